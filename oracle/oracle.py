"""ctypes front end of the CPU checkers (test infrastructure only).

Array conventions follow the reference's native layer
(torchwi/propagator/td2d/wrapper_cpu.cpp:44-112): padded velocity and fields
are flat ``[dimy*dimx]`` with x fastest, gathers are ``[nt, nx]`` and the
adjoint source (residual) is ``[nt, nx]``.  The operator-level helpers
``shot_gather`` / ``shot_gradient`` mirror ``Time2d(device='cpu')``
(torchwi/operator/TimeOperator.py:55-58 and TimeFunction.py:111-146): the
user model is ``(nx, nz)`` with z fastest, it is transposed and
edge-replicated by ``ne`` cells, and the gradient is cropped and transposed
back.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "_build", "libtwi_oracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libtd2d_ref.so")
_lock = threading.Lock()
_libs: dict[str, ctypes.CDLL] = {}


class OracleError(RuntimeError):
    pass


def reference_root() -> str | None:
    """The TorchWI checkout the reference build reads: $REFROOT, else a
    directory named ``reference`` beside this repository; None when neither
    holds the ``torchwi`` package."""
    cand = os.environ.get("REFROOT") or os.path.join(os.path.dirname(os.path.dirname(_HERE)),
                                                      "reference")
    return cand if os.path.isdir(os.path.join(cand, "torchwi")) else None


def build(ref: bool = True) -> None:
    """Compile the checkers with ``make`` (the reference part only when its
    sources are present)."""
    env = dict(os.environ)
    if os.path.exists("/usr/bin/g++"):
        env["CXX"] = "/usr/bin/g++"  # some toolchains on PATH lack libgomp
    targets = ["oracle"]
    refroot = reference_root()
    if ref and refroot is not None:
        env["REFROOT"] = refroot
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", _HERE, *targets], check=True, env=env)


_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double


def _load(path: str) -> ctypes.CDLL:
    with _lock:
        if path not in _libs:
            if not os.path.exists(path):
                if path == _ORACLE_SO:
                    build(ref=False)
                else:
                    raise OracleError(f"{path} missing (reference not built)")
            lib = ctypes.CDLL(path)
            if path == _ORACLE_SO:
                lib.twio_forward_f32.argtypes = [_F, _F, _F, _F, _i, _i, _i, _i,
                                                 _f, _f, _f, _f, _f]
                lib.twio_forward_f64.argtypes = [_D, _D, _D, _D, _i, _i, _i, _i,
                                                 _d, _d, _d, _d, _d]
                lib.twio_backward_f32.argtypes = [_F, _F, _F, _F, _i, _i, _i, _i,
                                                  _f, _f, _f, _i]
                lib.twio_backward_f64.argtypes = [_D, _D, _D, _D, _i, _i, _i, _i,
                                                  _d, _d, _d, _i]
                _S = ctypes.POINTER(ctypes.c_int16)
                lib.twio_exa_forward_f32.argtypes = [_F, _F, _S, _F, _F, _i, _i, _i, _i,
                                                     _f, _f, _f, _f, _f]
                lib.twio_exa_forward_cuda_order_f32.argtypes = lib.twio_exa_forward_f32.argtypes
                lib.twio_exa_backward_f32.argtypes = [_F, _F, _S, _F, _F, _i, _i, _i, _i,
                                                      _f, _f, _f]
                for fn in ("twio_forward_f32", "twio_forward_f64",
                           "twio_backward_f32", "twio_backward_f64",
                           "twio_exa_forward_f32", "twio_exa_forward_cuda_order_f32",
                           "twio_exa_backward_f32"):
                    getattr(lib, fn).restype = _i
            else:
                lib.ref_fdm_forward.argtypes = [_F] * 7 + [_i] * 4 + [_f] * 5
                lib.ref_fdm_backward.argtypes = [_F] * 7 + [_i] * 4 + [_f] * 3
                lib.ref_fdm_forward_only.argtypes = [_F] * 6 + [_i] * 4 + [_f] * 5
                for fn in ("ref_fdm_forward", "ref_fdm_backward",
                           "ref_fdm_forward_only"):
                    getattr(lib, fn).restype = None
            _libs[path] = lib
        return _libs[path]


def have_ref() -> bool:
    return os.path.exists(_REF_SO)


def _ptr(a: np.ndarray, kind=_F):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(kind)


def _check(status: int) -> None:
    if status != 0:
        raise OracleError({1: "order must be 2, 4 or 8",
                           2: "source outside the model",
                           3: "receiver row outside the grid",
                           4: "nt above 32767 (16-bit step index)"}.get(status, str(status)))


# ----------------------------------------------------------------------------
# native-layer calls (padded flat layout)
# ----------------------------------------------------------------------------

def twio_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry,
                 store_virt=True, dtype=np.float32):
    """Own restatement, forward pass.  Returns (frd[nt, nx], virt[nt, dimxy]
    or None)."""
    lib = _load(_ORACLE_SO)
    f64 = np.dtype(dtype) == np.float64
    dt_ = np.float64 if f64 else np.float32
    kind = _D if f64 else _F
    vpad = np.ascontiguousarray(vpad, dtype=dt_).ravel()
    w = np.ascontiguousarray(w, dtype=dt_).ravel()
    nx = dimx - order
    frd = np.zeros((nt, nx), dtype=dt_)
    virt = np.zeros((nt, dimx * dimy), dtype=dt_) if store_virt else None
    fn = lib.twio_forward_f64 if f64 else lib.twio_forward_f32
    _check(fn(_ptr(frd, kind), _ptr(virt, kind) if virt is not None else None,
              _ptr(vpad, kind), _ptr(w, kind), order, dimx, dimy, nt,
              h, dt, sx, sy, ry))
    return frd, virt


def twio_backward(virt, vpad, resid, order, dimx, dimy, nt, h, dt, ry,
                  kahan=False, dtype=np.float32):
    """Own restatement, adjoint pass.  Returns grad[dimxy] (padded layout)."""
    lib = _load(_ORACLE_SO)
    f64 = np.dtype(dtype) == np.float64
    dt_ = np.float64 if f64 else np.float32
    kind = _D if f64 else _F
    virt = np.ascontiguousarray(virt, dtype=dt_)
    vpad = np.ascontiguousarray(vpad, dtype=dt_).ravel()
    resid = np.ascontiguousarray(resid, dtype=dt_)
    grad = np.zeros(dimx * dimy, dtype=dt_)
    fn = lib.twio_backward_f64 if f64 else lib.twio_backward_f32
    _check(fn(_ptr(grad, kind), _ptr(virt, kind), _ptr(vpad, kind),
              _ptr(resid, kind), order, dimx, dimy, nt, h, dt, ry, int(kahan)))
    return grad


def twio_exa_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry, cuda_order=False):
    """Excitation-amplitude forward pass: (frd[nt, nx], exa[dimxy], iexa[dimxy] int16).
    cuda_order forms the virtual source with the reference CUDA kernel's
    operand order (td2d_cuda.cu:189) instead of the CPU propagator's."""
    lib = _load(_ORACLE_SO)
    vpad = np.ascontiguousarray(vpad, dtype=np.float32).ravel()
    w = np.ascontiguousarray(w, dtype=np.float32).ravel()
    frd = np.zeros((nt, dimx - order), dtype=np.float32)
    exa = np.zeros(dimx * dimy, dtype=np.float32)
    iexa = np.zeros(dimx * dimy, dtype=np.int16)
    fn = lib.twio_exa_forward_cuda_order_f32 if cuda_order else lib.twio_exa_forward_f32
    _check(fn(_ptr(frd), _ptr(exa), iexa.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)),
              _ptr(vpad), _ptr(w), order, dimx, dimy, nt, h, dt, sx, sy, ry))
    return frd, exa, iexa


def twio_exa_backward(exa, iexa, vpad, resid, order, dimx, dimy, nt, h, dt, ry):
    lib = _load(_ORACLE_SO)
    exa = np.ascontiguousarray(exa, dtype=np.float32)
    iexa = np.ascontiguousarray(iexa, dtype=np.int16)
    vpad = np.ascontiguousarray(vpad, dtype=np.float32).ravel()
    resid = np.ascontiguousarray(resid, dtype=np.float32)
    grad = np.zeros(dimx * dimy, dtype=np.float32)
    _check(lib.twio_exa_backward_f32(_ptr(grad), _ptr(exa), iexa.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)),
                                     _ptr(vpad), _ptr(resid), order, dimx, dimy, nt, h, dt, ry))
    return grad


def ref_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry, return_fields=False):
    """The reference's compiled c_fdm_forward.  Returns (frd, virt), and with
    return_fields the three work arrays u1, u2, u3 as the call left them."""
    lib = _load(_REF_SO)
    vpad = np.ascontiguousarray(vpad, dtype=np.float32).ravel().copy()
    w = np.ascontiguousarray(w, dtype=np.float32).ravel().copy()
    dimxy = dimx * dimy
    frd = np.zeros((nt, dimx - order), dtype=np.float32)
    virt = np.zeros((nt, dimxy), dtype=np.float32)
    u = [np.zeros(dimxy, dtype=np.float32) for _ in range(3)]
    lib.ref_fdm_forward(_ptr(frd), _ptr(virt), *(_ptr(a) for a in u), _ptr(vpad),
                        _ptr(w), order, dimx, dimy, nt, h, dt, sx, sy, ry)
    return (frd, virt, u) if return_fields else (frd, virt)


def ref_forward_only(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry, return_fields=False):
    lib = _load(_REF_SO)
    vpad = np.ascontiguousarray(vpad, dtype=np.float32).ravel().copy()
    w = np.ascontiguousarray(w, dtype=np.float32).ravel().copy()
    dimxy = dimx * dimy
    frd = np.zeros((nt, dimx - order), dtype=np.float32)
    u = [np.zeros(dimxy, dtype=np.float32) for _ in range(3)]
    lib.ref_fdm_forward_only(_ptr(frd), *(_ptr(a) for a in u), _ptr(vpad),
                             _ptr(w), order, dimx, dimy, nt, h, dt, sx, sy, ry)
    return (frd, u) if return_fields else frd


def ref_backward(virt, vpad, resid, order, dimx, dimy, nt, h, dt, ry, return_fields=False):
    lib = _load(_REF_SO)
    virt = np.ascontiguousarray(virt, dtype=np.float32)
    vpad = np.ascontiguousarray(vpad, dtype=np.float32).ravel().copy()
    resid = np.ascontiguousarray(resid, dtype=np.float32).copy()
    dimxy = dimx * dimy
    grad = np.zeros(dimxy, dtype=np.float32)
    u = [np.zeros(dimxy, dtype=np.float32) for _ in range(3)]
    lib.ref_fdm_backward(_ptr(grad), _ptr(virt), *(_ptr(a) for a in u), _ptr(vpad),
                         _ptr(resid), order, dimx, dimy, nt, h, dt, ry)
    return (grad, u) if return_fields else grad


# ----------------------------------------------------------------------------
# operator-level helpers (user layout)
# ----------------------------------------------------------------------------

def pad_model(vel, order, dtype=np.float32):
    """(nx, nz) z-fastest model -> flat padded [dimz*dimx] x-fastest, edge
    replicated by ne = order/2 (TimeOperator.py:55-58 on the CPU path)."""
    ne = order // 2
    v = np.asarray(vel, dtype=dtype).T  # (nz, nx)
    return np.pad(v, ((ne, ne), (ne, ne)), mode="edge").astype(dtype).ravel()


def shot_gather(vel, w, h, dt, order, sx, sy, ry, backend="oracle",
                dtype=np.float32, store_virt=False):
    """One shot of ``Time2d(device='cpu')``: returns gather [nt, nx] (and virt
    when ``store_virt``)."""
    nx, nz = np.asarray(vel).shape
    dimx, dimy = nx + order, nz + order
    vpad = pad_model(vel, order, dtype)
    nt = len(w)
    if backend == "ref":
        frd, virt = ref_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry)
    else:
        frd, virt = twio_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry,
                                 store_virt=store_virt, dtype=dtype)
    return (frd, virt) if store_virt else frd


def shot_gradient(vel, w, h, dt, order, sx, sy, ry, resid_fn, backend="oracle",
                  dtype=np.float32, kahan=False):
    """Forward + adjoint for one shot.  ``resid_fn(frd) -> resid[nt, nx]``
    (for the L2 misfit 0.5*sum((frd-obs)^2) this is frd-obs).  Returns
    (frd, grad[nx, nz])."""
    nx, nz = np.asarray(vel).shape
    dimx, dimy = nx + order, nz + order
    ne = order // 2
    vpad = pad_model(vel, order, dtype)
    nt = len(w)
    if backend == "ref":
        frd, virt = ref_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry)
        resid = np.asarray(resid_fn(frd), dtype=np.float32)
        g = ref_backward(virt, vpad, resid, order, dimx, dimy, nt, h, dt, ry)
    else:
        frd, virt = twio_forward(vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry,
                                 store_virt=True, dtype=dtype)
        resid = np.asarray(resid_fn(frd), dtype=dtype)
        g = twio_backward(virt, vpad, resid, order, dimx, dimy, nt, h, dt, ry,
                          kahan=kahan, dtype=dtype)
    g = g.reshape(dimy, dimx)[ne:ne + nz, ne:ne + nx].T.copy()
    return frd, g
