"""Drop-in for the reference's native module ``torchwi.propagator.td2d_cuda``
(torchwi/propagator/td2d/wrapper_cuda.cpp:45-119): the same two functions
with the same arguments, backed by the sm_100a kernels through the C ABI.

    forward(frd, virt, u1, u2, u3, vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry)
    backward(virt, u1, u2, u3, vpad, resid, order, dimx, dimy, nt, h, dt, ry) -> grad

Arrays follow the reference layout (padded grid [dimy][dimx] x fastest,
frd/resid [nt][nx] with nx = dimx - order, virt [nt][dimy*dimx]); `w` may
live on the host, as the reference keeps it.  Results are those of the
reference's CPU propagator, bit for bit.  Errors raise RuntimeError like the
reference's TORCH_CHECKs.
"""

from __future__ import annotations

import ctypes

import torch

from .. import _capi


def _cuda_input(t: torch.Tensor, name: str):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name}must be contiguous")
    if t.dtype != torch.float32:
        raise RuntimeError(f"{name} must be float32")


def _check_sizes(order, dimx, dimy, nt, grid=(), trace=(), history=(), w=None):
    """The kernels address every array by the sizes passed in, so each must
    hold at least that many samples: `grid` arrays dimy*dimx, `trace` arrays
    (frd, resid) nt*nx with nx = dimx - order, `history` arrays (virt)
    nt*dimy*dimx, and the wavelet nt.  A shorter array is an error here, not
    an out-of-bounds access on the device.  (The reference's CUDA path passes
    an (nt, nx_org) residual with the 16-padded nx when nx_org % 16 != 0,
    propagator_cuda.cu:142 with TimeFunction.py:128,137; that case stops
    here.)"""
    nx, dimxy = int(dimx) - int(order), int(dimx) * int(dimy)
    need = [(t, n, dimxy) for t, n in grid] + [(t, n, int(nt) * nx) for t, n in trace]
    need += [(t, n, int(nt) * dimxy) for t, n in history]
    if w is not None:
        need.append((w, "w", int(nt)))
    for t, name, n in need:
        if t.numel() < n:
            raise RuntimeError(f"{name} holds {t.numel()} samples; order={order}, dimx={dimx}, "
                               f"dimy={dimy}, nt={nt} need {n}")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _run(status):
    if status != _capi.TWI_OK:
        raise RuntimeError(_capi.last_error())


def forward(frd, virt, u1, u2, u3, vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry):
    for t, n in ((frd, "frd"), (virt, "source_wavefield"), (u1, "u1"), (u2, "u2"), (u3, "u3"),
                 (vpad, "vel")):
        _cuda_input(t, n)
    if not w.is_contiguous():
        raise RuntimeError("w must be contiguous")
    w = w.to(torch.float32)
    _check_sizes(order, dimx, dimy, nt, grid=((vpad, "vel"), (u1, "u1"), (u2, "u2"), (u3, "u3")),
                 trace=((frd, "frd"),), history=((virt, "source_wavefield"),), w=w)
    with torch.cuda.device(frd.device):
        _run(_capi.lib().twi_fdm_forward(_ptr(frd), _ptr(virt), _ptr(u1), _ptr(u2), _ptr(u3),
                                         _ptr(vpad), _ptr(w), int(order), int(dimx), int(dimy),
                                         int(nt), float(h), float(dt), float(sx), float(sy),
                                         float(ry), _stream()))


def backward(virt, u1, u2, u3, vpad, resid, order, dimx, dimy, nt, h, dt, ry):
    for t, n in ((virt, "source_wavefield"), (u1, "u1"), (u2, "u2"), (u3, "u3"), (vpad, "vel"),
                 (resid, "resid")):
        _cuda_input(t, n)
    _check_sizes(order, dimx, dimy, nt, grid=((vpad, "vel"), (u1, "u1"), (u2, "u2"), (u3, "u3")),
                 trace=((resid, "resid"),), history=((virt, "source_wavefield"),))
    grad = torch.zeros_like(vpad)
    with torch.cuda.device(vpad.device):
        _run(_capi.lib().twi_fdm_backward(_ptr(grad), _ptr(virt), _ptr(u1), _ptr(u2), _ptr(u3),
                                          _ptr(vpad), _ptr(resid), int(order), int(dimx),
                                          int(dimy), int(nt), float(h), float(dt), float(ry),
                                          _stream()))
    return grad
