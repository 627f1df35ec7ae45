"""The allocation-free forward entry point, through the C ABI.

Some callers cannot allocate GPU memory (they run inside another framework's
memory pool or a fixed arena, or on hosts that forbid allocation after
start-up); twi_fdm_forward_only_noalloc serves them from a fixed 32 MiB
device array built into the library.  Its gathers must equal those of the
allocating entry point twi_fdm_forward_only -- bit for bit, the tolerance of
the other reference-arithmetic tests -- on two calls in a row (the second
call sees the first call's leftovers in the shared array).  This file is
collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from torchwi_b200 import _capi, synthetic

pytestmark = pytest.mark.gpu


def _vpad(vel, order):
    ne = order // 2
    v = np.asarray(vel, dtype=np.float32).T
    return np.pad(v, ((ne, ne), (ne, ne)), mode="edge").astype(np.float32).ravel()


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _case(nx, nz, nt, order, seed, shot):
    s = synthetic.small_case(nx=nx, nz=nz, nt=nt, order=order, nshots=3, seed=seed)
    dev = torch.device("cuda")
    vel = torch.from_numpy(_vpad(s.vel, order)).to(dev)
    w = torch.from_numpy(s.w).to(dev)
    return s, vel, w, (order, nx + order, nz + order, nt, s.h, s.dt,
                       float(s.sx[shot]), float(s.sy[shot]), float(s.ry[shot]))


def _allocating(vel, w, args):
    order, dimx, dimy, nt = args[:4]
    dev = vel.device
    frd = torch.zeros(nt * (dimx - order), device=dev)
    u = torch.zeros(dimx * dimy, device=dev)
    L = _capi.lib()
    st = L.twi_fdm_forward_only(_p(frd), _p(u), _p(u), _p(u), _p(vel), _p(w), *args[:4],
                                *args[4:], ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, _capi.last_error()
    return frd


def _no_alloc(vel, w, args):
    order, dimx, dimy, nt = args[:4]
    frd = torch.full((nt * (dimx - order),), float("nan"), device=vel.device)
    L = _capi.lib()
    st = L.twi_fdm_forward_only_noalloc(_p(frd), _p(vel), _p(w), *args[:4], *args[4:],
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, _capi.last_error()
    return frd


def _same(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return np.array_equal(a.view(np.int32), b.view(np.int32))


def test_no_alloc_matches_allocating_entry_point_twice():
    # first call: order 4, second call: a different grid, order and shot, so
    # stale contents of the shared scratch from call 1 would show up
    cases = [_case(150, 60, 240, 4, seed=1, shot=1), _case(97, 41, 180, 8, seed=2, shot=2)]
    for _, vel, w, args in cases:
        ref = _allocating(vel, w, args)
        got = _no_alloc(vel, w, args)
        assert _same(got, ref)
    # and the same call twice in a row
    _, vel, w, args = cases[0]
    assert _same(_no_alloc(vel, w, args), _no_alloc(vel, w, args))


def test_no_alloc_rejects_oversized_grid():
    dev = torch.device("cuda")
    dimx, dimy, nt = 4000 + 4, 1200 + 4, 10   # 5 * 4096 * 1204 * 4 B > 32 MiB
    vel = torch.full((dimx * dimy,), 2000.0, device=dev)
    w = torch.zeros(nt, device=dev)
    frd = torch.zeros(nt * 4000, device=dev)
    L = _capi.lib()
    st = L.twi_fdm_forward_only_noalloc(_p(frd), _p(vel), _p(w), 4, dimx, dimy, nt, 10.0, 1e-3,
                                        100.0, 20.0, 20.0,
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _capi.TWI_ERR_INVALID
    assert "too large" in _capi.last_error()

