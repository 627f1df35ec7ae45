"""Drop-in for ``torchwi.propagator.td2d_forward_cuda``
(torchwi/propagator/td2d/wrapper_forward_cuda.cpp:30-73)."""

from __future__ import annotations

import torch

from .. import _capi
from .td2d_b200 import _check_sizes, _cuda_input, _ptr, _run, _stream


def forward(frd, u1, u2, u3, vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry):
    for t, n in ((frd, "frd"), (u1, "u1"), (u2, "u2"), (u3, "u3"), (vpad, "vel")):
        _cuda_input(t, n)
    if not w.is_contiguous():
        raise RuntimeError("w must be contiguous")
    w = w.to(torch.float32)
    _check_sizes(order, dimx, dimy, nt, grid=((vpad, "vel"), (u1, "u1"), (u2, "u2"), (u3, "u3")),
                 trace=((frd, "frd"),), w=w)
    with torch.cuda.device(frd.device):
        _run(_capi.lib().twi_fdm_forward_only(_ptr(frd), _ptr(u1), _ptr(u2), _ptr(u3),
                                              _ptr(vpad), _ptr(w), int(order), int(dimx),
                                              int(dimy), int(nt), float(h), float(dt),
                                              float(sx), float(sy), float(ry), _stream()))


def backward():
    return torch.zeros(1)
