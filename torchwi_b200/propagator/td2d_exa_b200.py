"""Drop-in for ``torchwi.propagator.td2d_exa_cuda``
(torchwi/propagator/td2d/wrapper_exa_cuda.cpp:9-89): excitation-amplitude
forward and backward with the reference's arguments; `iexa` is int16."""

from __future__ import annotations

import torch

from .. import _capi
from .td2d_b200 import _check_sizes, _cuda_input, _ptr, _run, _stream


def forward(frd, exa, iexa, u1, u2, u3, vpad, w, order, dimx, dimy, nt, h, dt, sx, sy, ry):
    for t, n in ((frd, "frd"), (exa, "exa"), (u1, "u1"), (u2, "u2"), (u3, "u3"), (vpad, "vel")):
        _cuda_input(t, n)
    if not iexa.is_cuda or iexa.dtype != torch.int16 or not iexa.is_contiguous():
        raise RuntimeError("iexa must be a contiguous int16 CUDA tensor")
    w = w.contiguous().to(torch.float32)
    _check_sizes(order, dimx, dimy, nt, grid=((vpad, "vel"), (exa, "exa"), (iexa, "iexa"),
                                             (u1, "u1"), (u2, "u2"), (u3, "u3")),
                 trace=((frd, "frd"),), w=w)
    with torch.cuda.device(frd.device):
        _run(_capi.lib().twi_fdm_exa_forward(_ptr(frd), _ptr(exa), _ptr(iexa), _ptr(u1), _ptr(u2),
                                             _ptr(u3), _ptr(vpad), _ptr(w), int(order), int(dimx),
                                             int(dimy), int(nt), float(h), float(dt), float(sx),
                                             float(sy), float(ry), _stream()))


def backward(exa, iexa, u1, u2, u3, vpad, resid, order, dimx, dimy, nt, h, dt, ry):
    for t, n in ((exa, "exa"), (u1, "u1"), (u2, "u2"), (u3, "u3"), (vpad, "vel"), (resid, "resid")):
        _cuda_input(t, n)
    if not iexa.is_cuda or iexa.dtype != torch.int16 or not iexa.is_contiguous():
        raise RuntimeError("iexa must be a contiguous int16 CUDA tensor")
    _check_sizes(order, dimx, dimy, nt, grid=((vpad, "vel"), (exa, "exa"), (iexa, "iexa"),
                                             (u1, "u1"), (u2, "u2"), (u3, "u3")),
                 trace=((resid, "resid"),))
    grad = torch.zeros_like(vpad)
    with torch.cuda.device(vpad.device):
        _run(_capi.lib().twi_fdm_exa_backward(_ptr(grad), _ptr(exa), _ptr(iexa), _ptr(u1), _ptr(u2),
                                              _ptr(u3), _ptr(vpad), _ptr(resid), int(order), int(dimx),
                                              int(dimy), int(nt), float(h), float(dt), float(ry),
                                              _stream()))
    return grad
