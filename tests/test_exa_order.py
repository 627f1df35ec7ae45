"""The excitation-amplitude mode forms its virtual source in the CPU
propagator's operand order, cons/(v*v*v) * ((u^{n-1} - 2u^n) + u^{n+1})
(propagator_cpu.cpp:70), like every other mode here.  The reference's only
EXA implementation is CUDA and writes ((u^{n+1} - 2u^n) + u^{n-1})
(td2d_cuda.cu:189).  This measures, with the oracle restatement run both
ways on the same propagation, what that order changes: the last bits of a
few stored amplitudes, and the gradient far below the 1e-4 tolerance."""
import numpy as np

import oracle as O
from oracle import oracle as OO
from torchwi_b200 import synthetic


def test_exa_operand_order_changes_only_last_bits():
    nx, nz, nt, order = 120, 60, 600, 4
    s = synthetic.small_case(nx=nx, nz=nz, nt=nt, order=order, nshots=1, seed=3, freq=10.0)
    dimx, dimy = nx + order, nz + order
    vpad, vtrue = O.pad_model(s.vel_start, order), O.pad_model(s.vel, order)
    args = (order, dimx, dimy, nt, s.h, s.dt)
    obs, _, _ = OO.twio_exa_forward(vtrue, s.w, *args, s.sx[0], s.sy[0], s.ry[0])
    out = {}
    for cuda_order in (False, True):
        frd, exa, iexa = OO.twio_exa_forward(vpad, s.w, *args, s.sx[0], s.sy[0], s.ry[0],
                                             cuda_order=cuda_order)
        g = OO.twio_exa_backward(exa, iexa, vpad, (frd - obs).astype(np.float32), *args, s.ry[0])
        out[cuda_order] = (exa, iexa, g.reshape(dimy, dimx)[2:-2, 2:-2].astype(np.float64))
    (e0, i0, g0), (e1, i1, g1) = out[False], out[True]
    differ = np.mean(e0.view(np.int32) != e1.view(np.int32))
    steps = np.mean(i0 != i1)
    err = np.linalg.norm(g1 - g0) / np.linalg.norm(g0)
    print(f"EXA operand order: amplitudes differing {differ:.2e} of cells, steps {steps:.2e}, "
          f"gradient rel L2 {err:.2e}")
    assert differ < 1e-2 and err < 1e-6
