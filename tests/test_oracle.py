"""The CPU checker (oracle) against the reference: golden vectors produced by
running TorchWI's own Time2d(device='cpu'), and -- where the reference's CPU
propagator was compiled from its sources -- a direct bit-for-bit comparison.
No GPU needed."""
import numpy as np
import pytest

import oracle as O
from golden_io import SMALL_CASES, bits_equal, load_json, load_small, rel_l2, sha
from torchwi_b200 import synthetic


@pytest.mark.parametrize("name", SMALL_CASES)
def test_oracle_matches_reference_golden(name):
    g = load_small(name)
    order, h, dt, w = g["order"], g["h"], g["dt"], g["w"]
    grad_sum = None
    for k in range(len(g["sx"])):
        sx, sy, ry = g["sx"][k], g["sy"][k], g["ry"][k]
        obs = O.shot_gather(g["vel"], w, h, dt, order, sx, sy, ry)
        assert bits_equal(obs, g["obs"][k])
        obs_k = g["obs"][k]
        frd, grad = O.shot_gradient(g["vel_start"], w, h, dt, order, sx, sy, ry,
                                    lambda f: (f - obs_k).astype(np.float32))
        assert bits_equal(frd, g["frd"][k])
        loss = 0.5 * np.sum((frd.astype(np.float32) - obs_k) ** 2, dtype=np.float32)
        assert abs(float(loss) - float(g["losses"][k])) <= 1e-5 * abs(float(g["losses"][k]))
        grad_sum = grad if grad_sum is None else (grad_sum + grad).astype(np.float32)
    assert bits_equal(grad_sum, g["grad"])


def test_oracle_config1_hashes():
    rec = load_json("config1.json")
    s = synthetic.config1()
    for k, shot in enumerate(rec["shots"][:3]):
        g = O.shot_gather(s.vel, s.w, s.h, s.dt, s.order, s.sx[k], s.sy[k], s.ry[k])
        assert sha(g) == shot["sha256"], k
    dec = np.load(__import__("os").path.join(__import__("golden_io").GOLDEN,
                                             "config1_shot0_decimated.npy"))
    g0 = O.shot_gather(s.vel, s.w, s.h, s.dt, s.order, s.sx[0], s.sy[0], s.ry[0])
    assert bits_equal(g0[::4, ::2], dec)


@pytest.mark.slow
def test_oracle_config2_shot_hashes():
    """Full-size (1000x300, nt=4000) shot: gathers and gradient equal the
    reference's bit for bit."""
    rec = load_json("config2_shot.json")
    s = synthetic.config2(nshots=64, nt=4000)
    k = rec["shot"]
    obs = O.shot_gather(s.vel, s.w, s.h, s.dt, s.order, s.sx[k], s.sy[k], s.ry[k])
    assert sha(obs) == rec["obs_sha256"]
    frd, grad = O.shot_gradient(s.vel_start, s.w, s.h, s.dt, s.order, s.sx[k], s.sy[k],
                                s.ry[k], lambda f: (f - obs).astype(np.float32))
    assert sha(frd) == rec["frd_sha256"]
    assert sha(grad) == rec["grad_sha256"]


@pytest.mark.skipif(not O.have_ref(), reason="reference CPU propagator not built")
@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("shape", [(33, 19, 150), (52, 40, 220)])
def test_oracle_bitexact_vs_reference_build(order, shape):
    nx, nz, nt = shape
    s = synthetic.small_case(nx=nx, nz=nz, nt=nt, order=order, nshots=1, seed=order + nx)
    vpad = O.pad_model(s.vel, order)
    dimx, dimy = nx + order, nz + order
    args = (order, dimx, dimy, nt, s.h, s.dt, s.sx[0], s.sy[0], s.ry[0])
    f_ref, v_ref = O.ref_forward(vpad, s.w, *args)
    f_own, v_own = O.twio_forward(vpad, s.w, *args)
    assert bits_equal(f_ref, f_own) and bits_equal(v_ref, v_own)
    assert bits_equal(O.ref_forward_only(vpad, s.w, *args), f_own)
    resid = (0.5 * f_ref).astype(np.float32)
    g_ref = O.ref_backward(v_ref, vpad, resid, order, dimx, dimy, nt, s.h, s.dt, s.ry[0])
    g_own = O.twio_backward(v_own, vpad, resid, order, dimx, dimy, nt, s.h, s.dt, s.ry[0])
    assert bits_equal(g_ref, g_own)


def test_fp64_oracle_close_to_fp32():
    """The FP64 run of the same scheme stays within the FP32 noise floor of
    the FP32 run (sanity check of the double instantiation)."""
    s = synthetic.small_case(nx=40, nz=30, nt=300, order=4, nshots=1)
    f32 = O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[0], s.sy[0], s.ry[0])
    f64 = O.shot_gather(s.vel.astype(np.float64), s.w.astype(np.float64), s.h, s.dt, 4,
                        s.sx[0], s.sy[0], s.ry[0], dtype=np.float64)
    assert 0 < rel_l2(f32, f64) < 1e-5


def test_oracle_rejects_bad_input():
    s = synthetic.small_case(nx=20, nz=12, nt=10, order=4, nshots=1)
    vpad = O.pad_model(s.vel, 4)
    with pytest.raises(O.OracleError):
        O.twio_forward(vpad, s.w, 6, 24, 16, 10, s.h, s.dt, 10.0, 20.0, 20.0)
    with pytest.raises(O.OracleError):
        O.twio_forward(vpad, s.w, 4, 24, 16, 10, s.h, s.dt, 1000.0, 20.0, 20.0)
