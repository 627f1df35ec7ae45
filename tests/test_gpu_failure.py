"""The kernels' failure path, exercised without a fault: a wait that can
never complete runs out after its limit, the device error word is reported,
and the context keeps working."""
import ctypes

import pytest
import torch

import oracle as O
from golden_io import bits_equal
from torchwi_b200 import PlanOptions, ShotPlan, _capi, synthetic

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives():
    L = _capi.lib()
    ms = ctypes.c_float()
    st = L.twi_check_wait_timeout(20000, ctypes.byref(ms),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _capi.TWI_OK, _capi.last_error()
    assert 19.0 <= ms.value < 2000.0, ms.value
    # the context is still usable: a plan runs and matches the CPU checker
    s = synthetic.small_case(nx=40, nz=20, nt=60, nshots=1)
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 4, nshots=1, options=PlanOptions())
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    p.set_model(torch.from_numpy(s.vel).cuda())
    frd = p.forward(save_checkpoints=False).clone()
    p.check()
    assert bits_equal(frd[0].cpu().numpy(), O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[0], s.sy[0], s.ry[0]))


def test_counter_wait_runs_out_or_leaves_on_error_and_context_survives():
    """The wait a chained or persistent launch's CTA makes for its shot group
    of the earlier steps: a counter that never reaches its target runs out
    after the limit and raises the error word; an error word another CTA has
    already raised ends the wait at once."""
    L = _capi.lib()
    st_ = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ms = ctypes.c_float()
    assert L.twi_check_counter_wait(20000, 0, ctypes.byref(ms), st_) == _capi.TWI_OK, _capi.last_error()
    assert 19.0 <= ms.value < 2000.0, ms.value
    assert L.twi_check_counter_wait(2000000, 1, ctypes.byref(ms), st_) == _capi.TWI_OK, _capi.last_error()
    assert ms.value < 100.0, ms.value
    # chained launches still run and match stream order bit for bit
    s = synthetic.small_case(nx=97, nz=41, nt=80, nshots=5)
    out = []
    for chained in (True, False):
        p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 4, nshots=s.nshots, options=PlanOptions(chained=chained))
        p.set_wavelet(torch.from_numpy(s.w))
        p.set_shots(s.sx, s.sy, s.ry)
        p.set_model(torch.from_numpy(s.vel).cuda())
        out.append(p.forward(save_checkpoints=False).clone())
        p.check()
    assert bits_equal(out[0].cpu().numpy(), out[1].cpu().numpy())


def test_wait_limit_is_validated_on_the_host():
    L = _capi.lib()
    assert L.twi_check_wait_timeout(0, None, None) == _capi.TWI_ERR_INVALID
    assert L.twi_check_counter_wait(0, 0, None, None) == _capi.TWI_ERR_INVALID
    assert L.twi_check_counter_wait(10, 2, None, None) == _capi.TWI_ERR_INVALID
