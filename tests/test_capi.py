"""The C-ABI library loads, exports every symbol declared in include/*.h and
validates problems on the host -- no GPU needed (no compute calls)."""
import ctypes
import glob
import os
import re

import pytest

from torchwi_b200 import _capi
from torchwi_b200.build import LIB

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"^\s*(?:int|const char\*|void)\s+\**\s*(twi_\w+)\s*\(", src, re.M))
    return sorted(names)


def test_library_built_in_tree():
    assert os.path.exists(LIB), "run python -m torchwi_b200.build"


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    names = _declared_symbols()
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(_declared_symbols()) <= set(_capi.SIGNATURES)


def _problem(**kw):
    base = dict(order=4, nx=100, nz=50, nt=200, h=10.0, dt=1e-3, nshots=4, ckpt_interval=0,
                exact=1, accumulate=0, shots_per_cta=0, rows_per_warp=0, use_graphs=1,
                wavelet_per_shot=0, forward_only=0)
    base.update(kw)
    return _capi.Problem(**base)


def _create(**kw):
    L = _capi.lib()
    h = ctypes.c_void_p()
    st = L.twi_plan_create(ctypes.byref(_problem(**kw)), ctypes.byref(h))
    return st, h


def test_plan_layout_on_host():
    L = _capi.lib()
    st, h = _create(nt=4000, nshots=64, nx=1000, nz=300, ckpt_interval=50)
    assert st == _capi.TWI_OK
    lay = _capi.Layout()
    assert L.twi_plan_layout(h, ctypes.byref(lay)) == 0
    assert (lay.dimx, lay.dimz, lay.pitch) == (1004, 304, 1024)
    assert lay.ckpt_interval == 50 and lay.nsegments == 80
    # fields: (1 + 64*(6 + 2*79)) slots + 64*50 virtual-source slots, 1024*304 floats each
    slot = 1024 * 304 * 4
    assert lay.workspace_bytes >= (1 + 64 * 164 + 64 * 50) * slot
    assert lay.workspace_bytes < (1 + 64 * 164 + 64 * 50 + 40) * slot + 2 * 64 * 4000 * 1000 * 4
    assert lay.workspace_bytes % 256 == 0
    assert L.twi_plan_destroy(h) == 0


@pytest.mark.parametrize("bad", [dict(order=6), dict(nx=0), dict(nt=0), dict(nshots=0),
                                 dict(h=0.0), dict(rows_per_warp=3), dict(ckpt_interval=1)])
def test_plan_rejects_invalid_problem(bad):
    st, h = _create(**bad)
    assert st == _capi.TWI_ERR_INVALID
    assert _capi.last_error()


@pytest.mark.parametrize("rz,expect", [(0, (4, 2)), (2, (2, 2)), (4, (4, 4)), (8, (8, 8))])
def test_rows_per_warp_per_mode(rz, expect):
    # left open, the adjoint runs on 2-row tiles and the rest on 4; an
    # explicit value applies to every mode
    L = _capi.lib()
    st, h = _create(rows_per_warp=rz)
    assert st == _capi.TWI_OK
    lay = _capi.Layout()
    assert L.twi_plan_layout(h, ctypes.byref(lay)) == 0
    assert (lay.rows_per_warp, lay.adjoint_rows_per_warp) == expect
    L.twi_plan_destroy(h)


@pytest.mark.parametrize("spc,nshots,expect", [(0, 64, (4, 8)), (0, 6, (4, 6)), (0, 3, (3, 3)),
                                              (2, 64, (2, 2)), (8, 64, (8, 8))])
def test_shots_per_cta_per_mode(spc, nshots, expect):
    # left open, adjoint launches take 8 shots per CTA (one Kahan pair per
    # group) and the rest 4; an explicit value applies to every mode
    L = _capi.lib()
    st, h = _create(shots_per_cta=spc, nshots=nshots)
    assert st == _capi.TWI_OK
    lay = _capi.Layout()
    assert L.twi_plan_layout(h, ctypes.byref(lay)) == 0
    assert (lay.shots_per_cta, lay.adjoint_shots_per_cta) == expect
    L.twi_plan_destroy(h)


def test_shots_per_cta_is_bounded():
    for spc in (-1, 33):
        st, _ = _create(shots_per_cta=spc, nshots=64)
        assert st == _capi.TWI_ERR_INVALID
        assert "shots_per_cta" in _capi.last_error()
    st, h = _create(shots_per_cta=32, nshots=64)
    assert st == _capi.TWI_OK
    _capi.lib().twi_plan_destroy(h)


def test_persistent_plans_run_one_step_per_item():
    st, _ = _create(persistent=1, time_block=2)
    assert st == _capi.TWI_ERR_INVALID
    assert "persistent" in _capi.last_error()
    for kw in (dict(persistent=1), dict(persistent=1, reconstruct=1), dict(persistent=1, forward_only=1)):
        st, h = _create(**kw)
        assert st == _capi.TWI_OK, kw
        lay = _capi.Layout()
        assert _capi.lib().twi_plan_layout(h, ctypes.byref(lay)) == 0
        assert lay.time_block == 1
        _capi.lib().twi_plan_destroy(h)


def test_chained_launch_option():
    st, _ = _create(unchained=2)
    assert st == _capi.TWI_ERR_INVALID
    assert "unchained" in _capi.last_error()
    # chaining needs one counter per shot group: the workspace grows by at most a few hundred bytes
    sizes = []
    for kw in (dict(unchained=0), dict(unchained=1), dict(unchained=0, persistent=1)):
        st, h = _create(**kw)
        assert st == _capi.TWI_OK, kw
        lay = _capi.Layout()
        assert _capi.lib().twi_plan_layout(h, ctypes.byref(lay)) == 0
        sizes.append(lay.workspace_bytes)
        _capi.lib().twi_plan_destroy(h)
    assert 0 < sizes[0] - sizes[1] <= 4096
    assert sizes[2] != sizes[0]


def test_two_rows_per_warp_runs_one_step_per_launch():
    st, h = _create(rows_per_warp=2, time_block=2)
    assert st == _capi.TWI_ERR_INVALID
    assert "rows_per_warp" in _capi.last_error()


def test_calls_out_of_sequence_are_errors():
    L = _capi.lib()
    st, h = _create()
    assert st == 0
    assert L.twi_forward(h, 1, None) == _capi.TWI_ERR_STATE
    assert L.twi_gradient(h, None) == _capi.TWI_ERR_STATE
    assert "workspace" in _capi.last_error()
    L.twi_plan_destroy(h)


def test_default_checkpoint_interval_is_sqrt_2nt():
    L = _capi.lib()
    st, h = _create(nt=4000)
    lay = _capi.Layout()
    L.twi_plan_layout(h, ctypes.byref(lay))
    assert lay.ckpt_interval == 89 and lay.nsegments == 45
    L.twi_plan_destroy(h)


def test_forward_only_plan_is_small():
    L = _capi.lib()
    full = _capi.Layout()
    st, h = _create(nt=4000, nshots=64, nx=1000, nz=300)
    L.twi_plan_layout(h, ctypes.byref(full))
    L.twi_plan_destroy(h)
    fo = _capi.Layout()
    st, h = _create(nt=4000, nshots=64, nx=1000, nz=300, forward_only=1)
    L.twi_plan_layout(h, ctypes.byref(fo))
    L.twi_plan_destroy(h)
    slot = 1024 * 304 * 4
    assert fo.workspace_bytes < (1 + 64 * 3 + 2) * slot + 2 * 64 * 4000 * 1000 * 4
    assert full.workspace_bytes > 10 * fo.workspace_bytes


def test_exa_plan_ignores_kahan():
    """Excitation amplitude assigns one value per cell and shot: its plans keep
    one gradient slot per shot whatever the accumulation switch says."""
    L = _capi.lib()
    sizes = []
    for acc in (0, 1):
        lay = _capi.Layout()
        st, h = _create(nt=300, nshots=8, nx=70, nz=33, exa=1, accumulate=acc)
        assert st == 0
        L.twi_plan_layout(h, ctypes.byref(lay))
        L.twi_plan_destroy(h)
        sizes.append(lay.workspace_bytes)
    assert sizes[0] == sizes[1]


def test_footprint_and_autotune_scratch_on_host():
    L = _capi.lib()
    n = ctypes.c_size_t()
    p = _problem(nt=300, nshots=8, nx=70, nz=33)
    assert L.twi_plan_footprint_bytes(ctypes.byref(p), ctypes.byref(n)) == 0
    st, h = _create(nt=300, nshots=8, nx=70, nz=33)
    lay = _capi.Layout()
    L.twi_plan_layout(h, ctypes.byref(lay))
    L.twi_plan_destroy(h)
    assert n.value == lay.workspace_bytes
    m = ctypes.c_size_t()
    assert L.twi_autotune_scratch_bytes(ctypes.byref(p), ctypes.byref(m)) == 0
    assert 0 < m.value < n.value            # short copies of the problem
    bad = _problem(order=6)
    assert L.twi_autotune_scratch_bytes(ctypes.byref(bad), ctypes.byref(m)) == _capi.TWI_ERR_INVALID


def test_time_block_option_on_host():
    L = _capi.lib()
    for tb, want in ((0, 1), (1, 1), (2, 2)):
        st, h = _create(nt=100, nshots=2, time_block=tb)
        assert st == 0
        lay = _capi.Layout()
        L.twi_plan_layout(h, ctypes.byref(lay))
        L.twi_plan_destroy(h)
        assert lay.time_block == want
    st, h = _create(time_block=3)
    assert st == _capi.TWI_ERR_INVALID
    st, h = _create(nt=100, nshots=2, time_block=2, exa=1)   # excitation amplitude: one step
    lay = _capi.Layout()
    L.twi_plan_layout(h, ctypes.byref(lay))
    L.twi_plan_destroy(h)
    assert lay.time_block == 1


def test_reconstruction_plan_trades_checkpoints_for_boundaries():
    """Config-3 sizes: boundary saving needs a fraction of the checkpointed
    plan's memory, and runs one step per launch."""
    L = _capi.lib()
    sizes = {}
    for rec in (0, 1):
        p = _problem(nt=6000, nshots=256, nx=1000, nz=300, ckpt_interval=50, reconstruct=rec)
        n = ctypes.c_size_t()
        assert L.twi_plan_footprint_bytes(ctypes.byref(p), ctypes.byref(n)) == 0
        sizes[rec] = n.value
    assert sizes[1] < 0.3 * sizes[0]
    boundary = 2 * 2 * 300 + 2 * 1004
    assert sizes[1] >= 6001 * 256 * boundary * 4
    st, h = _create(reconstruct=1, time_block=2)
    assert st == _capi.TWI_ERR_INVALID
