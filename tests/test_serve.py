"""Host-side logic of the serving loop (no GPU): shot chunking for HBM
admission, FIFO latency model of the plain per-request form, request stream."""
import numpy as np
import pytest

from torchwi_b200 import synthetic
from torchwi_b200.serve import chunk_shots, fifo_latencies


def test_chunk_shots_fits_and_covers():
    for n in (1, 7, 64, 128):
        for per in (1, 3, 10):
            budget = 50
            parts = chunk_shots(n, lambda k: 5 + per * k, budget)
            covered = []
            for s in parts:
                assert 5 + per * (s.stop - s.start) <= budget
                covered.extend(range(s.start, s.stop))
            assert covered == list(range(n))
            sizes = [s.stop - s.start for s in parts]
            assert max(sizes) - min(sizes) <= 1 or len(parts) == 1 or sizes[-1] <= sizes[0]


def test_chunk_shots_rejects_single_shot_too_big():
    with pytest.raises(MemoryError):
        chunk_shots(4, lambda k: 100 * k, 50)


def test_fifo_latencies():
    lat = fifo_latencies([0.0, 0.5, 0.6], [1.0, 1.0, 0.1])
    np.testing.assert_allclose(lat, [1.0, 1.5, 1.5])


def test_config5_stream_is_seeded_and_sorted():
    m1, r1 = synthetic.config5(rate=50.0, nreq=20)
    m2, r2 = synthetic.config5(rate=50.0, nreq=20)
    assert [r["arrival"] for r in r1] == [r["arrival"] for r in r2]
    assert all(a["arrival"] < b["arrival"] for a, b in zip(r1, r1[1:]))
    assert {r["kind"] for r in r1} <= {"forward", "gradient"}
    assert set(m1) == {f"layered_{nx}x{nz}" for nx, nz in synthetic.SERVE_GRIDS}
    for r in r1:
        nx, nz = m1[r["model"]].shape
        assert 1 <= len(r["sx"]) <= 128 and 2000 <= len(r["w"]) <= 8000
        assert np.all(r["sx"] < nx * 10.0)


def _server_stub(policy, inflight_cells):
    """A Server with only the admission state (no device, no engine)."""
    from torchwi_b200.serve import Server

    srv = Server.__new__(Server)
    srv.policy, srv.budget, srv.used = policy, 100, 0
    srv.saturation_cells, srv.backfill_cells = 1000, 50
    srv.inflight = {0: object()} if inflight_cells else {}
    srv.active_cells = inflight_cells
    return srv


def _chunk(name, cells, work, footprint=10):
    from torchwi_b200.serve import _Chunk

    c = _Chunk(req=None, shots=slice(0, 1), footprint=footprint, cells=cells, work=work)
    c.name = name
    return c


def test_fifo_admission_keeps_large_requests_in_line_and_backfills_small_ones():
    srv = _server_stub("fifo", inflight_cells=900)          # a large request is running
    srv.queue = [_chunk("big1", 800, 8e6), _chunk("big2", 500, 5e6), _chunk("small", 40, 4e4)]
    assert srv._next_chunk().name == "small"                 # runs alongside
    assert srv._next_chunk() is None                         # the large ones wait, in order
    srv.inflight, srv.active_cells = {}, 0
    assert [srv._next_chunk().name for _ in range(1)] == ["big1"]
    srv.active_cells, srv.inflight = 800, {0: object()}
    assert srv._next_chunk() is None                         # big2 would oversubscribe


def test_sjf_admission_takes_the_shortest_first():
    srv = _server_stub("sjf", inflight_cells=0)
    srv.queue = [_chunk("big", 800, 8e6), _chunk("mid", 300, 3e5), _chunk("small", 40, 4e4)]
    assert srv._next_chunk().name == "small"
    srv.inflight, srv.active_cells = {0: object()}, 40
    assert srv._next_chunk().name == "mid"
    srv.active_cells = 340
    assert srv._next_chunk() is None                         # 340 + 800 > saturation


def test_admission_respects_the_hbm_budget():
    srv = _server_stub("fifo", inflight_cells=0)
    srv.used = 95
    srv.queue = [_chunk("small", 40, 4e4, footprint=10)]
    assert srv._next_chunk() is None
