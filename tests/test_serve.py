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
