"""The wavelet generators against fixtures written by the reference's own
torchwi/source/wavelets.py (tests/golden/make_wavelet_golden.py): every
sample bit for bit, float32 and float64, over 60 frequencies x 5 time steps,
and the full arrays of the benchmark configurations."""
import hashlib
import json
import os
import warnings

import numpy as np
import pytest

from torchwi_b200.source import wavelets as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DTYPES = {"float32": np.float32, "float64": np.float64}


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


@pytest.fixture(scope="module")
def table():
    with open(os.path.join(GOLDEN, "wavelets.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("fn", ["ricker", "fdgaus"])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_wavelet_grid_matches_reference(table, fn, dtype):
    bad = []
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)   # the reference divides 0/0 for some cases too
        for dt in table["dts"]:
            for f in table["freqs"]:
                got = getattr(W, fn)(f, dt, table["nt"], dtype=DTYPES[dtype])
                assert got.dtype == DTYPES[dtype]
                if _digest(got) != table["sha256_16"][f"{fn}/{f:g}/{dt:g}/{dtype}"]:
                    bad.append((f, dt))
    assert not bad, f"{len(bad)} {fn}/{dtype} cases differ from the reference, e.g. {bad[:5]}"


def test_benchmark_wavelets_match_reference():
    ref = np.load(os.path.join(GOLDEN, "wavelets.npz"))
    for name in ref.files:
        fn, freq, dt, nt, dt_name = name.split("_")
        f = float(freq[:-2])
        step = float(dt[2:-2]) * 1e-3
        n = int(nt[2:])
        got = getattr(W, fn)(f, step, n, dtype=np.float32 if dt_name == "f32" else np.float64)
        assert np.array_equal(got.view(np.uint8), ref[name].view(np.uint8)), name
