"""RSF and shot-gather files (CPU).  Fixtures in tests/golden/rsf/ were
written and read back by the reference's own RSF module
(tests/golden/make_rsf_golden.py)."""
import json
import os

import numpy as np
import pytest
import torch

from torchwi_b200.io import (TimeDataset, TimeForwardDataset, load_gathers, read_survey, rsf,
                             save_gathers, time_dataloader, time_distributed_dataloader,
                             time_forward_dataloader)

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rsf")
CASES = ["vel", "wavelet", "shot", "cube_int", "cplx", "ascii"]


@pytest.fixture
def expected():
    return dict(np.load(os.path.join(GOLD, "rsf_expected.npz")))


@pytest.mark.parametrize("name", CASES)
def test_reads_what_the_reference_reads(name, expected, monkeypatch):
    monkeypatch.chdir(GOLD)
    keys = [k.split(".", 1)[1] for k in expected if k.startswith(name + ".") and not k.endswith("_source")]
    got = rsf.fromfile(name + ".rsf", " ".join(keys))
    for k, v in zip(keys, got):
        want = expected[f"{name}.{k}"]
        if k == "data":
            assert v.dtype == want.dtype and v.shape == want.shape
            assert v.tobytes() == want.tobytes()
        else:
            assert np.asarray(v) == want, k


def test_last_occurrence_wins(expected, monkeypatch):
    monkeypatch.chdir(GOLD)
    n1, n2, d1, label1, data = rsf.fromfile("history.rsf", "n1 n2 d1 label1 data")
    assert (n1, n2, d1, label1) == (int(expected["history.n1"]), int(expected["history.n2"]),
                                    float(expected["history.d1"]), str(expected["history.label1"]))
    assert label1 == "Depth below datum"
    assert data.tobytes() == expected["history.data"].tobytes()


@pytest.mark.parametrize("name", CASES)
def test_writes_the_reference_header_and_bytes(name, expected, tmp_path, monkeypatch):
    headers = json.load(open(os.path.join(GOLD, "headers.json")))
    monkeypatch.chdir(GOLD)
    with rsf.input(name + ".rsf") as f:
        keys = {}
        for i in range(1, f.dimension + 1):
            ax = f.get(f"ax{i}")
            keys.update({f"n{i}": ax.n, f"o{i}": ax.o, f"d{i}": ax.d})
            if ax.label:
                keys[f"label{i}"] = ax.label
            if ax.unit:
                keys[f"unit{i}"] = ax.unit
        fmt = f.data_format
    data = expected[f"{name}.data"]
    monkeypatch.chdir(tmp_path)
    rsf.tofile(name + ".rsf", data, abspath=False, data_format=fmt, **keys)
    assert open(name + ".rsf").read() == headers[name]
    assert open(name + ".rsf@", "rb").read() == open(os.path.join(GOLD, name + ".rsf@"), "rb").read()


def test_one_dimensional_native_data_read_as_a_vector(monkeypatch):
    monkeypatch.chdir(GOLD)
    nt, dt, w = rsf.fromfile("wavelet.rsf", "n1 d1 data")
    assert w.shape == (nt,) and dt == 0.001


def test_traces_and_absolute_paths(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    path = str(tmp_path / "a.rsf")
    rsf.tofile(path, a, n1=4, n2=3)
    assert os.path.isabs(rsf.fromfile(path, "in"))
    with rsf.input(path) as f:
        trcs = list(f.traces())
    assert [t.tolist() for t in trcs] == a.tolist()


def test_errors_exit_with_status_one(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    with pytest.raises(SystemExit) as e:
        rsf.output("x.rsf", n1=3, bogus=1)
    assert e.value.code == 1
    open("noin.rsf", "w").write("n1=3\n")
    with pytest.raises(rsf.RSFError):
        rsf.fromfile("noin.rsf", "data")
    open("gone.rsf", "w").write('in="nowhere.rsf@" n1=3\n')
    with pytest.raises(rsf.RSFError, match="not exists"):
        rsf.fromfile("gone.rsf", "data")
    with pytest.raises(rsf.RSFError, match="Wrong type"):
        rsf.tofile("y.rsf", np.zeros(3), n1=3, data_format="native_double")   # fails at the write


def test_read_survey_as_the_examples_do(monkeypatch):
    monkeypatch.chdir(GOLD)
    s = read_survey("vel.rsf", "wavelet.rsf", "shot.rsf")
    assert (s.nx, s.ny, s.h, s.nt, s.dt, s.nshot) == (40, 30, 10.0, 100, 0.001, 5)
    assert s.vel.shape == (40, 30) and s.w.shape == (100,) and s.sxy.shape == (5, 2)
    np.testing.assert_array_equal(s.sx, np.arange(5) * 50.0 + 25.0)


def _gathers(n=5, nt=7, nx=6):
    return torch.from_numpy(np.random.default_rng(3).standard_normal((n, nt, nx)).astype(np.float32))


def test_gathers_round_trip_and_datasets(tmp_path):
    g = _gathers()
    pat = str(tmp_path / "shots" / "seismo.%04d")
    save_gathers(g, pat, range(5))
    assert os.path.getsize(pat % 3) == 7 * 6 * 4
    back = load_gathers(pat, [4, 1, 2], 7, 6)
    assert torch.equal(back, g[[4, 1, 2]])

    sxy = torch.tensor([[10.0 * k, 20.0] for k in range(5)])
    ds = TimeDataset(sxy, pat, with_index=True, shape=(7, 6))
    sx, sy, obs, idx = ds[2]
    assert idx == 2 and torch.equal(obs, g[2]) and float(sx) == 20.0
    flat = TimeDataset(sxy, pat)[1][2]
    assert flat.shape == (42,)
    assert torch.equal(TimeDataset(sxy, pat, shape=(7, 6), transpose=True)[0][2], g[0].T)
    assert len(TimeForwardDataset(sxy)) == 5 and TimeForwardDataset(sxy)[3][2] == 3

    batches = list(time_dataloader(pat, sxy, shape=(7, 6)))
    assert len(batches) == 5 and batches[0][2].shape == (1, 7, 6)
    assert [int(b[2]) for b in time_forward_dataloader(sxy)] == list(range(5))


def test_distributed_loader_splits_shots(tmp_path):
    pat = str(tmp_path / "s.%d")
    save_gathers(_gathers(), pat, range(5))
    sxy = torch.zeros(5, 2)
    seen = []
    for rank in (0, 1):
        seen += [int(b[3]) for b in time_distributed_dataloader(pat, sxy, size=2, rank=rank)]
    assert sorted(set(seen)) == list(range(5)) and len(seen) == 6   # sampler pads to equal shares


def test_load_gathers_rejects_short_files(tmp_path):
    pat = str(tmp_path / "s.%d")
    save_gathers(_gathers(n=2), pat, range(2))
    with pytest.raises(ValueError):
        load_gathers(pat, [0, 1], 7, 7)
