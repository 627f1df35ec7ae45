"""Write the RSF fixtures with the reference's own RSF module.

Run from anywhere where the reference sources are available:

    python tests/golden/make_rsf_golden.py [<TorchWI checkout>]

It imports torchwi/io/rsf.py by path (nothing else of the reference), writes
seeded datasets into tests/golden/rsf/ with relative `in=` paths, and records
what the reference's reader returns for each (rsf_expected.npz) plus each
header's exact text (headers.json), so the tests need no reference at run
time.  numpy 2 removed `np.product`, which the reference's `RSF.size` calls;
it is aliased to `np.prod` (same result) before the import.
"""
import importlib.util
import json
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rsf")


def _load_reference_rsf(root):
    if not hasattr(np, "product"):
        np.product = np.prod
    path = os.path.join(root, "torchwi", "io", "rsf.py")
    spec = importlib.util.spec_from_file_location("reference_rsf", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(root):
    rsf = _load_reference_rsf(root)
    os.makedirs(OUT, exist_ok=True)
    here = os.getcwd()
    os.chdir(OUT)
    rng = np.random.default_rng(77)
    cases = {
        # velocity model as the examples read it: n1 = nz (fast), n2 = nx, d1 = h
        "vel": (rng.uniform(1500, 4500, (40, 30)).astype(np.float32),
                dict(n1=30, n2=40, d1=10.0, d2=10.0, o1=0.0, o2=0.0, label1="Depth", unit1="m",
                     label2="Distance", unit2="m")),
        "wavelet": (rng.standard_normal(100).astype(np.float32), dict(n1=100, d1=0.001, o1=0.0,
                                                                        label1="Time", unit1="s")),
        "shot": (np.stack([np.arange(5) * 50.0 + 25.0, np.full(5, 20.0)], 1).astype(np.float32),
                 dict(n1=2, n2=5, d1=1.0, d2=1.0)),
        "cube_int": (rng.integers(-1000, 1000, (3, 4, 5)).astype(np.int32),
                     dict(n1=5, n2=4, n3=3, data_format="native_int")),
        "cplx": ((rng.standard_normal((6, 7)) + 1j * rng.standard_normal((6, 7))).astype(np.complex64),
                 dict(n1=7, n2=6, o2=-3.5, d2=0.25, data_format="native_complex")),
        "ascii": (np.linspace(-1.0, 1.0, 9).astype(np.float32),
                  dict(n1=9, d1=0.5, data_format="ascii_float")),
    }
    expected, headers = {}, {}
    for name, (data, keys) in cases.items():
        fname = name + ".rsf"
        rsf.tofile(fname, data, abspath=False, **keys)
        with open(fname) as fh:
            headers[name] = fh.read()
        n = [k for k in ("n1", "n2", "n3") if k in keys]
        got = rsf.fromfile(fname, " ".join(n + ["d1", "o1", "esize", "data_format"]))
        for k, v in zip(n + ["d1", "o1", "esize", "data_format"], got):
            expected[f"{name}.{k}"] = np.asarray(v)
        try:
            expected[f"{name}.data"] = np.asarray(rsf.fromfile(fname, "data"))
            expected[f"{name}.data_source"] = np.asarray("reference reader")
        except TypeError:
            # the reference's RSF.shape fails for one-dimensional datasets
            # (rsf.py:240-246): record the samples it wrote instead
            expected[f"{name}.data"] = np.fromfile(fname + "@", dtype=data.dtype)
            expected[f"{name}.data_source"] = np.asarray("bytes written by the reference")
    # a header with an appended history: the last occurrence of a key wins
    with open("history.rsf", "w") as fh:
        fh.write(headers["vel"].replace('in="vel.rsf@"', 'in="missing.rsf@"')
                 + '\nsfwindow:\nin="vel.rsf@" n2=20 d1=12.5 label1="Depth below datum"\n')
    got = rsf.fromfile("history.rsf", "n1 n2 d1 label1 data")
    for k, v in zip(["n1", "n2", "d1", "label1", "data"], got):
        expected[f"history.{k}"] = np.asarray(v)
    np.savez(os.path.join(OUT, "rsf_expected.npz"), **expected)
    with open(os.path.join(OUT, "headers.json"), "w") as fh:
        json.dump(headers, fh, indent=1, sort_keys=True)
    os.chdir(here)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    default = os.environ.get("REFROOT") or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(here))),
                                                        "reference")
    main(sys.argv[1] if len(sys.argv) > 1 else default)
