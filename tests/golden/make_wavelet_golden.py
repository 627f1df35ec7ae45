"""Write the wavelet fixtures with the reference's own wavelet module.

    python tests/golden/make_wavelet_golden.py [<TorchWI checkout>]

Imports torchwi/source/wavelets.py by path (nothing else of the reference)
and records, for ricker and fdgaus over a grid of frequencies and time
steps in float32 and float64, a truncated SHA-256 of the output bytes
(wavelets.json), plus full arrays of the configurations the benchmarks use
(wavelets.npz).  The tests compare torchwi_b200.source.wavelets with these
files only; they never need the reference at run time.
"""

from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

FREQS = [1.5 + 0.5 * k for k in range(60)]          # 1.5 .. 31 Hz
DTS = [2.5e-4, 5e-4, 8e-4, 1e-3, 2e-3]
NT = 1000
DTYPES = {"float32": np.float32, "float64": np.float64}
FULL = {  # name -> (function, freq, dt, nt, dtype)
    "ricker_8hz_dt0.8ms_nt4000_f32": ("ricker", 8.0, 8e-4, 4000, "float32"),
    "ricker_10hz_dt1ms_nt1000_f32": ("ricker", 10.0, 1e-3, 1000, "float32"),
    "ricker_10hz_dt1ms_nt1000_f64": ("ricker", 10.0, 1e-3, 1000, "float64"),
    "fdgaus_10hz_dt1ms_nt1000_f32": ("fdgaus", 10.0, 1e-3, 1000, "float32"),
    "fdgaus_10hz_dt1ms_nt1000_f64": ("fdgaus", 10.0, 1e-3, 1000, "float64"),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def case_key(fn, freq, dt, dtype):
    return f"{fn}/{freq:g}/{dt:g}/{dtype}"


def main(root):
    path = os.path.join(root, "torchwi", "source", "wavelets.py")
    if not os.path.exists(path):
        raise SystemExit(f"{path} not found: pass the TorchWI checkout or set REFROOT")
    spec = importlib.util.spec_from_file_location("reference_wavelets", path)
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    hashes = {}
    for fn in ("ricker", "fdgaus"):
        for dname, dt_ in DTYPES.items():
            for dt in DTS:
                for f in FREQS:
                    hashes[case_key(fn, f, dt, dname)] = digest(getattr(ref, fn)(f, dt, NT, dtype=dt_))
    with open(os.path.join(HERE, "wavelets.json"), "w") as fh:
        json.dump({"nt": NT, "freqs": FREQS, "dts": DTS, "sha256_16": hashes}, fh, indent=0)
    full = {name: getattr(ref, fn)(f, dt, nt, dtype=DTYPES[d]) for name, (fn, f, dt, nt, d) in FULL.items()}
    np.savez_compressed(os.path.join(HERE, "wavelets.npz"), **full)
    print(f"wrote {len(hashes)} hashes and {len(full)} full arrays")


if __name__ == "__main__":
    here_repo = os.path.dirname(os.path.dirname(HERE))
    default = os.environ.get("REFROOT") or os.path.join(os.path.dirname(here_repo), "reference")
    main(sys.argv[1] if len(sys.argv) > 1 else default)
