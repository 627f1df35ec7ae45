"""Source wavelets (restated from torchwi/source/wavelets.py:3-52).

Both generators return FP64 numpy arrays, as the reference does; callers
cast to FP32 before propagation.  Samples are evaluated one at a time with
scalar ``np.exp`` so the values match the reference bit for bit (the
vectorised exp differs in the last ulp).
"""

import numpy as np


def ricker(freq, dt, nt, dtype=np.float64):
    """Ricker wavelet with peak parameter ``freq/2/1.08`` delayed so that the
    first sample is ~1e-3 of the peak (torchwi/source/wavelets.py:3-23)."""
    vm2 = (freq / 2.0 / 1.08) ** 2
    pi2 = np.pi ** 2

    def shape(tt):
        arg = pi2 * tt ** 2
        return (1.0 - 2.0 * vm2 * arg) * np.exp(-vm2 * arg)

    a0 = shape(0.0)
    t0 = 0.0
    for i in range(nt):                   # first sample below 1e-3 of a(0)
        if abs(shape(i * dt)) < a0 * 1.0e-3:
            t0 = i * dt
            break
    return np.array([shape(t0 - i * dt) for i in range(nt)], dtype=dtype)


def fdgaus(cutoff, dt, nt, dtype=np.float64):
    """First derivative of a Gaussian, normalised to unit peak
    (torchwi/source/wavelets.py:26-52)."""
    a = np.pi * (5.0 * cutoff / 8.0) ** 2
    amp = np.sqrt(a / np.pi)

    def gauss(tt):
        return amp * np.exp(max(-a * tt ** 2, -32.0))

    threshold = 0.001 * gauss(0.0)
    t0 = 0.0
    for i in range(nt):
        if gauss(i * dt) < threshold:
            t0 = (i - 1) * dt
            break
    sqpi = np.sqrt(np.pi)
    w = np.array([-2.0 * np.sqrt(a) * a * (i * dt - t0)
                  * np.exp(max(-a * (i * dt - t0) ** 2, -32.0)) / sqpi
                  for i in range(nt)], dtype=np.float64)
    w /= w.max()
    return w.astype(dtype)
