"""Source wavelets (restated from torchwi/source/wavelets.py:3-52).

Both generators work in the requested storage type the way the reference
does: every sample is evaluated in FP64 with scalar ``np.exp`` (the
vectorised exp differs in the last ulp) and rounded to ``dtype`` when it is
stored; the onset search compares stored samples in ``dtype`` arithmetic,
and ``fdgaus`` normalises the stored samples in place, in ``dtype``.  With
``dtype=np.float32`` the samples therefore equal the reference's float32
output bit for bit (not a float64 result cast at the end).
"""

import numpy as np


def _sampled(fn, n, dt, dtype):
    """fn(i*dt) for i in [0, n), each value rounded to `dtype` on store."""
    out = np.empty(n, dtype=dtype)
    for i in range(n):
        out[i] = fn(i * dt)
    return out


def ricker(freq, dt, nt, dtype=np.float64):
    """Ricker wavelet with peak parameter ``freq/2/1.08``, delayed to the
    first sample whose magnitude drops below 1e-3 of the zero-lag value
    (torchwi/source/wavelets.py:3-23)."""
    vm2 = (freq / 2.0 / 1.08) ** 2
    pi2 = np.pi ** 2

    def shape(tt):
        arg = pi2 * tt ** 2
        return (1.0 - 2.0 * vm2 * arg) * np.exp(-vm2 * arg)

    undelayed = _sampled(shape, nt, dt, dtype)
    floor = undelayed[0] * 1.0e-3          # dtype arithmetic, as the reference's array
    onset = next((i for i in range(nt) if np.abs(undelayed[i]) < floor), 0)
    t0 = onset * dt
    return _sampled(lambda tt: shape(t0 - tt), nt, dt, dtype)


def fdgaus(cutoff, dt, nt, dtype=np.float64):
    """First derivative of a Gaussian, normalised to unit peak
    (torchwi/source/wavelets.py:26-52)."""
    a = np.pi * (5.0 * cutoff / 8.0) ** 2
    amp = np.sqrt(a / np.pi)
    sqpi = np.sqrt(np.pi)

    def expo(tt):                          # exp(-a t^2), exponent floored at -32
        return np.exp(max(-a * tt ** 2, -32.0))

    gauss = _sampled(lambda tt: amp * expo(tt), nt, dt, dtype)
    threshold = 0.001 * gauss[0]
    t0 = 0.0
    for i in range(nt):
        if gauss[i] < threshold:
            t0 = (i - 1) * dt
            break
    w = _sampled(lambda tt: -2.0 * np.sqrt(a) * a * (tt - t0) * expo(tt - t0) / sqpi, nt, dt, dtype)
    w /= w.max()
    return w
