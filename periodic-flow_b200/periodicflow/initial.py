"""Initial fields (host NumPy set-up, like the reference's example scripts).

* ``taylor_green(x)``: u = sin x cos y cos z, v = -cos x sin y cos z, w = 0
  (examples/tgv3d.py:4-11).
* ``spectral_random_field(space, seed)``: random solenoidal field whose shell
  spectrum is E(k) ~ k^4 exp(-2 (k/kp)^2), total energy ``energy_total``:
  Gaussian physical-space noise from ``numpy.random.default_rng(seed)`` is
  transformed (so the field is exactly Hermitian), Leray-projected, the k = 0
  mode removed and every integer shell rescaled to the target spectrum.
"""
from __future__ import annotations

import numpy as np


def taylor_green(x):
    shape = np.broadcast_shapes(*[xi.shape for xi in x])
    u = np.zeros((3,) + shape)
    u[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    u[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    return u


def _half_weight(N):
    w = np.full(N[-1] // 2 + 1, 2.0)
    w[0] = 1.0
    if N[-1] % 2 == 0:
        w[-1] = 1.0
    return w


def spectral_random_field(space, seed, kp=4.0, energy_total=0.5):
    """u_hat (complex128, reference layout) for a FourierSpace-like ``space``."""
    N = list(space.N)
    d = len(N)
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((d,) + tuple(N))
    axes = tuple(range(1, d + 1))
    uh = np.fft.rfftn(z, axes=axes) / float(np.prod(N))
    k, k2 = space.k, space.k2
    kk2 = k / np.where(k2 == 0, 1, k2)
    p = np.sum(kk2 * uh, axis=0)
    uh = (uh - p[None] * k) * np.where(k2 == 0, 0, 1)
    lengths = [b - a for a, b in space.domain]
    shell = np.floor(np.sqrt(k2) * lengths[0] / (2 * np.pi) + 0.5).astype(np.int64)
    nb = int(shell.max()) + 1
    w = _half_weight(N).reshape([1] * (d - 1) + [-1])
    e = 0.5 * w * np.sum(np.abs(uh) ** 2, axis=0)
    cur = np.bincount(shell.ravel(), weights=np.broadcast_to(e, shell.shape).ravel(),
                      minlength=nb)[:nb]
    kk = np.arange(nb, dtype=np.float64)
    target = kk ** 4 * np.exp(-2.0 * (kk / kp) ** 2)
    target[0] = 0.0
    target *= energy_total / target.sum()
    scale = np.where(cur > 0, np.sqrt(target / np.where(cur > 0, cur, 1.0)), 0.0)
    return uh * scale[shell][None]
