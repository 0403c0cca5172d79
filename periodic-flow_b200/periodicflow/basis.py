"""Host-side description of the periodic box (the reference's basis.py:10-92).

The device computes wavenumbers from mode indices; the arrays built here are
the host views the reference exposes (``x``, ``k``, ``k2``, ``k_over_k2``,
``nyquist_mask``) for user code such as the example scripts.
"""
from __future__ import annotations

import numpy as np

DEALIAS_RULES = {"3/2": "pad", "pad": "pad", "2/3": "truncate", "truncate": "truncate"}


def parse_domain(domain, dim):
    """Domain forms accepted by basis.py:50-60."""
    if isinstance(domain, float):
        return [(0.0, domain) for _ in range(dim)]
    if isinstance(domain, (list, tuple)):
        if all(isinstance(i, (list, tuple)) for i in domain):
            return [tuple(float(v) for v in d) for d in domain]
        if all(isinstance(i, float) for i in domain):
            return [tuple(domain) for _ in range(dim)]
        raise ValueError("Invalid domain.")
    raise ValueError("Input domain must be either float, list or tuple.")


class FourierSpace:
    """Wavenumbers, mesh and masks of an (n0, n1[, n2]) periodic box.

    Last axis real-to-complex (rfftfreq ordering, Nyquist at +n/2); other axes
    complex (fftfreq ordering, Nyquist at -n/2); wavenumbers scaled by 2 pi/L.
    """

    def __init__(self, comm, mpi_rank, N, domain=2 * np.pi, dealias="3/2",
                 mask_nyquist=False, fft_plan="FFTW_MEASURE", decomposition="slab"):
        self.comm = comm
        self.mpi_rank = mpi_rank
        self.N = [int(n) for n in N]
        self.dim = len(self.N)
        self.domain = parse_domain(domain, self.dim)
        rule = DEALIAS_RULES.get(dealias)
        if rule is None:
            raise ValueError(f"FourierSpace: Invalid dealiasing rule: {dealias}.")
        self.dealias = dealias
        self.dealias_rule = rule
        self.fft_plan = fft_plan
        self.decomposition = decomposition
        d = self.dim
        self.lengths = [float(b - a) for a, b in self.domain]
        self.shape_spectral = tuple(self.N[:-1]) + (self.N[-1] // 2 + 1,)
        self.shape_physical = tuple(self.N)
        kint = []
        for ax in range(d):
            n = self.N[ax]
            kk = (np.arange(n // 2 + 1, dtype=np.float64) if ax == d - 1
                  else np.fft.fftfreq(n, 1.0 / n))
            shp = [1] * d
            shp[ax] = kk.size
            kint.append(kk.reshape(shp))
        self.k = np.array([np.broadcast_to(kint[ax] * (2 * np.pi / self.lengths[ax]),
                                           self.shape_spectral) for ax in range(d)])
        self.k2 = np.sum(self.k ** 2, axis=0)
        self.k_over_k2 = self.k / np.where(self.k2 == 0, 1, self.k2)
        self.x = []
        for ax in range(d):
            a, _ = self.domain[ax]
            shp = [1] * d
            shp[ax] = self.N[ax]
            self.x.append((a + self.lengths[ax] * np.arange(self.N[ax]) / self.N[ax]).reshape(shp))
        if mask_nyquist:
            keep = np.ones(self.shape_spectral, dtype=bool)
            for ax in range(d):
                idx = np.zeros(self.shape_spectral[ax], dtype=bool)
                if self.N[ax] % 2 == 0:
                    idx[self.N[ax] // 2] = True
                shp = [1] * d
                shp[ax] = idx.size
                keep &= ~idx.reshape(shp)
            self.nyquist_mask = keep.astype(np.float64)
        else:
            self.nyquist_mask = None
