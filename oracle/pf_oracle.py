"""FP64 NumPy restatement of periodicflow's RHS + time-stepping path (the oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  Nothing in the product imports it.

Every function cites the reference file:line it restates (paths are relative to
the periodic-flow project root).  The FFT layer stands in for the third-party
package shenfun (unpinned in setup.py:11-14, absent from this image); its
conventions are ASSUMED, not pinned by any reference test:

* forward transform normalised by 1/prod(N), backward unnormalised;
* last axis real-to-complex (rfftfreq wavenumbers), other axes complex
  (fftfreq wavenumbers, Nyquist at -N/2);
* '2/3' dealiasing zeroes modes with 3|k_i| >= N_i on a copy of the input of
  the backward transform (the spectral state keeps all modes);
* Nyquist mask zeroes index N_i/2 on every axis.

Noise parity is pinned two ways: reference-order NumPy draws injected into both
codes, and a counter-based Philox4x32-10 generator restated here bit-for-bit in
its integer part (Salmon et al., "Parallel random numbers: as easy as 1, 2, 3",
SC'11) with a Box-Muller transform.

Features absent from the reference (its add_forcing is a no-op,
space_solver.py:267-271) are restated here from their definitions so the new
device code has a checker: linear band forcing at constant injection rate, a
CFL-adaptive dt, the k^4 exp(-2(k/4)^2) random solenoidal initial field and the
energy / enstrophy / spectrum reductions.
"""
from __future__ import annotations

import math as _m
import numpy as np
import scipy.fft as sfft

__all__ = [
    "Grid", "curl", "cross", "apply_linear_operator", "leray_projection",
    "symmetrize", "noise_divergence", "INTEGRATORS", "OracleSolver",
    "philox4x32_10", "philox_noise_fields", "numpy_noise_fields",
    "spectral_random_field", "taylor_green", "energy", "enstrophy", "spectrum",
    "NOISE_FACTORS",
]

FFT_WORKERS = None  # None -> scipy default (1); bench sets os.cpu_count()


# ----------------------------------------------------------------------------
# Discretisation: basis.py:34-92
# ----------------------------------------------------------------------------
class Grid:
    """Wavenumbers, masks and transforms of one periodic box.

    Restates basis.py:50-77 (domain parsing, wavenumbers, k2, k/k^2) and the
    dealias rule table of basis.py:79-92 for the '2/3' / 'truncate' rule.
    """

    def __init__(self, N, domain=2 * np.pi, dealias="2/3", mask_nyquist=False):
        N = [int(n) for n in N]
        self.N = N
        self.dim = len(N)
        # basis.py:50-60
        if isinstance(domain, float):
            self.domain = [(0, domain) for _ in range(self.dim)]
        elif isinstance(domain, (list, tuple)):
            if all(isinstance(i, (list, tuple)) for i in domain):
                self.domain = [tuple(d) for d in domain]
            elif all(isinstance(i, float) for i in domain):
                self.domain = [tuple(domain) for _ in range(self.dim)]
            else:
                raise ValueError("Invalid domain.")
        else:
            raise ValueError("Input domain must be either float, list or tuple.")
        self.lengths = [float(b - a) for a, b in self.domain]
        if dealias not in ("3/2", "pad", "2/3", "truncate"):
            raise ValueError(f"FourierSpace: Invalid dealiasing rule: {dealias}.")
        self.dealias = dealias
        d = self.dim
        self.spec_shape = tuple(N[:-1]) + (N[-1] // 2 + 1,)
        self.phys_shape = tuple(N)
        # integer wavenumbers per axis (fftfreq / rfftfreq ordering)
        kint = []
        for ax in range(d):
            if ax == d - 1:
                kk = np.arange(N[ax] // 2 + 1, dtype=np.float64)
            else:
                kk = np.fft.fftfreq(N[ax], 1.0 / N[ax])
            shp = [1] * d
            shp[ax] = kk.size
            kint.append(kk.reshape(shp))
        self.kint1d = kint
        # basis.py:65,75-77: scaled, broadcast wavenumbers
        self.k = np.array([np.broadcast_to(kint[ax] * (2 * np.pi / self.lengths[ax]),
                                           self.spec_shape) for ax in range(d)])
        self.k2 = np.sum(self.k ** 2, axis=0)
        self.k_over_k2 = self.k / np.where(self.k2 == 0, 1, self.k2)
        # space_solver.py:143
        self.mask_k0 = np.where(self.k2 == 0, 0, 1).astype(np.float64)
        # 2/3 rule as an index predicate (see module docstring)
        keep = np.ones(self.spec_shape, dtype=bool)
        for ax in range(d):
            keep = keep & (3 * np.abs(kint[ax]) < N[ax])
        self.dealias_mask = keep.astype(np.float64)
        # basis.py:72 get_mask_nyquist
        if mask_nyquist:
            nyq = np.ones(self.spec_shape, dtype=bool)
            for ax in range(d):
                idx = np.zeros(self.spec_shape[ax], dtype=bool)
                if N[ax] % 2 == 0:
                    idx[N[ax] // 2] = True
                shp = [1] * d
                shp[ax] = idx.size
                nyq = nyq & ~idx.reshape(shp)
            self.nyquist_mask = nyq.astype(np.float64)
        else:
            self.nyquist_mask = None
        # basis.py:74 local_mesh: x_j = a + L j / N, sparse broadcastable arrays
        self.x = []
        for ax in range(d):
            a, _ = self.domain[ax]
            xx = a + self.lengths[ax] * np.arange(N[ax]) / N[ax]
            shp = [1] * d
            shp[ax] = N[ax]
            self.x.append(xx.reshape(shp))
        self.prodN = float(np.prod(N))
        # half-spectrum weights: planes k_last = 0 and Nyquist count once
        w = np.full(self.spec_shape[-1], 2.0)
        w[0] = 1.0
        if N[-1] % 2 == 0:
            w[-1] = 1.0
        shp = [1] * d
        shp[-1] = w.size
        self.half_weight = w.reshape(shp)

    # shenfun V.forward / V.backward (space_solver.py:215-225)
    def forward(self, u):
        axes = tuple(range(-self.dim, 0))
        return sfft.rfftn(u, axes=axes, workers=FFT_WORKERS) / self.prodN

    def backward(self, uh):
        axes = tuple(range(-self.dim, 0))
        return sfft.irfftn(uh, s=self.N, axes=axes, workers=FFT_WORKERS) * self.prodN

    def backward_dealiased(self, uh):
        """Vp.backward / Wp.backward of space_solver.py:284,291.

        '2/3': backward of the truncated copy.  '3/2' (basis.py:80-81): the
        spectrum padded onto M = 3N/2 per axis (Nyquist modes of even sides
        split in half between +N/2 and -N/2; halved on the last axis), then the
        unnormalised backward transform on the M grid.
        """
        if self.dealias in ("2/3", "truncate"):
            return self.backward(uh * self.dealias_mask)
        M = self.padded_shape()
        axes = tuple(range(-self.dim, 0))
        return sfft.irfftn(self.pad(uh), s=M, axes=axes, workers=FFT_WORKERS) * float(np.prod(M))

    def forward_dealiased(self, u):
        """Vp.forward of space_solver.py:296: '2/3' plain forward; '3/2' forward
        on the M grid (normalised by 1/prod M) folded back to the N grid."""
        if self.dealias in ("2/3", "truncate"):
            return self.forward(u)
        M = self.padded_shape()
        axes = tuple(range(-self.dim, 0))
        return self.truncate(sfft.rfftn(u, axes=axes, workers=FFT_WORKERS) / float(np.prod(M)))

    def padded_shape(self):
        return [3 * n // 2 for n in self.N]

    @staticmethod
    def _sl(ndim, axis, lo, hi):
        idx = [slice(None)] * ndim
        idx[axis] = slice(lo, hi)
        return tuple(idx)

    def pad(self, uh):
        """N-grid half spectrum (leading component axes allowed) -> M grid."""
        out = np.asarray(uh)
        nd = out.ndim
        for ax in range(self.dim):
            a = nd - self.dim + ax
            N, M = self.N[ax], 3 * self.N[ax] // 2
            h = N // 2
            last = ax == self.dim - 1
            shp = list(out.shape)
            shp[a] = M // 2 + 1 if last else M
            new = np.zeros(shp, dtype=np.complex128)
            S = lambda lo, hi: self._sl(nd, a, lo, hi)  # noqa: E731
            if last:
                new[S(0, h)] = out[S(0, h)]
                new[S(h, h + 1)] = (0.5 if N % 2 == 0 else 1.0) * out[S(h, h + 1)]
            else:
                new[S(0, h)] = out[S(0, h)]
                new[S(M - h + 1, M)] = out[S(N - h + 1, N)]
                new[S(h, h + 1)] = 0.5 * out[S(h, h + 1)]
                new[S(M - h, M - h + 1)] = 0.5 * out[S(h, h + 1)]
            out = new
        return out

    def truncate(self, P):
        """M-grid half spectrum -> N grid: the last axis first (its Nyquist
        entry gains the conjugate of the mirror mode, i.e. the -N/2 partner),
        then every complex axis folds +N/2 and -N/2 into the Nyquist index."""
        out = np.asarray(P)
        nd = out.ndim
        a = nd - 1
        N = self.N[-1]
        h = N // 2
        out = out[self._sl(nd, a, 0, h + 1)].copy()
        if N % 2 == 0:
            nyq = out[self._sl(nd, a, h, h + 1)]
            mir = nyq
            for ax in range(self.dim - 1):
                b = nd - self.dim + ax
                mir = np.roll(np.flip(mir, axis=b), 1, axis=b)
            out[self._sl(nd, a, h, h + 1)] = nyq + np.conj(mir)
        for ax in range(self.dim - 1):
            b = nd - self.dim + ax
            N, M = self.N[ax], 3 * self.N[ax] // 2
            h = N // 2
            shp = list(out.shape)
            shp[b] = N
            new = np.zeros(shp, dtype=np.complex128)
            S = lambda lo, hi: self._sl(nd, b, lo, hi)  # noqa: E731
            new[S(0, h)] = out[S(0, h)]
            new[S(N - h + 1, N)] = out[S(M - h + 1, M)]
            new[S(h, h + 1)] = out[S(h, h + 1)] + out[S(M - h, M - h + 1)]
            out = new
        return out


# ----------------------------------------------------------------------------
# Pointwise kernels: math.py:4-100
# ----------------------------------------------------------------------------
def cross(a, b):
    """math.py:4-28. 2D: (a1*b, -a0*b) with scalar b; 3D: full cross product."""
    if a.shape[0] == 2:
        return np.stack([a[1] * b, -a[0] * b])
    return np.stack([a[1] * b[2] - a[2] * b[1],
                     a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]])


def curl(k, a):
    """math.py:31-49. 2D: scalar i(k0 a1 - k1 a0); 3D: i k x a."""
    if a.shape[0] == 2:
        return 1j * (k[0] * a[1] - k[1] * a[0])
    return np.stack([1j * (k[1] * a[2] - k[2] * a[1]),
                     1j * (k[2] * a[0] - k[0] * a[2]),
                     1j * (k[0] * a[1] - k[1] * a[0])])


def apply_linear_operator(L, u):
    """math.py:52-68: Lu[i] = L * u[i]."""
    return L[None] * u


def leray_projection(u, k, k_over_k2):
    """math.py:71-100: p = (k/k^2).u ; u -= p k.  Returns (projected u, p)."""
    p = np.sum(k_over_k2 * u, axis=0)
    return u - p[None] * k, p


# ----------------------------------------------------------------------------
# Noise kernels: space_solver.py:15-64, 227-265
# ----------------------------------------------------------------------------
def symmetrize(w):
    """space_solver.py:15-42: W_sym = (W + W^T) sqrt(1/2), d x d row-major."""
    d = int(round(np.sqrt(w.shape[0])))
    ws = np.empty_like(w)
    f = np.sqrt(0.5)
    for a in range(d):
        for b in range(d):
            ws[a * d + b] = (w[a * d + b] + w[b * d + a]) * f
    return ws


def noise_divergence(wsym, k):
    """space_solver.py:45-64: noise_a = i sum_b k_b W_sym[a, b]."""
    d = k.shape[0]
    out = []
    for a in range(d):
        acc = 0
        for b in range(d):
            acc = acc + k[b] * wsym[a * d + b]
        out.append(1j * acc)
    return np.stack(out)


def noise_normal_factor(grid):
    """space_solver.py:143-145: mask(k != 0) / sqrt(prod N) / sqrt(2 - 2/d)."""
    return grid.mask_k0 / np.sqrt(grid.prodN) / np.sqrt(2 - 2 / grid.dim)


def noise_components(grid, noise_type):
    """Number of complex components of w1/w2 (space_solver.py:169)."""
    return grid.dim ** 2 if noise_type == "thermal" else grid.dim


def numpy_noise_fields(grid, noise_type, rng=None):
    """space_solver.py:227-238 in its RNG order: w1.re, w1.im, w2.re, w2.im.

    ``rng`` defaults to NumPy's global legacy generator, as the reference uses.
    """
    r = np.random if rng is None else rng
    shape = (noise_components(grid, noise_type),) + grid.spec_shape
    w1 = r.standard_normal(shape) + 1j * r.standard_normal(shape)
    w2 = r.standard_normal(shape) + 1j * r.standard_normal(shape)
    f = noise_normal_factor(grid)
    return w1 * f, w2 * f


# ---- Philox4x32-10 (Salmon et al. SC'11), restated in NumPy integer math ----
_PHILOX_M0 = np.uint64(0xD2511F53)
_PHILOX_M1 = np.uint64(0xCD9E8D57)
_PHILOX_W0 = np.uint32(0x9E3779B9)
_PHILOX_W1 = np.uint32(0xBB67AE85)
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Ten rounds of Philox4x32 on uint32 counter words and a 2-word key."""
    c0 = np.asarray(c0, dtype=np.uint32)
    c1 = np.asarray(c1, dtype=np.uint32)
    c2 = np.asarray(c2, dtype=np.uint32)
    c3 = np.asarray(c3, dtype=np.uint32)
    k0 = np.uint32(k0)
    k1 = np.uint32(k1)
    with np.errstate(over="ignore"):
        for r in range(10):
            if r > 0:
                k0 = np.uint32(k0 + _PHILOX_W0)
                k1 = np.uint32(k1 + _PHILOX_W1)
            p0 = _PHILOX_M0 * c0.astype(np.uint64)
            p1 = _PHILOX_M1 * c2.astype(np.uint64)
            hi0 = (p0 >> np.uint64(32)).astype(np.uint32)
            lo0 = (p0 & _MASK32).astype(np.uint32)
            hi1 = (p1 >> np.uint64(32)).astype(np.uint32)
            lo1 = (p1 & _MASK32).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
    return c0, c1, c2, c3


def _box_muller(x, y):
    """Two standard normals from two uint32 words: 24-bit uniforms in (0,1)."""
    u = ((x >> np.uint32(8)).astype(np.float64) + 0.5) * (1.0 / 16777216.0)
    v = ((y >> np.uint32(8)).astype(np.float64) + 0.5) * (1.0 / 16777216.0)
    r = np.sqrt(-2.0 * np.log(u))
    return r * np.cos(2.0 * np.pi * v), r * np.sin(2.0 * np.pi * v)


def _hermitian_canonical(grid):
    """Per half-spectrum mode: (index used for the draw, conjugate flag, real flag).

    On the self-conjugate planes (last-axis index 0 and, for even N, N/2) the
    mode (k_0..k_{d-2}) and its mirror (-k) share one draw: the
    lexicographically smaller index draws, the other takes the conjugate, and
    a mode equal to its mirror is real with sqrt(2) * Re so every mode has
    E|w|^2 = 2 before the normal factor.
    """
    N = grid.N
    d = grid.dim
    shp = grid.spec_shape
    idx = np.arange(int(np.prod(shp)), dtype=np.int64).reshape(shp)
    draw = idx.copy()
    conj = np.zeros(shp, dtype=bool)
    real = np.zeros(shp, dtype=bool)
    planes = [0] + ([N[-1] // 2] if N[-1] % 2 == 0 and N[-1] > 1 else [])
    for pl in planes:
        grids = np.meshgrid(*[np.arange(n) for n in N[:-1]], indexing="ij")
        mir = [(-g) % n for g, n in zip(grids, N[:-1])]
        # lexicographic comparison of (k0, k1, ..) vs mirror
        less = np.zeros(grids[0].shape, dtype=bool)
        equal = np.ones(grids[0].shape, dtype=bool)
        for g, m in zip(grids, mir):
            less = less | (equal & (g < m))
            equal = equal & (g == m)
        mir_lin = np.zeros(grids[0].shape, dtype=np.int64)
        for ax, m in enumerate(mir):
            mir_lin = mir_lin * N[ax] + m
        mir_lin = mir_lin * shp[-1] + pl
        sl = (Ellipsis, pl)
        d_sl = draw[sl]
        d_sl[~(less | equal)] = mir_lin[~(less | equal)]
        draw[sl] = d_sl
        conj[sl] = ~(less | equal)
        real[sl] = equal
    return draw, conj, real


def philox_noise_fields(grid, noise_type, seed, step):
    """Counter-based Gaussian w1, w2 for one time step (normal factor applied).

    counter = (draw mode index, pair index, step lo, step hi), key = seed words.
    Complex value v = field * ncomp + comp uses pair v // 2 and the normals
    from words (0,1) when v is even, (2,3) when odd.
    """
    ncomp = noise_components(grid, noise_type)
    draw, conj, real = _hermitian_canonical(grid)
    draw32 = draw.astype(np.uint32)
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    step = int(step) & 0xFFFFFFFFFFFFFFFF
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    s_lo, s_hi = step & 0xFFFFFFFF, step >> 32
    out = np.empty((2, ncomp) + grid.spec_shape, dtype=np.complex128)
    npairs = (2 * ncomp + 1) // 2
    for p in range(npairs):
        x0, x1, x2, x3 = philox4x32_10(draw32, np.uint32(p), np.uint32(s_lo),
                                       np.uint32(s_hi), k0, k1)
        for half, (a, b) in enumerate(((x0, x1), (x2, x3))):
            v = 2 * p + half
            if v >= 2 * ncomp:
                continue
            zr, zi = _box_muller(a, b)
            z = np.where(real, np.sqrt(2.0) * zr, zr) + 1j * np.where(
                real, 0.0, np.where(conj, -zi, zi))
            out[v // ncomp, v % ncomp] = z
    f = noise_normal_factor(grid)
    return out[0] * f, out[1] * f


# ----------------------------------------------------------------------------
# Time integrators: time_integrator.py:7-318
# ----------------------------------------------------------------------------
class _Integrator:
    """time_integrator.py:17-33: shares L, precomputes (1 - dt/2 L)^-1."""

    n_stages = 0
    noise_factor = ()

    def __init__(self, dt, linear_operator):
        self.dt = dt
        self._lin_op = linear_operator
        self._lin_op_inv = 1 / (1 - self.dt / 2 * linear_operator)

    def update_linear_operator(self, L):
        self._lin_op[...] = L
        self._lin_op_inv = 1 / (1 - self.dt / 2 * L)


class ExplicitPC(_Integrator):
    """time_integrator.py:36-56: u = u0 + a dt (N + Lu + f) + sqrt(dt/2) xi."""
    n_stages = 2
    noise_factor = (0.0, 1.0)
    _a = (0.5, 1.0)

    def stepping(self, unew, u0, stage, N, Lu, f, xi):
        a = self._a[stage]
        unew[...] = u0 + a * self.dt * (N + Lu + f) + np.sqrt(0.5 * self.dt) * xi


class ImplicitPC(_Integrator):
    """time_integrator.py:93-119: last stage recomputes Lu = L u0 (:116-117)."""
    n_stages = 2
    noise_factor = (0.0, 1.0)
    _ab = ((0.5, 0.0), (1.0, 0.5))

    def stepping(self, unew, u0, stage, N, Lu, f, xi):
        a, b = self._ab[stage]
        dt = self.dt
        if stage == self.n_stages - 1:
            Lu[...] = apply_linear_operator(self._lin_op, u0)
        unew[...] = self._lin_op_inv * (u0 + a * dt * (N + f) + b * dt * Lu
                                        + np.sqrt(0.5 * dt) * xi)


class RK2(_Integrator):
    """time_integrator.py:161-180 (TVD RK2, no noise).  noise_factor is not
    defined by the reference (solve() would raise there); zeros are supplied."""
    n_stages = 2
    noise_factor = (0.0, 0.0)
    _ab = ((0.0, 1.0), (0.5, 0.5))

    def stepping(self, unew, u0, stage, N, Lu, f, xi):
        a, b = self._ab[stage]
        unew[...] = a * u0 + b * (unew + self.dt * (N + Lu + f))


class RK3(_Integrator):
    """time_integrator.py:213-241 (stochastic TVD RK3)."""
    n_stages = 3
    noise_factor = ((2 * np.sqrt(2) + np.sqrt(3)) / 5,
                    (-4 * np.sqrt(2) + 3 * np.sqrt(3)) / 5,
                    (np.sqrt(2) - 2 * np.sqrt(3)) / 10)
    _ab = ((0.0, 1.0), (3.0 / 4.0, 1.0 / 4.0), (1.0 / 3.0, 2.0 / 3.0))

    def stepping(self, unew, u0, stage, N, Lu, f, xi):
        a, b = self._ab[stage]
        dt = self.dt
        unew[...] = a * u0 + b * (unew + dt * (N + Lu + f) + np.sqrt(dt) * xi)


class RK4(_Integrator):
    """time_integrator.py:278-293 (low-storage RK4, no noise)."""
    n_stages = 4
    noise_factor = (0.0, 0.0, 0.0, 0.0)
    _a = (1.0 / 4.0, 1.0 / 3.0, 1.0 / 2.0, 1.0)

    def stepping(self, unew, u0, stage, N, Lu, f, xi):
        unew[...] = u0 + self._a[stage] * self.dt * (N + Lu + f)


INTEGRATORS = {"explicit_pc": ExplicitPC, "implicit_pc": ImplicitPC,
               "rk2": RK2, "rk3": RK3, "rk4": RK4}
NOISE_FACTORS = {k: tuple(v.noise_factor) for k, v in INTEGRATORS.items()}


# ----------------------------------------------------------------------------
# Diagnostics, forcing, CFL, initial fields (new: absent from the reference)
# ----------------------------------------------------------------------------
def energy(grid, uh):
    """E = 1/2 sum over the full spectrum of |u_hat|^2 (half spectrum, weighted)."""
    return 0.5 * float(np.sum(grid.half_weight * np.sum(np.abs(uh) ** 2, axis=0)))


def enstrophy(grid, uh):
    """Z = 1/2 sum |k|^2 |u_hat|^2 over the full spectrum."""
    return 0.5 * float(np.sum(grid.half_weight * grid.k2 * np.sum(np.abs(uh) ** 2, axis=0)))


def shell_index(grid):
    """Shell bin of every mode: nearest integer of |k| in units of 2 pi / L_0."""
    kmag = np.sqrt(grid.k2) * grid.lengths[0] / (2 * np.pi)
    return np.floor(kmag + 0.5).astype(np.int64)


def spectrum(grid, uh, nbins=None):
    """Shell-summed energy spectrum E(k) (FP64)."""
    sidx = shell_index(grid)
    if nbins is None:
        nbins = int(sidx.max()) + 1
    e = 0.5 * grid.half_weight * np.sum(np.abs(uh) ** 2, axis=0)
    return np.bincount(sidx.ravel(), weights=np.broadcast_to(e, sidx.shape).ravel(),
                       minlength=nbins)[:nbins]


def forcing_mask(grid, kf):
    """Forced band 0 < |k| <= kf (scaled wavenumbers)."""
    return ((grid.k2 > 0) & (grid.k2 <= kf * kf)).astype(np.float64)


def linear_forcing(grid, uh, eps, kf):
    """f = eps / (2 E_f) u_hat on the band, E_f its energy: injects eps exactly."""
    m = forcing_mask(grid, kf)
    ef = 0.5 * float(np.sum(grid.half_weight * m * np.sum(np.abs(uh) ** 2, axis=0)))
    if ef <= 0.0:
        return np.zeros_like(uh)
    return (eps / (2.0 * ef)) * m[None] * uh


def cfl_dt(grid, uh, cfl):
    """dt = CFL / max_x sum_i |u_i| / dx_i on the dealiased physical field."""
    u = grid.backward_dealiased(uh)  # on the 3N/2 grid for the 3/2 rule
    acc = np.zeros(u.shape[1:])
    for i in range(grid.dim):
        acc += np.abs(u[i]) / (grid.lengths[i] / grid.N[i])
    s = float(acc.max())
    return cfl / s


def spectral_random_field(grid, seed, kp=4.0, energy_total=0.5):
    """Random solenoidal field with E(k) ~ k^4 exp(-2 (k/kp)^2) (NumPy generator).

    Gaussian physical-space noise is transformed (so the field is exactly
    Hermitian), Leray-projected, and each integer shell is rescaled to the
    target spectrum; the total energy is ``energy_total``.
    """
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((grid.dim,) + grid.phys_shape)
    uh = grid.forward(z)
    uh, _ = leray_projection(uh, grid.k, grid.k_over_k2)
    uh = uh * grid.mask_k0
    sidx = shell_index(grid)
    nb = int(sidx.max()) + 1
    cur = spectrum(grid, uh, nb)
    kk = np.arange(nb, dtype=np.float64)
    target = kk ** 4 * np.exp(-2.0 * (kk / kp) ** 2)
    target[0] = 0.0
    target *= energy_total / target.sum()
    scale = np.where(cur > 0, np.sqrt(target / np.where(cur > 0, cur, 1.0)), 0.0)
    return uh * scale[sidx][None]


def taylor_green(grid):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 (examples/tgv3d.py:4-11)."""
    x = grid.x
    u = np.zeros((3,) + grid.phys_shape)
    u[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    u[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    return u


# ----------------------------------------------------------------------------
# SpaceSolver + Solver loop: space_solver.py:107-310, simulation.py:161-225
# ----------------------------------------------------------------------------
class OracleSolver:
    """The reference loop restated on the Grid above.

    noise: 'philox' (device-matching counter draws, ``seed``), 'numpy'
    (reference RNG order from ``rng``) or a callable ``noise(step) -> (w1, w2)``.
    """

    def __init__(self, N, dt, is_nonlinear=True, time_integrator="rk2",
                 viscosity=1e-3, noise_type="thermal", noise_mag=0.0,
                 domain=2 * np.pi, dealias="2/3", mask_nyquist=False,
                 noise="philox", seed=0, rng=None, forcing=None, cfl=None):
        self.grid = Grid(N, domain, dealias, mask_nyquist)
        g = self.grid
        if g.dim not in (2, 3):
            raise ValueError("NS solver only supports 2D and 3D problems.")
        if noise_type not in ("thermal", "correlated"):
            raise ValueError(f"Invalid noise type '{noise_type}'. Options are 'thermal' or 'correlated'.")
        self.is_nonlinear = is_nonlinear
        self.viscosity = viscosity
        self.noise_type = noise_type
        self.noise_mag = noise_mag
        self.noise = noise
        self.seed = seed
        self.rng = rng
        self.forcing_cfg = forcing  # (eps, kf) or None
        self.cfl = cfl
        # space_solver.py:147-148
        self.linear_operator = -viscosity * g.k2
        self.correlation_func = np.zeros(g.spec_shape)
        if time_integrator not in INTEGRATORS:
            raise ValueError(f"Time integrator '{time_integrator}' not found.")
        self.integrator = INTEGRATORS[time_integrator](dt, self.linear_operator)
        self.u_hat = np.zeros((g.dim,) + g.spec_shape, dtype=np.complex128)
        self.step = 0
        self.t = 0.0
        self.dt = dt

    # simulation.py:161-180 + space_solver.py:180-225
    def initialize(self, u0, space="physical", project=True, mask_zero_mode=True):
        g = self.grid
        if space.casefold() == "physical":
            self.u_hat = g.forward(np.asarray(u0, dtype=np.float64))
        elif space.casefold() == "fourier":
            self.u_hat = np.array(u0, dtype=np.complex128)
            if mask_zero_mode:
                self.u_hat = self.u_hat * g.mask_k0
        else:
            raise ValueError("SpaceSolver.initialize_velocity: Invalid space type. "
                             "Options are 'physical' or 'fourier'.")
        if project:
            self.u_hat, _ = leray_projection(self.u_hat, g.k, g.k_over_k2)

    def set_linear_operator(self, L):
        """simulation.py:182-184."""
        self.linear_operator[...] = L
        self.integrator.update_linear_operator(L)

    def set_correlation_function(self, C):
        """simulation.py:186-187."""
        self.correlation_func = np.array(C, dtype=np.float64)

    def _noise_fields(self):
        g = self.grid
        if self.noise == "philox":
            return philox_noise_fields(g, self.noise_type, self.seed, self.step)
        if self.noise == "numpy":
            return numpy_noise_fields(g, self.noise_type, self.rng)
        return self.noise(self.step)

    def rhs_nonlinear(self, uh):
        """space_solver.py:279-300."""
        g = self.grid
        w = g.backward_dealiased(curl(g.k, uh))
        u = g.backward_dealiased(uh)
        N = g.forward_dealiased(cross(u, w))
        N, _ = leray_projection(N, g.k, g.k_over_k2)
        if g.nyquist_mask is not None:
            N = N * g.nyquist_mask
        return N

    def noise_term(self, w1, w2, a):
        """space_solver.py:240-265."""
        g = self.grid
        w = w1 + a * w2
        if self.noise_type == "thermal":
            xi = noise_divergence(symmetrize(w), g.k)
        else:
            xi = apply_linear_operator(self.correlation_func, w)
        xi, _ = leray_projection(xi, g.k, g.k_over_k2)
        return xi * self.noise_mag

    def _noise_fields_for(self, step):
        """The noise fields advance() draws for time step `step` (1-based)."""
        keep = self.step
        self.step = step
        try:
            return self._noise_fields()
        finally:
            self.step = keep

    def compute_rhs(self, a=0.0, w1=None, w2=None):
        """space_solver.py:302-310 as separate arrays: rhs_linear (:273-277),
        rhs_nonlinear (:279-300), noise and p_hat (:240-265; p_hat is the
        output of add_noise's projection, the last one compute_rhs makes) and
        forcing (new).  w1, w2 default to the next step's noise fields; with
        noise_mag == 0 no fields are drawn and noise, p_hat are zero."""
        g = self.grid
        uh = self.u_hat
        out = {"rhs_linear": apply_linear_operator(self.linear_operator, uh),
               "rhs_nonlinear": (self.rhs_nonlinear(uh) if self.is_nonlinear
                                 else np.zeros_like(uh))}
        if self.noise_mag != 0.0:
            if w1 is None:
                w1, w2 = self._noise_fields_for(self.step + 1)
            w = w1 + a * w2
            if self.noise_type == "thermal":
                xi = noise_divergence(symmetrize(w), g.k)
            else:
                xi = apply_linear_operator(self.correlation_func, w)
            xi, p = leray_projection(xi, g.k, g.k_over_k2)
            out["noise"], out["p_hat"] = xi * self.noise_mag, p
        else:
            out["noise"] = np.zeros_like(uh)
            out["p_hat"] = np.zeros(g.spec_shape, dtype=np.complex128)
        out["forcing"] = (linear_forcing(g, uh, *self.forcing_cfg)
                          if self.forcing_cfg is not None else np.zeros_like(uh))
        return out

    def advance(self, nsteps=1, diagnostics=False):
        """simulation.py:205-217 for a fixed number of steps."""
        g = self.grid
        integ = self.integrator
        hist = []
        for _ in range(nsteps):
            if self.cfl is not None:
                integ.dt = cfl_dt(g, self.u_hat, self.cfl)
                integ._lin_op_inv = 1 / (1 - integ.dt / 2 * integ._lin_op)
            self.dt = integ.dt
            self.t += integ.dt
            self.step += 1
            u0 = self.u_hat.copy()
            # noise_mag == 0 multiplies the noise by zero: counter-based draws
            # are skipped (other sources still draw, keeping the reference's
            # generator sequence)
            skip = self.noise_mag == 0.0 and self.noise == "philox"
            w1, w2 = (0.0, 0.0) if skip else self._noise_fields()
            Nl = np.zeros_like(self.u_hat)
            Lu = np.zeros_like(self.u_hat)
            for stage in range(integ.n_stages):
                a = integ.noise_factor[stage]
                Lu = apply_linear_operator(self.linear_operator, self.u_hat)
                if self.is_nonlinear:
                    Nl = self.rhs_nonlinear(self.u_hat)
                xi = (self.noise_term(w1, w2, a) if self.noise_mag != 0.0
                      else np.zeros_like(self.u_hat))
                if self.forcing_cfg is not None:
                    f = linear_forcing(g, self.u_hat, *self.forcing_cfg)
                else:
                    f = np.zeros_like(self.u_hat)
                integ.stepping(self.u_hat, u0, stage, Nl, Lu, f, xi)
            if diagnostics:
                hist.append((energy(g, self.u_hat), enstrophy(g, self.u_hat)))
        return hist
