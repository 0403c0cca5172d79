"""Generate the golden fixtures under tests/golden/ from the reference's own code.

Run in a container that has the reference checkout (it is read from
``--ref`` or the PERIODICFLOW_REF environment variable) and numba:

    python tests/golden/make_golden.py --ref <periodic-flow checkout>

What runs is the reference's code, unchanged:
  * ``periodicflow.math``            (cross, curl, apply_linear_operator,
                                      leray_projection; math.py:4-100)
  * ``periodicflow.time_integrator`` (the five integrator classes and their
                                      Numba 'optimized' and NumPy 'regular'
                                      stepping paths; time_integrator.py:7-318)
  * ``_symmetrize`` / ``_noise_divergence`` from space_solver.py:15-64, taken
    out of the module source with ``ast`` (the module itself imports shenfun
    and mpi4py, which are not installable here) and compiled with numba.

shenfun, mpi4py and h5py are absent, so the glue around those kernels is
restated here, independently of oracle/: wavenumbers (basis.py:62-77),
normal factor (space_solver.py:143-147), random_fields RNG order
(space_solver.py:227-238), compute_rhs (space_solver.py:273-310) and the solve
loop body (simulation.py:205-213), with scipy.fft standing in for shenfun's
transforms (forward normalised by 1/prod(N); 2/3 rule zeroes 3|k_i| >= N_i on a
copy of the backward input).  The fixtures are the outputs of that pipeline.
"""
from __future__ import annotations

import argparse
import ast
import json
import os
import sys
import types

import numpy as np
import scipy.fft as sfft

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import periodicflow.math as rmath  # noqa: E402
    import periodicflow.time_integrator as rti  # noqa: E402
    import numba as nb  # noqa: E402

    src_path = os.path.join(ref_root, "src", "periodicflow", "space_solver.py")
    tree = ast.parse(open(src_path).read(), filename=src_path)
    wanted = {"_symmetrize", "_noise_divergence"}
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in wanted]
    mod = ast.Module(body=body, type_ignores=[])
    ns = {"np": np, "nb": nb}
    exec(compile(mod, src_path, "exec"), ns)
    noise = types.SimpleNamespace(symmetrize=ns["_symmetrize"],
                                  noise_divergence=ns["_noise_divergence"])
    return rmath, rti, noise


# ---------------- glue restated from the shenfun-dependent modules ----------
class Box:
    def __init__(self, N, L=2 * np.pi, mask_nyquist=False):
        self.N = list(N)
        self.d = len(N)
        self.L = [L] * self.d if np.isscalar(L) else list(L)
        d = self.d
        self.spec = tuple(N[:-1]) + (N[-1] // 2 + 1,)
        ks = []
        for ax in range(d):
            kk = (np.arange(N[ax] // 2 + 1) if ax == d - 1
                  else np.fft.fftfreq(N[ax], 1.0 / N[ax])).astype(np.float64)
            shp = [1] * d
            shp[ax] = kk.size
            ks.append(kk.reshape(shp))
        self.kint = ks
        self.k = np.array([np.broadcast_to(ks[a] * 2 * np.pi / self.L[a], self.spec)
                           for a in range(d)])
        self.k2 = sum(self.k[a] ** 2 for a in range(d))
        self.k_over_k2 = np.array([self.k[a] / np.where(self.k2 == 0, 1, self.k2)
                                   for a in range(d)])
        keep = np.ones(self.spec, bool)
        for a in range(d):
            keep &= 3 * np.abs(ks[a]) < N[a]
        self.dealias = keep
        self.nyq = None
        if mask_nyquist:
            nyq = np.ones(self.spec, bool)
            for a in range(d):
                idx = np.zeros(self.spec[a], bool)
                idx[N[a] // 2] = True
                shp = [1] * d
                shp[a] = idx.size
                nyq &= ~idx.reshape(shp)
            self.nyq = nyq
        self.prodN = float(np.prod(N))
        self.x = [(self.L[a] * np.arange(N[a]) / N[a]).reshape(
            [N[a] if b == a else 1 for b in range(d)]) for a in range(d)]

    def fwd(self, u):
        return sfft.rfftn(u, axes=tuple(range(-self.d, 0))) / self.prodN

    def bwd(self, uh):
        return sfft.irfftn(uh, s=self.N, axes=tuple(range(-self.d, 0))) * self.prodN


def run_pipeline(rmath, rti, rnoise, box, integ_name, dt, nsteps, nu, nonlinear,
                 uh0, noise_type="thermal", noise_mag=0.0, noise_seed=None,
                 L=None, C=None, optimization=True):
    """compute_rhs + stepping with the reference kernels; returns states/noise."""
    d = box.d
    spec = box.spec
    lin = -nu * box.k2
    integ = rti.DICT_TIME_INTEGRATORS[integ_name](dt, lin, optimization)
    if L is not None:
        # simulation.py:182-184
        lin[...] = L
        integ.update_linear_operator(L)
    corr = np.zeros(spec) if C is None else C.astype(np.float64)
    noise_factor = getattr(integ, "noise_factor", (0.0,) * integ.n_stages)
    ncomp = d * d if noise_type == "thermal" else d
    f = np.where(box.k2 == 0, 0, 1) / np.sqrt(box.prodN) / np.sqrt(2 - 2 / d)
    rs = np.random.RandomState(noise_seed if noise_seed is not None else 0)
    u_hat = uh0.astype(np.complex128).copy()
    rhs_nl = np.zeros_like(u_hat)
    rhs_lin = np.zeros_like(u_hat)
    forcing = np.zeros_like(u_hat)
    noise = np.zeros_like(u_hat)
    p_hat = np.zeros(spec, dtype=np.complex128)
    w1s, w2s, states = [], [], []
    for _ in range(nsteps):
        u0 = u_hat.copy()
        shape = (ncomp,) + spec
        w1 = rs.randn(*shape) + 1j * rs.randn(*shape)
        w2 = rs.randn(*shape) + 1j * rs.randn(*shape)
        w1 *= f
        w2 *= f
        w1s.append(w1)
        w2s.append(w2)
        for stage in range(integ.n_stages):
            a = noise_factor[stage]
            rmath.apply_linear_operator(rhs_lin, lin, u_hat)
            if nonlinear:
                vort_hat = np.zeros((3,) + spec if d == 3 else spec, dtype=np.complex128)
                rmath.curl(vort_hat, box.k, u_hat)
                vort = box.bwd(vort_hat * box.dealias)
                u = box.bwd(u_hat * box.dealias)
                uw = np.zeros_like(u)
                rmath.cross(uw, u, vort)
                rhs_nl[...] = box.fwd(uw)
                rmath.leray_projection(rhs_nl, box.k, box.k_over_k2, p_hat)
                if box.nyq is not None:
                    rhs_nl *= box.nyq
            w_hat = w1 + a * w2
            if noise_type == "thermal":
                w_sym = np.zeros_like(w_hat)
                rnoise.symmetrize(w_sym, w_hat)
                rnoise.noise_divergence(noise, w_sym, box.k)
            else:
                rmath.apply_linear_operator(noise, corr, w_hat)
            rmath.leray_projection(noise, box.k, box.k_over_k2, p_hat)
            noise *= noise_mag
            integ.stepping(u_hat, u0, stage, rhs_nl, rhs_lin, forcing, noise)
        states.append(u_hat.copy())
    return dict(states=np.array(states), w1=np.array(w1s), w2=np.array(w2s))


def random_solenoidal(box, seed, amp=1.0):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((box.d,) + tuple(box.N))
    uh = box.fwd(u)
    p = np.sum(box.k_over_k2 * uh, axis=0)
    uh = (uh - p * box.k) * np.where(box.k2 == 0, 0, 1)
    # damp high modes so nonlinear runs stay smooth
    return amp * uh * np.exp(-box.k2 / (0.25 * max(box.N)) ** 2)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PERIODICFLOW_REF"),
                    required="PERIODICFLOW_REF" not in os.environ,
                    help="root of a periodic-flow checkout (or set PERIODICFLOW_REF)")
    args = ap.parse_args()
    rmath, rti, rnoise = load_reference(args.ref)
    rng = np.random.default_rng(20240601)
    out = {}

    # ---- 1. pointwise kernel known answers on random data ------------------
    for d, N in ((2, (8, 8)), (3, (8, 8, 8))):
        box = Box(N)
        spec = box.spec
        uh = rng.standard_normal((d,) + spec) + 1j * rng.standard_normal((d,) + spec)
        c = np.zeros((3,) + spec if d == 3 else spec, dtype=np.complex128)
        rmath.curl(c, box.k, uh)
        out[f"k{d}_uh"] = uh
        out[f"k{d}_curl"] = c
        u = rng.standard_normal((d,) + tuple(N))
        w = rng.standard_normal((3,) + tuple(N) if d == 3 else tuple(N))
        cr = np.zeros_like(u)
        rmath.cross(cr, u, w)
        out[f"k{d}_u"], out[f"k{d}_w"], out[f"k{d}_cross"] = u, w, cr
        Lop = rng.standard_normal(spec)
        Lu = np.zeros_like(uh)
        rmath.apply_linear_operator(Lu, Lop, uh)
        out[f"k{d}_L"], out[f"k{d}_Lu"] = Lop, Lu
        up = uh.copy()
        p = np.zeros(spec, dtype=np.complex128)
        rmath.leray_projection(up, box.k, box.k_over_k2, p)
        out[f"k{d}_leray_u"], out[f"k{d}_leray_p"] = up, p
        W = rng.standard_normal((d * d,) + spec) + 1j * rng.standard_normal((d * d,) + spec)
        Ws = np.zeros_like(W)
        rnoise.symmetrize(Ws, W)
        div = np.zeros((d,) + spec, dtype=np.complex128)
        rnoise.noise_divergence(div, Ws, box.k)
        out[f"k{d}_W"], out[f"k{d}_Wsym"], out[f"k{d}_noisediv"] = W, Ws, div

    # ---- 2. every integrator, every stage, both code paths -----------------
    for d, N in ((2, (8, 8)), (3, (4, 4, 4))):
        box = Box(N)
        spec = box.spec
        shp = (d,) + spec
        cz = lambda: rng.standard_normal(shp) + 1j * rng.standard_normal(shp)  # noqa: E731
        Lop = -0.3 * box.k2
        for name in ("explicit_pc", "implicit_pc", "rk2", "rk3", "rk4"):
            for opt in (False, True):
                integ = rti.DICT_TIME_INTEGRATORS[name](0.01, Lop.copy(), opt)
                for stage in range(integ.n_stages):
                    unew, u0, Nl, Lu, fo, xi = cz(), cz(), cz(), cz(), cz(), cz()
                    key = f"st{d}_{name}_{int(opt)}_{stage}"
                    out[key + "_in"] = np.stack([unew, u0, Nl, Lu, fo, xi])
                    integ.stepping(unew, u0, stage, Nl, Lu, fo, xi)
                    out[key + "_out"] = unew
                    out[key + "_Lu"] = Lu
        out[f"st{d}_L"] = Lop

    # ---- 3. pipelines: reference kernels + restated glue -------------------
    cases = []
    box = Box((16, 16, 16))
    u_tg = np.zeros((3, 16, 16, 16))
    x = box.x
    u_tg[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    u_tg[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    cases.append(("tgv16_rk4", box, dict(integ_name="rk4", dt=0.005, nsteps=4, nu=1 / 1600,
                                          nonlinear=True, uh0=box.fwd(u_tg))))
    cases.append(("rand16_rk3", box, dict(integ_name="rk3", dt=0.01, nsteps=3, nu=2e-3,
                                           nonlinear=True, uh0=random_solenoidal(box, 1, 4.0))))
    cases.append(("rand16_ipc", box, dict(integ_name="implicit_pc", dt=0.01, nsteps=2,
                                           nu=0.01, nonlinear=True,
                                           uh0=random_solenoidal(box, 2, 4.0))))
    boxa = Box((16, 8, 32), L=[2 * np.pi, np.pi, 4 * np.pi])
    cases.append(("aniso_rk2", boxa, dict(integ_name="rk2", dt=0.005, nsteps=2, nu=0.01,
                                          nonlinear=True, uh0=random_solenoidal(boxa, 3, 4.0))))
    box2 = Box((32, 32))
    cases.append(("twod32_epc", box2, dict(integ_name="explicit_pc", dt=0.01, nsteps=3,
                                            nu=0.01, nonlinear=True,
                                            uh0=random_solenoidal(box2, 4, 8.0))))
    cases.append(("twod32_rk3_noise", box2, dict(integ_name="rk3", dt=0.01, nsteps=3,
                                                  nu=0.01, nonlinear=True,
                                                  uh0=random_solenoidal(box2, 5, 8.0),
                                                  noise_mag=0.05, noise_seed=11)))
    boxn = Box((32, 32), mask_nyquist=True)
    cases.append(("twod32_nyq_rk4", boxn, dict(integ_name="rk4", dt=0.01, nsteps=2, nu=0.01,
                                                nonlinear=True,
                                                uh0=random_solenoidal(boxn, 6, 8.0))))
    box2s = Box((16, 16))
    kBT, nu = 1e-3, 0.1
    for name in ("explicit_pc", "implicit_pc", "rk3"):
        cases.append((f"stokes2d_thermal_{name}", box2s, dict(
            integ_name=name, dt=0.01, nsteps=4, nu=nu, nonlinear=False,
            uh0=np.zeros((2,) + box2s.spec), noise_type="thermal",
            noise_mag=np.sqrt(2 * nu * kBT), noise_seed=7)))
    box3s = Box((8, 8, 8))
    cases.append(("stokes3d_thermal_ipc", box3s, dict(
        integ_name="implicit_pc", dt=0.02, nsteps=3, nu=nu, nonlinear=False,
        uh0=random_solenoidal(box3s, 8, 0.1), noise_type="thermal",
        noise_mag=np.sqrt(2 * nu * kBT), noise_seed=8)))
    # correlated noise as in examples/fluctuating_stokes_correlated_noise.py:33-50,86-90
    l = 0.3
    dx = box2s.x[0][1, 0] - box2s.x[0][0, 0]
    kx, ky = box2s.k
    Cl = np.exp(-0.5 * ((l * kx) ** 2 + (l * ky) ** 2)) * (np.sqrt(2 * np.pi * l ** 2) / dx) ** 2
    Cl = Cl * np.where(box2s.k2 == 0, 0, 1)
    cases.append(("stokes2d_corr_ipc", box2s, dict(
        integ_name="implicit_pc", dt=0.01, nsteps=4, nu=nu, nonlinear=False,
        uh0=random_solenoidal(box2s, 9, 0.1), noise_type="correlated",
        noise_mag=np.sqrt(2 * nu * kBT), noise_seed=9, L=-nu * Cl, C=np.sqrt(Cl))))

    meta = []
    for name, bx, kw in cases:
        res = run_pipeline(rmath, rti, rnoise, bx, **kw)
        pre = f"p_{name}_"
        out[pre + "uh0"] = kw["uh0"].astype(np.complex128)
        out[pre + "states"] = res["states"]
        if kw.get("noise_mag", 0.0) != 0.0:
            out[pre + "w1"] = res["w1"]
            out[pre + "w2"] = res["w2"]
        if kw.get("L") is not None:
            out[pre + "L"] = kw["L"]
        if kw.get("C") is not None:
            out[pre + "C"] = kw["C"]
        meta.append(dict(name=name, N=list(bx.N), L=list(bx.L),
                         mask_nyquist=bx.nyq is not None,
                         **{k: v for k, v in kw.items()
                            if k not in ("uh0", "L", "C", "noise_seed")},
                         has_L=kw.get("L") is not None, has_C=kw.get("C") is not None))
    out["pipeline_meta"] = np.array(json.dumps(meta, default=float))
    path = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
