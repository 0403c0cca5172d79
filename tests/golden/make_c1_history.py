"""Generate tests/golden/tgv64_fp64_rk4_400.npz: the Taylor-Green benchmark
configuration run for its full length through the reference's own kernels.

Configuration: 64^3 grid on [0, 2 pi)^3, FP64, u = sin x cos y cos z,
v = -cos x sin y cos z, w = 0, nu = 1/1600, 2/3 rule, rk4, dt = 0.005,
400 steps; stored are the kinetic energy and enstrophy after every step
(E = 1/2 sum |u_hat|^2, Z = 1/2 sum |k|^2 |u_hat|^2 over the full spectrum,
half-spectrum planes k_z = 0 and Nyquist counted once) and the final state's
modes with |k_x|, |k_y| <= 3 and k_z <= 3.

What runs is the reference's periodicflow.math (curl, cross,
leray_projection, apply_linear_operator) and periodicflow.time_integrator
(RK4, Numba path), unchanged, with the glue of make_golden.py (scipy.fft in
place of shenfun).  Needs the reference checkout and numba:

    python tests/golden/make_c1_history.py --ref <periodic-flow checkout>
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import Box, load_reference  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PERIODICFLOW_REF"),
                    required="PERIODICFLOW_REF" not in os.environ,
                    help="root of a periodic-flow checkout (or set PERIODICFLOW_REF)")
    ap.add_argument("--steps", type=int, default=400)
    args = ap.parse_args()
    rmath, rti, _ = load_reference(args.ref)
    n, nu, dt = 64, 1 / 1600, 0.005
    box = Box((n, n, n))
    x = box.x
    u = np.zeros((3, n, n, n))
    u[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    u[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    u_hat = box.fwd(u)
    spec = box.spec
    lin = -nu * box.k2
    integ = rti.DICT_TIME_INTEGRATORS["rk4"](dt, lin, True)
    w = np.full(spec[-1], 2.0)
    w[0] = 1.0
    w[-1] = 1.0
    rhs_nl = np.zeros_like(u_hat)
    rhs_lin = np.zeros_like(u_hat)
    zero = np.zeros_like(u_hat)
    p_hat = np.zeros(spec, dtype=np.complex128)
    hist = []
    for _ in range(args.steps):
        u0 = u_hat.copy()
        for stage in range(integ.n_stages):
            rmath.apply_linear_operator(rhs_lin, lin, u_hat)
            vort_hat = np.zeros((3,) + spec, dtype=np.complex128)
            rmath.curl(vort_hat, box.k, u_hat)
            vort = box.bwd(vort_hat * box.dealias)
            uu = box.bwd(u_hat * box.dealias)
            uw = np.zeros_like(uu)
            rmath.cross(uw, uu, vort)
            rhs_nl[...] = box.fwd(uw)
            rmath.leray_projection(rhs_nl, box.k, box.k_over_k2, p_hat)
            integ.stepping(u_hat, u0, stage, rhs_nl, rhs_lin, zero, zero)
        e = np.sum(np.abs(u_hat) ** 2, axis=0)
        hist.append((0.5 * np.sum(w * e), 0.5 * np.sum(w * box.k2 * e)))
    idx = np.r_[0:4, n - 3:n]
    low = u_hat[:, idx][:, :, idx][..., 0:4]
    np.savez_compressed(os.path.join(HERE, "tgv64_fp64_rk4_400.npz"), energy_enstrophy=np.array(hist),
                        final_low_modes=low, meta=np.array([n, nu, dt, args.steps]))
    print("E, Z at the end:", hist[-1])


if __name__ == "__main__":
    main()
