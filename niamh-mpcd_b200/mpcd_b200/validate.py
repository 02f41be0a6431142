"""Transport validation: kinematic viscosity of an SRD fluid from the decay
of transverse momentum modes.

A transverse momentum mode of the smallest wavevector of a periodic box,
j_a(k e_b) = sum_i v_i,a exp(-i k x_i,b) with a != b and k = 2 pi / L,
decays as exp(-nu k^2 t) (nu = eta / rho, the kinematic viscosity).  The
normalised autocorrelation C(t) = Re<j(t0 + t) j*(t0)> / <|j(t0)|^2>,
averaged over the six (a, b) pairs and all time origins, is fitted to
exp(-nu k^2 t) over the lags where C > c_min.  The reference program has no
such analysis tool; `theory_nu_srd3d` gives the analytic values it is
compared with (Gompper, Ihle, Kroll and Winkler, Adv. Polym. Sci. 221
(2009), random-axis SRD in 3D: kinetic and collisional parts).

    python -m mpcd_b200.validate --L 32 --steps 40000 --every 10 --form mixed
"""
import argparse
import json
import math

import numpy as np

from . import abi
from . import workloads as W
from .gpu import Solver


def theory_nu_srd3d(n, alpha, dt, kbt=1.0, m=1.0, a=1.0):
    """Kinetic and collisional kinematic viscosity of 3D random-axis SRD."""
    en = n - 1.0 + math.exp(-n)
    kin = kbt * dt / (2.0 * m) * (5.0 * n / (en * (2.0 - math.cos(alpha) - math.cos(2 * alpha))) - 1.0)
    col = a * a / (18.0 * dt) * en / n * (1.0 - math.cos(alpha))
    return kin, col


def transverse_modes(Q, V, L):
    """The six transverse modes j_a(k e_b), k = 2 pi / L_b, as complex numbers
    (host restatement of mpcd_transverse_modes, same pair order)."""
    out = []
    for b in range(3):
        ph = np.exp(-2j * np.pi * Q[:, b] / L[b])
        for a in range(3):
            if a != b:
                out.append(np.dot(V[:, a], ph))
    return np.array(out)


def measure_viscosity(L=32, ppc=10, steps=40000, every=10, precision=abi.PREC_MIXED,
                      seed=11, c_min=0.25, max_lag=None):
    cfg = W.cfg_srd3d((L, L, L), precision=precision, seed=seed)
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=seed + 1)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    g.step(200, 1)  # forget the initial state
    samples = []
    step = 201
    for _ in range(steps // every):
        g.step(every, step)
        step += every
        samples.append(g.transverse_modes())
    g.close()
    J = np.array(samples)  # (T, 6)
    T = len(J)
    nlag = max_lag or min(T // 4, 400)
    norm = np.mean(np.abs(J) ** 2)
    C = np.array([np.mean((J[lag:] * np.conj(J[:T - lag])).real) / norm for lag in range(nlag)])
    t = np.arange(nlag) * every * cfg.dt
    k2 = (2 * np.pi / L) ** 2
    below = np.nonzero(C[1:] <= c_min)[0]
    last = int(below[0]) + 1 if len(below) else nlag
    use = np.arange(1, max(last, 3))  # lags before C first drops to c_min
    slope, _ = np.polyfit(t[use], np.log(C[use]), 1)
    nu = -slope / k2
    # error from the scatter of independent blocks of the run
    nblk = 8
    nus = []
    for blk in np.array_split(np.arange(T), nblk):
        Jb = J[blk]
        Tb = len(Jb)
        nb = np.mean(np.abs(Jb) ** 2)
        Cb = np.array([np.mean((Jb[lag:] * np.conj(Jb[:Tb - lag])).real) / nb
                       for lag in range(max(use) + 1)])
        ok = Cb[use] > 0
        if ok.sum() >= 2:
            s, _ = np.polyfit(t[use][ok], np.log(Cb[use][ok]), 1)
            nus.append(-s / k2)
    err = float(np.std(nus) / math.sqrt(len(nus))) if len(nus) > 1 else float("nan")
    return {"nu": float(nu), "nu_err": err, "lags_fitted": int(len(use)),
            "samples": T, "L": L, "steps": steps, "every": every,
            "precision": "fp64" if precision == abi.PREC_FP64 else "mixed"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--form", default="mixed", choices=["mixed", "fp64"])
    args = ap.parse_args()
    prec = abi.PREC_MIXED if args.form == "mixed" else abi.PREC_FP64
    res = measure_viscosity(L=args.L, steps=args.steps, every=args.every, precision=prec)
    kin, col = theory_nu_srd3d(10.0, math.radians(130.0), 0.1)
    res["theory_kinetic"] = kin
    res["theory_collisional"] = col
    res["theory_total"] = kin + col
    print(json.dumps(res))


if __name__ == "__main__":
    main()
