"""Transport validation: kinematic viscosity (1) of an SRD fluid from the
decay of transverse momentum modes, (2) of a walled channel from the
curvature of its steady Poiseuille profile.

A transverse momentum mode of the smallest wavevector of a periodic box,
j_a(k e_b) = sum_i v_i,a exp(-i k x_i,b) with a != b and k = 2 pi / L,
decays as exp(-nu k^2 t) (nu = eta / rho, the kinematic viscosity).  The
normalised autocorrelation C(t) = Re<j(t0 + t) j*(t0)> / <|j(t0)|^2>,
averaged over the six (a, b) pairs and all time origins, is fitted to
exp(-nu k^2 t) over the lags where C > c_min.  The reference program has no
such analysis tool; `theory_nu_srd3d` gives the analytic values it is
compared with (Gompper, Ihle, Kroll and Winkler, Adv. Polym. Sci. 221
(2009), random-axis SRD in 3D: kinetic and collisional parts).

A channel between two no-slip walls at y = 0 and y = H, driven by the body
force g along x, reaches the profile v_x(y) = g y (H - y) / (2 nu); the
fit of a parabola to the time-averaged, mass-weighted layer velocities gives
nu = -g / (2 c2) from its curvature c2 alone (a slip length moves the
parabola, not its curvature).  `theory_nu_reference` restates the analytic
kinematic viscosity the reference prints to synopsis.dat (theory_trans,
init.c:800-942; Noguchi and Gompper, PRE 78, 016706 (2008)).

    python -m mpcd_b200.validate --L 32 --steps 40000 --every 10 --form mixed
    python -m mpcd_b200.validate --channel --form fp64
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


def theory_nu_reference(coll_op, dim, n, rot_ang=math.pi / 2, dt=0.1, kbt=1.0, m=1.0):
    """Kinematic viscosity (kinetic, collisional) of theory_trans
    (init.c:800-942) for one species of mass m at number density n, a = 1:
    the correlation factors A, B of the operator (ARBAXIS, MPC-AT, MPC-AT+a),
    then the kinetic and collisional dynamic viscosities divided by n m.

    The factor M = n / (n - 1 + e^-n) of the operators without angular
    momentum conservation is computed there with smrtPow(e, -n)
    (mtools.c:38-50), whose integer-exponent branch multiplies x by itself
    "y times" in a loop that does not run for a negative y, so it returns 1
    for every integer density: M = 1 whenever n is a whole number.  That is
    what the reference prints (synopsis.dat) and what this restatement
    returns; theory_nu_srd3d gives the textbook value."""
    en = math.exp(-n)
    # smrtPow(e, -n): 1 for an integer n (see above), e^-n otherwise
    en_pow = 1.0 if float(n).is_integer() else en
    Mf = n / (n - 1.0 + en_pow)
    if coll_op == abi.COLL_ARBAXIS:
        A = 2.0 / dim * (1.0 - math.sin(rot_ang) / rot_ang)
        if dim == 2:
            B = 1.0 - 0.5 * math.sin(2.0 * rot_ang) / rot_ang
        else:
            B = 0.4 * (2.0 - 1.5 * math.sin(rot_ang) / rot_ang)
    elif coll_op in (abi.COLL_MPCAT, abi.COLL_RAT):
        A = B = 1.0
    else:
        raise ValueError("no analytic viscosity for this operator")
    if coll_op == abi.COLL_RAT:
        cm = B * (1.0 - en * (1.0 + n)) + (A + B / dim) * n * en / (dim + 2.0)
        cm += 0.5 * (A * dim - 0.5 * B * (3.0 * dim + 2.0)) * \
            (1.0 - en * (1.0 + n + 0.5 * n * n)) / n
        col = A * m / (24.0 * dt) * (n - 1.4 + en * (1.4 + 0.4 * n + (1.0 / dim - 0.3) * n * n))
    else:
        cm = B / Mf
        col = A * n / Mf * m / (12.0 * dt)
    kin = n * kbt * dt * (1.0 / cm - 0.5)
    return kin / (n * m), col / (n * m)


def channel_viscosity(L=(32, 32, 16), ppc=20, g=5e-4, warm=12000, steps=24000, every=10,
                      precision=abi.PREC_MIXED, seed=21, edge=2, nblk=8, start="rest"):
    """Kinematic viscosity from the steady profile of the MPC-AT+a channel
    (phantom no-slip walls at y = 0 and y = L1, periodic x and z, body force
    g along x): mass-weighted x velocity per y layer, averaged over time,
    fitted by a parabola over the layers at least `edge` cells from a wall.
    start="parabola" starts the flow from the steady profile of the analytic
    viscosity (theory_trans) instead of rest, so that a run much shorter than
    the channel's momentum diffusion time H^2 / (pi^2 nu) samples the steady
    state."""
    cfg = W.cfg_channel3d(tuple(L), g=g, precision=precision, seed=seed)
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=seed + 1)
    Q[:, 1] = 0.02 + Q[:, 1] * (L[1] - 0.04) / L[1]  # off the walls' planes
    if start == "parabola":
        kin, col = theory_nu_reference(abi.COLL_RAT, 3, float(ppc))
        H = float(L[1])
        V[:, 0] += g * Q[:, 1] * (H - Q[:, 1]) / (2.0 * (kin + col))
    s = Solver(cfg)
    s.upload(Q, V, U, sp)
    s.step(warm, 1)
    step = warm + 1
    H = int(L[1])
    mv, mm = [], []
    for _ in range(steps // every):
        s.step(every, step)
        step += every
        _, mass, vcm, _ = s.cell_props()
        mv.append((mass * vcm[..., 0])[:L[0], :H, :L[2]].sum(axis=(0, 2)))
        mm.append(mass[:L[0], :H, :L[2]].sum(axis=(0, 2)))
    s.close()
    res = fit_channel(np.array(mv), np.array(mm), g, edge=edge, nblk=nblk)
    res.update(L=list(L), g=g, warm=warm, steps=steps, every=every,
               precision="fp64" if precision == abi.PREC_FP64 else "mixed")
    return res


def fit_channel(mv, mm, g, edge=2, nblk=8):
    """nu from per-sample layer sums mv[t, y] (mass times x velocity) and
    mm[t, y] (mass): the time-averaged profile v = sum mv / sum mm is fitted
    by c0 + c1 y + c2 y^2 at the layer centres y + 1/2 at least `edge` layers
    from a wall, nu = -g / (2 c2); the error is the scatter of the fits of
    nblk consecutive blocks of samples."""
    H = mv.shape[1]
    y = np.arange(H) + 0.5
    use = slice(edge, H - edge)

    def fit(a, b):
        v = a.sum(axis=0) / b.sum(axis=0)
        c2, c1, c0 = np.polyfit(y[use], v[use], 2)
        return -g / (2.0 * c2), v, np.array([c2, c1, c0])

    nu, v, coef = fit(mv, mm)
    nus = [fit(a, b)[0] for a, b in zip(np.array_split(mv, nblk), np.array_split(mm, nblk))]
    err = float(np.std(nus) / math.sqrt(len(nus)))
    resid = v[use] - np.polyval(coef, y[use])
    return {"nu": float(nu), "nu_err": err, "v_max": float(v.max()),
            "fit_rms": float(np.sqrt(np.mean(resid ** 2))), "profile": v.tolist()}


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


def fit_decay(t, s, noise, snr_min=10.0):
    """Decay rate of a signal s(t) = s0 exp(-rate t) + noise: a straight line
    through ln s over the samples (from the first) where s is still above
    snr_min times the noise; returns the rate and the number of samples
    used."""
    ok = s > snr_min * noise
    last = int(np.argmin(ok)) if not ok.all() else len(s)
    use = np.arange(max(last, 3))
    slope, _ = np.polyfit(t[use], np.log(np.abs(s[use])), 1)
    return -slope, len(use)


def shear_wave_viscosity(L=64, ppc=10, amp=0.1, nrep=16, steps=2400, every=20,
                         precisions=(abi.PREC_FP64, abi.PREC_MIXED), seed=100):
    """Kinematic viscosity of the 3D SRD fluid (130 degrees, dt 0.1) from the
    decay of an imposed transverse shear wave: v_x += amp sin(k y), k =
    2 pi / L, on the thermal state, whose mode j = sum v_x exp(-i k y)
    (mpcd_transverse_modes, pair a = x, b = y) relaxes as exp(-nu k^2 t) --
    the decay of a transverse momentum fluctuation that the autocorrelation
    C(k, t) measures, driven far above the thermal noise.  nrep replicas
    (independent states and draws), each stepped in every given form from the
    same state with the same draws, so that the forms' difference is paired.
    Returns per form the mean nu and its standard error, and the paired
    differences to the first form."""
    k = 2.0 * math.pi / L
    nus = {p: [] for p in precisions}
    for r in range(nrep):
        for p in precisions:
            cfg = W.cfg_srd3d((L, L, L), precision=p, seed=seed + 7 * r)
            Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=seed + 7 * r + 1)
            V[:, 0] += amp * np.sin(k * Q[:, 1])
            V[:, 0] -= V[:, 0].mean()
            n = len(Q)
            noise = math.sqrt(n * cfg.kbt / 2.0)
            g = Solver(cfg)
            g.upload(Q, V, U, sp)
            sig = [-g.transverse_modes()[2].imag]
            for s in range(0, steps, every):
                g.step(every, 1 + s)
                sig.append(-g.transverse_modes()[2].imag)
            g.close()
            t = np.arange(len(sig)) * every * cfg.dt
            rate, _ = fit_decay(t, np.array(sig), noise)
            nus[p].append(rate / (k * k))
    out = {"L": L, "ppc": ppc, "amp": amp, "replicas": nrep, "steps": steps, "every": every}
    base = np.array(nus[precisions[0]])
    for p in precisions:
        a = np.array(nus[p])
        name = "fp64" if p == abi.PREC_FP64 else "mixed"
        out[name] = {"nu": float(a.mean()), "nu_err": float(a.std(ddof=1) / math.sqrt(len(a)))}
        if p != precisions[0]:
            d = a / base - 1.0
            out[name]["rel_diff_to_" + ("fp64" if precisions[0] == abi.PREC_FP64 else "mixed")] = \
                {"mean": float(d.mean()), "err": float(d.std(ddof=1) / math.sqrt(len(d)))}
    kin, col = theory_nu_srd3d(ppc, math.radians(130.0), 0.1)
    out["theory_textbook"] = kin + col
    rk, rc = theory_nu_reference(abi.COLL_ARBAXIS, 3, float(ppc), math.radians(130.0), 0.1)
    out["theory_reference_synopsis"] = rk + rc
    return out


def main():
    """Command line of the transport checks:
      --shear                 64^3 SRD viscosity from the shear-wave decay,
                              FP64 and mixed paired (--reps, --amp)
      --channel [--full]      MPC-AT+a channel viscosity from the steady
                              profile (--full: configuration 3, 128x64x64,
                              g = 1e-4, started from the parabola)
      (neither)               SRD viscosity from the transverse-momentum
                              autocorrelation of an equilibrium run."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--form", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--channel", action="store_true",
                    help="Poiseuille channel (MPC-AT+a, phantom walls) instead of SRD modes")
    ap.add_argument("--full", action="store_true",
                    help="channel of configuration 3: 128x64x64, g = 1e-4, parabola start")
    ap.add_argument("--shear", action="store_true",
                    help="64^3 SRD viscosity from the decay of an imposed shear wave")
    ap.add_argument("--reps", type=int, default=32)
    ap.add_argument("--amp", type=float, default=0.25)
    ap.add_argument("--warm", type=int, default=12000)
    args = ap.parse_args()
    prec = abi.PREC_MIXED if args.form == "mixed" else abi.PREC_FP64
    if args.shear:
        print(json.dumps(shear_wave_viscosity(L=64, nrep=args.reps, amp=args.amp)))
        return
    if args.channel:
        if args.full:
            res = channel_viscosity(L=(128, 64, 64), ppc=20, g=1e-4, warm=20000, steps=40000,
                                    every=200, precision=prec, edge=3, start="parabola")
        else:
            res = channel_viscosity(warm=args.warm,
                                    steps=args.steps if args.steps != 40000 else 24000,
                                    every=args.every, precision=prec)
        kin, col = theory_nu_reference(abi.COLL_RAT, 3, 20.0)
        res.update(theory_kinetic=kin, theory_collisional=col, theory_total=kin + col)
        res.pop("profile")
        print(json.dumps(res))
        return
    res = measure_viscosity(L=args.L, steps=args.steps, every=args.every, precision=prec)
    kin, col = theory_nu_srd3d(10.0, math.radians(130.0), 0.1)
    res["theory_kinetic"] = kin
    res["theory_collisional"] = col
    res["theory_total"] = kin + col
    print(json.dumps(res))


if __name__ == "__main__":
    main()
