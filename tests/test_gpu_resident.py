"""The resident SRD kernel family (mixed precision, particles kept in place,
cell sums accumulated in 64-bit fixed point) against the CPU oracle and
against the sorted kernel family of the same precision.

Fixed-point sums are exact and order-independent, so the resident family's
results must not depend on the particle order in memory: runs that re-sort
the state at different intervals agree bit for bit.
"""
import math

import numpy as np
import pytest

from checkers import Oracle
from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu


def _solid_channel(L):
    """Periodic in x and z, bounce-back walls at y=0 and y=L[1] without
    phantom particles (so the SRD operator stays on the resident path)."""
    w = W.channel_walls(L)
    for i in (2, 3):
        w[i].phantom = 0
    return w


def _case(name, precision):
    if name == "srd3d":
        return W.cfg_srd3d((9, 7, 6), precision=precision, seed=101), 10
    if name == "srd2d":
        return W.base_config(2, (11, 9), coll_op=abi.COLL_ARBAXIS, rot_ang=math.radians(130.0),
                             precision=precision, seed=102), 12
    if name == "heavy":
        return W.cfg_srd3d((6, 6, 6), species=[W._species(mass=2.5)], kbt=1.7, dt=0.25,
                           precision=precision, seed=103), 10
    if name == "species":
        return W.cfg_srd3d((7, 6, 5), species=[W._species(mass=1.0), W._species(mass=3.0)],
                           precision=precision, seed=104), 10
    if name == "walls_grav":
        L = (8, 6, 5)
        return W.base_config(3, L, coll_op=abi.COLL_ARBAXIS, rot_ang=math.radians(130.0),
                             walls=_solid_channel(L), grav=(1e-2, 0.0, 0.0),
                             precision=precision, seed=105), 15
    raise KeyError(name)


def _state(cfg, ppc, seed):
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=seed)
    if cfg.n_species > 1:
        sp = (np.arange(len(Q)) % cfg.n_species).astype(np.int32)
    if any(cfg.walls[i].phantom == 0 and cfg.walls[i].DN == 0.0 for i in range(cfg.n_walls)):
        # keep particles off the walls' planes
        Q[:, 1] = 0.02 + Q[:, 1] * (cfg.L[1] - 0.04) / cfg.L[1]
    return Q, V, U, sp


NAMES = ["srd3d", "srd2d", "heavy", "species", "walls_grav"]


def _min_image(d, L):
    return d - np.round(d / L) * L


@pytest.mark.parametrize("name", NAMES)
def test_resident_tracks_oracle_one_step(name):
    cfg, ppc = _case(name, abi.PREC_FP64)
    cfgm, _ = _case(name, abi.PREC_MIXED)
    Q, V, U, sp = _state(cfg, ppc, 7)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgm)
    g.set_kernel(abi.KERNEL_RESIDENT)
    g.upload(Q, V, U, sp)
    o.step(1)
    kg, ag = g.timestep(1)
    assert g.launches_per_step() >= 2
    qo, vo, _ = o.particles()
    qg, vg, _ = g.download()
    L = np.array([cfg.L[d] if d < cfg.dim else 1 for d in range(3)], dtype=float)
    dv = np.abs(vg - vo).max(axis=1)
    dq = np.abs(_min_image(qg - qo, L)).max(axis=1)
    bad = np.mean((dv > 1e-5) | (dq > 1e-5))
    assert bad < 2e-3, (bad, dv.max(), dq.max())
    ko, ao = o.globals()
    assert kg == pytest.approx(ko, rel=1e-5)
    np.testing.assert_allclose(ag, ao, rtol=0, atol=1e-6)
    st = g.status()
    assert st.escaped == 0 and st.bounce_limit == 0 and st.nonfinite == 0
    assert st.sync_timeout == 0


@pytest.mark.parametrize("name", NAMES)
def test_resident_matches_sorted_family_multistep(name):
    # same precision, same draws: the resident and the sorted (split) family
    # differ only in how the FP64 cell sums are formed (~1e-10), so they
    # agree to FP32 precision over many steps
    cfgm, ppc = _case(name, abi.PREC_MIXED)
    Q, V, U, sp = _state(cfgm, ppc, 8)
    out = []
    for kernel in (abi.KERNEL_RESIDENT, abi.KERNEL_SPLIT):
        g = Solver(cfgm)
        g.set_kernel(kernel)
        g.upload(Q, V, U, sp)
        glob = [g.timestep(s) for s in range(1, 11)]
        out.append((g.download(), glob))
    (qa, va, _), ga = out[0]
    (qb, vb, _), gb = out[1]
    L = np.array([cfgm.L[d] if d < cfgm.dim else 1 for d in range(3)], dtype=float)
    dv = np.abs(va - vb).max(axis=1)
    dq = np.abs(_min_image(qa - qb, L)).max(axis=1)
    bad = np.mean((dv > 1e-4) | (dq > 1e-5))
    assert bad < 5e-3, (bad, dv.max(), dq.max())
    for (ka, aa), (kb, ab) in zip(ga, gb):
        assert ka == pytest.approx(kb, rel=1e-5)


@pytest.mark.parametrize("name", ["srd3d", "species", "walls_grav"])
def test_resident_result_independent_of_sort_interval(name):
    cfgm, ppc = _case(name, abi.PREC_MIXED)
    Q, V, U, sp = _state(cfgm, ppc, 9)
    res = []
    for interval in (1, 3, 1000):
        g = Solver(cfgm)
        g.set_kernel(abi.KERNEL_RESIDENT)
        g.set_sort_interval(interval)
        g.upload(Q, V, U, sp)
        g.step(12, 1)
        q, v, _ = g.download()
        res.append((q, v, g.globals()))
    for q, v, gl in res[1:]:
        assert np.array_equal(q, res[0][0])
        assert np.array_equal(v, res[0][1])
        # the global measures are floating-point reductions whose order
        # follows the particle order: equal to rounding only
        assert gl[0] == pytest.approx(res[0][2][0], rel=1e-7)


def test_resident_switching_families_mid_run():
    # resident -> split -> resident must continue the same trajectory as a
    # run that stays on one family (to FP32 precision)
    cfgm, ppc = _case("srd3d", abi.PREC_MIXED)
    Q, V, U, sp = _state(cfgm, ppc, 10)
    a = Solver(cfgm)
    a.set_kernel(abi.KERNEL_SPLIT)
    a.upload(Q, V, U, sp)
    a.step(9, 1)
    b = Solver(cfgm)
    b.upload(Q, V, U, sp)
    for s0, kern in ((1, abi.KERNEL_RESIDENT), (4, abi.KERNEL_SPLIT), (7, abi.KERNEL_RESIDENT)):
        b.set_kernel(kern)
        b.step(3, s0)
    qa, va, _ = a.download()
    qb, vb, _ = b.download()
    dv = np.abs(va - vb).max(axis=1)
    assert np.mean(dv > 1e-4) < 5e-3, dv.max()


def test_resident_conserves_momentum_exactly_in_fixed_point():
    # SRD conserves each cell's momentum; with exact fixed-point sums the
    # total drifts only by the FP32 rounding of the rotated velocities
    cfgm = W.cfg_srd3d((16, 16, 16), precision=abi.PREC_MIXED, seed=11)
    Q, V, U, sp = W.synthetic_state(cfgm, 10, seed=12)
    g = Solver(cfgm)
    g.upload(Q, V, U, sp)
    p0 = V.sum(axis=0)
    g.step(50, 1)
    _, v, _ = g.download()
    assert np.abs(v.sum(axis=0) - p0).max() / np.abs(V).sum() < 1e-6


def _cell_momenta(Q, V, L):
    idx = np.floor(Q[:, :3]).astype(np.int64)
    lin = (idx[:, 0] * L[1] + idx[:, 1]) * L[2] + idx[:, 2]
    n = int(np.prod(L))
    p = np.zeros((n, 3))
    for d in range(3):
        p[:, d] = np.bincount(lin, weights=V[:, d], minlength=n)
    return p


# Per-cell momentum bound of the collision.  FP64: round-off of FP64 sums,
# below 1e-10 of the cell's momentum scale.  Mixed: v' = u + R (v - u) is
# formed and stored in FP32; each component of v' carries about ten
# roundings (2^-24 relative each) of terms no larger than |v - u|, so a
# cell's momentum changes by at most ~6e-7 sum_i |v_i - u| per component --
# below 5e-7 of the test's scale (the mean per-cell sum of |v| over the three
# components, about 24 at 10 particles per cell, kT = 1) for cells of up to
# about 25 particles.  No 32-bit velocity store can meet 1e-10: its
# rounding alone is 2^-24 of |v| per particle.
@pytest.mark.parametrize("prec,kernel,tol", [
    (abi.PREC_FP64, abi.KERNEL_SPLIT, 1e-10),
    (abi.PREC_FP64, abi.KERNEL_RESIDENT, 1e-10),
    (abi.PREC_FP64, abi.KERNEL_PERSIST, 1e-10),
    (abi.PREC_MIXED, abi.KERNEL_SPLIT, 5e-7),
    (abi.PREC_MIXED, abi.KERNEL_RESIDENT, 5e-7),
])
def test_collision_conserves_each_cells_momentum(prec, kernel, tol):
    # no grid shift and no streaming to speak of (dt = 1e-30): the collision
    # cells are the unshifted cells and positions do not move, so each
    # cell's momentum before and after the step must agree (SRD conserves
    # it per cell)
    L = (10, 9, 8)
    cfg = W.cfg_srd3d(L, precision=prec, seed=21, galinv=0, dt=1e-30)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=22)
    g = Solver(cfg)
    g.set_kernel(kernel)
    g.upload(Q, V, U, sp)
    q0, v0, _ = g.download()
    g.step(1, 1)
    q1, v1, _ = g.download()
    np.testing.assert_allclose(q1, q0, rtol=0, atol=1e-12)
    p0 = _cell_momenta(q0, v0, L)
    p1 = _cell_momenta(q1, v1, L)
    scale = np.abs(v0).sum() / len(p0)
    assert np.abs(p1 - p0).max() / scale < tol
    # and something did happen
    assert np.abs(v1 - v0).max() > 0.1


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-9), (abi.PREC_MIXED, 1e-4)])
def test_transverse_modes_match_host_restatement(prec, tol):
    from mpcd_b200.validate import transverse_modes
    L = (12, 10, 8)
    cfg = W.cfg_srd3d(L, precision=prec, seed=31)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=32)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    g.step(3, 1)
    q, v, _ = g.download()
    dev = g.transverse_modes()
    host = transverse_modes(q, v, L)
    scale = np.abs(v).sum()
    assert np.abs(dev - host).max() / scale < tol


def test_mixed_upload_rejects_bad_input_on_the_device():
    """The mixed form converts uploads on the device: a position outside the
    grid or a non-finite velocity is an error, and nothing is left to step."""
    from mpcd_b200.gpu import MPCDError
    cfg = W.cfg_srd3d((6, 6, 6), precision=abi.PREC_MIXED, seed=5)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=6)
    g = Solver(cfg)
    for bad in ("pos", "vel"):
        Qb, Vb = Q.copy(), V.copy()
        if bad == "pos":
            Qb[11, 0] = 6.0 + 1.5
        else:
            Vb[13, 2] = np.nan
        with pytest.raises(MPCDError):
            g.upload(Qb, Vb, U, sp)
        with pytest.raises(MPCDError):
            g.step(1, 1)
    g.upload(Q, V, U, sp)
    g.step(2, 1)
    q, v, _ = g.download()
    assert np.all(np.isfinite(v)) and np.all((q >= 0) & (q < 6))
    g.close()


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-10), (abi.PREC_MIXED, 5e-7)])
def test_collision_conserves_each_cells_momentum_64cubed(prec, tol):
    """The per-cell bound above on the 64^3 workload (2,621,440 particles,
    262,144 cells), default kernel family of each form."""
    L = (64, 64, 64)
    cfg = W.cfg_srd3d(L, precision=prec, seed=23, galinv=0, dt=1e-30)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=24)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    q0, v0, _ = g.download()
    g.step(1, 1)
    q1, v1, _ = g.download()
    np.testing.assert_allclose(q1, q0, rtol=0, atol=1e-12)
    p0 = _cell_momenta(q0, v0, L)
    p1 = _cell_momenta(q1, v1, L)
    scale = np.abs(v0).sum() / len(p0)
    assert np.abs(p1 - p0).max() / scale < tol
    assert np.abs(v1 - v0).max() > 0.1
    g.close()
