"""Edge cases of the default SRD path (the resident kernel families of both
precision forms) through the C ABI, against the CPU oracle:

- one cell holding thousands of particles next to an ordinary fluid: the
  mixed form's per-block sum table and the FP64 form's atomics take any
  population, so the dense cell collides like the oracle's (the tile
  kernels' staging limit does not apply here);
- particles whose mass-weighted velocity is above the mixed form's limb
  range (|m v| >= 256), which skip the shared-memory table and add
  straight to the 64-bit global sums;
- an empty state: the upload is accepted and a step is refused with an
  error status, without a launch.
"""
import math

import numpy as np
import pytest

from checkers import Oracle
from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import MPCDError, Solver

pytestmark = pytest.mark.gpu


def _dense_cell_state(cfg, ppc, seed, cell, extra):
    """Uniform fluid of ppc particles per cell, plus `extra` particles
    inside one cell (away from its faces), velocities Maxwellian kT = 1."""
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=seed)
    rng = np.random.default_rng(seed + 1)
    q = np.zeros((extra, 3))
    for d in range(cfg.dim):
        q[:, d] = cell[d] + 0.05 + 0.9 * rng.random(extra)
    v = np.zeros((extra, 3))
    v[:, :cfg.dim] = rng.standard_normal((extra, cfg.dim))
    Q = np.concatenate([Q, q])
    V = np.concatenate([V, v])
    U = np.concatenate([U, np.zeros((extra, 3))])
    return Q, V, U, np.zeros(len(Q), dtype=np.int32)


def _compare(prec, qg, vg, qo, vo, L, vtol_rel):
    d = qg - qo
    d -= np.round(d / L) * L
    dq = np.abs(d).max(axis=1)
    scale = np.maximum(1.0, np.abs(vo).max(axis=1))
    dv = np.abs(vg - vo).max(axis=1) / scale
    if prec == abi.PREC_FP64:
        assert dv.max() < 1e-11 and dq.max() < 1e-11 * L.max(), (dv.max(), dq.max())
    else:
        # FP32 velocities and cell records: a few particles may land a
        # rounding away from a cell face and take another cell's rotation
        bad = np.mean((dv > vtol_rel) | (dq > 1e-4))
        assert bad < 2e-3, (bad, dv.max(), dq.max())


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_FP64])
def test_dense_cell_collides_like_the_oracle(prec):
    L = (6, 6, 6)
    cfg = W.cfg_srd3d(L, seed=61)
    cfgp = W.cfg_srd3d(L, precision=prec, seed=61)
    Q, V, U, sp = _dense_cell_state(cfg, 10, 62, (2, 3, 1), 5000)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgp)
    g.set_kernel(abi.KERNEL_RESIDENT)
    g.set_sort_interval(2)  # re-sort with the dense cell too
    g.upload(Q, V, U, sp)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(L, dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.overflow == 0 and st.nonfinite == 0
    # momentum is conserved by every collision (exactly in the mixed form's
    # fixed-point sums, to FP32 rounding in its velocities)
    p0, p1 = V.sum(axis=0), g.download()[1].sum(axis=0)
    tol = 1e-9 if prec == abi.PREC_FP64 else 2e-6 * np.abs(V).sum()
    assert np.abs(p1 - p0).max() < tol


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_FP64])
def test_fast_particles_in_populated_cells(prec):
    # |v| of 260-400 at dt = 0.01: up to 4 cells per step in an 8-cell box,
    # inside cells of 10 ordinary particles, so that they collide
    L = (8, 8, 8)
    cfg = W.cfg_srd3d(L, seed=63, dt=0.01)
    cfgp = W.cfg_srd3d(L, precision=prec, seed=63, dt=0.01)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=64)
    rng = np.random.default_rng(65)
    fast = rng.choice(len(Q), 40, replace=False)
    V[fast] = rng.uniform(260.0, 400.0, (40, 3)) * np.where(rng.random((40, 3)) < 0.5, -1, 1)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgp)
    g.set_kernel(abi.KERNEL_RESIDENT)
    g.upload(Q, V, U, sp)
    for s in (1, 2):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(L, dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    p0, p1 = V.sum(axis=0), g.download()[1].sum(axis=0)
    tol = 1e-8 if prec == abi.PREC_FP64 else 2e-6 * np.abs(V).sum()
    assert np.abs(p1 - p0).max() < tol


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_FP64])
def test_empty_state_is_refused_not_stepped(prec):
    cfg = W.cfg_srd3d((4, 4, 4), precision=prec, seed=66)
    g = Solver(cfg)
    g.upload(np.zeros((0, 3)), np.zeros((0, 3)))
    with pytest.raises(MPCDError):
        g.step(1, 1)
    assert g.status().steps == 0


@pytest.mark.parametrize("prec,kernel", [
    (abi.PREC_FP64, abi.KERNEL_AUTO), (abi.PREC_FP64, abi.KERNEL_RESIDENT),
    (abi.PREC_FP64, abi.KERNEL_TILE), (abi.PREC_FP64, abi.KERNEL_SPLIT),
    (abi.PREC_FP64, abi.KERNEL_GROUP), (abi.PREC_MIXED, abi.KERNEL_RESIDENT),
    (abi.PREC_MIXED, abi.KERNEL_TILE)])
@pytest.mark.parametrize("vdist", [abi.VDIST_RANDVEL, abi.VDIST_GAUSS, abi.VDIST_HOMO])
def test_bounce_limit_rethermalises_like_the_oracle(prec, kernel, vdist):
    """Particles that cross a 0.01-wide gap between two walls about a
    hundred times in a step pass the bounce limit (bc.c:1461-1488): the
    device lengthens the rewinds, then gives them a fresh velocity of the
    species' distribution, as the oracle (pinned to the reference) does."""
    from cases import thin_gap
    cfg, Q, V, sp = thin_gap(precision=abi.PREC_FP64)
    cfgp, _, _, _ = thin_gap(precision=prec)
    o = Oracle(cfg, Q, V, None, sp)
    o.set_vdist([vdist])
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.set_vdist([vdist])
    g.upload(Q, V, None, sp)
    L = np.array(cfg.L[:3], dtype=float)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
    qo, vo, _ = o.particles()
    qg, vg, _ = g.download()
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    assert o.bounce_limit() > 50
    if prec == abi.PREC_FP64:
        assert st.bounce_limit == o.bounce_limit()
        _compare(prec, qg, vg, qo, vo, L, 0)
    else:
        # FP32 velocities: a particle near the limit may take one bounce
        # more or less than the oracle's and draw differently
        assert abs(st.bounce_limit - o.bounce_limit()) <= 0.1 * o.bounce_limit()
        dv = np.abs(vg - vo).max(axis=1) / np.maximum(1.0, np.abs(vo).max(axis=1))
        assert np.mean(dv > 1e-4) < 0.1, np.mean(dv > 1e-4)
        d = qg - qo
        d -= np.round(d / L) * L
        same = dv <= 1e-4
        assert np.all(np.isfinite(vg)) and np.abs(d[same]).max() < 1e-4


@pytest.mark.parametrize("op,dim,kernel", [
    (abi.COLL_ARBAXIS, 3, abi.KERNEL_AUTO), (abi.COLL_ARBAXIS, 3, abi.KERNEL_RESIDENT),
    (abi.COLL_ARBAXIS, 3, abi.KERNEL_TILE), (abi.COLL_ARBAXIS, 3, abi.KERNEL_SPLIT),
    (abi.COLL_ARBAXIS, 3, abi.KERNEL_GROUP), (abi.COLL_RAT, 3, abi.KERNEL_PERSIST),
    (abi.COLL_RAT, 3, abi.KERNEL_TILE), (abi.COLL_MPCAT, 2, abi.KERNEL_TILE),
    ("lc", 2, abi.KERNEL_AUTO)])
def test_escaped_particles_are_replaced_like_the_oracle(op, dim, kernel):
    """Particles that leave the grid through an open side are re-placed at
    the end of the step as the reference's re-bin does (bin, mpc.c:969-982,
    the oracle pinned to the reference): the same positions, velocities,
    orientations and escape count, FP64, every kernel family."""
    from cases import open_bottom
    cfg, Q, V, U, sp = open_bottom(op, dim=dim)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.set_kernel(kernel)
    g.upload(Q, V, U, sp)
    L = np.array(cfg.L[:3], dtype=float)
    for s in (1, 2, 3, 4):
        o.step(s)
        g.step(1, s)
    qo, vo, uo = o.particles()
    qg, vg, ug = g.download()
    st = g.status()
    assert o.escaped() > 20 and st.escaped == o.escaped(), (st.escaped, o.escaped())
    _compare(abi.PREC_FP64, qg, vg, qo, vo, L, 0)
    if U is not None:
        assert np.abs(ug - uo).max() < 1e-11
    g.close()
    o.close()


@pytest.mark.parametrize("kernel", [abi.KERNEL_RESIDENT, abi.KERNEL_TILE, abi.KERNEL_SPLIT])
def test_mixed_form_replaces_escaped_particles(kernel):
    """The mixed form re-places particles that leave the grid too (its
    fixed-point positions stop at the grid's lower face, so a particle in
    [-1, 0) is held at 0 and leaves one step later than in the FP64 form):
    every particle ends inside the grid with a finite velocity, and the
    escapes are counted."""
    from cases import open_bottom
    cfg, Q, V, U, sp = open_bottom(abi.COLL_ARBAXIS, precision=abi.PREC_MIXED)
    g = Solver(cfg)
    g.set_kernel(kernel)
    g.upload(Q, V, U, sp)
    for s in range(1, 6):
        g.step(1, s)
    q, v, _ = g.download()
    st = g.status()
    assert st.escaped > 20 and st.nonfinite == 0
    assert np.all(np.isfinite(v)) and np.all(q >= 0.0) and np.all(q <= 6.0)
    g.close()


@pytest.mark.parametrize("prec,kernel,dim", [
    (abi.PREC_FP64, abi.KERNEL_TILE, 3), (abi.PREC_FP64, abi.KERNEL_PERSIST, 3),
    (abi.PREC_FP64, abi.KERNEL_AUTO, 2), (abi.PREC_FP64, abi.KERNEL_TILE, 2),
    (abi.PREC_MIXED, abi.KERNEL_TILE, 3), (abi.PREC_MIXED, abi.KERNEL_TILE, 2)])
def test_langevin_operator_matches_the_oracle(prec, kernel, dim):
    """The Langevin MPC operator (langevinMPC, mpc.c:1674-1780) on the tile
    and persistent kernel families against the oracle (pinned to the
    reference): two species, damping, a no-slip wall pair."""
    L = (6, 5, 7) if dim == 3 else (12, 10)
    sp = [W._species(mass=1.0, damp=0.1), W._species(mass=2.5, damp=0.1)]
    w = None
    if dim == 3:
        w = [abi.make_wall((1, 0, 0), (0, 0, 0), 0.0, DN=6.0),
             abi.make_wall((-1, 0, 0), (6, 0, 0), 0.0, DN=6.0),
             abi.make_wall((0, 1, 0), (0, 0, 0), 0.0, MVN=-1.0, MVT=-1.0),
             abi.make_wall((0, -1, 0), (0, 5, 0), 0.0, MVN=-1.0, MVT=-1.0),
             abi.make_wall((0, 0, 1), (0, 0, 0), 0.0, DN=7.0),
             abi.make_wall((0, 0, -1), (0, 0, 7), 0.0, DN=7.0)]
    cfg = W.base_config(dim, L, coll_op=abi.COLL_LANG, fricco=0.7, species=sp, walls=w,
                        seed=88)
    cfgp = W.base_config(dim, L, coll_op=abi.COLL_LANG, fricco=0.7, species=sp, walls=w,
                         seed=88, precision=prec)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=89)
    if dim == 3:
        Q[:, 1] = 0.02 + Q[:, 1] * (L[1] - 0.04) / L[1]  # off the walls' planes
    spid = (np.arange(len(Q)) % 3 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()


@pytest.mark.parametrize("prec,kernel,dim", [
    (abi.PREC_FP64, abi.KERNEL_TILE, 3), (abi.PREC_FP64, abi.KERNEL_PERSIST, 3),
    (abi.PREC_FP64, abi.KERNEL_AUTO, 2), (abi.PREC_MIXED, abi.KERNEL_TILE, 3),
    (abi.PREC_MIXED, abi.KERNEL_AUTO, 3)])
def test_orthogonal_axis_srd_matches_the_oracle(prec, kernel, dim):
    """SRD about a random Cartesian axis (stochrotMPC with RTECH ORTHAXIS,
    mpc.c:1289; rotate, mpc.c:1206-1236) on the tile and persistent kernel
    families against the oracle (pinned to the reference)."""
    L = (6, 5, 7) if dim == 3 else (12, 10)
    cfg = W.base_config(dim, L, coll_op=abi.COLL_ORTHAXIS, rot_ang=math.radians(130), seed=91)
    cfgp = W.base_config(dim, L, coll_op=abi.COLL_ORTHAXIS, rot_ang=math.radians(130),
                         seed=91, precision=prec)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=92)
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()


@pytest.mark.parametrize("op,prec,kernel,dim", [
    (abi.COLL_ACT_ARBAXIS, abi.PREC_FP64, abi.KERNEL_TILE, 3),
    (abi.COLL_ACT_ORTHAXIS, abi.PREC_FP64, abi.KERNEL_PERSIST, 3),
    (abi.COLL_ACT_ARBAXIS, abi.PREC_FP64, abi.KERNEL_AUTO, 2),
    (abi.COLL_ACT_ORTHAXIS, abi.PREC_MIXED, abi.KERNEL_TILE, 3),
    (abi.COLL_ACT_ARBAXIS, abi.PREC_MIXED, abi.KERNEL_AUTO, 2)])
def test_active_srd_matches_the_oracle(op, prec, kernel, dim):
    """Active SRD (activeSRD, mpc.c:2037-2077) on the tile and persistent
    kernel families against the oracle (pinned to the reference), with a net
    flow so that the cells' VCM have a direction."""
    L = (6, 5, 7) if dim == 3 else (12, 10)
    sp = [W._species(mass=1.0, act=0.3), W._species(mass=2.0, act=0.3)]
    kw = dict(coll_op=op, rot_ang=math.radians(110), species=sp, seed=93)
    cfg = W.base_config(dim, L, **kw)
    cfgp = W.base_config(dim, L, precision=prec, **kw)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=94)
    V[:, 0] += 0.4
    spid = (np.arange(len(Q)) % 4 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()


def test_active_srd_refuses_species_of_different_activity():
    """activeSRD takes the cell's activity from the last particle of its list,
    whose order the reference's re-binning sets: species of different
    activity are refused."""
    sp = [W._species(mass=1.0, act=0.3), W._species(mass=1.0, act=0.0)]
    cfg = W.base_config(3, (4, 4, 4), coll_op=abi.COLL_ACT_ARBAXIS, species=sp)
    with pytest.raises(MPCDError):
        Solver(cfg)


@pytest.mark.parametrize("op,prec,kernel,dim", [
    (abi.COLL_VICSEK_MPCAT, abi.PREC_FP64, abi.KERNEL_TILE, 3),
    (abi.COLL_VICSEK_LANG, abi.PREC_FP64, abi.KERNEL_PERSIST, 3),
    (abi.COLL_VICSEK_MPCAT, abi.PREC_FP64, abi.KERNEL_AUTO, 2),
    (abi.COLL_VICSEK_LANG, abi.PREC_FP64, abi.KERNEL_TILE, 2),
    (abi.COLL_VICSEK_MPCAT, abi.PREC_MIXED, abi.KERNEL_TILE, 3),
    (abi.COLL_VICSEK_LANG, abi.PREC_MIXED, abi.KERNEL_AUTO, 2)])
def test_vicsek_aligned_operators_match_the_oracle(op, prec, kernel, dim):
    """MPC-AT and Langevin MPC with Vicsek alignment (vicsekAndersenMPC,
    mpc.c:2204-2290; vicsekLangevinMPC, mpc.c:2409-2480) on the tile and
    persistent kernel families against the oracle (pinned to the
    reference): an active and a passive species, a net flow."""
    L = (6, 5, 7) if dim == 3 else (12, 10)
    sp = [W._species(mass=1.0, act=0.8, damp=0.3), W._species(mass=2.0, act=0.0, damp=0.3)]
    kw = dict(coll_op=op, species=sp, relax=0.5, fricco=0.8, seed=95)
    cfg = W.base_config(dim, L, **kw)
    cfgp = W.base_config(dim, L, precision=prec, **kw)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=96)
    V[:, 0] += 0.3
    spid = (np.arange(len(Q)) % 3 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()


@pytest.mark.parametrize("prec,kernel,dim", [
    (abi.PREC_FP64, abi.KERNEL_TILE, 3), (abi.PREC_FP64, abi.KERNEL_PERSIST, 3),
    (abi.PREC_FP64, abi.KERNEL_AUTO, 2), (abi.PREC_MIXED, abi.KERNEL_TILE, 3),
    (abi.PREC_MIXED, abi.KERNEL_AUTO, 2)])
def test_vicsek_matches_the_oracle(prec, kernel, dim):
    """Vicsek (vicsek, mpc.c:2098-2135, with genrand_cone, rand.c:438-454)
    on the tile and persistent kernel families against the oracle (pinned to
    the reference), a net flow."""
    L = (6, 5, 7) if dim == 3 else (12, 10)
    sp = [W._species(mass=1.0, act=0.7)]
    cfg = W.base_config(dim, L, coll_op=abi.COLL_VICSEK, species=sp, seed=97)
    cfgp = W.base_config(dim, L, coll_op=abi.COLL_VICSEK, species=sp, seed=97, precision=prec)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=98)
    V[:, 0] += 0.3
    V[:, 1] += 0.2
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()


@pytest.mark.parametrize("prec,kernel", [(abi.PREC_FP64, abi.KERNEL_TILE),
                                         (abi.PREC_FP64, abi.KERNEL_PERSIST),
                                         (abi.PREC_MIXED, abi.KERNEL_AUTO)])
def test_chate_matches_the_oracle(prec, kernel):
    """Chate (chate, mpc.c:2151-2186) against the oracle (pinned to the
    reference), 2D: the cells' director from the normalised velocities, a
    cone draw about it and a random sign.  A persistent-kernel request runs
    on the tile kernel, which holds the cells' director."""
    L = (12, 10)
    sp = [W._species(mass=1.0, act=0.6)]
    cfg = W.base_config(2, L, coll_op=abi.COLL_CHATE, species=sp, seed=99)
    cfgp = W.base_config(2, L, coll_op=abi.COLL_CHATE, species=sp, seed=99, precision=prec)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=100)
    V[:, 0] += 0.3
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()


def test_chate_in_3d_is_refused():
    """The 3D director needs the reference's 3x3 eigensystem, not built."""
    cfg = W.base_config(3, (4, 4, 4), coll_op=abi.COLL_CHATE)
    with pytest.raises(MPCDError):
        Solver(cfg)


@pytest.mark.parametrize("prec,kernel", [(abi.PREC_FP64, abi.KERNEL_TILE),
                                         (abi.PREC_FP64, abi.KERNEL_AUTO),
                                         (abi.PREC_MIXED, abi.KERNEL_AUTO)])
def test_chate_aligned_mpcat_matches_the_oracle(prec, kernel):
    """MPC-AT with Chate alignment (chateAndersenMPC, mpc.c:2300-2408), 2D,
    against the oracle (pinned to the reference): an active and a passive
    species, a net flow."""
    L = (12, 10)
    sp = [W._species(mass=1.0, act=0.8, damp=0.2), W._species(mass=2.0, act=0.0, damp=0.2)]
    kw = dict(coll_op=abi.COLL_CHATE_MPCAT, species=sp, relax=0.5, seed=101)
    cfg = W.base_config(2, L, **kw)
    cfgp = W.base_config(2, L, precision=prec, **kw)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=102)
    V[:, 0] += 0.3
    spid = (np.arange(len(Q)) % 3 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, spid)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        _compare(prec, qg, vg, qo, vo, np.array(cfg.L[:3], dtype=float), 1e-5)
    st = g.status()
    assert st.escaped == 0 and st.nonfinite == 0
    g.close()
    o.close()
