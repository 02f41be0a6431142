"""Live comparison of the CPU oracle with the reference's own timestep
(oracle/_ref/libmpcdref.so, built from the reference sources) on cases larger
than the golden ones; skipped where the reference build is absent."""
import math

import numpy as np
import pytest

from checkers import Oracle, Reference
from mpcd_b200 import abi
from mpcd_b200 import workloads as W

pytestmark = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("builder,kw,ppc", [
    (W.cfg_srd3d, dict(L=(12, 10, 9)), 10),
    (W.cfg_channel3d, dict(L=(10, 12, 6), g=5e-3), 20),
    (W.cfg_passive2d, dict(L=(30, 30)), 20),
    (W.base_config, dict(dim=3, L=(7, 6, 8), coll_op=abi.COLL_RAT), 12),
])
def test_oracle_tracks_reference(builder, kw, ppc):
    cfg = builder(**kw, seed=4242)
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=99)
    o = Oracle(cfg, Q, V, U, sp)
    r = Reference(cfg, Q, V, U, sp)
    for s in range(1, 7):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(cfg.L))
    np.testing.assert_array_equal(o.cells()[0], r.cells()[0])
    ko, ao = o.globals()
    kr, ar = r.globals()
    assert ko == pytest.approx(kr, rel=1e-12)


@pytest.mark.parametrize("coll_op,dim,n,ra,dt", [
    (abi.COLL_ARBAXIS, 3, 10.0, 2.2689280275926285, 0.1),
    (abi.COLL_ARBAXIS, 2, 20.0, 1.5707963267948966, 0.1),
    (abi.COLL_ARBAXIS, 3, 5.0, 1.0, 0.25),
    (abi.COLL_ARBAXIS, 3, 9.5, 2.2689280275926285, 0.1),
    (abi.COLL_MPCAT, 2, 12.25, 1.5707963267948966, 0.1),
    (abi.COLL_MPCAT, 2, 20.0, 1.5707963267948966, 0.1),
    (abi.COLL_MPCAT, 3, 10.0, 1.5707963267948966, 0.05),
    (abi.COLL_RAT, 3, 20.0, 1.5707963267948966, 0.1),
    (abi.COLL_RAT, 2, 20.0, 1.5707963267948966, 0.1),
    (abi.COLL_RAT, 3, 7.5, 1.5707963267948966, 0.2),
])
def test_theory_restatement_matches_reference(coll_op, dim, n, ra, dt):
    """The restated analytic viscosity (mpcd_b200.validate.theory_nu_reference)
    against the compiled reference's own theory_trans."""
    from mpcd_b200 import validate as V
    kin, col = V.theory_nu_reference(coll_op, dim, n, ra, dt=dt)
    nu, _, mfp = Reference.theory_visc(coll_op, dim, n, ra, dt)
    assert kin + col == pytest.approx(nu, rel=1e-12)
    assert mfp == pytest.approx(dt, rel=1e-15)


@pytest.mark.parametrize("vdist", [abi.VDIST_RANDVEL, abi.VDIST_HOMO, abi.VDIST_HOMOAXIS,
                                   abi.VDIST_GAUSS])
def test_bounce_limit_rethermalisation_tracks_reference(vdist):
    """Particles past the bounce limit: the oracle's longer rewinds and
    re-thermalisations (bc.c:1461-1488, velocities of the species' VDIST
    from the re-thermalisation stream) follow the reference's.  SRD keeps
    the fast particles fast through the collision (an Andersen collision
    would redraw them thermal first)."""
    from cases import thin_gap
    cfg, Q, V, sp = thin_gap()
    o = Oracle(cfg, Q, V, None, sp)
    o.set_vdist([vdist])
    r = Reference(cfg, Q, V, None, sp)
    r.set_vdist([vdist])
    for s in range(1, 4):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    assert o.bounce_limit() > 50 and o.escaped() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11)


def test_bounce_limit_rethermalisation_draws_the_species_distribution():
    """The re-thermalised velocities follow VDIST: the same run with
    uniform and with Maxwell-Boltzmann re-thermalisation differs."""
    from cases import thin_gap
    out = []
    for vdist in (abi.VDIST_RANDVEL, abi.VDIST_GAUSS):
        cfg, Q, V, sp = thin_gap()
        o = Oracle(cfg, Q, V, None, sp)
        o.set_vdist([vdist])
        for s in range(1, 4):
            o.step(s)
        out.append(o.particles()[1])
    assert not np.array_equal(out[0], out[1])


@pytest.mark.parametrize("op,dim", [(abi.COLL_ARBAXIS, 3), (abi.COLL_RAT, 3),
                                    (abi.COLL_MPCAT, 2), ("lc", 2)])
def test_escape_replacement_tracks_reference(op, dim):
    """Particles that leave the grid through an open side: the oracle's
    re-placement (bin, mpc.c:969-982; replacePos_WithCheck, init.c:1462-1483,
    with the ceiling rejecting positions above it) and fresh velocities and
    orientations follow the reference's, draw for draw."""
    from cases import open_bottom
    cfg, Q, V, U, sp = open_bottom(op, dim=dim)
    o = Oracle(cfg, Q, V, U, sp)
    r = Reference(cfg, Q, V, U, sp)
    for s in range(1, 5):
        o.step(s)
        r.step(s)
    qo, vo, uo = o.particles()
    qr, vr, ur = r.particles()
    assert r.unexpected_draws() == 0
    assert o.escaped() > 20
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11)
    if U is not None:
        np.testing.assert_allclose(uo, ur, rtol=0, atol=1e-11)
    assert np.all(qo[:, 1] > -1.0)  # nothing left outside the grid


@pytest.mark.parametrize("dim,L,fricco,damp", [(3, (7, 6, 8), 1.0, 0.0), (2, (20, 16), 0.5, 0.2),
                                                (3, (6, 6, 6), 2.0, 0.1)])
def test_langevin_operator_tracks_reference(dim, L, fricco, damp):
    """The Langevin MPC operator (langevinMPC, mpc.c:1674-1780: the plain mean
    of the noise, friction factors a and b per species) of the oracle against
    the reference's own, with two species."""
    sp = [W._species(mass=1.0, damp=damp), W._species(mass=2.5, damp=damp)]
    cfg = W.base_config(dim, L, coll_op=abi.COLL_LANG, fricco=fricco, species=sp, seed=515)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=516)
    spid = (np.arange(len(Q)) % 3 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))
    ko, _ = o.globals()
    kr, _ = r.globals()
    assert ko == pytest.approx(kr, rel=1e-12)


@pytest.mark.parametrize("dim,L,ra", [(3, (7, 6, 8), 130.0), (3, (6, 6, 6), 90.0),
                                      (2, (20, 16), 120.0)])
def test_orthogonal_axis_srd_tracks_reference(dim, L, ra):
    """SRD about a random Cartesian axis (RTECH ORTHAXIS: stochrotMPC,
    mpc.c:1289, with rotate's matrices, mpc.c:1206-1236, including the x-axis
    matrix's -.1*S) of the oracle against the reference's own."""
    cfg = W.base_config(dim, L, coll_op=abi.COLL_ORTHAXIS, rot_ang=math.radians(ra), seed=525)
    Q, V, U, spid = W.synthetic_state(cfg, 10, seed=526)
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))
    if dim == 3:
        # the x-axis matrix shrinks |v - u| along z: kinetic energy is not conserved
        ko, _ = o.globals()
        kr, _ = r.globals()
        assert ko == pytest.approx(kr, rel=1e-12)


@pytest.mark.parametrize("op,dim,L,act", [(9, 3, (7, 6, 8), 0.3), (10, 3, (6, 6, 6), 0.5),
                                          (9, 2, (20, 16), 0.2)])
def test_active_srd_tracks_reference(op, dim, L, act):
    """Active SRD (activeSRD, mpc.c:2037-2077: the SRD rotation, then every
    particle turned toward the cell's VCM by ACT times their angle) of the
    oracle against the reference's own, random and Cartesian axes, two
    species of one activity."""
    sp = [W._species(mass=1.0, act=act), W._species(mass=2.0, act=act)]
    cfg = W.base_config(dim, L, coll_op=op, rot_ang=math.radians(110), species=sp, seed=535)
    Q, V, U, spid = W.synthetic_state(cfg, 10, seed=536)
    V[:, 0] += 0.4  # a net flow, so that the cells' VCM have a direction
    spid = (np.arange(len(Q)) % 4 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))


@pytest.mark.parametrize("op,dim,L,relax", [(11, 3, (7, 6, 8), 0.5), (12, 3, (6, 6, 6), 0.3),
                                            (11, 2, (20, 16), 0.7), (12, 2, (16, 14), 0.5)])
def test_vicsek_aligned_operators_track_reference(op, dim, L, relax):
    """MPC-AT and Langevin MPC with Vicsek alignment (vicsekAndersenMPC,
    mpc.c:2204-2290; vicsekLangevinMPC, mpc.c:2409-2480: RELAX (ACT VCMdir -
    V) for active species, no damping) of the oracle against the
    reference's own: an active and a passive species, a net flow."""
    sp = [W._species(mass=1.0, act=0.8, damp=0.3), W._species(mass=2.0, act=0.0, damp=0.3)]
    cfg = W.base_config(dim, L, coll_op=op, species=sp, relax=relax, fricco=0.8, seed=545)
    Q, V, U, spid = W.synthetic_state(cfg, 10, seed=546)
    V[:, 0] += 0.3
    spid = (np.arange(len(Q)) % 3 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))


@pytest.mark.parametrize("dim,L,act", [(3, (7, 6, 8), 0.7), (3, (6, 6, 6), 0.2), (2, (20, 16), 0.6)])
def test_vicsek_tracks_reference(dim, L, act):
    """Vicsek (vicsek, mpc.c:2098-2135: each particle keeps its speed and
    takes a direction on the cone genrand_cone, rand.c:438-454, builds about
    the cell's VCM direction) of the oracle against the reference's own, a
    net flow."""
    sp = [W._species(mass=1.0, act=act)]
    cfg = W.base_config(dim, L, coll_op=abi.COLL_VICSEK, species=sp, seed=555)
    Q, V, U, spid = W.synthetic_state(cfg, 10, seed=556)
    V[:, 0] += 0.3
    V[:, 1] += 0.2
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))


@pytest.mark.parametrize("L,act,seed", [((20, 16), 0.6, 565), ((16, 18), 0.2, 566)])
def test_chate_tracks_reference(L, act, seed):
    """Chate (chate, mpc.c:2151-2186: the cells' director from the order
    tensor of the normalised velocities, then a cone draw about it with a
    random sign) of the oracle against the reference's own, 2D."""
    sp = [W._species(mass=1.0, act=act)]
    cfg = W.base_config(2, L, coll_op=abi.COLL_CHATE, species=sp, seed=seed)
    Q, V, U, spid = W.synthetic_state(cfg, 10, seed=seed + 1)
    V[:, 0] += 0.3
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))


@pytest.mark.parametrize("L,relax", [((20, 16), 0.5), ((16, 18), 0.2)])
def test_chate_aligned_mpcat_tracks_reference(L, relax):
    """MPC-AT with Chate alignment (chateAndersenMPC, mpc.c:2300-2408: the
    active velocity pmOne RELAX (ACT - |V|) DIR joins the thermal one, no
    damping) of the oracle against the reference's own, 2D, an active and a
    passive species."""
    sp = [W._species(mass=1.0, act=0.8, damp=0.2), W._species(mass=2.0, act=0.0, damp=0.2)]
    cfg = W.base_config(2, L, coll_op=abi.COLL_CHATE_MPCAT, species=sp, relax=relax, seed=575)
    Q, V, U, spid = W.synthetic_state(cfg, 10, seed=576)
    V[:, 0] += 0.3
    spid = (np.arange(len(Q)) % 3 == 0).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    r = Reference(cfg, Q, V, U, spid)
    for s in range(1, 6):
        o.step(s)
        r.step(s)
    qo, vo, _ = o.particles()
    qr, vr, _ = r.particles()
    assert r.unexpected_draws() == 0
    np.testing.assert_allclose(vo, vr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qo, qr, rtol=0, atol=1e-11 * max(L))
