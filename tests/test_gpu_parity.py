"""GPU library (through its C ABI) against the CPU oracle on the same seeded
inputs and the same counter-based draws.

FP64 form: same algorithm and draws, only summation order and FMA
contraction differ -> agreement to 1e-12 (velocities O(1), positions O(L)).
Mixed form: FP32 offsets/velocities -> 1e-5 absolute on velocities after
one step, cell populations compared through the reported mismatch rate.
"""
import numpy as np
import pytest

from cases import CASES, build, state
from checkers import Oracle
from mpcd_b200 import abi
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu


def _min_image(d, L):
    return d - np.round(d / L) * L


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_oracle(name):
    cfg, ppc, sseed, nsteps = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    for s in range(1, nsteps + 1):
        o.step(s)
        kg, ag = g.timestep(s)
        qo, vo, _ = o.particles()
        qg, vg, ug = g.download()
        np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-12 * 10)
        np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-12 * max(cfg.L))
        if cfg.lc:
            np.testing.assert_allclose(ug, o.particles()[2], rtol=0, atol=1e-11)
        ko, ao = o.globals()
        assert kg == pytest.approx(ko, rel=1e-12)
        np.testing.assert_allclose(ag, ao, rtol=0, atol=1e-13)
    st = g.status()
    assert st.escaped == 0 and st.bounce_limit == 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_tracks_oracle(name):
    cfg, ppc, sseed, _ = build(name)
    cfgm, _, _, _ = build(name, precision=abi.PREC_MIXED)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgm)
    g.upload(Q, V, U, sp)
    o.step(1)
    kg, ag = g.timestep(1)
    qo, vo, uo = o.particles()
    qg, vg, ug = g.download()
    L = np.array([cfg.L[d] if d < cfg.dim else 1 for d in range(3)], dtype=float)
    if cfg.lc:
        # nematic: orientation (sign-free) tracks to FP32 precision
        du = np.minimum(np.abs(ug - uo).max(axis=1), np.abs(ug + uo).max(axis=1))
        assert np.mean(du > 1e-4) < 2e-3, du.max()
    dv = np.abs(vg - vo).max(axis=1)
    dq = np.abs(_min_image(qg - qo, L)).max(axis=1)
    # a particle within ~1e-7 of a cell face may bin differently in FP32
    # offsets and collide with other partners: allow a tiny fraction
    bad = np.mean((dv > 1e-5) | (dq > 1e-5))
    assert bad < 2e-3, (bad, dv.max(), dq.max())
    ko, ao = o.globals()
    assert kg == pytest.approx(ko, rel=1e-4)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_srd_conserves_momentum_and_energy(prec):
    from mpcd_b200 import workloads as W
    cfg = W.cfg_srd3d((16, 16, 16), precision=prec, seed=9)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=5)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    p0 = V.sum(axis=0)
    e0 = (V ** 2).sum()
    g.step(20, 1)
    _, v, _ = g.download()
    scale = np.abs(V).sum()
    tol = 1e-12 if prec == abi.PREC_FP64 else 1e-6
    assert np.abs(v.sum(axis=0) - p0).max() / scale < tol
    assert abs((v ** 2).sum() - e0) / e0 < (1e-12 if prec == abi.PREC_FP64 else 1e-5)


@pytest.mark.parametrize("strategy", [abi.STRATEGY_SCATTER, abi.STRATEGY_RECOMPUTE])
@pytest.mark.parametrize("name", ["srd3d", "srd2d", "rat2d", "channel3d", "mpcat3d_damp"])
@pytest.mark.parametrize("tile", [0, 64, 4096])
@pytest.mark.parametrize("kernel", [abi.KERNEL_AUTO, abi.KERNEL_TILE, abi.KERNEL_GROUP])
def test_strategies_and_tiles_agree_with_oracle(name, strategy, tile, kernel):
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.set_strategy(strategy, tile)
    g.set_kernel(kernel)
    g.upload(Q, V, U, sp)
    for s in range(1, 4):
        o.step(s)
        g.step(1, s)
    qo, vo, _ = o.particles()
    qg, vg, _ = g.download()
    np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-11 * max(cfg.L))


def _clumped_state(cfg, ppc, seed, clumps, per_clump):
    """Uniform fluid plus dense clumps of particles in a few cells, so that
    some cell tiles hold more particles than their staging capacity."""
    from mpcd_b200 import workloads as W
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=seed)
    rng = np.random.default_rng(seed + 1)
    extra_q = []
    for cidx in clumps:
        q = np.zeros((per_clump, 3))
        for d in range(cfg.dim):
            q[:, d] = cidx[d] + 0.05 + 0.9 * rng.random(per_clump)
        extra_q.append(q)
    Qx = np.concatenate([Q] + extra_q)
    n_extra = len(Qx) - len(Q)
    Vx = np.concatenate([V, np.zeros((n_extra, 3))])
    Vx[len(V):, :cfg.dim] = rng.standard_normal((n_extra, cfg.dim))
    Ux = np.concatenate([U, np.zeros((n_extra, 3))])
    spx = np.zeros(len(Qx), dtype=np.int32)
    return Qx, Vx, Ux, spx


@pytest.mark.parametrize("kernel", [abi.KERNEL_AUTO, abi.KERNEL_TILE, abi.KERNEL_GROUP])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_dense_tiles_are_subdivided(prec, kernel):
    # 40 dense cells of 200 particles: tiles far above capacity are split
    # into sub-tiles; every particle must still match the oracle.
    from mpcd_b200 import workloads as W
    cfg = W.cfg_srd3d((10, 10, 10), precision=abi.PREC_FP64, seed=31)
    cfgp = W.cfg_srd3d((10, 10, 10), precision=prec, seed=31)
    clumps = [(i % 10, (i // 10) % 10, 3 + (i % 4)) for i in range(40)]
    clumps += [(0, 0, z) for z in range(8)]  # one 32-cell group far above capacity
    Q, V, U, sp = _clumped_state(cfg, 10, 8, clumps, 200)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgp)
    g.set_kernel(kernel)
    g.upload(Q, V, U, sp)
    o.step(1)
    g.step(1, 1)
    qo, vo, _ = o.particles()
    qg, vg, _ = g.download()
    tol = 1e-11 if prec == abi.PREC_FP64 else 1e-5
    bad = np.mean(np.abs(vg - vo).max(axis=1) > tol)
    assert bad < (1e-12 if prec == abi.PREC_FP64 else 2e-3)
    assert g.status().overflow == 0


@pytest.mark.parametrize("kernel", [abi.KERNEL_TILE, abi.KERNEL_GROUP])
def test_overfull_cell_is_reported_not_collided(kernel):
    # one cell holding more particles than a tile can stage: its particles
    # stream without collision and are counted in status.overflow
    # (no grid shift, so the clump stays in one cell)
    from mpcd_b200 import workloads as W
    cfg = W.cfg_srd3d((6, 6, 6), seed=32, galinv=0)
    Q, V, U, sp = _clumped_state(cfg, 10, 9, [(2, 2, 2)], 5000)
    g = Solver(cfg)
    g.set_kernel(kernel)
    g.upload(Q, V, U, sp)
    g.step(1, 1)
    assert g.status().overflow >= 5000


def test_split_kernel_collides_any_cell_population():
    # the thread-per-cell pass has no staging limit: a 5000-particle cell
    # collides exactly like the oracle's
    from mpcd_b200 import workloads as W
    cfg = W.cfg_srd3d((6, 6, 6), seed=32, galinv=0)
    Q, V, U, sp = _clumped_state(cfg, 10, 9, [(2, 2, 2)], 5000)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.set_kernel(abi.KERNEL_SPLIT)
    g.upload(Q, V, U, sp)
    o.step(1)
    g.step(1, 1)
    np.testing.assert_allclose(g.download()[1], o.particles()[1], rtol=0, atol=1e-11)
    assert g.status().overflow == 0


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_nematic_multistep_conservation_and_order(prec):
    # 2D active nematic: orientations stay unit vectors, the mean order
    # parameter stays in [0, 1], and the FP64 form tracks the oracle over
    # several steps
    from mpcd_b200 import workloads as W
    cfg = W.cfg_nematic2d((16, 16), precision=prec, seed=77)
    cfg64 = W.cfg_nematic2d((16, 16), seed=77)
    Q, V, U, sp = W.synthetic_state(cfg, 20, seed=78)
    o = Oracle(cfg64, Q, V, U, sp)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    for s in range(1, 6):
        o.step(s)
        g.step(1, s)
    _, vg, ug = g.download()
    _, vo, uo = o.particles()
    n = np.linalg.norm(ug[:, :2], axis=1)
    assert np.abs(n - 1).max() < (1e-12 if prec == abi.PREC_FP64 else 1e-5)
    if prec == abi.PREC_FP64:
        np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-10)
        np.testing.assert_allclose(ug, uo, rtol=0, atol=1e-10)
