"""The FP64 form's resident kernel family (MPCD_KERNEL_RESIDENT with
MPCD_PREC_FP64) through the C ABI, against the CPU oracle.

It uses the FP64 form's arithmetic; only the order of the FP64 cell sums
differs (atomics instead of the sorted order), so it meets the FP64 form's
parity bar: 1e-12 on velocities and 1e-12 L on positions, step after step.
"""
import numpy as np
import pytest

from cases import build, state
from checkers import Oracle
from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu


def _walled_srd(seed=777):
    """3D SRD between two plain (non-phantom) no-slip walls at y = 0 and
    y = L1, periodic x and z, with gravity along x."""
    L = (6, 7, 5)
    walls = [w for w in W.channel_walls(L)]
    for w in walls:
        w.phantom = 0
    return W.base_config(3, L, coll_op=abi.COLL_ARBAXIS, walls=walls, grav=(5e-3, 0.0, 0.0),
                         seed=seed)


@pytest.mark.parametrize("name", ["srd3d", "srd2d", "srd3d_heavy", "walled", "two_species"])
def test_fp64_resident_matches_oracle(name):
    if name == "walled":
        cfg, ppc, sseed, nsteps = _walled_srd(), 10, 31, 5
    elif name == "two_species":
        cfg = W.cfg_srd3d((7, 6, 5), species=[W._species(mass=1.0), W._species(mass=3.0)],
                          seed=778)
        ppc, sseed, nsteps = 10, 32, 4
    else:
        cfg, ppc, sseed, nsteps = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    if cfg.n_species > 1:
        sp = (np.arange(len(Q)) % cfg.n_species).astype(np.int32)
    if name == "walled":
        Q[:, 1] = 0.02 + Q[:, 1] * (cfg.L[1] - 0.04) / cfg.L[1]  # off the walls' planes
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.set_kernel(abi.KERNEL_RESIDENT)
    g.set_sort_interval(2)  # exercise the locality re-sort too
    g.upload(Q, V, U, sp)
    for s in range(1, nsteps + 1):
        o.step(s)
        kg, ag = g.timestep(s)
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-12 * 10)
        np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-12 * max(cfg.L))
        ko, ao = o.globals()
        assert kg == pytest.approx(ko, rel=1e-12)
        np.testing.assert_allclose(ag, ao, rtol=0, atol=1e-13)
    st = g.status()
    assert st.escaped == 0 and st.bounce_limit == 0


def test_fp64_resident_matches_split_family_over_many_steps():
    """Resident and split families of the FP64 form on the same state: the
    same trajectory to rounding over 30 steps (the sums differ only in
    order)."""
    cfg = W.cfg_srd3d((9, 7, 6), seed=41)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=42)
    out = []
    for kernel in (abi.KERNEL_RESIDENT, abi.KERNEL_SPLIT):
        g = Solver(cfg)
        g.set_kernel(kernel)
        g.upload(Q, V, U, sp)
        g.step(30, 1)
        out.append(g.download())
        g.close()
    (qa, va, _), (qb, vb, _) = out
    np.testing.assert_allclose(va, vb, rtol=0, atol=1e-9)
    np.testing.assert_allclose(qa, qb, rtol=0, atol=1e-9 * 9)


def test_fp64_resident_conserves_momentum_and_energy():
    cfg = W.cfg_srd3d((8, 8, 8), seed=43)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=44)
    g = Solver(cfg)
    g.set_kernel(abi.KERNEL_RESIDENT)
    g.upload(Q, V, U, sp)
    p0 = V.sum(axis=0)
    e0 = (V ** 2).sum()
    g.step(25, 1)
    _, v, _ = g.download()
    scale = np.abs(V).sum()
    assert np.abs(v.sum(axis=0) - p0).max() / scale < 1e-12
    assert abs((v ** 2).sum() - e0) / e0 < 1e-12
