"""The persistent kernel family (MPCD_KERNEL_PERSIST: a small FP64 box held in
the shared memory of the blocks of one cooperative launch, many steps per
launch) against the CPU oracle: every isotropic operator of the golden cases
(SRD, MPC-AT with damping, MPC-AT+a, the phantom-wall channel, a heavy
species), stepped in launches of several steps, to the FP64 form's parity bar
(1e-12 on velocities, 1e-12 L on positions), with the cell populations of the
next step compared bit for bit."""
import numpy as np
import pytest

from cases import CASES, build, state
from checkers import Oracle
from mpcd_b200 import abi, gpu
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu

ISOTROPIC = sorted(n for n in CASES if not n.startswith("nematic"))


@pytest.mark.parametrize("name", ISOTROPIC)
def test_persist_matches_oracle(name):
    cfg, ppc, sseed, nsteps = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.set_kernel(abi.KERNEL_PERSIST)
    g.upload(Q, V, U, sp)
    s = 1
    for chunk in (1, 2, nsteps):  # launches of 1, 2 and nsteps steps
        kb, av = g.step_record(chunk, s)
        for k in range(chunk):
            o.step(s + k)
        s += chunk
        qo, vo, _ = o.particles()
        qg, vg, _ = g.download()
        np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-12 * 10)
        np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-12 * max(cfg.L))
        np.testing.assert_array_equal(g.debug_cell_counts(), o.shifted_counts(s))
        ko, ao = o.globals()
        assert kb[-1] == pytest.approx(ko, rel=1e-12)
        np.testing.assert_allclose(av[-1], ao, rtol=0, atol=1e-13)
    st = g.status()
    assert st.escaped == 0 and st.bounce_limit == 0
    g.close()


def test_persist_two_species_and_gravity():
    """Two species of different mass (and damping) under gravity, MPC-AT+a."""
    sp_ = [W._species(mass=1.0, damp=0.1), W._species(mass=2.5, damp=0.0)]
    cfg = W.base_config(3, (5, 6, 4), coll_op=abi.COLL_RAT, species=sp_, grav=(2e-3, 0, -1e-3),
                        seed=91)
    Q, V, U, spid = W.synthetic_state(cfg, 12, seed=92)
    spid = (np.arange(len(Q)) % 2).astype(np.int32)
    o = Oracle(cfg, Q, V, U, spid)
    g = Solver(cfg)
    g.set_kernel(abi.KERNEL_PERSIST)
    g.upload(Q, V, U, spid)
    g.step(4, 1)
    for s in range(1, 5):
        o.step(s)
    qo, vo, _ = o.particles()
    qg, vg, _ = g.download()
    np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-12 * 6)
    g.close()


def test_persist_matches_resident_on_a_larger_box():
    """A 3D SRD box of 24,000 particles: the persistent family and the FP64
    resident family (different summation orders) agree over 20 steps."""
    cfg = W.cfg_srd3d((20, 12, 10), seed=93)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=94)
    a, b = Solver(cfg), Solver(cfg)
    a.set_kernel(abi.KERNEL_PERSIST)
    b.set_kernel(abi.KERNEL_RESIDENT)
    a.upload(Q, V, U, sp)
    b.upload(Q, V, U, sp)
    a.step(20, 1)
    b.step(20, 1)
    qa, va, _ = a.download()
    qb, vb, _ = b.download()
    np.testing.assert_allclose(va, vb, rtol=0, atol=1e-10)
    np.testing.assert_allclose(qa, qb, rtol=0, atol=1e-10 * 20)
    a.close()
    b.close()


def test_persist_auto_for_small_fp64_boxes_and_refuses_large_ones():
    cfg = W.cfg_passive2d((30, 30), seed=95)
    Q, V, U, sp = W.synthetic_state(cfg, 20, seed=96)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    g.step(10, 1)
    assert g.launches_per_step() == 1  # one persistent launch for the 10 steps
    g.close()
    big = W.cfg_srd3d((128, 128, 128), seed=97)  # 21M particles: beyond the blocks' memory
    Qb, Vb, Ub, spb = W.synthetic_state(big, 10, seed=98)
    g = Solver(big)
    g.set_kernel(abi.KERNEL_PERSIST)
    g.upload(Qb, Vb, Ub, spb)
    with pytest.raises(gpu.MPCDError, match="-2"):
        g.step(1, 1)
    g.close()
