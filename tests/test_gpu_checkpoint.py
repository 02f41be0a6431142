"""Checkpoint and resume through the reference's text format on the GPU:
a run stopped after k steps, written as a precise checkpoint, read into a
new handle and continued equals the run that never stopped.  FP64 form:
the same within the parity bound (the continued run sums cells in another
particle order).  Mixed form: identical, because its cell sums are exact
integers, so the particle order does not matter."""
import numpy as np
import pytest

from cases import build, init_case, state
from checkers import Reference
from mpcd_b200 import abi
from mpcd_b200.gpu import Checkpoint, Solver

pytestmark = pytest.mark.gpu


def _resume(cfg, Q, V, U, sp, k, m, tmp_path, precise=True):
    a = Solver(cfg)
    a.upload(Q, V, U, sp)
    a.step(k + m, 1)
    qa, va, ua = a.download()
    b = Solver(cfg)
    b.upload(Q, V, U, sp)
    b.step(k, 1)
    ck = Checkpoint(cfg=cfg)
    ck.capture(b)
    path = tmp_path / "resume.dat"
    ck.write(path, precise=precise)
    rd = Checkpoint(path)
    c2 = rd.config()
    c2.precision = cfg.precision
    c = Solver(c2)
    rd.upload(c)
    c.step(m, k + 1)
    qc, vc, uc = c.download()
    for s in (a, b, c):
        s.close()
    return (qa, va, ua), (qc, vc, uc)


@pytest.mark.parametrize("name", ["srd3d", "channel3d", "rat2d", "nematic2d_dipole"])
def test_fp64_resume_matches_uninterrupted_run(tmp_path, name):
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    (qa, va, ua), (qc, vc, uc) = _resume(cfg, Q, V, U, sp, 5, 5, tmp_path)
    np.testing.assert_allclose(vc, va, rtol=0, atol=1e-11)
    np.testing.assert_allclose(qc, qa, rtol=0, atol=1e-11 * max(cfg.L))
    if cfg.lc:
        np.testing.assert_allclose(uc, ua, rtol=0, atol=1e-10)


@pytest.mark.parametrize("name", ["srd3d", "channel3d", "rat3d"])
def test_mixed_resume_is_identical(tmp_path, name):
    cfg, ppc, sseed, _ = build(name, precision=abi.PREC_MIXED)
    Q, V, U, sp = state(cfg, ppc, sseed)
    (qa, va, _), (qc, vc, _) = _resume(cfg, Q, V, U, sp, 6, 6, tmp_path)
    np.testing.assert_array_equal(qc, qa)
    np.testing.assert_array_equal(vc, va)


def test_capture_carries_species_and_reference_reads_it(tmp_path):
    """A two-species state built on the device, captured and written, is
    what the reference's own reader sees."""
    cfg, params = init_case("init_two_species")
    g = Solver(cfg)
    g.init_state(params)
    g.step(3, 1)
    Q, V, _ = g.download()
    sp = g.species()
    assert np.array_equal(np.bincount(sp), [1500, 900])
    ck = Checkpoint(cfg=cfg)
    ck.capture(g)
    q2, v2, _, sp2 = ck.particles()
    np.testing.assert_array_equal(q2, Q)
    np.testing.assert_array_equal(sp2, sp)
    if Reference.available():
        path = tmp_path / "two.dat"
        ck.write(path, precise=True)
        rc, Qr, Vr, _, spr, *_ = Reference.checkpoint_read(path, abi.Config)
        np.testing.assert_array_equal(Qr, Q)
        np.testing.assert_array_equal(Vr, V)
        np.testing.assert_array_equal(spr, sp)
    g.close()
