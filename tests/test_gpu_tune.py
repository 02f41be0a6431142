"""The autotuner on the GPU (mpcd_autotune): it times the plans that apply,
applies the fastest, and leaves the state, the error counters and the step
bookkeeping as they were, so the tuned handle still follows the oracle."""
import numpy as np
import pytest

from cases import build, state
from checkers import Oracle
from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["srd3d", "rat2d", "channel3d", "nematic2d_dipole"])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_tuned_plan_still_matches_oracle(name, prec, tmp_path):
    cfg, ppc, sseed, _ = build(name)
    cfgp, _, _, _ = build(name, precision=prec)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgp)
    g.upload(Q, V, U, sp)
    o.step(1)
    g.step(1, 1)
    st0 = g.status()
    c = g.autotune(trial_steps=8, cache_path=tmp_path / "tune.txt")
    assert c.candidates >= 2 and c.from_cache == 0 and c.us_per_step > 0
    st1 = g.status()
    assert (st1.steps, st1.escaped, st1.sync_timeout) == (st0.steps, st0.escaped, 0)
    for s in (2, 3):
        o.step(s)
        g.step(1, s)
    qo, vo, uo = o.particles()
    qg, vg, ug = g.download()
    if prec == abi.PREC_FP64:
        np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-11)
        np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-11 * max(cfg.L))
    else:
        bad = np.mean(np.abs(vg - vo).max(axis=1) > 1e-4)
        assert bad < 5e-3, bad
    # a second handle of the same workload takes the cached plan
    h2 = Solver(cfgp)
    h2.upload(Q, V, U, sp)
    c2 = h2.autotune(trial_steps=8, cache_path=tmp_path / "tune.txt")
    assert c2.from_cache == 1 and c2.candidates == 0
    assert (c2.kernel, c2.strategy, c2.tile_particles, c2.sort_interval) == \
        (c.kernel, c.strategy, c.tile_particles, c.sort_interval)
    g.close()
    h2.close()
