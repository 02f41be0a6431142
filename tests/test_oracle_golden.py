"""The CPU oracle (oracle/mpcd_oracle.c) against golden vectors produced by
the reference's own timestep with the same injected draws
(tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from cases import CASES, build, state
from checkers import Oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# FP64, same algorithm, summation order differs (reference: linked-list
# order; oracle: particle index order): agreement to round-off.
ATOL = 1e-12


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg, ppc, sseed, nsteps = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    np.testing.assert_array_equal(Q, g["Q0"])
    np.testing.assert_array_equal(V, g["V0"])
    o = Oracle(cfg, Q, V, U, sp)
    assert o.gndnst() == pytest.approx(float(g["gndnst"]), abs=0)
    for s in range(1, nsteps + 1):
        o.step(s)
        q, v, u = o.particles()
        kb, av = o.globals()
        if cfg.lc:
            np.testing.assert_allclose(u, g[f"U{s}"], rtol=0, atol=1e-11)
        pop, _, _, _ = o.cells()
        np.testing.assert_allclose(q, g[f"Q{s}"], rtol=0, atol=ATOL * max(cfg.L))
        np.testing.assert_allclose(v, g[f"V{s}"], rtol=0, atol=ATOL * 10)
        assert kb == pytest.approx(float(g[f"kbt{s}"]), rel=1e-13)
        np.testing.assert_allclose(av, g[f"av{s}"], rtol=0, atol=1e-14)
        np.testing.assert_array_equal(pop, g[f"pop{s}"])
    assert o.escaped() == 0
