"""Live comparison of the CPU oracle with the reference's own timestep
(oracle/_ref/libmpcdref.so, built from the reference sources) on cases larger
than the golden ones; skipped where the reference build is absent."""
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
