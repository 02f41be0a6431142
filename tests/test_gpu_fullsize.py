"""Parity at the benchmark sizes: the 64^3 SRD fluid (2,621,440 particles),
the 128x64x64 MPC-AT+a channel between phantom walls (10,485,760) and the
256^2 active nematic (1,310,720), each on the default kernel family of each
form, against the CPU oracle on the same seeded state and draws.

Size-dependent code paths run only here: the resident table's slot packing
(set from L), the 4x4x4 brick sort keys, scans of many tiles, the 22-bit
offset words near 64 cells and beyond, the channel's walls at 128x64x64.

FP64 form: the cell populations of every step's shifted grid are compared
bit for bit with the oracle's binning (the reference's bin(), mpc.c:948-992),
velocities and orientations to 1e-11 and positions to 1e-12 L.  Mixed form
(quirk Q9): the fraction of cells whose population differs, and of particles
that differ from the FP64 oracle by more than 1e-5, are bounded."""
import numpy as np
import pytest

from checkers import Oracle
from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu

CONFIGS = {
    # name: (builder, kwargs, particles per cell, steps compared)
    "srd64": (W.cfg_srd3d, dict(L=(64, 64, 64)), 10, 3),
    "channel128x64x64": (W.cfg_channel3d, dict(L=(128, 64, 64), g=1e-4), 20, 1),
    "nematic256": (W.cfg_nematic2d, dict(L=(256, 256)), 20, 1),
}


def _min_image(d, L):
    return d - np.round(d / L) * L


def _setup(name, prec):
    builder, kw, ppc, nsteps = CONFIGS[name]
    cfg = builder(**kw, precision=abi.PREC_FP64, seed=4242)
    cfgp = builder(**kw, precision=prec, seed=4242)
    Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=4243)
    if name.startswith("channel"):
        Q[:, 1] = 0.02 + Q[:, 1] * (cfg.L[1] - 0.04) / cfg.L[1]  # off the walls' planes
    return cfg, cfgp, Q, V, U, sp, nsteps


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_fullsize_fp64_matches_oracle(name):
    cfg, _, Q, V, U, sp, nsteps = _setup(name, abi.PREC_FP64)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    del Q, V
    for s in range(1, nsteps + 1):
        o.step(s)
        kg, ag = g.timestep(s)
        np.testing.assert_array_equal(g.debug_cell_counts(), o.shifted_counts(s + 1))
        qo, vo, uo = o.particles()
        qg, vg, ug = g.download()
        dv = np.abs(vg - vo).max()
        assert dv <= 1e-11, (s, dv, np.unravel_index(np.argmax(np.abs(vg - vo)), vg.shape))
        assert np.abs(qg - qo).max() <= 1e-12 * max(cfg.L)
        if cfg.lc:
            assert np.abs(ug - uo).max() <= 1e-11
        ko, ao = o.globals()
        assert kg == pytest.approx(ko, rel=1e-12)
        np.testing.assert_allclose(ag, ao, rtol=0, atol=1e-13)
    st = g.status()
    assert st.escaped == 0 and st.bounce_limit == 0 and st.overflow == 0
    g.close()
    o.close()


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_fullsize_mixed_tracks_oracle(name):
    cfg, cfgm, Q, V, U, sp, _ = _setup(name, abi.PREC_MIXED)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgm)
    g.upload(Q, V, U, sp)
    del Q, V
    o.step(1)
    kg, _ = g.timestep(1)
    a, b = g.debug_cell_counts(), o.shifted_counts(2)
    assert a.sum() == b.sum()
    assert np.mean(a != b) < 0.01, np.mean(a != b)
    qo, vo, uo = o.particles()
    qg, vg, ug = g.download()
    L = np.array([cfg.L[d] if d < cfg.dim else 1 for d in range(3)], dtype=float)
    dv = np.abs(vg - vo).max(axis=1)
    dq = np.abs(_min_image(qg - qo, L)).max(axis=1)
    bad = np.mean((dv > 1e-5) | (dq > 1e-5))
    assert bad < 3e-3, (bad, dv.max(), dq.max())
    if cfg.lc:
        du = np.minimum(np.abs(ug - uo).max(axis=1), np.abs(ug + uo).max(axis=1))
        assert np.mean(du > 1e-4) < 3e-3
    ko, _ = o.globals()
    assert kg == pytest.approx(ko, rel=1e-4)
    st = g.status()
    assert st.escaped == 0 and st.overflow == 0
    g.close()
    o.close()
