"""Initial state built on the device (mpcd_init_state) against the CPU
oracle's restatement of the reference's initialisation, which the CPU suite
pins bit for bit to the reference's own code (tests/test_init.py).

FP64 form: positions and the drawn velocities and orientations come from the
same counter-based draws with the same rounding, so positions are equal bit
for bit; the velocity scaling's sums are block trees on the device and serial
on the CPU, so velocities agree to a few ulp (1e-14), orientations to the
last ulp of cos/sin/atan2 (1e-14).  Mixed form: positions within one 2^-22
fixed-point step, velocities and orientations within FP32 rounding."""
import math

import numpy as np
import pytest

from cases import INIT_CASES, init_case, slab_walls
from checkers import Oracle, oracle_init_state
from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import MPCDError, Solver

pytestmark = pytest.mark.gpu

# orientation codes a 2D nematic state cannot hold (a z component)
_Z_ODIST = (abi.ODIST_ALIGNZ, abi.ODIST_PLANEY, abi.ODIST_PLANEX)


def _gpu_case(name, precision=abi.PREC_FP64):
    """init_case with the 2D nematic's z-component codes replaced by
    RANDORIENT (the oracle takes the same parameters)."""
    cfg, params = init_case(name, precision)
    if cfg.lc and cfg.dim == 2:
        for s in range(cfg.n_species):
            if params.odist[s] in _Z_ODIST:
                params.odist[s] = abi.ODIST_RANDORIENT
    return cfg, params


@pytest.mark.parametrize("name", sorted(INIT_CASES))
def test_fp64_init_matches_oracle(name):
    cfg, params = _gpu_case(name)
    Qo, Vo, Uo, _, ko = oracle_init_state(cfg, params)
    g = Solver(cfg)
    kg = g.init_state(params)
    Qg, Vg, Ug = g.download()
    np.testing.assert_array_equal(Qg, Qo)
    np.testing.assert_allclose(Vg, Vo, rtol=0, atol=1e-14)
    if cfg.lc:
        np.testing.assert_allclose(Ug[:, :2], Uo[:, :2], rtol=0, atol=1e-14)
    assert kg == pytest.approx(ko, rel=1e-13)
    g.close()


@pytest.mark.parametrize("name", sorted(INIT_CASES))
def test_mixed_init_matches_oracle(name):
    cfg, params = _gpu_case(name)
    cfgm, _ = _gpu_case(name, precision=abi.PREC_MIXED)
    Qo, Vo, Uo, _, ko = oracle_init_state(cfg, params)
    g = Solver(cfgm)
    kg = g.init_state(params)
    Qg, Vg, Ug = g.download()
    np.testing.assert_allclose(Qg, Qo, rtol=0, atol=2.0 ** -22)
    np.testing.assert_allclose(Vg, Vo, rtol=0, atol=1e-6 * np.abs(Vo).max())
    if cfg.lc:
        np.testing.assert_allclose(Ug[:, :2], Uo[:, :2], rtol=0, atol=1e-6)
    assert kg == pytest.approx(ko, rel=1e-13)  # computed in FP64 before conversion
    g.close()


def test_init_is_reproducible_and_keyed_by_seed_and_replica():
    cfg, params = init_case("init_slab_homo")
    runs = []
    for seed, replica in ((777, 0), (777, 0), (778, 0), (777, 1)):
        cfg.seed, cfg.replica = seed, replica
        g = Solver(cfg)
        g.init_state(params)
        runs.append(g.download())
        g.close()
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)
    assert not np.array_equal(runs[0][0], runs[2][0])
    assert not np.array_equal(runs[0][0], runs[3][0])


@pytest.mark.parametrize("name", ["init_slab_homo", "init_two_species", "init_nematic_odist"])
def test_init_then_steps_match_oracle(name):
    """The device-built state steps as the oracle does from its own
    initial state (the FP64 parity bound of the timestep)."""
    cfg, params = _gpu_case(name)
    Qo, Vo, Uo, sp, _ = oracle_init_state(cfg, params)
    o = Oracle(cfg, Qo, Vo, Uo if cfg.lc else None, sp)
    g = Solver(cfg)
    g.init_state(params)
    for s in range(1, 5):
        o.step(s)
        kg, ag = g.timestep(s)
        qo, vo, uo = o.particles()
        qg, vg, ug = g.download()
        np.testing.assert_allclose(vg, vo, rtol=0, atol=1e-11)
        np.testing.assert_allclose(qg, qo, rtol=0, atol=1e-11 * max(cfg.L))
        if cfg.lc:
            np.testing.assert_allclose(ug[:, :2], uo[:, :2], rtol=0, atol=1e-10)
        ko, ao = o.globals()
        assert kg == pytest.approx(ko, rel=1e-11)
    st = g.status()
    assert st.escaped == 0 and st.bounce_limit == 0
    g.close()


def test_init_full_size_matches_oracle():
    """The 64^3 SRD fluid at 10 particles per cell (2,621,440 particles),
    Maxwell-Boltzmann, built on the device: equal to the oracle's state."""
    cfg = W.cfg_srd3d((64, 64, 64), seed=2026)
    params = abi.init_params([10 * 64 ** 3], vdist=abi.VDIST_GAUSS)
    Qo, Vo, _, _, ko = oracle_init_state(cfg, params)
    g = Solver(cfg)
    kg = g.init_state(params)
    Qg, Vg, _ = g.download()
    np.testing.assert_array_equal(Qg, Qo)
    # the scaling factor comes from 2.6 M-term sums taken in another order
    np.testing.assert_allclose(Vg, Vo, rtol=2e-13, atol=1e-15)
    assert kg == pytest.approx(ko, rel=1e-12)
    assert kg == pytest.approx(1.0, abs=1e-5)
    g.close()


def test_init_rejects_bad_requests():
    L = (10, 12, 8)
    g = Solver(W.base_config(3, L, coll_op=abi.COLL_MPCAT, walls=slab_walls(L, 9.0, 3.0)))
    with pytest.raises(MPCDError, match=r"-1 "):  # no accessible volume
        g.init_state(abi.init_params([100]))
    assert g.n == 0
    g.close()
    g = Solver(W.cfg_srd3d((4, 4, 4)))
    with pytest.raises(MPCDError, match=r"-2 "):  # vDist READ is an upload
        g.init_state(abi.init_params([100], vdist=1))
    p = abi.init_params([100])
    p.population[1] = 5  # a species the config does not have
    with pytest.raises(MPCDError, match=r"-1 "):
        g.init_state(p)
    assert g.init_state(abi.init_params([0])) == 0.0
    g.close()
    cfg, params = init_case("init_nematic_odist")
    g = Solver(cfg)
    with pytest.raises(MPCDError, match=r"-2 "):  # z components in 2D
        g.init_state(params)
    g.close()
