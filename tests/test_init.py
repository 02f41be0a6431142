"""Initial state and accessible volume on the CPU: the oracle's restatement
of the reference's initialisation (setcoord, galileantrans, VSC scaling;
init.c:1565-1600, 2092-2170) against golden states from the reference's own
code with the same injected draws, and the library's exact accessible volume
against the reference's Monte Carlo estimate (accessibleVolume,
init.c:954-989) with its own generator (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from cases import INIT_CASES, init_case, slab_walls
from checkers import oracle_init_state
from mpcd_b200 import abi, gpu
from mpcd_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(INIT_CASES))
def test_oracle_init_matches_reference_golden(name):
    """Same draws, same arithmetic, sums in the same serial order: the
    oracle's state equals the reference's bit for bit."""
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg, params = init_case(name)
    Q, V, U, sp, kbt = oracle_init_state(cfg, params)
    np.testing.assert_array_equal(sp, g["spid"])
    np.testing.assert_array_equal(Q, g["Q"])
    np.testing.assert_array_equal(V, g["V"])
    np.testing.assert_array_equal(U, g["U"])
    assert kbt == float(g["kbt"])


def test_init_cases_exercise_rejection_and_distributions():
    """The slab cases re-place particles (a uniform first draw lands in the
    walls for 31% / 56% of them), every particle ends outside its walls, and
    the velocity distributions have their defining shapes."""
    for name, lo, hi in (("init_slab_homo", 1.5, 9.75), ("init_slab_inv_homoaxis", 2.25, 7.5)):
        g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        y = g["Q"][:, 1]
        assert y.min() > lo and y.max() < hi
    g = np.load(os.path.join(GOLDEN, "init_slab_homo.npz"))
    cfg, params = init_case("init_slab_homo")
    speed = np.linalg.norm(g["V"], axis=1)
    assert np.ptp(speed) < 1e-12 * speed.max()  # HOMO: one speed for all
    g = np.load(os.path.join(GOLDEN, "init_slab_inv_homoaxis.npz"))
    a = np.abs(g["V"])
    assert np.ptp(a) < 1e-12 * a.max()  # HOMOAXIS: +-s on every axis
    g = np.load(os.path.join(GOLDEN, "init_srd3d_randvel.npz"))
    V = g["V"]
    s = np.abs(V).max(axis=0)
    assert np.all(s < 1.0 * 1.01 * np.sqrt(3.0)) and np.all(s > 0.9)


@pytest.mark.parametrize("name", sorted(INIT_CASES))
def test_accessible_volume_matches_reference_monte_carlo(name):
    """The reference estimates the volume from 1000 points per unit volume;
    the exact product of intervals lies within 5 standard errors of it."""
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg, _ = init_case(name)
    box = float(np.prod([cfg.L[d] for d in range(3)]))
    for s in range(cfg.n_species):
        exact = gpu.accessible_volume(cfg, s)
        mc = float(g["volume_mc"][s])
        p = exact / box
        se = box * np.sqrt(max(p * (1 - p), 1e-12) / (1000 * box))
        assert abs(mc - exact) <= 5 * se + 1e-9, (s, mc, exact)


def test_accessible_volume_hand_values():
    L = (10, 12, 8)
    c = W.base_config(3, L, coll_op=abi.COLL_MPCAT)
    assert gpu.accessible_volume(c) == 960.0
    c = W.base_config(3, L, coll_op=abi.COLL_MPCAT, walls=slab_walls(L, 1.5, 9.75))
    assert gpu.accessible_volume(c) == pytest.approx(10 * 8.25 * 8, abs=1e-12)
    c = W.base_config(3, L, coll_op=abi.COLL_MPCAT, walls=slab_walls(L, 2.25, 7.5, True))
    assert gpu.accessible_volume(c) == pytest.approx(10 * 5.25 * 8, abs=1e-12)
    # walls that leave nothing: the fluid side of each lies beyond the other
    c = W.base_config(3, L, coll_op=abi.COLL_MPCAT, walls=slab_walls(L, 9.0, 3.0))
    assert gpu.accessible_volume(c) == 0.0
    # a species that ignores the walls sees the whole box; 2D counts z as 1
    cfg, _ = init_case("init_two_species")
    assert gpu.accessible_volume(cfg, 1) == 240.0
    assert gpu.accessible_volume(cfg, 0) == pytest.approx(6 * (7.5 - 1.25) * 5, abs=1e-12)
    c = W.cfg_passive2d((30, 20))
    assert gpu.accessible_volume(c) == 600.0
    with pytest.raises(gpu.MPCDError):
        gpu.accessible_volume(c, 1)
