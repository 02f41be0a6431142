"""Transport checks on the GPU path: the curvature of a steady Poiseuille
profile in the MPC-AT+a channel between phantom no-slip walls gives the
kinematic viscosity, which both forms must reproduce, and which must agree
with the analytic value the reference prints (theory_trans, init.c:800-942).
A CPU test pins the restated analytic values."""
import math

import numpy as np
import pytest

from mpcd_b200 import abi
from mpcd_b200 import validate as V


def test_theory_restatement():
    """theory_trans for MPC-AT+a at n = 20 and random-axis SRD at n = 10,
    130 degrees, dt = 0.1 (values worked by hand from init.c:800-942)."""
    kin, col = V.theory_nu_reference(abi.COLL_RAT, 3, 20.0)
    assert kin == pytest.approx(0.1 * (1.0 / 0.9375 - 0.5) * 1.0, rel=1e-6)
    assert col == pytest.approx((20.0 - 1.4) / 2.4 / 20.0, rel=1e-6)
    kin, col = V.theory_nu_reference(abi.COLL_ARBAXIS, 3, 10.0, math.radians(130.0))
    a = 2.0 / 3.0 * (1.0 - math.sin(math.radians(130.0)) / math.radians(130.0))
    # integer density: the reference's smrtPow(e, -n) is 1, so M = 1
    assert col == pytest.approx(a / 12.0 / 0.1, rel=1e-9)
    # a non-integer density takes e^-n
    _, col = V.theory_nu_reference(abi.COLL_ARBAXIS, 3, 9.5, math.radians(130.0))
    assert col == pytest.approx(a * (9.5 - 1.0 + math.exp(-9.5)) / 12.0 / 0.1 / 9.5, rel=1e-9)


def test_channel_fit_recovers_viscosity():
    """The profile fit on noisy synthetic layer sums of a known parabola
    (with a wall slip, which shifts the parabola but not its curvature)."""
    rng = np.random.default_rng(5)
    H, T, g, nu = 16, 400, 2e-3, 0.44
    y = np.arange(H) + 0.5
    v = g * (y + 0.3) * (H + 0.3 - y) / (2 * nu)
    mm = np.full((T, H), 2560.0)
    mv = mm * (v + rng.normal(0, 0.01, (T, H)))
    r = V.fit_channel(mv, mm, g, nblk=4)
    assert r["nu"] == pytest.approx(nu, rel=0.02)
    assert r["nu_err"] < 0.01
    assert r["fit_rms"] < 1e-3


def test_channel_driver_with_fake_solver(monkeypatch):
    """channel_viscosity's loop and layer sums, against a stand-in solver
    whose cells hold the exact parabola (no GPU)."""
    g, nu = 2e-3, 0.5

    class Fake:
        def __init__(self, cfg):
            self.shp = tuple(int(cfg.L[d]) + 1 for d in range(3))
            self.steps = 0

        def upload(self, *a):
            pass

        def step(self, n, s0):
            self.steps += n

        def cell_props(self):
            H = self.shp[1] - 1
            y = np.arange(self.shp[1]) + 0.5
            vx = np.where(y < H, g * y * (H - y) / (2 * nu), 0.0)
            mass = np.ones(self.shp) * 20.0
            vcm = np.zeros(self.shp + (3,))
            vcm[..., 0] = vx[None, :, None]
            return None, mass, vcm, None

        def close(self):
            pass

    monkeypatch.setattr(V, "Solver", Fake)
    r = V.channel_viscosity(L=(8, 12, 4), g=g, warm=10, steps=40, every=10, nblk=2)
    assert r["nu"] == pytest.approx(nu, rel=1e-9)
    assert len(r["profile"]) == 12


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_FP64])
def test_channel_profile_viscosity(prec):
    r = V.channel_viscosity(L=(16, 16, 8), g=2e-3, warm=3000, steps=6000, every=10,
                            precision=prec, nblk=4)
    kin, col = V.theory_nu_reference(abi.COLL_RAT, 3, 20.0)
    assert r["fit_rms"] < 0.03 * r["v_max"], r
    assert r["nu"] == pytest.approx(kin + col, rel=0.15), r


def test_decay_fit_recovers_rate():
    """fit_decay on a noisy synthetic exponential: the rate to 1%."""
    rng = np.random.default_rng(9)
    t = np.arange(120) * 2.0
    s = 5e4 * np.exp(-0.004 * t) + rng.normal(0.0, 300.0, t.size)
    rate, used = V.fit_decay(t, s, 300.0)
    assert rate == pytest.approx(0.004, rel=0.01)
    assert 10 < used <= t.size
