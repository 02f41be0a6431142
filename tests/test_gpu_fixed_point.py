"""Exact streaming in the mixed form, on the GPU, through both SRD kernel
families: particles alone in their cells (no collision partner, so their
velocity is unchanged) must move by exactly rint(float32(dt * v) * 2^22)
units of 2^-22 cell, the resolution of the mixed form's position words."""
import numpy as np
import pytest

from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu


def _isolated_state(L, seed):
    """One particle in every second cell along each axis (so no shifted cell
    ever holds two), at positions that are exact multiples of 2^-22, with
    velocities spanning many magnitudes, both signs and exact ties."""
    rng = np.random.default_rng(seed)
    idx = np.stack(np.meshgrid(*[np.arange(0, l - 1, 2) for l in L], indexing="ij"), -1)
    idx = idx.reshape(-1, 3)
    n = len(idx)
    frac = np.floor(rng.random((n, 3)) * 2.0 ** 22) * 2.0 ** -22
    frac = 0.25 + 0.5 * frac  # away from the cell faces
    frac = np.round(frac * 2.0 ** 22) * 2.0 ** -22
    Q = idx + frac
    mag = np.exp2(rng.integers(-30, 1, size=(n, 3))) * (1.0 + rng.random((n, 3)))
    V = (np.where(rng.random((n, 3)) < 0.5, -1.0, 1.0) * mag).astype(np.float32)
    V[: n // 4] = (rng.integers(-99, 100, size=(n // 4, 3)) * 2 + 1) * 2.0 ** -20  # ties at dt=1/8
    return Q, V.astype(np.float64)


@pytest.mark.parametrize("kernel", [abi.KERNEL_RESIDENT, abi.KERNEL_SPLIT])
def test_isolated_particles_stream_exactly(kernel):
    L = (12, 10, 8)
    cfg = W.cfg_srd3d(L, precision=abi.PREC_MIXED, seed=5, dt=0.125)
    Q, V = _isolated_state(L, 6)
    g = Solver(cfg)
    g.set_kernel(kernel)
    g.upload(Q, V, None, np.zeros(len(Q), dtype=np.int32))
    g.step(1, 1)
    q, v, _ = g.download()
    np.testing.assert_array_equal(v, V)
    dx = (np.float32(0.125) * V.astype(np.float32)).astype(np.float64)
    disp = np.rint(dx * 2.0 ** 22)  # ties to even
    expect = (np.round(Q * 2.0 ** 22) + disp) * 2.0 ** -22
    np.testing.assert_array_equal(q, expect)


@pytest.mark.parametrize("kernel", [abi.KERNEL_RESIDENT, abi.KERNEL_SPLIT])
def test_fast_isolated_particles_stream_exactly(kernel):
    # displacements of more than one cell per step take the 64-bit path
    L = (16, 16, 16)
    cfg = W.cfg_srd3d(L, precision=abi.PREC_MIXED, seed=7, dt=0.125)
    Q = np.array([[2.25, 2.5, 2.75], [10.5, 3.25, 9.125], [5.5, 12.75, 4.25],
                  [13.25, 9.5, 13.75]])
    V = np.array([[12.5, -9.25, 15.75], [-14.125, 8.0, -11.5], [9.0625, -15.5, 13.25],
                  [-10.75, 11.125, -8.5]])
    g = Solver(cfg)
    g.set_kernel(kernel)
    g.upload(Q, V, None, np.zeros(len(Q), dtype=np.int32))
    g.step(1, 1)
    q, v, _ = g.download()
    np.testing.assert_array_equal(v, V)
    expect = np.mod(Q + 0.125 * V, 16.0)
    np.testing.assert_array_equal(q, expect)
