"""The ensemble API (mpcd_batch_*): boxes of different sizes stepped
together must follow, bit for bit, the trajectories of single-box handles of
the resident family with the same generator keys (seed, replica = box
index), and keep each box's momentum and temperature."""
import numpy as np
import pytest

from mpcd_b200 import abi
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Batch, Solver

pytestmark = pytest.mark.gpu

SIZES = [(8, 8, 8), (12, 12, 12), (16, 16, 16), (8, 12, 16), (12, 8, 8), (24, 24, 24)]
SEEDS = [101, 202, 303, 404, 505, 606]


def _states(ppc=10):
    out = []
    for b, L in enumerate(SIZES):
        cfg = W.cfg_srd3d(L, precision=abi.PREC_MIXED, seed=SEEDS[b])
        Q, V, _, _ = W.synthetic_state(cfg, ppc, seed=1000 + b)
        out.append((cfg, Q, V))
    return out


def test_batch_matches_single_box_handles():
    states = _states()
    base = W.cfg_srd3d(SIZES[0], precision=abi.PREC_MIXED, seed=SEEDS[0])
    bat = Batch(base, SIZES, SEEDS)
    npart = [len(Q) for _, Q, _ in states]
    bat.upload(npart, np.concatenate([Q for _, Q, _ in states]),
               np.concatenate([V for _, _, V in states]), step0=1)
    nsteps = 25  # includes the periodic re-sort
    bat.step(nsteps)
    Qb, Vb = bat.download()
    kb, av = bat.globals()
    off = 0
    for b, (cfg, Q, V) in enumerate(states):
        cfg.replica = b
        g = Solver(cfg)
        g.set_kernel(abi.KERNEL_RESIDENT)
        g.upload(Q, V, None, np.zeros(len(Q), dtype=np.int32))
        g.step(nsteps, 1)
        q, v, _ = g.download()
        kg, ag = g.globals()
        n = len(Q)
        assert np.array_equal(Qb[off:off + n], q), b
        assert np.array_equal(Vb[off:off + n], v), b
        assert kb[b] == pytest.approx(kg, rel=1e-6)
        np.testing.assert_allclose(av[b], ag, rtol=0, atol=1e-9)
        off += n
        g.close()
    bat.close()


def test_batch_conserves_per_box_momentum_and_temperature():
    states = _states()
    base = W.cfg_srd3d(SIZES[0], precision=abi.PREC_MIXED, seed=7)
    bat = Batch(base, SIZES, SEEDS)
    npart = [len(Q) for _, Q, _ in states]
    V0 = np.concatenate([V for _, _, V in states])
    bat.upload(npart, np.concatenate([Q for _, Q, _ in states]), V0, step0=1)
    bat.step(40)
    _, V1 = bat.download()
    kb, _ = bat.globals()
    off = 0
    for b, n in enumerate(npart):
        p0 = V0[off:off + n].sum(axis=0)
        p1 = V1[off:off + n].sum(axis=0)
        assert np.abs(p1 - p0).max() / np.abs(V0[off:off + n]).sum() < 1e-6
        e0 = (V0[off:off + n] ** 2).sum()
        e1 = (V1[off:off + n] ** 2).sum()
        assert abs(e1 - e0) / e0 < 1e-5
        assert kb[b] == pytest.approx(e1 / (3 * n), rel=1e-3)
        off += n
    bat.close()


def test_batch_rejects_unsupported_configs():
    base = W.cfg_srd3d((8, 8, 8), precision=abi.PREC_FP64)
    with pytest.raises(Exception):
        Batch(base, [(8, 8, 8)])


def test_batch_runs_on_the_legacy_default_stream():
    # the step graphs are captured on a private stream, so any launch stream
    # works, the legacy default stream (handle 0) included
    states = _states()[:3]
    base = W.cfg_srd3d(SIZES[0], precision=abi.PREC_MIXED, seed=3)
    out = []
    for use_default in (False, True):
        bat = Batch(base, SIZES[:3], SEEDS[:3])
        if use_default:
            bat.set_stream(0)
        bat.upload([len(Q) for _, Q, _ in states], np.concatenate([Q for _, Q, _ in states]),
                   np.concatenate([V for _, _, V in states]), step0=5)
        bat.step(4)
        out.append(bat.download())
        bat.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_batch_upload_rejects_positions_outside_their_box():
    """The device-side conversion of an upload checks every position against
    its own box; a rejected upload leaves nothing to step, and a valid one
    afterwards works."""
    base = W.cfg_srd3d((8, 8, 8), precision=abi.PREC_MIXED, seed=3)
    bat = Batch(base, [(8, 8, 8), (6, 6, 6)])
    rng = np.random.default_rng(3)
    q1, q2 = rng.random((500, 3)) * 8, rng.random((300, 3)) * 6
    q2[7, 2] = 6.5  # inside the first box's size, outside its own
    v = rng.standard_normal((800, 3))
    with pytest.raises(Exception):
        bat.upload([500, 300], np.vstack([q1, q2]), v)
    with pytest.raises(Exception):
        bat.step(1)
    q2[7, 2] = 5.5
    bat.upload([500, 300], np.vstack([q1, q2]), v)
    bat.step(2)
    q, vv = bat.download()
    assert q.shape == (800, 3) and np.all(np.isfinite(vv))
    assert np.all(q[:500] < 8) and np.all(q[500:] < 6)
    bat.close()


def test_batch_per_box_momentum_and_temperature_against_fp64():
    """Each box of the mixed ensemble against the FP64 form of the same box
    (a single-box FP64 handle with the same generator key, so the same grid
    shifts, axes and initial state): after 40 steps (a re-sort included) the
    box's temperature (TEMP, therm.c:209-235) agrees to 1e-5 relative and its
    momentum to 1e-6 of the box's momentum scale, the FP32 rounding of the
    mixed form; the FP64 boxes conserve momentum to 1e-12 of that scale."""
    states = _states()
    base = W.cfg_srd3d(SIZES[0], precision=abi.PREC_MIXED, seed=SEEDS[0])
    bat = Batch(base, SIZES, SEEDS)
    npart = [len(Q) for _, Q, _ in states]
    bat.upload(npart, np.concatenate([Q for _, Q, _ in states]),
               np.concatenate([V for _, _, V in states]), step0=1)
    nsteps = 40
    bat.step(nsteps)
    Qb, Vb = bat.download()
    kb, _ = bat.globals()
    off = 0
    for b, (cfg, Q, V) in enumerate(states):
        c64 = W.cfg_srd3d(SIZES[b], precision=abi.PREC_FP64, seed=SEEDS[b])
        c64.replica = b
        g = Solver(c64)
        g.upload(Q, V, None, np.zeros(len(Q), dtype=np.int32))
        g.step(nsteps, 1)
        _, v64, _ = g.download()
        k64, _ = g.globals()
        n = len(Q)
        scale = np.abs(V).sum()
        p0 = V.sum(axis=0)
        assert np.abs(v64.sum(axis=0) - p0).max() / scale < 1e-12, b
        assert np.abs(Vb[off:off + n].sum(axis=0) - v64.sum(axis=0)).max() / scale < 1e-6, b
        assert kb[b] == pytest.approx(k64, rel=1e-5), b
        off += n
        g.close()
    bat.close()
