"""The reference-facing boundary through the C ABI, against the CPU oracle:

- the strided calls that read and write the reference's particleMPC records
  in place (SRDclss.h:34-44: Q, V, U, T doubles, then the ids), orientations
  included;
- the output cell fields computed on the device (mpcd_cell_props: the re-bin
  and localPROP at the end of timestep, mpc.c:4936-4942);
- the step's own per-cell populations on the shifted grid
  (mpcd_debug_cell_counts), bit-exact against the cell lists of the
  reference's bin() (mpc.c:948-992) in the FP64 form;
- every step's global measures from mpcd_step_record;
- uploads that the device-side conversion rejects.
"""
import numpy as np
import pytest

from cases import build, state
from checkers import Oracle
from mpcd_b200 import abi, gpu
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu

# the reference's particleMPC: Q[3], V[3], U[3], T[3] doubles, then S_flag,
# SPID, q (int), and two pointers -- 128 bytes
REC = np.dtype([("Q", "<f8", 3), ("V", "<f8", 3), ("U", "<f8", 3), ("T", "<f8", 3),
                ("S_flag", "<i4"), ("SPID", "<i4"), ("q", "<i4"), ("pad", "<i4"),
                ("next", "<u8"), ("prev", "<u8")])
assert REC.itemsize == 128


def _records(Q, V, U, sp):
    r = np.zeros(len(Q), dtype=REC)
    r["Q"], r["V"], r["U"], r["SPID"] = Q, V, U, sp
    r["T"] = 7.0  # a field the library must leave alone
    return r


def _upload_strided(g, recs):
    import ctypes as C
    lib = g.lib
    off = REC.fields
    r = lib.mpcd_upload_particles_strided(g.h, len(recs), recs.ctypes.data_as(C.c_void_p),
                                          REC.itemsize, off["Q"][1], off["V"][1], off["U"][1],
                                          off["SPID"][1])
    assert r == 0, r
    g.n = len(recs)


def _download_strided(g, recs):
    import ctypes as C
    off = REC.fields
    r = g.lib.mpcd_download_particles_strided(g.h, recs.ctypes.data_as(C.c_void_p), REC.itemsize,
                                              off["Q"][1], off["V"][1], off["U"][1])
    assert r == 0, r


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_strided_records_carry_orientations(prec):
    """A nematic state through the reference's own record layout: the
    orientations go in through off_U and come back out through it."""
    cfg, ppc, sseed, _ = build("nematic2d_dipole")
    cfgp, _, _, _ = build("nematic2d_dipole", precision=prec)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgp)
    recs = _records(Q, V, U, sp)
    _upload_strided(g, recs)
    for s in (1, 2):
        o.step(s)
        g.step(1, s)
    _download_strided(g, recs)
    qo, vo, uo = o.particles()
    assert np.all(recs["T"] == 7.0)
    if prec == abi.PREC_FP64:
        np.testing.assert_allclose(recs["V"], vo, rtol=0, atol=1e-11)
        np.testing.assert_allclose(recs["U"], uo, rtol=0, atol=1e-11)
    else:
        du = np.minimum(np.abs(recs["U"] - uo).max(axis=1), np.abs(recs["U"] + uo).max(axis=1))
        assert np.mean(du > 1e-4) < 5e-3, du.max()
    g.close()


def _unshifted_props(cfg, Q, V, sp):
    """Re-bin on the unshifted grid and localPROP's sums in numpy."""
    dim = cfg.dim
    N1 = [cfg.L[d] + 1 if d < dim else 2 for d in range(3)]
    idx = np.zeros((len(Q), 3), dtype=np.int64)
    for d in range(dim):
        idx[:, d] = np.clip(np.trunc(Q[:, d]).astype(np.int64), 0, cfg.L[d])
    k = (idx[:, 0] * N1[1] + idx[:, 1]) * N1[2] + idx[:, 2]
    nc = N1[0] * N1[1] * N1[2]
    return np.bincount(k, minlength=nc)


@pytest.mark.parametrize("name", ["srd3d", "rat2d", "channel3d", "nematic2d_dipole",
                                  "srd3d_heavy"])
def test_cell_props_on_device_match_oracle(name):
    """POP bit-exact, MASS/VCM (and CM where localPROP computes it) to the
    FP64 form's 1e-12, after a few steps."""
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    for s in (1, 2, 3):
        o.step(s)
        g.step(1, s)
    pop, mass, vcm, cm = g.cell_props()
    po, mo, vo, co = o.cells()
    np.testing.assert_array_equal(pop.ravel(), po)
    np.testing.assert_allclose(mass.ravel(), mo, rtol=1e-13, atol=0)
    np.testing.assert_allclose(vcm.reshape(-1, 3), vo, rtol=0, atol=1e-12)
    if cfg.coll_op == abi.COLL_RAT or cfg.lc:
        np.testing.assert_allclose(cm.reshape(-1, 3), co, rtol=0, atol=1e-12 * max(cfg.L))
    g.close()


def test_cell_props_mixed_rebin_their_own_positions():
    """Mixed form: the device re-bin counts exactly the cells of the
    positions the download returns."""
    cfg = W.cfg_srd3d((12, 10, 8), precision=abi.PREC_MIXED, seed=61)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=62)
    g = Solver(cfg)
    g.upload(Q, V, U, sp)
    g.step(3, 1)
    qg, vg, _ = g.download()
    pop, mass, vcm, _ = g.cell_props()
    np.testing.assert_array_equal(pop.ravel(), _unshifted_props(cfg, qg, vg, sp))
    np.testing.assert_allclose(mass.ravel(), pop.ravel().astype(float), rtol=0, atol=1e-12)
    g.close()


KERNELS = {"auto": abi.KERNEL_AUTO, "split": abi.KERNEL_SPLIT, "tile": abi.KERNEL_TILE}


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", ["srd3d", "srd2d", "rat3d", "channel3d", "srd3d_heavy",
                                  "nematic2d_rat"])
def test_step_cell_counts_bit_exact_fp64(name, kernel):
    """FP64 form: the populations the step's kernels hold for the next
    step's collision equal, cell by cell, those of the reference's bin() on
    the same positions and shift (the oracle's restatement, pinned to the
    reference by the golden vectors)."""
    cfg, ppc, sseed, nsteps = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfg)
    g.set_kernel(KERNELS[kernel])
    g.upload(Q, V, U, sp)
    with pytest.raises(gpu.MPCDError):
        g.debug_cell_counts()  # no step yet
    for s in range(1, nsteps + 1):
        o.step(s)
        g.step(1, s)
        np.testing.assert_array_equal(g.debug_cell_counts(), o.shifted_counts(s + 1))
    g.close()


@pytest.mark.parametrize("name", ["srd3d", "srd2d", "channel3d", "nematic2d_dipole"])
def test_step_cell_counts_mixed_mismatch_rate(name):
    """Mixed form (quirk Q9): particles within 2^-22 of a shifted cell face,
    or whose FP32 velocity rounds across one, may bin differently; the
    fraction of cells whose population differs from the FP64 oracle's after
    one step stays below 1%."""
    cfg, ppc, sseed, _ = build(name)
    cfgm, _, _, _ = build(name, precision=abi.PREC_MIXED)
    Q, V, U, sp = state(cfg, ppc, sseed)
    o = Oracle(cfg, Q, V, U, sp)
    g = Solver(cfgm)
    g.upload(Q, V, U, sp)
    o.step(1)
    g.step(1, 1)
    a, b = g.debug_cell_counts(), o.shifted_counts(2)
    assert a.sum() == b.sum()
    assert np.mean(a != b) < 0.01, np.mean(a != b)
    g.close()


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_step_record_returns_every_steps_globals(prec):
    """mpcd_step_record over 70 steps (three read-back batches) returns what
    70 calls of mpcd_timestep return on a twin handle.  The mixed form's KE
    is summed in FP32 per thread, and the re-sort's ranks (atomics) decide
    which thread takes which particle, so its twins agree to FP32 rounding;
    its velocities are bitwise the same (exact fixed-point cell sums)."""
    cfg = W.cfg_srd3d((8, 8, 8), precision=prec, seed=63)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=64)
    a, b = Solver(cfg), Solver(cfg)
    a.upload(Q, V, U, sp)
    b.upload(Q, V, U, sp)
    kb, av = a.step_record(70, 5)
    rel = 1e-12 if prec == abi.PREC_FP64 else 1e-6
    for k in range(70):
        kt, at = b.timestep(5 + k)
        assert kb[k] == pytest.approx(kt, rel=rel)
        np.testing.assert_allclose(av[k], at, rtol=0, atol=1e-13)
    qa, va, _ = a.download()
    qb, vb, _ = b.download()
    np.testing.assert_allclose(va, vb, rtol=0, atol=1e-12)
    a.close()
    b.close()


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_upload_rejects_bad_values_on_device(prec):
    cfg = W.cfg_srd3d((6, 6, 6), precision=prec, species=[W._species(), W._species(mass=2.0)],
                      seed=65)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=66)
    g = Solver(cfg)
    bad = V.copy()
    bad[17, 1] = np.nan
    with pytest.raises(gpu.MPCDError, match="-1"):
        g.upload(Q, bad, U, sp)
    spb = sp.copy()
    spb[3] = 2  # no third species
    with pytest.raises(gpu.MPCDError, match="-1"):
        g.upload(Q, V, U, spb)
    with pytest.raises(gpu.MPCDError, match="-5"):
        g.step(1, 1)  # a rejected upload leaves no state
    g.upload(Q, V, U, sp)
    g.step(1, 1)
    g.close()
