"""Checkpoints in the reference's text format (host side, no GPU).

The reference writes checkpoints with checkpoint() (pout.c:2325-2396) and
reads them with readchckpnt() (read.c:669-834).  Pinned here:
  - a file the reference wrote (committed fixture, and live where the
    compiled reference is present) reads into the library and writes back
    byte for byte;
  - the configuration and particles the library takes from it equal the
    state the reference wrote, to the file's six decimals;
  - a file the library writes is read by the reference's own reader: in the
    precise form exactly, in the reference's form to six decimals;
  - runs using features outside the library are reported as unsupported.
"""
import gzip
import os

import numpy as np
import pytest

from cases import build, state
from checkers import Reference
from mpcd_b200 import abi, gpu
from mpcd_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
live = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")


def _golden_file(tmp_path):
    path = tmp_path / "ref_ckpt.dat"
    with gzip.open(os.path.join(GOLDEN, "ckpt_rat2d.dat.gz"), "rb") as g:
        path.write_bytes(g.read())
    return path


def _state_after(name, steps=3):
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    return cfg, Q, V, U, sp


def test_golden_reference_checkpoint_round_trips_byte_for_byte(tmp_path):
    src = _golden_file(tmp_path)
    ck = gpu.Checkpoint(src)
    out = tmp_path / "lib.dat"
    ck.write(out)
    assert out.read_bytes() == src.read_bytes()


def test_golden_reference_checkpoint_fields(tmp_path):
    """rat2d (8 x 7, MPC-AT+a, 20 per cell) after three reference steps."""
    ck = gpu.Checkpoint(_golden_file(tmp_path))
    cfg0, _, _, _ = build("rat2d")
    cfg = ck.config()
    assert (cfg.dim, list(cfg.L), cfg.coll_op, cfg.lc, cfg.galinv) == (2, [8, 7, 1], 3, 0, 1)
    assert cfg.dt == cfg0.dt and cfg.kbt == cfg0.kbt and cfg.seed == cfg0.seed
    assert cfg.rot_ang == pytest.approx(cfg0.rot_ang, abs=5e-7)
    assert cfg.n_walls == cfg0.n_walls and cfg.n_species == 1
    for w in range(cfg.n_walls):
        a, b = cfg.walls[w], cfg0.walls[w]
        assert list(a.A) == list(b.A) and list(a.Q) == list(b.Q)
        assert (a.DN, a.MVN, a.MVT, a.inv, a.phantom) == (b.DN, b.MVN, b.MVT, b.inv, b.phantom)
        assert list(a.inter) == list(b.inter)
    run = ck.run()
    assert (run.runtime, run.warmtime, run.sim_steps) == (3, 0, 1000)
    assert ck.count() == 20 * 56
    g = np.load(os.path.join(GOLDEN, "rat2d.npz"))
    Q, V, U, sp = ck.particles()
    np.testing.assert_allclose(Q, g["Q3"], rtol=0, atol=5e-7)
    np.testing.assert_allclose(V, g["V3"], rtol=0, atol=5e-7)
    assert np.all(sp == 0)


@live
@pytest.mark.parametrize("name", ["channel3d", "nematic2d_dipole", "mpcat3d_damp"])
def test_reference_checkpoints_round_trip_byte_for_byte(tmp_path, name):
    cfg, Q, V, U, sp = _state_after(name)
    r = Reference(cfg, Q, V, U, sp)
    for s in range(1, 3):
        r.step(s)
    src = tmp_path / "ref.dat"
    r.checkpoint_write(src, 2, 0)
    ck = gpu.Checkpoint(src)
    out = tmp_path / "lib.dat"
    ck.write(out)
    assert out.read_bytes() == src.read_bytes()
    qr, vr, ur = r.particles()
    q, v, u, _ = ck.particles()
    np.testing.assert_allclose(q, qr, rtol=0, atol=5e-7)
    np.testing.assert_allclose(v, vr, rtol=0, atol=5e-7)
    if cfg.lc:
        np.testing.assert_allclose(u, ur, rtol=0, atol=5e-7)


@live
@pytest.mark.parametrize("name", ["channel3d", "nematic2d_dipole", "rat3d"])
def test_library_checkpoint_read_by_reference(tmp_path, name):
    """A checkpoint the library makes from a config and particles, read by
    the reference's own readchckpnt."""
    cfg, Q, V, U, sp = _state_after(name)
    ck = gpu.Checkpoint(cfg=cfg)
    ck.set_particles(Q, V, U if cfg.lc else None, sp)
    run = abi.CkptRun(sim_steps=500, warmup_steps=0, runtime=42, warmtime=0, kbtnow=0.97)
    ck.set_run(run)
    for precise in (True, False):
        path = tmp_path / f"lib_{int(precise)}.dat"
        ck.write(path, precise=precise)
        rc, Qr, Vr, Ur, spr, rt, wt, kb, av = Reference.checkpoint_read(path, abi.Config)
        tol = 0 if precise else 5e-7
        assert (rt, wt) == (42, 0) and kb == pytest.approx(0.97, abs=tol)
        np.testing.assert_allclose(Qr, Q, rtol=0, atol=tol)
        np.testing.assert_allclose(Vr, V, rtol=0, atol=tol)
        if cfg.lc:
            np.testing.assert_allclose(Ur, U, rtol=0, atol=tol)
        np.testing.assert_array_equal(spr, sp)
        assert (rc.dim, list(rc.L), rc.coll_op, rc.lc, rc.n_walls, rc.n_species) == \
            (cfg.dim, list(cfg.L), cfg.coll_op, cfg.lc, cfg.n_walls, cfg.n_species)
        assert rc.rot_ang == pytest.approx(cfg.rot_ang, abs=tol)
        assert rc.dt == cfg.dt and rc.kbt == cfg.kbt and rc.seed == cfg.seed
        assert (rc.fricco, rc.relax) == (cfg.fricco, cfg.relax)
        for w in range(cfg.n_walls):
            a, b = rc.walls[w], cfg.walls[w]
            assert list(a.A) == list(b.A) and list(a.Q) == list(b.Q)
            assert (a.DN, a.MVN, a.MVT, a.inv, a.phantom, a.coll_type) == \
                (b.DN, b.MVN, b.MVT, b.inv, b.phantom, b.coll_type)
        for s in range(cfg.n_species):
            assert rc.species[s].mass == cfg.species[s].mass
            assert rc.species[s].act == pytest.approx(cfg.species[s].act, abs=tol)
        # and the library reads back what it wrote
        back = gpu.Checkpoint(path)
        c2 = back.config()
        assert c2.rot_ang == pytest.approx(cfg.rot_ang, abs=tol)
        assert (c2.fricco, c2.relax) == (cfg.fricco, cfg.relax)
        q2, v2, _, sp2 = back.particles()
        np.testing.assert_allclose(q2, Q, rtol=0, atol=tol)
        np.testing.assert_array_equal(sp2, sp)


def test_checkpoint_species_populations_follow_particles(tmp_path):
    two = W.base_config(3, (4, 4, 4), coll_op=abi.COLL_MPCAT,
                        species=[W._species(1.0), W._species(2.0)])
    ck = gpu.Checkpoint(cfg=two)
    n = 300
    rng = np.random.default_rng(5)
    sp = (rng.random(n) < 0.3).astype(np.int32)
    ck.set_particles(rng.random((n, 3)) * 4, rng.standard_normal((n, 3)), None, sp)
    path = tmp_path / "two.dat"
    ck.write(path)
    lines = path.read_text().splitlines()
    assert lines[10].split() == [str(n), "2"]  # GPOP NSPECI
    # each species' first line holds MASS POP ...
    pops = [int(lines[21 + 3 * s].split()[1]) for s in range(2)]
    assert pops == [int((sp == 0).sum()), int((sp == 1).sum())]
    with pytest.raises(gpu.MPCDError):
        ck.set_particles(np.zeros((2, 3)), np.zeros((2, 3)), None, np.array([0, 2]))


def _edit(path, line, field, value):
    lines = path.read_text().splitlines(keepends=True)
    toks = lines[line].split()
    toks[field] = value
    lines[line] = " ".join(toks) + "\n"
    path.write_text("".join(lines))


@pytest.mark.parametrize("line,field,value", [
    (4, 3, "1"),            # TSTECH: a thermostat
    (9, 0, "1"),            # MD coupling
    (6, 0, "1"),            # noHI
    (8, 2, "0.500000"),     # magnetic field
    (4, 4, "5"),            # another collision operator
])
def test_unsupported_runs_are_reported(tmp_path, line, field, value):
    path = _golden_file(tmp_path)
    _edit(path, line, field, value)
    ck = gpu.Checkpoint(path)  # the file itself still reads
    with pytest.raises(gpu.MPCDError, match=r"-2 "):
        ck.config()


def test_moving_wall_is_reported(tmp_path):
    path = _golden_file(tmp_path)
    ck = gpu.Checkpoint(path)
    nbc_line = 21 + 3 * 1 + 1  # one species: 3 lines, then GnDNST
    lines = path.read_text().splitlines()
    assert int(lines[nbc_line].split()[0]) == ck.config().n_walls
    _edit(path, nbc_line + 1, 6, "0.100000")  # first wall's V[0]
    with pytest.raises(gpu.MPCDError, match=r"-2 "):
        gpu.Checkpoint(path).config()


def test_truncated_or_malformed_files_are_rejected(tmp_path):
    src = _golden_file(tmp_path)
    data = src.read_bytes()
    cut = tmp_path / "cut.dat"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(gpu.MPCDError, match=r"-1 "):
        gpu.Checkpoint(cut)
    bad = tmp_path / "bad.dat"
    bad.write_bytes(data.replace(b"\n", b" x\n", 1))
    with pytest.raises(gpu.MPCDError, match=r"-1 "):
        gpu.Checkpoint(bad)
    with pytest.raises(gpu.MPCDError, match=r"-1 "):
        gpu.Checkpoint(tmp_path / "missing.dat")


def test_operator_parameters_travel_in_checkpoints(tmp_path):
    """FRICCO (Langevin operators) and TAU (RELAX of the Vicsek-aligned
    operators) are written where the reference's checkpoint keeps them and
    read back, with the operator."""
    cfg = W.base_config(3, (4, 4, 4), coll_op=abi.COLL_VICSEK_LANG, fricco=0.75, relax=0.25,
                        species=[W._species(mass=1.0, act=0.5)])
    Q, V, U, sp = W.synthetic_state(cfg, 3, seed=7)
    ck = gpu.Checkpoint(cfg=cfg)
    ck.set_particles(Q, V, None, sp)
    path = tmp_path / "ops.dat"
    ck.write(path, precise=True)
    c2 = gpu.Checkpoint(path).config()
    assert (c2.coll_op, c2.fricco, c2.relax) == (abi.COLL_VICSEK_LANG, 0.75, 0.25)
    assert c2.species[0].act == 0.5
