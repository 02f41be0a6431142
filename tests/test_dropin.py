"""The drop-in on the reference program itself: oracle/_ref/mpcd_dropin is the
reference's own executable (its main(), JSON reader, initialisation and
output writers, built from its sources) with timestep() answered by
libmpcd_gpu.so (oracle/ref/dropin_timestep.c).  The runs read a JSON input
in the reference's format and are checked through the reference's own output
file avVel.dat (pout.c:1590, one row per avVelOut steps: t, the centre-of-mass
velocity AVNOW, KBTNOW and the mean velocity gradient).

Skipped where oracle/_ref was not built (it needs the reference sources)."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "mpcd_dropin")
HEADER_LINES = 13  # the reference's banner and column names above the rows

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/mpcd_dropin not built")


def run(tmp_path, name, inp, env=None):
    d = tmp_path / name
    (d / "out").mkdir(parents=True)
    (d / "in.json").write_text(json.dumps(inp, indent=1))
    e = dict(os.environ)
    e.update(env or {})
    p = subprocess.run([EXE, "-i", str(d / "in.json"), "-o", str(d / "out") + "/"],
                       cwd=d, env=e, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    lines = (d / "out" / "avVel.dat").read_text().splitlines()
    assert lines[HEADER_LINES - 1].split()[:5] == ["t", "VcmX", "VcmY", "VcmZ", "KBT"]
    rows = np.array([[float(x) for x in ln.split()] for ln in lines[HEADER_LINES:] if ln.strip()])
    return p, rows


# a fixed "seed" (read.c:1114): 0 would seed the reference's generator, and so
# its initial state and the GPU's draws, from the clock
def periodic2d(steps=100, coll=2, L=(24, 24), dens=20, seed=4711):
    return {"domain": list(L), "simSteps": steps, "collOp": coll, "seed": seed,
            "species": [{"dens": dens}],
            "domainWalls": 1, "checkpointOut": 0, "avVelOut": 10, "energyOut": 10}


def srd3d(steps=100, L=(12, 12, 12), dens=10, seed=4712):
    return {"domain": list(L), "simSteps": steps, "collOp": 0, "rotAng": 2.2689280, "seed": seed,
            "species": [{"dens": dens}], "domainWalls": 1, "checkpointOut": 0, "avVelOut": 10}


def channel2d(steps=400, L=(60, 20), g=0.003, seed=4713):
    def wall(q, a, phantom, dn, mv):
        return {"phantom": phantom, "Q": q, "aInv": a, "P": [1, 1, 1, 1], "R": 0,
                "DN": dn, "MVN": mv, "MVT": mv}
    return {"domain": list(L), "simSteps": steps, "collOp": 2, "grav": [g, 0, 0], "seed": seed,
            "species": [{"dens": 20}], "checkpointOut": 0, "avVelOut": 20,
            "BC": [wall([0, 0, 0], [1, 0, 0], 0, L[0], 1),
                   wall([L[0], 0, 0], [-1, 0, 0], 0, L[0], 1),
                   wall([0, 0, 0], [0, 1, 0], 1, 0, -1),
                   wall([0, L[1], 0], [0, -1, 0], 1, 0, -1)]}


def test_reference_path_without_gpu_library(tmp_path):
    """With the GPU path switched off (or no GPU) the executable is the
    reference program: its own timestep runs and its writers see the state."""
    p, rows = run(tmp_path, "off", periodic2d(steps=40), env={"MPCD_DROPIN_OFF": "1"})
    assert "dropin: solvent timestep on the GPU" not in p.stderr
    assert len(rows) == 5
    assert np.all(np.abs(rows[:, 4] - 1.0) < 0.1)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dropin_mpcat_periodic(tmp_path, prec):
    """2D MPC-AT (collOp 2) in a periodic box: every collision draws the cell's
    velocities from the thermostat, so KBT stays at kT = 1 within the
    equipartition noise of 11,520 particles."""
    p, rows = run(tmp_path, prec, periodic2d(), env={"MPCD_DROPIN_PRECISION": prec})
    assert f"dropin: solvent timestep on the GPU ({prec}" in p.stderr
    assert len(rows) == 11
    assert np.all(np.abs(rows[:, 4] - 1.0) < 0.05)
    assert abs(rows[:, 4].mean() - 1.0) < 0.02


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dropin_srd_conserves_energy(tmp_path, prec):
    """3D random-axis SRD (collOp 0, 130 degrees) in a periodic box conserves
    kinetic energy: every row of avVel.dat keeps the KBT of the first to the
    printed 6 digits (FP64) or to 1e-4 (FP32 velocities)."""
    p, rows = run(tmp_path, prec, srd3d(), env={"MPCD_DROPIN_PRECISION": prec})
    assert f"dropin: solvent timestep on the GPU ({prec}" in p.stderr
    tol = 2e-5 if prec == "fp64" else 1e-4
    assert np.all(np.abs(rows[:, 4] - rows[0, 4]) < tol), rows[:, 4]


@pytest.mark.gpu
def test_dropin_downloads_only_for_output(tmp_path):
    """The particles come back to the host only on output and checkpoint
    steps; the device state evolves the same whether or not they do, so the
    reference's writers produce the same files as with a download on every
    step (MPCD_DROPIN_SYNC)."""
    inp = periodic2d(steps=60)
    run(tmp_path, "sparse", inp, env={"MPCD_DROPIN_PRECISION": "mixed"})
    run(tmp_path, "sync", inp, env={"MPCD_DROPIN_PRECISION": "mixed", "MPCD_DROPIN_SYNC": "1"})
    for f in ("avVel.dat", "energy.dat"):
        a = (tmp_path / "sparse" / "out" / f).read_text()
        b = (tmp_path / "sync" / "out" / f).read_text()
        assert a == b, f


@pytest.mark.gpu
def test_dropin_channel_matches_reference_run(tmp_path):
    """2D gravity-driven channel between phantom no-slip walls (the layout of
    the reference's channelFlow sample, smaller): the GPU run and the
    reference's own run of the same input (different random streams) agree on
    the centre-of-mass velocity the flow reaches, to its thermal noise."""
    pg, g = run(tmp_path, "gpu", channel2d())
    assert "dropin: solvent timestep on the GPU (fp64" in pg.stderr
    _, r = run(tmp_path, "ref", channel2d(), env={"MPCD_DROPIN_OFF": "1"})
    assert g.shape == r.shape
    late = slice(len(g) // 2, None)
    assert g[late, 1].mean() > 0.02  # the flow is driven along x
    np.testing.assert_allclose(g[late, 1].mean(), r[late, 1].mean(), atol=0.025)
    np.testing.assert_allclose(g[late, 4].mean(), r[late, 4].mean(), atol=0.02)


def nematic2d(steps=400, L=(24, 24), seed=4714, act=0.0):
    """2D nematic with the local Maier-Saupe collision and dipole activity
    (collOp 16, lc 1); passive for act = 0.  The orientations start random
    (oDist 0, RANDORIENT, init.c:1310; the reference's default is 2, aligned
    along y); the director field and the local order parameter of every cell
    are written every 50 steps (dirSOut: directorfield.dat, pout.c:2021)."""
    return {"domain": list(L), "simSteps": steps, "collOp": 16, "lc": 1, "seed": seed,
            "species": [{"dens": 20, "act": act, "oDist": 0}], "domainWalls": 1,
            "checkpointOut": 0, "avVelOut": 10, "dirSOut": 50}


def local_order(path):
    """Mean over the cells of the local scalar order parameter S per output
    time of directorfield.dat (rows: t, i, j, k, DIR[3], S)."""
    by_t = {}
    for ln in path.read_text().splitlines():
        f = ln.split()
        if len(f) != 8:
            continue
        try:
            t, S = float(f[0]), float(f[7])
        except ValueError:
            continue
        by_t.setdefault(t, []).append(S)
    return np.array([np.mean(by_t[t]) for t in sorted(by_t)])


@pytest.mark.gpu
def test_dropin_nematic_carries_orientations(tmp_path):
    """The reference's own program runs a 2D nematic with the GPU timestep:
    the orientations cross the binding in both directions (the strided
    calls' off_U), and the reference's own localPROP/tensOrderParam computes
    each cell's order parameter from the downloaded orientations.  The mean
    local order starts low from the random initial orientations (every
    mesogen starting at (1, 0) would give S = 1), rises to the nematic's
    local order, and matches the reference's own run of the same input
    (different random streams) to its noise."""
    pg, _ = run(tmp_path, "gpu", nematic2d())
    assert "dropin: solvent timestep on the GPU (fp64" in pg.stderr
    _, _ = run(tmp_path, "ref", nematic2d(), env={"MPCD_DROPIN_OFF": "1"})
    g = local_order(tmp_path / "gpu" / "out" / "directorfield.dat")
    r = local_order(tmp_path / "ref" / "out" / "directorfield.dat")
    assert g.shape == r.shape and len(g) >= 8
    assert g[0] < 0.5 and r[0] < 0.5
    assert g[-3:].mean() > g[0] + 0.2  # the nematic orders locally
    np.testing.assert_allclose(g[-3:].mean(), r[-3:].mean(), atol=0.03)
