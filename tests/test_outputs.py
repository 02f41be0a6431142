"""The reference's output files of the cell fields and global measures
(coarsegrain, velfield, densityfield, flowfield, avVel, energy .dat) written
by the library's host writers from the reference's own arrays are the
reference's own writers' files byte for byte, over two output steps."""
import filecmp
import os

import numpy as np
import pytest

from cases import build, init_case, state
from checkers import Reference, oracle_init_state
from mpcd_b200 import gpu

pytestmark = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")

FILES = ["avVel.dat", "coarsegrain.dat", "densityfield.dat", "energy.dat", "flowfield.dat",
         "velfield.dat"]


def _kinetic(cfg, V, sp):
    """enout's MPCD_kin in its own order (pout.c:1393-1399)."""
    ke = 0.0
    for i in range(len(V)):
        e = 0.0
        for d in range(cfg.dim):
            e += V[i, d] * V[i, d]
        ke += e * 0.5 * cfg.species[int(sp[i])].mass
    return ke


def _compare(tmp_path, cfg, Q, V, U, sp, every=3, nsteps=6):
    ref_dir, lib_dir = tmp_path / "ref", tmp_path / "lib"
    ref_dir.mkdir()
    lib_dir.mkdir()
    r = Reference(cfg, Q, V, U, sp)
    r.set_flow(True)
    fw = gpu.FieldWriter(cfg, lib_dir)
    nsum = 0
    for s in range(1, nsteps + 1):
        r.step(s)
        nsum += 1
        if s % every:
            continue
        flow = r.flow()
        pop, mass, vcm, _ = r.cells()
        spc = r.cell_species() if cfg.n_species > 1 else None
        kb, _ = r.globals()
        _, v, _ = r.particles()
        fw.write(s * cfg.dt, pop, mass, vcm, spc, kb, _kinetic(cfg, v, sp), flow, nsum)
        r.write_outputs(ref_dir, s, nsum, header=(s == every))
        nsum = 0
    for f in FILES:
        assert filecmp.cmp(ref_dir / f, lib_dir / f, shallow=False), f


@pytest.mark.parametrize("name", ["srd3d", "channel3d", "rat2d", "mpcat3d_damp"])
def test_output_files_match_reference_writers(tmp_path, name):
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    _compare(tmp_path, cfg, Q, V, U, sp)


def test_output_files_two_species(tmp_path):
    cfg, params = init_case("init_two_species")
    Q, V, _, sp, _ = oracle_init_state(cfg, params)
    _compare(tmp_path, cfg, Q, V, None, sp)


@pytest.mark.parametrize("name", ["srd2d", "srd3d"])
def test_velocity_gradient_of_a_linear_shear(name):
    """v_x = a y: every bulk cell's dv_x/dy is a (the stencil is exact on a
    linear field), the edges copy it, so the box mean is a; repeated calls
    give the same."""
    import ctypes as C
    cfg, _, _, _ = build(name)
    N1 = [cfg.L[d] + 1 if d < cfg.dim else 2 for d in range(3)]
    a = 0.0375
    y = np.arange(N1[1], dtype=float)
    vcm = np.zeros((N1[0], N1[1], N1[2], 3))
    vcm[..., 0] = a * y[None, :, None]
    vcm = vcm.reshape(-1, 3).copy()
    E = np.zeros(9 * len(vcm))
    g1, g2 = np.zeros(9), np.zeros(9)
    lib = gpu.load()
    p = lambda x: x.ctypes.data_as(C.c_void_p)
    assert lib.mpcd_vel_grad(C.byref(cfg), p(vcm), p(E), p(g1)) == 0
    assert lib.mpcd_vel_grad(C.byref(cfg), p(vcm), p(E), p(g2)) == 0
    np.testing.assert_array_equal(g1, g2)
    want = np.zeros(9)
    want[1] = a
    np.testing.assert_allclose(g1, want, rtol=0, atol=1e-15)
