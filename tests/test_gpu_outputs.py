"""Output fields from the device: the end-of-step cell fields, per-species
populations, the flow field's running sum and the kinetic energy, written
through the reference's formats, against the reference's own writers run on
the same trajectory (FP64 form: the state agrees to the parity bound, so the
printed values agree to their last printed digit; mixed form: within FP32
rounding).  The banner and column headers are compared as text."""
import numpy as np
import pytest

from cases import build, init_case, state
from checkers import Oracle, Reference, oracle_init_state
from mpcd_b200 import abi
from mpcd_b200.gpu import FieldWriter, Solver

pytestmark = pytest.mark.gpu

FILES = ["avVel.dat", "coarsegrain.dat", "densityfield.dat", "energy.dat", "flowfield.dat",
         "velfield.dat"]
HEAD = 13  # banner (11 lines and a blank) and the column header


def _load(path):
    lines = path.read_text().splitlines()
    return lines[:HEAD], np.array([[float(x) for x in ln.split()] for ln in lines[HEAD:]])


def _run(tmp_path, cfg, cfg_gpu, Q, V, U, sp, rtol, atol):
    ref_dir, gpu_dir = tmp_path / "ref", tmp_path / "gpu"
    ref_dir.mkdir()
    gpu_dir.mkdir()
    r = Reference(cfg, Q, V, U, sp)
    r.set_flow(True)
    g = Solver(cfg_gpu)
    g.upload(Q, V, U, sp)
    g.flow_enable(True)
    fw = FieldWriter(cfg_gpu, gpu_dir)
    for s in range(1, 7):
        r.step(s)
        kb, _ = g.timestep(s)
        if s % 3 == 0:
            r.write_outputs(ref_dir, s, 3, header=(s == 3))
            fw.write_from(g, s * cfg.dt, kb, flow_interval=3)
    for f in FILES:
        hr, ar = _load(ref_dir / f)
        hg, ag = _load(gpu_dir / f)
        assert hr == hg, f
        assert ar.shape == ag.shape, f
        np.testing.assert_allclose(ag, ar, rtol=rtol, atol=atol, err_msg=f)
    g.close()


@pytest.mark.parametrize("name", ["srd3d", "channel3d", "rat2d"])
def test_fp64_outputs_match_reference_writers(tmp_path, name):
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    # printed with 6 significant digits: one unit in the last place
    _run(tmp_path, cfg, cfg, Q, V, U, sp, rtol=2e-5, atol=1e-9)


@pytest.mark.parametrize("name", ["srd3d", "channel3d"])
def test_mixed_outputs_track_reference_writers(tmp_path, name):
    cfg, ppc, sseed, _ = build(name)
    cfgm, _, _, _ = build(name, precision=abi.PREC_MIXED)
    Q, V, U, sp = state(cfg, ppc, sseed)
    _run(tmp_path, cfg, cfgm, Q, V, U, sp, rtol=1e-3, atol=1e-5)


def test_species_counts_flow_sum_and_kinetic_energy_against_oracle():
    cfg, params = init_case("init_two_species")
    Q, V, _, sp, _ = oracle_init_state(cfg, params)
    o = Oracle(cfg, Q, V, None, sp)
    g = Solver(cfg)
    g.upload(Q, V, None, sp)
    g.flow_enable(True)
    flow = None
    for s in range(1, 5):
        o.step(s)
        g.step(1, s)
        _, _, vcm, _ = o.cells()
        flow = vcm if flow is None else flow + vcm
    f, k = g.flow_read()
    assert k == 4
    np.testing.assert_allclose(f, flow, rtol=0, atol=1e-11)
    q, v, _ = o.particles()
    L = [cfg.L[d] + 1 for d in range(3)]
    idx = np.clip(q.astype(int), 0, np.array(cfg.L[:3]))
    lin = (idx[:, 0] * L[1] + idx[:, 1]) * L[2] + idx[:, 2]
    want = np.zeros((2, L[0] * L[1] * L[2]), dtype=np.int32)
    np.add.at(want, (sp, lin), 1)
    np.testing.assert_array_equal(g.cell_species(), want)
    m = np.array([cfg.species[i].mass for i in sp])
    assert g.kinetic_energy() == pytest.approx(0.5 * np.sum(m * np.sum(v * v, axis=1)),
                                               rel=1e-10)
    f, _ = g.flow_read(reset=True)
    f, k = g.flow_read()
    assert k == 0 and not f.any()
    g.close()
