"""Generates tests/golden/*.npz from the reference's own timestep.

The reference (NIAMH-MPCD) is built from its sources into oracle/_ref/ with
the draw-injecting harness (oracle/ref/ref_harness.c), fed the seeded state of
each case in tests/cases.py, and stepped; positions, velocities, the step's
global measures and the cell populations after every step are stored.

Initial-state cases (INIT_CASES): the reference's own initialisation
(setcoord, galileantrans, the VSC scaling) with the injected draws, and its
Monte Carlo accessible volume per species with its own generator.

"checkpoint": the reference's own checkpoint file (checkpoint(),
pout.c:2325-2396) of the rat2d case after three steps.

    make -C oracle/ref REF=$MPCD_REFERENCE_DIR && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "niamh-mpcd_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

from cases import CASES, INIT_CASES, build, init_case, state  # noqa: E402
from checkers import Reference  # noqa: E402


def make_init(name):
    cfg, params = init_case(name)
    ref, Q, V, U, sp, kbt = Reference.from_init(cfg, params)
    assert ref.unexpected_draws() == 0, name
    out = {"Q": Q, "V": V, "U": U, "spid": sp, "kbt": kbt}
    out["volume_mc"] = np.array([Reference.accessible_volume(cfg, s)
                                 for s in range(cfg.n_species)])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, len(Q), "particles")


def make_checkpoint(name="rat2d", steps=3):
    """The reference's own checkpoint() of a golden case after a few steps,
    gzip-compressed."""
    import gzip
    import tempfile
    cfg, ppc, sseed, _ = build(name)
    Q, V, U, sp = state(cfg, ppc, sseed)
    ref = Reference(cfg, Q, V, U, sp)
    for s in range(1, steps + 1):
        ref.step(s)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ckpt.dat")
        ref.checkpoint_write(path, steps, 0)
        with open(path, "rb") as f:
            data = f.read()
    with gzip.GzipFile(os.path.join(HERE, f"ckpt_{name}.dat.gz"), "wb", mtime=0) as g:
        g.write(data)
    print("checkpoint", name, len(data), "bytes")


def main(names=None):
    for name in (names or list(CASES) + list(INIT_CASES) + ["checkpoint"]):
        if name == "checkpoint":
            make_checkpoint()
            continue
        if name in INIT_CASES:
            make_init(name)
            continue
        cfg, ppc, sseed, nsteps = build(name)
        Q, V, U, sp = state(cfg, ppc, sseed)
        ref = Reference(cfg, Q, V, U, sp)
        out = {"Q0": Q, "V0": V, "U0": U, "gndnst": ref.gndnst()}
        for s in range(1, nsteps + 1):
            ref.step(s)
            q, v, u = ref.particles()
            if cfg.lc:
                out[f"U{s}"] = u
            kb, av = ref.globals()
            pop, _, _, _ = ref.cells()
            out[f"Q{s}"] = q
            out[f"V{s}"] = v
            out[f"kbt{s}"] = kb
            out[f"av{s}"] = av
            out[f"pop{s}"] = pop
        assert ref.unexpected_draws() == 0, name
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, len(Q), "particles,", nsteps, "steps")


if __name__ == "__main__":
    main(sys.argv[1:] or None)
