"""Generates tests/golden/*.npz from the reference's own timestep.

The reference (NIAMH-MPCD) is built from its sources into oracle/_ref/ with
the draw-injecting harness (oracle/ref/ref_harness.c), fed the seeded state of
each case in tests/cases.py, and stepped; positions, velocities, the step's
global measures and the cell populations after every step are stored.

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

from cases import CASES, build, state  # noqa: E402
from checkers import Reference  # noqa: E402


def main(names=None):
    for name in (names or CASES):
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
