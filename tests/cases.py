"""Small parity cases: each is a workload of the benchmark configurations at
a size the CPU checkers finish in seconds."""
import math

from mpcd_b200 import abi
from mpcd_b200 import workloads as W

# name -> (builder, builder kwargs, particles per cell, state seed, steps)
CASES = {
    "srd3d": (W.cfg_srd3d, dict(L=(6, 5, 4)), 10, 11, 4),
    "srd2d": (W.base_config, dict(dim=2, L=(7, 6), coll_op=abi.COLL_ARBAXIS,
                                  rot_ang=math.radians(130.0)), 10, 12, 4),
    "rat2d": (W.cfg_passive2d, dict(L=(8, 7)), 20, 13, 4),
    "rat3d": (W.base_config, dict(dim=3, L=(5, 5, 4), coll_op=abi.COLL_RAT), 10, 14, 4),
    "mpcat2d": (W.base_config, dict(dim=2, L=(8, 7), coll_op=abi.COLL_MPCAT), 20, 15, 4),
    "mpcat3d_damp": (W.base_config, dict(dim=3, L=(4, 5, 4), coll_op=abi.COLL_MPCAT,
                                         species=[W._species(mass=1.0, damp=0.3)]), 10, 16, 4),
    "channel3d": (W.cfg_channel3d, dict(L=(8, 6, 4), g=1e-2), 20, 17, 4),
    "srd3d_heavy": (W.cfg_srd3d, dict(L=(4, 4, 4), species=[W._species(mass=2.5)],
                                      kbt=1.7, dt=0.25), 10, 18, 4),
    "nematic2d_dipole": (W.cfg_nematic2d, dict(L=(8, 7), coll_op=16), 20, 19, 4),
    "nematic2d_av": (W.cfg_nematic2d, dict(L=(7, 6), coll_op=17), 20, 20, 4),
    "nematic2d_rat": (W.cfg_nematic2d, dict(L=(6, 8), coll_op=3), 20, 21, 4),
}


def build(name, precision=abi.PREC_FP64, seed=777):
    builder, kw, ppc, sseed, nsteps = CASES[name]
    kw = dict(kw)
    cfg = builder(**kw, precision=precision, seed=seed)
    return cfg, ppc, sseed, nsteps


def state(cfg, ppc, sseed):
    return W.synthetic_state(cfg, ppc, seed=sseed)
