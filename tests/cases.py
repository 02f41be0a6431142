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


def slab_walls(L, ylo, yhi, inverted=False):
    """Periodic box with two solid walls inside it across y, at ylo (normal
    +y) and yhi (normal -y, or +y inverted): the fluid fills ylo < y < yhi,
    so a uniform placement in the box is often rejected."""
    w = list(abi.periodic_walls(3, L))
    w.append(abi.make_wall((0, 1, 0), (0, ylo, 0), 0.0, MVN=-1.0, MVT=-1.0))
    if inverted:
        w.append(abi.make_wall((0, 1, 0), (0, yhi, 0), 0.0, MVN=-1.0, MVT=-1.0, inv=1))
    else:
        w.append(abi.make_wall((0, -1, 0), (0, yhi, 0), 0.0, MVN=-1.0, MVT=-1.0))
    return w


def _two_species_channel(L):
    """Channel of two species (masses 1 and 2.5); species 1 ignores the
    y walls, so the two see different accessible volumes."""
    cfg = W.base_config(3, L, coll_op=abi.COLL_MPCAT,
                        species=[W._species(1.0), W._species(2.5)],
                        walls=slab_walls(L, 1.25, L[1] - 0.5))
    for w in range(cfg.n_walls):
        cfg.walls[w].inter[0] = 1
        cfg.walls[w].inter[1] = 1 if w < cfg.n_walls - 2 else 0
    return cfg


def _nematic_all_odist(L):
    """2D nematic with ten species, species s initialised with oDist s."""
    sp = [W._species(mass=1.0 + 0.25 * s, rfc=0.01, tumble=0.5, chihi=0.5, act=0.05,
                     mfpot=10.0) for s in range(abi.MAX_SPECIES)]
    cfg = W.base_config(2, L, coll_op=abi.COLL_DIPOLE_DIR_SUM, lc=abi.LC_LOCAL, species=sp)
    for w in range(cfg.n_walls):
        for s in range(abi.MAX_SPECIES):
            cfg.walls[w].inter[s] = 1
    return cfg


_VD = (abi.VDIST_RANDVEL, abi.VDIST_HOMO, abi.VDIST_HOMOAXIS, abi.VDIST_GAUSS)

# initial-state cases: name -> (config builder, populations, vdist, odist,
# rframe); every config uses generator key 777
INIT_CASES = {
    "init_srd3d_gauss": (lambda: W.cfg_srd3d((8, 8, 8)), [2560], abi.VDIST_GAUSS, 0, 1),
    "init_srd3d_randvel": (lambda: W.cfg_srd3d((8, 8, 8)), [2560], abi.VDIST_RANDVEL, 0, 0),
    "init_slab_homo": (lambda: W.base_config(3, (10, 12, 8), coll_op=abi.COLL_MPCAT,
                                             walls=slab_walls((10, 12, 8), 1.5, 9.75)),
                       [6000], abi.VDIST_HOMO, 0, 1),
    "init_slab_inv_homoaxis": (lambda: W.base_config(3, (10, 12, 8), coll_op=abi.COLL_RAT,
                                                     walls=slab_walls((10, 12, 8), 2.25, 7.5,
                                                                      True)),
                               [4000], abi.VDIST_HOMOAXIS, 0, 1),
    "init_two_species": (lambda: _two_species_channel((6, 8, 5)), [1500, 900],
                         [abi.VDIST_GAUSS, abi.VDIST_RANDVEL], 0, 1),
    "init_nematic_odist": (lambda: _nematic_all_odist((12, 10)), [60] * abi.MAX_SPECIES,
                           [_VD[s % 4] for s in range(abi.MAX_SPECIES)],
                           list(range(abi.MAX_SPECIES)), 1),
}


def init_case(name, precision=abi.PREC_FP64):
    """(config, InitParams) of an initial-state case."""
    builder, pops, vd, od, rframe = INIT_CASES[name]
    cfg = builder()
    cfg.precision = precision
    cfg.seed = 777
    return cfg, abi.init_params(pops, vdist=vd, odist=od, rframe=rframe)


def thin_gap(op=abi.COLL_ARBAXIS, precision=abi.PREC_FP64, n=400, vy=10.0, seed=99):
    """A 4^3 box, periodic in x and z, whose fluid fills a gap 0.01 wide
    between two no-slip walls across y: particles of |v_y| ~ vy cross it
    about a hundred times in one step, past the reference's bounce limit
    (NBOUNCE, bc.c:1461-1488), so the longer rewinds and then the
    re-thermalisation run.  (Much faster particles rewind out of the box
    and escape, and the reference's escape re-placement then draws from
    its own generator.)  Returns (config, Q, V, species)."""
    import numpy as np
    L = (4, 4, 4)
    w = [abi.make_wall((1, 0, 0), (0, 0, 0), 0.0, DN=4.0),
         abi.make_wall((-1, 0, 0), (4, 0, 0), 0.0, DN=4.0),
         abi.make_wall((0, 0, 1), (0, 0, 0), 0.0, DN=4.0),
         abi.make_wall((0, 0, -1), (0, 0, 4), 0.0, DN=4.0),
         abi.make_wall((0, 1, 0), (0, 1.0, 0), 0.0, MVN=-1.0, MVT=-1.0),
         abi.make_wall((0, -1, 0), (0, 1.01, 0), 0.0, MVN=-1.0, MVT=-1.0)]
    cfg = W.base_config(3, L, coll_op=op, walls=w, seed=seed, precision=precision)
    rng = np.random.default_rng(seed)
    Q = np.zeros((n, 3))
    Q[:, 0] = rng.random(n) * 4
    Q[:, 2] = rng.random(n) * 4
    Q[:, 1] = 1.0005 + rng.random(n) * 0.009
    V = rng.standard_normal((n, 3))
    V[: n // 4, 1] = vy * np.sign(V[: n // 4, 1])
    return cfg, Q, V, np.zeros(n, dtype=np.int32)


def open_bottom(op=abi.COLL_ARBAXIS, precision=abi.PREC_FP64, dim=3, n=600, vy=15.0, seed=7):
    """A box of 6 cells per side, periodic across x (and z in 3D), with a
    no-slip ceiling at y = 4 and no wall below: the fastest particles leave
    through the bottom within a step or two, and the reference's end-of-step
    re-bin re-places them (bin, mpc.c:969-982) at a uniform position that
    no wall excludes (the ceiling rejects y >= 4) with a fresh thermal
    velocity and, for the nematic (2D), orientation.  (A particle that ends
    a step in [-1, 0) is binned to cell 0 by truncation and leaves at a
    later step; none can end one in [L, L + 1), below the ceiling, where the
    reference's shifted bin would re-place it instead.)  Returns (config, Q,
    V, U, species)."""
    import numpy as np
    L = (6, 6, 6)[:dim] + (1,) * (3 - dim)
    w = [abi.make_wall((1, 0, 0), (0, 0, 0), 0.0, DN=6.0),
         abi.make_wall((-1, 0, 0), (6, 0, 0), 0.0, DN=6.0),
         abi.make_wall((0, -1, 0), (0, 4.0, 0), 0.0, MVN=-1.0, MVT=-1.0)]
    if dim == 3:
        w += [abi.make_wall((0, 0, 1), (0, 0, 0), 0.0, DN=6.0),
              abi.make_wall((0, 0, -1), (0, 0, 6), 0.0, DN=6.0)]
    if op == "lc":
        cfg = W.cfg_nematic2d(L=L[:2], walls=w, seed=seed, precision=precision, gndnst=10.0)
    else:
        cfg = W.base_config(dim, L, coll_op=op, walls=w, seed=seed, precision=precision)
    rng = np.random.default_rng(seed)
    Q = np.zeros((n, 3))
    Q[:, 0] = rng.random(n) * 6
    Q[:, 1] = 0.1 + rng.random(n) * 3.8
    if dim == 3:
        Q[:, 2] = rng.random(n) * 6
    V = rng.standard_normal((n, 3))
    V[: n // 4, 1] = -vy
    if dim == 2:
        V[:, 2] = 0.0
    U = None
    if op == "lc":
        a = rng.random(n) * 2 * np.pi
        U = np.stack([np.cos(a), np.sin(a), np.zeros(n)], axis=1)
    return cfg, Q, V, U, np.zeros(n, dtype=np.int32)
