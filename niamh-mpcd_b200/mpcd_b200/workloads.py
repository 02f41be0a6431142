"""Synthetic MPCD workloads of the shapes the benchmark configurations name.

Inputs are generated from a seed (no dataset is involved): positions uniform
in the box, velocities Maxwell-Boltzmann at kT with the net momentum removed,
nematic orientations uniform on the unit circle/sphere.  This mirrors how the
reference initialises a fluid (setcoord/push/orient, init.c:1219-1605) without
reproducing its random sequence.
"""
import math

import numpy as np

from . import abi


def _species(mass=1.0, **kw):
    s = abi.Species()
    s.mass = mass
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def base_config(dim, L, *, coll_op, dt=0.1, kbt=1.0, rot_ang=math.pi / 2,
                lc=0, grav=(0.0, 0.0, 0.0), walls=None, seed=12345,
                precision=abi.PREC_FP64, species=None, gndnst=0.0, galinv=1, fricco=1.0,
                relax=0.5):
    cfg = abi.Config()
    cfg.dim = dim
    for d in range(3):
        cfg.L[d] = int(L[d]) if d < dim else 1
        cfg.grav[d] = float(grav[d])
    cfg.dt = dt
    cfg.kbt = kbt
    cfg.coll_op = coll_op
    cfg.lc = lc
    cfg.rot_ang = rot_ang
    cfg.galinv = galinv
    cfg.precision = precision
    cfg.gndnst = gndnst
    cfg.seed = seed
    cfg.replica = 0
    sp = species if species is not None else [_species()]
    cfg.n_species = len(sp)
    for i, s in enumerate(sp):
        cfg.species[i] = s
    w = walls if walls is not None else abi.periodic_walls(dim, L)
    cfg.n_walls = len(w)
    for i, wl in enumerate(w):
        cfg.walls[i] = wl
    cfg.capacity = 0
    cfg.fricco = fricco
    cfg.relax = relax
    return cfg


def cfg_passive2d(L=(30, 30), **kw):
    """2D passive fluid, MPC-AT+a (collOp 3), periodic (configuration 1)."""
    return base_config(2, L, coll_op=abi.COLL_RAT, **kw)


def cfg_srd3d(L=(64, 64, 64), **kw):
    """3D SRD fluid, random axis, 130 degrees, periodic (configuration 2)."""
    kw.setdefault("rot_ang", math.radians(130.0))
    return base_config(3, L, coll_op=abi.COLL_ARBAXIS, **kw)


def channel_walls(L):
    """Periodic in x and z, no-slip phantom bounce-back walls at y=0 and
    y=L[1] (the sampleInputs/channelFlow BC pattern, in 3D)."""
    w = []
    w.append(abi.make_wall((1, 0, 0), (0, 0, 0), 0.0, DN=float(L[0])))
    w.append(abi.make_wall((-1, 0, 0), (L[0], 0, 0), 0.0, DN=float(L[0])))
    w.append(abi.make_wall((0, 1, 0), (0, 0, 0), 0.0, MVN=-1.0, MVT=-1.0,
                           phantom=1))
    w.append(abi.make_wall((0, -1, 0), (0, L[1], 0), 0.0, MVN=-1.0, MVT=-1.0,
                           phantom=1))
    w.append(abi.make_wall((0, 0, 1), (0, 0, 0), 0.0, DN=float(L[2])))
    w.append(abi.make_wall((0, 0, -1), (0, 0, L[2]), 0.0, DN=float(L[2])))
    return w


def cfg_channel3d(L=(128, 64, 64), g=1e-4, **kw):
    """3D Poiseuille channel, MPC-AT+a, body force along x (configuration 3)."""
    return base_config(3, L, coll_op=abi.COLL_RAT, walls=channel_walls(L),
                       grav=(g, 0.0, 0.0), **kw)


def cfg_nematic2d(L=(256, 256), **kw):
    """2D active nematic, LC collision with dipole activity (configuration 4)."""
    sp = [_species(mass=1.0, rfc=0.01, tumble=0.5, chihi=0.5, act=0.05,
                   mfpot=10.0, sigwidth=0.0, sigpos=0.0, minactratio=0.0)]
    kw.setdefault("coll_op", abi.COLL_DIPOLE_DIR_SUM)
    return base_config(2, L, lc=abi.LC_LOCAL, species=sp, **kw)


def box_size(cfg):
    return [cfg.L[d] for d in range(cfg.dim)]


def synthetic_state(cfg, ppc, seed=2024, dtype=np.float64):
    """Seeded particle state: returns Q, V, U as (n,3) float64 arrays and the
    species ids.  ppc particles per cell on average (n = ppc * volume)."""
    rng = np.random.default_rng(seed)
    dim = cfg.dim
    L = np.array([cfg.L[d] if d < dim else 1 for d in range(3)], dtype=np.float64)
    vol = int(np.prod(L[:dim]))
    n = int(ppc * vol)
    Q = np.zeros((n, 3))
    Q[:, :dim] = rng.random((n, dim)) * L[:dim]
    mass = cfg.species[0].mass
    V = np.zeros((n, 3))
    V[:, :dim] = rng.standard_normal((n, dim)) * math.sqrt(cfg.kbt / mass)
    V[:, :dim] -= V[:, :dim].mean(axis=0)
    U = np.zeros((n, 3))
    if dim == 2:
        th = rng.random(n) * 2 * math.pi
        U[:, 0] = np.cos(th)
        U[:, 1] = np.sin(th)
    else:
        u = rng.standard_normal((n, 3))
        U[:] = u / np.linalg.norm(u, axis=1, keepdims=True)
    spid = np.zeros(n, dtype=np.int32)
    return Q, V, U, spid


def ensemble_sides(nboxes, seed=5000):
    """Side lengths of configuration 5's ensemble: nboxes cubic boxes with
    sides drawn uniformly from {8, 12, 16, 24, 32}, the same on every rank."""
    rng = np.random.default_rng(seed)
    return rng.choice([8, 12, 16, 24, 32], size=nboxes)


def shard_boxes(work, world, rank):
    """The boxes rank `rank` of `world` steps when an ensemble is split
    across GPUs: boxes are independent (no data crosses between them), so
    each goes whole to one rank, the largest first to the least-loaded rank
    (ties to the lower rank), which keeps the ranks' particle counts within
    one box of each other.  Every rank computes the same split from the same
    per-box work (particle counts); returns the rank's box indices in
    ascending order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    load = [0] * world
    owner = [0] * len(work)
    for b in sorted(range(len(work)), key=lambda j: (-int(work[j]), j)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[b] = r
        load[r] += int(work[b])
    return [b for b in range(len(work)) if owner[b] == rank]
