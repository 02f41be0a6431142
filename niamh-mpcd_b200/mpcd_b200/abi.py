"""ctypes mirror of include/mpcd_gpu.h (the C ABI of libmpcd_gpu.so).

The structures below must match the C header field for field; a CPU test
checks their sizes against the compiled library's own sizeof().
"""
import ctypes as C

ABI_VERSION = 4

MAX_SPECIES = 10
MAX_WALLS = 16

OK = 0
ERR_ARG = -1
ERR_UNSUPPORTED = -2
ERR_CUDA = -3
ERR_NOMEM = -4
ERR_STATE = -5
ERR_SIZE = -6

COLL_ARBAXIS = 0
COLL_ORTHAXIS = 1
COLL_VICSEK = 7
COLL_CHATE = 8
COLL_MPCAT = 2
COLL_LANG = 4
COLL_RAT = 3
COLL_ACT_ARBAXIS = 9
COLL_ACT_ORTHAXIS = 10
COLL_VICSEK_MPCAT = 11
COLL_VICSEK_LANG = 12
COLL_CHATE_MPCAT = 13
COLL_DIPOLE_DIR_SUM = 16
COLL_DIPOLE_DIR_AV = 17

LC_ISOTROPIC = 0
LC_LOCAL = 1

PREC_FP64 = 0
PREC_MIXED = 1

KERNEL_AUTO = 0
KERNEL_TILE = 1
KERNEL_GROUP = 2
KERNEL_SPLIT = 3
KERNEL_RESIDENT = 4
KERNEL_PERSIST = 5

STRATEGY_SCATTER = 0
STRATEGY_RECOMPUTE = 1

ERRORS = {
    ERR_ARG: "bad argument",
    ERR_UNSUPPORTED: "unsupported option",
    ERR_CUDA: "CUDA error",
    ERR_NOMEM: "device allocation failed",
    ERR_STATE: "call out of order",
    ERR_SIZE: "size above compiled-in maximum",
}


class Species(C.Structure):
    _fields_ = [
        ("mass", C.c_double),
        ("damp", C.c_double),
        ("rfc", C.c_double),
        ("tumble", C.c_double),
        ("chihi", C.c_double),
        ("act", C.c_double),
        ("mfpot", C.c_double),
        ("sigwidth", C.c_double),
        ("sigpos", C.c_double),
        ("minactratio", C.c_double),
    ]


class Wall(C.Structure):
    _fields_ = [
        ("A", C.c_double * 3),
        ("Q", C.c_double * 3),
        ("R", C.c_double),
        ("inv", C.c_int),
        ("phantom", C.c_int),
        ("coll_type", C.c_int),
        ("pad_", C.c_int),
        ("DN", C.c_double),
        ("DT", C.c_double),
        ("DVN", C.c_double),
        ("DVT", C.c_double),
        ("MVN", C.c_double),
        ("MVT", C.c_double),
        ("DVxyz", C.c_double * 3),
        ("MUN", C.c_double),
        ("MUT", C.c_double),
        ("MUxyz", C.c_double * 3),
        ("DUxyz", C.c_double * 3),
        ("inter", C.c_int * MAX_SPECIES),
    ]


class Config(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("L", C.c_int * 3),
        ("dt", C.c_double),
        ("kbt", C.c_double),
        ("coll_op", C.c_int),
        ("lc", C.c_int),
        ("rot_ang", C.c_double),
        ("galinv", C.c_int),
        ("precision", C.c_int),
        ("grav", C.c_double * 3),
        ("gndnst", C.c_double),
        ("seed", C.c_uint64),
        ("replica", C.c_uint32),
        ("n_species", C.c_int),
        ("species", Species * MAX_SPECIES),
        ("n_walls", C.c_int),
        ("walls", Wall * MAX_WALLS),
        ("capacity", C.c_int),
        ("fricco", C.c_double),
        ("relax", C.c_double),
    ]


class TuneChoice(C.Structure):
    _fields_ = [
        ("kernel", C.c_int),
        ("strategy", C.c_int),
        ("tile_particles", C.c_int),
        ("sort_interval", C.c_int),
        ("us_per_step", C.c_double),
        ("from_cache", C.c_int),
        ("candidates", C.c_int),
    ]


# initial distributions: the reference's vDist / oDist codes
VDIST_RANDVEL = 0
VDIST_HOMO = 2
VDIST_HOMOAXIS = 3
VDIST_GAUSS = 4
ODIST_RANDORIENT = 0
ODIST_ALIGNX = 1
ODIST_ALIGNY = 2
ODIST_ALIGNZ = 3
ODIST_ALIGN45 = 4
ODIST_PLANEZ = 5
ODIST_PLANEY = 6
ODIST_PLANEX = 7
ODIST_ALIGNTR = 8
ODIST_ALIGNDEFECTPAIR = 9


class InitParams(C.Structure):
    _fields_ = [
        ("population", C.c_int * MAX_SPECIES),
        ("vdist", C.c_int * MAX_SPECIES),
        ("odist", C.c_int * MAX_SPECIES),
        ("rframe", C.c_int),
        ("pad_", C.c_int),
    ]


def init_params(population, vdist=VDIST_RANDVEL, odist=ODIST_ALIGNY, rframe=1):
    """InitParams for per-species populations; vdist/odist a code or a
    per-species list (defaults: the reference's JSON defaults vDist 0,
    oDist 2, rFrame 1)."""
    p = InitParams()
    pops = list(population)
    for s, n in enumerate(pops):
        p.population[s] = int(n)
        p.vdist[s] = int(vdist[s] if hasattr(vdist, "__len__") else vdist)
        p.odist[s] = int(odist[s] if hasattr(odist, "__len__") else odist)
    p.rframe = int(rframe)
    return p


class CkptRun(C.Structure):
    _fields_ = [
        ("sim_steps", C.c_int),
        ("warmup_steps", C.c_int),
        ("runtime", C.c_int),
        ("warmtime", C.c_int),
        ("kbtnow", C.c_double),
        ("avv", C.c_double * 3),
        ("avnow", C.c_double * 3),
    ]


class Status(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64),
        ("escaped", C.c_uint64),
        ("bounce_limit", C.c_uint64),
        ("nonfinite", C.c_uint64),
        ("overflow", C.c_uint64),
        ("sync_timeout", C.c_uint64),
    ]


def make_wall(A, Q, R=0.0, *, DN=0.0, MVN=1.0, MVT=1.0, phantom=0, inv=0,
              DT=0.0, DVN=0.0, DVT=0.0, DVxyz=(0, 0, 0), MUN=1.0, MUT=1.0,
              coll_type=1):
    """A planar wall as readJson builds one from a JSON "BC" entry
    (mpcd/subroutines/read.c:1141-1428): A = 1/aInv."""
    w = Wall()
    for d in range(3):
        w.A[d] = A[d]
        w.Q[d] = Q[d]
        w.DVxyz[d] = DVxyz[d]
        w.MUxyz[d] = 1.0
        w.DUxyz[d] = 0.0
    w.R = R
    w.inv = inv
    w.phantom = phantom
    w.coll_type = coll_type
    w.DN, w.DT, w.DVN, w.DVT = DN, DT, DVN, DVT
    w.MVN, w.MVT, w.MUN, w.MUT = MVN, MVT, MUN, MUT
    for s in range(MAX_SPECIES):
        w.inter[s] = 1
    return w


def periodic_walls(dim, L):
    """The 2*dim periodic planes of the 'domainWalls' default
    (read.c:1441-1583 with domainWalls=1): left/right, bottom/top, near/far."""
    walls = []
    for ax in range(dim):
        a_lo = [0.0, 0.0, 0.0]
        a_lo[ax] = 1.0
        a_hi = [0.0, 0.0, 0.0]
        a_hi[ax] = -1.0
        walls.append(make_wall(a_lo, (0, 0, 0), 0.0, DN=float(L[ax])))
        walls.append(make_wall(a_hi, (0, 0, 0), -float(L[ax]), DN=float(L[ax])))
    return walls
