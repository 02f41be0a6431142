"""TEST INFRASTRUCTURE ONLY: ctypes wrappers of the CPU checkers.

- Oracle: oracle/libmpcd_oracle.so, the plain-C restatement of the reference
  solvent timestep (oracle/mpcd_oracle.c).
- Reference: oracle/_ref/libmpcdref.so, the reference's own timestep built
  from its sources with injected counter-based draws
  (oracle/ref/ref_harness.c); libmpcdref_time.so is the same with the
  reference's own Mersenne-Twister generator, for timing.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, never by the product.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libmpcd_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmpcdref.so")
REF_TIME_LIB = os.path.join(HERE, "_ref", "libmpcdref_time.so")


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """CPU restatement of the reference timestep."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(ORACLE_LIB)
            lib.oracle_create.restype = C.c_void_p
            lib.oracle_create.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 4
            lib.oracle_destroy.argtypes = [C.c_void_p]
            lib.oracle_step.argtypes = [C.c_void_p, C.c_uint32]
            lib.oracle_get_particles.argtypes = [C.c_void_p] * 4
            lib.oracle_get_globals.argtypes = [C.c_void_p] * 3
            lib.oracle_get_cells.argtypes = [C.c_void_p] * 5
            lib.oracle_gndnst.restype = C.c_double
            lib.oracle_gndnst.argtypes = [C.c_void_p]
            lib.oracle_ncells.argtypes = [C.c_void_p]
            lib.oracle_escaped.restype = C.c_long
            lib.oracle_escaped.argtypes = [C.c_void_p]
            lib.oracle_shifted_counts.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
            lib.oracle_init_state.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + \
                [C.c_void_p] * 5
            lib.oracle_bounce_limit.restype = C.c_long
            lib.oracle_bounce_limit.argtypes = [C.c_void_p]
            lib.oracle_set_vdist.argtypes = [C.c_void_p, C.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, cfg, Q, V, U=None, spid=None):
        self.cfg = cfg
        lib = self.lib()
        self.n = len(Q)
        Q, V = _f64(Q), _f64(V)
        U = None if U is None else _f64(U)
        spid = None if spid is None else np.ascontiguousarray(spid, dtype=np.int32)
        self.h = lib.oracle_create(C.byref(cfg), self.n, _p(Q), _p(V), _p(U), _p(spid))
        if not self.h:
            raise RuntimeError("oracle_create failed")

    def step(self, step):
        r = self.lib().oracle_step(self.h, step)
        if r != 0:
            raise RuntimeError(f"oracle_step returned {r}")

    def particles(self):
        Q = np.zeros((self.n, 3))
        V = np.zeros((self.n, 3))
        U = np.zeros((self.n, 3))
        self.lib().oracle_get_particles(self.h, _p(Q), _p(V), _p(U))
        return Q, V, U

    def globals(self):
        kb = C.c_double()
        av = np.zeros(3)
        self.lib().oracle_get_globals(self.h, C.byref(kb), _p(av))
        return kb.value, av

    def cells(self):
        nc = self.lib().oracle_ncells(self.h)
        pop = np.zeros(nc, dtype=np.int32)
        mass = np.zeros(nc)
        vcm = np.zeros((nc, 3))
        cm = np.zeros((nc, 3))
        self.lib().oracle_get_cells(self.h, _p(pop), _p(mass), _p(vcm), _p(cm))
        return pop, mass, vcm, cm

    def gndnst(self):
        return self.lib().oracle_gndnst(self.h)

    def shifted_counts(self, step):
        """Populations of the cells of step `step`'s shifted grid from the
        current positions (the cell lists that step collides)."""
        nc = self.lib().oracle_ncells(self.h)
        pop = np.zeros(nc, dtype=np.int32)
        self.lib().oracle_shifted_counts(self.h, step, _p(pop))
        return pop

    def escaped(self):
        return self.lib().oracle_escaped(self.h)

    def bounce_limit(self):
        """Particles that exceeded the bounce limit (summed over steps)."""
        return self.lib().oracle_bounce_limit(self.h)

    def set_vdist(self, vdist):
        v = np.zeros(10, dtype=np.int32)
        v[:len(vdist)] = vdist
        self.lib().oracle_set_vdist(self.h, _p(v))

    def close(self):
        if self.h:
            self.lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def oracle_init_state(cfg, params, max_attempts=1 << 22):
    """The oracle's initial state (oracle_init_state): Q, V, U (n x 3), spid
    and TEMP after the scaling."""
    n = sum(params.population)
    Q, V, U = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    sp = np.zeros(n, dtype=np.int32)
    kb = C.c_double()
    r = Oracle.lib().oracle_init_state(C.byref(cfg), C.byref(params), max_attempts, _p(Q),
                                       _p(V), _p(U), _p(sp), C.byref(kb))
    if r != 0:
        raise RuntimeError("oracle_init_state failed")
    return Q, V, U, sp, kb.value


class Reference:
    """The reference's own timestep (process-global state: one at a time)."""

    _libs = {}

    @classmethod
    def available(cls, timing=False):
        return os.path.exists(REF_TIME_LIB if timing else REF_LIB)

    @classmethod
    def lib(cls, timing=False):
        path = REF_TIME_LIB if timing else REF_LIB
        if path not in cls._libs:
            lib = C.CDLL(path)
            lib.ref_init.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 4
            lib.ref_step.argtypes = [C.c_uint32]
            lib.ref_run_timed.restype = C.c_double
            lib.ref_run_timed.argtypes = [C.c_int, C.c_uint32]
            lib.ref_get_particles.argtypes = [C.c_void_p] * 3
            lib.ref_get_globals.argtypes = [C.c_void_p] * 2
            lib.ref_get_cells.argtypes = [C.c_void_p] * 4
            lib.ref_gndnst.restype = C.c_double
            lib.ref_unexpected_draws.restype = C.c_long
            lib.ref_theory_visc.restype = C.c_double
            lib.ref_init_state.argtypes = [C.c_void_p] * 7
            lib.ref_accessible_volume.restype = C.c_double
            lib.ref_accessible_volume.argtypes = [C.c_int]
            lib.ref_checkpoint_write.argtypes = [C.c_char_p, C.c_int, C.c_int]
            lib.ref_checkpoint_read.argtypes = [C.c_char_p] + [C.c_void_p] * 6
            lib.ref_checkpoint_particles.argtypes = [C.c_void_p] * 4
            lib.ref_set_flow.argtypes = [C.c_int]
            lib.ref_set_vdist.argtypes = [C.c_void_p]
            lib.ref_get_flow.argtypes = [C.c_void_p]
            lib.ref_get_cell_species.argtypes = [C.c_void_p]
            lib.ref_write_outputs.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int]
            lib.ref_theory_visc.argtypes = [C.c_int, C.c_int] + [C.c_double] * 5 + \
                [C.c_void_p, C.c_void_p]
            cls._libs[path] = lib
        return cls._libs[path]

    def __init__(self, cfg, Q, V, U=None, spid=None, timing=False):
        self.cfg = cfg
        self.n = len(Q)
        self._lib = self.lib(timing)
        Q, V = _f64(Q), _f64(V)
        U = None if U is None else _f64(U)
        spid = None if spid is None else np.ascontiguousarray(spid, dtype=np.int32)
        r = self._lib.ref_init(C.byref(cfg), self.n, _p(Q), _p(V), _p(U), _p(spid))
        if r != 0:
            raise RuntimeError("ref_init failed")

    @classmethod
    def from_init(cls, cfg, params, timing=False):
        """The reference's own initialisation (setcoord, galileantrans, the
        VSC scaling) through ref_init_state; returns the Reference, which can
        step on from there, and the arrays Q, V, U, spid and TEMP after the
        scaling."""
        self = cls.__new__(cls)
        self.cfg = cfg
        self.n = n = sum(params.population)
        self._lib = cls.lib(timing)
        Q, V, U = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        sp = np.zeros(n, dtype=np.int32)
        kb = C.c_double()
        r = self._lib.ref_init_state(C.byref(cfg), C.byref(params), _p(Q), _p(V), _p(U),
                                     _p(sp), C.byref(kb))
        if r != 0:
            raise RuntimeError("ref_init_state failed")
        return self, Q, V, U, sp, kb.value

    @classmethod
    def accessible_volume(cls, cfg, species=0):
        """The reference's Monte Carlo accessibleVolume (init.c:954-989) with
        its own generator (the timing build), for cfg's walls."""
        lib = cls.lib(timing=True)
        z = np.zeros(3)
        if lib.ref_init(C.byref(cfg), 0, _p(z), _p(z), None, None) != 0:
            raise RuntimeError("ref_init failed")
        return lib.ref_accessible_volume(species)

    def set_vdist(self, vdist):
        """The species' VDIST (re-thermalised velocities)."""
        v = np.zeros(10, dtype=np.int32)
        v[:len(vdist)] = vdist
        self._lib.ref_set_vdist(_p(v))

    def set_flow(self, on=True):
        """Sum the cell velocities into FLOW after every step (flow output)."""
        self._lib.ref_set_flow(int(bool(on)))

    def flow(self):
        nc = self._lib.ref_ncells()
        f = np.zeros((nc, 3))
        self._lib.ref_get_flow(_p(f))
        return f

    def cell_species(self):
        nc = self._lib.ref_ncells()
        out = np.zeros(self.cfg.n_species * nc, dtype=np.int32)
        self._lib.ref_get_cell_species(_p(out))
        return out.reshape(self.cfg.n_species, nc)

    def write_outputs(self, outdir, runtime, flow_interval=0, header=False):
        """The reference's own writers of the current state into outdir."""
        d = str(outdir).rstrip("/") + "/"
        if self._lib.ref_write_outputs(d.encode(), runtime, flow_interval, int(header)) != 0:
            raise RuntimeError("ref_write_outputs failed")

    def checkpoint_write(self, path, runtime, warmtime=0):
        """The reference's checkpoint() of the current state to path."""
        if self._lib.ref_checkpoint_write(str(path).encode(), runtime, warmtime) != 0:
            raise RuntimeError("ref_checkpoint_write failed")

    @classmethod
    def checkpoint_read(cls, path, abi_config):
        """The reference's readchckpnt() of path: (config as the reference
        holds it, Q, V, U, spid, runtime, warmtime, KBTNOW, AVNOW)."""
        lib = cls.lib()
        cfg = abi_config()
        n, rt, wt, kb = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        av = np.zeros(3)
        lib.ref_checkpoint_read(str(path).encode(), C.byref(cfg), C.byref(n), C.byref(rt),
                                C.byref(wt), C.byref(kb), _p(av))
        m = n.value
        Q, V, U = np.zeros((m, 3)), np.zeros((m, 3)), np.zeros((m, 3))
        sp = np.zeros(m, dtype=np.int32)
        lib.ref_checkpoint_particles(_p(Q), _p(V), _p(U), _p(sp))
        return cfg, Q, V, U, sp, rt.value, wt.value, kb.value, av

    @classmethod
    def theory_visc(cls, coll_op, dim, n, rot_ang, dt, kbt=1.0, m=1.0):
        """The reference's own theory_trans (init.c:800-942): kinematic
        viscosity, self-diffusion coefficient and mean free path."""
        sd, mfp = C.c_double(), C.c_double()
        nu = cls.lib().ref_theory_visc(coll_op, dim, n, rot_ang, dt, kbt, m, C.byref(sd),
                                       C.byref(mfp))
        return nu, sd.value, mfp.value

    def step(self, step):
        self._lib.ref_step(step)

    def run_timed(self, nsteps, step0=1):
        return self._lib.ref_run_timed(nsteps, step0)

    def particles(self):
        Q = np.zeros((self.n, 3))
        V = np.zeros((self.n, 3))
        U = np.zeros((self.n, 3))
        self._lib.ref_get_particles(_p(Q), _p(V), _p(U))
        return Q, V, U

    def globals(self):
        kb = C.c_double()
        av = np.zeros(3)
        self._lib.ref_get_globals(C.byref(kb), _p(av))
        return kb.value, av

    def cells(self):
        nc = self._lib.ref_ncells()
        pop = np.zeros(nc, dtype=np.int32)
        mass = np.zeros(nc)
        vcm = np.zeros((nc, 3))
        cm = np.zeros((nc, 3))
        self._lib.ref_get_cells(_p(pop), _p(mass), _p(vcm), _p(cm))
        return pop, mass, vcm, cm

    def gndnst(self):
        return self._lib.ref_gndnst()

    def unexpected_draws(self):
        return self._lib.ref_unexpected_draws()
