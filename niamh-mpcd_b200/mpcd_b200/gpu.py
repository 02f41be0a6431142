"""Python binding of libmpcd_gpu.so (the C ABI of include/mpcd_gpu.h).

The library is built in-tree (niamh-mpcd_b200/build.sh); if it is missing,
loading raises instead of falling back to any CPU path.
"""
import ctypes as C
import os

import numpy as np

from . import abi

LIB_PATH = os.environ.get(
    "MPCD_GPU_LIB",
    os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "libmpcd_gpu.so"))

EXPORTS = [
    "mpcd_abi_version", "mpcd_create", "mpcd_destroy", "mpcd_upload_state",
    "mpcd_upload_particles_strided", "mpcd_init_state", "mpcd_set_species_vdist",
    "mpcd_accessible_volume",
    "mpcd_download_state",
    "mpcd_download_particles_strided", "mpcd_step", "mpcd_timestep",
    "mpcd_globals", "mpcd_cell_props", "mpcd_get_status", "mpcd_set_stream",
    "mpcd_launches_per_step", "mpcd_set_strategy", "mpcd_set_kernel",
    "mpcd_set_sort_interval", "mpcd_set_timing", "mpcd_kernel_time",
    "mpcd_transverse_modes", "mpcd_step_record", "mpcd_debug_cell_counts",
    "mpcd_autotune", "mpcd_tune_key", "mpcd_tune_cache_lookup", "mpcd_tune_cache_store",
    "mpcd_srd_step_noalloc", "mpcd_batch_create", "mpcd_batch_destroy", "mpcd_batch_upload",
    "mpcd_batch_step", "mpcd_batch_download", "mpcd_batch_globals",
    "mpcd_batch_set_sort_interval", "mpcd_batch_set_stream", "mpcd_batch_info",
    "mpcd_download_species", "mpcd_get_config", "mpcd_particle_count", "mpcd_ckpt_read", "mpcd_ckpt_create",
    "mpcd_ckpt_free", "mpcd_ckpt_write", "mpcd_ckpt_config", "mpcd_ckpt_get_run",
    "mpcd_ckpt_set_run", "mpcd_ckpt_count", "mpcd_ckpt_particles", "mpcd_ckpt_set_particles",
    "mpcd_ckpt_upload", "mpcd_ckpt_capture", "mpcd_cell_species", "mpcd_flow_enable",
    "mpcd_flow_read", "mpcd_kinetic_energy", "mpcd_write_coarse", "mpcd_write_velfield",
    "mpcd_write_densityfield", "mpcd_write_flowfield", "mpcd_write_avvel", "mpcd_write_energy",
    "mpcd_vel_grad", "mpcd_av_vel",
]

_lib = None


class MPCDError(RuntimeError):
    pass


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MPCDError(f"libmpcd_gpu.so not built ({LIB_PATH}); run build()")
        lib = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        lib.mpcd_create.argtypes = [vp, C.POINTER(vp)]
        lib.mpcd_destroy.argtypes = [vp]
        lib.mpcd_upload_state.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        lib.mpcd_upload_particles_strided.argtypes = [vp, C.c_int, vp, C.c_size_t,
                                                      C.c_size_t, C.c_size_t, C.c_size_t,
                                                      C.c_size_t]
        lib.mpcd_init_state.argtypes = [vp, vp, vp]
        lib.mpcd_set_species_vdist.argtypes = [vp, vp]
        lib.mpcd_accessible_volume.argtypes = [vp, C.c_int, vp]
        lib.mpcd_download_state.argtypes = [vp, vp, vp, vp]
        lib.mpcd_download_species.argtypes = [vp, vp]
        lib.mpcd_particle_count.argtypes = [vp, vp]
        lib.mpcd_get_config.argtypes = [vp, vp]
        lib.mpcd_ckpt_read.argtypes = [C.c_char_p, C.POINTER(vp)]
        lib.mpcd_ckpt_create.argtypes = [vp, C.POINTER(vp)]
        lib.mpcd_ckpt_free.argtypes = [vp]
        lib.mpcd_ckpt_write.argtypes = [vp, C.c_char_p, C.c_int]
        lib.mpcd_ckpt_config.argtypes = [vp, vp]
        lib.mpcd_ckpt_get_run.argtypes = [vp, vp]
        lib.mpcd_ckpt_set_run.argtypes = [vp, vp]
        lib.mpcd_ckpt_count.argtypes = [vp, vp]
        lib.mpcd_ckpt_particles.argtypes = [vp, vp, vp, vp, vp]
        lib.mpcd_ckpt_set_particles.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        lib.mpcd_ckpt_upload.argtypes = [vp, vp]
        lib.mpcd_ckpt_capture.argtypes = [vp, vp]
        lib.mpcd_cell_species.argtypes = [vp, vp]
        lib.mpcd_flow_enable.argtypes = [vp, C.c_int]
        lib.mpcd_flow_read.argtypes = [vp, vp, vp, C.c_int]
        lib.mpcd_kinetic_energy.argtypes = [vp, vp]
        lib.mpcd_write_coarse.argtypes = [C.c_char_p, vp, C.c_double, vp, vp, vp, C.c_int]
        lib.mpcd_write_velfield.argtypes = [C.c_char_p, vp, C.c_double, vp, C.c_int]
        lib.mpcd_write_densityfield.argtypes = [C.c_char_p, vp, C.c_double, vp, vp, vp, C.c_int]
        lib.mpcd_write_flowfield.argtypes = [C.c_char_p, vp, C.c_double, vp, C.c_int, C.c_int]
        lib.mpcd_write_avvel.argtypes = [C.c_char_p, C.c_double, vp, C.c_double, vp, C.c_int]
        lib.mpcd_write_energy.argtypes = [C.c_char_p, C.c_double, C.c_double, C.c_double,
                                          C.c_int]
        lib.mpcd_vel_grad.argtypes = [vp, vp, vp, vp]
        lib.mpcd_av_vel.argtypes = [vp, vp, vp]
        lib.mpcd_download_particles_strided.argtypes = [vp, vp, C.c_size_t, C.c_size_t,
                                                        C.c_size_t, C.c_size_t]
        lib.mpcd_step.argtypes = [vp, C.c_int, C.c_uint32]
        lib.mpcd_timestep.argtypes = [vp, C.c_uint32, vp, vp]
        lib.mpcd_globals.argtypes = [vp, vp, vp]
        lib.mpcd_cell_props.argtypes = [vp, vp, vp, vp, vp]
        lib.mpcd_step_record.argtypes = [vp, C.c_int, C.c_uint32, vp, vp]
        lib.mpcd_debug_cell_counts.argtypes = [vp, vp]
        lib.mpcd_autotune.argtypes = [vp, C.c_int, C.c_char_p, vp]
        lib.mpcd_tune_key.argtypes = [vp, C.c_int, C.c_char_p, C.c_char_p, C.c_size_t]
        lib.mpcd_tune_cache_lookup.argtypes = [C.c_char_p, C.c_char_p, vp]
        lib.mpcd_tune_cache_store.argtypes = [C.c_char_p, C.c_char_p, vp]
        lib.mpcd_get_status.argtypes = [vp, vp]
        lib.mpcd_set_stream.argtypes = [vp, vp]
        lib.mpcd_launches_per_step.argtypes = [vp]
        lib.mpcd_set_strategy.argtypes = [vp, C.c_int, C.c_int]
        lib.mpcd_set_kernel.argtypes = [vp, C.c_int]
        lib.mpcd_set_sort_interval.argtypes = [vp, C.c_int]
        lib.mpcd_set_timing.argtypes = [vp, C.c_int]
        lib.mpcd_transverse_modes.argtypes = [vp, vp, C.POINTER(C.c_int)]
        lib.mpcd_batch_create.argtypes = [vp, C.c_int, vp, vp, vp]
        lib.mpcd_batch_destroy.argtypes = [vp]
        lib.mpcd_batch_upload.argtypes = [vp, vp, vp, vp, C.c_uint32]
        lib.mpcd_batch_step.argtypes = [vp, C.c_int]
        lib.mpcd_batch_download.argtypes = [vp, vp, vp]
        lib.mpcd_batch_globals.argtypes = [vp, vp, vp]
        lib.mpcd_batch_set_sort_interval.argtypes = [vp, C.c_int]
        lib.mpcd_batch_set_stream.argtypes = [vp, vp]
        lib.mpcd_batch_info.argtypes = [vp, vp, vp, vp]
        lib.mpcd_kernel_time.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.mpcd_srd_step_noalloc.argtypes = [vp, C.c_int, vp, vp, C.c_uint32, vp, vp, vp]
        _lib = lib
    return _lib


def _check(r, what):
    if r != 0:
        raise MPCDError(f"{what} failed: {r} ({abi.ERRORS.get(r, 'unknown')})")


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def tune_key(cfg, n, device):
    """The autotuner's cache key of a workload on a device (no GPU needed)."""
    lib = load()
    buf = C.create_string_buffer(512)
    _check(lib.mpcd_tune_key(C.byref(cfg), n, device.encode(), buf, 512), "mpcd_tune_key")
    return buf.value.decode()


def tune_cache_lookup(path, key):
    """The cached choice for key (abi.TuneChoice) or None (no GPU needed)."""
    lib = load()
    c = abi.TuneChoice()
    r = lib.mpcd_tune_cache_lookup(str(path).encode(), key.encode(), C.byref(c))
    if r < 0:
        _check(r, "mpcd_tune_cache_lookup")
    return c if r == 1 else None


def tune_cache_store(path, key, choice):
    lib = load()
    _check(lib.mpcd_tune_cache_store(str(path).encode(), key.encode(), C.byref(choice)),
           "mpcd_tune_cache_store")


def accessible_volume(cfg, species=0):
    """Volume accessible to a species (mpcd_accessible_volume; host only)."""
    lib = load()
    v = C.c_double()
    _check(lib.mpcd_accessible_volume(C.byref(cfg), species, C.byref(v)),
           "mpcd_accessible_volume")
    return v.value


class FieldWriter:
    """The reference's output files (coarsegrain, velfield, densityfield,
    flowfield, avVel, energy .dat) from cell arrays, through the library's
    host writers.  Keeps the velocity-gradient array between calls, as the
    reference's cells keep theirs."""

    def __init__(self, cfg, outdir):
        self.lib = load()
        self.cfg = cfg
        self.dir = str(outdir)
        L = [cfg.L[d] if d < cfg.dim else 1 for d in range(3)]
        self.nc = (L[0] + 1) * (L[1] + 1) * (L[2] + 1)
        self.E = np.zeros(9 * self.nc)
        self.started = set()

    def _path(self, name):
        return os.path.join(self.dir, name + ".dat").encode()

    def _hdr(self, name):
        first = name not in self.started
        self.started.add(name)
        return int(first)

    def write(self, t, pop, mass, vcm, spc, kbtnow, kinetic, flow=None, interval=0):
        """One output step: arrays over the (L+1)^D grid (vcm and flow as
        (nc, 3)); spc per species (ns, nc) or None for one species."""
        cfg = C.byref(self.cfg)
        pop = np.ascontiguousarray(pop, dtype=np.int32)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        vcm = np.ascontiguousarray(vcm, dtype=np.float64)
        sp = None if spc is None else np.ascontiguousarray(spc, dtype=np.int32)
        lib = self.lib
        _check(lib.mpcd_write_coarse(self._path("coarsegrain"), cfg, t, _p(pop), _p(vcm), _p(sp),
                                     self._hdr("coarsegrain")), "mpcd_write_coarse")
        _check(lib.mpcd_write_velfield(self._path("velfield"), cfg, t, _p(vcm),
                                       self._hdr("velfield")), "mpcd_write_velfield")
        _check(lib.mpcd_write_densityfield(self._path("densityfield"), cfg, t, _p(pop), _p(mass),
                                           _p(sp), self._hdr("densityfield")),
               "mpcd_write_densityfield")
        if flow is not None:
            fl = np.ascontiguousarray(flow, dtype=np.float64)
            _check(lib.mpcd_write_flowfield(self._path("flowfield"), cfg, t, _p(fl), interval,
                                            self._hdr("flowfield")), "mpcd_write_flowfield")
        grad = np.zeros(9)
        av = np.zeros(3)
        _check(lib.mpcd_vel_grad(cfg, _p(vcm), _p(self.E), _p(grad)), "mpcd_vel_grad")
        _check(lib.mpcd_av_vel(cfg, _p(vcm), _p(av)), "mpcd_av_vel")
        _check(lib.mpcd_write_avvel(self._path("avVel"), t, _p(av), kbtnow, _p(grad),
                                    self._hdr("avVel")), "mpcd_write_avvel")
        _check(lib.mpcd_write_energy(self._path("energy"), t, kinetic, kbtnow,
                                     self._hdr("energy")), "mpcd_write_energy")

    def write_from(self, solver, t, kbtnow, flow_interval=0):
        """One output step from a Solver's state (cell fields on the device;
        the flow sum read and emptied when flow_interval > 0)."""
        pop, mass, vcm, _ = solver.cell_props()
        pop, mass, vcm = pop.reshape(-1), mass.reshape(-1), vcm.reshape(-1, 3)
        spc = solver.cell_species() if self.cfg.n_species > 1 else None
        flow = solver.flow_read(reset=True)[0] if flow_interval > 0 else None
        self.write(t, pop, mass, vcm, spc, kbtnow, solver.kinetic_energy(), flow, flow_interval)


class Checkpoint:
    """A checkpoint in the reference's text format (mpcd_ckpt_*): read from
    a file or made from a config; host-side except upload/capture."""

    def __init__(self, path=None, cfg=None):
        self.lib = load()
        h = C.c_void_p()
        if path is not None:
            _check(self.lib.mpcd_ckpt_read(str(path).encode(), C.byref(h)), "mpcd_ckpt_read")
        else:
            _check(self.lib.mpcd_ckpt_create(C.byref(cfg), C.byref(h)), "mpcd_ckpt_create")
        self.h = h

    def write(self, path, precise=False):
        _check(self.lib.mpcd_ckpt_write(self.h, str(path).encode(), int(bool(precise))),
               "mpcd_ckpt_write")

    def config(self):
        cfg = abi.Config()
        _check(self.lib.mpcd_ckpt_config(self.h, C.byref(cfg)), "mpcd_ckpt_config")
        return cfg

    def run(self):
        r = abi.CkptRun()
        _check(self.lib.mpcd_ckpt_get_run(self.h, C.byref(r)), "mpcd_ckpt_get_run")
        return r

    def set_run(self, run):
        _check(self.lib.mpcd_ckpt_set_run(self.h, C.byref(run)), "mpcd_ckpt_set_run")

    def count(self):
        n = C.c_int()
        _check(self.lib.mpcd_ckpt_count(self.h, C.byref(n)), "mpcd_ckpt_count")
        return n.value

    def particles(self):
        n = self.count()
        Q, V, U = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        sp = np.zeros(n, dtype=np.int32)
        _check(self.lib.mpcd_ckpt_particles(self.h, _p(Q), _p(V), _p(U), _p(sp)),
               "mpcd_ckpt_particles")
        return Q, V, U, sp

    def set_particles(self, Q, V, U=None, spid=None):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        spid = None if spid is None else np.ascontiguousarray(spid, dtype=np.int32)
        _check(self.lib.mpcd_ckpt_set_particles(self.h, len(Q), _p(Q), _p(V), _p(U), _p(spid)),
               "mpcd_ckpt_set_particles")

    def upload(self, solver):
        _check(self.lib.mpcd_ckpt_upload(self.h, solver.h), "mpcd_ckpt_upload")
        solver.n = self.count()

    def capture(self, solver):
        _check(self.lib.mpcd_ckpt_capture(self.h, solver.h), "mpcd_ckpt_capture")

    def close(self):
        if self.h:
            self.lib.mpcd_ckpt_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def srd_step_noalloc(cfg, n, q_dev_ptr, v_dev_ptr, step, globals_dev_ptr=None, stream=None,
                     counters_dev_ptr=None):
    """One SRD timestep on caller-owned device arrays (AoS, 3 doubles per
    particle) with no allocation (mpcd_srd_step_noalloc).  counters_dev_ptr:
    optional device array of 3 uint64 (escaped, bounce_limit, nonfinite) to
    which the step adds its counts."""
    lib = load()

    def vp(x):
        return C.c_void_p(x) if x else None

    _check(lib.mpcd_srd_step_noalloc(C.byref(cfg), n, C.c_void_p(q_dev_ptr),
                                     C.c_void_p(v_dev_ptr), step, vp(globals_dev_ptr),
                                     vp(counters_dev_ptr), vp(stream)),
           "mpcd_srd_step_noalloc")


class Solver:
    """One simulation box on the current CUDA device."""

    def __init__(self, cfg):
        self.lib = load()
        self.cfg = cfg
        h = C.c_void_p()
        _check(self.lib.mpcd_create(C.byref(cfg), C.byref(h)), "mpcd_create")
        self.h = h
        self.n = 0

    def upload(self, Q, V, U=None, spid=None):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        spid = None if spid is None else np.ascontiguousarray(spid, dtype=np.int32)
        _check(self.lib.mpcd_upload_state(self.h, len(Q), _p(Q), _p(V), _p(U), _p(spid)),
               "mpcd_upload_state")
        self.n = len(Q)

    def init_state(self, params):
        """Build the initial state on the device (mpcd_init_state) from an
        abi.InitParams; returns TEMP after the temperature scaling."""
        k = C.c_double()
        self.n = 0  # a failed initialisation leaves no state
        _check(self.lib.mpcd_init_state(self.h, C.byref(params), C.byref(k)), "mpcd_init_state")
        self.n = sum(params.population)
        return k.value

    def set_vdist(self, vdist):
        """The species' velocity distributions (VDIST codes), which a
        particle past the wall bounce limit is re-thermalised from."""
        v = np.zeros(abi.MAX_SPECIES, dtype=np.int32)
        v[:len(vdist)] = vdist
        _check(self.lib.mpcd_set_species_vdist(self.h, _p(v)), "mpcd_set_species_vdist")

    def config(self):
        """The handle's configuration, gndnst the value in use."""
        cfg = abi.Config()
        _check(self.lib.mpcd_get_config(self.h, C.byref(cfg)), "mpcd_get_config")
        return cfg

    def cell_species(self):
        """Per-species populations of the end-of-step cells, (ns, nc)."""
        ns = self.cfg.n_species
        L = [self.cfg.L[d] if d < self.cfg.dim else 1 for d in range(3)]
        nc = (L[0] + 1) * (L[1] + 1) * (L[2] + 1)
        out = np.zeros(ns * nc, dtype=np.int32)
        _check(self.lib.mpcd_cell_species(self.h, _p(out)), "mpcd_cell_species")
        return out.reshape(ns, nc)

    def flow_enable(self, on=True):
        _check(self.lib.mpcd_flow_enable(self.h, int(bool(on))), "mpcd_flow_enable")

    def flow_read(self, reset=False):
        """(flow sum (nc, 3), steps summed)."""
        L = [self.cfg.L[d] if d < self.cfg.dim else 1 for d in range(3)]
        nc = (L[0] + 1) * (L[1] + 1) * (L[2] + 1)
        f = np.zeros((nc, 3))
        k = C.c_longlong()
        _check(self.lib.mpcd_flow_read(self.h, _p(f), C.byref(k), int(bool(reset))),
               "mpcd_flow_read")
        return f, k.value

    def kinetic_energy(self):
        e = C.c_double()
        _check(self.lib.mpcd_kinetic_energy(self.h, C.byref(e)), "mpcd_kinetic_energy")
        return e.value

    def species(self):
        """Species id of every particle, in the original order."""
        sp = np.zeros(self.n, dtype=np.int32)
        _check(self.lib.mpcd_download_species(self.h, _p(sp)), "mpcd_download_species")
        return sp

    def step(self, nsteps, step0):
        _check(self.lib.mpcd_step(self.h, nsteps, step0), "mpcd_step")

    def timestep(self, runtime):
        av = np.zeros(3)
        kb = C.c_double()
        _check(self.lib.mpcd_timestep(self.h, runtime, _p(av), C.byref(kb)), "mpcd_timestep")
        return kb.value, av

    def step_record(self, nsteps, step0):
        """nsteps steps from step0 with every step's (KBTNOW, AVNOW)
        (mpcd_step_record): arrays of shapes (nsteps,) and (nsteps, 3)."""
        kb = np.zeros(nsteps)
        av = np.zeros((nsteps, 3))
        _check(self.lib.mpcd_step_record(self.h, nsteps, step0, _p(kb), _p(av)),
               "mpcd_step_record")
        return kb, av

    def debug_cell_counts(self):
        """Populations of the cells of the next step's shifted grid as the
        device holds them (mpcd_debug_cell_counts), flat over (L+1)^D."""
        nc = int(np.prod([int(self.cfg.L[d]) + 1 for d in range(3)]))
        pop = np.zeros(nc, dtype=np.int32)
        _check(self.lib.mpcd_debug_cell_counts(self.h, _p(pop)), "mpcd_debug_cell_counts")
        return pop

    def globals(self):
        av = np.zeros(3)
        kb = C.c_double()
        _check(self.lib.mpcd_globals(self.h, C.byref(kb), _p(av)), "mpcd_globals")
        return kb.value, av

    def download(self, out=None):
        """Positions, velocities and orientations in the original particle
        order.  out=(Q, V) writes into the caller's (n, 3) float64 arrays
        (pinned host memory makes the copies direct) and skips the
        orientations; the third result is then None."""
        if out is not None:
            Q, V = out
            assert Q.shape == (self.n, 3) and V.shape == (self.n, 3)
            assert Q.dtype == np.float64 and V.dtype == np.float64
            assert Q.flags.c_contiguous and V.flags.c_contiguous
            _check(self.lib.mpcd_download_state(self.h, _p(Q), _p(V), None),
                   "mpcd_download_state")
            return Q, V, None
        Q = np.zeros((self.n, 3))
        V = np.zeros((self.n, 3))
        U = np.zeros((self.n, 3))
        _check(self.lib.mpcd_download_state(self.h, _p(Q), _p(V), _p(U)),
               "mpcd_download_state")
        return Q, V, U

    def cell_props(self):
        """Per-cell population, mass, centre-of-mass velocity and centre of
        mass on the unshifted (L+1)^D grid, as arrays shaped (L0+1, L1+1,
        L2+1) (the last two with a trailing axis of 3)."""
        shp = tuple(int(self.cfg.L[d]) + 1 for d in range(3))
        nc = shp[0] * shp[1] * shp[2]
        pop = np.zeros(nc, dtype=np.int32)
        mass = np.zeros(nc)
        vcm = np.zeros((nc, 3))
        cm = np.zeros((nc, 3))
        _check(self.lib.mpcd_cell_props(self.h, _p(pop), _p(mass), _p(vcm), _p(cm)),
               "mpcd_cell_props")
        return (pop.reshape(shp), mass.reshape(shp), vcm.reshape(shp + (3,)),
                cm.reshape(shp + (3,)))

    def status(self):
        st = abi.Status()
        _check(self.lib.mpcd_get_status(self.h, C.byref(st)), "mpcd_get_status")
        return st

    def launches_per_step(self):
        return self.lib.mpcd_launches_per_step(self.h)

    def set_strategy(self, strategy=-1, tile_particles=0):
        _check(self.lib.mpcd_set_strategy(self.h, strategy, tile_particles),
               "mpcd_set_strategy")

    def set_kernel(self, kernel):
        _check(self.lib.mpcd_set_kernel(self.h, kernel), "mpcd_set_kernel")

    def transverse_modes(self):
        """The transverse momentum modes as complex numbers (6 in 3D)."""
        out = np.zeros(12)
        nm = C.c_int()
        _check(self.lib.mpcd_transverse_modes(self.h, _p(out), C.byref(nm)),
               "mpcd_transverse_modes")
        return out[0:2 * nm.value:2] + 1j * out[1:2 * nm.value:2]

    def set_timing(self, enable=True):
        _check(self.lib.mpcd_set_timing(self.h, 1 if enable else 0), "mpcd_set_timing")

    def kernel_time(self):
        """(summed ms, launches) of the timed particle-pass launches."""
        ms = C.c_double()
        nl = C.c_int()
        _check(self.lib.mpcd_kernel_time(self.h, C.byref(ms), C.byref(nl)), "mpcd_kernel_time")
        return ms.value, nl.value

    def set_sort_interval(self, steps):
        _check(self.lib.mpcd_set_sort_interval(self.h, steps), "mpcd_set_sort_interval")

    def autotune(self, trial_steps=0, cache_path=None):
        """Time the applicable execution plans and apply the fastest
        (mpcd_autotune); returns the abi.TuneChoice."""
        c = abi.TuneChoice()
        _check(self.lib.mpcd_autotune(self.h, trial_steps,
                                      None if cache_path is None else str(cache_path).encode(),
                                      C.byref(c)), "mpcd_autotune")
        return c

    def set_stream(self, stream_ptr):
        _check(self.lib.mpcd_set_stream(self.h, C.c_void_p(stream_ptr)), "mpcd_set_stream")

    def close(self):
        if self.h:
            self.lib.mpcd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """An ensemble of periodic 3D SRD boxes stepped together (mpcd_batch_*)."""

    def __init__(self, base_cfg, sizes, seeds=None):
        self.lib = load()
        self.sizes = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32).reshape(-1, 3))
        self.nb = len(self.sizes)
        self.seeds = (None if seeds is None
                      else np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64)))
        self.h = C.c_void_p()
        _check(self.lib.mpcd_batch_create(C.byref(base_cfg), self.nb, _p(self.sizes),
                                          _p(self.seeds) if self.seeds is not None else None,
                                          C.byref(self.h)), "mpcd_batch_create")
        self.npart = None

    def upload(self, npart, Q, V, step0=1):
        self.npart = np.ascontiguousarray(np.asarray(npart, dtype=np.int32))
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        _check(self.lib.mpcd_batch_upload(self.h, _p(self.npart), _p(Q), _p(V), step0),
               "mpcd_batch_upload")

    def step(self, nsteps=1):
        _check(self.lib.mpcd_batch_step(self.h, nsteps), "mpcd_batch_step")

    def download(self, out=None):
        """Positions and velocities of all boxes in the upload's order;
        out=(Q, V) writes into the caller's (n, 3) float64 arrays (pinned
        host memory makes the copies direct)."""
        n = int(self.npart.sum())
        if out is not None:
            Q, V = out
            assert Q.shape == (n, 3) and V.shape == (n, 3)
            assert Q.dtype == np.float64 and V.dtype == np.float64
            assert Q.flags.c_contiguous and V.flags.c_contiguous
        else:
            Q = np.zeros((n, 3))
            V = np.zeros((n, 3))
        _check(self.lib.mpcd_batch_download(self.h, _p(Q), _p(V)), "mpcd_batch_download")
        return Q, V

    def globals(self):
        kb = np.zeros(self.nb)
        av = np.zeros((self.nb, 3))
        _check(self.lib.mpcd_batch_globals(self.h, _p(kb), _p(av)), "mpcd_batch_globals")
        return kb, av

    def set_sort_interval(self, steps):
        _check(self.lib.mpcd_batch_set_sort_interval(self.h, steps),
               "mpcd_batch_set_sort_interval")

    def set_stream(self, stream_ptr):
        _check(self.lib.mpcd_batch_set_stream(self.h, C.c_void_p(stream_ptr)),
               "mpcd_batch_set_stream")

    def info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.mpcd_batch_info(self.h, C.byref(a), C.byref(b), C.byref(c)),
               "mpcd_batch_info")
        return a.value, b.value, c.value

    def close(self):
        if self.h:
            self.lib.mpcd_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
