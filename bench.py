"""Benchmark of the MPCD solvent timestep on B200.

Workload (one step = one solvent timestep of every particle): the 3D SRD
fluid of 64^3 periodic cells, 10 particles per cell (2,621,440 particles),
kT=1, dt=0.1, rotation angle 130 degrees about a random axis per cell, random
grid shift, synthetic seeded state.  The headline is the mixed-precision form;
the plain FP64 form is measured in the same run ("fp64" key).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs independent replica boxes, one per rank (the path has no data
exchange between replicas): weak scaling, value summed over ranks, time the
max over ranks.  --workload ensemble with N > 1 splits one ensemble of boxes
across the ranks, balanced by particle count: strong scaling.  --impl
reference times the reference's own serial C timestep (built from its
sources into oracle/_ref/) on a bounded sample of the same workload on this
host's cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "niamh-mpcd_b200"))

METRIC = "MPCD particle-steps/s, mixed vs FP64 on 1 B200; achieved HBM GB/s"
UNIT = "particle-steps/s"
L_BOX = (64, 64, 64)
PPC = 10
# algorithmic bytes per particle-step (state read+written once, cell record
# written+read once per ppc particles): 3D SRD mixed 62.4 B, FP64 102.4 B
ALG_BYTES = {"mixed": 62.4, "fp64": 102.4}
SORT_INTERVAL = 30  # the library's default re-sort interval of the resident families
WORKLOAD = "3D SRD fluid, periodic 64^3 cells, 10 particles/cell (2,621,440), rot 130 deg"
L2_NOTE = {
    "none": ("not flushed: steps run back to back; each step reads and writes 2 x 84 MB of "
             "particle state plus 26 MB of cell sums and records, more than the 126 MB L2; "
             "ms_per_step_l2_flushed gives steps with L2 flushed before each"),
    "write+read": "flushed between timed steps: 256 MB write, then 256 MB read (L2 left holding clean lines)",
    "write": "flushed between timed steps: 256 MB write",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--forms", default="fp64,mixed",
                    help="comma list of state forms to time (fp64, mixed)")
    ap.add_argument("--strategy", type=int, default=-1,
                    help="-1 default, 0 scatter, 1 recompute")
    ap.add_argument("--tile", type=int, default=0, help="particles per tile (0 default)")
    ap.add_argument("--kernel", type=int, default=0,
                    help="cell-kernel family: 0 auto, 1 tile, 2 group, 3 split, 4 resident")
    ap.add_argument("--workload", default="srd64",
                    choices=["srd64", "ensemble", "rat2d", "channel", "nematic"],
                    help="srd64: the 64^3 SRD fluid (default); ensemble: 512 periodic SRD "
                         "boxes of sides 8-32 stepped together")
    ap.add_argument("--boxes", type=int, default=512, help="ensemble: number of boxes")
    ap.add_argument("--flush", default="none", choices=["none", "write+read", "write"],
                    help="L2 between timed steps: none (the step's working set is larger "
                         "than L2), or a flush before each step")
    ap.add_argument("--sort-interval", type=int, default=0,
                    help="resident family: steps between re-sorts (0 = library default)")
    return ap.parse_args()


def max_over_ranks(x, world, device="cuda"):
    """The maximum of x over all ranks (every rank gets it): the job's time
    is its slowest rank's."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(n_per_rank, world, steps, seconds):
    """Whole-job particle-steps/s: every rank advances its own replica of
    n_per_rank particles by `steps` steps; the job takes `seconds` (the max
    over ranks)."""
    return n_per_rank * world * steps / seconds


def traffic_per_launch():
    """DRAM bytes (read + write) of one particle-pass launch on this
    workload, from the committed ncu summary of that kernel, or None."""
    path = os.path.join(ROOT, "profiles", "k_res_parts_srd64_mixed.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """SM clock and clock-event reasons of this process's GPU, sampled during
    the timed region: NVML read every 10 ms by a thread (the timed region of
    the default run is a fraction of a second), or nvidia-smi every 200 ms
    where NVML cannot be loaded.  The GPU is found by its PCI address, so
    the samples are this device's whatever CUDA_VISIBLE_DEVICES says.  Each
    sample carries the host time of its reading, and stop() keeps those that
    fall inside [t0, t1] (the nearest one if the region was shorter than a
    sampling period).  Only reads: no clock or setting is changed."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, dev):
        import torch
        pr = torch.cuda.get_device_properties(dev)
        self.busid = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        self.samples = []  # (host time, sm MHz, max sm MHz, set of reason names)
        self.p = None
        self.nv = None
        self.halt = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(self.busid.encode())
            self.nv = pynvml
            self.bits = [(nm, getattr(pynvml, "nvmlClocksEventReason" + cap))
                         for nm, cap in zip(self.NAMES, ["HwSlowdown", "HwThermalSlowdown",
                                                         "SwThermalSlowdown", "SwPowerCap"])]
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.th = threading.Thread(target=self._poll, daemon=True)
        except Exception:
            self.nv = None
            try:
                self.p = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.busid}", f"--query-gpu={self.Q}",
                     "--format=csv,noheader,nounits", "-lms", "200"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            except Exception:
                self.p = None
                return
            self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _poll(self):
        nv = self.nv
        while not self.halt.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                return
            self.samples.append((time.time(), sm, self.smax,
                                 {nm for nm, bit in self.bits if mask & bit}))
            self.halt.wait(0.01)

    def _read(self):
        for line in self.p.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, smax = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            rs = {nm for nm, val in zip(self.NAMES, parts[5:9])
                  if val.lower().startswith("active")}
            self.samples.append((time.time(), sm, smax, rs))

    def wait_ready(self, timeout=15.0):
        t0 = time.time()
        while (self.p is not None or self.nv is not None) and not self.samples \
                and time.time() - t0 < timeout:
            time.sleep(0.01)

    def stop(self, t0, t1):
        if self.nv is None and self.p is None:
            return None
        if self.nv is not None:
            self.halt.set()
            self.th.join(timeout=2)
            slack = 0.01
        else:
            time.sleep(0.25)  # let the sample that covers t1 arrive
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            slack = 0.2
        inside = [s for s in self.samples if t0 <= s[0] <= t1 + slack]
        if not inside and self.samples:
            inside = [min(self.samples, key=lambda s: abs(s[0] - 0.5 * (t0 + t1)))]
        if not inside:
            return None
        reasons = set().union(*(s[3] for s in inside))
        return {"sm_mhz": statistics.median(s[1] for s in inside),
                "sm_max_mhz": max(s[2] for s in inside),
                "reasons": sorted(reasons), "samples": len(inside),
                "source": "nvml" if self.nv is not None else "nvidia-smi",
                "timed_region_s": round(t1 - t0, 3)}


def run_gpu(args, rank, world):
    import numpy as np
    import torch

    from mpcd_b200 import abi
    from mpcd_b200 import workloads as W
    from mpcd_b200.gpu import Solver

    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    # the flush writes 256 MB, then reads another 256 MB so that the lines it
    # leaves in L2 are clean (otherwise the timed step pays the write-back of
    # the flush's own dirty lines); none of the step's data stays in L2
    flush_rd = torch.ones(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    flush_sink = torch.empty(1, dtype=torch.float32, device="cuda")
    results = {}

    def flush_l2(kind):
        flush.zero_()
        if kind == "write+read":
            torch.sum(flush_rd, dim=0, out=flush_sink[0])

    forms = [f for f in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED))
             if f[0] in args.forms.split(",")]
    for form, prec in forms:
        cfg = W.cfg_srd3d(L_BOX, precision=prec, seed=20240 + rank)
        cfg.replica = rank
        Q, V, U, sp = W.synthetic_state(cfg, PPC, seed=7 + rank)
        n = len(Q)
        g = Solver(cfg)
        g.set_stream(stream.cuda_stream)
        g.set_strategy(args.strategy, args.tile)
        g.set_kernel(args.kernel)
        g.upload(Q, V, U, sp)
        g.step(args.warmup, 1)
        # a new re-sort cycle: the first timed step re-sorts, so a window of K
        # steps carries ceil(K / interval) sorts (at least the steady
        # state's share, 1 per interval)
        g.set_sort_interval(args.sort_interval if args.sort_interval > 0 else SORT_INTERVAL)
        torch.cuda.synchronize()
        clk = Clocks(dev) if form == "mixed" else None
        if clk:
            clk.wait_ready()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        launches = 0
        step0 = 1 + args.warmup
        t_begin = time.time()
        if args.flush == "none":
            # back to back: the step's working set (state 2 x 84 MB, cell
            # sums and records 26 MB at 64^3) is larger than L2, so no step
            # finds the previous one's data there
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for k in range(args.steps):
                g.step(1, step0 + k)
                launches += g.launches_per_step()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = [e0.elapsed_time(e1) / args.steps]
            total = e0.elapsed_time(e1)
        else:
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
            for k in range(args.steps):
                flush_l2(args.flush)
                ev[k][0].record(stream)
                g.step(1, step0 + k)
                ev[k][1].record(stream)
                launches += g.launches_per_step()
            torch.cuda.synchronize()
            ms = [a.elapsed_time(b) for a, b in ev]
            total = float(sum(ms))
        t_end = time.time()
        clocks = clk.stop(t_begin, t_end) if clk else None
        step0 += args.steps
        # For comparison, steps with L2 flushed before each one (256 MB
        # write, then 256 MB read), each timed on its own.
        nf = min(args.steps, 200)
        evf = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(nf)]
        for k in range(nf):
            flush_l2("write+read")
            evf[k][0].record(stream)
            g.step(1, step0 + k)
            evf[k][1].record(stream)
        torch.cuda.synchronize()
        ms_flushed = sum(a.elapsed_time(b) for a, b in evf) / nf
        step0 += nf
        # The particle pass alone: a run of flushed steps with the library's
        # CUDA events around each particle-pass launch (kept out of the
        # timed steps above, where an event between the cell and particle
        # passes would hold back the particle pass's early start).
        g.set_timing(True)
        for k in range(nf):
            flush_l2("write+read")
            g.step(1, step0 + k)
        torch.cuda.synchronize()
        kern_ms, kern_n = g.kernel_time()
        g.set_timing(False)
        if world > 1:
            torch.distributed.barrier()
        total_ms = max_over_ranks(total, world)
        kb, av = g.globals()
        st = g.status()
        kernel_ms = max_over_ranks(kern_ms / max(kern_n, 1), world)
        results[form] = {
            "n": n, "ms_total": total_ms, "ms_per_step": total_ms / args.steps,
            "ms_min": min(ms), "ms_per_step_l2_flushed": max_over_ranks(ms_flushed, world),
            "launches": launches, "clocks": clocks,
            "kbt": kb, "escaped": int(st.escaped), "kernel_ms": kernel_ms,
            "kernel_launches": kern_n,
        }
        # e2e through the C ABI with host buffers: upload from pinned host
        # memory, K steps with every step's global measures (TEMP, avVel)
        # returned to the host (mpcd_step_record), download of the final
        # state into pinned arrays
        if form == "mixed":
            Qh = torch.from_numpy(Q).pin_memory().numpy()
            Vh = torch.from_numpy(V).pin_memory().numpy()
            # the caller's result arrays, pinned like its inputs
            Qo = torch.empty(Q.shape, dtype=torch.float64).pin_memory().numpy()
            Vo = torch.empty(V.shape, dtype=torch.float64).pin_memory().numpy()
            # one species: no species ids to upload (the library takes every
            # particle as species 0)
            spx = sp if cfg.n_species > 1 else None

            def e2e_pass():
                g.upload(Qh, Vh, None, spx)
                g.step_record(args.steps, 1000)
                return g.download(out=(Qo, Vo))

            # an untimed pass first, as for the device-timed steps (first
            # launches, first use of the caller's pinned buffers)
            e2e_pass()
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            t0 = time.perf_counter()
            q2, v2, _ = e2e_pass()
            torch.cuda.synchronize()
            e2e_s = max_over_ranks(time.perf_counter() - t0, world)
            results["e2e"] = {
                "value": job_rate(n, world, args.steps, e2e_s), "unit": UNIT,
                "h2d_bytes_per_step": (Q.nbytes + V.nbytes + (spx.nbytes if spx is not None else 0))
                / args.steps,
                "d2h_bytes_per_step": (q2.nbytes + v2.nbytes) / args.steps + 32,
                "path": "mpcd_upload_state, mpcd_step_record (every step's TEMP and avVel "
                        "to the host), mpcd_download_state",
            }
        g.close()
        del Q, V, U
    return results


# The other configurations, timed as back-to-back steps of both forms (their
# states, 0.6 MB to 0.5 GB, are timed as they are; the config says whether
# they exceed L2): name -> (description, builder, builder kwargs, particles per
# cell, algorithmic bytes per particle-step (mixed, FP64)).
OTHER = {
    "rat2d": ("2D MPC-AT+a, periodic 30^2 cells, 20 particles/cell (18,000), FP64 plain method",
              "cfg_passive2d", dict(L=(30, 30)), 20, (48.0, 72.0)),
    "channel": ("3D MPC-AT+a channel 128x64x64, phantom no-slip walls at y = 0 and 64, "
                "g = 1e-4 along x, 20 particles/cell (10,485,760)",
                "cfg_channel3d", dict(L=(128, 64, 64), g=1e-4), 20, (73.6, 113.6)),
    "nematic": ("2D active nematic 256^2, dipole LC collision (collOp 16), "
                "20 particles/cell (1,310,720)",
                "cfg_nematic2d", dict(L=(256, 256)), 20, (72.0, 112.0)),
}


FP64_WORKLOADS = ("rat2d",)


def run_other(args, rank, world):
    """One of the other configurations: back-to-back steps of the mixed and
    the FP64 form, timed with CUDA events around the whole run."""
    import torch

    from mpcd_b200 import abi
    from mpcd_b200 import workloads as W
    from mpcd_b200.gpu import Solver

    desc, builder, kw, ppc, alg = OTHER[args.workload]
    stream = torch.cuda.current_stream()
    out = {}
    for form, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        cfg = getattr(W, builder)(**kw, precision=prec, seed=30300 + rank)
        cfg.replica = rank
        Q, V, U, sp = W.synthetic_state(cfg, ppc, seed=31 + rank)
        g = Solver(cfg)
        g.set_stream(stream.cuda_stream)
        g.set_strategy(args.strategy, args.tile)
        g.upload(Q, V, U, sp)
        g.step(args.warmup, 1)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(args.steps, 1 + args.warmup)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        st = g.status()
        n = len(Q)
        out[form] = {"n": n, "ms_per_step": ms / args.steps,
                     "value": job_rate(n, world, args.steps, ms / 1e3),
                     "state_mb": n * (32 if form == "mixed" else 52) / 1e6,
                     "escaped": int(st.escaped), "overflow": int(st.overflow)}
        g.close()
    if rank == 0:
        peak, peak_kind = peaks()
        mix = out["mixed"]
        ach = alg[0] * mix["n"] / (mix["ms_per_step"] / 1e3) / 1e9
        ach64 = alg[1] * out["fp64"]["n"] / (out["fp64"]["ms_per_step"] / 1e3) / 1e9
        # the configuration's own form is the headline: FP64 for the plain
        # method of configuration 1, mixed elsewhere
        head = "fp64" if args.workload in FP64_WORKLOADS else "mixed"
        hv = out[head]
        print(json.dumps({
            "metric": METRIC, "value": hv["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": hv["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else "f32+f64 (mixed)", "data": "synthetic",
            "form": head,
            "mixed": {"value": mix["value"], "ms_per_step": mix["ms_per_step"],
                      "achieved_gbs": ach, "frac": ach / peak},
            "config": {"workload": desc, "global_batch": mix["n"] * world,
                       "parallelism": f"replicas x{world}",
                       "l2": (f"not flushed: back-to-back steps; mixed state "
                              f"{mix['state_mb']:.1f} MB ("
                              + ("larger" if mix["state_mb"] > 126 else "smaller")
                              + " than the 126 MB L2)")},
            "fp64": {"value": out["fp64"]["value"], "ms_per_step": out["fp64"]["ms_per_step"],
                     "achieved_gbs": ach64, "frac": ach64 / peak},
            "mixed_over_fp64": mix["value"] / out["fp64"]["value"],
            "roofline": {"bound": "hbm", "achieved": ach64 if head == "fp64" else ach,
                         "peak": peak, "unit": "GB/s",
                         "frac": (ach64 if head == "fp64" else ach) / peak, "traffic": None,
                         "kernel": "whole step",
                         "alg_bytes_per_particle_step": alg[1] if head == "fp64" else alg[0],
                         "peak_source": peak_kind},
            "status": {f: {"escaped": out[f]["escaped"], "overflow": out[f]["overflow"]}
                       for f in out},
        }))


def run_ensemble(args, rank, world):
    """Configuration 5: --boxes periodic 3D SRD boxes with sides drawn from
    {8, 12, 16, 24, 32}, 10 particles/cell, independent seeds, all stepped
    together (one launch per kernel, each step a CUDA graph replay).  With
    N > 1 the one ensemble is split across the ranks by box, balanced by
    particle count (no data crosses between boxes, so no collective): strong
    scaling.  The ensemble's state (about 1.7 GB for 512 boxes) is far larger
    than L2, so no flush is needed between steps."""
    import numpy as np
    import torch

    from mpcd_b200 import abi
    from mpcd_b200 import workloads as W
    from mpcd_b200.gpu import Batch

    sides_all = W.ensemble_sides(args.boxes)
    work = [10 * int(L) ** 3 for L in sides_all]
    mine = W.shard_boxes(work, world, rank)
    if not mine:
        raise SystemExit(f"rank {rank}: no box of the {args.boxes} to step")
    sides = sides_all[mine]
    sizes = np.stack([sides, sides, sides], axis=1)
    # each box's seed and state from its own stream: the same box gets the
    # same data whichever rank steps it
    seeds = np.array([np.random.default_rng([5000, b]).integers(1, 2 ** 62, dtype=np.uint64)
                      for b in mine], dtype=np.uint64)
    nparts, qs, vs = [], [], []
    for b, L in zip(mine, sides):
        rng = np.random.default_rng([5001, b])
        L = int(L)
        n = 10 * L ** 3
        q = rng.random((n, 3)) * L
        v = rng.standard_normal((n, 3))
        v -= v.mean(axis=0)
        nparts.append(n)
        qs.append(q)
        vs.append(v)
    base = W.cfg_srd3d((8, 8, 8), precision=abi.PREC_MIXED, seed=1)
    bat = Batch(base, sizes, seeds)
    stream = torch.cuda.current_stream()
    bat.set_stream(stream.cuda_stream)
    Q = np.concatenate(qs)
    V = np.concatenate(vs)
    del qs, vs
    bat.upload(nparts, Q, V, step0=1)
    n = int(sum(nparts))
    bat.step(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = Clocks(torch.cuda.current_device())
    clk.wait_ready()
    a = torch.cuda.Event(enable_timing=True)
    z = torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    a.record(stream)
    bat.step(args.steps)
    z.record(stream)
    torch.cuda.synchronize()
    t1 = time.time()
    clocks = clk.stop(t0, t1)
    ms = max_over_ranks(a.elapsed_time(z), world)
    kb, _ = bat.globals()
    nb_, slots, cells = bat.info()
    # e2e: upload from pinned host memory, the steps, download; an untimed
    # pass first
    Qh = torch.from_numpy(Q).pin_memory().numpy()
    Vh = torch.from_numpy(V).pin_memory().numpy()
    Qo = torch.empty(Q.shape, dtype=torch.float64).pin_memory().numpy()
    Vo = torch.empty(V.shape, dtype=torch.float64).pin_memory().numpy()
    for timed in (False, True):
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        bat.upload(nparts, Qh, Vh, step0=10 ** 6)
        bat.step(args.steps)
        bat.download(out=(Qo, Vo))
        torch.cuda.synchronize()
        if timed:
            e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    bat.close()
    n_job = int(sum(work))
    return {
        "n": n, "n_job": n_job, "boxes": len(mine), "ms_total": ms, "clocks": clocks,
        "kbt_mean": float(np.mean(kb)),
        "e2e": {"value": job_rate(n_job, 1, args.steps, e2e_s), "unit": UNIT,
                "h2d_bytes_per_step": (Q.nbytes + V.nbytes) / args.steps,
                "d2h_bytes_per_step": (Qo.nbytes + Vo.nbytes) / args.steps},
        "slots": slots, "cells": cells,
    }


def cpu_baseline(args, force_port=False):
    """The reference's own serial timestep (oracle/_ref/libmpcdref_time.so,
    built from its sources) on a bounded sample: the same 64^3 SRD state,
    a few steps, one core.  Falls back to the CPU oracle port if the
    reference build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from checkers import Oracle, Reference
    from mpcd_b200 import workloads as W

    cfg = W.cfg_srd3d(L_BOX, seed=20240)
    Q, V, U, sp = W.synthetic_state(cfg, PPC, seed=7)
    n = len(Q)
    k = max(1, args.cpu_sample_steps)
    if Reference.available(timing=True) and not force_port:
        r = Reference(cfg, Q, V, U, sp, timing=True)
        r.run_timed(1, 1)  # warm-up step
        secs = r.run_timed(k, 2)
        kind = "reference"
    else:
        o = Oracle(cfg, Q, V, U, sp)
        o.step(1)
        t0 = time.perf_counter()
        for s in range(k):
            o.step(2 + s)
        secs = time.perf_counter() - t0
        kind = "port"
    return {"value": n * k / secs, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{k} timesteps of the 64^3 SRD state ({n} particles) after 1 warm-up "
                      f"step, serial, host {os.cpu_count()} cores available"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_baseline(args)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
                "n_gpus": args.gpus, "steps": args.cpu_sample_steps, "warmup": 1,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "global_batch": 2621440, "form": "reference C"},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload in OTHER:
        run_other(args, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "ensemble":
        e = run_ensemble(args, rank, world)
        if rank == 0:
            # the whole ensemble's particles over the slowest rank's time
            n = e["n_job"]
            value = job_rate(n, 1, args.steps, e["ms_total"] / 1e3)
            peak, peak_kind = peaks()
            # bytes per GPU: this rank's share of the ensemble
            ach = ALG_BYTES["mixed"] * e["n"] / (e["ms_total"] / args.steps / 1e3) / 1e9
            print(json.dumps({
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": e["ms_total"] / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64 (mixed)",
                "data": "synthetic",
                "config": {"workload": f"ensemble of {args.boxes} periodic 3D SRD boxes, "
                                       "sides from {8,12,16,24,32}, 10 particles/cell",
                           "global_batch": n,
                           "parallelism": f"boxes sharded by particle count over {world} GPUs "
                                          f"({e['boxes']} boxes on rank 0)",
                           "l2": "not flushed: the ensemble's state is larger than L2",
                           "slots_with_padding": e["slots"], "cells_with_padding": e["cells"]},
                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                             "frac": ach / peak, "traffic": None,
                             "kernel": "whole step (graph replay)", "peak_source": peak_kind},
                "clocks": e["clocks"], "e2e": e["e2e"], "kbt_mean": e["kbt_mean"]}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    res = run_gpu(args, rank, world)
    if rank == 0 and not ("mixed" in res and "fp64" in res):
        print(json.dumps({k: v for k, v in res.items()}))
    elif rank == 0:
        mix, f64 = res["mixed"], res["fp64"]
        n = mix["n"]
        value = job_rate(n, world, args.steps, mix["ms_total"] / 1e3)
        v64 = job_rate(n, world, args.steps, f64["ms_total"] / 1e3)
        peak, peak_kind = peaks()
        # dominant kernel: the particle pass (reads and writes every particle)
        ach = ALG_BYTES["mixed"] * n / (mix["kernel_ms"] / 1e3) / 1e9
        step_gbs = ALG_BYTES["mixed"] * n / (mix["ms_total"] / args.steps / 1e3) / 1e9
        ach64 = ALG_BYTES["fp64"] * n / (f64["ms_total"] / args.steps / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": mix["ms_total"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": n * world, "form": "mixed",
                       "parallelism": f"replicas x{world}",
                       "l2": L2_NOTE[args.flush],
                       "sort_interval": args.sort_interval or SORT_INTERVAL,
                       "sorts_in_window": -(-args.steps // (args.sort_interval or SORT_INTERVAL))},
            "fp64": {"value": v64, "ms_per_step": f64["ms_total"] / args.steps,
                     "achieved_gbs": ach64, "frac": ach64 / peak},
            "mixed_over_fp64": value / v64,
            "ms_per_step_l2_flushed": mix["ms_per_step_l2_flushed"],
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "traffic": traffic_per_launch(),
                         "kernel": "k_res_parts<3, RES_STEP> (particle pass)",
                         "kernel_ms": mix["kernel_ms"],
                         "alg_bytes_per_launch": ALG_BYTES["mixed"] * n,
                         "step_achieved": step_gbs, "step_frac": step_gbs / peak,
                         "peak_source": peak_kind},
            "gpu_launches": mix["launches"],
            "clocks": mix["clocks"],
            "e2e": res["e2e"],
        }
        if not args.no_cpu:
            try:
                line["cpu_baseline"] = cpu_baseline(args)
            except Exception as e:  # noqa: BLE001
                line["cpu_baseline"] = {"error": str(e)}
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
