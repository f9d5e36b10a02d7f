#!/usr/bin/env python
"""Benchmark of the LJ hot path: pair-interactions per second on the 1,048,576-molecule FCC box
(rho 0.75, T 0.9, rc 3.0, dt 0.002, truncated-shifted LJ), FP32 pair arithmetic with FP64
accumulation on one B200 (one independent box per GPU when run on several).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision mixed|fp64]
  python bench.py --workload c3|batched|checkpoint|rigid|adjoint [--charges]

One step = Leapfrog kick+drift, periodic wrap + linked-cell binning, the pair traversal (forces,
Upot, virial) and the closing kick with sum m v^2, i.e. Simulation::simulateStep's hot path. The
other workloads: the 4M-molecule two-species slab (c3), the 512-box ensemble (batched), phase-space
file write and read of the 1M-molecule box (checkpoint), and 1M rigid two-centre molecules with
quaternion integration, optionally with point charges (rigid).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "LJ pair-interactions/s, 1M atoms, 1 B200: FP32/FP64-acc vs FP64 at ≤1e-5 err"
UNIT = "pair-interactions/s"
FLOPS_PER_PAIR = 31  # algorithmic flops per unordered pair within rc (FMA = 2): dr 3, r^2 5, 1/r^2 1, s^2 1, s^6 2, s^12 1, s^12-s^6 1, u 2, fac 3, f 3, virial 5, U 1


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 drop-in comparison leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=25.0, help="bound of the CPU baseline sample")
    ap.add_argument("--fcc-cells", type=int, default=64,
                    help="FCC unit cells per box edge (64 -> 1,048,576 molecules; smaller for profiling)")
    ap.add_argument("--pair-kernel", choices=["brick", "gather"], default="brick")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--skin", type=float, default=None,
                    help="Verlet skin of the step (0: cells and candidates rebuilt every step, as the reference); "
                         "default 0.4 for the single boxes (c2, c3), 0.3 for the others")
    ap.add_argument("--prune", type=float, default=0.15,
                    help="inner skin of the pruned lists of the single boxes (0: the steps evaluate the build lists)")
    ap.add_argument("--workload", choices=["c2", "c3", "batched", "checkpoint", "rigid", "adjoint"], default="c2",
                    help="c2: the 1M-molecule box (headline); c3: the 4M-molecule two-species slab; "
                         "batched: the 512-box ensemble; checkpoint: phase-space file write and read of the "
                         "1M-molecule box through the C ABI; rigid: a fluid of 1M two-centre LJ molecules")
    ap.add_argument("--boxes", type=int, default=512, help="boxes of the batched ensemble")
    ap.add_argument("--charges", action="store_true",
                    help="rigid workload: two-centre molecules with point charges +-0.5 (charge pairs besides LJ)")
    ap.add_argument("--loop-steps", type=int, default=20,
                    help="steps of the loop-over-single-box comparison of the batched workload")
    ap.add_argument("--adjoint-precision", choices=["fp64", "mixed"], default="fp64",
                    help="adjoint workload: arithmetic of the forward steps and the adjoint kernel")
    ap.add_argument("--liquid-steps", type=int, default=1500,
                    help="untimed steps before the liquid sub-record of the headline box (0: none)")
    args = ap.parse_args()
    if args.skin is None:
        args.skin = 0.4 if args.workload in ("c2", "c3") else 0.3
    return args


def workload_config(system, precision, skin=0.0, prune=0.0):
    if system.name.startswith("c3"):
        head = {"workload": f"lj_slab_two_species_{system.n}", "n_molecules": int(system.n),
                "box": [float(x) for x in system.length], "density": "liquid 0.70 (middle third), vapour 0.02",
                "temperature": 0.85, "cutoff": float(system.cutoff), "dt": float(system.dt),
                "potential": "LJ 12-6 truncated-shifted, A/B 50/50, sigma 1.0/0.9, eps 1.0/0.8, Lorentz-Berthelot"}
    else:
        head = {"workload": f"lj_fcc_{system.n}_rho0.75_T0.9_rc3.0", "n_molecules": int(system.n), "density": 0.75,
                "temperature": 0.9, "cutoff": float(system.cutoff), "dt": float(system.dt),
                "potential": "LJ 12-6 truncated-shifted, single species"}
    return {**head, "ensemble": "NVE",
            "pair_arithmetic": "fp32, fp64 accumulation" if precision == "mixed" else "fp64",
            "verlet_skin": skin,
            "pair_search": (f"candidate lists of radius rc + {skin} rebuilt (with the binning) when a molecule moved "
                            f"more than {skin / 2:g} since the last build; exact r^2 < rc^2 test on every pair")
            if skin > 0 else "cells rebuilt and candidates searched every step",
            "list_prune": (f"the steps evaluate the list entries within rc + {prune:g} at the last prune, re-pruned "
                           f"after each build and when the summed largest drifts reach {prune / 2:g}")
            if 0 < prune < skin else None,
            "l2": "not flushed: each step reads the whole state (molecule arrays and candidate lists, "
                  "several times the 126 MB L2); the timed steps run as one mdgpu_run_async"}


# ---------------------------------------------------------------------------- distributed plumbing

class Dist:
    def __init__(self, want):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock, power and clock-event reasons sampled during the timed region (read-only queries):
    an NVML polling thread every 5 ms (timed regions of a few ms still get samples), else
    nvidia-smi at 200 ms."""

    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.thread = None
        self.rows = []

    def _nvml_loop(self, nv, h):
        while not self.done:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except AttributeError:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((float(sm), float(mx), int(rs)))
            except Exception:
                pass
            time.sleep(0.005)

    def start(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            # NVML enumerates all GPUs; map the CUDA-visible index through the PCI bus id
            import torch

            pr = torch.cuda.get_device_properties(self.gpu)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            h = nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
            self.done = False
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            while not self.rows and self.thread.is_alive():
                time.sleep(0.002)
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.done = True
            self.thread.join(timeout=2)
            rows = self.rows[1:] if len(self.rows) > 1 else self.rows   # the first one precedes the region
            if not rows:
                return None
            reasons = sorted({k for r in rows for k, bit in self.REASONS.items() if r[2] & bit})
            return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                    "reasons": reasons, "samples": len(rows), "source": "NVML, 5 ms period"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms period"}


# ---------------------------------------------------------------------------- our arm

def make_system(rank: int, fcc_cells: int = 64, workload: str = "c2"):
    from madpac_b200 import workloads as W

    if workload == "c3":
        return W.config_c3(seed=3 + rank)
    if fcc_cells == 64:
        return W.config_c2(seed=2 + rank)
    return W.lj_fcc_box(fcc_cells, 0.75, 0.9, 2 + rank, 3.0, [W.Component(1.0, 1.0, 1.0, True)])


def time_device_resident(M, lc, system, steps, warmup, stream):
    """Device-resident steps: inputs in HBM, all `steps` steps enqueued as one mdgpu_run_async
    (consecutive steps share the kick between them), CUDA events on the library's stream around
    them. No L2 flush: every step reads the whole state (molecule arrays and candidate lists,
    several times the 126 MB L2). Returns (seconds, pairs, records, launches)."""
    import torch

    dt = system.dt
    lc.runAsync(warmup, dt)
    lc.readSteps(warmup)
    launches0 = lc.profileRead()[1][3]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    lc.runAsync(steps, dt)
    e1.record(stream)
    rec = lc.readSteps(steps)
    torch.cuda.synchronize()
    launches = int(lc.profileRead()[1][3] - launches0)
    seconds = e0.elapsed_time(e1) * 1e-3
    return seconds, float(rec[:, 3].sum()), rec, launches


def time_kernels(lc, system, steps):
    """Per-kernel-group device time (CUDA events on the library's stream) over `steps` steps."""
    lc.profileRead(reset=True)
    lc.profileEnable(True)
    lc.runAsync(steps, system.dt)
    rec = lc.readSteps(steps)
    t, cnt = lc.profileRead(reset=True)
    lc.profileEnable(False)
    return t, cnt, rec


def time_e2e(M, lc, system, steps, stream):
    """The same steps through the C ABI with host buffers: per step the caller uploads r, v from
    pinned host memory, runs mdgpu_step and downloads r, v, F and the step's scalars."""
    import torch

    n = system.n
    pin = lambda: torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    r, v, F = pin(), pin(), pin()
    st = lc.getParticles()
    r[:], v[:] = st["r"], st["v"]
    pairs = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        lc.setState(r=r, v=v)
        out = lc.step(system.dt, 1.0)
        pairs += out[3]
        st = lc.lib.mdgpu_get_particles(lc.h, n, None, None, r.ctypes.data, v.ctypes.data, F.ctypes.data)
        if st != 0:
            raise M.MdgpuError(st, lc.lib.mdgpu_last_error(lc.h).decode())
    e1.record(stream)
    torch.cuda.synchronize()
    seconds = e0.elapsed_time(e1) * 1e-3
    return seconds, pairs, 48 * n, 72 * n + 32


def time_e2e_run(M, lc, system, steps, stream):
    """The same steps as a user runs them through the C ABI: the state (r, v) copied in from pinned
    host memory (mdgpu_set_state), then `steps` calls of mdgpu_step, each returning its step record
    {Upot, virial, sum m v^2, pairs} to the host, then the final r, v, F copied out to pinned host
    memory. Returns (seconds, pairs, h2d bytes, d2h bytes) of the whole run."""
    import torch

    n = system.n
    pin = lambda: torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    r, v, F = pin(), pin(), pin()
    st = lc.getParticles()
    r[:], v[:] = st["r"], st["v"]
    pairs = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    lc.setState(r=r, v=v)
    for _ in range(steps):
        out = lc.step(system.dt, 1.0)
        pairs += out[3]
    st = lc.lib.mdgpu_get_particles(lc.h, n, None, None, r.ctypes.data, v.ctypes.data, F.ctypes.data)
    if st != 0:
        raise M.MdgpuError(st, lc.lib.mdgpu_last_error(lc.h).decode())
    e1.record(stream)
    torch.cuda.synchronize()
    seconds = e0.elapsed_time(e1) * 1e-3
    return seconds, pairs, 48 * n, 72 * n + 32 * steps


def count_pairs_host(system) -> float:
    from scipy.spatial import cKDTree

    tree = cKDTree(np.mod(system.r, system.length), boxsize=system.length)
    return (tree.count_neighbors(tree, system.cutoff) - system.n) / 2.0


def cpu_baseline(system, seconds_bound: float, pairs=None):
    """The reference's own CPU path on a bounded sample of the same workload: the reference
    harness (oracle/_ref/ref_driver, the unmodified MarDyn sources) when it was built, else the
    oracle's C restatement; single-threaded like the reference's sequential build."""
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if pairs is None:
        pairs = count_pairs_host(system)
    if os.path.exists(ref):
        from madpac_b200 import workloads as W

        tmp = tempfile.mkdtemp(prefix="mdref_")
        W.write_inp(system, os.path.join(tmp, "sys.inp"))
        W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
        nsteps = 3
        out = subprocess.run([ref, "--time", "sys.cfg", str(nsteps)], cwd=tmp, capture_output=True, text=True,
                             timeout=max(120.0, 8 * seconds_bound))
        sec = json.loads(out.stdout.strip().splitlines()[-1])["seconds_per_step"]
        kind, sample = "reference", f"{nsteps} steps of the full {system.n}-molecule box (after prepare_start)"
    else:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        o = O.Oracle(system)
        o.init()
        o.prepare_start()
        nsteps = 2
        t0 = time.perf_counter()
        for _ in range(nsteps):
            o.step()
        sec = (time.perf_counter() - t0) / nsteps
        kind, sample = "port", f"{nsteps} steps of the full {system.n}-molecule box on the oracle"
    return {"value": pairs / sec, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample,
            "seconds_per_step": sec, "pairs_per_step": pairs}


def run_ours(args, dist: Dist):
    import torch

    from madpac_b200 import mdgpu as M

    torch.cuda.set_device(dist.local)
    precision = M.MIXED if args.precision == "mixed" else M.FP64
    system = make_system(dist.rank, args.fcc_cells, args.workload)
    lc = M.LinkedCells.from_system(system, precision, device=dist.local)
    kernel = 0 if args.pair_kernel == "brick" else 1
    lc.setPairKernel(kernel)
    lc.update()
    lc.traversePairs()
    lc.setSkin(args.skin)
    lc.setListPrune(args.prune)
    stream = torch.cuda.ExternalStream(lc.stream())

    st0 = lc.getParticles()
    dist.barrier()
    clocks = ClockSampler(dist.local)
    clocks.start()
    seconds, pairs, rec, launches = time_device_resident(M, lc, system, args.steps, args.warmup, stream)
    clk = clocks.stop()
    dist.barrier()
    t_max = dist.max(seconds)
    pairs_all = dist.sum(pairs)
    value = pairs_all / t_max

    # kernel-level timing for the roofline: a profiled pass over the same steps (the start state
    # again, its forces, the warm-up steps, then the timed steps with events around each group)
    lc.setState(r=st0["r"], v=st0["v"])
    lc.update()
    lc.traversePairs()
    lc.setSkin(args.skin)
    lc.run(args.warmup, system.dt, record=False)
    builds0 = lc.skinBuilds() if args.skin > 0 else 0
    prunes0 = lc.listPrunes() if args.skin > 0 else 0
    tk, cnt, rec2 = time_kernels(lc, system, args.steps)
    rebuilds = (lc.skinBuilds() - builds0) if args.skin > 0 else args.steps
    prunes = (lc.listPrunes() - prunes0) if args.skin > 0 else 0
    # one rebinning pass alone: the same state set again before each of a few single steps, so that
    # every step rebins (the binning group then holds exactly one active k_rebuild per step)
    bin_pass_ms = None
    if args.skin > 0:
        st_b = lc.getParticles()
        lc.profileRead(reset=True)
        lc.profileEnable(True)
        for _ in range(5):
            lc.setState(r=st_b["r"], v=st_b["v"])
            lc.run(1, system.dt, record=False)
        bin_pass_ms = lc.profileRead(reset=True)[0][0] / 5
        lc.profileEnable(False)
    pair_ms = tk[1] / args.steps   # all pair launches of a step (the build is gated off in most steps)
    pairs_per_launch = float(rec2[:, 3].mean())
    fp32_peak, fp64_peak = M.device_peaks(dist.local)
    peak = fp32_peak if precision == M.MIXED else fp64_peak
    achieved = pairs_per_launch * FLOPS_PER_PAIR / (pair_ms * 1e-3) / 1e12
    traffic = None
    tf = os.path.join(ROOT, "profiles", "pair_kernel_traffic.json")
    if os.path.exists(tf):
        d = json.load(open(tf)).get(args.precision)
        if d:
            traffic = d["dram_bytes_per_pair"] * pairs_per_launch
    n = system.n
    bin_bytes = n * 184.0
    int_bytes = n * (124.0 + 76.0)
    hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs") if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0

    # end to end through the C ABI with host buffers
    e2e_each = None
    if args.no_e2e:
        e2e_value, h2d, d2h = None, 0, 0
    else:
        e2e_steps = max(3, args.steps)
        e2e_s, e2e_pairs, h2d_run, d2h_run = time_e2e_run(M, lc, system, e2e_steps, stream)
        e2e_s = dist.max(e2e_s)
        e2e_value = dist.sum(e2e_pairs) / e2e_s
        h2d, d2h = h2d_run / e2e_steps, d2h_run / e2e_steps
        # the whole state through the host every step (a caller that changes r, v between steps)
        each_steps = max(3, args.steps // 2)
        es, ep, eh, ed = time_e2e(M, lc, system, each_steps, stream)
        es = dist.max(es)
        e2e_each = {"value": dist.sum(ep) / es, "unit": UNIT, "h2d_bytes_per_step": eh, "d2h_bytes_per_step": ed,
                    "ms_per_step": es / each_steps * 1e3,
                    "note": "every step: r, v uploaded from pinned host memory, mdgpu_step, r, v, F downloaded"}

    out = {
        "metric": METRIC if args.workload == "c2" else "LJ pair-interactions/s, 4M-molecule two-species slab, 1 B200",
        "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair arithmetic, f64 accumulation" if precision == M.MIXED else "f64",
        "data": "synthetic (seeded FCC lattice, Maxwell-Boltzmann velocities)",
        "config": workload_config(system, args.precision, args.skin, args.prune),
        "steps_per_s": args.steps / t_max,
        "pairs_per_step": pairs / args.steps,
        "roofline": {"bound": "fp32" if precision == M.MIXED else "fp64", "kernel": "pair traversal",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": "measured FMA microbenchmark (mdgpu_device_peaks)",
                     "flops_per_pair": FLOPS_PER_PAIR, "launch_ms": pair_ms,
                     "timed": "pair kernels of one step (list evaluation, plus the list build in steps that "
                              "rebuild), CUDA events on the library stream; algorithmic flops = unordered pairs "
                              "within rc x 31"},
        "kernels_ms_per_step": {"binning": tk[0] / args.steps, "pairs": tk[1] / args.steps,
                                "integration": tk[2] / args.steps},
        "rebuilds_per_step": rebuilds / args.steps,
        "prunes_per_step": prunes / args.steps,
        "hbm_kernels": {"binning_gbs": (bin_bytes / (bin_pass_ms * 1e-3) / 1e9) if bin_pass_ms else
                                       bin_bytes * max(rebuilds, 1) / (tk[0] * 1e-3) / 1e9,
                        "binning_ms_per_pass": bin_pass_ms,
                        "binning_gated_us_per_step": ((tk[0] - rebuilds * bin_pass_ms) / max(args.steps - rebuilds, 1)
                                                      * 1e3) if bin_pass_ms else None,
                        "binning_note": "184 algorithmic bytes per molecule over one rebinning pass (wrap, bin, sort: "
                                        "k_rebuild), timed over steps that each rebin; the gated-off launch of the "
                                        "other steps is given apart" if bin_pass_ms else
                                        "per binning pass (wrap, bin, sort), over the binning time of the timed steps",
                        "integration_gbs": (int_bytes / (tk[2] / args.steps * 1e-3) / 1e9) if args.skin == 0 else None,
                        "integration_note": "in the Verlet-skin mode the closing kick, opening kick and drift run in "
                                            "the pair kernels' epilogue (no separate pass)" if args.skin > 0 else
                                            "fused closing/opening kick pass",
                        "peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "through the C ABI as a user runs it: r, v uploaded from pinned host memory, then "
                        "mdgpu_step per step with its record {Upot, virial, sum m v^2, pairs} read back to the "
                        "host each step, then the final r, v, F downloaded to pinned host memory; bytes per "
                        "step are the run's copies divided by its steps",
                "state_through_host_every_step": e2e_each},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if args.liquid_steps > 0 and dist.world == 1:
        # the same box once the lattice has melted: liquid_steps untimed steps on the device, then
        # the same number of timed steps as the headline, in this form and in the other precision
        # from the same liquid state
        lc.runAsync(args.liquid_steps, system.dt)
        lc.readSteps(args.liquid_steps)
        sl, pl, recl, _ = time_device_resident(M, lc, system, args.steps, 3, stream)
        st_l = lc.getParticles()
        other_l = M.FP64 if precision == M.MIXED else M.MIXED
        y = M.LinkedCells.from_system(system, other_l, device=dist.local)
        y.setPairKernel(kernel)
        y.setState(r=st_l["r"], v=st_l["v"])
        y.update()
        y.traversePairs()
        y.setSkin(args.skin)
        y.setListPrune(args.prune)
        so, po, _, _ = time_device_resident(M, y, system, args.steps, 3, torch.cuda.ExternalStream(y.stream()))
        y.close()
        ratio = (pl / sl) / (po / so)
        out["liquid"] = {
            "value": pl / sl, "unit": UNIT, "ms_per_step": sl / args.steps * 1e3, "steps": args.steps,
            "untimed_steps_before": args.liquid_steps + args.warmup + 2 * args.steps,
            "pairs_per_step": pl / args.steps,
            "fp64_dropin" if other_l == M.FP64 else "mixed": {"value": po / so, "ms_per_step": so / args.steps * 1e3},
            "mixed_over_fp64": ratio if precision == M.MIXED else 1.0 / ratio,
            "note": "the headline box after the untimed steps (the FCC lattice has melted); same timing as value"}
    if not args.no_compare and dist.world == 1:
        other = M.FP64 if precision == M.MIXED else M.MIXED
        csteps = min(args.steps, 50)

        def arm(prec, skin):
            x = M.LinkedCells.from_system(system, prec, device=dist.local)
            x.setPairKernel(kernel)
            x.update()
            x.traversePairs()
            x.setSkin(skin)
            x.setListPrune(args.prune if skin > 0 else 0.0)
            s2, p2, _, _ = time_device_resident(M, x, system, csteps, args.warmup,
                                                torch.cuda.ExternalStream(x.stream()))
            x.close()
            return {"value": p2 / s2, "ms_per_step": s2 / csteps * 1e3, "steps": csteps, "verlet_skin": skin}

        out["fp64_dropin" if other == M.FP64 else "mixed"] = arm(other, args.skin)
        if args.skin > 0:
            out["rebinned_every_step"] = {"mixed": arm(M.MIXED, 0.0), "fp64": arm(M.FP64, 0.0),
                                          "note": "the reference's sequence: wrap, binning and candidate search "
                                                  "in every step"}
        # accuracy of the mixed form against the FP64 drop-in on the evolved (thermalised)
        # positions the benchmark ended with; the FCC start has zero net forces by symmetry
        r_end = lc.getParticles()["r"]
        a = M.LinkedCells.from_system(system, M.MIXED, device=dist.local)
        b = M.LinkedCells.from_system(system, M.FP64, device=dist.local)
        a.setState(r=r_end)
        b.setState(r=r_end)
        a.update()
        b.update()
        ua, wa, _ = a.traversePairs()
        ub, wb, _ = b.traversePairs()
        Fa, Fb = a.getParticles()["F"], b.getParticles()["F"]
        rms = float(np.sqrt(np.mean(np.sum(Fb * Fb, axis=1))))
        out["accuracy_vs_fp64"] = {
            "force_err_rms": float(np.sqrt(np.mean(np.sum((Fa - Fb) ** 2, axis=1)))) / rms,
            "force_err_max": float(np.max(np.linalg.norm(Fa - Fb, axis=1))) / rms,
            "upot_rel": abs(ua - ub) / abs(ub), "virial_rel": abs(wa - wb) / abs(wb)}
        for x in (a, b):
            x.close()
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(system, args.cpu_seconds, pairs=float(rec[0, 3]))
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    lc.close()
    return out


# ---------------------------------------------------------------------------- batched ensemble

BATCH_METRIC = "LJ pair-interactions/s, 512-box ensemble (N 256-8192), 1 B200"


def _ref_box_time(args_):
    """Seconds per step of the reference harness on one box (runs in a worker process)."""
    ref, system, nsteps = args_
    from madpac_b200 import workloads as W

    tmp = tempfile.mkdtemp(prefix="mdref_")
    W.write_inp(system, os.path.join(tmp, "sys.inp"))
    W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
    out = subprocess.run([ref, "--time", "sys.cfg", str(nsteps)], cwd=tmp, capture_output=True, text=True, timeout=600)
    return json.loads(out.stdout.strip().splitlines()[-1])["seconds_per_step"]


def batched_cpu_baseline(systems, pairs_per_box, cores=8, sample_boxes=32, nsteps=20):
    """The reference harness on a sample of the boxes (every k-th by size), `cores` processes at a
    time, as 512 separate reference runs would go; throughput = sampled pairs*steps / wall time."""
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(ref):
        return {"value": None, "error": "oracle/_ref/ref_driver was not built"}
    import multiprocessing as mp

    order = np.argsort([s.n for s in systems])
    pick = order[:: max(1, len(systems) // sample_boxes)][:sample_boxes]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        secs = pool.map(_ref_box_time, [(ref, systems[k], nsteps) for k in pick])
    wall = time.perf_counter() - t0
    # wall includes process start and input writing; the per-box step times give the stepping rate
    step_rate = sum(pairs_per_box[k] for k in pick) / sum(secs) * cores
    return {"value": step_rate, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{len(pick)} of {len(systems)} boxes (every {max(1, len(systems) // sample_boxes)}-th by size), "
                      f"{nsteps} steps each, {cores} concurrent single-threaded reference processes; "
                      f"rate = sum(pairs per step) / sum(seconds per step) x {cores}",
            "wall_seconds": wall}


def run_batched(args, dist: Dist):
    import torch

    from madpac_b200 import mdgpu as M
    from madpac_b200 import workloads as W

    torch.cuda.set_device(dist.local)
    precision = M.MIXED if args.precision == "mixed" else M.FP64
    systems = W.config_c4(seed=4 + dist.rank, n_boxes=args.boxes)
    dt = systems[0].dt
    b = M.Batch.from_systems(systems, precision, device=dist.local)
    b.setSkin(args.skin)
    prep = b.prepare()
    best, cand_ms = b.autotune(dt, trial_steps=5)
    b.run(args.warmup, dt, record=False)
    dist.barrier()
    clocks = ClockSampler(dist.local)
    clocks.start()
    recs = b.run(args.steps, dt)
    clk = clocks.stop()
    seconds = dist.max(b.lastRunMs() * 1e-3)
    pairs = float(recs[:, :, 3].sum())
    value = dist.sum(pairs) / seconds
    ntot = sum(s.n for s in systems)

    # end to end: host arrays in, records and the final state out, through the batch C ABI
    e2e = None
    if not args.no_e2e:
        st = b.getParticles()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.setParticles(st["id"], st["cid"], st["r"], st["v"])
        b.prepare()
        r2 = b.run(args.steps, dt)
        b.getParticles()
        e2e_s = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.sum(float(r2[:, :, 3].sum())) / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": (60 * ntot) / args.steps, "d2h_bytes_per_step": 32 * len(systems) + 84 * ntot / args.steps,
               "note": "one upload of id, cid, r, v and one download of the final state per run of `steps` steps"}

    # the comparison: one single-box context per box, stepped in a host loop (own stream each)
    loop = None
    if args.loop_steps > 0:
        ctxs = []
        for s in systems:
            lc = M.LinkedCells.from_system(s, precision, device=dist.local)
            lc.update()
            lc.traversePairs()
            lc.setSkin(args.skin)
            ctxs.append(lc)
        for lc in ctxs:
            lc.runAsync(2, dt)
        for lc in ctxs:
            lc.readSteps(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.loop_steps):
            for lc in ctxs:
                lc.runAsync(1, dt)
        lpairs = 0.0
        for lc in ctxs:
            lpairs += float(lc.readSteps(args.loop_steps)[:, 3].sum())
        torch.cuda.synchronize()
        lsec = time.perf_counter() - t0
        launches = sum(lc.profileRead()[1][3] for lc in ctxs)
        for lc in ctxs:
            lc.close()
        loop = {"value": lpairs / lsec, "ms_per_step": lsec / args.loop_steps * 1e3, "steps": args.loop_steps,
                "timing": "host wall clock around the loop, synchronised at both ends",
                "launches_per_step": launches / (args.loop_steps + 2)}
    out = {
        "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": seconds / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair arithmetic, f64 accumulation" if precision == M.MIXED else "f64",
        "data": "synthetic (seeded FCC subsets, Maxwell-Boltzmann velocities)",
        "config": {"workload": f"c4_{len(systems)}_boxes", "n_boxes": len(systems), "n_molecules": ntot,
                   "n_min": min(s.n for s in systems), "n_max": max(s.n for s in systems), "cutoff": 2.5,
                   "dt": dt, "ensemble": "NVE", "verlet_skin": args.skin,
                   "skin_builds": b.skinBuilds() if args.skin > 0 else None, "tiles": {"list_cap": best[0], "ctas_per_sm": best[1],
                                                         "brick_queue": best[2]},
                   "autotune_ms_per_step": {f"cap{c}_ctas{t}_q{q}": v for (c, t, q), v in cand_ms.items()},
                   "l2": f"working set larger than L2 ({ntot * 200 / 1e6:.0f} MB of molecule arrays)"},
        "steps_per_s": args.steps / seconds, "box_steps_per_s": len(systems) * args.steps / seconds,
        "pairs_per_step": pairs / args.steps,
        "timing": "CUDA events around the graph launch of all timed steps",
        "gpu_launches": args.steps,
        "e2e": e2e, "loop_single_box": loop,
        "speedup_vs_loop": (value / loop["value"]) if loop else None,
        "clocks": clk,
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = batched_cpu_baseline(systems, prep[:, 3])
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    b.close()
    return out


# ---------------------------------------------------------------------------- phase-space files

def run_checkpoint(args, dist: Dist):
    """Write (the reference's checkpoint layout, 6 digits, and 17 digits) and read back the
    1,048,576-molecule box through mdgpu_write_checkpoint / mdgpu_read_phase_space: host wall clock
    around each call, device transfers included; beside it the reference writing the same box's
    checkpoint (Domain::writeCheckpoint via oracle/_ref/ref_driver --time-checkpoint)."""
    import torch

    from madpac_b200 import mdgpu as M
    from madpac_b200 import workloads as W

    torch.cuda.set_device(dist.local)
    system = make_system(dist.rank, args.fcc_cells)
    lc = M.LinkedCells.from_system(system, M.FP64, device=dist.local)
    tmp = tempfile.mkdtemp(prefix="mdck_")
    res = {}
    for digits in (6, 17):
        path = os.path.join(tmp, f"ck{digits}.txt")
        lc.writeCheckpoint(path, 0.0, system.temperature, digits=digits if digits != 6 else 0)   # warm-up
        times_w, times_r = [], []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            lc.writeCheckpoint(path, 0.0, system.temperature, digits=digits if digits != 6 else 0)
            times_w.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            lc.readPhaseSpace(path)
            torch.cuda.synchronize()
            times_r.append(time.perf_counter() - t0)
        size = os.path.getsize(path)
        res[digits] = {"write_s": statistics.median(times_w), "read_s": statistics.median(times_r), "bytes": size}
    n = system.n
    w6 = res[6]["write_s"]
    out = {
        "metric": "phase-space checkpoint write, molecules/s (1M-molecule box, C ABI, reference layout)",
        "value": n / w6, "unit": "molecules/s", "n_gpus": dist.world, "steps": args.steps, "warmup": 1,
        "ms_per_step": w6 * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded FCC lattice, Maxwell-Boltzmann velocities)",
        "config": {"workload": "checkpoint_1048576", "n_molecules": n, "format": "ICRVQD",
                   "timing": "host wall clock per call (median of steps), device-to-host and host-to-device "
                             "copies included; file on the host's local disk"},
        "write_6_digits": {"seconds": w6, "molecules_per_s": n / w6, "bytes": res[6]["bytes"],
                           "MB_per_s": res[6]["bytes"] / w6 / 1e6},
        "read_6_digits": {"seconds": res[6]["read_s"], "molecules_per_s": n / res[6]["read_s"]},
        "write_17_digits": {"seconds": res[17]["write_s"], "molecules_per_s": n / res[17]["write_s"],
                            "bytes": res[17]["bytes"]},
        "read_17_digits": {"seconds": res[17]["read_s"], "molecules_per_s": n / res[17]["read_s"]},
        "threads": os.cpu_count(),
    }
    lc.close()
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if dist.rank == 0 and not args.no_cpu_baseline and os.path.exists(ref):
        W.write_inp(system, os.path.join(tmp, "sys.inp"))
        W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
        r = subprocess.run([ref, "--time-checkpoint", "sys.cfg", "ref_ck.txt"], cwd=tmp, capture_output=True, text=True,
                           timeout=600)
        secs = json.loads(r.stdout.strip().splitlines()[-1])["seconds"]
        out["cpu_baseline"] = {"value": n / secs, "unit": "molecules/s", "cores": 1, "kind": "reference",
                               "sample": "Domain::writeCheckpoint of the full box after prepare_start", "seconds": secs}
    shutil.rmtree(tmp, ignore_errors=True)
    return out


# ---------------------------------------------------------------------------- rigid molecules

RIGID_METRIC = "LJ centre-pair interactions/s, 1M two-centre LJ molecules (2CLJ), 1 B200"
RIGID_Q_METRIC = "site-pair interactions/s (LJ + charge pairs), 1M two-centre LJ molecules with point charges, 1 B200"
RIGID_UNIT = "centre-pair interactions/s"
# algorithmic flops per LJ centre pair (FMA = 2): site distance 6, r^2 5, 1/r^2 1, s^2 1, s^6 2, s^12 1,
# s^12-s^6 1, u 2, fac 3, f 3, virial drm.f 5, torque d x f 9, U 1
FLOPS_PER_CENTRE_PAIR = 40
# per charge pair: site distance 6, r^2 5, 1/r^2 1, sqrt 1, u 2, fac 1, f 3, virial 5, torque 9, U 1
FLOPS_PER_CHARGE_PAIR = 34


def run_rigid(args, dist: Dist):
    """Steps of a fluid of rigid two-centre LJ molecules (workloads.config_2clj: 4 fcc_cells^3
    molecules, elongation 0.5, rho 0.3, T 2.0, rc 3.0 on the molecule centres, dt 0.002): Leapfrog with
    quaternions, wrap and binning of the centres, site rotation, the centre-pair forces and torques,
    closing kicks. Every step evaluates all centre pairs of every molecule pair within rc (4 here)."""
    import torch

    from madpac_b200 import mdgpu as M
    from madpac_b200 import workloads as W

    torch.cuda.set_device(dist.local)
    system = W.config_2clj(seed=6 + dist.rank, n_cells=args.fcc_cells, charged=args.charges)
    n = system.n
    dt = system.dt
    ncentre = 8 if args.charges else 4   # LJ centre pairs (+ charge pairs) per molecule pair

    def device_run(precision, steps, warmup, skin=args.skin):
        lc = M.RigidLinkedCells.from_system(system, precision, device=dist.local)
        lc.update()
        lc.traversePairs()
        if skin > 0.0:
            lc.setSkin(skin)
        lc.run(warmup, dt, record=False)
        b0 = lc.skinBuilds() if skin > 0.0 else 0
        stream = torch.cuda.ExternalStream(lc.stream())
        l0 = lc.launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        rec = lc.run(steps, dt)
        e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3
        launches = lc.launches() - l0
        device_run.builds = (lc.skinBuilds() - b0) if skin > 0.0 else None
        # kernel groups over a few more steps
        lc.profileRead(reset=True)
        lc.profileEnable(True)
        kk = max(3, min(steps, 20))
        krec = lc.run(kk, dt)
        t, cnt = lc.profileRead(reset=True)
        lc.profileEnable(False)
        return lc, sec, rec, launches, t / kk, cnt, krec

    clocks = ClockSampler(dist.local)
    clocks.start()
    lc, sec, rec, launches, groups_ms, cnt, krec = device_run(M.MIXED, args.steps, args.warmup)
    builds = device_run.builds
    clk = clocks.stop()
    sec = dist.max(sec)
    mol_pairs = float(rec[:, 4].sum())
    value = dist.sum(mol_pairs * ncentre) / sec
    fp32_peak, fp64_peak = M.device_peaks(dist.local)
    pair_ms = float(groups_ms[1])
    pairs_per_step = float(krec[:, 4].mean())
    flops_per_mol_pair = 4 * FLOPS_PER_CENTRE_PAIR + (4 * FLOPS_PER_CHARGE_PAIR if args.charges else 0)
    achieved = pairs_per_step * flops_per_mol_pair / (pair_ms * 1e-3) / 1e12

    # e2e: host arrays in (id, cid, r, v, q, D), one run of `steps` steps, the final state out
    st = lc.getParticles()
    pin = lambda shape, dt_=np.float64: torch.empty(shape, dtype=getattr(torch, np.dtype(dt_).name),  # noqa: E731
                                                    pin_memory=True).numpy()
    hr, hv, hq, hD = pin((n, 3)), pin((n, 3)), pin((n, 4)), pin((n, 3))
    hr[:], hv[:], hq[:], hD[:] = st["r"], st["v"], st["q"], st["D"]
    e2e_steps = max(3, args.steps // 2)
    stream = torch.cuda.ExternalStream(lc.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    lc.addParticles(st["id"], st["cid"], hr, hv, hq, hD)
    lc.update()
    lc.traversePairs()
    erec = lc.run(e2e_steps, dt)
    out_state = lc.getParticles()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_sec = e0.elapsed_time(e1) * 1e-3
    e2e_value = float(erec[:, 4].sum()) * ncentre / e2e_sec
    h2d = n * (8 + 4 + 8 * 14)
    d2h = n * (8 + 4 + 8 * 22) + 40 * e2e_steps
    del out_state
    lc.close()

    # the FP64 form of the same steps
    fp64 = None
    rebinned = None
    if not args.no_compare:
        lc64, sec64, rec64, *_ = device_run(M.FP64, args.steps, args.warmup)
        sec64 = dist.max(sec64)
        fp64 = {"value": dist.sum(float(rec64[:, 4].sum()) * ncentre) / sec64, "ms_per_step": sec64 / args.steps * 1e3}
        lc64.close()
        if args.skin > 0.0:
            # the reference's sequence: binning and candidate search every step
            lcb, secb, recb, *_ = device_run(M.MIXED, args.steps, args.warmup, skin=0.0)
            secb = dist.max(secb)
            rebinned = {"value": dist.sum(float(recb[:, 4].sum()) * ncentre) / secb,
                        "ms_per_step": secb / args.steps * 1e3}
            lcb.close()

    out = {
        "metric": RIGID_Q_METRIC if args.charges else RIGID_METRIC, "value": value,
        "unit": "site-pair interactions/s" if args.charges else RIGID_UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 centre-pair arithmetic, f64 accumulation",
        "data": "synthetic (seeded FCC lattice of molecule centres, random orientations, Maxwell-Boltzmann "
                "translational and rotational velocities)",
        "config": {"workload": f"rigid_{system.name}", "n_molecules": n, "centres_per_molecule": 2,
                   "charges_per_molecule": 2 if args.charges else 0, "elongation": 0.5,
                   "density": 0.3, "temperature": 2.0, "cutoff": float(system.cutoff), "dt": dt, "ensemble": "NVE",
                   "potential": "2CLJ, LJ 12-6 truncated-shifted per centre pair" +
                                (", point charges +-0.5 at z = +-0.35 (plain Coulomb)" if args.charges else "") +
                                ", cutoff on the molecule centres",
                   "pair_search": (f"lists of the molecule pairs within rc + {args.skin:g}, rebuilt (with the "
                                   f"binning) when a centre moved more than {args.skin / 2:g}; exact rc test on every "
                                   "list entry") if args.skin > 0.0 else "cells rebuilt and candidates searched every step",
                   "l2": f"not flushed: each step reads the whole state ({n * 230 / 1e6:.0f} MB of molecule arrays, "
                         "above the 126 MB L2)"},
        "molecule_pairs_per_step": mol_pairs / args.steps,
        "timing": "CUDA events on the library stream around one mdgpu_rigid_run of the timed steps",
        "gpu_launches": int(launches),
        "kernel_ms_per_step": {"binning": float(groups_ms[0]), "site_rotation_and_pairs": pair_ms,
                               "integration": float(groups_ms[2])},
        "roofline": {"bound": "fp32", "kernel": "site rotation + centre-pair forces", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                     "peak_source": "measured FMA microbenchmark (mdgpu_device_peaks)",
                     "flops_per_molecule_pair": flops_per_mol_pair,
                     "timed": "k_rigid_sites + k_rigid_pairs per step, CUDA events on the library stream"},
        "fp64": fp64,
        "speedup_vs_fp64": (value / fp64["value"]) if fp64 else None,
        "rebuilds_per_step": (builds / args.steps) if builds is not None else None,
        "rebinned_every_step": rebinned,
        "e2e": {"value": e2e_value, "unit": RIGID_UNIT, "h2d_bytes_per_step": h2d / e2e_steps,
                "d2h_bytes_per_step": d2h / e2e_steps,
                "note": f"one upload of id, cid, r, v, q, D and one download of the final state per run of "
                        f"{e2e_steps} steps, plus the step records"},
        "clocks": clk,
    }
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline and os.path.exists(ref):
        tmp = tempfile.mkdtemp(prefix="mdrig_")
        W.write_inp(system, os.path.join(tmp, "sys.inp"))
        W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
        probe = subprocess.run([ref, "--time", "sys.cfg", "1"], cwd=tmp, capture_output=True, text=True, timeout=900)
        t1 = json.loads(probe.stdout.strip().splitlines()[-1])["seconds_per_step"]
        k = max(1, min(args.steps, int(args.cpu_seconds / max(t1, 1e-3))))
        r = subprocess.run([ref, "--time", "sys.cfg", str(k)], cwd=tmp, capture_output=True, text=True, timeout=900)
        secs = json.loads(r.stdout.strip().splitlines()[-1])["seconds_per_step"]
        out["cpu_baseline"] = {"value": float(rec[0, 4]) * ncentre / secs, "unit": RIGID_UNIT, "cores": 1,
                               "kind": "reference", "seconds_per_step": secs,
                               "sample": f"{k} steps of the full {n}-molecule box (bounded to ~{args.cpu_seconds:g} s) "
                                         "after prepare_start and one untimed probe step, single-threaded"}
        shutil.rmtree(tmp, ignore_errors=True)
    return out


# ---------------------------------------------------------------------------- reference arm

def run_reference(args, dist: Dist):
    """The reference's own CPU implementation (unmodified MarDyn sources, sequential build) on the
    same workload; rank 0 only."""
    system = make_system(0, args.fcc_cells)
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    pairs = count_pairs_host(system)
    if os.path.exists(ref):
        from madpac_b200 import workloads as W

        tmp = tempfile.mkdtemp(prefix="mdref_")
        W.write_inp(system, os.path.join(tmp, "sys.inp"))
        W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
        # bounded: at most ~150 s of stepping
        probe = subprocess.run([ref, "--time", "sys.cfg", "1"], cwd=tmp, capture_output=True, text=True)
        t1 = json.loads(probe.stdout.strip().splitlines()[-1])["seconds_per_step"]
        nsteps = max(1, min(args.steps, int(150.0 / max(t1, 1e-3))))
        out = subprocess.run([ref, "--time", "sys.cfg", str(nsteps)], cwd=tmp, capture_output=True, text=True)
        sec = json.loads(out.stdout.strip().splitlines()[-1])["seconds_per_step"]
        kind, sample = "reference", (f"{nsteps} timed steps (of {args.steps} asked; bounded to ~150 s) of the full "
                                     f"{system.n}-molecule box, after prepare_start and one untimed probe step")
    else:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        o = O.Oracle(system)
        o.init()
        o.prepare_start()
        for _ in range(min(args.warmup, 1)):
            o.step()
        nsteps = max(1, min(args.steps, 10))
        t0 = time.perf_counter()
        for _ in range(nsteps):
            o.step()
        sec = (time.perf_counter() - t0) / nsteps
        kind, sample = "port", f"{nsteps} steps of the full {system.n}-molecule box on the C restatement"
    value = pairs / sec
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**{k: v for k, v in workload_config(system, "fp64").items() if k != "l2"},
                       "l2": "the reference's own CPU path (single-threaded, sequential build)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


class _Solo:
    """Rank bookkeeping without a process group (the reference arm runs on rank 0 only)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))


ADJ_METRIC = "LJ trajectory gradients/s, 16,384-molecule two-species box, 50 Leapfrog steps, 1 B200"
FLOPS_PER_ADJ_PAIR = 60  # FP64 flops per ordered pair of the adjoint kernel (FMA = 2)


def run_adjoint(args, dist: Dist):
    """Gradient of L = sum |F - F_t|^2 + 0.1 (U - U_t)^2 after 50 NVE steps (checkpoints every 10)
    with respect to the start positions, velocities and eps_ab / sigma_ab, on the 16,384-molecule
    two-species box (targets at eps_AB x 1.1, sigma_AB x 0.95), forward and backward on the device."""
    import torch

    from madpac_b200 import mdgpu as M
    from madpac_b200 import workloads as W
    from madpac_b200.trajectory import TrajectoryAdjoint

    torch.cuda.set_device(dist.local)
    precision = M.MIXED if args.adjoint_precision == "mixed" else M.FP64
    s = W.config_c5(seed=5 + dist.rank)
    lc = M.LinkedCells.from_system(s, M.FP64, device=dist.local)
    lc.update()
    lc.traversePairs()
    lc.run(100, s.dt, record=False)
    st = lc.getParticles()
    lc.close()
    s.r, s.v = st["r"], st["v"]
    # targets: the same molecules with the cross-species pair at eps x 1.1, sigma x 0.95
    t = W.System(**{**s.__dict__})
    t.mix = np.array(s.mix, dtype=np.float64).reshape(-1, 2) * np.array([[1.1, 0.95]])
    tl = M.LinkedCells.from_system(t, M.FP64, device=dist.local)
    tl.update()
    Ut, _, _ = tl.traversePairs()
    Ft = tl.getParticles()["F"]
    tl.close()
    steps, every = 50, 10
    tr = TrajectoryAdjoint(s, steps, every, device=dist.local, precision=precision)
    stream = torch.cuda.ExternalStream(tr.lc.stream())

    def one():
        r, v, F, U = tr.forward(s.r, s.v)
        return tr.backward(2 * (F - Ft), 0.2 * (U - Ut))

    for _ in range(max(args.warmup, 1)):
        one()
    reps = max(1, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    clocks = ClockSampler(dist.local)
    clocks.start()
    torch.cuda.synchronize()
    launches0 = tr.lc.profileRead()[1][3]
    e0.record(stream)
    for _ in range(reps):
        gr, gv, ge, gs = one()
    e1.record(stream)
    launches = int(tr.lc.profileRead()[1][3] - launches0)
    torch.cuda.synchronize()
    clk = clocks.stop()
    sec = dist.max(e0.elapsed_time(e1) * 1e-3)
    # adjoint kernel alone: CUDA events around its launches in one more (profiled) backward pass
    tr.lc.profileEnable(True)
    one()
    tr.lc.profileEnable(False)
    adj_ms, adj_launches = tr.lc.trajAdjointTime()
    tr.lc.setState(r=s.r)
    tr.lc.update()
    _, _, upairs = tr.lc.traversePairs()
    fp32_peak, fp64_peak = M.device_peaks(dist.local)
    peak = fp32_peak if precision == M.MIXED else fp64_peak
    flops_launch = 2.0 * upairs * FLOPS_PER_ADJ_PAIR
    achieved = flops_launch / (adj_ms / max(adj_launches, 1) * 1e-3) / 1e12
    tr.close()
    out = {
        "metric": ADJ_METRIC, "value": dist.sum(reps / sec), "unit": "trajectory gradients/s", "n_gpus": dist.world,
        "steps": reps, "warmup": max(args.warmup, 1), "ms_per_step": sec / reps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if precision == M.FP64 else "f32 pair terms, f64 sums",
        "data": "synthetic (seeded FCC lattice thermalised 100 steps, Maxwell-Boltzmann velocities)",
        "config": {"workload": "two-species LJ box, N=16,384, rho 0.8, T 1.0, A/B 50/50 (sigma_B 0.9, eps_B 0.8), "
                               "rc 2.5, dt 0.002; L = sum|F - F_t|^2 + 0.1 (U - U_t)^2 after 50 NVE steps, targets "
                               "at eps_AB x 1.1, sigma_AB x 0.95; gradients in r0, v0, eps_ab, sigma_ab",
                   "checkpoint_every": every, "trajectory_steps": steps,
                   "l2": "not flushed (one gradient = 50 forward + 50 recomputed + 50 backward steps)"},
        "ms_per_gradient": sec / reps * 1e3, "md_steps_per_gradient": 3 * steps,
        "roofline": {"bound": "fp64" if precision == M.FP64 else "fp32", "kernel": "adjoint (vector-Jacobian product)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                     "peak_source": "measured FMA microbenchmark (mdgpu_device_peaks)",
                     "flops_per_ordered_pair": FLOPS_PER_ADJ_PAIR, "launch_ms": adj_ms / max(adj_launches, 1),
                     "launches": adj_launches},
        "gradient_norms": {"dL_dr0_rms": float(np.sqrt(np.mean(gr ** 2))), "dL_deps_AB": float(ge[0, 1]),
                           "dL_dsigma_AB": float(gs[0, 1])},
        "gpu_launches": launches, "launches_per_gradient": launches / reps, "clocks": clk,
        "e2e": {"value": dist.sum(reps / sec), "unit": "trajectory gradients/s",
                "h2d_bytes_per_step": 2 * 48 * s.n, "d2h_bytes_per_step": 4 * 24 * s.n,
                "note": "each gradient uploads r0, v0 and gF and downloads the final state and dL/dr0, dL/dv0"},
    }
    return out


def main():
    args = parse()
    if args.impl == "reference":
        solo = _Solo()
        if solo.rank == 0:
            print(json.dumps(run_reference(args, solo)), flush=True)
        return
    dist = Dist(args.gpus)
    if args.workload == "batched":
        out = run_batched(args, dist)
    elif args.workload == "checkpoint":
        out = run_checkpoint(args, dist)
    elif args.workload == "rigid":
        out = run_rigid(args, dist)
    elif args.workload == "adjoint":
        out = run_adjoint(args, dist)
    else:
        out = run_ours(args, dist)
    if dist.rank == 0:
        print(json.dumps(out), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
