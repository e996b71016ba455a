"""Benchmark of the B200 FARGO3D hydro step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload p3disof|fargo2d] [--precision fp64|fp32]

A step is one hydro step (main.c:361-448 of the reference) of the workload.
Default workload: the 3D spherical isothermal disk with one planet
(setups/p3disof physics, 512 x 256 x 48 zones, FP64 plain path).  Inputs are
seeded synthetic disks of that shape (no dataset is involved).

value       cell-updates/s of the whole job, device-timed with CUDA events on
            the disk's stream, state resident in HBM (max over ranks)
e2e         same metric through the public API from pinned host buffers:
            H2D of the initial state, K steps, D2H of the final state
roofline    the dominant launch of a step against the measured HBM copy peak
cpu_baseline  the reference's own C sources (oracle/_ref, built from the
            reference tree) timed on this host's cores on a bounded sample

Under torchrun each rank advances its own disk (independent disks: weak
scaling, no collective in the data path).  `--impl reference` times the
reference's CPU implementation of the same workload on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
# compulsory state words per cell-update (read rho, cs, v; write rho, v)
ALG_WORDS = {"2d": 7, "3d": 9}
# compulsory words per active cell of each launch group
LAUNCH_WORDS = {
    "2d": {"rowsum": 1, "cfl": 4, "sources": 6, "bnd_vtemp": 0, "rowsum_vtemp": 1,
           "sweep_cols": 8, "sweep_x": 11, "newvel": 8, "bnd": 0},
    "3d": {"rowsum": 1, "cfl": 5, "sources": 8, "bnd_vtemp": 0, "rowsum_vtemp": 1,
           "sweep_cols": 26, "sweep_x": 15, "newvel": 11, "bnd": 0},
}
KERNELS_PER_GROUP = {"2d": {"sweep_cols": 1, "bnd": 1, "bnd_vtemp": 1},
                     "3d": {"sweep_cols": 2, "bnd": 2, "bnd_vtemp": 2}}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(name: str):
    from fargo3d_b200 import config_fargo2d, config_p3disof
    if name == "fargo2d":
        return config_fargo2d(384, 128, seed=0), "fargo2d 384x128 (2D cylindrical, 1 planet, nu=1e-5)"
    return config_p3disof(512, 256, 48, seed=0), "p3disof 512x256x48 (3D spherical, 1 planet, nu=1e-5)"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch
    from fargo3d_b200 import Disk, initial_state
    torch.cuda.set_device(local_rank)
    cfg, wname = workload(args.workload)
    dim = "3d" if cfg.is3d else "2d"
    esz = 8 if args.precision == "fp64" else 4
    init = initial_state(cfg)
    d = Disk(cfg, args.precision, device=local_rank)
    d.set_state(*init)
    d.initialize()
    stream = torch.cuda.ExternalStream(d.stream)
    for _ in range(args.warmup):
        d.step()
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            d.step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms = float(t.item())
        tdist.barrier()
    cells = cfg.active_cells
    value = cells * args.steps * world / (ms / 1e3)
    # per-launch timing of two extra steps (dominant kernel for the roofline)
    from fargo3d_b200 import _abi
    import ctypes as C
    L = _abi.lib()
    L.fb_disk_profile(d._h, 1)
    prof = {}
    for _ in range(2):
        d.step()
        msa = (C.c_float * 32)()
        nms = (C.c_char_p * 32)()
        n = L.fb_disk_profile_read(d._h, msa, nms, 32)
        for i in range(n):
            prof.setdefault(nms[i].decode(), []).append(msa[i])
    L.fb_disk_profile(d._h, 0)
    prof = {k: float(np.mean(v)) for k, v in prof.items() if k != "host_scalars"}
    launches_per_step = sum(KERNELS_PER_GROUP[dim].get(k, 1) for k in prof)
    dom = max((k for k in prof if k in LAUNCH_WORDS[dim]), key=lambda k: prof[k])
    hbm, peak_kind = peaks()
    dom_bytes = LAUNCH_WORDS[dim][dom] * esz * cells
    achieved = dom_bytes / (prof[dom] / 1e3) / 1e9
    # end-to-end through the public API from pinned host buffers
    pinned = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in init]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d2 = Disk(cfg, args.precision, device=local_rank)
    d2.set_state(*[p.numpy() for p in pinned])
    d2.initialize()
    for _ in range(args.steps):
        d2.step()
    st = d2.state()
    t_e2e = time.perf_counter() - t0
    d2.close()
    ncell = int(np.prod(cfg.shape))
    h2d = 5 * ncell * 8 / args.steps
    d2h = (4 * ncell * 8) / args.steps + 8
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32", "data": "synthetic",
        "config": {"workload": wname, "precision": args.precision, "active_cells": cells,
                   "parallelism": "independent disks, one per GPU" if world > 1 else "single disk",
                   "l2": "state (%d MB) larger than L2 (126 MB); no flush needed" %
                         (ncell * esz * 5 // 2 ** 20)},
        "e2e": {"value": cells * args.steps * world / t_e2e, "unit": "cell-updates/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": None,
                     "alg_bytes_per_launch": dom_bytes, "launch_ms": prof[dom],
                     "step_alg_frac": ALG_WORDS[dim] * esz * cells * args.steps * world / (ms / 1e3) / 1e9 / hbm},
        "launch_ms": prof,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
        "rho_check": float(np.sum(st["rho"])),
    }
    d.close()
    return line


def cpu_reference_time(cfg, steps):
    """Time the reference's own sources (oracle/_ref) on `steps` hydro steps of
    the workload, single process on one core (the reference has no threading
    and MPI is not available on this image)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fargo3d_b200 import initial_state
    kind = "reference"
    try:
        d = pyoracle.Disk(cfg, "ref")
    except FileNotFoundError:
        pyoracle.build()
        try:
            d = pyoracle.Disk(cfg, "ref")
        except FileNotFoundError:
            d = pyoracle.Disk(cfg, "oracle")
            kind = "port"
    d.set_state(*initial_state(cfg))
    d.initialize()
    d.step()  # warm the caches / first-touch
    t0 = time.perf_counter()
    for _ in range(steps):
        d.step()
    t = time.perf_counter() - t0
    d.close()
    return cfg.active_cells * steps / t, kind, t


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="p3disof", choices=["p3disof", "fargo2d"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--cpu-steps", type=int, default=0, help="reference steps for cpu_baseline (0: auto)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg (profiling runs)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    cfg, wname = workload(args.workload)
    cpu_steps = args.cpu_steps or (2 if cfg.is3d else 400)
    if args.impl == "reference":
        if rank != 0:
            return
        steps = max(1, min(args.steps, cpu_steps))
        v, kind, t = cpu_reference_time(cfg, steps)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": world,
                "steps": steps, "warmup": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                "config": {"workload": wname, "precision": "fp64"},
                "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": kind,
                                 "sample": "%d hydro steps of the full workload, one process on one core (%s)"
                                           % (steps, cpu_model())},
                "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
    line = run_ours(args, rank, world, local_rank)
    if rank == 0 and not args.no_cpu:
        v, kind, t = cpu_reference_time(cfg, cpu_steps)
        line["cpu_baseline"] = {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": kind,
                                "sample": "%d hydro steps of the full workload, one process on one core, %.1f s (%s)"
                                          % (cpu_steps, t, cpu_model())}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
