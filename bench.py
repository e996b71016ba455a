"""Benchmark of the B200 FARGO3D hydro step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|p3disof|fargo2d] [--precision fp64|fp32]

A step is one hydro step (main.c:361-448 of the reference) of every disk of
the workload.  Workloads (seeded synthetic disks of the stated shapes; no
dataset is involved):
  batched  (default) 64 independent 2D disks of uneven sizes (N_phi in
           {128..1024}, N_r in {64..512}; alpha viscosity, one planet each),
           FP32 transport and sources with FP64 shift / means / planets,
           every stage one launch over all disks, steps replayed from a CUDA
           graph.  The plain FP64 path on the same disks, one disk at a time,
           is measured beside it ("fp64_plain").
  p3disof  one 3D spherical disk 512 x 256 x 48 (plain path, --precision)
  fargo2d  one 2D cylindrical disk 384 x 128 (plain path, --precision)
  multifluid  one 2D disk 768 x 256 with gas + 4 dust species coupled by
           implicit drag (plain path, --precision)
  serving  the continuous-batching server: --requests requests (default
           100) arriving as a Poisson process (--rate, 20/s), sizes
           {256x64, 512x128, 1024x256, 2048x512} weighted {.4,.3,.2,.1}, each
           run for --orbits orbits (default 0.25, a bounded stand-in for the
           50-orbit requests), FP32; reports p50/p99 request latency beside
           throughput.  The default (batched) run adds the same measurement
           as its "serving" object.

value       cell-updates/s of the whole job, device-timed with CUDA events on
            the launching stream, state resident in HBM (max over ranks)
e2e         the same through the public API from pinned host buffers: create,
            H2D of the initial state, K steps, D2H of the final state (the
            median of five such runs)
roofline    the dominant launch group of a step against the measured HBM copy
            peak (MEASURED_PEAKS.json)
cpu_baseline  the reference's own C sources (oracle/_ref, built from the
            reference tree) timed on this host on a bounded sample

Multi-GPU: `--gpus N` without a torchrun environment starts N ranks itself
(torch.distributed.run on 127.0.0.1).  The batched workload is then ONE list
of 64 x N disks split over the ranks by the LPT rule (fargo3d_b200/shard.py):
about 64 disks per GPU (weak scaling), no collective in the data path; the
single-disk workloads run one replica per rank.  `--impl reference` times the
reference's CPU implementation (its own C sources with its stock -O3) of the
same workload on rank 0 only, every host core running independent disks, for
the same step count as the GPU arm.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
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
           "sweep_cols": 8, "sweep_x": 11, "newvel": 8, "bnd": 0, "scalars": 0},
    "3d": {"rowsum": 1, "cfl": 5, "sources": 8, "bnd_vtemp": 0, "rowsum_vtemp": 1,
           "sweep_cols": 26, "sweep_x": 15, "newvel": 11, "bnd": 0, "scalars": 0},
}
KERNELS_PER_GROUP = {"2d": {"sweep_cols": 1, "bnd": 1, "bnd_vtemp": 1},
                     "3d": {"sweep_cols": 2, "bnd": 2, "bnd_vtemp": 2}}


def build_hash() -> str:
    """Digest of the library's sources: a DRAM-traffic figure applies to the
    build it was captured on only."""
    import hashlib
    h = hashlib.sha256()
    for d in (os.path.join(ROOT, "fargo3d_b200", "csrc"), os.path.join(ROOT, "include")):
        for f in sorted(os.listdir(d)):
            with open(os.path.join(d, f), "rb") as fh:
                h.update(f.encode() + b"\0" + fh.read())
    return h.hexdigest()[:16]


def traffic_bytes(workload: str, precision: str, group: str):
    """DRAM bytes (read + write) per launch of a launch group from the last
    ncu capture (profiles/traffic.json), or None unless that capture was
    taken on this very build and workload."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as fh:
            t = json.load(fh)
    except (OSError, ValueError):
        return None
    if t.get("build") != build_hash() or t.get("workload") != "%s:%s" % (workload, precision):
        return None
    return t.get("bytes_per_launch", {}).get(group)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(name: str, rank: int = 0, world: int = 1):
    """This rank's disks and the workload's description.  Batched: rank's LPT
    share of one global list of 64 x world disks (seeded once, seed 0)."""
    from fargo3d_b200 import config_batched, config_fargo2d, config_p3disof
    from fargo3d_b200.shard import shard_disks
    if name == "fargo2d":
        return [config_fargo2d(384, 128, seed=rank)], "fargo2d 384x128 (2D cylindrical, 1 planet, nu=1e-5)"
    if name == "p3disof":
        return [config_p3disof(512, 256, 48, seed=rank)], "p3disof 512x256x48 (3D spherical, 1 planet, nu=1e-5)"
    if name == "multifluid":
        from fargo3d_b200 import config_multifluid
        return [config_multifluid(768, 256, seed=rank)], ("multifluid 768x256, gas + 4 dust species (1/St = 1000, "
                                                          "100, 10, 1), implicit drag, 1 planet")
    if name == "serving":
        from fargo3d_b200 import serving_requests
        return [r.cfg for r in serving_requests(64, seed=rank)], ("serving requests, sizes {256x64, 512x128, "
                                                                  "1024x256, 2048x512} weighted {.4,.3,.2,.1}")
    return shard_disks(config_batched(64 * world, seed=0), rank, world), (
        "%d independent 2D disks (%d per GPU), N_phi x N_r in {128..1024} x {64..512}, alpha viscosity, "
        "1 planet each" % (64 * world, 64))


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
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
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


E2E_REPS = 5   # end-to-end runs per bench line (the median is reported)


def read_profile(L, fn, h, *extra):
    """{launch group: ms summed over its occurrences (one per fluid)}, and the
    number of occurrences of each group."""
    import ctypes as C
    ms = (C.c_float * 40)()
    names = (C.c_char_p * 40)()
    n = fn(h, *extra, ms, names, 40)
    out, count = {}, {}
    for i in range(max(n, 0)):
        k = names[i].decode()
        out[k] = out.get(k, 0.0) + float(ms[i])
        count[k] = count.get(k, 0) + 1
    return out, count


# --------------------------------------------------------------------------
def time_plain_fp64(cfgs, steps, device):
    """The plain FP64 path, one disk at a time (host-synchronised steps)."""
    import torch
    from fargo3d_b200 import Disk, initial_state
    cells, t = 0, 0.0
    for c in cfgs:
        d = Disk(c, "fp64", device=device)
        d.set_state(*initial_state(c))
        d.initialize()
        d.run(2)
        stream = torch.cuda.ExternalStream(d.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        d.run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1e3
        cells += c.active_cells * steps
        d.close()
    return cells / t


def run_serving(n_requests: int, rate: float, orbits: float, device: int, seed: int = 0):
    """The serving workload through the continuous-batching server: Poisson
    arrivals submitted in real time by a thread, every request run to its end
    time; latency = finished - submitted on the server's clock.  The initial
    states are built before the clock starts."""
    from fargo3d_b200 import Server, initial_state, serving_requests
    reqs = serving_requests(n_requests, rate=rate, orbits=orbits, seed=seed)
    states = [initial_state(r.cfg) for r in reqs]
    srv = Server("fp32", device=device, max_disks=256, chunk_steps=10)
    # warm-up: one small request of each size class (kernel loading, graphs)
    warm = [srv.submit(r.cfg, 0.05, st) for r, st in zip(reqs[:4], states[:4])]
    for w in warm:
        srv.wait(w)
        srv.fetch(w)
    ids = [None] * len(reqs)

    def submitter():
        t0 = time.perf_counter()
        for k, (r, st) in enumerate(zip(reqs, states)):
            dt = r.arrival - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids[k] = srv.submit(r.cfg, r.t_end, st)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    infos = []
    for rid in ids:
        srv.wait(rid)
        infos.append(srv.fetch(rid)[1])
    srv.close()
    lat = np.array([i["finished"] - i["submitted"] for i in infos])
    work = sum(i["steps"] * i["cells"] for i in infos)
    span = max(i["finished"] for i in infos) - min(i["submitted"] for i in infos)
    return {"value": work / span, "unit": "cell-updates/s",
            "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3), "p99": float(np.percentile(lat, 99) * 1e3),
                           "max": float(lat.max() * 1e3)},
            "queue_wait_ms_p50": float(np.percentile([i["admitted"] - i["submitted"] for i in infos], 50) * 1e3),
            "requests": len(infos), "failed": int(sum(1 for i in infos if i["status"] != 1)),
            "workload": "%d requests, Poisson %.0f/s, sizes {256x64, 512x128, 1024x256, 2048x512} weighted "
                        "{.4,.3,.2,.1}, %.2g orbits each, FP32, continuous batching" % (len(infos), rate, orbits),
            "span_s": span}


def run_serving_fp64_sequential(n_requests: int, rate: float, orbits: float, device: int, seed: int = 0):
    """The same request stream served by the plain FP64 path one request at a
    time: each request runs alone (fb_disk_step, FP64) until its end time;
    requests queue in arrival order behind the one running.  Service times
    are measured (wall clock around each request's steps, state uploaded
    before), the queue is then replayed on the measured times:
    finish_k = max(arrival_k, finish_{k-1}) + service_k."""
    from fargo3d_b200 import Disk, initial_state, serving_requests
    reqs = serving_requests(n_requests, rate=rate, orbits=orbits, seed=seed)
    service, work = [], 0
    for r in reqs:
        d = Disk(r.cfg, "fp64", device=device)
        d.set_state(*initial_state(r.cfg))
        d.initialize()
        t0 = time.perf_counter()
        steps = 0
        while d.scalars()[0] < r.t_end * (1.0 - 1e-12):
            d.step(r.t_end)
            steps += 1
        service.append(time.perf_counter() - t0)
        work += steps * r.cfg.active_cells
        d.close()
    fin, lat = 0.0, []
    for r, sv in zip(reqs, service):
        fin = max(r.arrival, fin) + sv
        lat.append(fin - r.arrival)
    lat = np.array(lat)
    return {"value": work / (fin - reqs[0].arrival), "unit": "cell-updates/s",
            "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3), "p99": float(np.percentile(lat, 99) * 1e3),
                           "max": float(lat.max() * 1e3)},
            "orbits_per_request": orbits, "requests": len(reqs),
            "how": "plain FP64 path (fb_disk_step), one request at a time in arrival order, measured service "
                   "times replayed through the FIFO queue"}


def fp32_errors(device: int):
    """Per-field error of the FP32 path against the FP64 path after each
    configuration's own step count, native CFL steps: the 64 batched disks
    (1000 steps; FP64 batched path as the reference, it follows the CPU oracle
    to round-off), the 3D spherical disk 512x256x48 (500 steps) and the
    multifluid disk 768x256 x 5 fluids (1000 steps; plain paths).  Relative
    L1 and L-infinity over the active cells."""
    from fargo3d_b200 import Batch, Disk, config_batched, config_multifluid, config_p3disof

    def err(a, b, k, is3d):
        sl = (slice(3, -3) if is3d else slice(None), slice(3, -3), slice(None))
        x, y = a[k][sl], b[k][sl]
        den = np.sum(np.abs(y))
        return {"l1": float(np.sum(np.abs(x - y)) / den) if den > 0 else 0.0,
                "linf": float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))}

    out = {}
    cfgs = config_batched(64)
    st = {}
    for prec in ("fp64", "fp32"):
        b = Batch(cfgs, prec, device=device)
        b.load_initial_states()
        b.run(1000)
        st[prec] = [b.state(i) for i in range(len(cfgs))]
        b.close()
    per = {k: [err(st["fp32"][i], st["fp64"][i], k, False) for i in range(len(cfgs))] for k in ("rho", "vx", "vy")}
    out["batched_64_disks_1000_steps"] = {
        k: {"l1_max": max(e["l1"] for e in v), "l1_median": float(np.median([e["l1"] for e in v])),
            "linf_max": max(e["linf"] for e in v)} for k, v in per.items()}
    out["batched_64_disks_1000_steps"]["disks_over_1e-5_l1_rho"] = sum(1 for e in per["rho"] if e["l1"] > 1e-5)
    for name, cfg, n in (("p3disof_512x256x48_500_steps", config_p3disof(512, 256, 48), 500),
                         ("multifluid_768x256x5_1000_steps", config_multifluid(768, 256), 1000)):
        res = {}
        for prec in ("fp64", "fp32"):
            d = Disk(cfg, prec, device=device)
            d.load_initial_state()
            d.run(n)
            res[prec] = [d.state(f) for f in range(cfg.nfluids)]
            d.close()
        keys = ("rho", "vx", "vy", "vz") if cfg.is3d else ("rho", "vx", "vy")
        out[name] = {("fluid%d_" % f if cfg.nfluids > 1 else "") + k: err(res["fp32"][f], res["fp64"][f], k, cfg.is3d)
                     for f in range(cfg.nfluids) for k in keys}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from fargo3d_b200 import Batch, Disk, initial_state
    from fargo3d_b200 import _abi
    torch.cuda.set_device(local_rank)
    cfgs, wname = workload(args.workload, rank, world)
    batched = args.workload == "batched"
    precision = "fp32" if batched and args.precision_default else args.precision
    dim = "3d" if cfgs[0].is3d else "2d"
    esz = 8 if precision == "fp64" else 4
    cells = sum(c.active_cells for c in cfgs)
    L = _abi.bind_batch(_abi.lib())
    nf = cfgs[0].nfluids
    inits = [[initial_state(c, f) for f in range(nf)] for c in cfgs]   # [disk][fluid]
    if batched:
        runner = Batch(cfgs, precision, device=local_rank)
        if args.chains:
            runner.set_chains(args.chains)
        for i, sts in enumerate(inits):
            for f, st in enumerate(sts):
                runner.set_state(i, *st, fluid=f)
        runner.initialize()
        stream = torch.cuda.ExternalStream(runner.stream)
        runner.run(max(args.warmup, 10))   # includes the graph capture
        runner.sync()
        step_fn = lambda n: runner.run(n)
    else:
        runner = Disk(cfgs[0], precision, device=local_rank)
        for f, st in enumerate(inits[0]):
            runner.set_state(*st, fluid=f)
        runner.initialize()
        stream = torch.cuda.ExternalStream(runner.stream)
        runner.run(args.warmup)
        step_fn = lambda n: runner.run(n)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        step_fn(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        from fargo3d_b200.shard import max_over_ranks
        ms = max_over_ranks(ms, device="cuda")   # the job's time is its slowest rank's
        tdist.barrier()
    # the whole job's cells: every rank's share of the global list (batched)
    # or one replica per rank
    if batched:
        from fargo3d_b200 import config_batched
        total_cells = sum(c.active_cells for c in config_batched(64 * world, seed=0))
    else:
        total_cells = cells * world
    value = total_cells * args.steps / (ms / 1e3)
    # per-launch-group timing of one extra step (dominant kernel, roofline)
    if batched:
        prof, count = read_profile(L, L.fb_batch_profile_step, runner._h, 1e30)
    else:
        L.fb_disk_profile(runner._h, 1)
        runner.step()
        prof, count = read_profile(L, L.fb_disk_profile_read, runner._h)
        L.fb_disk_profile(runner._h, 0)
    prof.pop("host_scalars", None)
    count.pop("host_scalars", None)
    launches_per_step = sum(KERNELS_PER_GROUP[dim].get(k, 1) * count[k] for k in prof)
    if batched:   # every chain that holds disks launches its own groups
        launches_per_step *= min(runner.chains(), len(cfgs))
    dom = max((k for k in prof if LAUNCH_WORDS[dim].get(k, 0) > 0), key=lambda k: prof[k])
    hbm, peak_kind = peaks()
    # a group's time covers all its fluids: its words per cell, once per fluid
    dom_bytes = LAUNCH_WORDS[dim][dom] * esz * cells * (count[dom] if dom not in ("cfl", "rowsum") else nf)
    achieved = dom_bytes / (prof[dom] / 1e3) / 1e9
    runner.close()
    # end-to-end through the public API from page-locked host buffers: per
    # fluid, one page-locked block holds every member's input fields and one
    # its result fields, disk after disk in the order of the call (rho, vx,
    # vy, [vz,] cs in; rho, vx, vy, [vz] out), as an application keeping a
    # batch's state in one host buffer does
    in_q = (0, 1, 2, 3, 4) if dim == "3d" else (0, 1, 2, 4)
    keys = ("rho", "vx", "vy", "vz") if dim == "3d" else ("rho", "vx", "vy")

    def carve(block, shapes):
        out, o = [], 0
        for shp in shapes:
            n = int(np.prod(shp))
            out.append(block[o:o + n].view(*shp))
            o += n
        return out

    pinned, results = [], [[None] * nf for _ in cfgs]
    for f in range(nf):
        shapes = [c.shape for c in cfgs for _ in in_q]
        blk = torch.empty(sum(int(np.prod(s)) for s in shapes), dtype=torch.float64).pin_memory()
        views = iter(carve(blk, shapes))
        per = []
        for i in range(len(cfgs)):
            st = [None] * 5
            for q in in_q:
                v = next(views)
                v.copy_(torch.from_numpy(np.ascontiguousarray(inits[i][f][q]).reshape(cfgs[i].shape)))
                st[q] = v
            per.append(st)
        pinned.append(per)
        shapes = [c.shape for c in cfgs for _ in keys]
        rblk = torch.empty(sum(int(np.prod(s)) for s in shapes), dtype=torch.float64).pin_memory()
        rviews = iter(carve(rblk, shapes))
        for i in range(len(cfgs)):
            results[i][f] = {k: next(rviews).numpy() for k in keys}
    torch.cuda.synchronize()
    np_ = lambda st: [None if p is None else p.numpy() for p in st]

    def e2e_once():
        t0 = time.perf_counter()
        if batched:
            r2 = Batch(cfgs, precision, device=local_rank)
            for f in range(nf):
                r2.set_states([np_(st) for st in pinned[f]], fluid=f)
            r2.initialize()
            r2.run(args.steps)
            for f in range(nf):
                r2.states(f, out=[results[i][f] for i in range(len(cfgs))])
        else:
            r2 = Disk(cfgs[0], precision, device=local_rank)
            for f in range(nf):
                r2.set_state(*np_(pinned[f][0]), fluid=f)
            r2.initialize()
            r2.run(args.steps)
            for f in range(nf):
                r2.state(f, out=results[0][f])
        t = time.perf_counter() - t0
        r2.close()
        if dist:
            from fargo3d_b200.shard import max_over_ranks
            t = max_over_ranks(t, device="cuda")
        return t

    # the whole job (create, upload, K steps, read-back) E2E_REPS times; the
    # median (a run's host-side set-up and PCIe timing vary with the load
    # other jobs put on the shared host)
    e2e_samples = [e2e_once() for _ in range(E2E_REPS)]
    t_e2e = float(np.median(e2e_samples))
    nstored = sum(int(np.prod(c.shape)) for c in cfgs) * nf
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if precision == "fp64" else "f32", "data": "synthetic",
        "config": {"workload": wname, "precision": precision, "disks_per_gpu": len(cfgs),
                   "active_cells_per_gpu": cells,
                   "disk_seeds": [c.seed for c in cfgs] if batched else [cfgs[0].seed],
                   "parallelism": "independent disks per GPU (no collective)" if world > 1 else "one GPU",
                   "mode": ("batched launches + CUDA graph, %s concurrent chains" % (args.chains or "default")
                            if batched else "plain, one disk"),
                   "l2": "state (%d MB) larger than L2 (126 MB); no flush needed" % (nstored * esz * 5 // 2 ** 20)},
        "e2e": {"value": total_cells * args.steps / t_e2e, "unit": "cell-updates/s",
                "how": "median of %d runs of the whole job through the public API" % E2E_REPS,
                "samples_ms": [round(t * 1e3, 3) for t in e2e_samples],
                "h2d_bytes_per_step": (5 if dim == "3d" else 4) * nstored * 8 / args.steps,
                "d2h_bytes_per_step": len(keys) * nstored * 8 / args.steps + (0 if batched else 16)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": traffic_bytes(args.workload, precision, dom),
                     "build": build_hash(),
                     "alg_bytes_per_launch": dom_bytes, "launch_ms": prof[dom],
                     "step_alg_frac": (ALG_WORDS[dim] + (ALG_WORDS[dim] - 1) * (nf - 1)) * esz * cells
                                      * args.steps / (ms / 1e3) / 1e9 / hbm},
        "launch_ms": prof,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
        "rho_checksum": float(sum(np.sum(results[i][f]["rho"]) for i in range(len(cfgs)) for f in range(nf))),
    }
    if batched and rank == 0:
        v64 = time_plain_fp64(cfgs, 5, local_rank)
        line["fp64_plain"] = {"value": v64, "unit": "cell-updates/s",
                              "how": "same disks, plain FP64 path one disk at a time, 5 steps each"}
        line["speedup_vs_fp64_plain"] = value / world / v64
    return line


# --------------------------------------------------------------------------
def _ref_disk_worker(job):
    """One disk advanced by the reference's own sources (oracle/_ref, built
    with the reference's stock -O3; the parity build if that is missing):
    `warmup` untimed steps, then `steps` timed ones."""
    cfg, steps, warmup = job
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fargo3d_b200 import initial_state
    d, kind = None, "port"
    for k in ("ref_o3", "ref"):
        try:
            d = pyoracle.Disk(cfg, k)
            kind = "reference" if k == "ref_o3" else "reference (-O2 parity build)"
            break
        except FileNotFoundError:
            continue
    if d is None:
        d = pyoracle.Disk(cfg, "oracle")
    for f in range(cfg.nfluids):
        d.set_state(*initial_state(cfg, f), fluid=f)
    d.initialize()
    for _ in range(warmup):
        d.step()
    t0 = time.time()
    for _ in range(steps):
        d.step()
    t1 = time.time()
    d.close()
    return cfg.active_cells * steps, t0, t1, kind


def cpu_reference(cfgs, steps, warmup=0):
    """Throughput of the reference's CPU implementation: independent disks as
    independent single-threaded processes over the host's cores (the
    reference has no threading; MPI is absent on this image).  Returns
    (cell-updates/s, kind, cores, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libfargo_ref_cyl2d.so")):
        pyoracle.build()
    cores = max(1, min(len(cfgs), os.cpu_count() or 1))
    # largest disks first so the makespan is not set by a late big disk
    jobs = sorted([(c, steps, warmup) for c in cfgs], key=lambda j: -j[0].active_cells)
    if cores == 1:
        res = [_ref_disk_worker(j) for j in jobs]
        wall = sum(r[2] - r[1] for r in res)
    else:
        with mp.get_context("spawn").Pool(cores) as pool:
            res = pool.map(_ref_disk_worker, jobs, chunksize=1)
        # makespan of the stepping itself (process start-up excluded)
        wall = max(r[2] for r in res) - min(r[1] for r in res)
    work = sum(r[0] for r in res)
    kinds = sorted(set(r[3] for r in res))
    kind = kinds[0] if len(kinds) == 1 else "mixed: " + ", ".join(kinds)
    return work / wall, kind, cores, wall


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_steps_for(cfgs, steps, cores):
    """Steps of the CPU sample: the GPU arm's count, capped so the sample is
    about 30 s of host work (at ~3 M cell-updates/s per core)."""
    work = sum(c.active_cells * c.nfluids for c in cfgs)
    cap = max(1, int(30.0 * 3.0e6 * max(1, min(cores, len(cfgs))) / max(work, 1)))
    return max(1, min(steps, cap))


def print_plan(args, rank: int, world: int):
    """Each rank's share of the workload, gathered on rank 0 over the same
    rank set-up as a run (gloo: it needs no GPU)."""
    cfgs, wname = workload(args.workload, rank, world)
    mine = {"rank": rank, "disks": len(cfgs), "cells": sum(c.active_cells for c in cfgs),
            "seeds": [c.seed for c in cfgs]}
    allp = [mine]
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        tdist.init_process_group("gloo", timeout=timedelta(seconds=60))
        allp = [None] * world
        tdist.all_gather_object(allp, mine)
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"plan": True, "n_gpus": world, "workload": wname, "ranks": allp}), flush=True)


def relaunch_with_ranks(n: int) -> int:
    """`--gpus N` outside torchrun: start N ranks of this same command."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "p3disof", "fargo2d", "multifluid", "serving"])
    ap.add_argument("--requests", type=int, default=100, help="serving: number of requests")
    ap.add_argument("--orbits", type=float, default=0.25, help="serving: orbits per request")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: arrivals per second")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg of the default run")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP32-vs-FP64 error leg of the default run")
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg (profiling runs)")
    ap.add_argument("--chains", type=int, default=0,
                    help="batched: concurrent step chains (0 = the library's default; 1 for per-launch profiles)")
    ap.add_argument("--plan", action="store_true",
                    help="print every rank's share of the workload and exit (no GPU work; gloo when N > 1)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_with_ranks(args.gpus))
    args.precision_default = args.precision is None
    if args.precision is None:
        args.precision = "fp32" if args.workload == "batched" else "fp64"
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.plan:
        print_plan(args, rank, world)
        return
    if args.impl == "reference":
        if rank != 0:
            return
        # the GPU arm's workload (for N > 1 its first 64 disks: a bounded
        # sample of the same distribution), the GPU arm's step count
        gcfgs, wname = workload(args.workload, 0, 1)
        cores = max(1, min(len(gcfgs), os.cpu_count() or 1))
        steps = cpu_steps_for(gcfgs, args.steps, cores)
        warm = min(args.warmup, steps)
        v, kind, cores, wall = cpu_reference(gcfgs, steps, warm)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": world,
                "steps": steps, "warmup": warm, "ms_per_step": wall / steps * 1e3, "higher_is_better": True,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": wname, "precision": "fp64 (the reference CPU build, stock -O3)"},
                "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                                 "sample": "%d hydro steps of each of %d disks, %d single-threaded processes, "
                                           "%.1f s (%s)" % (steps, len(gcfgs), cores, wall, cpu_model())},
                "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if args.workload == "serving":
        if rank != 0:
            return
        sv = run_serving(args.requests, args.rate, args.orbits, local_rank)
        sv["fp64_one_at_a_time"] = run_serving_fp64_sequential(args.requests, args.rate, args.orbits, local_rank)
        line = {"metric": METRIC, "value": sv["value"], "unit": "cell-updates/s", "n_gpus": 1,
                "steps": sv["requests"], "warmup": 4, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": sv["workload"], "parallelism": "one GPU"},
                "latency_ms": sv["latency_ms"], "serving": sv}
        print(json.dumps(line), flush=True)
        return
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
    line = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and args.workload == "batched" and not args.no_serving:
        line["serving"] = run_serving(args.requests, args.rate, args.orbits, local_rank)
        line["serving"]["fp64_one_at_a_time"] = run_serving_fp64_sequential(args.requests, args.rate, args.orbits,
                                                                            local_rank)
    if rank == 0 and world == 1 and args.workload == "batched" and not args.no_accuracy:
        line["fp32_error"] = fp32_errors(local_rank)
    if rank == 0 and world == 1 and not args.no_cpu:
        cfgs, _ = workload(args.workload, 0, 1)
        cores = max(1, min(len(cfgs), os.cpu_count() or 1))
        steps = cpu_steps_for(cfgs, args.steps, cores)
        v, kind, cores, wall = cpu_reference(cfgs, steps)
        line["cpu_baseline"] = {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                                "sample": "%d hydro steps of each of %d disks, %d single-threaded processes, "
                                          "%.1f s (%s)" % (steps, len(cfgs), cores, wall, cpu_model())}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
