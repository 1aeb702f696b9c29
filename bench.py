"""Benchmark of the CGFDM hot path on B200 (one JSON line on stdout).

A step is one full RK4 time step (sources, four fused stages, stations, PGV)
over the whole grid of the workload.  Metric: grid-point updates per second
per RK4 step (Gpt-updates/s).  Multi-GPU: independent replicas (the path is
not sharded), weak scaling, max time over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3-1201]
                  [--precision fp32] [--impl ours|reference]

The default workload is the 1201 x 1201 x 401 PerformanceTest shape in FP32
with the scaled-FP16 form timed beside it; an accuracy block runs the
Gaussian-hill configuration (401 x 401 x 201, 2000 steps) in FP64, FP32 and
scaled FP16 and reports each one's relative L2 error against FP64.

--impl reference times the reference's own scalar CPU build (oracle/_ref,
compiled in place from the reference sources, run on all host cores as MPI
ranks through the shared-memory MPI shim) on the same workload.
"""
import argparse
import contextlib
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cgfdm-fp16_sve_sme_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from cgfdm import scenarios as S  # noqa: E402

REF_EXE = os.path.join(ROOT, "oracle", "_ref", "cgfdm_ref_fp32")
METRIC = "Gpt-updates/s per RK4 step"
UNIT = "Gpt-updates/s"
# Algorithmic HBM bytes per grid point per RK4 step of the fused stage kernels
# in FP32: per stage 9 stage-input + 12 coefficient reads and 9 output
# writes; W_n reads in stages 1-2; the RK accumulator written in stage 0,
# read+written in stages 1-2, read in stage 3 (4 bytes each).
BYTES_PER_POINT_STEP = {"fp32": 768, "fp64": 1536, "fp16": 384, "bf16": 384}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------
# workloads (synthetic inputs with the shapes of the benchmark configurations)
# --------------------------------------------------------------------------
def make_workload(name, nsteps_total):
    if name == "c2":
        return S.c2_workload(nsteps_total)
    m = re.fullmatch(r"c3-(\d+)", name)
    if m:
        return S.c3_workload(int(m.group(1)), nsteps_total)
    raise SystemExit("unknown workload " + name)


def write_workload(w, d):
    S.write_run_dir(d, w["params"], stations=w["stations"], terrain=w.get("terrain"),
                    layers=w.get("layers"), source=w.get("source"))


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


# --------------------------------------------------------------------------
# reference arm / CPU baseline: the reference's own CPU build, all host cores
# --------------------------------------------------------------------------
def pick_decomposition(p, cores):
    """PX*PY*PZ <= cores with every rank at least max(nPML, 8) cells per axis
    (init_grid.cpp:109-117): the largest rank count, and among those the
    split with the fewest padded points (the least halo)."""
    lim = max(p["nPML"], 8)
    best, best_key = (1, 1, 1), None
    for px in range(1, cores + 1):
        if p["NX"] // px < lim:
            break
        for py in range(1, cores // px + 1):
            if p["NY"] // py < lim:
                break
            for pz in range(1, cores // (px * py) + 1):
                if p["NZ"] // pz < lim:
                    break
                pad = (p["NX"] + 6 * px) * (p["NY"] + 6 * py) * (p["NZ"] + 6 * pz)
                key = (px * py * pz, -pad)
                if best_key is None or key > best_key:
                    best, best_key = (px, py, pz), key
    return best


def reference_bytes(p, ranks):
    """Host memory the reference holds during its time loop: 49 FLOAT fields
    per padded point of every rank (13 CJM + 4 x 9 wavefield, run.cpp:63-96,
    propagate.cpp:65-92) plus the PML auxiliaries (4 x 9 floats per slab
    point), with each rank's halo counted."""
    px, py, pz = ranks
    padded = 0
    for X in range(px):
        nx = p["NX"] // px + (1 if X < p["NX"] % px else 0)
        for Y in range(py):
            ny = p["NY"] // py + (1 if Y < p["NY"] % py else 0)
            for Z in range(pz):
                nz = p["NZ"] // pz + (1 if Z < p["NZ"] % pz else 0)
                padded += (nx + 6) * (ny + 6) * (nz + 6)
    n = p["nPML"]
    slab = 2 * n * p["NY"] * p["NZ"] + 2 * p["NX"] * n * p["NZ"] + p["NX"] * p["NY"] * n
    return 4 * 49 * padded + 4 * 36 * slab


def mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def run_reference(w, nsteps, cores, timeout_s=1500):
    """Runs the reference on a copy of the workload with MPI ranks = cores
    and returns (seconds per step, ranks used, steps timed).  The reference
    prints a `Step time loss` line for step 0 and then one per 10 steps
    (propagate.cpp:183-195); the per-step time is the mean of the 10-step
    blocks after the first (nsteps >= 20), or of the one 10-step block after
    step 0 (nsteps < 20, for grids whose steps take tens of seconds)."""
    if not os.path.exists(REF_EXE):
        raise RuntimeError("reference build missing at %s (make -C oracle ref)" % REF_EXE)
    p = dict(w["params"])
    dt = np.float32(p["DT"])
    nblocks = 1 if nsteps < 20 else max(2, math.ceil(nsteps / 10))
    total = 10 * nblocks + 1
    p["TMAX"] = float((total + 0.5) * dt)
    px, py, pz = pick_decomposition(p, cores)
    p.update(PX=px, PY=py, PZ=pz)
    need, avail = reference_bytes(p, (px, py, pz)), mem_available()
    if avail is not None and need * 1.2 > avail:
        raise RuntimeError("the reference needs about %.0f GB of host memory for %s on %d ranks, "
                           "%.0f GB available" % (need / 1e9, w["name"], px * py * pz, avail / 1e9))
    d = tempfile.mkdtemp(prefix="cgfdm_ref_")
    try:
        ww = dict(w)
        ww["params"] = p
        write_workload(ww, d)
        env = dict(os.environ, CGFDM_SHIM_NPROC=str(px * py * pz),
                   CGFDM_SHIM_TIMEOUT=str(timeout_s))
        r = subprocess.run([REF_EXE], cwd=d, env=env, capture_output=True, text=True,
                           timeout=timeout_s, start_new_session=True)
        if r.returncode != 0:
            raise RuntimeError("reference run failed (%d): %s" % (r.returncode, r.stdout[-400:] +
                                                                  r.stderr[-400:]))
        times = [float(m.group(1)) for m in
                 re.finditer(r"Step time loss:\s*([0-9.eE+-]+)s", r.stdout)]
        blocks = times[1:]  # it = 0 is the first step alone; later lines cover 10 steps
        if len(blocks) > 1:
            blocks = blocks[1:]  # first 10-step block is warm-up
        if not blocks:
            raise RuntimeError("no timing lines in the reference output")
        return sum(blocks) / (10.0 * len(blocks)), px * py * pz, 10 * len(blocks)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def cpu_sample_workload(name):
    """The bounded CPU-baseline sample of a workload: the grid itself up to
    401 x 401 x 401 points of columns, else the same generator at 401 x 401
    columns (the reference's per-point cost does not depend on the grid
    size; a 1201^2 step takes about half a minute on 16 cores)."""
    m = re.fullmatch(r"c3-(\d+)", name)
    if m and int(m.group(1)) > 401:
        return "c3-401"
    return name


# --------------------------------------------------------------------------
def _propagate(cgfdm, setup, prec, kern, device, nsteps):
    d0 = setup["desc"]
    desc = cgfdm.make_desc(d0.nx, d0.ny, d0.nz, d0.npml, d0.dh, d0.dt, nsteps, prec, kern,
                           device)
    has_fault = setup["src_index"].size > 0
    return cgfdm.propagate(
        desc, setup["cjm"], setup["rdz"], point=setup["point"], rickerfc=setup["rickerfc"],
        src_index=setup["src_index"] if has_fault else None,
        moment_rate=setup["moment_rate"] if has_fault else None,
        src_nt=setup["src_nt"], src_dt=setup["src_dt"], stations=setup["stations"])


def measure_accuracy(cgfdm, wname, nsteps, precisions, device):
    """Relative L2 error of the seismograms (Vx, Vy, Vz of every station over
    all steps) and of the final free-surface velocity snapshot of each
    precision (the streaming kernels, KERNEL_AUTO) against an FP64 run of the
    same workload on the GPU (the exact-order kernel templated on double),
    all through propagate().  Returns {precision: {...}}."""
    w = make_workload(wname, nsteps + 2)
    rel = lambda a, b: float(np.linalg.norm((a - b).ravel().astype(np.float64)) /
                             max(np.linalg.norm(b.ravel().astype(np.float64)), 1e-300))

    def run(prec):
        d = tempfile.mkdtemp(prefix="cgfdm_acc_")
        try:
            write_workload(w, d)
            st = cgfdm.setup_from_directory(d, prec)
        finally:
            shutil.rmtree(d, ignore_errors=True)
        t0 = time.perf_counter()
        sta, _, fs = _propagate(cgfdm, st, prec, cgfdm.KERNEL_AUTO, device, nsteps)
        nsta = len(st["stations"])
        return sta.reshape(nsta, -1, 9)[:, :nsteps, :3], fs, time.perf_counter() - t0

    ref_sta, ref_fs, t64 = run(cgfdm.FP64)
    out = {"workload": w["name"], "steps": nsteps,
           "reference": "fp64 GPU run of the same workload (exact-order kernel on double)",
           "fp64_seconds": t64, "max_abs_ref_v": float(np.abs(ref_sta).max())}
    names = {cgfdm.FP32: "fp32", cgfdm.FP16: "fp16", cgfdm.BF16: "bf16"}
    for prec in precisions:
        sta, fs, _ = run(prec)
        out[names[prec]] = {"rel_l2_stations_v": rel(sta, ref_sta),
                            "rel_l2_free_surface_v": rel(fs, ref_fs)}
    return out


# --------------------------------------------------------------------------
# batched scenarios (c4) and serving (c5)
# --------------------------------------------------------------------------
def _setup_scenario(cgfdm, w, prec):
    d = tempfile.mkdtemp(prefix="cgfdm_bench_")
    try:
        write_workload(dict(w, name="s"), d)
        return cgfdm.setup_from_directory(d, prec)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def _sim_of(cgfdm, setup, prec, nt, device):
    """A handle of one scenario; its tile form and work-item depth are the
    autotuner's (alone), or its depth for the 32 x 16 form (in a batch)."""
    d0 = setup["desc"]
    sim = cgfdm.Simulation(cgfdm.make_desc(d0.nx, d0.ny, d0.nz, d0.npml, d0.dh, d0.dt, nt, prec,
                                           cgfdm.KERNEL_AUTO, device))
    sim.set_model(setup["cjm"], setup["rdz"])
    if setup["point"] is not None:
        sim.set_point_source(*setup["point"], setup["rickerfc"])
    if setup["src_index"].size:
        sim.set_fault_source(setup["src_index"], setup["moment_rate"], setup["src_nt"],
                             setup["src_dt"], scaled=True)
    sim.set_stations(setup["stations"])
    return sim


def bench_batch(args, cgfdm, torch, local, prec):
    """48 seeded scenarios (NX, NY in [121, 401], NZ in [101, 201], own
    medium, hill and double-couple source) advanced together as one batch
    (persistent streaming launches spanning all of them, one CUDA graph per
    step) against the same scenarios run back to back alone."""
    n = args.batch_n
    total = args.warmup + args.steps + 2
    setups = [_setup_scenario(cgfdm, S.sample_scenario(1000 + q, nsteps=total), prec)
              for q in range(n)]
    pts = [s["desc"].nx * s["desc"].ny * s["desc"].nz for s in setups]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    alone_ms = 0.0
    for st in setups:  # back to back
        sim = _sim_of(cgfdm, st, prec, total, local)
        sim.run(args.warmup, stream.cuda_stream)
        torch.cuda.synchronize()
        ev0.record(stream)
        sim.run(args.steps, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        alone_ms += ev0.elapsed_time(ev1)
        sim.close()
    sims = [_sim_of(cgfdm, st, prec, total, local) for st in setups]
    batch = cgfdm.Batch(sims, graph=True)
    batch.run(args.warmup, stream.cuda_stream)
    torch.cuda.synchronize()
    depths = {}
    for sim in sims:
        ch = sim.tuning()[1]
        depths[str(ch)] = depths.get(str(ch), 0) + 1
    with ClockSampler(local) as clk:
        ev0.record(stream)
        batch.run(args.steps, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    batch.synchronize()
    ms = ev0.elapsed_time(ev1)
    batch.close()
    for sim in sims:
        sim.close()
    upd = float(sum(pts)) * args.steps
    return {
        "metric": "aggregate Gpt-updates/s, batched scenarios", "value": upd / (ms / 1e3) / 1e9,
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": _dtype(args.precision), "data": "synthetic",
        "config": {"workload": "c4-batched-%d-scenarios" % n, "precision": args.precision,
                   "points_total": int(sum(pts)), "points_min": int(min(pts)),
                   "points_max": int(max(pts)), "graph": True, "tile_form": 16,
                   "chunk_planes_histogram": depths,
                   "steps_note": "bounded sample of the 1500-step runs"},
        "serial": {"value": upd / (alone_ms / 1e3) / 1e9, "unit": UNIT,
                   "note": "the same scenarios run alone back to back (no batch, no graph; "
                           "each with its own autotuned tile form and depth)"},
        "speedup_vs_serial": alone_ms / ms,
        "clocks": clk.summary(),
    }


def bench_serving(args, cgfdm, torch, local):
    """A seeded Poisson stream of requests (grid points log-uniform in
    [1e6, 5e7], steps uniform in [500, 3000] times --step-scale, FP32 or
    FP16 each) through the library's server (continuous batching, graphs,
    budget 160 GB), against serial single-request FP32 on the same GPU."""
    rng = np.random.default_rng(7)
    nreq = args.requests
    rate = float(rng.uniform(2.0, 20.0))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    reqs = []
    for q in range(nreq):
        points = float(np.exp(rng.uniform(math.log(1e6), math.log(5e7))))
        steps = max(1, int(round(rng.integers(500, 3001) * args.step_scale)))
        prec = cgfdm.FP16 if rng.random() < 0.5 else cgfdm.FP32
        w = S.sample_scenario(2000 + q, points=points, nsteps=steps + 2)
        reqs.append((_setup_scenario(cgfdm, w, prec), prec, steps))
    log("serving: %d requests generated" % nreq)

    def submit_args(st, prec, steps):
        d0 = st["desc"]
        desc = cgfdm.make_desc(d0.nx, d0.ny, d0.nz, d0.npml, d0.dh, d0.dt, steps, prec,
                               cgfdm.KERNEL_AUTO, local)
        fault = st["src_index"].size > 0
        return desc, dict(point=st["point"], rickerfc=st["rickerfc"],
                          src_index=st["src_index"] if fault else None,
                          moment_rate=st["moment_rate"] if fault else None,
                          src_nt=st["src_nt"], src_dt=st["src_dt"], stations=st["stations"])

    chunk = max(1, int(round(100 * args.step_scale)))
    free = torch.cuda.mem_get_info(local)[0]
    budget = int(min(160e9, free - 8e9))
    with cgfdm.Server(hbm_budget_bytes=budget, chunk=chunk, device=local, graph=True) as srv:
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            ids = []
            for q, (st, prec, steps) in enumerate(reqs):
                delay = arrivals[q] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                desc, kw = submit_args(st, prec, steps)
                ids.append(srv.submit(desc, st["cjm"], st["rdz"], **kw))
            for rid in ids:
                srv.wait(rid)
            wall = time.perf_counter() - t0
        stats = srv.stats()
    upd = float(sum(st["desc"].nx * st["desc"].ny * st["desc"].nz * steps
                    for st, _, steps in reqs))
    # serial single-request FP32: each request alone, end to end (upload, run, results)
    t_serial = 0.0
    for st, _, steps in reqs:
        desc, kw = submit_args(st, cgfdm.FP32, steps)
        t1 = time.perf_counter()
        cgfdm.propagate(desc, st["cjm"], st["rdz"], **kw)
        t_serial += time.perf_counter() - t1
    return {
        "metric": "serving: aggregate Gpt-updates/s with p50/p99 latency", "value": stats["gpts"],
        "unit": UNIT, "n_gpus": 1, "steps": int(sum(s for _, _, s in reqs)), "warmup": 0,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 and f16-storage/f32 (per request)", "data": "synthetic",
        "config": {"workload": "c5-serving-%d-requests" % nreq, "arrival_rate_per_s": rate,
                   "step_scale": args.step_scale, "chunk_steps": chunk,
                   "hbm_budget_bytes": budget, "graph": True,
                   "fp16_requests": sum(1 for _, p, _ in reqs if p == cgfdm.FP16)},
        "latency_ms": {"first_seismogram_p50": stats["first_p50_ms"],
                       "first_seismogram_p99": stats["first_p99_ms"],
                       "completion_p50": stats["done_p50_ms"],
                       "completion_p99": stats["done_p99_ms"]},
        "wall_s": wall, "peak_admitted_bytes": stats["peak_bytes"],
        "serial_fp32": {"value": upd / t_serial / 1e9, "unit": UNIT, "seconds": t_serial,
                        "note": "each request alone through cgfdm_propagate, FP32, back to back"},
        "speedup_vs_serial": stats["gpts"] / (upd / t_serial / 1e9),
        "clocks": clk.summary(),
    }


def _dtype(p):
    return {"fp32": "f32", "fp64": "f64", "fp16": "f16-storage/f32", "bf16": "bf16-storage/f32"}[p]


def measured_traffic(workload, kernel, precision, alg_bytes, launches):
    """DRAM read + write bytes per launch (one stage's streaming launches) of
    the kernel, from the one-pass ncu launch list of this workload, kernel and
    precision (profiles/stage_traffic.json: DRAM bytes per algorithmic byte),
    scaled to the algorithmic bytes of this run; None without a capture of
    that exact combination."""
    prof = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if not os.path.exists(prof) or launches <= 0:
        return None
    try:
        for e in json.load(open(prof))["captures"]:
            if (e["workload"], e["kernel"], e["precision"]) == (workload, kernel, precision):
                return e["traffic_over_alg"] * alg_bytes / launches
    except (OSError, ValueError, KeyError, TypeError):
        return None
    return None


def replica_throughput(torch, dist, seconds, points, steps, world, device):
    """Whole-job throughput of N independent replicas (one per rank, the
    same work each): the slowest rank's time bounds the job, so the value is
    world * points * steps / max over ranks of the time.  Returns (Gpt/s,
    max seconds).  Every rank must call it (one all-reduce)."""
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    if dist is not None and world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tmax = float(t.item())
    return world * float(points) * steps / tmax / 1e9, tmax


def setup_slots(params, local_ranks, avail):
    """How many of a node's ranks may run the host setup at once: all of
    them when the node's available memory holds their peak host footprint
    (the 13 coefficient fields about 2.5 times over: the setup's own arrays,
    the returned fields and their pinned copy), else as many as it holds
    (at least one).  Ranks beyond that wait for a turn, so that N replicas
    of a large grid do not drive the host out of memory."""
    cjm_bytes = 13 * (params["NX"] + 6) * (params["NY"] + 6) * (params["NZ"] + 6) * 4
    if not avail:
        return local_ranks
    return max(1, min(local_ranks, int(avail // (2.5 * cjm_bytes))))


class SetupTurn:
    """Holds one of `slots` node-wide setup slots (a file lock per slot under
    the temporary directory; local rank r uses slot r mod slots) while a host
    setup runs."""

    def __init__(self, local, slots):
        self.path = os.path.join(tempfile.gettempdir(),
                                 "cgfdm_bench_setup.%s.%d.lock" % (
                                     os.environ.get("MASTER_PORT", "0"), local % slots))
        self.f = None

    def __enter__(self):
        import fcntl
        self.f = open(self.path, "a")
        fcntl.flock(self.f, fcntl.LOCK_EX)
        return self

    def __exit__(self, *a):
        import fcntl
        fcntl.flock(self.f, fcntl.LOCK_UN)
        self.f.close()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c3-1201",
                    help="c2, c3-N (N x N x 401), c4 (batched scenarios) or c5 (serving)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16", "bf16", "fp64"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "exact", "stream"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--tile-rows", type=int, default=0, choices=[0, 8, 16, 64],
                    help="streaming-kernel tile form: 16 or 8 (32-column tiles of that height), "
                         "64 (paired-point 64 x 8 tiles, FP16 / BF16), 0: the library's "
                         "autotuner")
    ap.add_argument("--chunk", type=int, default=0,
                    help="planes per streaming work item in z (0: the library's default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp16", action="store_true",
                    help="skip the scaled-FP16 companion measurement of an FP32 run")
    ap.add_argument("--cpu-baseline-steps", type=int, default=20)
    ap.add_argument("--batch-n", type=int, default=48, help="scenarios of --workload c4")
    ap.add_argument("--requests", type=int, default=32, help="requests of --workload c5")
    ap.add_argument("--step-scale", type=float, default=1.0,
                    help="--workload c5: request step counts are U[500, 3000] times this")
    ap.add_argument("--accuracy-workload", default="c2",
                    help="workload of the accuracy block (FP64 must fit one GPU)")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="steps of the accuracy block: FP64, FP32 and scaled FP16 (and "
                         "--precision) through propagate(), relative L2 of the station "
                         "seismograms and the free-surface snapshot against FP64 "
                         "(0: no accuracy block)"),
    args = ap.parse_args()
    if args.e2e_steps < 1:
        ap.error("--e2e-steps must be at least 1 (the line always carries an end-to-end figure)")
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return 0
        if args.workload in ("c4", "c5"):
            print(json.dumps({"impl": "reference", "unavailable": "the reference runs one "
                              "scenario per process: no batched or serving mode"}))
            return 0
        w = make_workload(args.workload, args.warmup + args.steps + 2)
        cores = os.cpu_count() or 1
        npts_w = w["params"]["NX"] * w["params"]["NY"] * w["params"]["NZ"]
        # grids whose reference steps take tens of seconds: step 0 and one
        # timed 10-step block (a bounded sample of the run's steps)
        ref_steps = args.warmup + args.steps if npts_w <= 1e8 else 10
        try:
            sps, ranks, timed = run_reference(w, ref_steps, cores)
        except Exception as e:  # noqa: BLE001
            print(json.dumps({"impl": "reference", "unavailable": str(e)[:300]}))
            return 0
        npts = w["params"]["NX"] * w["params"]["NY"] * w["params"]["NZ"]
        v = npts / sps / 1e9
        sample = "%s (the whole grid), %d timed steps (%s), %d MPI ranks" % (
            w["name"], timed, "10-step blocks after a warm-up block" if timed > 10 else
            "one 10-step block after step 0", ranks)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
            "steps": timed, "warmup": args.warmup, "ms_per_step": sps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["name"], "precision": "fp32", "points": npts},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ranks, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return 0

    import torch
    import cgfdm

    torch.cuda.set_device(local)
    dist = None
    slots = 1
    if ws > 1:
        import datetime
        import torch.distributed as dist
        local_ranks = int(os.environ.get("LOCAL_WORLD_SIZE", str(ws)))
        if args.workload not in ("c4", "c5"):
            slots = setup_slots(make_workload(args.workload, 1)["params"], local_ranks,
                                mem_available())
        # ranks that wait for a setup turn reach the first barrier late: the
        # timeout covers the waits (about a minute of setup per turn)
        waits = (local_ranks + slots - 1) // slots - 1
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120 + 90 * waits),
                                device_id=torch.device("cuda", local))
    prec = {"fp32": cgfdm.FP32, "fp16": cgfdm.FP16, "bf16": cgfdm.BF16, "fp64": cgfdm.FP64}[
        args.precision]
    if args.workload in ("c4", "c5"):
        line = (bench_batch(args, cgfdm, torch, local, prec) if args.workload == "c4"
                else bench_serving(args, cgfdm, torch, local))
        if rank == 0:
            print(json.dumps(line))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    kern = {"auto": cgfdm.KERNEL_AUTO, "exact": cgfdm.KERNEL_EXACT,
            "stream": cgfdm.KERNEL_STREAM}[args.kernel]

    total_steps = args.warmup + args.steps
    w = make_workload(args.workload, max(total_steps, args.e2e_steps) + 2)
    d = tempfile.mkdtemp(prefix="cgfdm_bench_")
    write_workload(w, d)
    def pinned(a):
        t = torch.empty(a.shape, dtype={np.float32: torch.float32, np.int64: torch.int64}[
            a.dtype.type], pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    t0 = time.perf_counter()
    def setup_turn():
        # a slot of the node's setup lock when its memory cannot hold every
        # rank's setup at once (see setup_slots)
        if slots < int(os.environ.get("LOCAL_WORLD_SIZE", "1")):
            return SetupTurn(local, slots)
        return contextlib.nullcontext()

    with setup_turn():
        # FP16 / BF16 handles take the coefficients in the reference's scaled form
        setup = cgfdm.setup_from_directory(d, prec)
        # the model coefficients (13 fields, 31 GB at 1201 x 1201 x 401 in
        # FP32) are held once per rank, in pinned memory: the handles upload
        # them from there, and the end-to-end run below takes them as its
        # host input
        cjm = pinned(setup["cjm"])
        # the rest as copies of their own, so that the setup's buffers (the
        # library frees them with their last view: coefficients, coordinates
        # and medium, 45 GB at 1201 x 1201 x 401) go now
        setup = {k: (np.array(v) if isinstance(v, np.ndarray) else v)
                 for k, v in setup.items() if k not in ("cjm", "coord", "medium")}
    log("host setup %.1f s" % (time.perf_counter() - t0))
    shutil.rmtree(d, ignore_errors=True)
    desc0 = setup["desc"]
    npts = desc0.nx * desc0.ny * desc0.nz

    def new_sim(nt):
        desc = cgfdm.make_desc(desc0.nx, desc0.ny, desc0.nz, desc0.npml, desc0.dh, desc0.dt, nt,
                               prec, kern, local)
        sim = cgfdm.Simulation(desc)
        sim.set_tile_rows(args.tile_rows)
        sim.set_chunk(args.chunk)
        sim.set_model(cjm, setup["rdz"])
        if setup["point"] is not None:
            sim.set_point_source(*setup["point"], setup["rickerfc"])
        if setup["src_index"].size:
            sim.set_fault_source(setup["src_index"], setup["moment_rate"], setup["src_nt"],
                                 setup["src_dt"], scaled=True)
        sim.set_stations(setup["stations"])
        return sim

    sim = new_sim(total_steps)
    sim.set_timing(True)
    # a dedicated (non-null) stream: the work and the events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sim.run(args.warmup, stream.cuda_stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        sim.run(args.steps, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    tm = sim.timing_ms()
    ks = sim.kernel_stats()
    form, chunk, fast_top = sim.tuning3()
    stage_ms, stage_n = float(tm[1]), int(tm[2])
    sim.close()
    value, ms_max = replica_throughput(torch, dist, ms / 1e3, npts, args.steps, ws, "cuda")
    ms_max *= 1e3

    # end to end through the drop-in with host buffers (propagate()): the
    # model and source arrays sit in pinned host memory (staged before the
    # timed region), the run's outputs come back to host arrays
    e2e_steps = args.e2e_steps
    desc = cgfdm.make_desc(desc0.nx, desc0.ny, desc0.nz, desc0.npml, desc0.dh, desc0.dt,
                           e2e_steps, prec, kern, local)
    sta = setup["stations"]

    cjm_p, rdz_p = cjm, pinned(setup["rdz"])
    has_fault = setup["src_index"].size > 0
    idx_p = pinned(setup["src_index"]) if has_fault else None
    rate_p = pinned(setup["moment_rate"]) if has_fault else None
    t0 = time.perf_counter()
    out_sta, out_pgv, out_fs = cgfdm.propagate(
        desc, cjm_p, rdz_p, point=setup["point"], rickerfc=setup["rickerfc"],
        src_index=idx_p, moment_rate=rate_p,
        src_nt=setup["src_nt"], src_dt=setup["src_dt"], stations=sta)
    e2e_s = time.perf_counter() - t0
    del cjm_p, rdz_p, idx_p, rate_p
    e2e_value, e2e_max = replica_throughput(torch, dist, e2e_s, npts, e2e_steps, ws, "cuda")
    h2d = cjm.nbytes + setup["rdz"].nbytes + setup["moment_rate"].nbytes + \
        setup["src_index"].nbytes + sta.nbytes
    d2h = out_sta.nbytes + out_pgv.nbytes + out_fs.nbytes
    del cjm  # the FP32 model's host copy is not needed past this point

    # the scaled-FP16 form on the same workload, timed the same way (the
    # metric pairs it with FP32; its error against FP64 comes from the
    # accuracy block below)
    fp16 = None
    if args.precision == "fp32" and not args.no_fp16:
        d16 = tempfile.mkdtemp(prefix="cgfdm_bench_")
        try:
            write_workload(w, d16)
            with setup_turn():
                s16 = cgfdm.setup_from_directory(d16, cgfdm.FP16)
        finally:
            shutil.rmtree(d16, ignore_errors=True)
        e0 = s16["desc"]
        sim16 = cgfdm.Simulation(cgfdm.make_desc(e0.nx, e0.ny, e0.nz, e0.npml, e0.dh, e0.dt,
                                                 total_steps, cgfdm.FP16, kern, local))
        sim16.set_tile_rows(args.tile_rows)
        sim16.set_chunk(args.chunk)
        sim16.set_timing(True)  # as the FP32 run: per-stage events, no graphs
        sim16.set_model(s16["cjm"], s16["rdz"])
        if s16["point"] is not None:
            sim16.set_point_source(*s16["point"], s16["rickerfc"])
        if s16["src_index"].size:
            sim16.set_fault_source(s16["src_index"], s16["moment_rate"], s16["src_nt"],
                                   s16["src_dt"], scaled=True)
        sim16.set_stations(s16["stations"])
        del s16  # the setup's buffers go with their last view
        sim16.run(args.warmup, stream.cuda_stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        sim16.run(args.steps, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms16 = ev0.elapsed_time(ev1)
        ks16 = sim16.kernel_stats()
        form16, chunk16, top16 = sim16.tuning3()
        sim16.close()
        v16, ms16_max = replica_throughput(torch, dist, ms16 / 1e3, npts, args.steps, ws, "cuda")
        fp16 = {"value": v16, "unit": UNIT, "ms_per_step": ms16_max * 1e3 / args.steps,
                "speedup_vs_fp32": v16 / value, "tile_form": form16, "chunk_planes": chunk16,
                "surface_kernel": "tiled" if top16 else "exact-order",
                "bytes_per_point_step": BYTES_PER_POINT_STEP["fp16"]}
        if ks16["stream_ms"] > 0:
            a16 = ks16["stream_bytes"] / (ks16["stream_ms"] / 1e3) / 1e9
            pk16 = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs") \
                if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else None
            pk16 = pk16 or 6650.0
            kn16 = {64: "stage_pair_kernel", 16: "stage_stream_batch_kernel",
                    8: "stage_stream_kernel"}.get(form16, "stage_stream_kernel")
            fp16["roofline"] = {"bound": "hbm", "achieved": a16, "peak": pk16, "unit": "GB/s",
                                "frac": a16 / pk16,
                                "traffic": measured_traffic(w["name"], kn16, "fp16",
                                                            ks16["stream_bytes"],
                                                            ks16["stream_launches"]),
                                "kernel": kn16 + " (interior and PML launches)"}

    # error against FP64 of the precisions of this line, measured in this run
    # on a workload whose FP64 form fits one GPU
    accuracy = None
    if args.accuracy_steps > 0 and ws == 1:
        precs = [prec] + ([cgfdm.FP16] if fp16 and prec != cgfdm.FP16 else [])
        if prec == cgfdm.FP64:
            precs = []
        t0 = time.perf_counter()
        accuracy = measure_accuracy(cgfdm, args.accuracy_workload, args.accuracy_steps, precs,
                                    local)
        accuracy["seconds"] = time.perf_counter() - t0
        if fp16 and "fp16" in accuracy:
            fp16["accuracy"] = dict(accuracy["fp16"], workload=accuracy["workload"],
                                    steps=accuracy["steps"], against="fp64 GPU run")

    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    bpp = BYTES_PER_POINT_STEP[args.precision]
    # the dominant kernel: the streaming stage kernel (the exact-order kernel
    # when the precision has no streaming form)
    if ks["stream_launches"] > 0 and ks["stream_ms"] > 0:
        # tile height 16 runs the batched form of the kernel (a batch of one)
        kname = {16: "stage_stream_batch_kernel", 8: "stage_stream_kernel",
                 64: "stage_pair_kernel"}.get(form, "stage_stream_kernel")
        kms, klaunch = ks["stream_ms"], ks["stream_launches"]
        kbytes = ks["stream_bytes"]
    else:
        kname, kms, klaunch = "stage_exact_kernel", ks["exact_ms"], ks["stages"]
        kbytes = npts * bpp / 4.0 * ks["stages"]
    achieved = kbytes / (kms / 1e3) / 1e9 if kms > 0 else None
    # PML auxiliaries: every slab point below the free surface reads and
    # writes 27 / 45 / 45 / 27 floats in stages 0..3 (144 B per stage on average)
    npml = desc0.npml
    slab_pts = 0
    if npml > 0:
        kz = desc0.nz - 3
        slab_pts = 2 * npml * desc0.ny * kz + 2 * desc0.nx * npml * kz + desc0.nx * desc0.ny * npml
    aux_bytes = slab_pts * 144.0 * klaunch if kname != "stage_exact_kernel" else 0.0
    achieved_pml = (kbytes + aux_bytes) / (kms / 1e3) / 1e9 if kms > 0 else None
    traffic = measured_traffic(w["name"], kname, args.precision, kbytes, klaunch)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cw = make_workload(cpu_sample_workload(args.workload), 12)
        try:
            sps, ranks, timed = run_reference(cw, 10, os.cpu_count() or 1)
            npc = cw["params"]["NX"] * cw["params"]["NY"] * cw["params"]["NZ"]
            cpu = {"value": npc / sps / 1e9, "unit": UNIT, "cores": ranks, "kind": "reference",
                   "sample": "%s, %d timed steps on %d MPI ranks (reference FP32 CPU build)%s" % (
                       cw["name"], timed, ranks, "" if cw["name"] == w["name"] else
                       "; a bounded sample of %s (same generator, fewer columns)" % w["name"])}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": "unavailable: %s" % str(e)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "fp64": "f64", "fp16": "f16-storage/f32",
                      "bf16": "bf16-storage/f32"}[args.precision],
            "data": "synthetic",
            "config": {"workload": w["name"], "precision": args.precision,
                       "grid": [desc0.nx, desc0.ny, desc0.nz], "points": npts,
                       "kernel": args.kernel, "tile_form": form, "chunk_planes": chunk,
                       "surface_kernel": "tiled" if fast_top else "exact-order",
                       "parallelism": "replicas" if ws > 1 else "single",
                       "l2": "inputs larger than L2 (%.2f GB per wavefield buffer), no flush" % (
                           9 * (desc0.nx + 6) * (desc0.ny + 6) * (desc0.nz + 6) *
                           {"fp32": 4, "fp64": 8}.get(args.precision, 2) / 1e9)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": traffic,
                         "kernel": kname + " (interior and PML launches)", "launches": klaunch,
                         "achieved_incl_pml_aux": achieved_pml,
                         "frac_incl_pml_aux": achieved_pml / peak if achieved_pml else None,
                         "alg_bytes_per_launch": kbytes / max(klaunch, 1),
                         "kernel_ms_avg": kms / max(klaunch, 1),
                         "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_src == "measured" else peak_src,
                         "bytes_per_point_step": bpp,
                         "step_share": {"stream": ks["stream_ms"] / ms,
                                        "free_surface": ks["exact_ms"] / ms}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / e2e_steps,
                    "d2h_bytes_per_step": d2h / e2e_steps, "steps": e2e_steps,
                    "seconds": e2e_max},
            "gpu_launches": ks["launches"],
            "clocks": clk.summary(),
        }
        if accuracy:
            line["accuracy"] = accuracy
        if fp16:
            line["fp16"] = fp16
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
