#!/usr/bin/env python3
"""All-sources heat-method throughput on B200 (sources/s), FastCorticalWiring hot path.

Workload: the order-7 folded icosphere (163,842 vertices, 10% medial-wall cap
removed -> 147,458 cortical sources), t = (0.7 mm)^2, the runner's 12 area
fractions, 3 samples between scales (45 radii per source). A step is one batch
of `--batch` sources (in BFS order, walking through all cortical sources):
heat solve, normalised-gradient divergence, Poisson solve, shift, health,
MSD, distance to boundary, 12 radii + perimeters, 33 samples.

  python bench.py [--gpus N --steps K --warmup W]        # this engine
  python bench.py --impl reference [...]                  # the CPU path, all host cores

`value` is timed on the device (CUDA events, inputs resident in HBM, max over
ranks); `e2e` runs the same steps through the host-buffer public API with the
copies inside the timed region. Each rank holds a full replica of the mesh and
its factors and processes its own slice of the sources (weak scaling).
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "L5": dict(level=5, jitter=0.0), "L6": dict(level=6, jitter=0.2),
    "L7": dict(level=7, jitter=0.0), "L8": dict(level=8, jitter=0.2),
}
METRIC = "sources/s @164k verts"
N_BETWEEN = 3
L2_BYTES = 126 * 1024 * 1024

# DRAM bytes (read + write) per 1024-source block of each stage, mixed precision, from one
# ncu capture on the small L6 workload (36,866 cortical vertices; about 3.5 GB on the device):
#   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum --clock-control none
#       -c 90 -k 'regex:^k_(fwd|bwd|div_mixed|shift_stats|source_metrics|reach)$' --csv
#       python bench.py --workload L6 --batch 1024 --steps 1 --warmup 3 --quick --cpu-sample 0 --pipeline-depth 1
# (the first block's launches). Every stage moves n x K right-hand-side rows, so other meshes
# report these bytes scaled by their vertex count (n / 36,866), labelled as scaled.
TRAFFIC_L6_N = 36866
TRAFFIC_L6 = {
    "heat_fwd": 0.0720e9, "heat_bwd": 0.4775e9, "divergence": 0.4658e9, "poisson_fwd": 0.5230e9,
    "poisson_bwd": 0.3583e9, "shift": 0.2889e9, "metrics": 0.4322e9,
}


def _traffic(stage, n, block_k, precision):
    """(bytes, how) of a stage's DRAM traffic per block, or (None, None)."""
    if block_k != 1024 or precision != "mixed" or stage not in TRAFFIC_L6:
        return None, None
    if n == TRAFFIC_L6_N:
        return TRAFFIC_L6[stage], "ncu capture of this workload (L6)"
    return TRAFFIC_L6[stage] * n / TRAFFIC_L6_N, f"L6 ncu capture scaled by n = {n} / {TRAFFIC_L6_N}"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _mesh(workload, seed):
    from fastcorticalwiring_b200 import mesh as M
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    cfg = WORKLOADS[workload]
    m = folded_icosphere(cfg["level"], seed=seed, jitter=cfg["jitter"])
    return m, M.prepare(m.vertices, m.faces, m.cortex_mask)


# ---------------------------------------------------------------------------
# CPU path: the oracle's per-source pipeline (the reference's algorithm)
# ---------------------------------------------------------------------------
def _cpu_source(ho, pm, targets, s):
    import oracle

    d = ho.distances([int(s)])[0]
    return oracle.source_metrics(d, int(s), pm, targets)


def _cpu_worker(workload, seed, sources, q):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    import oracle
    from fastcorticalwiring_b200 import mesh as M

    _, pm = _mesh(workload, seed)
    targets = pm.targets(M.RUNNER_SCALES)
    ho = oracle.HeatOracle(pm.V, pm.F)
    _cpu_source(ho, pm, targets, sources[0])  # warm caches
    t0 = time.perf_counter()
    recs = [_cpu_source(ho, pm, targets, s) for s in sources]
    sec = time.perf_counter() - t0
    keep = ("radii", "perim", "extra_a", "msd_u", "msd_w", "dist_b", "bad")
    q.put((len(sources), sec, [{k: np.asarray(r[k]).tolist() for k in keep} for r in recs]))


def _start_cpu_baseline(workload, seed, n):
    from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: F401  (import check only)

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    _, pm = _mesh(workload, seed)
    bfs = pm.bfs
    sources = [int(x) for x in bfs[np.linspace(0, bfs.size - 1, n).astype(int)]]
    p = ctx.Process(target=_cpu_worker, args=(workload, seed, sources, q), daemon=True)
    p.start()
    return p, q, sources


def run_reference(args):
    """CPU arm: the oracle's per-source pipeline on every host core (fork after the factorisation)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    import oracle
    from fastcorticalwiring_b200 import mesh as M

    _, pm = _mesh(args.workload, args.seed)
    targets = pm.targets(M.RUNNER_SCALES)
    t0 = time.perf_counter()
    ho = oracle.HeatOracle(pm.V, pm.F)
    factor_s = time.perf_counter() - t0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    per_step = args.ref_sources_per_core
    bfs = pm.bfs
    ctx = mp.get_context("fork")  # no GPU is touched in this arm

    def step(i):
        idx = np.linspace(0, bfs.size - 1, cores * per_step * (args.steps + args.warmup)).astype(int)
        chunk = bfs[idx[i * cores * per_step:(i + 1) * cores * per_step]]
        return [chunk[c::cores] for c in range(cores)]

    global _REF_STATE
    _REF_STATE = (ho, pm, targets)
    times = []
    with ctx.Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            parts = step(i)
            t = time.perf_counter()
            pool.map(_ref_task, parts)
            if i >= args.warmup:
                times.append(time.perf_counter() - t)
    total = args.steps * cores * per_step
    sec = sum(times)
    value = total / sec
    line = {
        "metric": METRIC, "value": value, "unit": "sources/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(args, pm, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": "sources/s", "cores": cores, "kind": "port",
                         "sample": f"{per_step} sources per core per step, BFS-spaced over all "
                                   f"{pm.n_vertices} sources; factorisation ({factor_s:.1f} s) excluded"},
        "e2e": {"value": value, "unit": "sources/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


_REF_STATE = None


def _ref_task(srcs):
    ho, pm, targets = _REF_STATE
    for s in srcs:
        _cpu_source(ho, pm, targets, s)
    return len(srcs)


def _config(args, pm, world=1):
    return {"workload": f"{args.workload} folded icosphere, {pm.n_vertices} cortical sources, "
                        f"{pm.n_faces} faces, t=(0.7 mm)^2, 12 scales + {N_BETWEEN} samples between",
            "batch_sources_per_step": args.batch, "block_k": args.block_k, "precision": args.precision,
            "pipeline_depth": args.pipeline_depth, "leaf_size": args.leaf_size, "relax": args.relax,
            "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (n x K RHS blocks > 126 MB)"}


# ---------------------------------------------------------------------------
# ranks: one process per GPU
# ---------------------------------------------------------------------------
def rank_env():
    """(rank, world size, local rank) of this process, from torchrun's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def free_port():
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_ranks(script, argv, nproc, timeout_s=None):
    """Run `script argv` as nproc processes under torch.distributed.run on this node (rendezvous on
    127.0.0.1, one rank per GPU); returns the launcher's exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={int(nproc)}",
           "--master-addr", "127.0.0.1", f"--master-port={free_port()}", script, *argv]
    return subprocess.call(cmd, timeout=timeout_s)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device), "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
            os.unlink(self.path)
        except Exception:
            pass
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=reasons, samples=len(rows))
        return out


def _stage_bytes(stage, n, nf, K, nnz_factor, precision, nreached_rows=None):
    """Algorithmic bytes of one execution of a stage on a K-source block."""
    b = 4 if precision == "mixed" else 8
    if stage == "heat_bwd":
        return nnz_factor * 8 + 2 * n * K * 8
    if stage in ("poisson_fwd", "poisson_bwd"):
        return nnz_factor * b + 2 * n * K * b
    if stage == "divergence":
        return n * K * 8 + n * K * b + nf * (3 * 4 + 4 * 4) + 3 * nf * 5
    if stage == "shift":
        return 2 * n * K * b
    if stage == "metrics":
        return n * K * b + n * 32
    if stage == "heat_fwd":
        return nnz_factor * 8
    return 0


def shard_sources(order, world, rank):
    """Rank `rank`'s contiguous slice of the BFS order: every source on exactly one rank (the
    product's sharding, fastcorticalwiring_b200.sharded)."""
    from fastcorticalwiring_b200 import sharded

    return sharded.shard(order, world, rank)


def max_over_ranks(x, dist, device):
    """The slowest rank's value, on every rank (a multi-rank time is the max over ranks)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_gpu(args):
    rank, world, local = rank_env()
    cpu = None
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        cpu = _start_cpu_baseline(args.workload, args.seed, args.cpu_sample)  # before any CUDA call

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from fastcorticalwiring_b200 import engine as E
    from fastcorticalwiring_b200 import mesh as M

    dev = local if world > 1 else args.device
    torch.cuda.set_device(dev)
    _, pm = _mesh(args.workload, args.seed)
    targets = pm.targets(M.RUNNER_SCALES)
    tuned = None
    if args.autotune:
        from fastcorticalwiring_b200.autotune import autotune

        t0 = time.perf_counter()
        best, trials = autotune(pm, precision=args.precision, device=dev)
        args.block_k, args.pipeline_depth = best["block_k"], best["pipeline_depth"]
        tuned = {"chosen": best, "tune_s": time.perf_counter() - t0,
                 "trials": [{k: (round(v, 1) if isinstance(v, float) else v) for k, v in t.items()} for t in trials]}
    t0 = time.perf_counter()
    eng = E.HeatEngine(pm.V, pm.F, device=dev, block_k=args.block_k, pipeline_depth=args.pipeline_depth,
                       leaf_size=args.leaf_size, relax=args.relax, tc_sweeps=int(args.tc_sweeps))
    eng.graphs(not args.no_graphs)
    build_s = time.perf_counter() - t0
    info = eng.info()

    bfs = pm.bfs.astype(np.int32)
    share = shard_sources(bfs, world, rank)
    # a step never holds more sources than every rank's slice (the mesh may be smaller than a batch)
    B = args.batch = min(args.batch, bfs.size // world)
    stride = E._lib.metrics_stride(12, N_BETWEEN)
    src_dev = torch.from_numpy(share.copy()).to(f"cuda:{dev}")
    out_dev = torch.empty((B, stride), dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)
    nsteps_avail = max(1, share.size // B)

    def step_slice(i):
        j = i % nsteps_avail
        return src_dev[j * B:(j + 1) * B]

    def device_step(i, precision=args.precision):
        eng.compute_metrics_device(step_slice(i), targets, N_BETWEEN, 1e-6, precision, out_dev,
                                   stream.cuda_stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    for i in range(args.warmup):
        device_step(i)
    eng.synchronize(stream.cuda_stream)

    # --- device-timed region (no stage marks inside it; the launch counter restarts here) ---
    clocks = ClockSampler(dev)
    clocks.start()
    eng.profile(False)
    torch.cuda.synchronize()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        device_step(args.warmup + i)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    _, launches = eng.stage_times()
    clk = clocks.stop()
    eng.synchronize(stream.cuda_stream)

    # --- stage durations for the roofline: blocks one at a time, so a stage's
    # CUDA-event span is its own duration, not shared with the other streams ---
    nprof = 3
    K = args.block_k
    prof_out = torch.empty((K, stride), dtype=torch.float64, device=f"cuda:{dev}")  # a block's records
    eng.profile(True)
    for i in range(nprof):
        j = i % max(1, share.size // K)
        eng.compute_metrics_device(src_dev[j * K:(j + 1) * K], targets, N_BETWEEN, 1e-6, args.precision, prof_out,
                                   stream.cuda_stream)
        eng.synchronize(stream.cuda_stream)
    stages, _ = eng.stage_times()
    eng.profile(False)
    stages = {k: v / nprof for k, v in stages.items()}  # ms per block
    ms = max_over_ranks(ms, dist, f"cuda:{dev}")
    total_sources = B * args.steps * world
    value = total_sources / (ms / 1e3)

    # --- end to end through the host-buffer API (pinned host memory) ---
    h_src = torch.from_numpy(share[:B * min(nsteps_avail, args.steps)].copy()).pin_memory().numpy()
    h_out = torch.empty((B, stride), dtype=torch.float64).pin_memory().numpy()
    lib = E._lib.load()
    import ctypes

    tgt = np.ascontiguousarray(targets)
    prec = E._precision(args.precision)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        j = i % min(nsteps_avail, args.steps)
        s = h_src[j * B:(j + 1) * B]
        E._lib.check(lib.fcw_compute_metrics(eng.handle, ctypes.c_void_p(s.ctypes.data), s.size, prec,
                                             E._lib.ptr(tgt), tgt.size, N_BETWEEN, 1e-6, E._lib.ptr(h_out)))
    e2e_s = time.perf_counter() - t0
    barrier()
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{dev}")
    e2e = total_sources / e2e_s

    extra = {}
    if rank == 0 and not args.quick:
        extra = _fp64_forms_and_errors(eng, pm, targets, stream, args, dev)

    if rank == 0:
        hbm, peak_kind = _peaks()
        dom = max(stages, key=stages.get) if stages else None
        roof = None
        if dom and stages[dom] > 0:
            per_block_s = stages[dom] / 1e3
            byts = _stage_bytes(dom, pm.n_vertices, pm.n_faces, args.block_k, info["nnz_factor"], args.precision)
            ach = byts / per_block_s / 1e9
            traffic, traffic_from = _traffic(dom, pm.n_vertices, args.block_k, args.precision)
            roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "unit": "GB/s",
                    "frac": ach / hbm, "traffic": traffic, "traffic_from": traffic_from,
                    "peak_kind": peak_kind,
                    "bytes_per_launch": byts, "launch": f"one {dom} stage on a {args.block_k}-source block"}
        line = {
            "metric": METRIC, "value": value, "unit": "sources/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 heat / f32 Poisson" if args.precision == "mixed" else "f64",
            "data": "synthetic", "config": _config(args, pm, world),
            "e2e": {"value": e2e, "unit": "sources/s", "h2d_bytes_per_step": B * 4 * world,
                    "d2h_bytes_per_step": B * stride * 8 * world},
            "gpu_launches": launches,
            "roofline": roof,
            "stage_ms_per_block": {k: round(v, 3) for k, v in stages.items()},
            "clocks": clk,
            "engine": {"factor_ms": info["factor_ms"], "analyze_ms": info["analyze_ms"], "build_s": build_s,
                       "n_supernodes": info["n_supernodes"], "n_levels": info["n_levels"],
                       "nnz_factor": info["nnz_factor"], "nnz_l": info["nnz_l"],
                       "device_bytes": info["device_bytes"], "tc_sweeps": bool(args.tc_sweeps),
                       "pipeline_depth_held": info["pipeline_depth"], "cuda_graphs": not args.no_graphs},
        }
        line.update(extra)
        if tuned is not None:
            line["autotune"] = tuned
        if cpu is not None:
            p, q, cpu_sources = cpu
            try:
                cnt, sec, cpu_recs = q.get(timeout=args.cpu_timeout)
                line["cpu_baseline"] = {"value": cnt / sec, "unit": "sources/s", "cores": 1, "kind": "port",
                                        "sample": f"{cnt} BFS-spaced sources of the same mesh, one at a time, "
                                                  "single thread, factorisation excluded"}
                line["err_vs_oracle"] = _errors_vs_oracle(eng, cpu_sources, cpu_recs, targets)
            except Exception as exc:
                line["cpu_baseline"] = {"value": None, "unit": "sources/s", "cores": 1, "kind": "port",
                                        "sample": f"not finished: {exc!r}"}
            p.join(timeout=5)
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _errors_vs_oracle(eng, sources, recs, targets):
    """Largest relative error of the engine (both forms) against the oracle's FP64 records of the
    CPU-baseline sample, over the sources neither side flags; and the flag disagreements."""
    from fastcorticalwiring_b200 import engine as E

    src = np.asarray(sources, dtype=np.int32)
    obad = np.array([bool(r["bad"]) for r in recs])
    out = {"sources": int(src.size), "oracle_flagged": int(obad.sum())}
    for prec in ("fp64", "mixed"):
        r = E.split_records(eng.compute_metrics(src, targets, N_BETWEEN, precision=prec), 12, N_BETWEEN)
        ok = ~(obad | r["bad"])
        e = {"flag_mismatch": int(np.sum(obad != r["bad"]))}
        for key, okey in (("radii", "radii"), ("perim", "perim"), ("extra_a", "extra_a"), ("msd_u", "msd_u"),
                          ("msd_w", "msd_w"), ("dist_b", "dist_b")):
            ref = np.array([np.asarray(x[okey], float) for x in recs])
            got = np.asarray(r[key], float)
            rel = np.abs(got[ok] - ref[ok]) / np.maximum(np.abs(ref[ok]), 1e-300)
            e[key] = float(np.nanmax(rel)) if rel.size else None
        out[prec] = e
    return out


def _fp64_forms_and_errors(eng, pm, targets, stream, args, dev):
    """The plain FP64 drop-in (one source per call) and the accuracy of the mixed form."""
    import torch

    from fastcorticalwiring_b200 import engine as E

    bfs = pm.bfs.astype(np.int32)
    # drop-in: one source per call, FP64, all metrics, host result
    sample = bfs[np.linspace(0, bfs.size - 1, args.fp64_sample).astype(int)]
    eng.compute_metrics(sample[:1], targets, N_BETWEEN, precision="fp64")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in sample:
        eng.compute_metrics(np.array([s], np.int32), targets, N_BETWEEN, precision="fp64")
    dropin = len(sample) / (time.perf_counter() - t0)
    # the distances-only drop-in (fcw_compute_distance, the reference loop's engine call):
    # one source per call, field returned in a host array
    eng.compute_distance(int(sample[0]))
    n_dist = 4 * len(sample)
    dsample = bfs[np.linspace(0, bfs.size - 1, n_dist).astype(int)]
    t0 = time.perf_counter()
    for s in dsample:
        eng.compute_distance(int(s))
    dist_only = n_dist / (time.perf_counter() - t0)
    # batched FP64 (same blocks as the headline, device timed)
    B = min(args.batch, bfs.size)
    src = torch.from_numpy(bfs[:B].copy()).to(f"cuda:{dev}")
    stride = E._lib.metrics_stride(12, N_BETWEEN)
    out = torch.empty((B, stride), dtype=torch.float64, device=f"cuda:{dev}")
    eng.compute_metrics_device(src, targets, N_BETWEEN, 1e-6, "fp64", out, stream.cuda_stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(2):
        eng.compute_metrics_device(src, targets, N_BETWEEN, 1e-6, "fp64", out, stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    fp64_batched = 2 * B / (ev0.elapsed_time(ev1) / 1e3)
    # accuracy of the mixed form against the FP64 engine on one block
    n = min(args.block_k, bfs.size)
    chk = bfs[np.linspace(0, bfs.size - 1, n).astype(int)]
    r64 = E.split_records(eng.compute_metrics(chk, targets, N_BETWEEN, precision="fp64"), 12, N_BETWEEN)
    r32 = E.split_records(eng.compute_metrics(chk, targets, N_BETWEEN, precision="mixed"), 12, N_BETWEEN)
    ok = ~(r64["bad"] | r32["bad"])

    def rel(a, b):
        a, b = a[ok], b[ok]
        return float(np.nanmax(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) if a.size else None

    d64 = eng.compute_distances(chk[:4], precision="fp64")
    d32 = eng.compute_distances(chk[:4], precision="mixed")
    return {
        "fp64_forms": {"dropin_sources_per_s": dropin, "dropin_distance_only_per_s": dist_only,
                       "batched_sources_per_s": fp64_batched, "sample": f"{len(sample)} sources one per call"},
        "err_mixed_vs_fp64": {"radius": rel(r32["radii"], r64["radii"]), "perimeter": rel(r32["perim"], r64["perim"]),
                              "msd_unweighted": rel(r32["msd_u"], r64["msd_u"]),
                              "msd_weighted": rel(r32["msd_w"], r64["msd_w"]),
                              "sample_area": rel(r32["extra_a"], r64["extra_a"]),
                              "phi_max_abs_over_max": float(np.max(np.abs(d32 - d64)) / np.max(np.abs(d64))),
                              "flag_mismatch": int(np.sum(r64["bad"] != r32["bad"])), "sources": int(n)},
    }


def run_serving(args):
    """The serving stream (hemisphere jobs of mixed sizes arriving as a Poisson process).

    Jobs: 40% order-5, 40% order-6 (jitter 0.2), 20% order-7 folded icospheres, each with
    its own folding seed and a medial-wall cap of 8-12% of the vertices, all cortical
    sources per job. For each arrival rate the server admits jobs against the HBM
    budget and reports p50/p99 job latency (arrival to results on the host) and the
    stream's sources/s (all sources over the time from the first arrival to the last
    result). Meshes are generated before the stream starts.
    """
    import torch

    from fastcorticalwiring_b200 import serving
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    rng = np.random.default_rng(args.seed)
    n = args.serving_jobs
    levels = rng.choice([5, 6, 7], size=n, p=[0.4, 0.4, 0.2])
    jobs = []
    for i, lv in enumerate(levels):
        m = folded_icosphere(int(lv), seed=1000 + i, jitter=0.2 if lv == 6 else 0.0,
                             cap_fraction=float(rng.uniform(0.08, 0.12)))
        jobs.append(serving.Job(f"job{i}-L{lv}", m.vertices, m.faces, m.cortex_mask, precision=args.precision))
    torch.cuda.set_device(args.device)
    rows = []
    for rate in [float(x) for x in args.serving_rates.split(",")]:
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
        arrivals -= arrivals[0]
        srv = serving.Server(hbm_budget_bytes=args.hbm_budget_gb * 1e9, device=args.device,
                             engine_params=dict(block_k=args.block_k, pipeline_depth=2))
        try:
            t0 = time.perf_counter()
            res = srv.run(list(zip(arrivals.tolist(), jobs)))
            span = time.perf_counter() - t0
        finally:
            srv.close()
        lat = serving.latency_summary(res)
        total = sum(r.sources.size for r in res.values())
        by_level = {}
        for r in res.values():
            by_level.setdefault(r.job_id.split("-")[1], []).append(r.latency_s)
        rows.append({"rate_jobs_per_s": rate, "sources_per_s": total / span, "sources": int(total),
                     "span_s": span, **lat,
                     "p50_s_by_level": {k: float(np.percentile(v, 50)) for k, v in sorted(by_level.items())},
                     "peak_device_bytes_per_job": int(max(r.device_bytes for r in res.values()))})
    line = {"metric": "serving: job p50/p99 latency and sources/s", "unit": "s / sources/s", "n_gpus": 1,
            "jobs": n, "mix": {"L5": int((levels == 5).sum()), "L6": int((levels == 6).sum()),
                               "L7": int((levels == 7).sum())},
            "hbm_budget_gb": args.hbm_budget_gb, "precision": args.precision, "block_k": args.block_k,
            "data": "synthetic", "rates": rows}
    print(json.dumps(line))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="L7")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--batch", type=int, default=16384, help="sources per step")
    ap.add_argument("--block-k", type=int, default=1024)
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--pipeline-depth", type=int, default=4, help="blocks in flight on separate streams")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--leaf-size", type=int, default=64, help="nested-dissection leaf size")
    ap.add_argument("--relax", type=int, default=64, help="relaxed supernode amalgamation (columns)")
    ap.add_argument("--cpu-sample", type=int, default=24, help="sources timed on the CPU oracle (0 = skip)")
    ap.add_argument("--cpu-timeout", type=float, default=600.0)
    ap.add_argument("--fp64-sample", type=int, default=16)
    ap.add_argument("--ref-sources-per-core", type=int, default=2)
    ap.add_argument("--quick", action="store_true", help="skip the FP64 forms and the accuracy check")
    ap.add_argument("--no-graphs", action="store_true", help="launch each block's kernels directly")
    ap.add_argument("--tc-sweeps", type=int, default=0, choices=(0, 1),
                    help="mixed Poisson sweeps on the tensor cores (1) or on FMA register tiles (0)")
    ap.add_argument("--autotune", action="store_true", help="choose block size and depth on the mesh first")
    ap.add_argument("--serving", action="store_true", help="run the serving stream instead (own JSON line)")
    ap.add_argument("--serving-jobs", type=int, default=64)
    ap.add_argument("--serving-rates", default="0.5,2,8", help="Poisson arrival rates, jobs/s")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    args = ap.parse_args(argv)
    if args.serving:
        return run_serving(args)
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    _, world, _ = rank_env()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # one process per GPU: start the ranks here when no launcher did
        return launch_ranks(os.path.abspath(__file__), sys.argv[1:] if argv is None else list(argv), args.gpus)
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; start one rank per GPU "
              f"(torchrun --nproc-per-node {args.gpus}) or drop the launcher", file=sys.stderr)
        return 2
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
