"""Block-size autotuner: the sources per block (K) and blocks in flight for one mesh.

Each candidate (K, depth) builds an engine on the mesh, runs one untimed block
and then at least `min_sources` sources through the device metrics path, timed
with CUDA events on the caller's stream. The fastest candidate wins; ties go to
the smaller memory footprint (smaller K x depth). Candidates that do not fit on
the device (engine creation fails for memory) are skipped.
"""

from __future__ import annotations

import itertools
import time

import numpy as np

from . import _lib
from . import engine as E
from . import mesh as M

DEFAULT_K = (64, 128, 256, 512, 1024)
DEFAULT_DEPTH = (1, 2, 3, 4)


def autotune(pm: M.PreparedMesh, scales=M.RUNNER_SCALES, n_between=3, precision="mixed", ks=DEFAULT_K,
             depths=DEFAULT_DEPTH, min_sources=4096, device=0):
    """Returns (best {'block_k', 'pipeline_depth', 'sources_per_s'}, list of all trials)."""
    import torch

    torch.cuda.set_device(device)
    targets = pm.targets(scales)
    stride = _lib.metrics_stride(targets.size, n_between)
    bfs = pm.bfs.astype(np.int32)
    dev = f"cuda:{device}"
    stream = torch.cuda.Stream(device=device)
    trials = []
    for k, d in itertools.product(ks, depths):
        n = max(int(min_sources), k * d)
        src = torch.from_numpy(np.resize(bfs, n + k).copy()).to(dev)
        out = torch.empty((n + k, stride), dtype=torch.float64, device=dev)
        try:
            eng = E.HeatEngine(pm.V, pm.F, device=device, block_k=k, pipeline_depth=d)
        except _lib.FCWError as exc:
            if exc.code == _lib.FCW_E_NOMEM:
                continue
            raise
        try:
            held = eng.info()["pipeline_depth"]
            eng.compute_metrics_device(src[:k], targets, n_between, 1e-6, precision, out[:k], stream.cuda_stream)
            eng.synchronize(stream.cuda_stream)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            eng.compute_metrics_device(src[k:k + n], targets, n_between, 1e-6, precision, out[k:k + n],
                                       stream.cuda_stream)
            ev1.record(stream)
            eng.synchronize(stream.cuda_stream)
            ms = ev0.elapsed_time(ev1)
        finally:
            eng.close()
        if held < d:
            continue  # the device held fewer blocks in flight: counted under the smaller depth
        trials.append({"block_k": k, "pipeline_depth": d, "sources": n, "ms": ms, "sources_per_s": n / (ms / 1e3)})
    if not trials:
        raise RuntimeError("no block size fits on the device")
    best = max(trials, key=lambda t: (round(t["sources_per_s"], -1), -t["block_k"] * t["pipeline_depth"]))
    return dict(best), trials


def main(argv=None):
    """python -m fastcorticalwiring_b200.autotune --level 6: tune on a seeded folded icosphere."""
    import argparse
    import json

    from .meshgen import folded_icosphere

    ap = argparse.ArgumentParser()
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--jitter", type=float, default=0.2)
    ap.add_argument("--precision", default="mixed")
    args = ap.parse_args(argv)
    m = folded_icosphere(args.level, seed=args.seed, jitter=args.jitter)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    t0 = time.perf_counter()
    best, trials = autotune(pm, precision=args.precision)
    print(json.dumps({"best": best, "trials": trials, "tune_s": time.perf_counter() - t0}))


if __name__ == "__main__":
    main()
