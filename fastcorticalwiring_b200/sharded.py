"""One subject over several GPUs: the sources shard, the mesh and its factors replicate.

One process per GPU (started by torchrun, or any launcher that sets RANK, WORLD_SIZE and
LOCAL_RANK), each with its own engine on its own device. Rank r computes the metric records
of its contiguous slice of the BFS source order (every source on exactly one rank; slices
differ by at most one source). The records are then gathered, in rank order, to every rank
by one all_gather over the process group (NCCL between GPUs, gloo between CPU processes),
and each rank assembles the samples and the per-vertex arrays of the whole mesh from the
gathered records, as a one-GPU run does from its own. A source's field needs only the
replicated factors, so nothing is exchanged inside the solves.

The reference parallelises across subjects, one process per subject (run_pipeline.py:20-100,
326-342); runner.py keeps that grain on one GPU, and this module adds the finer one: one
subject's sources over several GPUs.
"""

from __future__ import annotations

import os
import time

import numpy as np

from . import _lib
from .analysis import WiringAnalysis


def shard(order, world: int, rank: int) -> np.ndarray:
    """Rank `rank`'s contiguous slice of `order`: every entry on exactly one rank, slices in
    rank order, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    return np.array_split(np.asarray(order), world)[rank]


def _group_info(group):
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1, None
    return dist.get_rank(group), dist.get_world_size(group), dist.get_backend(group)


def gather_rows(local: np.ndarray, group=None) -> np.ndarray:
    """The ranks' float64 row blocks (same number of columns, any number of rows), stacked in
    rank order, on every rank. One all_gather of blocks padded to the longest: CUDA tensors
    on the current device for NCCL, host tensors otherwise. Without a process group, the
    block itself."""
    local = np.ascontiguousarray(local, dtype=np.float64)
    rank, world, backend = _group_info(group)
    if backend is None:
        return local.copy()
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    cols = local.shape[1]
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(x.item()) for x in sizes]
    most = max(sizes)
    buf = torch.zeros((most, cols), dtype=torch.float64, device=dev)
    if local.shape[0]:
        buf[: local.shape[0]] = torch.from_numpy(local).to(dev)
    out = torch.empty((world * most, cols), dtype=torch.float64, device=dev)
    dist.all_gather_into_tensor(out, buf, group=group)
    out = out.cpu().numpy()
    return np.concatenate([out[r * most: r * most + sizes[r]] for r in range(world)])


class ShardedWiringAnalysis(WiringAnalysis):
    """WiringAnalysis whose compute_all_wiring_costs shards the sources over the ranks of a
    torch.distributed process group (`group`, default the world; with no process group it
    is WiringAnalysis on one device).

    Every rank constructs it with the same mesh and arguments and makes the same calls in
    the same order; every rank ends with the whole result. The engine goes to the device
    named by engine_kwargs["device"], by default LOCAL_RANK.
    """

    def __init__(self, vertices, faces, cortex_mask, engine_type="b200", engine_kwargs=None, group=None,
                 **kwargs):
        kw = dict(engine_kwargs or {})
        kw.setdefault("device", int(os.environ.get("LOCAL_RANK", "0")))
        self.group = group
        self.quiet = _group_info(group)[0] != 0  # rank 0 alone prints the run's reports
        super().__init__(vertices, faces, cortex_mask, engine_type=engine_type, engine_kwargs=kw, **kwargs)

    def compute_all_wiring_costs(self, scale=None, area_tol=None, vertex_subset=None, n_samples_between_scales=3,
                                 boundary_cap_fraction=None, batch_size=None, verbose=False):
        """As WiringAnalysis.compute_all_wiring_costs (core_analysis.py:1441-1672), with each rank
        computing its slice of the sources and the records gathered to every rank. Every rank
        returns the same arrays; rank 0 prints the end-of-run report."""
        t0 = time.perf_counter()
        scales, m, cap = self.run_arguments(scale, n_samples_between_scales, boundary_cap_fraction)
        targets = self._reset(scales, m, cap)
        order = self._sources(vertex_subset)
        rank, world, _ = _group_info(self.group)
        mine = shard(order, world, rank)
        eng = self.distance_engine.engine
        parts = [eng.compute_metrics(mine[b0:b0 + self.block_sources], targets, n_between=m, eps=self.eps,
                                     precision=self.precision)
                 for b0 in range(0, mine.size, self.block_sources)]
        stride = _lib.metrics_stride(len(targets), m)
        local = np.concatenate(parts) if parts else np.empty((0, stride), dtype=np.float64)
        rec = gather_rows(local, self.group)
        if order.size:
            self._absorb(order, rec, eng.assemble_samples(rec, targets, n_between=m, boundary_cap=cap))
        flagged = self._finish(order.size)
        self.report(order.size, flagged, time.perf_counter() - t0)
        return (self.msd_unweighted, self.msd_weighted), self.radius_function, self.perimeter_function
