"""A request loop for hemisphere jobs on one GPU: continuous batching under an HBM budget.

Jobs (a cortical mesh, its scales, the sources to run) arrive at any time. Builder
threads admit them when their device memory fits the budget (in arrival order,
except that a job that fits may pass a head job waiting for memory a bounded
number of times; a job whose estimate exceeds the whole budget is refused with a
result that carries the reason), prepare the mesh and factor it; the factors and the job's
right-hand-side blocks stay resident until the job is done. The dispatch loop
keeps the next chunk of source blocks of the few admitted jobs with the least
work left enqueued on each job's own stream, so their blocks overlap on the
device, and a job that arrives while others run starts as soon as memory frees
up and it is among the shortest. Each job
reports its latency (arrival to results on the host) beside the whole stream's
throughput.

The results are the per-source metric records of `fcw_compute_metrics` (see
include/fcw_b200.h), in the order of the job's sources.
"""

from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

from . import engine as E
from . import mesh as M


@dataclass
class Job:
    job_id: str
    vertices: np.ndarray
    faces: np.ndarray
    cortex_mask: np.ndarray
    scales: tuple = M.RUNNER_SCALES
    n_between: int = 3
    sources: np.ndarray | None = None  # cortical sub-indices; None = all, in BFS order
    precision: str = "mixed"
    eps: float = 1e-6
    prepared: M.PreparedMesh | None = None  # the mesh already prepared on the host (else done on admission)


@dataclass
class JobResult:
    job_id: str
    sources: np.ndarray
    records: np.ndarray
    t_arrive: float
    t_admit: float
    t_done: float
    device_bytes: int
    n_vertices: int
    estimate_bytes: int = 0
    engine_info: dict | None = None
    error: str | None = None  # set when the job was refused (no records)

    @property
    def latency_s(self) -> float:
        return self.t_done - self.t_arrive


@dataclass(eq=False)
class _Active:
    job: Job
    eng: E.HeatEngine
    sources: np.ndarray
    targets: np.ndarray
    src_dev: object
    out_dev: object
    stream: object
    reserved: int
    t_arrive: float
    t_admit: float
    estimate: int = 0
    next0: int = 0
    event: object = None
    chunk: int = 0


@dataclass
class _Pending:
    job: Job
    t_arrive: float
    estimate: int = 0


def _stride(nt, nb):
    return 7 + 2 * nt + 2 * (nt - 1) * nb


def estimate_device_bytes(n_vertices: int, n_faces: int, block_k: int, pipeline_depth: int, n_sources: int,
                          stride: int) -> int:
    """Upper estimate of a job's device memory before it is factored.

    Per workspace and right-hand side about 100 bytes per vertex (four FP64 n x K
    arrays, the near-vertex lists, the update rows at ~2.65 n, and the per-source
    face band of 20 bytes per face), plus factors and mesh arrays (~3 KB per
    vertex at these fills) and the job's source list and result records.
    """
    ws = int(block_k) * (n_vertices * 60 + n_faces * 20 + int(2.65 * n_vertices * 8) + stride * 8)
    return pipeline_depth * ws + 3000 * n_vertices + n_sources * (4 + stride * 8) + (64 << 20)


class Server:
    """Continuous batching of hemisphere jobs on one GPU under an HBM budget (bytes)."""

    def __init__(self, hbm_budget_bytes=150e9, device=0, chunk_blocks=8, engine_params=None, builders=4,
                 max_running=3, max_bypass=8):
        import torch

        self.torch = torch
        self.device = int(device)
        self.budget = int(hbm_budget_bytes)
        self.chunk_blocks = int(chunk_blocks)
        self.max_running = max(1, int(max_running))  # jobs with source blocks on the device at once
        self.max_bypass = int(max_bypass)  # admissions that may pass a head job waiting for memory
        self.params = dict(block_k=1024, pipeline_depth=2)
        self.params.update(engine_params or {})
        self._cv = threading.Condition()
        self._pending: deque[_Pending] = deque()
        self._ready: deque[_Active] = deque()
        self._reserved = 0
        self._bypassed = 0
        self._n_open = 0  # submitted and not finished
        self._closed = False
        self._error: BaseException | None = None
        self.results: dict[str, JobResult] = {}
        # builders prepare and factor admitted jobs in parallel (mesh preparation and
        # the symbolic analysis run on the host); admission itself stays in arrival order
        self._builders = [threading.Thread(target=self._build_loop, name=f"fcw-serving-builder-{i}", daemon=True)
                          for i in range(max(1, int(builders)))]
        for t in self._builders:
            t.start()

    # -- public ----------------------------------------------------------------
    def submit(self, job: Job) -> None:
        """Queue a job; its latency clock starts now."""
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._pending.append(_Pending(job, time.perf_counter()))
            self._n_open += 1
            self._cv.notify_all()

    def run(self, jobs_with_arrivals, poll_s=2e-4):
        """Submit (arrival_offset_s, Job) pairs at their offsets and serve until all are done."""
        schedule = sorted(jobs_with_arrivals, key=lambda x: x[0])
        t0 = time.perf_counter()
        i = 0
        active: list[_Active] = []
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            now = time.perf_counter() - t0
            while i < len(schedule) and schedule[i][0] <= now:
                self.submit(schedule[i][1])
                i += 1
            with self._cv:
                if self._error is not None:
                    raise self._error
                while self._ready:
                    active.append(self._ready.popleft())
                if i == len(schedule) and self._n_open == 0:
                    break
            progressed = False
            for a in list(active):
                if a.event is not None and a.event.query():
                    a.event = None
                    progressed = True
                    if a.next0 >= a.sources.size:
                        self._finish(a)
                        active.remove(a)
            # shortest remaining work first: the jobs with the fewest sources left keep a
            # chunk on the device; the others stay resident and wait their turn
            active.sort(key=lambda x: x.sources.size - x.next0)
            for a in active[:self.max_running]:
                if a.event is None and a.next0 < a.sources.size:
                    self._enqueue(a)
                    progressed = True
            if not progressed:
                time.sleep(poll_s)
        return self.results

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._builders:
            t.join(timeout=60)

    # -- internals -------------------------------------------------------------
    def _enqueue(self, a: _Active) -> None:
        n = min(self.chunk_blocks * a.eng.block_k, a.sources.size - a.next0)
        j = a.job
        a.eng.compute_metrics_device(a.src_dev[a.next0:a.next0 + n], a.targets, j.n_between, j.eps, j.precision,
                                     a.out_dev[a.next0:a.next0 + n], a.stream.cuda_stream)
        a.event = self.torch.cuda.Event()
        a.event.record(a.stream)
        a.next0 += n
        a.chunk += 1

    def _finish(self, a: _Active) -> None:
        a.stream.synchronize()
        a.eng.synchronize(a.stream.cuda_stream)  # surfaces kernel error flags
        rec = a.out_dev.cpu().numpy()
        t_done = time.perf_counter()
        info = a.eng.info()
        info_bytes = int(info["device_bytes"])
        a.eng.close()
        a.src_dev = a.out_dev = None  # back to the tensor cache; no device-wide free
        res = JobResult(a.job.job_id, a.sources, rec, a.t_arrive, a.t_admit, t_done, info_bytes,
                        int(a.sources.size), a.estimate, info)
        with self._cv:
            self.results[a.job.job_id] = res
            self._reserved -= a.reserved
            self._n_open -= 1
            self._cv.notify_all()

    def _build_loop(self):
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            with self._cv:
                # admission in arrival order: take the head job once it fits the budget
                # (or once nothing else is resident)
                while True:
                    if self._closed:
                        return
                    p = self._pick()
                    if p is not None:
                        self._reserved += p.estimate
                        break
                    self._cv.wait()
            try:
                act = self._admit(p)
            except BaseException as exc:  # surfaced by run()
                with self._cv:
                    self._reserved -= p.estimate
                    self._error = exc
                    self._cv.notify_all()
                return
            with self._cv:
                # hold the larger of the estimate and what the engine allocated
                act.reserved = max(act.reserved, p.estimate)
                act.estimate = p.estimate
                self._reserved += act.reserved - p.estimate
                self._ready.append(act)
                self._cv.notify_all()

    def _estimate(self, p: _Pending) -> int:
        if not p.estimate:
            job = p.job
            nv = int(np.count_nonzero(job.cortex_mask))
            nsrc = nv if job.sources is None else int(np.asarray(job.sources).size)
            p.estimate = estimate_device_bytes(nv, 2 * nv, self.params["block_k"], self.params["pipeline_depth"],
                                               nsrc, _stride(len(job.scales), job.n_between))
        return p.estimate

    def _pick(self):
        """The next job to admit (caller holds the lock): the head of the queue if it fits
        the budget (or nothing is resident); else the first later job that fits, while the
        head has been passed fewer than max_bypass times."""
        # a job whose estimate exceeds the whole budget can never be admitted: refuse it
        while self._pending and self._estimate(self._pending[0]) > self.budget:
            self._refuse(self._pending.popleft())
        if not self._pending:
            return None
        head = self._pending[0]
        if self._reserved == 0 or self._reserved + self._estimate(head) <= self.budget:
            self._bypassed = 0
            return self._pending.popleft()
        if self._bypassed >= self.max_bypass:
            return None
        for i in range(1, len(self._pending)):
            q = self._pending[i]
            if self._reserved + self._estimate(q) <= self.budget:
                del self._pending[i]
                self._bypassed += 1
                return q
        return None

    def _refuse(self, p: _Pending) -> None:
        """Record a job that cannot fit the HBM budget (caller holds the lock)."""
        now = time.perf_counter()
        msg = (f"job {p.job.job_id!r} needs an estimated {p.estimate / 1e9:.2f} GB of device memory, more than "
               f"the {self.budget / 1e9:.2f} GB budget")
        self.results[p.job.job_id] = JobResult(p.job.job_id, np.zeros(0, np.int32), np.zeros((0, 0)), p.t_arrive,
                                               now, now, 0, 0, p.estimate, None, error=msg)
        self._n_open -= 1
        self._cv.notify_all()

    def _admit(self, p: _Pending) -> _Active:
        torch = self.torch
        job = p.job
        pm = job.prepared if job.prepared is not None else M.prepare(job.vertices, job.faces, job.cortex_mask)
        eng = E.HeatEngine(pm.V, pm.F, device=self.device, **self.params)
        src = pm.bfs.astype(np.int32) if job.sources is None else np.asarray(job.sources, dtype=np.int32)
        targets = pm.targets(job.scales)
        stride = _stride(targets.size, job.n_between)
        dev = f"cuda:{self.device}"
        src_dev = torch.from_numpy(src.copy()).to(dev)
        out_dev = torch.empty((src.size, stride), dtype=torch.float64, device=dev)
        stream = torch.cuda.Stream(device=self.device)
        reserved = int(eng.info()["device_bytes"]) + src.size * (4 + stride * 8)
        return _Active(job, eng, src, targets, src_dev, out_dev, stream, reserved, p.t_arrive, time.perf_counter())


def latency_summary(results: dict) -> dict:
    lat = np.array([r.latency_s for r in results.values()])
    return {"jobs": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
