"""The serving loop's admission policy on the host (no device): arrival order under an HBM
budget, a bounded number of later jobs passing a head job that waits for memory, and the
memory estimate growing with the job."""
import threading
from collections import deque

import numpy as np

from fastcorticalwiring_b200 import serving as S


def _server(budget, max_bypass=2):
    srv = object.__new__(S.Server)  # the policy only; no builder threads, no device
    srv.budget = int(budget)
    srv.max_bypass = max_bypass
    srv.params = dict(block_k=1024, pipeline_depth=2)
    srv._cv = threading.Condition()
    srv._pending = deque()
    srv._reserved = 0
    srv._bypassed = 0
    srv.results = {}
    srv._n_open = 0
    return srv


def _pending(name, estimate):
    job = S.Job(name, np.zeros((3, 3)), np.zeros((1, 3), np.int32), np.ones(3, bool))
    return S._Pending(job, 0.0, estimate)


def test_head_first_then_bounded_bypass():
    srv = _server(budget=100)
    srv._pending.extend([_pending("big", 90), _pending("a", 20), _pending("b", 20), _pending("c", 20)])
    assert srv._pick().job.job_id == "big"      # nothing resident: the head goes first
    srv._reserved = 90
    srv._pending.appendleft(_pending("big2", 50))
    assert srv._pick() is None                   # neither the head nor a 20 fits beside 90
    srv._reserved = 60
    assert srv._pick().job.job_id == "a"         # the head (50) waits; a later job that fits passes
    srv._reserved += 20
    assert srv._pick().job.job_id == "b"         # 80 + 20 fits: a second pass (max_bypass = 2)
    srv._reserved = 60
    assert srv._pick() is None                   # the head has been passed twice: "c" waits behind it
    srv._reserved = 40
    assert srv._pick().job.job_id == "big2"      # the head fits now, and the bypass count resets
    assert srv._bypassed == 0
    assert srv._pick().job.job_id == "c"


def test_memory_estimate_grows_with_the_job():
    e = S.estimate_device_bytes
    base = e(40_000, 80_000, 1024, 2, 40_000, S._stride(12, 3))
    assert e(160_000, 320_000, 1024, 2, 160_000, S._stride(12, 3)) > 3 * base
    assert e(40_000, 80_000, 1024, 4, 40_000, S._stride(12, 3)) > base
    assert e(40_000, 80_000, 512, 2, 40_000, S._stride(12, 3)) < base


def test_job_larger_than_the_budget_is_refused_not_run():
    """A job that can never fit the HBM budget gets a result with the reason (no records), and the
    jobs behind it are admitted as usual."""
    srv = _server(budget=100)
    srv._pending.extend([_pending("huge", 150), _pending("a", 20)])
    srv._n_open = 2
    with srv._cv:  # the builders call _pick holding the lock
        assert srv._pick().job.job_id == "a"
    r = srv.results["huge"]
    assert r.error is not None and "budget" in r.error and r.records.size == 0
    assert srv._n_open == 1
