"""The block-size autotuner (needs a B200): it times every fitting candidate and keeps the fastest."""
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import autotune, mesh as M  # noqa: E402
from fastcorticalwiring_b200.meshgen import folded_icosphere  # noqa: E402


def test_autotune_picks_the_fastest_candidate():
    m = folded_icosphere(4, seed=5, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    best, trials = autotune.autotune(pm, ks=(64, 128), depths=(1, 2), min_sources=512)
    assert len(trials) == 4
    assert all(t["sources_per_s"] > 0 for t in trials)
    assert best["sources_per_s"] >= max(t["sources_per_s"] for t in trials) - 10.0
    assert (best["block_k"], best["pipeline_depth"]) in {(t["block_k"], t["pipeline_depth"]) for t in trials}
