"""ShardedWiringAnalysis over NCCL (needs a B200): a one-rank process group on this GPU runs the
same gather path as several GPUs do (CUDA tensors, all_gather over NCCL), and its arrays must
equal WiringAnalysis's on the same mesh (the band sums' atomics set the last bits of the
geometry, so to 1e-12; flags, counts and sample CSR exactly up to those bits)."""
import datetime
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCALES = [0.001, 0.004, 0.016]


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_rank_nccl_matches_wiring_analysis():
    import torch
    import torch.distributed as dist

    from fastcorticalwiring_b200.analysis import WiringAnalysis
    from fastcorticalwiring_b200.meshgen import folded_icosphere
    from fastcorticalwiring_b200.sharded import ShardedWiringAnalysis

    m = folded_icosphere(4, seed=11, jitter=0.1)
    args = (m.vertices, m.faces, m.cortex_mask)
    ref = WiringAnalysis(*args, allow_interior_nonmanifold=True)
    ref.compute_all_wiring_costs(scale=SCALES, n_samples_between_scales=2)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sh = ShardedWiringAnalysis(*args, allow_interior_nonmanifold=True, engine_kwargs={"device": 0})
        sh.compute_all_wiring_costs(scale=SCALES, n_samples_between_scales=2)
    finally:
        dist.destroy_process_group()
    assert np.array_equal(sh.field_flag, ref.field_flag)
    ok = ref.field_flag == 0
    for a, b in ((sh.msd_unweighted, ref.msd_unweighted), (sh.msd_weighted, ref.msd_weighted),
                 (sh.dist_to_boundary, ref.dist_to_boundary)):
        assert np.allclose(a[ok], b[ok], rtol=1e-6, atol=0, equal_nan=True)
    for s in SCALES:
        assert np.allclose(sh.radius_function[s], ref.radius_function[s], rtol=1e-6, equal_nan=True)
    assert np.array_equal(sh.sample_indptr, ref.sample_indptr)
    assert np.allclose(sh.sample_radii_flat, ref.sample_radii_flat, rtol=1e-6)
