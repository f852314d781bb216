"""The tensor-core split product of the FP32 sweeps (needs a B200).

fcw_tc_product_check runs one tile through the sweeps' shared-memory layouts, UMMA
descriptors and tcgen05.mma kind::tf32: each FP32 operand is split into two TF32
terms (hi = rna(x), lo = rna(x - hi)) and hi*hi + hi*lo + lo*hi accumulate in FP32 in
tensor memory. Against an FP64 product, the error of each entry must be at FP32
level: at most k * 2^-24 * (|A| |B|)_ij for depth k, the classical bound of an FP32
dot product of length k (the dropped lo*lo term is below 2^-22 |a||b| per product).
One TF32 term alone must be clearly worse (it is the 2^-11 rounding of TF32), which
shows the split is doing the work.

The tile shapes are those of the sweeps: K-major A (forward: a 64-row chunk of a
panel Q_s times the right-hand-side rows) and the transposed, MN-major read of the
same panel (backward: Q_s^T times gathered solution rows), M = 64 and 128, N = 64
and 128. A "real panel" is Q = L21 inv(L11) of a dense Cholesky factor of the
grounded cotan Laplacian of a folded mesh, the matrix the mixed Poisson solve uses.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from fastcorticalwiring_b200 import _lib  # noqa: E402

U32 = 2.0 ** -24


def _tc(A, B, terms=3, trans=False):
    import torch

    lib = _lib.load()
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    k, n = B.shape
    m = A.shape[1] if trans else A.shape[0]
    a = torch.from_numpy(A).cuda()
    b = torch.from_numpy(B).cuda()
    c = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    raw = torch.zeros((128, n), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.fcw_tc_product_check(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                  ctypes.c_void_p(c.data_ptr()), m, k, n, terms, int(trans),
                                  ctypes.c_void_p(raw.data_ptr()), ctypes.c_void_p(st.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0 and int(st.item()) == 0
    return c.cpu().numpy(), raw.cpu().numpy()


def _real_panel(rows=64, cols=48, seed=0):
    """Q = L21 inv(L11) of a dense Cholesky factor of a grounded cotan Laplacian."""
    import scipy.linalg as la

    import oracle
    from fastcorticalwiring_b200 import mesh as M
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    m = folded_icosphere(3, seed=seed, jitter=0.2)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    L = oracle.operators(pm.V, pm.F)[0].toarray()
    g = L.shape[0] - 1
    L[g, :] = 0.0
    L[:, g] = 0.0
    L[g, g] = 1.0
    C = la.cholesky(L, lower=True)
    c0 = L.shape[0] // 3
    L11 = C[c0:c0 + cols, c0:c0 + cols]
    L21 = C[c0 + cols:c0 + cols + rows, c0:c0 + cols]
    return L21 @ np.linalg.inv(L11)


def _check(A64, B64, got, trans, terms):
    A32 = A64.astype(np.float32).astype(np.float64)
    B32 = B64.astype(np.float32).astype(np.float64)
    Aop = A32.T if trans else A32
    exact = Aop @ B32
    scale = np.abs(Aop) @ np.abs(B32)
    err = np.abs(got - exact) / np.maximum(scale, 1e-300)
    return float(np.max(err))


@pytest.mark.parametrize("m,k,n,trans", [(64, 48, 128, False), (128, 64, 128, False), (40, 24, 64, False),
                                         (64, 64, 128, True), (48, 32, 64, True)])
def test_split_product_is_fp32_accurate_on_random_tiles(m, k, n, trans):
    rng = np.random.default_rng(m * 1000 + k + n + trans)
    A = rng.standard_normal((k, m) if trans else (m, k))
    B = rng.standard_normal((k, n))
    got3, _ = _tc(A, B, 3, trans)
    got1, _ = _tc(A, B, 1, trans)
    e3 = _check(A, B, got3, trans, 3)
    e1 = _check(A, B, got1, trans, 1)
    # an FP32 FMA loop on the same operands, for scale
    Aop = (A.T if trans else A).astype(np.float32)
    ef = _check(A, B, (Aop @ B.astype(np.float32)).astype(np.float64), trans, 0)
    print(f"\nTC m={m} k={k} n={n} trans={trans}: 3xTF32 {e3:.2e}  1xTF32 {e1:.2e}  fp32 {ef:.2e} (x |A||B|)")
    assert e3 <= k * U32, e3
    assert e1 > 4 * k * U32  # one TF32 term is visibly coarser: the split carries the accuracy


@pytest.mark.parametrize("trans", [False, True])
def test_split_product_on_a_real_panel(trans):
    Q = _real_panel()                      # 64 x 48, rows of Q_s
    rng = np.random.default_rng(7)
    if trans:                              # backward: Q^T (48 x 64) times 64 gathered rows
        B = rng.standard_normal((Q.shape[0], 128))
        got, _ = _tc(Q, B, 3, True)
    else:                                  # forward: Q (64 x 48) times 48 right-hand-side rows
        B = rng.standard_normal((Q.shape[1], 128))
        got, _ = _tc(Q, B, 3, False)
    e = _check(Q, B, got, trans, 3)
    print(f"\nTC real panel trans={trans}: 3xTF32 {e:.2e} (x |Q||B|)")
    assert e <= Q.shape[0 if trans else 1] * U32, e


@pytest.mark.parametrize("level,jitter", [(4, 0.2), (5, 0.0)])
def test_tensor_core_sweeps_match_fma_sweeps(level, jitter):
    """The mixed Poisson solve with tensor-core sweeps against the same solve on FMA register
    tiles and against the FP64 engine, over several 64-column tiles and split-K supernodes.
    Two TF32 terms carry 22 of an FP32 value's 24 significant bits, so the factor and the
    right-hand sides the tensor cores see are perturbed about 4x more than in FP32: the
    solution error may be up to 8x the FMA tiles' (measured 3-5x)."""
    from fastcorticalwiring_b200 import engine, mesh as M
    from fastcorticalwiring_b200.meshgen import folded_icosphere

    m = folded_icosphere(level, seed=5, jitter=jitter)
    pm = M.prepare(m.vertices, m.faces, m.cortex_mask)
    src = pm.bfs[np.linspace(0, pm.n_vertices - 1, 256).astype(int)]
    out = {}
    for tc in (1, 0):
        eng = engine.HeatEngine(pm.V, pm.F, block_k=256, tc_sweeps=tc)
        try:
            out[tc] = eng.compute_distances(src, precision="mixed")
            if tc:
                out["fp64"] = eng.compute_distances(src, precision="fp64")
        finally:
            eng.close()
    scale = np.max(np.abs(out["fp64"]), axis=1)
    e_tc = np.max(np.abs(out[1] - out["fp64"]), axis=1) / scale
    e_fma = np.max(np.abs(out[0] - out["fp64"]), axis=1) / scale
    d = np.max(np.abs(out[1] - out[0]), axis=1) / scale
    print(f"\nTC sweeps L{level}: vs fp64 {e_tc.max():.2e} (FMA tiles {e_fma.max():.2e}), tc vs fma {d.max():.2e}")
    assert e_tc.max() <= max(8 * e_fma.max(), 1e-6)
    assert e_tc.max() <= 1e-4
