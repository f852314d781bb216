"""The per-source kernel's sub-bin rules, checked on the reference's own distance fields.

k_source_metrics splits each distance bin (the reference's rule kb = int(hi / w),
lean_geometry.py:99-180) into 16 sub-bins by the same quotient q = hi / w, and an
evaluation at radius r visits only the sub-bins [j0, j1) of the two-bin band
(lean_geometry.py:183-244): the faces below j0 enter as whole areas and the faces
from j1 on are skipped. This restates those rules in numpy and checks, on the
golden fields, that the skipped terms are exactly what `_face_cdf` would return
(whole area below j0, zero from j1 on), so the area equals the reference's
prefix + band sum.
"""
import os

import numpy as np
import pytest

from fastcorticalwiring_b200 import mesh as M
from tests.conftest import GOLDEN

SB = 16  # sub-bins per bin (the kernel's kSubBins when the bins fit)


def _face_cdf(lo, mi, hi, A, r):
    """Area of {d <= r} per face (lean_geometry.py:66-88), vectorised."""
    ar = np.where(r >= hi, A, 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        lower = (r > lo) & (r < mi)
        upper = (r >= mi) & (r < hi) & (r > lo)
        x = r - lo
        ar = np.where(lower, A * x * x / ((mi - lo) * (hi - lo)), ar)
        y = hi - r
        ar = np.where(upper, A * (1.0 - y * y / ((hi - lo) * (hi - mi))), ar)
    return ar


def _f32_down(x):
    """x rounded down to float32 (the kernel's __double2float_rd), as float64."""
    f = x.astype(np.float32)
    f = np.where(f.astype(np.float64) > x, np.nextafter(f, np.float32(-np.inf)), f)
    return f.astype(np.float64)


@pytest.fixture(scope="module")
def l4():
    z = dict(np.load(os.path.join(GOLDEN, "golden_heat_L4.npz")))
    z["pm"] = M.prepare(z["V"], z["F"], z["mask"])
    return z


@pytest.mark.parametrize("as_f32", [False, True])
def test_subbins_skip_only_exact_terms(l4, as_f32):
    pm = l4["pm"]
    w = float(pm.bin_width)
    A = pm.lean_area
    checked = 0
    for j in range(l4["phi"].shape[0]):
        d = l4["phi"][j]
        if as_f32:  # the mixed form's fields are float32
            d = d.astype(np.float32).astype(np.float64)
        c = np.sort(d[pm.F], axis=1)
        lo, mi, hi = c[:, 0], c[:, 1], c[:, 2]
        q = hi / w
        kb = np.where(q < 1.0, 0, q.astype(np.int64))
        sub = np.clip(np.floor((q - kb) * SB).astype(np.int64), 0, SB - 1)
        jb = kb * SB + sub
        nsub = int(jb.max()) + 1
        minlo = np.full(nsub + 1, np.inf)
        np.minimum.at(minlo, jb, _f32_down(lo))
        suffix = np.minimum.accumulate(minlo[::-1])[::-1]
        radii = np.concatenate([l4["radii"][j], l4["extra_r"][j]])
        for r in radii[np.isfinite(radii) & (radii > 0)]:
            kr = int(r / w)
            kend = kr + 2
            qr = r / w
            j0 = kr * SB + min(max(int(np.floor((qr - kr) * SB)), 0), SB - 1)
            j1 = j0 + 1
            while j1 < kend * SB and not (suffix[j1] >= r):
                j1 += 1
            below = jb < j0
            skipped = (jb >= j1) & (kb < kend)
            assert np.all(hi[below] < r)          # whole areas
            assert np.all(lo[skipped] >= r)       # zero terms
            band = (kb >= kr) & (kb < kend)
            ref = A[kb < kr].sum() + _face_cdf(lo[band], mi[band], hi[band], A[band], r).sum()
            vis = (jb >= j0) & (jb < j1)
            new = A[below].sum() + _face_cdf(lo[vis], mi[vis], hi[vis], A[vis], r).sum()
            assert abs(new - ref) <= 1e-13 * ref
            checked += 1
    assert checked > 100
