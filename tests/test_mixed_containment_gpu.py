"""What the mixed-precision leaf stage rests on, checked on float data: each
point's exact FP32 best k over its leaf blocks must lie inside the best kq
candidates that the tensor-core tiles select by their rounded keys, so that
the FP32 re-rank can recover it.

With no propagation, the plain FP32 build returns exactly that exact best k
(every key of the union of the point's blocks, ranked by (key, id)), and the
mixed build returns the exact best k of its kq candidates.  The two rows are
equal exactly when the containment holds, so the share of equal rows is the
containment rate.  Where a row differs, the mixed row can only be worse
entry by entry, never better.

Cases: Gaussian mixtures (EUCLIDEAN, float32), unit-norm rows stored as FP16
(COSINE, the shape of the normalised-mixture workload), d from 128 to 256,
k = 10, 16 and 24 (kq = 32 < 2k for k = 24).  Every case must reach a
containment rate of at least 0.98; the rates are printed."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

CASES = [  # (name, n, d, k, metric, fp16 input, precision names)
    ("mixture_d200_k10", 30000, 200, 10, 0, False),
    ("mixture_d256_k16", 30000, 256, 16, 0, False),
    ("mixture_d128_k24", 30000, 128, 24, 0, False),
    ("unit_fp16_d96_k10", 40000, 96, 10, 2, True),
    ("unit_fp16_d256_k16", 30000, 256, 16, 2, True),
]


def _points(acknn, n, d, metric, fp16, seed):
    if metric == 2:
        return acknn.workloads.normalized_mixture(seed=seed, n=n, d=d, clusters=200,
                                                  dtype=np.float16 if fp16 else np.float32)
    return acknn.workloads.gaussian_mixture(n, d, 24, seed=seed)


def _precisions(acknn):
    out = {"bf16": acknn.PREC_BF16_RERANK}
    if hasattr(acknn, "PREC_F16_RERANK"):
        out["f16"] = acknn.PREC_F16_RERANK
    return out


@pytest.mark.parametrize("name,n,d,k,metric,fp16", CASES, ids=[c[0] for c in CASES])
def test_exact_best_k_inside_tensor_core_candidates(name, n, d, k, metric, fp16, capsys):
    acknn = load_package()
    x = _points(acknn, n, d, metric, fp16, seed=d + k)
    trees, leaf = 4, 256
    pi, pd = acknn.knn_build(x, k, trees, leaf, 0, metric, seed=2)
    for pname, prec in _precisions(acknn).items():
        mi, md = acknn.knn_build(x, k, trees, leaf, 0, metric, seed=2, precision=prec)
        same = np.all(mi == pi, axis=1) & np.all(md.view(np.uint32) == pd.view(np.uint32), axis=1)
        rate = float(same.mean())
        # the mixed rows are drawn from the same candidate union: never better
        assert np.all(md >= pd), f"{pname}: a mixed entry beats the exact best k"
        with capsys.disabled():
            print(f"\n[containment] {name} {pname}: {rate:.5f} of {n} rows equal the exact best {k}")
        assert rate >= 0.98, (pname, rate)
