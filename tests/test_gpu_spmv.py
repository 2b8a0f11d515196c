"""The stand-alone BSR SpMV (drape_spmv_benchmark) on a block-diagonal batch of drapes against numpy (needs a
B200): every kernel shape, f32 blocks and x on both sides (relative L2 1e-6)."""
import numpy as np
import pytest

from drape_b200 import api
from drape_b200.scenes import sheet_matrix

pytestmark = pytest.mark.gpu


def test_batched_spmv_matches_numpy_for_every_shape():
    parts, offset = [], 0
    for n, seed in ((17, 1), (33, 2), (17, 3)):
        rp, ci, blk = sheet_matrix(n, seed, 0.25, 5e5)
        parts.append((rp, ci + offset, blk))
        offset += len(rp) - 1
    rp = np.concatenate([[0]] + [p[0][1:] + sum(q[0][-1] for q in parts[:i]) for i, p in enumerate(parts)])
    ci = np.concatenate([p[1] for p in parts])
    blk = np.concatenate([p[2] for p in parts])
    R = len(rp) - 1
    x = np.random.default_rng(0).standard_normal(3 * R).astype(np.float32)
    rows = np.repeat(np.arange(R), np.diff(rp))
    ref = np.zeros((R, 3))
    np.add.at(ref, rows, np.einsum("kab,kb->ka", blk.reshape(-1, 3, 3).astype(np.float64),
                                   x.reshape(-1, 3).astype(np.float64)[ci]))
    for lanes in (4, 8, 16, 32):
        for threads in (128, 256):
            ms, y = api.spmv_benchmark(rp, ci, blk, x, 3, lanes, threads, result=True)
            assert ms > 0
            assert np.linalg.norm(y - ref.reshape(-1)) <= 1e-6 * np.linalg.norm(ref), (lanes, threads)


def test_spmv_benchmark_rejects_bad_columns():
    with pytest.raises(api.DrapeError):
        api.spmv_benchmark(np.array([0, 1]), np.array([5]), np.ones(9, np.float32), np.ones(3, np.float32))
