"""The ordering network of the migration's large destination buckets
(k_mig_order_large in rhybrid_b200/csrc/k_fast.cuh), stepped here exactly as
the kernel's loops step it: a bitonic sort of (key, mover index) over the
bucket padded to a power of two with (all-ones, all-ones). It must give the
order the radix sorts give: by key, equal keys by mover index."""
import numpy as np
import pytest

MIG_SMALL, MIG_LARGE, THREADS = 64, 2048, 256


def order_large(keys: np.ndarray, vals: np.ndarray) -> np.ndarray:
    k = len(keys)
    m = 1
    while m < k:
        m <<= 1
    skey = np.full(m, np.iinfo(np.uint64).max, dtype=np.uint64)
    sval = np.full(m, np.iinfo(np.uint32).max, dtype=np.uint32)
    skey[:k], sval[:k] = keys, vals
    size = 2
    while size <= m:
        stride = size >> 1
        while stride > 0:
            # every thread of the block takes i = tid, tid + THREADS, ... ; one stage per barrier
            for i in range(m):
                j = i ^ stride
                if j > i:
                    up = (i & size) == 0
                    gt = skey[i] > skey[j] or (skey[i] == skey[j] and sval[i] > sval[j])
                    if gt == up:
                        skey[i], skey[j] = skey[j], skey[i]
                        sval[i], sval[j] = sval[j], sval[i]
            stride >>= 1
        size <<= 1
    return sval[:k]


@pytest.mark.parametrize("k", [MIG_SMALL + 1, 100, 255, 256, 257, 1000, MIG_LARGE])
def test_large_bucket_order_equals_radix_order(k):
    rng = np.random.default_rng(k)
    # keys as the push writes them: source segment << 32 | index, a few repeated
    keys = (rng.integers(0, 5000, k).astype(np.uint64) << np.uint64(32)) | rng.integers(0, 300, k).astype(np.uint64)
    keys[rng.integers(0, k, k // 10)] = keys[0]
    vals = rng.permutation(10 * k)[:k].astype(np.uint32)
    want = vals[np.lexsort((vals, keys))]
    assert np.array_equal(order_large(keys, vals), want)
