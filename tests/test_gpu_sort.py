"""The plan builder's own device sort and scan against numpy.

The radix sort must be stable (equal keys keep their input order: the plan's
sample order inside a run of equal keys is the accessor's row order, which
fixes the order of floating-point additions) and must order by bits
[0, end_bit) only; both are checked bit-exactly against numpy's stable sort,
on sizes that end inside a tile, keys with many duplicates, and keys with
bits set above end_bit.  The scan is checked for sum, min and max, inclusive
and exclusive, in place and on unaligned lengths."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,end_bit,spread", [
    (1, 64, 10), (2, 8, 3), (4095, 36, 1 << 36), (4097, 12, 7), (100_003, 40, 1 << 20),
    (1_000_000, 64, 1 << 64), (3_000_001, 33, 1 << 33), (257, 0, 5)])
def test_sort_pairs_stable_against_numpy(ygmod, n, end_bit, spread):
    from yandasoft_b200.gridder import sort_pairs
    rng = np.random.default_rng(n + end_bit)
    if spread >= 1 << 63:
        keys = rng.integers(0, 1 << 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    else:
        keys = rng.integers(0, spread, n, dtype=np.uint64)
    vals = np.arange(n, dtype=np.uint32)
    k, v = sort_pairs(keys, vals, end_bit)
    mask = np.uint64((1 << end_bit) - 1) if end_bit < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    order = np.argsort(keys & mask, kind="stable")
    assert np.array_equal(v, vals[order])
    assert np.array_equal(k, keys[order])


def test_sort_pairs_sorted_runs_of_plan_keys(ygmod):
    """Plan-like keys: long runs of equal high bits (tile, CF), short low bits."""
    from yandasoft_b200.gridder import sort_pairs
    rng = np.random.default_rng(3)
    n = 2_000_000
    tile = rng.integers(0, 300, n, dtype=np.uint64)
    cf = rng.integers(0, 64, n, dtype=np.uint64)
    pos = rng.integers(0, 1024, n, dtype=np.uint64)
    keys = (tile << np.uint64(16)) | (cf << np.uint64(10)) | pos
    keys[rng.random(n) < 0.01] = np.uint64((300 << 16) + 1)   # the invalid key: after every valid one
    vals = rng.permutation(n).astype(np.uint32)
    k, v = sort_pairs(keys, vals, 25)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(v, vals[order]) and np.array_equal(k, keys[order])


@pytest.mark.parametrize("n", [1, 5, 2047, 2048, 2049, 1_000_003])
@pytest.mark.parametrize("op", ["sum", "min", "max"])
@pytest.mark.parametrize("exclusive", [False, True])
def test_scan_i32_against_numpy(ygmod, n, op, exclusive):
    from yandasoft_b200.gridder import scan_i32
    rng = np.random.default_rng(n)
    x = rng.integers(-1000, 1000, n, dtype=np.int32) if op != "sum" else rng.integers(0, 100, n, dtype=np.int32)
    y = scan_i32(x, op, exclusive)
    f = {"sum": np.cumsum, "min": np.minimum.accumulate, "max": np.maximum.accumulate}[op]
    ident = {"sum": 0, "min": np.iinfo(np.int32).max, "max": np.iinfo(np.int32).min}[op]
    inc = f(x.astype(np.int64)).astype(np.int32)
    ref = np.concatenate([[ident], inc[:-1]]).astype(np.int32) if exclusive else inc
    assert np.array_equal(y, ref)
