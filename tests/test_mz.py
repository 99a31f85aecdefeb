"""The minimizer-bucketed table's key map (gpu-ibs_b200/csrc/mz_core.cuh,
compiled for the host): the scan kernel's query-side computation equals the
build-side one on every position of either strand, and (bucket, slot)
identifies a k-mer exactly."""
import ctypes

import numpy as np
import pytest

import corpus

vp = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(vp)


def locate(shim, codes, k, nb):
    codes = np.ascontiguousarray(codes, np.uint64)
    b = np.zeros(len(codes), np.uint64)
    s = np.zeros(len(codes), np.uint64)
    shim.mz_locate(_ptr(codes), ctypes.c_uint64(len(codes)), ctypes.c_uint32(k), ctypes.c_uint64(nb),
                   _ptr(b), _ptr(s))
    return b, s


def query(shim, bases, k, nb):
    bases = np.ascontiguousarray(bases, np.uint8)
    n = max(len(bases) - k + 1, 0)
    b = np.zeros(n, np.uint64)
    s = np.zeros(n, np.uint64)
    shim.mz_query(_ptr(bases), ctypes.c_uint64(len(bases)), ctypes.c_uint32(k), ctypes.c_uint64(nb),
                  _ptr(b), _ptr(s))
    return b, s


def min_lines_log2(k):
    """log2 of the fewest lines whose slots fit the sector: 31-bit slots of
    B8x32 sectors (format MZ8) up to k = 27, 40-bit slots of B6x40 sectors
    (format MZ6) above."""
    return 2 * k - 27 if k <= 27 else 2 * k - 36


def slot_bits(k):
    return 31 if k <= 27 else 40


@pytest.mark.parametrize("k", [16, 21, 25, 27, 28, 31])
def test_query_side_equals_build_side(native_shim, k):
    rng = np.random.default_rng(k)
    nb = 4 << max(min_lines_log2(k), 20)  # four sectors per line
    # random sequence plus repeats that force minimizer ties
    seq = rng.integers(0, 4, 200_000).astype(np.uint8)
    unit = rng.integers(0, 4, 17).astype(np.uint8)
    seq[5000:5000 + 17 * 40] = np.tile(unit, 40)
    seq[9000:9200] = 0
    rc = (3 - seq[::-1]).copy()
    for s_ in (seq, rc):
        qb, qs = query(native_shim, s_, k, nb)
        text = bytes(np.frombuffer(b"ACGT", np.uint8)[s_])
        codes = corpus.canonical_codes_np(text, k)
        lb, ls = locate(native_shim, codes, k, nb)
        assert np.array_equal(qb, lb) and np.array_equal(qs, ls)


@pytest.mark.parametrize("k", [20, 25, 27, 28, 31])
def test_bucket_and_slot_identify_the_kmer(native_shim, k):
    rng = np.random.default_rng(100 + k)
    nb = 4 << max(min_lines_log2(k), 18)
    codes = np.unique(corpus.random_codes(rng, 400_000, k))
    b, s = locate(native_shim, codes, k, nb)
    assert (b < nb).all()
    assert (s < (1 << slot_bits(k))).all(), "slot values must stay below the sector's sentinels"
    pairs = np.unique(np.stack([b, s], axis=1), axis=0)
    assert len(pairs) == len(codes)


def test_buckets_are_uniform_over_minimizers(native_shim):
    # k-mers of one sequence cluster by minimizer; the clusters must spread
    # evenly over the buckets (a minimizer's hash is biased towards 0)
    k, nb = 25, 1 << 18
    rng = np.random.default_rng(7)
    seq = rng.integers(0, 4, 1_000_000).astype(np.uint8)
    qb, _ = query(native_shim, seq, k, nb)
    lines = qb >> np.uint64(2)  # four 32-byte sectors per line
    keys = np.unique(lines)  # lines touched, one per distinct minimizer (mostly)
    frac_low = (keys < nb // 8).mean()
    assert 0.47 < frac_low < 0.53
    counts = np.bincount(lines.astype(np.int64), minlength=nb // 4)
    # load of the first and last eighths of the lines agree within 5%
    a, b = counts[: nb // 32].sum(), counts[-nb // 32:].sum()
    assert abs(a - b) / max(a, b) < 0.05
    # the sector inside a line comes from the k-mer: a run of positions sharing
    # a minimizer spreads over the line's four sectors
    sectors = np.bincount((qb & np.uint64(3)).astype(np.int64), minlength=4) / len(qb)
    assert (abs(sectors - 0.25) < 0.01).all()
