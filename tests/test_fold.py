"""The associative window-statistics fold the scan kernel uses
(gpu-ibs_b200/csrc/ibs_core.cuh, compiled for the host) equals the
reference's sequential loop for every split of a window into segments."""
import ctypes

import numpy as np
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

import oracle as orc


def fold(shim, valid, hit, cuts, k):
    valid = np.ascontiguousarray(valid, np.uint8)
    hit = np.ascontiguousarray(hit, np.uint8)
    cuts = np.ascontiguousarray(sorted(cuts), np.uint64)
    out = (ctypes.c_int32 * 4)()
    shim.fold_segments(valid.ctypes.data_as(ctypes.c_void_p), hit.ctypes.data_as(ctypes.c_void_p),
                       ctypes.c_uint64(len(valid)), cuts.ctypes.data_as(ctypes.c_void_p),
                       ctypes.c_uint64(len(cuts)), ctypes.c_int(k), out)
    return tuple(out)


def sequential(valid, hit, k):
    h = [int(x) for v, x in zip(valid, hit) if v]  # invalid positions are skipped
    r = orc.stats_from_hits(h, k)
    return (int(r["total_kmers"]), int(r["observed_kmers"]), int(r["variations"]),
            int(r["kmer_distance"]))


@settings(max_examples=400, deadline=None)
@given(st.data())
def test_fold_equals_sequential_loop(native_shim, data):
    n = data.draw(st.integers(0, 300))
    k = data.draw(st.sampled_from([4, 15, 25, 31, 32]))
    valid = data.draw(st.lists(st.booleans(), min_size=n, max_size=n))
    hit = [v and data.draw(st.booleans()) for v in valid]
    cuts = data.draw(st.lists(st.integers(0, n), max_size=12))
    assert fold(native_shim, valid, hit, cuts, k) == sequential(valid, hit, k)


@pytest.mark.parametrize("bits", [2, 8, 14, 20])
def test_table_hash_is_a_bijection(native_shim, bits):
    native_shim.hash_collisions.restype = ctypes.c_uint64
    assert native_shim.hash_collisions(ctypes.c_uint32(bits)) == 0


def span_fold(shim, valid, hit, k):
    valid = np.ascontiguousarray(valid, np.uint8)
    hit = np.ascontiguousarray(hit, np.uint8)
    out = (ctypes.c_int32 * 4)()
    shim.span_fold(valid.ctypes.data_as(ctypes.c_void_p), hit.ctypes.data_as(ctypes.c_void_p),
                   ctypes.c_uint64(len(valid)), ctypes.c_int(k), out)
    return tuple(out)


@settings(max_examples=400, deadline=None)
@given(st.data())
def test_span_fold_equals_sequential_loop(native_shim, data):
    # the scan kernels' span fold (32-position blocks kept one per lane,
    # summaries combined by the shuffle tree), its 32 lanes emulated; runs of
    # hits and misses of every length, invalid positions anywhere, spans of
    # several 32-block flushes
    n = data.draw(st.integers(0, 2600))
    k = data.draw(st.sampled_from([4, 15, 25, 31, 32]))
    p_hit = data.draw(st.sampled_from([0.0, 0.1, 0.5, 0.9, 0.99, 1.0]))
    p_valid = data.draw(st.sampled_from([1.0, 0.95, 0.5]))
    seed = data.draw(st.integers(0, 2**32 - 1))
    rng = np.random.default_rng(seed)
    valid = rng.random(n) < p_valid
    hit = valid & (rng.random(n) < p_hit)
    assert span_fold(native_shim, valid, hit, k) == sequential(valid, hit, k)
