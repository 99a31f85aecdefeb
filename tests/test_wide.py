"""k > 32 on the CPU: the reference's string path (every k > 32 database,
src/KmerDatabase.hpp:100-124, :675-708) restated by the oracle, and the
128-bit code reader of the wide scan kernel (gpu-ibs_b200/csrc/wide_core.cuh
compiled for the host) against it. The oracle itself is pinned to the
reference's binary by the edge_k33 / edge_k41 / edge_k64 golden TSVs
(tests/test_oracle.py)."""
import ctypes

import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

WIDE_CASES = ["edge_k33", "edge_k41", "edge_k64"]


def _ascii(rng, n):
    """ACGT and acgt, with an invalid byte (N, R or n) at about 1 in 300
    positions, so that k-mers of 64 bases are still mostly valid."""
    a = np.frombuffer(b"ACGTacgt", np.uint8)[rng.integers(0, 8, n)].copy()
    bad = rng.random(n) < 1 / 300
    a[bad] = np.frombuffer(b"NRn", np.uint8)[rng.integers(0, 3, int(bad.sum()))]
    return bytes(a)


@pytest.mark.parametrize("k", [33, 41, 56, 63, 64])
def test_codec128_matches_numpy_restatement(k):
    rng = np.random.default_rng(k)
    s = _ascii(rng, 6000)
    lo, hi = orc.canonical_codes128(s, k)
    nlo, nhi = corpus.canonical_codes128_np(s, k)
    assert len(lo) > 0
    assert np.array_equal(lo, nlo) and np.array_equal(hi, nhi)


def test_codec128_is_the_string_rule():
    # the smaller of the k-mer and its reverse complement as strings
    # (getCanonicalKmersLegacy, src/Utils.hpp:102-125)
    rng = np.random.default_rng(9)
    k = 45
    s = _ascii(rng, 400)
    lo, hi = orc.canonical_codes128(s, k)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    want = []
    up = s.upper()
    for i in range(len(up) - k + 1):
        kmer = up[i:i + k]
        if kmer.strip(b"ACGT"):
            continue
        rc = kmer.translate(comp)[::-1]
        want.append(min(kmer, rc))
    got = []
    for a, b in zip(lo.tolist(), hi.tolist()):
        v = (b << 64) | a
        got.append(bytes(b"ACGT"[(v >> (2 * (k - 1 - j))) & 3] for j in range(k)))
    assert got == want


@pytest.mark.parametrize("k", [33, 40, 47, 64])
def test_kernel_code_reader_matches_oracle(native_shim, k):
    """The wide scan kernel's reader (three packed words, funnel shifts, a
    2-bit symbol reversal for the forward strand, the complement for the
    reverse one) at every start of every contig, against the oracle's
    string-path codes."""
    rng = np.random.default_rng(100 + k)
    seqs = [_ascii(rng, n) for n in (3000, k, k - 1, 777, 64 * 5 + 3)]
    packed, nmask, lens = ib.pack_ascii(seqs)
    f = native_shim.wide_codes_packed
    f.restype = None
    f.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32] + [ctypes.c_void_p] * 3
    base = 0
    for s in seqs:
        n = max(0, len(s) - k + 1)
        lo = np.zeros(max(n, 1), np.uint64)
        hi = np.zeros(max(n, 1), np.uint64)
        ok = np.zeros(max(n, 1), np.uint8)
        if n:
            f(packed.ctypes.data, nmask.ctypes.data, base, n, k, lo.ctypes.data, hi.ctypes.data, ok.ctypes.data)
        sel = ok[:n].astype(bool)
        wlo, whi = orc.canonical_codes128(s, k)
        assert np.array_equal(lo[:n][sel], wlo) and np.array_equal(hi[:n][sel], whi)
        base += (len(s) + 63) // 64 * 64


@pytest.mark.parametrize("name", WIDE_CASES)
def test_index_lists_exactly_the_written_keys128(name, build_case):
    case = build_case(name)
    ix = orc.Index(str(case["prefix"]))
    assert ix.k == case["k"]
    lo, hi = ix.list_codes128()
    assert len(lo) == ix.total
    assert len({(a, b) for a, b in zip(lo.tolist(), hi.tolist())}) == ix.total
    assert ix.probe128(lo[:2000], hi[:2000]).all()
    # a code one past each listed code (mostly absent) stays consistent with
    # the listing
    keys = {(a, b) for a, b in zip(lo.tolist(), hi.tolist())}
    q_lo = lo[:500] ^ np.uint64(1)
    got = ix.probe128(q_lo, hi[:500])
    want = [1 if (a, b) in keys else 0 for a, b in zip(q_lo.tolist(), hi[:500].tolist())]
    assert got.tolist() == want


def test_wide_table_lines_spread(native_shim):
    """The level hash of the wide table spreads keys over the lines about
    evenly (a Poisson load of 4 keys per line rarely passes 8)."""
    f = native_shim.wide_line_of
    f.restype = ctypes.c_uint64
    f.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64]
    rng = np.random.default_rng(3)
    lo, hi = corpus.random_codes128(rng, 40000, 41)
    lines = 10000
    counts = np.bincount([f(int(a), int(b), 0, lines) for a, b in zip(lo, hi)], minlength=lines)
    # Poisson(4): P(X > 8) = 2.1%, and a line above 20 keys is a 1e-10 event
    assert counts.max() <= 20
    assert (counts > 8).mean() < 0.04
    # another level hashes the same keys elsewhere
    other = [f(int(a), int(b), 1, lines) for a, b in zip(lo[:1000], hi[:1000])]
    same = [f(int(a), int(b), 0, lines) for a, b in zip(lo[:1000], hi[:1000])]
    assert np.mean(np.array(other) == np.array(same)) < 0.01


def test_wide_entry_points_are_exported():
    for name in ("ibs_table_from_codes128", "ibs_probe128"):
        assert hasattr(ib._lib, name)
    assert hasattr(ib._tools, "ibs_kmc_write128")
