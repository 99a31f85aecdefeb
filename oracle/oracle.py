"""ctypes binding of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

The oracle is a plain-C restatement of the reference GPU-IBS CPU scan path
(see ibs_oracle.h). Only the tests, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it, and only as the checker or the timed CPU baseline;
the product (gpu-ibs_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "liboracle.so"
REF_DIR = ORACLE_DIR / "_ref"

WINDOW_DTYPE = np.dtype([("start", "<i4"), ("end", "<i4"), ("total_kmers", "<i4"),
                         ("observed_kmers", "<i4"), ("variations", "<i4"),
                         ("kmer_distance", "<i4")])


def build():
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "liboracle.so"], check=True)


if not LIB_PATH.exists():
    build()
_o = C.CDLL(str(LIB_PATH))
vp = C.c_void_p


def _sig(name, res, args):
    f = getattr(_o, name)
    f.restype = res
    f.argtypes = args
    return f


_read = _sig("orc_read_sequence_file", vp, [C.c_char_p, C.c_int])
_count = _sig("orc_seqfile_count", C.c_size_t, [vp])
_id = _sig("orc_seqfile_id", C.c_char_p, [vp, C.c_size_t])
_seq = _sig("orc_seqfile_seq", vp, [vp, C.c_size_t, C.POINTER(C.c_size_t)])
_free = _sig("orc_seqfile_free", None, [vp])
_iopen = _sig("orc_index_open", vp, [C.c_char_p])
_iclose = _sig("orc_index_close", None, [vp])
_iparams = _sig("orc_index_params", None, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)])
_probe_many = _sig("orc_probe_many", None, [vp, vp, C.c_size_t, vp])
_list = _sig("orc_index_list", C.c_size_t, [vp, vp, C.c_size_t])
_canon = _sig("orc_canonical_codes", C.c_size_t, [C.c_char_p, C.c_size_t, C.c_uint32, vp])
_canon128 = _sig("orc_canonical_codes128", C.c_size_t, [C.c_char_p, C.c_size_t, C.c_uint32, vp, vp])
_probe128 = _sig("orc_probe128", C.c_int, [vp, C.c_uint64, C.c_uint64])
_list128 = _sig("orc_index_list128", C.c_size_t, [vp, vp, vp, C.c_size_t])
_wcount = _sig("orc_window_count", C.c_size_t, [C.c_size_t, C.c_uint32, C.c_uint32])
_scan_contigs = _sig("orc_scan_contigs", C.c_int,
                     [vp, C.POINTER(C.c_char_p), vp, C.c_size_t, C.c_uint32, C.c_uint32, C.c_int, vp])
_stats = _sig("orc_stats_from_hits", None, [vp, C.c_size_t, C.c_uint32, vp])
_err = _sig("orc_error", C.c_char_p, [])


class OracleError(RuntimeError):
    pass


def read_sequence_file(path: str, compressed: bool | None = None):
    """(ids, seqs) as the reference's readSequenceFile returns them."""
    if compressed is None:
        compressed = ".gz" in str(path)
    h = _read(str(path).encode(), int(compressed))
    if not h:
        raise OracleError(_err().decode())
    try:
        ids, seqs = [], []
        for i in range(_count(h)):
            ids.append(_id(h, i).decode(errors="surrogateescape"))
            n = C.c_size_t()
            p = _seq(h, i, C.byref(n))
            seqs.append(C.string_at(p, n.value))
        return ids, seqs
    finally:
        _free(h)


class Index:
    """The reference's KmcRaIndex restated: KMC 3 files -> probe."""

    def __init__(self, prefix: str):
        self._h = _iopen(str(prefix).encode())
        if not self._h:
            raise OracleError(_err().decode())
        p = (C.c_uint32 * 6)()
        t = C.c_uint64()
        _iparams(self._h, p, C.byref(t))
        self.k, self.p, self.sig_len, self.suffix_bytes, self.counter_bytes, self.n_bins = list(p)
        self.total = t.value

    @property
    def handle(self):
        return self._h

    def probe(self, codes) -> np.ndarray:
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        hits = np.zeros(len(codes), dtype=np.uint8)
        _probe_many(self._h, codes.ctypes.data, len(codes), hits.ctypes.data)
        return hits

    def list_codes(self) -> np.ndarray:
        out = np.zeros(max(self.total, 1), dtype=np.uint64)
        n = _list(self._h, out.ctypes.data, len(out))
        return out[:n]

    def probe128(self, lo, hi) -> np.ndarray:
        """k > 32: membership of codes given as low / high word arrays."""
        lo = np.ascontiguousarray(lo, dtype=np.uint64)
        hi = np.ascontiguousarray(hi, dtype=np.uint64)
        return np.array([_probe128(self._h, int(a), int(b)) for a, b in zip(lo, hi)], dtype=np.uint8)

    def list_codes128(self):
        """k > 32: every k-mer as (low words, high words)."""
        lo = np.zeros(max(self.total, 1), dtype=np.uint64)
        hi = np.zeros(max(self.total, 1), dtype=np.uint64)
        n = _list128(self._h, lo.ctypes.data, hi.ctypes.data, len(lo))
        return lo[:n], hi[:n]

    def close(self):
        if self._h:
            _iclose(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def canonical_codes(seq: bytes, k: int) -> np.ndarray:
    out = np.zeros(max(len(seq), 1), dtype=np.uint64)
    n = _canon(seq, len(seq), k, out.ctypes.data)
    return out[:n]


def canonical_codes128(seq: bytes, k: int):
    """k > 32: the string path's canonical k-mers as (low words, high words)."""
    lo = np.zeros(max(len(seq), 1), dtype=np.uint64)
    hi = np.zeros(max(len(seq), 1), dtype=np.uint64)
    n = _canon128(seq, len(seq), k, lo.ctypes.data, hi.ctypes.data)
    return lo[:n], hi[:n]


def window_count(length: int, W: int, k: int) -> int:
    return _wcount(length, W, k)


def scan(index: Index | None, seqs: list[bytes], W: int, k: int, threads: int = 1) -> np.ndarray:
    """Rows of every window of every sequence; index None = the synthetic
    predicate of the reference's phase-2 test."""
    lens = np.array([len(s) for s in seqs], dtype=np.uint64)
    n = sum(window_count(len(s), W, k) for s in seqs)
    rows = np.zeros(max(n, 1), dtype=WINDOW_DTYPE)
    arr = (C.c_char_p * max(1, len(seqs)))(*seqs)
    rc = _scan_contigs(index.handle if index else None, arr, lens.ctypes.data, len(seqs), W, k, threads,
                       rows.ctypes.data)
    if rc:
        raise OracleError(_err().decode())
    return rows[:n]


def stats_from_hits(hits, k: int) -> np.ndarray:
    hits = np.ascontiguousarray(hits, dtype=np.uint8)
    row = np.zeros(1, dtype=WINDOW_DTYPE)
    _stats(hits.ctypes.data, len(hits), k, row.ctypes.data)
    return row[0]


def tsv_text(ids: list[str], seqs_lens: list[int], rows: np.ndarray, W: int, k: int) -> str:
    """The TSV the reference writes for one reference file."""
    out = ["seqname\tstart\tend\ttotal_kmers\tobserved_kmers\tvariations\tkmer_distance\n"]
    r = 0
    for cid, ln in zip(ids, seqs_lens):
        for _ in range(window_count(ln, W, k)):
            x = rows[r]
            out.append(f"{cid}\t{x['start']}\t{x['end']}\t{x['total_kmers']}\t{x['observed_kmers']}\t"
                       f"{x['variations']}\t{x['kmer_distance']}\n")
            r += 1
    return "".join(out)


def position_codes(seq: bytes, k: int):
    """(canonical code, valid) of every k-mer start of seq, as the reference's
    KmerCodec::encodePositions gives them (src/KmerCodec.hpp:38-61): a start
    is valid when its k bases are ACGT/acgt."""
    s = np.frombuffer(seq, dtype=np.uint8)
    n = len(s) - k + 1
    if n <= 0:
        return np.zeros(0, np.uint64), np.zeros(0, bool)
    lut = np.full(256, 4, dtype=np.uint8)
    for i, c in enumerate(b"ACGT"):
        lut[c] = lut[c + 32] = i
    v = lut[s]
    cb = np.concatenate([[0], np.cumsum(v > 3)])
    valid = (cb[k:] - cb[:-k])[:n] == 0
    v = np.where(v > 3, 0, v).astype(np.uint64)
    fwd = np.zeros(n, np.uint64)
    rc = np.zeros(n, np.uint64)
    for t in range(k):
        fwd = (fwd << np.uint64(2)) | v[t:t + n]
        rc |= (np.uint64(3) - v[t:t + n]) << np.uint64(2 * t)
    return np.minimum(fwd, rc), valid


def position_codes128(seq: bytes, k: int):
    """k > 32: (low words, high words, valid) of every k-mer start of seq, the
    string path's canonical k-mers (src/Utils.hpp:102-125) by position."""
    s = np.frombuffer(seq, dtype=np.uint8)
    n = len(s) - k + 1
    if n <= 0:
        return np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0, bool)
    lut = np.full(256, 4, dtype=np.uint8)
    for i, c in enumerate(b"ACGT"):
        lut[c] = lut[c + 32] = i
    v = lut[s]
    cb = np.concatenate([[0], np.cumsum(v > 3)])
    valid = (cb[k:] - cb[:-k])[:n] == 0
    v = np.where(v > 3, 0, v).astype(np.uint64)
    flo, fhi, rlo, rhi = (np.zeros(n, np.uint64) for _ in range(4))
    for t in range(k):
        b = v[t:t + n]
        fb = 2 * (k - 1 - t)
        if fb >= 64:
            fhi |= b << np.uint64(fb - 64)
        else:
            flo |= b << np.uint64(fb)
        c = np.uint64(3) - b
        if 2 * t >= 64:
            rhi |= c << np.uint64(2 * t - 64)
        else:
            rlo |= c << np.uint64(2 * t)
    fwd = (fhi < rhi) | ((fhi == rhi) & (flo <= rlo))
    return np.where(fwd, flo, rlo), np.where(fwd, fhi, rhi), valid


def coverage(index: Index, seq: bytes, k: int) -> np.ndarray:
    """Per-base k-mer coverage of one contig: the reference's difference array
    (+1 at a hit start, -1 k bases on) and its prefix sum
    (KmerDatabase::getMappingFromSequence, src/KmerDatabase.hpp:774-801;
    for k > 32 its string path, getMappingFromSequenceLegacy, :803-848)."""
    if k > 32:
        lo, hi, valid = position_codes128(seq, k)
        codes = lo
        probe = lambda: index.probe128(lo, hi)  # noqa: E731
    else:
        codes, valid = position_codes(seq, k)
        probe = lambda: index.probe(codes)  # noqa: E731
    diff = np.zeros(len(seq) + 1, np.int64)
    if len(codes):
        hit = valid & (probe().astype(bool))
        idx = np.nonzero(hit)[0]
        np.add.at(diff, idx, 1)
        np.add.at(diff, idx + k, -1)
    return np.cumsum(diff)[: len(seq)]


def mapping_text(index: Index, ids: list[str], seqs: list[bytes], k: int) -> bytes:
    """The mapper's output file: per contig its id, then the coverage values
    joined by commas (serializeCoverage, src/KmerDatabase.hpp:754-772;
    the writer, :1195-1203)."""
    out = []
    for cid, s in zip(ids, seqs):
        cov = coverage(index, s, k)
        out.append(cid.encode(errors="surrogateescape") + b"\n" + ",".join(map(str, cov.tolist())).encode() + b"\n")
    return b"".join(out)


def reference_binary() -> Path | None:
    p = REF_DIR / "fastibs"
    return p if p.exists() else None
