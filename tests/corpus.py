"""Seeded test corpora (test infrastructure).

Two kinds of inputs:

* workloads from gpu-ibs_b200's configs (counter-based generators in
  libibs_tools), written as FASTA + KMC 3 database;
* an edge-case corpus shaped like the reference's scripts/make_test_corpus.sh:
  a main contig whose sample copy has ~1% SNPs and dropout blocks, a
  lowercase contig, a contig with N runs of 1, k-1, k and 3k, a contig
  shorter than k, one of exactly k, and a lowercase+N contig. The sample
  database holds the canonical k-mers of the copy plus random k-mers.

Every case is a pure function of its parameters; tests regenerate the inputs
and check their sha256 against the committed golden records before
comparing results.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "gpu-ibs_b200" / "python"))
sys.path.insert(0, str(REPO / "oracle"))

import ibs_b200 as ib  # noqa: E402
from ibs_b200 import configs  # noqa: E402

GOLDEN = REPO / "tests" / "golden"
BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
LOWER = np.frombuffer(b"acgt", dtype=np.uint8)


def sha256_file(path) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


# ---------------------------------------------------------------------------
# edge-case corpus
# ---------------------------------------------------------------------------
def _random_bases(rng, n, lower=False) -> np.ndarray:
    return (LOWER if lower else BASES)[rng.integers(0, 4, n)]


def _put_n(a: np.ndarray, k: int):
    """N runs of 1, k-1, k and 3k at fixed offsets (make_test_corpus.sh:60-66)."""
    for at, ln in ((1000, 1), (5000, k - 1), (9000, k), (13000, 3 * k)):
        if at + ln <= len(a):
            a[at:at + ln] = ord("N")


def edge_contigs(k: int, seed: int, main_len: int = 200_000):
    """[(name, reference bytes, sample-copy bytes)]: the copy has ~1% SNPs
    and dropout blocks (make_test_corpus.sh:68-101)."""
    rng = np.random.default_rng(seed)
    out = []

    def add(name, n, lower=False, with_n=False, drops=()):
        ref = _random_bases(rng, n, lower)
        up = np.frombuffer(bytes(ref).upper(), dtype=np.uint8).copy()
        snp = rng.random(n) < 0.01
        copy = up.copy()
        copy[snp] = BASES[rng.integers(0, 4, int(snp.sum()))]
        keep = np.ones(n, dtype=bool)
        for a, b in drops:
            keep[a:min(b, n)] = False
        if with_n:
            _put_n(ref, k)
        out.append((name, bytes(ref), bytes(copy[keep])))

    add("chr1", main_len, drops=((60_000, 65_000), (120_000, 122_000), (180_000, 180_100)))
    add("chr2_lowercase", 30_000, lower=True)
    add("chr3_withN", 20_000, with_n=True)
    add("chr4_short", k - 3)
    add("chr5_exactk", k)
    add("chr6_mixed", 20_000, lower=True, with_n=True)
    return out


def fasta_bytes(records, width=80, crlf=False) -> bytes:
    nl = b"\r\n" if crlf else b"\n"
    parts = []
    for name, seq in records:
        parts.append(b">" + name.encode() + nl)
        for i in range(0, len(seq), width):
            parts.append(seq[i:i + width] + nl)
    return b"".join(parts)


def fastq_bytes(records) -> bytes:
    parts = []
    for name, seq in records:
        parts += [b"@" + name.encode() + b"\n", seq + b"\n", b"+\n", b"I" * len(seq) + b"\n"]
    return b"".join(parts)


def canonical_codes_np(seq: bytes, k: int) -> np.ndarray:
    """Canonical codes of the ACGT-only k-mers of seq (numpy; case-folded)."""
    s = np.frombuffer(seq.upper(), dtype=np.uint8)
    lut = np.full(256, 4, dtype=np.uint8)
    for i, c in enumerate(b"ACGT"):
        lut[c] = i
    v = lut[s]
    n = len(v) - k + 1
    if n <= 0:
        return np.zeros(0, dtype=np.uint64)
    bad = (v > 3).astype(np.int64)
    cb = np.concatenate([[0], np.cumsum(bad)])
    ok = (cb[k:] - cb[:-k]) == 0
    v = np.where(v > 3, 0, v).astype(np.uint64)
    fwd = np.zeros(n, dtype=np.uint64)
    rc = np.zeros(n, dtype=np.uint64)
    for t in range(k):
        fwd = (fwd << np.uint64(2)) | v[t:t + n]
        rc = rc | ((np.uint64(3) - v[t:t + n]) << np.uint64(2 * t))
    can = np.minimum(fwd, rc)
    return can[ok[:n]]


def _split_codes(v: np.ndarray, k: int):
    """Forward and reverse-complement codes of every k-mer start of the base
    values v (0..3) as (fwd_lo, fwd_hi, rc_lo, rc_hi), k > 32: base t of a
    k-mer sits at bit 2 (k - 1 - t) of the forward code and, complemented,
    at bit 2 t of the reverse complement."""
    n = len(v) - k + 1
    z = lambda: np.zeros(max(n, 0), dtype=np.uint64)  # noqa: E731
    flo, fhi, rlo, rhi = z(), z(), z(), z()
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
    return flo, fhi, rlo, rhi


def min128(alo, ahi, blo, bhi):
    a_first = (ahi < bhi) | ((ahi == bhi) & (alo <= blo))
    return np.where(a_first, alo, blo), np.where(a_first, ahi, bhi)


def canonical_codes128_np(seq: bytes, k: int):
    """k > 32: (lo, hi) words of the canonical codes of the ACGT-only k-mers
    of seq (case-folded), in order."""
    s = np.frombuffer(seq.upper(), dtype=np.uint8)
    lut = np.full(256, 4, dtype=np.uint8)
    for i, c in enumerate(b"ACGT"):
        lut[c] = i
    v = lut[s]
    n = len(v) - k + 1
    if n <= 0:
        return np.zeros(0, dtype=np.uint64), np.zeros(0, dtype=np.uint64)
    cb = np.concatenate([[0], np.cumsum(v > 3)])
    ok = ((cb[k:] - cb[:-k]) == 0)[:n]
    v = np.where(v > 3, 0, v).astype(np.uint64)
    lo, hi = min128(*_split_codes(v, k))
    return lo[ok], hi[ok]


def random_codes128(rng, n, k):
    """n random canonical k-mers (k > 32) as (lo, hi)."""
    v = rng.integers(0, 4, (n, k)).astype(np.uint64)
    flo, fhi, rlo, rhi = (np.zeros(n, dtype=np.uint64) for _ in range(4))
    for t in range(k):
        fb = 2 * (k - 1 - t)
        if fb >= 64:
            fhi |= v[:, t] << np.uint64(fb - 64)
        else:
            flo |= v[:, t] << np.uint64(fb)
        c = np.uint64(3) - v[:, t]
        if 2 * t >= 64:
            rhi |= c << np.uint64(2 * t - 64)
        else:
            rlo |= c << np.uint64(2 * t)
    return min128(flo, fhi, rlo, rhi)


def random_codes(rng, n, k) -> np.ndarray:
    mask = (1 << (2 * k)) - 1 if k < 32 else (1 << 64) - 1
    x = rng.integers(0, 1 << 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    x &= np.uint64(mask)
    # canonical: min(x, revcomp(x))
    rc = np.zeros(n, dtype=np.uint64)
    y = x.copy()
    for _ in range(k):
        rc = (rc << np.uint64(2)) | (np.uint64(3) - (y & np.uint64(3)))
        y >>= np.uint64(2)
    return np.minimum(x, rc)


# ---------------------------------------------------------------------------
# cases
# ---------------------------------------------------------------------------
EDGE_CASES = {
    # name: k, KMC params, windows, reference file flavour
    "edge_k25": dict(k=25, p=5, version=0x200, counter_size=1, windows=[5000, 50000], fmt="fasta"),
    "edge_k31": dict(k=31, p=7, version=0x200, counter_size=2, windows=[5000], fmt="fasta"),
    "edge_k32": dict(k=32, p=8, version=0x200, counter_size=1, windows=[1000], fmt="fasta"),
    "edge_k15": dict(k=15, p=7, version=0x200, counter_size=0, windows=[100, 5000], fmt="fasta"),
    "edge_k25_kmc1": dict(k=25, p=5, version=0, counter_size=1, windows=[5000], fmt="fasta"),
    "edge_k25_crlf": dict(k=25, p=9, version=0x200, counter_size=1, windows=[5000], fmt="crlf"),
    "edge_k25_fastq": dict(k=25, p=5, version=0x200, counter_size=1, windows=[5000], fmt="fastq"),
    "edge_k25_gz": dict(k=25, p=5, version=0x200, counter_size=1, windows=[5000], fmt="gz"),
    # k > 32: the reference's string path (two-word codes here)
    "edge_k33": dict(k=33, p=9, version=0x200, counter_size=1, windows=[5000], fmt="fasta"),
    "edge_k41": dict(k=41, p=5, version=0x200, counter_size=2, windows=[1000, 5000], fmt="fasta"),
    "edge_k64": dict(k=64, p=8, version=0, counter_size=0, windows=[5000], fmt="fasta"),
}


def ref_filename(fmt: str) -> str:
    return {"fasta": "test_genome.fasta", "crlf": "test_genome.fa", "fastq": "test_genome.fna",
            "gz": "test_genome.fasta.gz"}[fmt]


def build_edge_case(name: str, root: Path):
    """Writes <root>/<name>/{db/sample.kmc_*, refs/<file>}; returns paths."""
    spec = EDGE_CASES[name]
    k = spec["k"]
    seed = 7000 + sum(map(ord, name))
    d = root / name
    (d / "db").mkdir(parents=True, exist_ok=True)
    (d / "refs").mkdir(parents=True, exist_ok=True)
    recs = edge_contigs(k, seed)
    fmt = spec["fmt"]
    refs = [(n, r) for n, r, _ in recs]
    ref_path = d / "refs" / ref_filename(fmt)
    if fmt == "fasta":
        data = fasta_bytes(refs)
    elif fmt == "crlf":
        data = fasta_bytes(refs, crlf=True)
    elif fmt == "fastq":
        data = fastq_bytes(refs)
    else:
        data = gzip.compress(fasta_bytes(refs), mtime=0)
    ref_path.write_bytes(data)
    rng = np.random.default_rng(seed + 1)
    prefix = d / "db" / "sample"
    kmc = dict(k=k, p=spec["p"], sig_len=9, n_bins=64, counter_size=spec["counter_size"], version=spec["version"],
               min_count=2 if spec["counter_size"] else 0, max_count=255 if spec["counter_size"] == 1 else 65535)
    if k > 32:
        parts = [canonical_codes128_np(c, k) for _, _, c in recs]
        total = sum(len(lo) for lo, _ in parts)
        parts.append(random_codes128(rng, total // 20, k))
        lo = np.concatenate([a for a, _ in parts])
        hi = np.concatenate([b for _, b in parts])
        ib.kmc_write128(str(prefix), lo, hi, **kmc)
    else:
        codes = [canonical_codes_np(c, k) for _, _, c in recs]
        total = sum(len(c) for c in codes)
        codes.append(random_codes(rng, total // 20, k))
        allc = np.concatenate(codes)
        ib.kmc_write(str(prefix), allc, len(allc), **kmc)
    return dict(db=d / "db", prefix=prefix, refs=d / "refs", ref=ref_path, k=k, windows=spec["windows"])


def build_workload(w: configs.Workload, root: Path):
    """Writes a configs workload (host generation) as FASTA + KMC DB."""
    d = root / w.name
    (d / "db").mkdir(parents=True, exist_ok=True)
    (d / "refs").mkdir(parents=True, exist_ok=True)
    seq, mask = w.ref.reference_host()
    codes = w.samples[0].codes_host(w.ref, seq, mask)
    prefix = d / "db" / "sample"
    ib.kmc_write(str(prefix), codes, len(codes), **w.kmc)
    ref_path = d / "refs" / "test_genome.fasta"
    w.ref.write_fasta(str(ref_path))
    return dict(db=d / "db", prefix=prefix, refs=d / "refs", ref=ref_path, k=w.k, windows=[w.window],
                seq=seq, mask=mask)


def input_hashes(case) -> dict:
    return {"ref": sha256_file(case["ref"]),
            "kmc_pre": sha256_file(str(case["prefix"]) + ".kmc_pre"),
            "kmc_suf": sha256_file(str(case["prefix"]) + ".kmc_suf")}


def golden_path(name: str) -> Path:
    return GOLDEN / f"{name}.json"


def load_golden(name: str) -> dict:
    return json.loads(golden_path(name).read_text())


def build_case(name: str, root: Path):
    if name in EDGE_CASES:
        return build_edge_case(name, root)
    return build_workload(getattr(configs, name)(), root)


GOLDEN_CASES = list(EDGE_CASES) + ["plain_1mbp"]


# ---------------------------------------------------------------------------
# intersection cases: two samples of one reference, in different KMC layouts
# ---------------------------------------------------------------------------
INTERSECT_CASES = {
    # name: k, and the KMC layouts of sample A and sample B
    "x_k25": dict(k=25, a=dict(p=5, version=0x200, counter_size=1), b=dict(p=9, version=0, counter_size=2)),
    "x_k31": dict(k=31, a=dict(p=7, version=0x200, counter_size=1), b=dict(p=3, version=0x200, counter_size=0)),
    "x_k15": dict(k=15, a=dict(p=7, version=0, counter_size=1), b=dict(p=3, version=0x200, counter_size=1)),
    "x_k32": dict(k=32, a=dict(p=8, version=0x200, counter_size=1), b=dict(p=4, version=0x200, counter_size=1)),
    # k > 32 (two-word codes; the reference's string path)
    "x_k41": dict(k=41, a=dict(p=5, version=0x200, counter_size=1), b=dict(p=9, version=0, counter_size=2)),
}


def _wide_sample_codes(seqs, k: int, seed: int, rate: float, present: float, extra: float):
    """k > 32 samples for the intersection cases: the canonical k-mers of a
    copy of the reference with SNPs at `rate`, keeping each 20 kbp block with
    probability `present`, plus random k-mers (`extra` per reference base)."""
    rng = np.random.default_rng(seed)
    lo, hi = [], []
    for s in seqs:
        a = np.frombuffer(s.upper(), dtype=np.uint8).copy()
        snp = rng.random(len(a)) < rate
        a[snp] = BASES[rng.integers(0, 4, int(snp.sum()))]
        for b0 in range(0, len(a), 20_000):
            if rng.random() < present:
                x, y = canonical_codes128_np(bytes(a[b0:b0 + 20_000]), k)
                lo.append(x)
                hi.append(y)
    x, y = random_codes128(rng, int(extra * sum(len(s) for s in seqs)), k)
    return np.concatenate(lo + [x]), np.concatenate(hi + [y])


def build_intersect_case(name: str, root: Path):
    """Writes <root>/<name>/{a,b}/sample.kmc_*: two samples of one seeded
    400 kbp reference (1% and 3% SNP copies, each with random extra k-mers,
    B keeping 60% of its blocks); returns their folders and prefixes."""
    spec = INTERSECT_CASES[name]
    k = spec["k"]
    seed = 900 + k
    ref = ib.RefSpec(seed=seed, lens=[300_000, 100_000], n_frac=0.002, n_run=(1, 200))
    seq, mask = ref.reference_host()
    out = dict(k=k)
    if k > 32:
        seqs = [ref.contig_ascii(c) for c in range(len(ref.lens))]
        for side, rate, present, extra in (("a", 0.01, 1.0, 0.05), ("b", 0.03, 0.6, 0.10)):
            lo, hi = _wide_sample_codes(seqs, k, seed * 10 + ord(side), rate, present, extra)
            lay = spec[side]
            d = root / name / side
            d.mkdir(parents=True, exist_ok=True)
            ib.kmc_write128(str(d / "sample"), lo, hi, k=k, p=lay["p"], sig_len=9, n_bins=64,
                            counter_size=lay["counter_size"], version=lay["version"],
                            min_count=2 if lay["counter_size"] else 0,
                            max_count=255 if lay["counter_size"] == 1 else 65535)
            out[side] = d
            out["prefix_" + side] = d / "sample"
        return out
    for side, rate, present, extra in (("a", 0.01, 1.0, 0.05), ("b", 0.03, 0.6, 0.10)):
        smp = ib.SampleSpec(seed=seed * 10 + ord(side), k=k, class_rate=(rate,), class_prob=(1.0,),
                            block_len=20_000, present_frac=present, random_frac=extra)
        codes = smp.codes_host(ref, seq, mask)
        lay = spec[side]
        d = root / name / side
        d.mkdir(parents=True, exist_ok=True)
        ib.kmc_write(str(d / "sample"), codes, len(codes), k=k, p=lay["p"], sig_len=9, n_bins=64,
                     counter_size=lay["counter_size"], version=lay["version"],
                     min_count=2 if lay["counter_size"] else 0,
                     max_count=255 if lay["counter_size"] == 1 else 65535)
        out[side] = d
        out["prefix_" + side] = d / "sample"
    return out


def intersect_hashes(case) -> dict:
    return {s + ext: sha256_file(str(case["prefix_" + s]) + ext) for s in ("a", "b")
            for ext in (".kmc_pre", ".kmc_suf")}
