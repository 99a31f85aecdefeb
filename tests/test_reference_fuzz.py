"""The oracle against the reference's own binaries on seeded random inputs
(CPU only; skipped where oracle/_ref/ was not built from the reference's
sources).

The golden files pin the oracle on fixed cases; this runs the reference's
fastibs (CPU-OPT, and its string path for k > 32) and fastibsmapper live on
small random references -- N runs of random lengths, lowercase runs, contigs
shorter than k and of exactly k, windows of a few k -- against databases
that hold part of the reference's own k-mers and random ones, for k on both
sides of 32, and compares the files byte for byte.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

REF_DIR = corpus.REPO / "oracle" / "_ref"
LETTERS = np.frombuffer(b"ACGT", np.uint8)


def _need(binary: str):
    exe = REF_DIR / binary
    if not exe.exists():
        pytest.skip(f"oracle/_ref/{binary} not built (needs the reference's sources)")
    return exe


def _contig(rng, n, k):
    a = LETTERS[rng.integers(0, 4, n)].copy()
    for _ in range(int(rng.integers(0, 4))):  # N runs, some of about k
        at = int(rng.integers(0, max(1, n)))
        a[at:at + int(rng.choice([1, k - 1, k, 2 * k, int(rng.integers(1, 300))]))] = ord("N")
    for _ in range(int(rng.integers(0, 3))):  # lowercase runs
        at = int(rng.integers(0, max(1, n)))
        seg = a[at:at + int(rng.integers(1, 500))]
        a[at:at + len(seg)] = np.where(seg == ord("N"), seg, seg + 32)
    return bytes(a)


def _case(tmp_path, seed: int, k: int):
    """A reference FASTA and a KMC database of about half its k-mers plus 5% random ones."""
    rng = np.random.default_rng(seed)
    seqs = [_contig(rng, int(rng.integers(2 * k, 20_000)), k) for _ in range(3)]
    seqs += [_contig(rng, k - 1, k), _contig(rng, k, k)]
    refs = tmp_path / "refs"
    refs.mkdir()
    (refs / "fz_genome.fasta").write_bytes(corpus.fasta_bytes([(f"c{i}", s) for i, s in enumerate(seqs)],
                                                              width=int(rng.integers(50, 120))))
    db = tmp_path / "db"
    db.mkdir()
    p = int(rng.choice([p for p in range(1, 12) if (k - p) % 4 == 0]))
    kmc = dict(k=k, p=p, sig_len=9 if k >= 9 else 5, n_bins=64, counter_size=int(rng.integers(0, 3)),
               version=int(rng.choice([0, 0x200])))
    if k > 32:
        lo, hi = [], []
        for s in seqs:
            a, b = orc.canonical_codes128(s, k)
            keep = rng.random(len(a)) < 0.5
            lo.append(a[keep])
            hi.append(b[keep])
        n = sum(len(x) for x in lo)
        a, b = corpus.random_codes128(rng, max(1, n // 20), k)
        ib.kmc_write128(str(db / "s"), np.concatenate(lo + [a]), np.concatenate(hi + [b]), **kmc)
    else:
        codes = [c[rng.random(len(c)) < 0.5] for c in (orc.canonical_codes(s, k) for s in seqs)]
        n = sum(len(c) for c in codes)
        codes.append(corpus.random_codes(rng, max(1, n // 20), k))
        allc = np.concatenate(codes)
        ib.kmc_write(str(db / "s"), allc, len(allc), **kmc)
    return seqs, refs, db


@pytest.mark.parametrize("seed,k", [(1, 21), (2, 31), (3, 32), (4, 33), (5, 47), (6, 58), (7, 64)])
def test_fastibs_matches_oracle_on_random_inputs(tmp_path, seed, k):
    exe = _need("fastibs")
    seqs, refs, db = _case(tmp_path, seed, k)
    ids, read = orc.read_sequence_file(str(refs / "fz_genome.fasta"))
    assert read == seqs
    ix = orc.Index(str(db / "s"))
    for W in (k + 1, 3 * k, 5000):
        out = tmp_path / f"out{W}"
        r = subprocess.run([str(exe), str(db), str(refs), str(out), str(W), "--cpu"], capture_output=True,
                           text=True, env=dict(os.environ, FASTIBS_THREADS="4"))
        assert r.returncode == 0, r.stderr[-2000:]
        (f,) = sorted(out.glob("*.tsv"))
        rows = orc.scan(ix, seqs, W, k, threads=4)
        assert f.read_text() == orc.tsv_text(ids, [len(s) for s in seqs], rows, W, k), (k, W)
        shutil.rmtree(out)


@pytest.mark.parametrize("seed,k", [(11, 25), (12, 41), (13, 64)])
def test_fastibsmapper_matches_oracle_on_random_inputs(tmp_path, seed, k):
    exe = _need("fastibsmapper")
    seqs, refs, db = _case(tmp_path, seed, k)
    ids, _ = orc.read_sequence_file(str(refs / "fz_genome.fasta"))
    out = tmp_path / "map"
    r = subprocess.run([str(exe), str(db), str(refs), str(out)], capture_output=True, text=True,
                       env=dict(os.environ, FASTIBS_THREADS="4"))
    assert r.returncode == 0, r.stderr[-2000:]
    (f,) = sorted(out.glob("*.txt"))
    assert f.read_bytes() == orc.mapping_text(orc.Index(str(db / "s")), ids, seqs, k)
