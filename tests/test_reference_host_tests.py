"""The reference's own host tests run against KMC databases written by this
repository's writer (libibs_tools' kmc_write).

tests/phase1_test.cpp of the reference (KmcRaIndex load and probe against the
vendored KMC API's CKMCFile: every listed k-mer is a hit, 2M random and
codec queries agree, the batched CPU probe agrees query for query) and
tests/phase2_test.cpp (the reference's window pipeline against its codec on
synthetic windows and on the database, with the database's own reference
FASTA) are compiled from the reference sources into oracle/_ref/ by
`make -C oracle ref`; without them these tests skip. CPU only.
"""
import subprocess

import pytest

import corpus

REF_BIN = corpus.REPO / "oracle" / "_ref"

# KMC layouts the writer produces: KMC2 (0x200) and KMC1 (0) files, counter
# widths 0..2, prefix lengths 5..9, k = 15, 25, 31, 32
CASES = ["edge_k25", "edge_k25_kmc1", "edge_k31", "edge_k32", "edge_k15", "edge_k25_crlf", "plain_1mbp"]


def _run(binary: str, *args, timeout=600):
    exe = REF_BIN / binary
    if not exe.exists():
        pytest.skip(f"oracle/_ref/{binary} not built (needs the reference sources)")
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=timeout)
    return r


@pytest.mark.parametrize("name", CASES)
def test_reference_phase1_accepts_the_writers_database(name, build_case):
    case = build_case(name)
    r = _run("phase1_test", case["prefix"])
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "ALL PHASE 1 HOST TESTS PASSED" in r.stdout
    assert "FAIL" not in r.stdout


@pytest.mark.parametrize("name", ["edge_k25", "edge_k31", "plain_1mbp"])
def test_reference_phase2_on_the_writers_database(name, build_case):
    case = build_case(name)
    ref = case["ref"]
    r = _run("phase2_test", case["prefix"], ref)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "ALL PHASE 2 HOST TESTS PASSED" in r.stdout
    assert "real db:" in r.stdout
