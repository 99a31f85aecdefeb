"""fastibsmapper (per-base k-mer coverage): the oracle against the files the
reference's own fastibsmapper writes (tests/golden/mapper.json, made by
tests/golden/make_mapper_golden.py), then the device coverage
(ibs_map_coverage), the device-written text (ibs_map_text) and the
fastibsmapper CLI against both."""
import hashlib
import json
import subprocess

import numpy as np
import pytest

import corpus
import oracle as orc

GOLD = json.loads((corpus.GOLDEN / "mapper.json").read_text())
CLI = corpus.REPO / "gpu-ibs_b200" / "bin" / "fastibsmapper"


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


@pytest.mark.parametrize("name", corpus.GOLDEN_CASES)
def test_oracle_matches_reference_mapper(name, build_case):
    case = build_case(name)
    assert corpus.input_hashes(case) == GOLD["cases"][name]["inputs_sha256"]
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    text = orc.mapping_text(orc.Index(str(case["prefix"])), ids, seqs, case["k"])
    assert len(text) == GOLD["cases"][name]["bytes"]
    assert sha(text) == GOLD["cases"][name]["sha256"]


def test_cli_usage_without_a_device():
    r = subprocess.run([str(CLI)], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stdout
    assert subprocess.run([str(CLI), "--help"], capture_output=True).returncode == 0
    r = subprocess.run([str(CLI), "/nonexistent/db", "/nonexistent/refs", "/tmp/x"], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("Error: KMC database folder not found")


@pytest.mark.gpu
@pytest.mark.parametrize("name", corpus.GOLDEN_CASES)
def test_device_mapping_matches_reference(name, build_case):
    import ibs_b200 as ib
    case = build_case(name)
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    ref = ib.Reference(seq, mask, lens)
    ix = orc.Index(str(case["prefix"]))
    want_cov = np.concatenate([orc.coverage(ix, s, case["k"]) for s in seqs])
    # k > 32 has one layout, the wide-key table
    formats = ([0] if case["k"] > 32 else [0, 2] + ([1] if case["k"] <= 25 else [])
               + ([4] if 16 <= case["k"] <= 27 else []) + ([6] if 16 <= case["k"] <= 31 else []))
    for fmt in formats:
        t = ib.Table.open(str(case["prefix"]), force_format=fmt)
        assert np.array_equal(ib.map_coverage(t, ref).astype(np.int64), want_cov), (name, fmt)
        text = ib.map_text(t, ref, [i.encode(errors="surrogateescape") for i in ids])
        assert sha(text) == GOLD["cases"][name]["sha256"], (name, fmt)
        t.close()
    ref.free()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["edge_k25", "edge_k25_crlf", "edge_k25_fastq", "edge_k25_gz", "edge_k41",
                                  "plain_1mbp"])
def test_cli_writes_the_reference_file(name, build_case, tmp_path):
    case = build_case(name)
    out = tmp_path / "out"
    r = subprocess.run([str(CLI), str(case["db"]), str(case["refs"]), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = GOLD["cases"][name]
    f = out / g["name"]
    assert f.exists(), sorted(out.iterdir())
    assert sha(f.read_bytes()) == g["sha256"]
    # a second run skips the existing output
    r = subprocess.run([str(CLI), str(case["db"]), str(case["refs"]), str(out)], capture_output=True, text=True)
    assert r.returncode == 0 and "already exists" in r.stdout
