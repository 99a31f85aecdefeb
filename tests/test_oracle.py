"""The CPU oracle against the golden fixtures made by the reference's own
fastibs binary (tests/golden/make_golden.py), and its parts against their
reference counterparts' documented behaviour."""
import numpy as np
import pytest

import corpus
import oracle as orc


@pytest.mark.parametrize("name", corpus.GOLDEN_CASES)
def test_oracle_matches_reference_golden(name, build_case):
    gold = corpus.load_golden(name)
    case = build_case(name)
    assert corpus.input_hashes(case) == gold["inputs_sha256"], "inputs differ from the golden run"
    ix = orc.Index(str(case["prefix"]))
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    for W in case["windows"]:
        rows = orc.scan(ix, seqs, W, case["k"], threads=4)
        text = orc.tsv_text(ids, [len(s) for s in seqs], rows, W, case["k"])
        assert text == gold["tsv"][str(W)]


@pytest.mark.parametrize("name", ["edge_k25", "edge_k31", "edge_k32", "edge_k15", "edge_k25_kmc1"])
def test_index_lists_exactly_the_written_keys(name, build_case):
    case = build_case(name)
    ix = orc.Index(str(case["prefix"]))
    listed = ix.list_codes()
    assert len(listed) == ix.total
    assert len(np.unique(listed)) == ix.total
    assert ix.probe(listed).all()


def test_codec_matches_numpy_restatement():
    rng = np.random.default_rng(5)
    for k in (4, 15, 25, 31, 32):
        s = bytes(np.frombuffer(b"ACGTacgtNRn", np.uint8)[rng.integers(0, 11, 5000)])
        assert np.array_equal(orc.canonical_codes(s, k), corpus.canonical_codes_np(s, k))


def test_window_rule():
    # chunkSequences: [j, min(j+W, len)) for j = 0, W-k, ... (src/Utils.hpp:296-327)
    assert orc.window_count(0, 100, 25) == 0
    assert orc.window_count(1, 100, 25) == 1
    assert orc.window_count(75, 100, 25) == 1
    assert orc.window_count(76, 100, 25) == 2
    assert orc.window_count(100, 100, 25) == 2
    assert orc.window_count(100, 25, 25) == 0  # W <= k is rejected


def test_gap_statistics_rules():
    k = 25
    # addVariationOriginal: d = g-(k-1); d <= 0 -> |d+1| (src/Window.hpp:29-36)
    def dist(g):
        d = g - (k - 1)
        return abs(d + 1) if d <= 0 else d
    r = orc.stats_from_hits([1, 0, 0, 1, 1, 0], k)
    assert (r["total_kmers"], r["observed_kmers"], r["variations"]) == (6, 3, 2)
    assert r["kmer_distance"] == dist(2) + dist(1)
    r = orc.stats_from_hits([0] * 30, k)
    assert (r["variations"], r["kmer_distance"]) == (1, dist(30))
    r = orc.stats_from_hits([], k)
    assert (r["total_kmers"], r["variations"], r["kmer_distance"]) == (0, 0, 0)


def test_reader_quirks(tmp_path):
    # ids keep the whole header line; '\r' stays in ids and sequences; empty
    # records are dropped; FASTQ quality lines are skipped (src/Utils.hpp:170-255)
    p = tmp_path / "x.fa"
    p.write_bytes(b">a b c\r\nAC\r\nGT\n>empty\n>b\nNNNN\n\n>c\nacgt")
    ids, seqs = orc.read_sequence_file(str(p))
    assert ids == ["a b c\r", "b", "c"]
    assert seqs == [b"AC\rGT", b"NNNN", b"acgt"]
    q = tmp_path / "x.fq"
    q.write_bytes(b"@r1\nACGT\n+\n@@@@\n@r2\nGG\n+\nII\n")
    ids, seqs = orc.read_sequence_file(str(q))
    assert ids == ["r1", "r2"] and seqs == [b"ACGT", b"GG"]
    bad = tmp_path / "bad.fa"
    bad.write_bytes(b"ACGT\n")
    with pytest.raises(orc.OracleError, match="Unknown file type"):
        orc.read_sequence_file(str(bad))
