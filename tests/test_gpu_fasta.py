"""FASTA text parsed and packed on the device (ibs_reference_from_fasta):
the same contigs, ids and packed words as the reference reader restated in
the oracle plus the host packer, and the golden TSVs when scanned."""
import gzip

import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

pytestmark = pytest.mark.gpu


def host_view(path, text):
    ids, seqs = orc.read_sequence_file(str(path))
    seq, mask, lens = ib.pack_ascii(seqs)
    return ids, lens, seq, mask


def check_against_host(ref, ids, lens, seq, mask):
    assert [i.decode(errors="surrogateescape") for i in ref.ids] == ids
    assert np.array_equal(ref.lens, lens)
    dseq, dmask = ref.copy_packed()
    assert np.array_equal(dseq, seq) and np.array_equal(dmask, mask)


@pytest.mark.parametrize("name", [n for n in corpus.GOLDEN_CASES if n != "edge_k25_fastq"])
def test_device_parse_matches_reader_and_goldens(name, build_case):
    case = build_case(name)
    raw = case["ref"].read_bytes()
    text = gzip.decompress(raw) if str(case["ref"]).endswith(".gz") else raw
    ref = ib.Reference.from_fasta(text)
    check_against_host(ref, *host_view(case["ref"], text))
    gold = corpus.load_golden(name)
    t = ib.Table.open(str(case["prefix"]))
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    for W in case["windows"]:
        rows = ib.scan(t, ref, W)
        assert orc.tsv_text(ids, [len(s) for s in seqs], rows, W, case["k"]) == gold["tsv"][str(W)], (name, W)
    t.close()
    ref.free()


def test_device_parse_edge_layouts(tmp_path):
    rng = np.random.default_rng(11)
    alphabet = np.frombuffer(b"ACGTacgtNnRYKM\r>", np.uint8)
    recs = []
    for i in range(40):
        n = int(rng.integers(0, 30_000)) if i % 7 else 0  # some records without sequence
        body = bytes(rng.choice(alphabet[:12], n, p=[.21] * 4 + [.02] * 8))
        if i % 5 == 1:
            body = body.replace(b"N", b">", 3)  # '>' inside a sequence line is a base
        recs.append((f"contig_{i} desc {i}".encode() + (b"\r" if i % 3 == 0 else b""), body))
    out = bytearray()
    for j, (hdr, body) in enumerate(recs):
        out += b">" + hdr + b"\n"
        width = int(rng.integers(1, 130))
        for a in range(0, len(body), width):
            line = body[a:a + width]
            if line.startswith(b">"):
                line = b"A" + line[1:]  # keep the line a sequence line
            out += line + (b"\r\n" if j % 4 == 2 else b"\n")
            if rng.random() < 0.01:
                out += b"\n"  # empty lines are skipped
    text = bytes(out[:-1])  # no newline at the end of the file
    path = tmp_path / "edge.fasta"
    path.write_bytes(text)
    ref = ib.Reference.from_fasta(text)
    check_against_host(ref, *host_view(path, text))
    ref.free()


def test_device_parse_refuses_what_it_does_not_read():
    with pytest.raises(ib.IbsError) as e:
        ib.Reference.from_fasta(b"@read\nACGT\n+\nIIII\n")
    assert e.value.status == 6
    with pytest.raises(ib.IbsError) as e:
        ib.Reference.from_fasta(b"ACGT\n")
    assert e.value.status == 3
    with pytest.raises(ib.IbsError) as e:
        ib.Reference.from_fasta(b"")
    assert e.value.status == 3
