"""k > 32 on the device: wide-key tables (format 8) and the scans, mapper and
intersection over them, against the golden files of the reference's own
binaries (whose k > 32 runs take the string path, src/KmerDatabase.hpp:
100-124) and the CPU oracle."""
import shutil
import subprocess

import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

pytestmark = pytest.mark.gpu

WIDE = ["edge_k33", "edge_k41", "edge_k64"]
FASTIBS = corpus.REPO / "gpu-ibs_b200" / "bin" / "fastibs"


def _tsv(case, table, W):
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    ref = ib.Reference(seq, mask, lens)
    rows = ib.scan(table, ref, W)
    ref.free()
    return orc.tsv_text(ids, [len(s) for s in seqs], rows, W, case["k"])


@pytest.mark.parametrize("kpb", [0.0, 7.5, 1.0])
@pytest.mark.parametrize("name", WIDE)
def test_wide_table_probe_and_scan(name, kpb, build_case):
    """Every listed k-mer is found, random and near-miss queries agree with
    the oracle, and the rows equal the reference's TSV, at the default load,
    at a load that sends many keys to later levels, and at a light one."""
    case = build_case(name)
    k = case["k"]
    ix = orc.Index(str(case["prefix"]))
    t = ib.Table.open(str(case["prefix"]), keys_per_bucket=kpb)
    info = t.info()
    assert info.format == 8 and info.k == k and info.n_keys == ix.total
    if kpb == 7.5:
        assert info.stash_keys > 0, "no key reached a later level"
    lo, hi = ix.list_codes128()
    assert t.probe128(lo, hi).all()
    rng = np.random.default_rng(k)
    qlo, qhi = corpus.random_codes128(rng, 20_000, k)
    qlo = np.concatenate([qlo, lo[:5000] ^ np.uint64(4)])
    qhi = np.concatenate([qhi, hi[:5000]])
    assert np.array_equal(t.probe128(qlo, qhi), ix.probe128(qlo, qhi))
    gold = corpus.load_golden(name)
    for W in case["windows"]:
        assert _tsv(case, t, W) == gold["tsv"][str(W)], (name, W, kpb)
    t.close()


@pytest.mark.parametrize("name", WIDE)
def test_wide_scan_paths_agree(name, build_case):
    """The end-to-end host-buffer scan and the device-row scan give the
    resident scan's rows."""
    import torch
    case = build_case(name)
    t = ib.Table.open(str(case["prefix"]))
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    ref = ib.Reference(seq, mask, lens)
    for W in case["windows"]:
        want = ib.scan(t, ref, W)
        assert np.array_equal(ib.scan_packed(t, seq, mask, lens, W), want)
        n = len(want)
        dev = torch.zeros(max(n, 1) * 6, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        ib.scan_async(t, ref, W, dev.data_ptr(), n, s.cuda_stream)
        s.synchronize()
        assert np.array_equal(dev.cpu().numpy().view(ib.WINDOW_DTYPE)[:n], want)
    ref.free()
    t.close()


def test_wide_table_from_codes_with_duplicates(build_case):
    case = build_case("edge_k41")
    ix = orc.Index(str(case["prefix"]))
    lo, hi = ix.list_codes128()
    order = np.random.default_rng(1).permutation(2 * len(lo))
    dlo, dhi = np.concatenate([lo, lo])[order], np.concatenate([hi, hi])[order]
    t = ib.Table.from_codes128(dlo, dhi, 41)
    assert t.info().n_keys == len(lo)
    assert t.probe128(lo, hi).all()
    gold = corpus.load_golden("edge_k41")
    assert _tsv(case, t, 5000) == gold["tsv"]["5000"]
    t.close()


def test_wide_panel_of_tables_equals_single_scans(build_case):
    case = build_case("edge_k41")
    a = ib.Table.open(str(case["prefix"]))
    b = ib.Table.open(str(case["prefix"]), keys_per_bucket=7.5)
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    ref = ib.Reference(seq, mask, lens)
    rows = ib.scan_panel([a, b], ref, 1000)
    single = ib.scan(a, ref, 1000)
    assert np.array_equal(rows[0], single) and np.array_equal(rows[1], single)
    ref.free()
    a.close()
    b.close()


def test_wide_tables_are_refused_where_codes_are_one_word(build_case):
    import torch
    case = build_case("edge_k41")
    t = ib.Table.open(str(case["prefix"]))
    with pytest.raises(ib.IbsError) as e:
        t.probe(np.zeros(4, np.uint64))
    assert e.value.status == 1
    with pytest.raises(ib.IbsError) as e:
        t.count_present(np.zeros(4, np.uint64))
    assert e.value.status == 1
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    dseq = torch.from_numpy(seq.view(np.int64)).cuda()
    dmask = torch.from_numpy(mask.view(np.int64)).cuda()
    rows = torch.zeros(6 * 64, dtype=torch.int32, device="cuda")
    with pytest.raises(ib.IbsError) as e:
        ib.scan_noalloc(t, dseq.data_ptr(), dmask.data_ptr(), lens, 5000, rows.data_ptr(), 64)
    assert e.value.status == 6
    with pytest.raises(ib.IbsError):
        ib.PanelTable(41, 1000)
    ref = ib.Reference(seq, mask, lens)
    with pytest.raises(ib.IbsError):
        ib.Server(ref, 5000, 41)
    ref.free()
    t.close()
    # one-word k and the wide layout do not mix
    c25 = build_case("edge_k25")
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(c25["prefix"]), force_format=8)
    assert e.value.status == 6
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(case["prefix"]), force_format=4)
    assert e.value.status == 6


@pytest.mark.parametrize("name", WIDE)
def test_wide_cli_files_match_reference_golden(name, build_case, tmp_path):
    gold = corpus.load_golden(name)
    case = build_case(name)
    for W in case["windows"]:
        out = tmp_path / f"o{W}"
        r = subprocess.run([str(FASTIBS), str(case["db"]), str(case["refs"]), str(out), str(W)],
                           capture_output=True, text=True, cwd=tmp_path)
        assert r.returncode == 0, r.stderr
        assert "wide-key" in r.stderr
        f = out / gold["tsv_name"][str(W)]
        assert f.read_bytes().decode("latin-1") == gold["tsv"][str(W)]


def test_wide_cli_panel_runs_single_scans(build_case, tmp_path):
    """A k > 32 panel is scanned database by database (src/FastIBS.cpp:155-180),
    writing the files single runs write."""
    case = build_case("edge_k41")
    db2 = tmp_path / "db2"
    shutil.copytree(case["db"], db2)
    out = tmp_path / "panel"
    r = subprocess.run([str(FASTIBS), str(case["db"]), str(case["refs"]), str(out), "5000", f"--db={db2}"],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "> 32 has no panel path" in r.stdout
    gold = corpus.load_golden("edge_k41")
    for db in ("db", "db2"):
        assert (out / f"{db}_v_test_5000.tsv").read_bytes().decode("latin-1") == gold["tsv"]["5000"]
