"""GPU parity: the sm_100a scan through the C-ABI against the golden TSVs of
the reference's own binary and against the CPU oracle."""
import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

pytestmark = pytest.mark.gpu


def tsv_of(ids, lens, rows, W, k):
    return orc.tsv_text(ids, lens, rows, W, k)


def rows_of_case(case, table, W, path="resident"):
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    if path == "resident":
        ref = ib.Reference(seq, mask, lens)
        rows = ib.scan(table, ref, W)
        ref.free()
    elif path == "packed":
        rows = ib.scan_packed(table, seq, mask, lens, W)
    elif path == "async":
        import torch
        ref = ib.Reference(seq, mask, lens)
        n = ib.window_count(lens, W, case["k"])
        dev = torch.zeros(max(n, 1) * 6, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        ib.scan_async(table, ref, W, dev.data_ptr(), n, s.cuda_stream)
        s.synchronize()
        rows = dev.cpu().numpy().view(ib.WINDOW_DTYPE)[:n]
        ref.free()
    return ids, [len(s) for s in seqs], rows


@pytest.mark.parametrize("name", corpus.GOLDEN_CASES)
def test_scan_matches_reference_golden(name, build_case):
    gold = corpus.load_golden(name)
    case = build_case(name)
    assert corpus.input_hashes(case) == gold["inputs_sha256"]
    t = ib.Table.open(str(case["prefix"]))
    for W in case["windows"]:
        for path in ("resident", "packed", "async"):
            ids, lens, rows = rows_of_case(case, t, W, path)
            assert tsv_of(ids, lens, rows, W, case["k"]) == gold["tsv"][str(W)], (name, W, path)
    t.close()


@pytest.mark.parametrize("fmt,kpb", [(1, 0.0), (2, 0.0), (1, 7.5), (2, 5.5), (0, 12.0)])
def test_table_formats_and_stash_agree_with_oracle(fmt, kpb, build_case):
    for name in ("edge_k25", "edge_k31", "edge_k32", "edge_k15"):
        case = build_case(name)
        if fmt == 1 and case["k"] > 25:
            continue  # B8x32 needs N >= 2^(2k-31) buckets: too large to force here
        t = ib.Table.open(str(case["prefix"]), force_format=fmt, keys_per_bucket=kpb)
        info = t.info()
        ix = orc.Index(str(case["prefix"]))
        listed = ix.list_codes()
        assert info.n_keys == ix.total
        assert t.probe(listed).all()
        rng = np.random.default_rng(5)
        q = corpus.random_codes(rng, 50_000, case["k"])
        assert np.array_equal(t.probe(q), ix.probe(q))
        gold = corpus.load_golden(name)
        W = case["windows"][0]
        ids, lens, rows = rows_of_case(case, t, W)
        assert tsv_of(ids, lens, rows, W, case["k"]) == gold["tsv"][str(W)]
        # B8x32 keeps >= 2^(2k-31) buckets, so only small k reach a high load
        slots = 8 if info.format == 1 else 6
        if info.n_keys / info.n_buckets >= 0.8 * slots:
            assert info.stash_keys > 0, "the stash path was not exercised"
        t.close()


def test_stash_is_exercised_and_exact(build_case):
    case = build_case("edge_k15")
    for fmt, kpb in ((1, 9.0), (2, 7.0)):
        t = ib.Table.open(str(case["prefix"]), force_format=fmt, keys_per_bucket=kpb)
        info = t.info()
        assert info.stash_keys > 0
        ix = orc.Index(str(case["prefix"]))
        listed = ix.list_codes()
        assert t.probe(listed).all()
        q = corpus.random_codes(np.random.default_rng(8), 100_000, 15)
        assert np.array_equal(t.probe(q), ix.probe(q))
        gold = corpus.load_golden("edge_k15")
        ids, lens, rows = rows_of_case(case, t, 100)
        assert tsv_of(ids, lens, rows, 100, 15) == gold["tsv"]["100"]
        t.close()


def test_panel_equals_single_scans(build_case):
    cases = [build_case(n) for n in ("edge_k25", "edge_k25_kmc1")]
    tables = [ib.Table.open(str(c["prefix"])) for c in cases]
    # both share k=25; scan one reference against both
    ids, seqs = orc.read_sequence_file(str(cases[0]["ref"]))
    seq, mask, lens = ib.pack_ascii(seqs)
    ref = ib.Reference(seq, mask, lens)
    panel = ib.scan_panel(tables + tables[:1], ref, 5000)
    for i, t in enumerate(tables + tables[:1]):
        single = ib.scan(t, ref, 5000)
        assert np.array_equal(panel[i], single)


def test_device_generator_matches_host(tmp_path):
    import torch
    from ibs_b200 import configs
    w = configs.plain_2gbp(scale=0.002)  # 4 Mbp, same shape
    seq, mask = w.ref.reference_host()
    sw, mw = w.ref.packed_words()
    dseq = torch.zeros(sw, dtype=torch.int64, device="cuda")
    dmask = torch.zeros(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    assert np.array_equal(dseq.cpu().numpy().view(np.uint64), seq)
    assert np.array_equal(dmask.cpu().numpy().view(np.uint64), mask)
    host_codes = w.samples[0].codes_host(w.ref, seq, mask)
    bound = w.samples[0].codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
    out = torch.zeros(bound, dtype=torch.int64, device="cuda")
    n = w.samples[0].codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), out.data_ptr(), bound)
    dev_codes = out[:n].cpu().numpy().view(np.uint64)
    assert np.array_equal(np.unique(dev_codes), np.unique(host_codes))
    # the device KMC writer writes the same files as the host writer
    a, b = tmp_path / "h", tmp_path / "d"
    ib.kmc_write(str(a), host_codes, len(host_codes), **w.kmc)
    ib.kmc_write(str(b), out.data_ptr(), n, on_device=True, **w.kmc)
    for ext in (".kmc_pre", ".kmc_suf"):
        assert corpus.sha256_file(str(a) + ext) == corpus.sha256_file(str(b) + ext)


def test_40mbp_against_oracle(tmp_path):
    from ibs_b200 import configs
    w = configs.plain_2gbp(scale=0.02)  # 40 Mbp in 10 contigs, ~44M k-mers
    case = corpus.build_workload(w, tmp_path)
    t = ib.Table.open(str(case["prefix"]))
    ix = orc.Index(str(case["prefix"]))
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    want = orc.scan(ix, seqs, w.window, w.k, threads=16)
    seq, mask, lens = ib.pack_ascii(seqs)
    assert np.array_equal(seq, case["seq"]) and np.array_equal(mask, case["mask"])
    ref = ib.Reference(seq, mask, lens)
    got = ib.scan(t, ref, w.window)
    assert np.array_equal(got, want)
    got2 = ib.scan_packed(t, seq, mask, lens, w.window)
    assert np.array_equal(got2, want)
    # size-independent properties
    assert got["total_kmers"].sum() > 0.9 * sum(lens)
    assert (got["observed_kmers"] <= got["total_kmers"]).all()


def test_scan_argument_errors(build_case):
    case = build_case("edge_k25")
    t = ib.Table.open(str(case["prefix"]))
    seq, mask, lens = ib.pack_ascii([b"ACGT" * 100])
    ref = ib.Reference(seq, mask, lens)
    with pytest.raises(ib.IbsError) as e:
        ib.scan(t, ref, 25)  # W <= k
    assert e.value.status == 1
    empty = ib.Reference(*ib.pack_ascii([b""])[:2], np.array([0], np.uint64))
    assert len(ib.scan(t, empty, 1000)) == 0


@pytest.mark.parametrize("name,fmt", [("edge_k25", 4), ("edge_k25_kmc1", 4), ("edge_k25_crlf", 4), ("plain_1mbp", 4),
                                      ("edge_k25_gz", 4), ("edge_k31", 6), ("edge_k25", 6), ("plain_1mbp", 6)])
def test_minimizer_table_matches_reference_golden(name, fmt, build_case):
    # format 4: B8x32 sectors (k <= 27); format 6: B6x40 sectors (k <= 31)
    gold = corpus.load_golden(name)
    case = build_case(name)
    t = ib.Table.open(str(case["prefix"]), force_format=fmt)
    info = t.info()
    assert info.format == fmt
    ix = orc.Index(str(case["prefix"]))
    assert t.probe(ix.list_codes()).all()
    q = corpus.random_codes(np.random.default_rng(6), 100_000, case["k"])
    assert np.array_equal(t.probe(q), ix.probe(q))
    for W in case["windows"]:
        for path in ("resident", "packed"):
            ids, lens, rows = rows_of_case(case, t, W, path)
            assert tsv_of(ids, lens, rows, W, case["k"]) == gold["tsv"][str(W)], (name, W, path)
    t.close()


def test_minimizer_table_40mbp_and_overflow(tmp_path):
    from ibs_b200 import configs
    w = configs.plain_2gbp(scale=0.02)
    case = corpus.build_workload(w, tmp_path)
    ix = orc.Index(str(case["prefix"]))
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    want = orc.scan(ix, seqs, w.window, w.k, threads=16)
    seq, mask, lens = ib.pack_ascii(seqs)
    ref = ib.Reference(seq, mask, lens)
    for kpb in (4.0, 7.0):  # 7 keys per bucket forces overflow into the stash
        t = ib.Table.open(str(case["prefix"]), force_format=4, keys_per_bucket=kpb)
        if kpb == 7.0:
            assert t.info().stash_keys > 0
        assert np.array_equal(ib.scan(t, ref, w.window), want)
        t.close()


@pytest.mark.parametrize("name,fmt", [("edge_k31", 4), ("edge_k32", 6), ("edge_k15", 4), ("edge_k15", 6)])
def test_minimizer_format_rejects_unsupported_k(name, fmt, build_case):
    case = build_case(name)
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(case["prefix"]), force_format=fmt)
    assert e.value.status == 6


@pytest.mark.parametrize("k,fmt", [(16, 4), (21, 4), (22, 4), (24, 4), (16, 6), (25, 6), (28, 6), (31, 6)])
def test_minimizer_table_at_other_k_equals_hash_table(k, fmt):
    # the minimizer kernel's generic-k instances (k = 25 in B8x32 sectors and
    # k = 31 in B6x40 sectors have their own), with minimizer lengths 16
    # (k <= 22) and k - 6; rows equal the hash table's, which the goldens pin
    # to the reference
    spec = ib.RefSpec(seed=40 + k, lens=[250_000, 70_000, 23, 5_000], n_frac=0.003, n_run=(1, 150))
    seq, mask = spec.reference_host()
    smp = ib.SampleSpec(seed=400 + k, k=k, class_rate=(0.0001, 0.01, 0.03), class_prob=(0.3, 0.5, 0.2),
                        block_len=10_000, present_frac=0.8, random_frac=0.05)
    codes = smp.codes_host(spec, seq, mask)
    ref = ib.Reference(seq, mask, spec.lens)
    th = ib.Table.from_codes(codes, len(codes), k, on_device=False, force_format=5)
    tm = ib.Table.from_codes(codes, len(codes), k, on_device=False, force_format=fmt)
    assert tm.info().format == fmt
    for W in (1000, 5000):
        assert np.array_equal(ib.scan(tm, ref, W), ib.scan(th, ref, W)), (k, W)
    q = np.concatenate([codes[:20_000], corpus.random_codes(np.random.default_rng(k), 20_000, k)])
    assert np.array_equal(tm.probe(q), th.probe(q))
    th.close()
    tm.close()
    ref.free()
