"""The joint panel table: one bucket load per position for up to 16 samples,
every sample's rows equal to its single-sample scan."""
import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

pytestmark = pytest.mark.gpu


def _samples(ref_spec, seq, mask, n, k=25):
    out = []
    for s in range(n):
        smp = ib.SampleSpec(seed=900 + s, k=k, class_rate=(0.0001, 0.005, 0.02, 0.05),
                            class_prob=(0.2, 0.4, 0.3, 0.1), block_len=20_000,
                            present_frac=0.3 + 0.7 * ((s * 7) % 10) / 10, random_frac=0.05)
        out.append(np.unique(smp.codes_host(ref_spec, seq, mask)))
    return out


@pytest.mark.parametrize("n_samples,k,fmt", [(1, 25, 3), (5, 25, 3), (16, 25, 3), (16, 31, 0),
                                             (1, 25, 7), (5, 25, 7), (16, 25, 7)])
def test_panel_rows_equal_single_scans(n_samples, k, fmt):
    """fmt 3: hash sectors; 7: minimizer lines; 0: by size (k = 31: hash)."""
    ref_spec = ib.RefSpec(seed=77, lens=[400_000, 123_457, 24, 31, 90_000], n_frac=0.003,
                          n_run=(1, 200), lower_frac=0.02)
    seq, mask = ref_spec.reference_host()
    samples = _samples(ref_spec, seq, mask, n_samples, k)
    union = len(np.unique(np.concatenate(samples)))
    pt = ib.PanelTable(k, union, force_format=fmt)
    for c in samples:
        pt.add_codes(c, len(c), on_device=False)
    info, ns = pt.info()
    assert ns == n_samples
    assert info.format == (fmt or 3)
    # masks against set membership
    rng = np.random.default_rng(3)
    q = np.concatenate([rng.choice(np.concatenate(samples), 20_000), corpus.random_codes(rng, 20_000, k)])
    masks = pt.probe(q)
    want = np.zeros(len(q), np.uint32)
    for i, c in enumerate(samples):
        want |= np.isin(q, c).astype(np.uint32) << np.uint32(i)
    assert np.array_equal(masks, want)
    ref = ib.Reference(seq, mask, ref_spec.lens)
    W = 5000
    panel = pt.scan(ref, W)
    import torch
    n = ib.window_count(ref_spec.lens, W, k)
    dev = torch.zeros(max(n * ns, 1) * 6, dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    for _ in range(3):  # capture, then graph replays
        dev.zero_()
        pt.scan_async(ref, W, dev.data_ptr(), n * ns, st.cuda_stream)
        st.synchronize()
        again = dev[: n * ns * 6].cpu().numpy().view(ib.WINDOW_DTYPE).reshape(ns, n)
        assert np.array_equal(again, panel)
    for i, c in enumerate(samples):
        t = ib.Table.from_codes(c, len(c), k, on_device=False)
        single = ib.scan(t, ref, W)
        assert np.array_equal(panel[i], single), f"sample {i}"
        t.close()
    pt.close()


def test_panel_from_kmc_matches_goldens(build_case):
    names = ["edge_k25", "edge_k25_kmc1", "plain_1mbp"]
    cases = [build_case(n) for n in names]
    ixs = [orc.Index(str(c["prefix"])) for c in cases]
    union = len(np.unique(np.concatenate([ix.list_codes() for ix in ixs])))
    pt = ib.PanelTable(25, union, keys_per_bucket=4.5)  # a dense table: the stash is used
    for c in cases:
        pt.add_kmc(str(c["prefix"]))
    # each golden case's reference against the whole panel: its own sample's rows match its golden
    for i, (name, c) in enumerate(zip(names, cases)):
        gold = corpus.load_golden(name)
        ids, seqs = orc.read_sequence_file(str(c["ref"]))
        seq, mask, lens = ib.pack_ascii(seqs)
        ref = ib.Reference(seq, mask, lens)
        W = c["windows"][0]
        rows = pt.scan(ref, W)
        assert orc.tsv_text(ids, [len(s) for s in seqs], rows[i], W, 25) == gold["tsv"][str(W)]
        for j, ix in enumerate(ixs):
            assert np.array_equal(rows[j], orc.scan(ix, seqs, W, 25, threads=4))
    pt.close()


def test_panel_stash_grows_when_keys_exceed_the_estimate():
    ref_spec = ib.RefSpec(seed=78, lens=[300_000, 50_000], n_frac=0.002, n_run=(1, 100))
    seq, mask = ref_spec.reference_host()
    samples = _samples(ref_spec, seq, mask, 4, k=15)  # k=15: no minimum bucket count
    union = len(np.unique(np.concatenate(samples)))
    pt = ib.PanelTable(15, union // 12)  # ~36 keys per 5-slot bucket: most keys overflow
    first = pt.info()[0].stash_buckets
    for c in samples:
        pt.add_codes(c, len(c), on_device=False)
    info, ns = pt.info()
    assert info.stash_buckets > first
    rng = np.random.default_rng(4)
    q = np.concatenate([np.concatenate(samples), corpus.random_codes(rng, 20_000, 15)])
    want = np.zeros(len(q), np.uint32)
    for i, c in enumerate(samples):
        want |= np.isin(q, c).astype(np.uint32) << np.uint32(i)
    assert np.array_equal(pt.probe(q), want)
    ref = ib.Reference(seq, mask, ref_spec.lens)
    panel = pt.scan(ref, 5000)
    for i, c in enumerate(samples):
        t = ib.Table.from_codes(c, len(c), 15, on_device=False)
        assert np.array_equal(panel[i], ib.scan(t, ref, 5000)), f"sample {i}"
        t.close()
    pt.close()


def test_panel_scan_in_bucket_range_passes_equals_one_pass():
    # a joint table scanned in several bucket-range passes (the masks of
    # each pass kept per position) gives the one-pass rows
    ref_spec = ib.RefSpec(seed=79, lens=[400_000, 90_000, 24], n_frac=0.003, n_run=(1, 200))
    seq, mask = ref_spec.reference_host()
    samples = _samples(ref_spec, seq, mask, 16)
    union = len(np.unique(np.concatenate(samples)))
    pt = ib.PanelTable(25, union)
    for c in samples:
        pt.add_codes(c, len(c), on_device=False)
    ref = ib.Reference(seq, mask, ref_spec.lens)
    one = pt.scan(ref, 5000)
    nbytes = pt.info()[0].n_buckets * 32
    assert nbytes > 3 << 20
    t = ib.get_tuning()
    t.panel_pass_mb = 1  # several passes over this table
    ib.set_tuning(t)
    try:
        many = pt.scan(ref, 5000)
        import torch
        n = ib.window_count(ref_spec.lens, 5000, 25)
        dev = torch.zeros(n * 16 * 6, dtype=torch.int32, device="cuda")
        st = torch.cuda.Stream()
        for _ in range(2):  # captured, then replayed
            pt.scan_async(ref, 5000, dev.data_ptr(), n * 16, st.cuda_stream)
            st.synchronize()
            assert np.array_equal(dev.cpu().numpy().view(ib.WINDOW_DTYPE).reshape(16, n), one)
    finally:
        t.panel_pass_mb = 0xffffffff
        ib.set_tuning(t)
    assert ib.get_tuning().panel_pass_mb == 0
    assert np.array_equal(many, one)
    pt.close()
    ref.free()


@pytest.mark.parametrize("serial", [False, True])
def test_dense_minimizer_line_panel_uses_partner_sectors_and_stash(serial):
    """A crowded joint minimizer-line table (k = 20: a small minimum line
    count, 4 keys per 5-slot sector): full sectors send keys to their
    partner sector and the stash; masks, panel rows and served rows still
    equal set membership and single-sample scans."""
    k, W = 20, 3000
    ref_spec = ib.RefSpec(seed=81, lens=[250_000, 60_000, 19, 20], n_frac=0.002, n_run=(1, 100))
    seq, mask = ref_spec.reference_host()
    samples = _samples(ref_spec, seq, mask, 16, k=k)
    union = len(np.unique(np.concatenate(samples)))
    pt = ib.PanelTable(k, union, keys_per_bucket=4.0, force_format=7)
    for c in samples:
        pt.add_codes(c, len(c), on_device=False)
    info, ns = pt.info()
    assert info.format == 7 and info.stash_buckets > 0
    rng = np.random.default_rng(5)
    q = np.concatenate([np.concatenate(samples), corpus.random_codes(rng, 20_000, k)])
    want = np.zeros(len(q), np.uint32)
    for i, c in enumerate(samples):
        want |= np.isin(q, c).astype(np.uint32) << np.uint32(i)
    assert np.array_equal(pt.probe(q), want)
    ref = ib.Reference(seq, mask, ref_spec.lens)
    panel = pt.scan(ref, W)
    singles = []
    for i, c in enumerate(samples):
        t = ib.Table.from_codes(c, len(c), k, on_device=False)
        singles.append(ib.scan(t, ref, W))
        assert np.array_equal(panel[i], singles[i]), f"sample {i}"
        t.close()
    # the same table served: whole contigs for every sample, batched or one per launch
    srv = ib.Server(ref, W, k, one_request_per_launch=serial)
    assert srv.add_panel(pt, release=True) == list(range(16))
    pt.close()
    reqs = [(s, c, 0, 0) for s in range(16) for c in range(len(ref_spec.lens))]
    for r in reqs:
        srv.submit(*r)
    done = []
    import time
    deadline = time.time() + 300
    while len(done) < len(reqs) and time.time() < deadline:
        done += srv.poll(64, timeout_ms=2000)
    assert len(done) == len(reqs), srv.stats()
    starts = np.concatenate([[0], np.cumsum([ib.window_count(ref_spec.lens[c:c + 1], W, k)
                                             for c in range(len(ref_spec.lens))])])
    for r in done:
        assert r["status"] == 0
        a = starts[r["contig"]]
        assert np.array_equal(r["rows"], singles[r["sample"]][a:a + r["n_windows"]]), (r["sample"], r["contig"])
    srv.close()
    ref.free()
