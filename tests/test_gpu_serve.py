"""The serving loop: every request's rows equal the same windows of a full
single-sample scan, alone and in a concurrent mix, with tables evicted and
reloaded under a memory budget."""
import threading
import time

import numpy as np
import pytest

import ibs_b200 as ib

pytestmark = pytest.mark.gpu

W, K = 5000, 25


@pytest.fixture(scope="module")
def world():
    ref_spec = ib.RefSpec(seed=321, lens=[3_000_000, 1_500_000, 700_000, 24, 0, 250_000], n_frac=0.002,
                          n_run=(1, 300))
    seq, mask = ref_spec.reference_host()
    ref = ib.Reference(seq, mask, ref_spec.lens)
    samples = []
    for s in range(6):
        smp = ib.SampleSpec(seed=500 + s, k=K, class_rate=(0.0001, 0.005, 0.02, 0.05),
                            class_prob=(0.2, 0.4, 0.3, 0.1), block_len=50_000, present_frac=0.4 + 0.1 * s,
                            random_frac=0.05)
        samples.append(smp.codes_host(ref_spec, seq, mask))
    # the full single-sample scans, alone
    full = []
    for c in samples:
        t = ib.Table.from_codes(c, len(c), K, on_device=False)
        full.append(ib.scan(t, ref, W))
        t.close()
    starts = np.concatenate([[0], np.cumsum([ib.window_count(ref_spec.lens[:i + 1], W, K) -
                                             ib.window_count(ref_spec.lens[:i], W, K)
                                             for i in range(len(ref_spec.lens))])])
    yield dict(ref=ref, ref_spec=ref_spec, samples=samples, full=full, starts=starts)
    ref.free()


def expected(world, r):
    rows = world["full"][r["sample"]]
    a = world["starts"][r["contig"]] + r["first_window"]
    return rows[a:a + r["n_windows"]]


def make_server(world, budget_tables=2.5, table_format=0, serial=False, iteration_launches=False,
                idle_exit_us=0):
    sizes = [ib.table_bytes_for(len(c), K, force_format=table_format) for c in world["samples"]]
    budget = int(max(sizes) * budget_tables)
    srv = ib.Server(world["ref"], W, K, memory_budget=budget, max_spans_per_launch=512, min_spans_per_request=8,
                    table_format=table_format, one_request_per_launch=serial,
                    iteration_launches=iteration_launches, idle_exit_us=idle_exit_us)
    ids = [srv.add_codes(c, len(c), on_device=False) for c in world["samples"]]
    assert ids == list(range(len(world["samples"])))
    return srv


def random_requests(world, n, seed):
    rng = np.random.default_rng(seed)
    lens = world["ref_spec"].lens
    reqs = []
    for _ in range(n):
        c = int(rng.integers(0, len(lens)))
        nw = ib.window_count(lens[c:c + 1], W, K)
        first = int(rng.integers(0, max(nw, 1)))
        cnt = int(rng.integers(1, max(nw - first, 1) + 1)) if nw else 0
        reqs.append((int(rng.integers(0, len(world["samples"]))), c, first, cnt))
    return reqs


def test_requests_alone_equal_full_scan_rows(world):
    srv = make_server(world)
    for req in random_requests(world, 25, 1):
        srv.submit(*req)
        got = srv.poll(1, timeout_ms=60_000)
        assert len(got) == 1, ("no result within 60 s", req, srv.stats())
        (r,) = got
        assert r["status"] == 0
        assert np.array_equal(r["rows"], expected(world, r)), req
    srv.close()


@pytest.mark.parametrize("iteration_launches", [False, True])
def test_requests_in_a_concurrent_mix_equal_full_scan_rows(world, iteration_launches):
    """Batched serving, through the persistent launch (default) and through
    one launch per loop iteration."""
    srv = make_server(world, budget_tables=2.2, iteration_launches=iteration_launches)
    reqs = random_requests(world, 300, 2) + [(s, 0, 0, 0) for s in range(6)]  # whole-contig requests too
    done = []

    def producer():
        rng = np.random.default_rng(9)
        for req in reqs:
            srv.submit(*req)
            time.sleep(float(rng.exponential(0.0005)))

    th = threading.Thread(target=producer)
    th.start()
    deadline = time.time() + 300
    while len(done) < len(reqs) and time.time() < deadline:
        done += srv.poll(64, timeout_ms=2000)
    th.join()
    assert len(done) == len(reqs), ("requests left unfinished", srv.stats())
    for r in done:
        assert r["status"] == 0
        assert np.array_equal(r["rows"], expected(world, r)), (r["sample"], r["contig"], r["first_window"])
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["evictions"] > 0 and st["reloads"] > 0, st
    assert st["latency_p99"] >= st["latency_p50"] > 0
    if iteration_launches:
        assert st["persistent_launches"] == 0
    else:
        # the whole burst went through a few resident launches, not one per iteration
        assert 1 <= st["persistent_launches"] < st["launches"], st
        assert st["wait_timeouts"] == 0, st
    srv.close()


def test_persistent_launch_ends_when_idle_and_comes_back(world):
    """The persistent kernel's wait for new work is bounded: with no request
    for longer than idle_exit_us the kernel ends by itself (the bound runs
    out and the kernel reports it), and the next request launches it again;
    results stay exact across the restarts."""
    srv = make_server(world, idle_exit_us=2000)
    # requests on contigs with windows (a request on the empty contig completes
    # at submission, without a launch)
    reqs = [r for r in random_requests(world, 12, 21) if world["ref_spec"].lens[r[1]] > 0][:6]
    for i, req in enumerate(reqs):
        srv.submit(*req)
        got = srv.poll(1, timeout_ms=60_000)
        assert len(got) == 1 and got[0]["status"] == 0, (req, srv.stats())
        assert np.array_equal(got[0]["rows"], expected(world, got[0])), req
        time.sleep(0.05)  # 25x the idle limit: the kernel has ended
        st = srv.stats()
        assert st["idle_exits"] == st["persistent_launches"] >= i + 1, st  # every launch ended idle
    st = srv.stats()
    assert st["wait_timeouts"] == 0, st
    srv.close()


def test_persistent_launch_batches_larger_than_its_grid(world):
    """Batches of more span tickets than the persistent grid has warps (every
    contig of every sample at once, all tables resident, no cap on the spans
    of a batch): warps go round for further tickets while others wait, and
    a warp that stamps its work while another reads the clock must not make
    the launch look idle. Every batch finishes in its first launch (no
    replay, no idle end before the stream is done), rows exact."""
    lens = world["ref_spec"].lens
    sizes = [ib.table_bytes_for(len(c), K) for c in world["samples"]]
    srv = ib.Server(world["ref"], W, K, memory_budget=int(sum(sizes) * 1.3))
    for c in world["samples"]:
        srv.add_codes(c, len(c), on_device=False)
    reqs = []
    for rnd in range(3):
        for s in range(len(world["samples"])):
            for c in range(len(lens)):
                nw = ib.window_count(lens[c:c + 1], W, K)
                if nw:
                    reqs.append((s, c, 0, nw))
    for req in reqs:
        srv.submit(*req)
    done, deadline = [], time.time() + 300
    while len(done) < len(reqs) and time.time() < deadline:
        done += srv.poll(64, timeout_ms=2000)
    st = srv.stats()
    assert len(done) == len(reqs), ("requests left unfinished", st)
    for r in done:
        assert r["status"] == 0
        assert np.array_equal(r["rows"], expected(world, r)), (r["sample"], r["contig"])
    # two span items per 5 kbp window: about 13,000 per round of requests
    assert st["persistent_launches"] >= 1 and st["spans"] >= 10_000, st
    assert st["replays"] == 0 and st["wait_timeouts"] == 0 and st["lookup_failures"] == 0, st
    srv.close()


@pytest.mark.parametrize("table_format,serial", [(4, False), (4, True), (6, False)])
def test_minimizer_tables_alone_and_in_a_mix(world, table_format, serial):
    """The server's single-sample tables in the minimizer-line layouts (MZ8,
    MZ6), one request per launch or batched, under a budget that forces
    evictions: every row equals the full scan's."""
    srv = make_server(world, budget_tables=2.2, table_format=table_format, serial=serial)
    for req in random_requests(world, 8, 11):
        srv.submit(*req)
        got = srv.poll(1, timeout_ms=60_000)
        assert len(got) == 1, ("no result within 60 s", req, srv.stats())
        assert got[0]["status"] == 0
        assert np.array_equal(got[0]["rows"], expected(world, got[0])), req
    reqs = random_requests(world, 120, 12) + [(s, 0, 0, 0) for s in range(6)]
    for req in reqs:
        srv.submit(*req)
    done, deadline = [], time.time() + 300
    while len(done) < len(reqs) and time.time() < deadline:
        done += srv.poll(64, timeout_ms=2000)
    assert len(done) == len(reqs), ("requests left unfinished", srv.stats())
    for r in done:
        assert r["status"] == 0
        assert np.array_equal(r["rows"], expected(world, r)), (r["sample"], r["contig"], r["first_window"])
    st = srv.stats()
    assert st["evictions"] > 0 and st["reloads"] > 0, st
    assert st["sample_probes"] == st["scanned"]  # single-sample tables: one sample per scanned position
    srv.close()


def make_panel_server(world, serial=False, force_format=0):
    """The six samples as one joint panel table (the library's layout for k,
    or force_format), plus sample 0 once more as a single-sample table (id
    6), in one server."""
    union = len(np.unique(np.concatenate(world["samples"])))
    pt = ib.PanelTable(K, union, force_format=force_format)
    if force_format:
        assert pt.info()[0].format == force_format
    for c in world["samples"]:
        pt.add_codes(c, len(c), on_device=False)
    srv = ib.Server(world["ref"], W, K, one_request_per_launch=serial)
    ids = srv.add_panel(pt, release=serial)  # either way the server keeps its own copy
    if serial:
        with pytest.raises(ib.IbsError) as e:
            pt.probe(world["samples"][0][:10])
        assert e.value.status == 9
    pt.close()
    assert ids == list(range(6))
    c = world["samples"][0]
    assert srv.add_codes(c, len(c), on_device=False) == 6
    return srv


def expected_any(world, r):
    s = r["sample"] if r["sample"] < 6 else 0
    rows = world["full"][s]
    a = world["starts"][r["contig"]] + r["first_window"]
    return rows[a:a + r["n_windows"]]


@pytest.mark.parametrize("serial,force_format", [(False, 0), (True, 0), (False, 3), (True, 3)])
def test_panel_server_alone_and_in_a_mix(world, serial, force_format):
    """Lone requests (one sample per work item: the lane-parallel fold) and
    overlapping bursts (several samples per item) over a joint table, in the
    minimizer-line layout (the default for k = 25) and in hash sectors."""
    srv = make_panel_server(world, serial, force_format)
    # alone
    for req in random_requests(world, 10, 3):
        srv.submit(*req)
        got = srv.poll(1, timeout_ms=60_000)
        assert len(got) == 1, ("no result within 60 s", req, srv.stats())
        assert got[0]["status"] == 0
        assert np.array_equal(got[0]["rows"], expected_any(world, got[0])), req
    # a burst that overlaps heavily: every sample (and the single-table copy) over the same regions
    reqs = [(s, c, 0, 0) for c in (0, 1, 5) for s in range(7)] + random_requests(world, 60, 4)
    for req in reqs:
        srv.submit(*req)
    done, deadline = [], time.time() + 300
    while len(done) < len(reqs) and time.time() < deadline:
        done += srv.poll(64, timeout_ms=2000)
    assert len(done) == len(reqs), ("requests left unfinished", srv.stats())
    for r in done:
        assert r["status"] == 0
        assert np.array_equal(r["rows"], expected_any(world, r)), (r["sample"], r["contig"], r["first_window"])
    st = srv.stats()
    assert st["sample_probes"] >= st["scanned"]
    if serial:
        assert st["scanned"] == st["probes"]  # one request per launch: nothing shared
    else:
        assert st["scanned"] < st["probes"]  # windows shared between requests were scanned once
    srv.close()
