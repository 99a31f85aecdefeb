"""ibs_scan_noalloc, the allocation-free scan, against ibs_scan.

Some callers cannot allocate device memory while they scan (a server whose
device memory belongs to its own pool, a host that fixes its allocations at
start-up, a latency-bound loop that cannot afford cudaMalloc's implicit
synchronization). ibs_scan_noalloc serves them with scratch in a fixed
device array inside the library. This file is collected last so that a run
stopping at its first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import ibs_b200 as ib
import oracle as orc

pytestmark = pytest.mark.gpu


def _device_inputs(seqs):
    import torch
    seq, mask, lens = ib.pack_ascii(seqs)
    dseq = torch.from_numpy(seq.view(np.int64)).cuda()
    dmask = torch.from_numpy(mask.view(np.int64)).cuda()
    return seq, mask, lens, dseq, dmask


@pytest.mark.parametrize("name,W,fmt", [("plain_1mbp", 50000, 0), ("edge_k25", 5000, 0), ("edge_k15", 100, 0),
                                        ("edge_k32", 1000, 0), ("edge_k25", 5000, 4), ("edge_k31", 5000, 6)])
def test_noalloc_matches_scan_twice(name, W, fmt, build_case):
    import torch
    case = build_case(name)
    table = ib.Table.open(str(case["prefix"]), force_format=fmt)  # 4, 6: minimizer tables
    ids, seqs = orc.read_sequence_file(str(case["ref"]))
    seq, mask, lens, dseq, dmask = _device_inputs(seqs)
    ref = ib.Reference(seq, mask, lens)
    want = ib.scan(table, ref, W)  # the existing entry point
    n = len(want)
    stream = torch.cuda.Stream()
    for call in range(2):  # two calls in a row share (and reuse) the fixed scratch
        rows = torch.full((max(n, 1) * 6,), -7, dtype=torch.int32, device="cuda")
        ib.scan_noalloc(table, dseq, dmask, lens, W, rows, n, stream.cuda_stream)
        stream.synchronize()
        got = rows[: n * 6].cpu().numpy().view(ib.WINDOW_DTYPE)
        assert np.array_equal(got, want), (name, call)
    ref.free()
    table.close()


def test_noalloc_rejects_scans_beyond_its_scratch(build_case):
    import torch
    case = build_case("edge_k25")
    table = ib.Table.open(str(case["prefix"]))
    tiny = torch.zeros(4, dtype=torch.int64, device="cuda")
    rows = torch.zeros(6, dtype=torch.int32, device="cuda")
    # 20 Gbp of contigs at W=100: far more span summaries than the fixed
    # scratch holds; refused on the host before any device access, ahead of
    # the row-capacity check (the honest capacity of `rows` is one row)
    lens = np.full(10, 2_000_000_000, dtype=np.uint64)
    with pytest.raises(ib.IbsError) as e:
        ib.scan_noalloc(table, tiny, tiny, lens, 100, rows, 1)
    assert e.value.status == 7  # IBS_ERR_CAPACITY
    assert "fixed maximum" in str(e.value)
    table.close()
