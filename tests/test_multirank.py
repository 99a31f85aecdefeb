"""The N-GPU path of bench.py on CPU ranks (gloo, world size 2): every rank
scans its own sample (distinct seeds, same workload shape) and the reported
time is the maximum over ranks; no collective touches the scan's data."""
import os
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def torch_sum(dist, value):
    import torch
    t = torch.tensor([value], dtype=torch.float64)
    dist.all_reduce(t)
    return int(t.item())


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "gpu-ibs_b200", "python"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    import bench
    from ibs_b200 import configs
    w = configs.plain_1mbp()
    smp = bench.sample_for_rank(w, rank)
    seed = int(smp.c.seed)
    # every rank's elapsed time differs; the reported one is the maximum
    got = bench.max_over_ranks(10.0 + rank, dist)
    # a rank's sample: same shape, its own seed; the rank writes its own
    # database and scans the whole reference against it (the oracle stands in
    # for the device scan on these CPU ranks); nothing is exchanged but the
    # timing and the probe count
    import tempfile
    import numpy as np
    import ibs_b200 as ib
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as orc
    seq, mask = w.ref.reference_host()
    codes = smp.codes_host(w.ref, seq, mask)
    n = len(np.unique(codes))
    with tempfile.TemporaryDirectory() as d:
        ib.kmc_write(os.path.join(d, "s"), codes, len(codes), **w.kmc)
        seqs = [w.ref.contig_ascii(c) for c in range(len(w.ref.lens))]
        rows = orc.scan(orc.Index(os.path.join(d, "s")), seqs, w.window, w.k, threads=2)
    observed = int(rows["observed_kmers"].astype(np.int64).sum())
    probes = bench.valid_positions(w.ref.lens, w.k, w.ref.n_runs())
    total = torch_sum(dist, probes)
    q.put((rank, seed, got, n, observed, total))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_weak_scaling():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    (r0, s0, t0, n0, o0, p0), (r1, s1, t1, n1, o1, p1) = res
    assert s0 != s1                     # different samples
    assert t0 == t1 == 11.0             # max over ranks
    assert abs(n0 - n1) / n0 < 0.05     # same workload shape
    assert o0 != o1 and o0 > 0 and o1 > 0  # each rank scanned its own sample
    assert p0 == p1 > 0                 # whole-job probes: the sum over ranks of the same reference's positions
