#!/usr/bin/env python3
"""Benchmark of the B200 fastibs window scan (reference k-mer probes/s).

Workload (default plain_2gbp): a seeded 2 Gbp reference in 10 contigs of
100-400 Mbp with 0.5% N runs, scanned in 50 kbp windows against one sample of
~2.2e9 canonical k=25 k-mers (block-divergence copy of the reference plus 10%
random k-mers). Synthetic data stands in for the reference project's
plant-genome inputs, which are not available here.

A step is one scan of the whole reference: every window's row. `value` is
probes/s with the table and the packed reference resident in HBM (CUDA events
on the launching stream, max over ranks); `e2e` is the same metric through the
host-buffer C-ABI call ibs_scan_packed (pinned host reference in, rows out,
copies inside the timed region). With N GPUs every rank scans its own sample
(weak scaling, no collective on the data path).

At N=1 the workload is also written as files (the sample's KMC 3 database,
the whole reference as FASTA; cached in /dev/shm): the table is built from
the database by ibs_open, the reference's own CPU-BATCHED fastibs (built from
its sources into oracle/_ref/) scans the whole reference as the CPU baseline,
the timed rows are compared with its TSV, and this repository's fastibs CLI
(the drop-in) runs on the same files and its TSV is compared byte for byte
(`parity`, `e2e_cli`).

--impl reference times the reference's CPU-BATCHED fastibs on all host
cores, one contig of the same workload per step; --prepare only writes the
input files (the reference arm runs it as a separate process when they are
missing).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "gpu-ibs_b200" / "python"))

BYTES_PER_PROBE = 32.0 + 0.375  # one 32-byte bucket sector + 2-bit base + N-mask bit
METRIC = "ref k-mer probes/s"
STARTED = time.time()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# workload helpers
# ---------------------------------------------------------------------------
def valid_positions_by_contig(lens, k, runs) -> list[int]:
    """Per contig, the k-mer start positions whose k bases are ACGT (from
    the contig's N runs)."""
    rc, rs, rl = runs
    out = []
    for c, L in enumerate(lens):
        L = int(L)
        npos = max(0, L - k + 1)
        if npos == 0:
            out.append(0)
            continue
        last = npos - 1  # last valid start
        iv = []
        sel = rc == c
        for s, ln in zip(rs[sel].tolist(), rl[sel].tolist()):
            x, y = max(0, s - k + 1), min(last, s + ln - 1)
            if x <= y:
                iv.append((x, y))
        iv.sort()
        bad, cur = 0, None
        for x, y in iv:
            if cur is None or x > cur[1] + 1:
                if cur:
                    bad += cur[1] - cur[0] + 1
                cur = [x, y]
            else:
                cur[1] = max(cur[1], y)
        if cur:
            bad += cur[1] - cur[0] + 1
        out.append(npos - bad)
    return out


def valid_positions(lens, k, runs) -> int:
    return sum(valid_positions_by_contig(lens, k, runs))


def sample_for_rank(w, rank: int):
    from ibs_b200 import SampleSpec
    s = w.samples[0]
    if rank == 0:
        return s
    c = s.c
    return SampleSpec(seed=int(c.seed) + 7919 * rank, k=int(c.k),
                      class_rate=tuple(c.class_rate)[: c.n_classes],
                      class_prob=tuple(c.class_prob)[: c.n_classes], block_len=int(c.block_len),
                      present_frac=float(c.present_frac), random_frac=float(c.random_frac))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest value over all ranks (every rank calls it, in the same order)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


def profiled_traffic(workload: str, table_format: int):
    """DRAM bytes per scan-kernel launch from the committed ncu summary of
    the kernel this table format runs, if any."""
    kernel = "scan_spans_mz" if table_format == 4 else "scan_spans"
    p = REPO / "profiles" / f"{kernel}_{workload}.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("dram_bytes_per_launch")
        except Exception:
            return None
    return None


# ---------------------------------------------------------------------------
# inputs on disk and the reference's own binary
# ---------------------------------------------------------------------------
REF_FASTIBS = REPO / "oracle" / "_ref" / "fastibs"
OUR_FASTIBS = REPO / "gpu-ibs_b200" / "bin" / "fastibs"
TSV_DTYPE = [("start", "<i8"), ("end", "<i8"), ("total_kmers", "<i8"), ("observed_kmers", "<i8"),
             ("variations", "<i8"), ("kmer_distance", "<i8")]


def cache_dir(w) -> Path:
    root = Path("/dev/shm") if Path("/dev/shm").is_dir() else Path(tempfile.gettempdir())
    return root / f"ibs_bench_{w.name}"


def input_paths(w) -> dict:
    """Where the workload's files live: the sample's KMC 3 database
    (db/sample.kmc_pre/.kmc_suf), the whole reference as one FASTA
    (genome/<workload>_genome.fasta) and each contig as its own FASTA
    (contigs/<contig>_genome.fasta)."""
    d = cache_dir(w)
    return {"root": d, "dbdir": d / "db", "prefix": d / "db" / "sample", "db_stamp": d / "db" / "complete",
            "genome_dir": d / "genome", "genome": d / "genome" / f"{w.name}_genome.fasta",
            "contig_dir": d / "contigs", "contig_stamp": d / "contigs" / "complete"}


def prepare_inputs(w, dcodes_ptr: int, n_codes: int) -> dict:
    """Writes the workload's input files once (kept across runs in the cache
    folder): the KMC 3 database of sample 0 from its codes in device memory,
    the whole-genome FASTA and the per-contig FASTAs. Returns input_paths(w)
    plus the number of distinct k-mers in the database."""
    import ibs_b200 as ib
    p = input_paths(w)
    if not p["db_stamp"].exists():
        p["dbdir"].mkdir(parents=True, exist_ok=True)
        t = time.time()
        written = ib.kmc_write(str(p["prefix"]), dcodes_ptr, n_codes, on_device=True, **w.kmc)
        p["db_stamp"].write_text(str(written))
        log(f"[bench] KMC database of {written} k-mers written in {time.time() - t:.1f} s")
    if not p["genome"].exists():
        p["genome_dir"].mkdir(parents=True, exist_ok=True)
        t = time.time()
        w.ref.write_fasta(str(p["genome"]) + ".partial")
        os.replace(str(p["genome"]) + ".partial", p["genome"])
        log(f"[bench] whole-genome FASTA written in {time.time() - t:.1f} s")
    if not p["contig_stamp"].exists():
        p["contig_dir"].mkdir(parents=True, exist_ok=True)
        text = p["genome"].read_bytes()
        heads = [0] + [m.start() + 1 for m in re.finditer(rb"\n>", text)]
        for i, h in enumerate(heads):
            rec = text[h: heads[i + 1] if i + 1 < len(heads) else len(text)]
            name = rec[1: rec.index(b"\n")].decode()
            (p["contig_dir"] / f"{name}_genome.fasta").write_bytes(rec)
        p["contig_stamp"].write_text(str(len(heads)))
        del text
    p["distinct_kmers"] = int(p["db_stamp"].read_text())
    return p


def prepare_main(args, w) -> int:
    """bench.py --prepare: generate the workload on the device and write its
    input files (a separate process, so that the process timing the
    reference's binary maps none of this repository's libraries)."""
    import torch
    import ibs_b200 as ib
    torch.cuda.set_device(0)
    sw, mw = w.ref.packed_words()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    smp = w.samples[0]
    bound = smp.codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
    dcodes = torch.empty(bound, dtype=torch.int64, device="cuda")
    n = smp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), dcodes.data_ptr(), bound)
    torch.cuda.synchronize()
    p = prepare_inputs(w, dcodes.data_ptr(), n)
    log(f"[prepare] {w.name}: {p['distinct_kmers']} distinct k-mers; files under {p['root']}")
    return 0


PHASES_RE = re.compile(r"Scan phases: setup ([\d.e+-]+) s, read ([\d.e+-]+) s, window ([\d.e+-]+) s, "
                       r"stats ([\d.e+-]+) s, write ([\d.e+-]+) s")


def run_fastibs(binary: Path, dbdir: Path, refdir: Path, outdir: Path, W: int, extra=(), env=None):
    """One run of a fastibs CLI (the reference's, or this repository's
    drop-in) over every reference file in refdir; returns the wall seconds,
    the per-reference 'Scan phases' (keyed by the reference name the CLI
    prints) and stdout."""
    shutil.rmtree(outdir, ignore_errors=True)
    t0 = time.perf_counter()
    r = subprocess.run([str(binary), str(dbdir), str(refdir), str(outdir), str(W), *extra],
                       env=env, capture_output=True, text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{binary.name} failed ({r.returncode}): {r.stdout[-800:]} {r.stderr[-800:]}")
    phases, cur = {}, None
    for line in r.stdout.splitlines():
        m = re.match(r"Processing reference: (\S+)", line)
        if m:
            cur = m.group(1)
        m = PHASES_RE.search(line)
        if m and cur:
            phases[cur] = dict(zip(("setup", "read", "window", "stats", "write"), map(float, m.groups())))
    return wall, phases, r.stdout


def reference_env(threads: int) -> dict:
    return dict(os.environ, FASTIBS_THREADS=str(threads), FASTIBS_CPU_BATCH="16")


def tsv_rows(path: Path):
    """(seqname column, numeric rows) of a fastibs TSV."""
    lines = path.read_bytes().split(b"\n")
    assert lines[0] == b"seqname\tstart\tend\ttotal_kmers\tobserved_kmers\tvariations\tkmer_distance"
    body = [ln.split(b"\t") for ln in lines[1:] if ln]
    names = [f[0] for f in body]
    nums = np.array([tuple(int(x) for x in f[1:]) for f in body], dtype=TSV_DTYPE)
    return names, nums


def rows_equal_tsv(rows, nums) -> bool:
    if len(rows) != len(nums):
        return False
    return all(np.array_equal(rows[f].astype(np.int64), nums[f]) for f in rows.dtype.names)


def sha256_file(path: Path) -> str:
    import hashlib
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for b in iter(lambda: f.read(1 << 24), b""):
            h.update(b)
    return h.hexdigest()


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def reference_cpu_run(w, p: dict, threads: int) -> dict:
    """The reference's CPU-BATCHED fastibs over the whole reference (one
    FASTA of every contig) against the sample's KMC database: its TSV and its
    own phase timings."""
    out = p["root"] / "ref_out"
    wall, phases, _ = run_fastibs(REF_FASTIBS, p["dbdir"], p["genome_dir"], out, w.window,
                                  ("--cpu", "--probe=batched"), env=reference_env(threads))
    tsv = out / f"db_v_{w.name}_{w.window}.tsv"
    return {"wall_s": wall, "phases": phases[w.name], "tsv": tsv}


def reference_check(w, tag: str, sample: int, contig: int, dcodes_ptr: int, n_codes: int, rows) -> dict:
    """Rows of one sample over one contig against the reference's own
    CPU-BATCHED fastibs on the same inputs: the sample's KMC database and the
    contig's FASTA are written (cached), the reference scans the contig, and
    its TSV is compared with `rows` (that contig's rows of the sample)."""
    import ibs_b200 as ib
    d = cache_dir(w) / f"check_{tag}_s{sample}_c{contig}"
    (d / "db").mkdir(parents=True, exist_ok=True)
    (d / "refs").mkdir(parents=True, exist_ok=True)
    stamp = d / "db" / "complete"
    if not stamp.exists():
        stamp.write_text(str(ib.kmc_write(str(d / "db" / "sample"), dcodes_ptr, n_codes, on_device=True,
                                          **w.kmc)))
    name = w.ref.names[contig]
    fa = d / "refs" / f"{name}_genome.fasta"
    if not fa.exists():
        seq = w.ref.contig_ascii(contig)
        with open(str(fa) + ".partial", "wb") as fh:
            fh.write(b">" + name.encode() + b"\n")
            for j in range(0, len(seq), 80):
                fh.write(seq[j:j + 80] + b"\n")
        os.replace(str(fa) + ".partial", fa)
    threads = os.cpu_count() or 1
    wall, phases, _ = run_fastibs(REF_FASTIBS, d / "db", d / "refs", d / "out", w.window,
                                  ("--cpu", "--probe=batched"), env=reference_env(threads))
    _, nums = tsv_rows(d / "out" / f"db_v_{name}_{w.window}.tsv")
    equal = rows_equal_tsv(rows, nums)
    return {"status": "bit-exact" if equal else "MISMATCH", "sample": sample, "contig": name,
            "sample_kmers": int(stamp.read_text()), "windows": int(len(nums)),
            "against": "oracle/_ref/fastibs --cpu --probe=batched on this sample's KMC database and this "
                       "contig's FASTA", "reference_wall_s": wall}


def gpu_arm(args, w, rank: int, world: int, local: int):
    import torch
    import ibs_b200 as ib

    torch.cuda.set_device(local)
    dev = local
    k, W = w.k, w.window
    lens = w.ref.lens
    runs = w.ref.n_runs()
    probes_per_scan = valid_positions(lens, k, runs)
    sw, mw = w.ref.packed_words()
    n_win = ib.window_count(lens, W, k)
    files = rank == 0 and world == 1  # the KMC database, FASTA files, CPU baseline and parity

    # random-sector ceiling of this GPU (before the big allocations)
    sector_rate = ib.random_sector_rate(16 << 30) if args.scale >= 0.5 else ib.random_sector_rate(4 << 30)

    # inputs generated on the device
    t0 = time.time()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    smp = sample_for_rank(w, rank)
    bound = smp.codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
    dcodes = torch.empty(bound, dtype=torch.int64, device="cuda")
    n_codes = smp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), dcodes.data_ptr(), bound)
    torch.cuda.synchronize()
    t_gen = time.time() - t0

    # the sample's table: rank 0 of a 1-GPU run decodes the KMC database the
    # reference reads (ibs_open: the .kmc_suf records decoded on the device);
    # the other ranks of a multi-GPU run build theirs from their own codes
    paths = None
    if files:
        paths = prepare_inputs(w, dcodes.data_ptr(), n_codes)
    del dcodes
    torch.cuda.empty_cache()
    t0 = time.time()
    if files:
        table = ib.Table.open(str(paths["prefix"]), device=dev, force_format=args.table_format,
                              keys_per_bucket=args.keys_per_bucket)
    else:
        dcodes = torch.empty(bound, dtype=torch.int64, device="cuda")
        n_codes = smp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), dcodes.data_ptr(), bound)
        table = ib.Table.from_codes(dcodes.data_ptr(), n_codes, k, on_device=True, device=dev,
                                    force_format=args.table_format, keys_per_bucket=args.keys_per_bucket)
        del dcodes
        torch.cuda.empty_cache()
    info = table.info()
    t_build = time.time() - t0
    build_call = "ibs_open (KMC 3 files decoded on the device)" if files else "ibs_table_from_codes"
    log(f"[bench r{rank}] generated {sum(map(int, lens)) / 1e9:.3f} Gbp + {n_codes / 1e9:.3f}e9 codes "
        f"in {t_gen:.1f} s; table of {info.n_keys} k-mers, {info.n_buckets * 32 / 1e9:.2f} GB (format "
        f"{info.format}, {info.stash_keys} stashed) by {build_call} in {t_build:.1f} s")

    # the reference's own CPU-BATCHED scan of the whole reference (its TSV is
    # the parity target of the rows timed below)
    cpu, ref_run = None, None
    if files and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            ref_run = reference_cpu_run(w, paths, threads)
            ph = ref_run["phases"]
            cpu = {"value": probes_per_scan / ph["stats"], "unit": "probes/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"the whole {w.name} workload ({sum(map(int, lens)) / 1e9:g} Gbp in {len(lens)} "
                             f"contigs) against the {paths['distinct_kmers'] / 1e9:.3f}e9-k-mer KMC database: "
                             f"oracle/_ref/fastibs --cpu --probe=batched (CPU-BATCHED), FASTIBS_THREADS={threads}; "
                             f"probes/s = valid positions / the 'stats' phase of its Scan phases line",
                   "phases_s": ph, "wall_s": ref_run["wall_s"]}
            log(f"[bench] reference CPU-BATCHED scan: {ph} (wall {ref_run['wall_s']:.1f} s)")
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "probes/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    ref = ib.Reference(dseq.data_ptr(), dmask.data_ptr(), lens, device=dev, on_device=True)
    rows_dev = torch.empty(max(n_win, 1) * 6, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()

    def step():
        ib.scan_async(table, ref, W, rows_dev.data_ptr(), n_win, stream.cuda_stream)

    # warm-up (allocates the scan plan on the first call)
    for _ in range(args.warmup):
        step()
    stream.synchronize()

    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ib.launch_count()
    with Clocks(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    launches = ib.launch_count() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, "cuda")
    if dist:
        dist.barrier()
    ms_step = ms / args.steps
    total_probes = probes_per_scan * world
    value = total_probes / (ms_step * 1e-3)
    rows = rows_dev[: n_win * 6].cpu().numpy().view(ib.WINDOW_DTYPE)

    # e2e: pinned host reference in, rows out, through ibs_scan_packed
    hseq = dseq.cpu().pin_memory()
    hmask = dmask.cpu().pin_memory()
    hrows = torch.empty(max(n_win, 1) * 6, dtype=torch.int32).pin_memory()
    for _ in range(2):
        ib.scan_packed(table, hseq.data_ptr(), hmask.data_ptr(), lens, W, hrows.data_ptr())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ib.scan_packed(table, hseq.data_ptr(), hmask.data_ptr(), lens, W, hrows.data_ptr())
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, dist, "cuda")
    e2e_rows = hrows[: n_win * 6].numpy().view(ib.WINDOW_DTYPE)
    assert np.array_equal(e2e_rows, rows), "e2e rows differ from the resident scan's"
    h2d = (sw + mw) * 8 + n_win * 32 + (n_win + 1) * 4
    d2h = n_win * 24

    # from FASTA text in host memory: parse + pack on the device, scan, rows
    # back (the fastibs CLI's path for a plain .fasta reference)
    fasta = None
    if files and not args.no_fasta_e2e:
        text = paths["genome"].read_bytes()
        secs, parse = [], []
        for it in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fref = ib.Reference.from_fasta(text, device=dev)
            t1 = time.perf_counter()
            frows = ib.scan(table, fref, W)
            secs.append(time.perf_counter() - t0)
            parse.append(t1 - t0)
            fref.free()
            assert np.array_equal(frows, rows), "rows from the device-parsed FASTA differ"
        best = min(secs[1:])
        fasta = {"value": total_probes / best, "unit": "probes/s", "seconds": best,
                 "seconds_per_call": [round(x, 4) for x in secs], "parse_seconds": [round(x, 4) for x in parse],
                 "fasta_bytes": len(text), "h2d_bytes_per_step": len(text), "d2h_bytes_per_step": int(d2h),
                 "call": "ibs_reference_from_fasta (FASTA bytes in host memory) + ibs_scan (rows to host)"}
        del text
    table_info = {"format": int(info.format), "buckets": int(info.n_buckets), "keys": int(info.n_keys),
                  "fp_bits": int(info.fp_bits), "stash_keys": int(info.stash_keys),
                  "device_gb": info.device_bytes / 1e9, "build_s": t_build, "build_call": build_call}
    table.close()
    ref.free()
    del rows_dev, hseq, hmask, hrows
    torch.cuda.empty_cache()

    # parity at full size: the timed scan's rows against the reference's own
    # TSV, and this repository's fastibs CLI (the drop-in: KMC files and FASTA
    # in, TSV out) byte for byte against it
    parity, cli = None, None
    if ref_run is not None:
        names, nums = tsv_rows(ref_run["tsv"])
        timed_equal = rows_equal_tsv(rows, nums)
        try:
            wall, phases, _ = run_fastibs(OUR_FASTIBS, paths["dbdir"], paths["genome_dir"],
                                          paths["root"] / "our_out", W)
            our_tsv = paths["root"] / "our_out" / ref_run["tsv"].name
            cli_identical = our_tsv.read_bytes() == ref_run["tsv"].read_bytes()
            cli = {"value": total_probes / wall, "unit": "probes/s", "seconds": wall,
                   "phases_s": phases.get(w.name),
                   "call": "gpu-ibs_b200/bin/fastibs <db> <refs> <out> 50000: KMC 3 files and the FASTA file "
                           "in, TSV out (process start to exit)",
                   "reference_seconds": ref_run["wall_s"]}
        except Exception as e:
            cli_identical = False
            cli = {"value": None, "unavailable": str(e)[-400:]}
        parity = {"status": "bit-exact" if timed_equal and cli_identical else "MISMATCH",
                  "against": "the reference's fastibs --cpu --probe=batched TSV of the whole workload",
                  "windows": int(len(nums)), "timed_rows_equal_reference_tsv": bool(timed_equal),
                  "cli_tsv_identical_to_reference_tsv": bool(cli_identical),
                  "tsv_sha256": sha256_file(ref_run["tsv"])}
        log(f"[bench] parity {parity}")

    peak, peak_kind = measured_peaks()
    achieved = probes_per_scan / (ms_step * 1e-3) * BYTES_PER_PROBE / 1e9
    checksum = int(rows["observed_kmers"].astype(np.int64).sum())
    out = {
        "metric": METRIC, "value": value, "unit": "probes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded generator; stands in for plant-genome inputs not available here)",
        "config": {"workload": w.name, "reference_bp": int(sum(map(int, lens))), "contigs": len(lens),
                   "sample_kmers": int(info.n_keys), "k": k, "window": W, "windows": int(n_win),
                   "probes_per_scan": int(probes_per_scan), "parallelism": f"{world} sample(s), one per GPU",
                   "l2": f"inputs larger than L2: {info.n_buckets * 32 / 1e9:.1f} GB table, "
                         f"{(sw + mw) * 8 / 1e9:.2f} GB packed reference"},
        "parity": parity,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": profiled_traffic(w.name, int(info.format)),
                     "bytes_per_probe": BYTES_PER_PROBE,
                     "random_sector_peak": sector_rate * BYTES_PER_PROBE / 1e9,
                     "random_sector_frac": (probes_per_scan / (ms_step * 1e-3)) / sector_rate,
                     "note": "achieved = probes/s x (32 B bucket sector + 0.375 B streamed reference); "
                             "random_sector_peak = live GUPS-style random 32 B reads x the same bytes; "
                             "with the minimizer table (format 4) consecutive probes share 128-byte "
                             "lines, so traffic (DRAM bytes per launch, ncu) sits below the algorithmic "
                             "bytes"},
        "e2e": {"value": total_probes / e2e_s, "unit": "probes/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_s * 1e3,
                "call": "ibs_scan_packed (pinned host 2-bit reference -> host rows)"},
        "e2e_from_fasta": fasta,
        "e2e_cli": cli,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "extra": {"gbp_x_samples_per_s": sum(map(int, lens)) * world / (ms_step * 1e-3) / 1e9,
                  "table": table_info, "generator_codes": int(n_codes),
                  "rows_checksum_observed": checksum, "gen_s": t_gen,
                  "tuning": getattr(args, "tuning_used", None)},
    }
    if cpu is not None:
        out["cpu_baseline"] = cpu
    return out


def panel_arm(args, rank: int):
    """Batched panel: 16 samples of uneven size against one reference, one
    joint table, the scan replayed as a CUDA graph; compared with the plain
    path (one table and one scan launch per sample) on the same GPU, and
    every sample's panel rows checked against its single-sample rows."""
    import torch
    import ibs_b200 as ib
    from ibs_b200 import configs
    if args.panel_workload == "served_2gbp":
        w = configs.served_2gbp(n_samples=args.panel_samples, scale=args.panel_scale)
    else:
        w = configs.panel_4gbp(n_samples=args.panel_samples, scale=args.panel_scale)
    k, W = w.k, w.window
    lens = w.ref.lens
    runs = w.ref.n_runs()
    positions = valid_positions(lens, k, runs)
    sw, mw = w.ref.packed_words()
    n_win = ib.window_count(lens, W, k)
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    ref = ib.Reference(dseq.data_ptr(), dmask.data_ptr(), lens, on_device=True)

    def sample_codes_bound(i):
        return w.samples[i].codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())

    def sample_codes(i):
        smp = w.samples[i]
        bound = sample_codes_bound(i)
        buf = torch.empty(bound, dtype=torch.int64, device="cuda")
        n = smp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), buf.data_ptr(), bound)
        return buf, n

    # the union's size from a 1/64 hash sample of every sample's k-mers
    t0 = time.time()
    sizes, sampled = [], []
    for i in range(len(w.samples)):
        buf, n = sample_codes(i)
        sizes.append(n)
        v = buf[:n]
        sel = v[((v * 0x9E3779B97F4A7C15) >> 58) == 0]
        sampled.append(torch.unique(sel))
        del buf, v, sel
        torch.cuda.empty_cache()
    # plain path: one table and one scan launch per sample (scan time only)
    stream = torch.cuda.Stream()
    rows_single = torch.empty(max(n_win, 1) * 6, dtype=torch.int32, device="cuda")
    singles, plain_ms = [], 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(len(w.samples)):
        buf, n = sample_codes(i)
        t = ib.Table.from_codes(buf.data_ptr(), n, k, on_device=True)
        del buf
        torch.cuda.empty_cache()
        ib.scan_async(t, ref, W, rows_single.data_ptr(), n_win, stream.cuda_stream)  # plan + warm
        stream.synchronize()
        e0.record(stream)
        ib.scan_async(t, ref, W, rows_single.data_ptr(), n_win, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
        singles.append(rows_single[: n_win * 6].cpu().numpy().view(ib.WINDOW_DTYPE).copy())
        t.close()
    del rows_single
    torch.cuda.empty_cache()

    # batched: joint tables of as many samples as fit next to the build's
    # scratch (one sample's codes); all 16 in one table when memory allows
    # joint-table load: the flag, else the library's default for the layout it
    # picks (minimizer lines at 2 keys per sector for 16 <= k <= 27, hash
    # sectors at the tuned load otherwise)
    kpb = args.panel_keys_per_bucket
    kpb_est = kpb or (1.5 if 16 <= k <= 27 else ib.get_tuning().panel_keys_per_bucket)
    free, _ = torch.cuda.mem_get_info()
    max_codes = max(sample_codes_bound(i) for i in range(len(w.samples))) * 8
    rows_bytes = n_win * len(w.samples) * 24 + 64 * n_win * len(w.samples)
    budget = free - max_codes - (2 << 30) * 2 - rows_bytes - (6 << 30)

    union_of = {}

    def joint_bytes(members):
        u = int(torch.unique(torch.cat([sampled[j] for j in members])).numel() * 64 * 1.02) + (1 << 20)
        union_of[tuple(members)] = u
        return u / kpb_est * 32 * 1.15

    groups, cur = [], []
    for i in range(len(w.samples)):
        if cur and joint_bytes(cur + [i]) > budget:
            groups.append(cur)
            cur = []
        cur.append(i)
    groups.append(cur)
    for members in groups:
        joint_bytes(members)
    log(f"[panel] {len(groups)} joint table group(s) {groups} under a {budget / 1e9:.1f} GB budget; "
        f"union estimates {[union_of[tuple(m)] for m in groups]}")
    del sampled
    panel_ms, launches, table_gb, union_est, got = 0.0, 0, [], [], [None] * len(w.samples)
    table_fmt = []
    build_s = 0.0
    for members in groups:
        tb = time.time()
        pt = ib.PanelTable(k, union_of[tuple(members)], keys_per_bucket=kpb)
        for i in members:
            buf, n = sample_codes(i)
            pt.add_codes(buf.data_ptr(), n, on_device=True)
            del buf
            torch.cuda.empty_cache()
        info, ns = pt.info()
        build_s += time.time() - tb
        table_gb.append(info.device_bytes / 1e9)
        table_fmt.append(int(info.format))
        union_est.append(union_of[tuple(members)])
        rows = torch.empty(max(n_win * ns, 1) * 6, dtype=torch.int32, device="cuda")
        for _ in range(args.warmup):
            pt.scan_async(ref, W, rows.data_ptr(), n_win * ns, stream.cuda_stream)
        stream.synchronize()
        launches0 = ib.launch_count()
        e0.record(stream)
        for _ in range(args.steps):
            pt.scan_async(ref, W, rows.data_ptr(), n_win * ns, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        panel_ms += e0.elapsed_time(e1) / args.steps
        launches += ib.launch_count() - launches0
        g = rows[: n_win * ns * 6].cpu().numpy().view(ib.WINDOW_DTYPE).reshape(ns, n_win)
        for j, i in enumerate(members):
            got[i] = g[j].copy()
        del rows
        pt.close()
        torch.cuda.empty_cache()
    t_build = time.time() - t0
    ns = len(w.samples)
    mismatched = [i for i in range(ns) if not np.array_equal(got[i], singles[i])]
    assert not mismatched, f"panel rows differ from single-sample rows for samples {mismatched}"
    # the smallest sample's rows over the shortest contig against the
    # reference's own CPU scan of the same inputs
    win_start = np.concatenate([[0], np.cumsum([ib.window_count(lens[c:c + 1], W, k) for c in range(len(lens))])])
    si = int(np.argmin(sizes))
    ci = int(np.argmin([int(x) for x in lens]))
    ref_check = None
    if REF_FASTIBS.exists() and not args.no_cpu_baseline:
        buf, n = sample_codes(si)
        ref_check = reference_check(w, "panel", si, ci, buf.data_ptr(), n,
                                    got[si][int(win_start[ci]):int(win_start[ci + 1])])
        del buf
        torch.cuda.empty_cache()
    probes = positions * ns
    out = {"workload": w.name, "samples": ns, "sample_kmers": sizes, "k": k, "window": W,
           "reference_bp": int(sum(map(int, lens))), "positions": int(positions),
           "groups": groups, "union_keys_estimate": union_est, "joint_table_gb": table_gb,
           "joint_table_format": table_fmt,
           "keys_per_bucket": kpb_est, "build_s": build_s, "setup_s": t_build,
           "batched_probes_per_s": probes / (panel_ms * 1e-3), "batched_ms_per_scan": panel_ms,
           "plain_probes_per_s": probes / (plain_ms * 1e-3), "plain_ms_all_samples": plain_ms,
           "speedup_vs_plain": plain_ms / panel_ms, "graph_launches_per_scan": launches / args.steps,
           "rows_equal_single_sample": True,
           "parity": {"status": "bit-exact" if ref_check is None or ref_check["status"] == "bit-exact"
                      else "MISMATCH",
                      "single_sample": "every sample's panel rows equal its single-sample scan's rows",
                      "reference": ref_check},
           "note": "batched = joint tables (one per group; one group when all samples fit), each scan a "
                   "replayed CUDA graph; plain = one table and one scan launch per sample; scan time only"}
    ref.free()
    return out


def served_arm(args, rank: int):
    """Served scan stream: a reference and a pool of 16 resident samples
    (served_2gbp by default); Poisson arrivals; each request one sample and a
    region log-uniform from 1 Mbp to a whole contig. The batching server over joint
    panel tables (requests sharing windows are scanned together) against the
    plain path (per-sample tables, one request per launch) on the same GPU.
    Every result is checked against its sample's full-scan rows."""
    import torch
    import ibs_b200 as ib
    from ibs_b200 import configs
    if args.serve_workload == "served_2gbp":
        w = configs.served_2gbp(n_samples=args.serve_samples, scale=args.serve_scale)
    else:
        w = configs.panel_4gbp(n_samples=args.serve_samples, scale=args.serve_scale,
                               sample_scale=args.serve_sample_scale)
    k, W = w.k, w.window
    lens = w.ref.lens
    sw, mw = w.ref.packed_words()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    ref = ib.Reference(dseq.data_ptr(), dmask.data_ptr(), lens, on_device=True)
    n_samples = len(w.samples)
    win_start = np.concatenate([[0], np.cumsum([ib.window_count(lens[c:c + 1], W, k) for c in range(len(lens))])])
    n_win = int(win_start[-1])
    t0 = time.time()

    def codes(i):
        sp = w.samples[i]
        bound = sp.codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
        buf = torch.empty(bound, dtype=torch.int64, device="cuda")
        n = sp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), buf.data_ptr(), bound)
        return buf, n

    # every sample's full-scan rows (to check the served results) and a 1/64
    # hash sample of its k-mers (to size the joint tables)
    full, n_keys, sampled, max_bound = [], [], [], 0
    rows_dev = torch.empty(n_win * 6, dtype=torch.int32, device="cuda")
    for i in range(n_samples):
        buf, n = codes(i)
        max_bound = max(max_bound, buf.numel())
        n_keys.append(n)
        v = buf[:n]
        sampled.append(torch.unique(v[((v * 0x9E3779B97F4A7C15) >> 58) == 0]))
        t = ib.Table.from_codes(buf.data_ptr(), n, k, on_device=True)
        del buf, v
        torch.cuda.empty_cache()
        ib.scan_async(t, ref, W, rows_dev.data_ptr(), n_win, 0)
        torch.cuda.synchronize()
        full.append(rows_dev.cpu().numpy().view(ib.WINDOW_DTYPE).copy())
        t.close()
    del rows_dev
    torch.cuda.empty_cache()
    # the full-scan rows every served row is checked against: one sample's
    # over one contig against the reference's own CPU scan
    si = int(np.argmin(n_keys))
    ci = int(np.argmin([int(x) for x in lens]))
    ref_check = None
    if REF_FASTIBS.exists() and not args.no_cpu_baseline:
        buf, n = codes(si)
        ref_check = reference_check(w, "served", si, ci, buf.data_ptr(), n,
                                    full[si][int(win_start[ci]):int(win_start[ci + 1])])
        del buf
        torch.cuda.empty_cache()
    setup_s = time.time() - t0

    # the request stream
    rng = np.random.default_rng(404)
    reqs = []
    step = W - k
    for _ in range(args.serve_requests):
        s_ = int(rng.integers(0, n_samples))
        c = int(rng.integers(0, len(lens)))
        L = int(lens[c])
        ln = int(np.exp(rng.uniform(np.log(1e6), np.log(max(L, 1e6 + 1)))))
        nw_c = int(win_start[c + 1] - win_start[c])
        first = int(rng.integers(0, max(1, (L - ln) // step + 1)))
        first = min(first, nw_c - 1)
        cnt = max(1, min(nw_c - first, ln // step))
        reqs.append((s_, c, first, cnt))
    unit_gaps = rng.exponential(1.0, len(reqs))  # arrival gaps at 1 req/s, scaled per rate
    rates = [float(x) for x in str(args.serve_rates).split(",") if x]

    def run(srv, rate):
        """rate = None: every request submitted at once (saturated); else
        Poisson arrivals at `rate` per second of the first requests (all of
        them at the highest rate, about args.serve_seconds worth below it)."""
        done = []
        stats0 = srv.stats()
        t_start = srv.now()
        if rate:
            n = len(reqs) if rate == max(rates) else min(len(reqs), max(50, int(rate * args.serve_seconds)))
            t_next = time.perf_counter()
            for req, g in zip(reqs[:n], unit_gaps[:n] / rate):
                t_next += g
                while time.perf_counter() < t_next:
                    try:
                        done += srv.poll(256, timeout_ms=0)
                    except ib.IbsError as e:
                        raise RuntimeError(f"{e}; stats {srv.stats()}") from e
                    time.sleep(0.0002)
                srv.submit(*req)
        else:
            n = len(reqs)
            for req in reqs:
                srv.submit(*req)
        deadline = time.time() + 600
        while len(done) < n and time.time() < deadline:
            done += srv.poll(256, timeout_ms=1000)
        assert len(done) == n, f"served requests unfinished: {srv.stats()}"
        makespan = srv.now() - t_start
        log(f"[served] rate {rate}: {n} requests in {makespan:.1f} s; stats {srv.stats()}")
        st = srv.stats()
        lat = np.array([r["done_time"] - r["submit_time"] for r in done])
        for r in done:
            assert r["status"] == 0, "a served request failed"
            a = int(win_start[r["contig"]] + r["first_window"])
            assert np.array_equal(r["rows"], full[r["sample"]][a:a + int(r["n_windows"])]), "served rows differ"
        probes = st["probes"] - stats0["probes"]
        busy = st["busy_seconds"] - stats0["busy_seconds"]
        sp = st["sample_probes"] - stats0["sample_probes"]
        return {"requests": n, "arrival_rate_per_s": rate, "probes": int(probes),
                "scanned": int(st["scanned"] - stats0["scanned"]), "sample_probes_computed": int(sp),
                "makespan_s": makespan, "probes_per_s": probes / makespan,
                "device_busy_s": busy, "probes_per_device_s": probes / max(busy, 1e-9),
                "sample_probes_per_device_s": sp / max(busy, 1e-9),
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_max_s": float(lat.max()), "launches": int(st["launches"] - stats0["launches"]),
                "reloads": int(st["reloads"] - stats0["reloads"]),
                "reload_bytes": int(st["reload_bytes"] - stats0["reload_bytes"]),
                "rows_equal_full_scan": True}

    out = {"workload": f"{w.name} reference x {n_samples} resident samples", "k": k, "window": W,
           "reference_bp": int(sum(map(int, lens))), "sample_kmers": n_keys, "requests": len(reqs),
           "arrival_rates_per_s": rates, "region": "log-uniform 1 Mbp .. whole contig",
           "setup_s": setup_s}

    # plain path: per-sample tables in the plain scan's layout (minimizer
    # lines at the tuned load), one request per launch. The budget leaves
    # room for registering a sample (its codes and a transient table)
    # single: the same per-sample tables under the batching server (windows
    # shared by pending requests of one sample are scanned once; no joint
    # table), optional
    for mode, serial in (("plain", True), ("single", False)):
        if mode not in args.serve_modes:
            continue
        free, _ = torch.cuda.mem_get_info()
        transient = max_bound * 8 + ib.table_bytes_for(max(n_keys), k) * 2 + (4 << 30)
        srv = ib.Server(ref, W, k, memory_budget=int(free - transient), one_request_per_launch=serial)
        for i in range(n_samples):
            buf, n = codes(i)
            srv.add_codes(buf.data_ptr(), n, on_device=True)
            del buf
            torch.cuda.empty_cache()
        out[f"{mode}_tables_gb"] = srv.stats()["resident_bytes"] / 1e9
        for r in rates:
            out[f"{mode}_poisson_{r:g}"] = run(srv, r)
        out[f"{mode}_saturated"] = run(srv, None)
        srv.close()
        torch.cuda.empty_cache()
    if "batched" not in args.serve_modes:
        return out

    # batched: joint panel tables (as many samples per table as memory allows)
    # joint-table load: the flag, else the library's default for the layout it
    # picks (minimizer lines at 2 keys per sector for 16 <= k <= 27, hash
    # sectors at the tuned load otherwise)
    kpb = args.panel_keys_per_bucket
    kpb_est = kpb or (1.5 if 16 <= k <= 27 else ib.get_tuning().panel_keys_per_bucket)
    free, _ = torch.cuda.mem_get_info()
    budget = free - max_bound * 8 - (4 << 30) - (8 << 30)
    union_of = {}

    def joint_bytes(members):
        u = int(torch.unique(torch.cat([sampled[j] for j in members])).numel() * 64 * 1.02) + (1 << 20)
        union_of[tuple(members)] = u
        return u / kpb_est * 32 * 1.15

    # a joint table holds as many samples as memory allows, or (--serve-group-gb)
    # as fit under a size cap: a smaller table keeps a lone request's random
    # probes inside the GPU's address-translation reach
    cap = args.serve_group_gb * 1e9 if args.serve_group_gb else float("inf")
    groups, cur = [], []
    for i in range(n_samples):
        if cur and (sum(joint_bytes(g) for g in groups) + joint_bytes(cur + [i]) > budget or
                    joint_bytes(cur + [i]) > cap):
            groups.append(cur)
            cur = []
        cur.append(i)
    groups.append(cur)
    del sampled
    per_iteration = "iterations" in args.serve_modes
    srv = ib.Server(ref, W, k, memory_budget=int(free - max_bound * 8 - (8 << 30)),
                    iteration_launches=per_iteration)
    out["batched_launch"] = "per loop iteration" if per_iteration else "one persistent launch"
    id_of, joint_fmt = {}, []
    for members in groups:
        pt = ib.PanelTable(k, union_of[tuple(members)], keys_per_bucket=kpb)
        for i in members:
            buf, n = codes(i)
            pt.add_codes(buf.data_ptr(), n, on_device=True)
            del buf
            torch.cuda.empty_cache()
        joint_fmt.append(int(pt.info()[0].format))
        for i, sid in zip(members, srv.add_panel(pt, release=True)):
            id_of[i] = sid
        pt.close()
        torch.cuda.empty_cache()
    assert all(id_of[i] == i for i in range(n_samples))
    out["batched_groups"] = groups
    out["batched_table_format"] = joint_fmt
    out["batched_tables_gb"] = srv.stats()["resident_bytes"] / 1e9
    for r in rates:
        out[f"batched_poisson_{r:g}"] = run(srv, r)
    out["batched_saturated"] = run(srv, None)
    srv.close()
    if "plain" not in args.serve_modes:
        return out
    out["saturated_speedup_vs_plain"] = (out["batched_saturated"]["probes_per_s"] /
                                         out["plain_saturated"]["probes_per_s"])
    out["p99_ratio_batched_over_plain"] = {f"{r:g}": out[f"batched_poisson_{r:g}"]["latency_p99_s"] /
                                           out[f"plain_poisson_{r:g}"]["latency_p99_s"] for r in rates}
    if "single" in args.serve_modes:
        out["single_saturated_speedup_vs_plain"] = (out["single_saturated"]["probes_per_s"] /
                                                    out["plain_saturated"]["probes_per_s"])
        out["p99_ratio_single_over_plain"] = {f"{r:g}": out[f"single_poisson_{r:g}"]["latency_p99_s"] /
                                              out[f"plain_poisson_{r:g}"]["latency_p99_s"] for r in rates}
    out["parity"] = {"status": "bit-exact" if ref_check is None or ref_check["status"] == "bit-exact"
                     else "MISMATCH",
                     "single_sample": "every served row equals the same window of its sample's full "
                                      "single-sample scan",
                     "reference": ref_check}
    out["note"] = ("probes = positions of the completed requests (a window shared by k requests counts k "
                   "times); scanned = positions the device scanned; sample_probes_computed = positions x "
                   "samples the scans answered")
    ref.free()
    return out


def wide_arm(args, rank: int):
    """k > 32 (wide-key tables, the reference's string-path k): the 2 Gbp
    reference scanned against a table of random 128-bit k = 41 keys (4 keys
    per 128-byte line), timed with CUDA events over --steps scans after
    --warmup. Throughput only: the rows of the k > 32 golden cases are
    checked by the tests; here every row's total is checked against the
    valid positions of its window."""
    import ctypes as C
    import torch
    import ibs_b200 as ib
    from ibs_b200 import configs
    w = configs.plain_2gbp(scale=args.scale) if args.scale != 1.0 else configs.plain_2gbp()
    k, W = 41, w.window
    lens = w.ref.lens
    sw, mw = w.ref.packed_words()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    ref = ib.Reference(dseq.data_ptr(), dmask.data_ptr(), lens, on_device=True)
    n = int(args.wide_keys)
    g = torch.Generator(device="cuda").manual_seed(41)
    lo = torch.randint(-2**63, 2**63 - 1, (n,), device="cuda", dtype=torch.int64, generator=g)
    hi = torch.randint(0, 2**(2 * k - 64), (n,), device="cuda", dtype=torch.int64, generator=g)
    codes = torch.stack([lo, hi], 1).contiguous()
    del lo, hi
    opts = ib.TableOpts(0, 0.0, 0)
    h = C.c_void_p()
    t0 = time.time()
    ib._check(ib._ibs_from_codes128(codes.data_ptr(), n, k, 1, C.byref(opts), C.byref(h)))
    build_s = time.time() - t0
    del codes
    torch.cuda.empty_cache()
    t = ib.Table(h.value)
    info = t.info()
    nwin = ib.window_count(lens, W, k)
    rows = torch.zeros(nwin * 6, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    for _ in range(args.warmup):
        ib.scan_async(t, ref, W, rows.data_ptr(), nwin, s.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.steps):
        ib.scan_async(t, ref, W, rows.data_ptr(), nwin, s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    got = rows.cpu().numpy().view(ib.WINDOW_DTYPE)
    bounds = ib.window_bounds(lens, W, k)
    probes = valid_positions(lens, k, w.ref.n_runs())
    t.close()
    ref.free()
    return {"k": k, "keys": n, "table_gb": info.device_bytes / 1e9, "later_level_keys": int(info.stash_keys),
            "build_s": build_s, "ms_per_scan": ms, "probes_per_scan": probes, "probes_per_s": probes / ms * 1e3,
            "bytes_per_probe": 128.375, "windows": int(nwin),
            "rows_consistent": bool(np.array_equal(got["start"], bounds["start"]) and
                                    np.array_equal(got["end"], bounds["end"]) and
                                    int(got["total_kmers"].sum()) >= probes),
            "table": "random keys (the throughput of one 128-byte line per probe; hits do not change it)"}


def admitted_arm(args, rank: int):
    """Memory-admitted serving beyond the device's share: 48 samples whose
    tables total about 3x the server's byte budget, Zipf(1.1) popularity,
    whole-genome (every contig) and regional requests. The batching server
    against one request per launch, both evicting least-recently-used tables
    and reloading them from pinned host images on a side stream. Every row
    is checked against its sample's full-scan rows."""
    import torch
    import ibs_b200 as ib
    from ibs_b200 import configs
    w = configs.admitted_4gbp(n_samples=args.admit_samples, scale=args.admit_scale,
                              sample_scale=args.admit_sample_scale)
    k, W = w.k, w.window
    lens = w.ref.lens
    sw, mw = w.ref.packed_words()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    ref = ib.Reference(dseq.data_ptr(), dmask.data_ptr(), lens, on_device=True)
    n_samples = len(w.samples)
    win_start = np.concatenate([[0], np.cumsum([ib.window_count(lens[c:c + 1], W, k) for c in range(len(lens))])])
    n_win = int(win_start[-1])
    t0 = time.time()

    def codes(i):
        sp = w.samples[i]
        bound = sp.codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
        buf = torch.empty(bound, dtype=torch.int64, device="cuda")
        n = sp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), buf.data_ptr(), bound)
        return buf, n

    full, n_keys, table_bytes = [], [], []
    rows_dev = torch.empty(n_win * 6, dtype=torch.int32, device="cuda")
    for i in range(n_samples):
        buf, n = codes(i)
        n_keys.append(n)
        t = ib.Table.from_codes(buf.data_ptr(), n, k, on_device=True, force_format=5)
        table_bytes.append(int(t.info().device_bytes))
        del buf
        torch.cuda.empty_cache()
        ib.scan_async(t, ref, W, rows_dev.data_ptr(), n_win, 0)
        torch.cuda.synchronize()
        full.append(rows_dev.cpu().numpy().view(ib.WINDOW_DTYPE).copy())
        t.close()
    del rows_dev
    torch.cuda.empty_cache()
    # one sample over one contig against the reference's own CPU scan
    si = int(np.argmin(n_keys))
    ci = int(np.argmin([int(x) for x in lens]))
    ref_check = None
    if REF_FASTIBS.exists() and not args.no_cpu_baseline:
        buf, n = codes(si)
        ref_check = reference_check(w, "admitted", si, ci, buf.data_ptr(), n,
                                    full[si][int(win_start[ci]):int(win_start[ci + 1])])
        del buf
        torch.cuda.empty_cache()
    setup_s = time.time() - t0
    budget = int(sum(table_bytes) / args.admit_overcommit)
    log(f"[admitted] {n_samples} samples, {sum(n_keys) / 1e9:.2f}e9 k-mers, tables {sum(table_bytes) / 1e9:.1f} GB "
        f"(pinned host images of that size per server), budget {budget / 1e9:.1f} GB, setup {setup_s:.0f} s")

    # requests: Zipf(1.1) over the samples; whole-genome (one request per
    # contig, timed as a group) or regional (log-uniform 1 Mbp .. a contig)
    rng = np.random.default_rng(606)
    pop = 1.0 / np.arange(1, n_samples + 1) ** 1.1
    pop /= pop.sum()
    order = rng.permutation(n_samples)
    reqs, group = [], []
    step = W - k
    for g in range(args.admit_requests):
        s_ = int(order[rng.choice(n_samples, p=pop)])
        if rng.random() < args.admit_whole_frac:
            for c in range(len(lens)):
                reqs.append((s_, c, 0, 0))
                group.append(g)
        else:
            c = int(rng.integers(0, len(lens)))
            L = int(lens[c])
            ln = int(np.exp(rng.uniform(np.log(1e6), np.log(max(L, 1e6 + 1)))))
            nw_c = int(win_start[c + 1] - win_start[c])
            first = min(int(rng.integers(0, max(1, (L - ln) // step + 1))), nw_c - 1)
            reqs.append((s_, c, first, max(1, min(nw_c - first, ln // step))))
            group.append(g)
    group = np.array(group)
    gaps = rng.exponential(1.0 / args.admit_rate, args.admit_requests)

    def run(srv, paced: bool):
        done = {}
        stats0 = srv.stats()
        t_start = srv.now()
        submit_t = {}
        i = 0
        if paced:
            t_next = time.perf_counter()
            for g in range(args.admit_requests):
                t_next += gaps[g]
                while time.perf_counter() < t_next:
                    for r in srv.poll(256, timeout_ms=0):
                        done[r["request_id"]] = r
                    time.sleep(0.0002)
                while i < len(reqs) and group[i] == g:
                    submit_t[srv.submit(*reqs[i])] = i
                    i += 1
        else:
            for req in reqs:
                submit_t[srv.submit(*req)] = len(submit_t)
        deadline = time.time() + 3600
        while len(done) < len(reqs) and time.time() < deadline:
            for r in srv.poll(256, timeout_ms=1000):
                done[r["request_id"]] = r
        assert len(done) == len(reqs), f"admitted requests unfinished: {srv.stats()}"
        makespan = srv.now() - t_start
        st = srv.stats()
        first_submit = np.full(args.admit_requests, np.inf)
        last_done = np.zeros(args.admit_requests)
        for rid, r in done.items():
            assert r["status"] == 0, "an admitted request failed"
            a = int(win_start[r["contig"]] + r["first_window"])
            assert np.array_equal(r["rows"], full[r["sample"]][a:a + int(r["n_windows"])]), "admitted rows differ"
            g = group[submit_t[rid]]
            first_submit[g] = min(first_submit[g], r["submit_time"])
            last_done[g] = max(last_done[g], r["done_time"])
        lat = last_done - first_submit
        probes = st["probes"] - stats0["probes"]
        return {"requests": args.admit_requests, "server_requests": len(reqs), "probes": int(probes),
                "scanned": int(st["scanned"] - stats0["scanned"]), "makespan_s": makespan,
                "probes_per_s": probes / makespan,
                "device_busy_s": st["busy_seconds"] - stats0["busy_seconds"],
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_max_s": float(lat.max()), "launches": int(st["launches"] - stats0["launches"]),
                "reloads": int(st["reloads"] - stats0["reloads"]),
                "reload_bytes": int(st["reload_bytes"] - stats0["reload_bytes"]),
                "evictions": int(st["evictions"] - stats0["evictions"])}

    out = {"workload": f"{w.name} reference x {n_samples} samples, tables {sum(table_bytes) / 1e9:.1f} GB "
                       f"against a {budget / 1e9:.1f} GB budget",
           "k": k, "window": W, "reference_bp": int(sum(map(int, lens))), "sample_kmers": n_keys,
           "table_gb_total": sum(table_bytes) / 1e9, "budget_gb": budget / 1e9,
           "requests": args.admit_requests, "whole_genome_frac": args.admit_whole_frac,
           "popularity": "Zipf(1.1)", "arrival_rate_per_s": args.admit_rate, "setup_s": setup_s}
    for mode in ("plain", "batched"):
        srv = ib.Server(ref, W, k, memory_budget=budget, one_request_per_launch=(mode == "plain"))
        for i in range(n_samples):
            buf, n = codes(i)
            srv.add_codes(buf.data_ptr(), n, on_device=True)
            del buf
            torch.cuda.empty_cache()
        log(f"[admitted] {mode}: {n_samples} samples registered")
        out[f"{mode}_saturated"] = run(srv, False)
        out[f"{mode}_poisson"] = run(srv, True)
        srv.close()
        torch.cuda.empty_cache()
    out["saturated_speedup_vs_plain"] = (out["batched_saturated"]["probes_per_s"] /
                                         out["plain_saturated"]["probes_per_s"])
    out["rows_equal_full_scan"] = True
    out["parity"] = {"status": "bit-exact" if ref_check is None or ref_check["status"] == "bit-exact"
                     else "MISMATCH",
                     "single_sample": "every admitted row equals the same window of its sample's full "
                                      "single-sample scan",
                     "reference": ref_check}
    out["note"] = ("latency of a whole-genome request = its last contig's completion - its submission; "
                   "both modes use per-sample tables under the same budget")
    ref.free()
    return out


def reference_arm(args, w):
    """--impl reference: the reference's own CPU-BATCHED fastibs (built from
    its sources into oracle/_ref/; FASTIBS_THREADS = all host threads) on the
    workload's files, one contig of the reference per step, in contig order
    and cycling: the warm-up steps and then `steps` timed ones (with at least
    as many steps as contigs, the timed ones cover the whole reference). The
    input files come from a separate `bench.py --prepare` process when they
    are not there yet, so this process runs nothing of this repository's
    libraries."""
    if not REF_FASTIBS.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/fastibs was not built (the reference "
                "sources are needed at build time)"}
    p = input_paths(w)
    if not (p["db_stamp"].exists() and p["genome"].exists() and p["contig_stamp"].exists()):
        cmd = [sys.executable, str(REPO / "bench.py"), "--prepare", "--workload", args.workload]
        if args.scale != 1.0:
            cmd += ["--scale", str(args.scale)]
        r = subprocess.run(cmd)
        if r.returncode != 0:
            return {"impl": "reference", "unavailable": f"input preparation failed ({r.returncode})"}
    k, W = w.k, w.window
    names = list(w.ref.names)
    per_contig = valid_positions_by_contig(w.ref.lens, k, w.ref.n_runs())
    n = args.warmup + args.steps
    steps = [i % len(names) for i in range(n)]
    refdir = p["root"] / "ref_steps"
    shutil.rmtree(refdir, ignore_errors=True)
    refdir.mkdir(parents=True)
    for i, c in enumerate(steps):
        os.symlink(p["contig_dir"] / f"{names[c]}_genome.fasta", refdir / f"s{i:03d}_{names[c]}_genome.fasta")
    threads = os.cpu_count() or 1
    wall, phases, _ = run_fastibs(REF_FASTIBS, p["dbdir"], refdir, p["root"] / "ref_steps_out", W,
                                  ("--cpu", "--probe=batched"), env=reference_env(threads))
    stats = [phases[f"s{i:03d}_{names[c]}"]["stats"] for i, c in enumerate(steps)]
    timed = range(args.warmup, n)
    probes = sum(per_contig[steps[i]] for i in timed)
    secs = sum(stats[i] for i in timed)
    value = probes / secs
    covered = sorted({steps[i] for i in timed})
    return {
        "metric": METRIC, "value": value, "unit": "probes/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "impl": "reference",
        "data": "synthetic (seeded generator; stands in for plant-genome inputs not available here)",
        "config": {"workload": w.name, "reference_bp": int(sum(map(int, w.ref.lens))), "contigs": len(names),
                   "sample_kmers": int(p["db_stamp"].read_text()), "k": k, "window": W,
                   "step": "one contig of the reference (in order, cycling) against the whole sample database",
                   "timed_contigs_covered": f"{len(covered)} of {len(names)}"},
        "cpu_baseline": {"value": value, "unit": "probes/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} timed + {args.warmup} warm-up contig scans of {w.name}; "
                                   f"oracle/_ref/fastibs --cpu --probe=batched (CPU-BATCHED, FASTIBS_THREADS="
                                   f"{threads}); probes/s = valid positions / 'stats' phase seconds",
                         "setup_s": phases[f"s000_{names[steps[0]]}"]["setup"], "wall_s": wall},
        "e2e": {"value": value, "unit": "probes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def apply_tuning(args):
    """The scan's launch shape and table layout: the committed autotuner
    result (or a given file), then any explicit flag on top."""
    import ibs_b200 as ib
    from ibs_b200 import autotune
    applied = None
    if args.tuning != "none":
        path = None if args.tuning == "auto" else args.tuning
        applied = autotune.apply(path)
    t = ib.get_tuning()
    for name in ("span_len", "blocks_in_flight", "block_threads", "ctas_per_sm"):
        v = getattr(args, name)
        if v:
            setattr(t, name, v)
    ib.set_tuning(t)
    args.tuning_used = {**t.as_dict(), "source": "flags over " + (args.tuning if applied else "library defaults")}
    log(f"[bench] tuning {args.tuning_used}")


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="plain_2gbp")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the workload (testing)")
    ap.add_argument("--prepare", action="store_true",
                    help="only write the workload's input files (KMC database, FASTA) and exit")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fasta-e2e", action="store_true", help="skip the from-FASTA end-to-end measurement")
    ap.add_argument("--table-format", type=int, default=0,
                    help="sample table layout: 0 library default, 1 B8x32, 2 B6x40, 4 minimizer-bucketed")
    ap.add_argument("--keys-per-bucket", type=float, default=0.0, help="table load (0: library default)")
    ap.add_argument("--tuning", default="auto",
                    help="launch shape: 'auto' = the committed gpu-ibs_b200/tuning/b200.json when present, "
                         "'none' = library defaults, or a path")
    ap.add_argument("--span-len", type=int, default=0)
    ap.add_argument("--blocks-in-flight", type=int, default=0)
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--no-panel", action="store_true",
                    help="skip the 16-sample batched panel (measured by default at N=1)")
    ap.add_argument("--panel-only", action="store_true")
    ap.add_argument("--panel-samples", type=int, default=16)
    ap.add_argument("--panel-scale", type=float, default=1.0)
    ap.add_argument("--panel-keys-per-bucket", type=float, default=0.0,
                    help="joint-table load (0: the tuned default)")
    ap.add_argument("--panel-workload", choices=["panel_4gbp", "served_2gbp"], default="panel_4gbp",
                    help="panel_4gbp (k=31); served_2gbp's 16 k=25 samples make small profiling cases")
    ap.add_argument("--no-serve", action="store_true",
                    help="skip the served request stream (measured by default at N=1)")
    ap.add_argument("--no-admitted", action="store_true",
                    help="skip memory-admitted serving (measured by default at N=1)")
    ap.add_argument("--serve-only", action="store_true")
    ap.add_argument("--serve-samples", type=int, default=16)
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-rates", default="5,20,50",
                    help="Poisson arrival rates (req/s); the highest runs every request")
    ap.add_argument("--serve-modes", default="plain,batched",
                    help="which servers the served stream runs (plain: one request per launch; "
                         "batched: joint tables; single: the batching server over per-sample tables; "
                         "adding iterations launches the batched server's kernels per loop iteration "
                         "instead of feeding one persistent launch)")
    ap.add_argument("--serve-seconds", type=float, default=20.0,
                    help="arrival time of the request prefix run at the lower rates")
    ap.add_argument("--serve-scale", type=float, default=1.0, help="reference length scale")
    ap.add_argument("--serve-group-gb", type=float, default=0.0,
                    help="largest joint table of the batched server (GB; 0: as many samples per table "
                         "as memory allows)")
    ap.add_argument("--admitted-only", action="store_true",
                    help="memory-admitted serving: 48 samples, tables ~3x the server's budget")
    ap.add_argument("--admit-samples", type=int, default=48)
    ap.add_argument("--admit-scale", type=float, default=1.0, help="reference length scale")
    ap.add_argument("--admit-sample-scale", type=float, default=0.1,
                    help="sample size scale: the pinned host images of all 48 tables must fit the "
                         "host's memory (196 GB on the B200 boxes here)")
    ap.add_argument("--admit-overcommit", type=float, default=3.0,
                    help="sum of the tables / the server's byte budget")
    ap.add_argument("--admit-requests", type=int, default=1500,
                    help="requests of the memory-admitted stream (the configuration names 5,000; the default "
                         "keeps the whole bench within minutes)")
    ap.add_argument("--admit-whole-frac", type=float, default=0.1)
    ap.add_argument("--admit-rate", type=float, default=100.0)
    ap.add_argument("--serve-workload", choices=["served_2gbp", "panel_4gbp"], default="served_2gbp",
                    help="the pool: the 2 Gbp reference with 16 samples, or the 4.2 Gbp panel's")
    ap.add_argument("--no-wide", action="store_true",
                    help="skip the k = 41 wide-key scan (measured by default at N=1)")
    ap.add_argument("--wide-keys", type=float, default=1e8, help="keys of the wide-key table")
    ap.add_argument("--arm-start-limit", type=float, default=1080.0,
                    help="seconds after start past which the batched, served and admitted arms are not "
                         "started (reported as skipped), so that the whole run stays bounded")
    ap.add_argument("--serve-sample-scale", type=float, default=0.5,
                    help="panel_4gbp pool: sample size scale (its 16 full-size samples do not fit "
                         "on one GPU together)")
    args = ap.parse_args()

    from ibs_b200 import configs
    fn = getattr(configs, args.workload)
    w = fn(scale=args.scale) if args.scale != 1.0 else fn()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.prepare:
        return prepare_main(args, w)
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(reference_arm(args, w)), flush=True)
        return 0

    apply_tuning(args)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    if args.serve_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"served": served_arm(args, rank)}), flush=True)
        return 0
    if args.panel_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"panel": panel_arm(args, rank)}), flush=True)
        return 0
    if args.admitted_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"admitted": admitted_arm(args, rank)}), flush=True)
        return 0
    out = gpu_arm(args, w, rank, world, local)
    # the batched and served forms, each on its own workload with its own
    # parity check against single-sample scans; one failing is reported in
    # the line, not fatal to it
    if world == 1:
        import torch
        for key, skip, fn in (("wide", args.no_wide, wide_arm),
                              ("panel", args.no_panel, panel_arm), ("served", args.no_serve, served_arm),
                              ("admitted", args.no_admitted, admitted_arm)):
            if skip:
                continue
            if time.time() - STARTED > args.arm_start_limit:
                out[key] = {"skipped": f"not started: {time.time() - STARTED:.0f} s after start is past "
                                       f"--arm-start-limit {args.arm_start_limit:.0f} s"}
                log(f"[bench] {key} arm skipped ({out[key]['skipped']})")
                continue
            torch.cuda.empty_cache()
            t0 = time.time()
            try:
                out[key] = fn(args, rank)
            except Exception as e:  # reported in the line
                import traceback
                traceback.print_exc()
                out[key] = {"error": f"{type(e).__name__}: {e}"[-600:]}
            out[key]["arm_wall_s"] = time.time() - t0
            log(f"[bench] {key} arm done in {time.time() - t0:.0f} s")
            torch.cuda.empty_cache()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
