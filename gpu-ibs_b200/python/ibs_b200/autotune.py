"""Autotuner of the window scans.

The single-sample scan: sweeps the table layout and load (bucket format and
keys per bucket) and the kernel launch shape (span length = positions per
warp task, 32-position blocks in flight per lane, threads per CTA, CTAs per
SM) on the device, times every point with CUDA events, and writes the sweep
and its best point to gpu-ibs_b200/tuning/<gpu>.json.

The batched (joint-table) scan, --panel: sweeps the joint table's load (keys
per 5-slot bucket), the persistent scan's span length, CTAs per SM and
blocks in flight, and the bucket-range pass size, on the 16-sample panel
workload scaled down; every point's rows are checked against the first
point's; the sweep and its best point go to the same file ("panel",
"panel_best"), next to the single-sample result.

    python -m ibs_b200.autotune [--scale 0.25] [--out PATH]
    python -m ibs_b200.autotune --panel [--panel-scale 0.5]

The launch shapes cover the region where earlier full sweeps (up to spans
of 16384, 8 blocks in flight, 128 threads, 4 CTAs per SM) found every
fastest point.

The workload is plain_2gbp scaled down (default 500 Mbp and ~5.5e8 k-mers:
tables of several GB, far beyond L2, so a point's timing is DRAM-bound as at
full size). `apply()` loads a committed result into the library.
"""
from __future__ import annotations

import argparse
import itertools
import json
import time
from pathlib import Path

import numpy as np

from . import (PKG_DIR, Reference, Table, Tuning, get_tuning, scan_async, set_tuning, window_count)
from . import configs

TUNING_DIR = PKG_DIR / "tuning"


def default_path() -> Path:
    return TUNING_DIR / "b200.json"


def apply(path: Path | None = None) -> dict | None:
    """Loads a tuning result (the best point) into the library; returns it."""
    path = Path(path) if path else default_path()
    if not path.exists():
        return None
    res = json.loads(path.read_text())
    best = res["best"]
    t = Tuning(span_len=best["span_len"], blocks_in_flight=best["blocks_in_flight"],
               block_threads=best["block_threads"], ctas_per_sm=best["ctas_per_sm"],
               keys_per_bucket=best["keys_per_bucket"], table_format=best["table_format"])
    pb = res.get("panel_best")
    if pb:
        t.panel_span_len = pb["panel_span_len"]
        t.panel_ctas_per_sm = pb["panel_ctas_per_sm"]
        t.panel_blocks_in_flight = pb["panel_blocks_in_flight"]
        t.panel_keys_per_bucket = pb["panel_keys_per_bucket"]
        t.panel_pass_mb = pb["panel_pass_mb"] or 0xFFFFFFFF
    set_tuning(t)
    return {**best, "panel": pb}


def sweep(scale: float = 0.25, reps: int = 3, quick: bool = False) -> dict:
    import torch
    w = configs.plain_2gbp(scale=scale)
    k, W = w.k, w.window
    lens = w.ref.lens
    sw, mw = w.ref.packed_words()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    bound = w.samples[0].codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
    codes = torch.empty(bound, dtype=torch.int64, device="cuda")
    n = w.samples[0].codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), codes.data_ptr(), bound)
    ref = Reference(dseq.data_ptr(), dmask.data_ptr(), lens, on_device=True)
    n_win = window_count(lens, W, k)
    rows = torch.empty(n_win * 6, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    base = get_tuning()
    layouts = [(1, 3.0), (4, 2.0)] if quick else [(1, 3.0), (1, 4.0), (4, 1.5), (4, 2.0), (4, 3.0)]
    shapes = list(itertools.product([4096] if quick else [1024, 2048, 4096],
                                    [2, 4] if quick else [1, 2, 4],
                                    [256, 512],
                                    [8, 16]))
    points, reference_rows = [], None
    for fmt, kpb in layouts:
        table = Table.from_codes(codes.data_ptr(), n, k, on_device=True, force_format=fmt, keys_per_bucket=kpb)
        info = table.info()
        for span, nb, threads, ctas in shapes:
            set_tuning(Tuning(span_len=span, blocks_in_flight=nb, block_threads=threads, ctas_per_sm=ctas))
            scan_async(table, ref, W, rows.data_ptr(), n_win, stream.cuda_stream)  # plan + warm-up
            stream.synchronize()
            got = rows.cpu().numpy().view(np.int32).copy()
            if reference_rows is None:
                reference_rows = got
            ok = bool(np.array_equal(got, reference_rows))
            e0.record(stream)
            for _ in range(reps):
                scan_async(table, ref, W, rows.data_ptr(), n_win, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            points.append(dict(table_format=fmt, keys_per_bucket=kpb, span_len=span, blocks_in_flight=nb,
                               block_threads=threads, ctas_per_sm=ctas, ms=ms, rows_equal=ok,
                               table_gb=info.device_bytes / 1e9, stash_keys=int(info.stash_keys)))
        table.close()
    set_tuning(base)
    good = [p for p in points if p["rows_equal"]]
    best = min(good, key=lambda p: p["ms"])
    ref.free()
    return {"gpu": torch.cuda.get_device_name(), "workload": w.name, "reference_bp": int(sum(map(int, lens))),
            "sample_kmers": int(n), "reps": reps, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            "best": best, "points": points}


def sweep_panel(scale: float = 0.5, reps: int = 3, quick: bool = False) -> dict:
    """The joint-table scan over the 16-sample panel workload at `scale`."""
    import torch
    from . import PanelTable
    w = configs.panel_4gbp(scale=scale)
    k, W = w.k, w.window
    lens = w.ref.lens
    sw, mw = w.ref.packed_words()
    dseq = torch.empty(sw, dtype=torch.int64, device="cuda")
    dmask = torch.empty(mw, dtype=torch.int64, device="cuda")
    w.ref.reference_device(dseq.data_ptr(), dmask.data_ptr())
    ref = Reference(dseq.data_ptr(), dmask.data_ptr(), lens, on_device=True)
    n_win = window_count(lens, W, k)
    ns = len(w.samples)

    def codes(i):
        sp = w.samples[i]
        bound = sp.codes_device_bound(w.ref, dseq.data_ptr(), dmask.data_ptr())
        buf = torch.empty(bound, dtype=torch.int64, device="cuda")
        n = sp.codes_device(w.ref, dseq.data_ptr(), dmask.data_ptr(), buf.data_ptr(), bound)
        return buf, n

    # the union's size, for the table's capacity: from a 1/64 hash sample of
    # every sample's k-mers
    seen = []
    for i in range(ns):
        buf, n = codes(i)
        v = buf[:n]
        seen.append(torch.unique(v[((v * 0x9E3779B97F4A7C15) >> 58) == 0]))
        del buf, v
    union = int(torch.unique(torch.cat(seen)).numel() * 64 * 1.02) + (1 << 20)
    del seen
    torch.cuda.empty_cache()
    rows = torch.empty(n_win * ns * 6, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    base = get_tuning()
    loads = [3.0] if quick else [2.5, 3.0, 3.5, 4.0]
    passes_mb = [0] if quick else [12 << 10, 24 << 10, 0]  # 0: the default (48 GiB)
    shapes = list(itertools.product([8192] if quick else [4096, 8192, 16384], [4, 6] if quick else [4, 6, 8],
                                    [2, 4], passes_mb))
    points, reference_rows = [], None
    for kpb in loads:
        pt = PanelTable(k, union, keys_per_bucket=kpb)
        for i in range(ns):
            buf, n = codes(i)
            pt.add_codes(buf.data_ptr(), n, on_device=True)
            del buf
        torch.cuda.empty_cache()
        info, _ = pt.info()
        for span, ctas, nb, pmb in shapes:
            t = get_tuning()
            t.panel_span_len, t.panel_ctas_per_sm, t.panel_blocks_in_flight = span, ctas, nb
            t.panel_pass_mb = pmb or 0xFFFFFFFF
            set_tuning(t)
            pt.scan_async(ref, W, rows.data_ptr(), n_win * ns, stream.cuda_stream)  # plan, graph, warm-up
            stream.synchronize()
            got = rows.cpu().numpy().copy()
            if reference_rows is None:
                reference_rows = got
            ok = bool(np.array_equal(got, reference_rows))
            e0.record(stream)
            for _ in range(reps):
                pt.scan_async(ref, W, rows.data_ptr(), n_win * ns, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            points.append(dict(panel_keys_per_bucket=kpb, panel_span_len=span, panel_ctas_per_sm=ctas,
                               panel_blocks_in_flight=nb, panel_pass_mb=pmb, ms=ms, rows_equal=ok,
                               table_gb=info.device_bytes / 1e9, stash_keys=int(info.stash_keys)))
        pt.close()
        torch.cuda.empty_cache()
    set_tuning(base)
    good = [p for p in points if p["rows_equal"]]
    best = min(good, key=lambda p: p["ms"])
    ref.free()
    return {"workload": w.name, "reference_bp": int(sum(map(int, lens))), "samples": ns,
            "union_keys_estimate": union,
            "reps": reps, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            "all_rows_equal": all(p["rows_equal"] for p in points), "best": best, "points": points}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--scale", type=float, default=0.25)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=str(default_path()))
    ap.add_argument("--panel", action="store_true", help="sweep the joint-table scan instead")
    ap.add_argument("--panel-scale", type=float, default=0.5)
    args = ap.parse_args()
    out = Path(args.out)
    if args.panel:
        # the joint-table sweep goes next to the single-sample result in the same file
        prev = json.loads(out.read_text()) if out.exists() else {}
        res = sweep_panel(args.panel_scale, args.reps, args.quick)
        prev["panel"] = res
        prev["panel_best"] = res["best"]
        out.parent.mkdir(parents=True, exist_ok=True)
        out.write_text(json.dumps(prev, indent=1) + "\n")
        print(json.dumps({"panel_best": res["best"], "points": len(res["points"]),
                          "all_rows_equal": res["all_rows_equal"]}))
        return
    res = sweep(args.scale, args.reps, args.quick)
    prev = json.loads(out.read_text()) if out.exists() else {}
    for key in ("panel", "panel_best"):  # keep a committed joint-table result
        if key in prev:
            res[key] = prev[key]
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text(json.dumps(res, indent=1) + "\n")
    b = res["best"]
    print(json.dumps({"best": b, "points": len(res["points"])}))


if __name__ == "__main__":
    main()
