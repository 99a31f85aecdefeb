"""Regenerates the golden fixtures in tests/golden/ (run in a container where
the reference sources are present; needs oracle/_ref/fastibs built by
`make -C oracle ref`).

For every case of tests/corpus.py: build the inputs from their seeds, run the
reference's own fastibs CLI in its three CPU modes (CPU-OPT: --cpu;
CPU-BATCHED: --cpu --probe=batched; CPU-BASE: FASTIBS_LEGACY=1 --cpu),
require the three TSVs to be byte-identical, and store that TSV together
with the sha256 of the inputs in <case>.json.

Usage: python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import corpus  # noqa: E402

REF_BIN = corpus.REPO / "oracle" / "_ref" / "fastibs"


def run_reference(case, W: int, workdir: Path) -> str:
    outs = {}
    modes = {"cpu_opt": (["--cpu"], {}),
             "cpu_batched": (["--cpu", "--probe=batched"], {"FASTIBS_CPU_BATCH": "16"}),
             "cpu_base": (["--cpu"], {"FASTIBS_LEGACY": "1"})}
    for mode, (args, env) in modes.items():
        out = workdir / f"out_{mode}_{W}"
        shutil.rmtree(out, ignore_errors=True)
        e = dict(os.environ, **env)
        r = subprocess.run([str(REF_BIN), str(case["db"]), str(case["refs"]), str(out), str(W)] + args,
                           env=e, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference {mode} failed: {r.stderr[-2000:]}")
        files = sorted(out.glob("*.tsv"))
        if len(files) != 1:
            raise RuntimeError(f"reference {mode}: expected one TSV, got {files}")
        outs[mode] = files[0].read_bytes().decode("latin-1")
        outs[mode + "_name"] = files[0].name
    if not (outs["cpu_opt"] == outs["cpu_batched"] == outs["cpu_base"]):
        raise RuntimeError("the reference's CPU modes disagree")
    return outs["cpu_opt"], outs["cpu_opt_name"]


def main(names):
    if not REF_BIN.exists():
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` first")
    for name in names or corpus.GOLDEN_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            case = corpus.build_case(name, Path(tmp))
            rec = {"case": name, "k": case["k"], "windows": case["windows"],
                   "inputs_sha256": corpus.input_hashes(case), "tsv": {}, "tsv_name": {},
                   "encoding": "latin-1", "made_by": "reference fastibs (src/FastIBS.cpp) --cpu / --probe=batched / FASTIBS_LEGACY=1"}
            for W in case["windows"]:
                tsv, fname = run_reference(case, W, Path(tmp))
                rec["tsv"][str(W)] = tsv
                rec["tsv_name"][str(W)] = fname
            corpus.golden_path(name).write_text(json.dumps(rec, indent=1) + "\n")
            rows = sum(t.count("\n") - 1 for t in rec["tsv"].values())
            print(f"{name}: {rows} rows, windows {case['windows']}")


if __name__ == "__main__":
    main(sys.argv[1:])
