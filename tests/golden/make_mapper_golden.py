"""Regenerates tests/golden/mapper.json: the coverage files the reference's
own fastibsmapper writes for the golden cases of tests/corpus.py (run where
the reference sources are present, after `make -C oracle ref` has built
oracle/_ref/fastibsmapper).

Every case runs in the reference's three CPU modes (CPU-OPT: default;
CPU-BATCHED: --cpu --probe=batched; CPU-BASE: FASTIBS_LEGACY=1), which must
write byte-identical files; the file's name, size and sha256 are stored
(the files themselves run to megabytes).

Usage: python tests/golden/make_mapper_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import corpus  # noqa: E402

REF_BIN = corpus.REPO / "oracle" / "_ref" / "fastibsmapper"
OUT = corpus.GOLDEN / "mapper.json"


def main():
    if not REF_BIN.exists():
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` first")
    rec = {"made_by": "reference fastibsmapper (src/FastIBSMapper.cpp), CPU-OPT / CPU-BATCHED / CPU-BASE",
           "cases": {}}
    modes = {"cpu_opt": ([], {}), "cpu_batched": (["--cpu", "--probe=batched"], {"FASTIBS_CPU_BATCH": "16"}),
             "cpu_base": ([], {"FASTIBS_LEGACY": "1"})}
    with tempfile.TemporaryDirectory() as tmp:
        for name in corpus.GOLDEN_CASES:
            case = corpus.build_case(name, Path(tmp))
            got = {}
            for mode, (args, env) in modes.items():
                out = Path(tmp) / f"map_{name}_{mode}"
                shutil.rmtree(out, ignore_errors=True)
                r = subprocess.run([str(REF_BIN), str(case["db"]), str(case["refs"]), str(out)] + args,
                                   env=dict(os.environ, **env), capture_output=True, text=True)
                if r.returncode != 0:
                    raise RuntimeError(f"{name} {mode}: {r.stderr[-2000:]}")
                (f,) = sorted(out.glob("*.txt"))
                got[mode] = (f.name, f.read_bytes())
            if len({v[1] for v in got.values()}) != 1:
                raise RuntimeError(f"{name}: the reference's CPU modes disagree")
            fname, data = got["cpu_opt"]
            rec["cases"][name] = {"name": fname, "bytes": len(data), "sha256": hashlib.sha256(data).hexdigest(),
                                  "inputs_sha256": corpus.input_hashes(case)}
            print(name, fname, len(data))
    OUT.write_text(json.dumps(rec, indent=1) + "\n")


if __name__ == "__main__":
    main()
