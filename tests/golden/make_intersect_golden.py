"""Regenerates tests/golden/intersect.json: the intersection sizes the
reference's own KDBIntersect prints for the pairs of tests/corpus.py's
INTERSECT_CASES (run where the reference sources are present, after
`make -C oracle ref` has built oracle/_ref/kdbintersect).

Each pair runs in both argument orders, on the reference's enumeration path
and on its KMC-API stream-and-probe path (FASTIBS_LEGACY=1); all four counts
must agree. A pair of databases with different k records the error line and
exit status.

Usage: python tests/golden/make_intersect_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import corpus  # noqa: E402

REF_BIN = corpus.REPO / "oracle" / "_ref" / "kdbintersect"
OUT = corpus.GOLDEN / "intersect.json"


def run(a, b, legacy: bool):
    env = dict(os.environ, FASTIBS_LEGACY="1") if legacy else dict(os.environ)
    env.pop("FASTIBS_LEGACY", None) if not legacy else None
    r = subprocess.run([str(REF_BIN), str(a), str(b)], env=env, capture_output=True, text=True)
    return r.returncode, r.stdout, r.stderr


def main():
    if not REF_BIN.exists():
        sys.exit(f"{REF_BIN} missing: run `make -C oracle ref` first")
    rec = {"made_by": "reference KDBIntersect (src/KDBIntersect.cpp), enumeration and FASTIBS_LEGACY=1 paths",
           "cases": {}}
    with tempfile.TemporaryDirectory() as tmp:
        cases = {n: corpus.build_intersect_case(n, Path(tmp)) for n in corpus.INTERSECT_CASES}
        for name, c in cases.items():
            counts = set()
            for a, b in ((c["a"], c["b"]), (c["b"], c["a"]), (c["a"], c["a"])):
                for legacy in (False, True):
                    rc, out, err = run(a, b, legacy)
                    if rc != 0:
                        raise RuntimeError(f"{name}: reference failed: {err}")
                    counts.add((a == b, int(out.strip())))
            pair = {v for same, v in counts if not same}
            selfc = {v for same, v in counts if same}
            if len(pair) != 1 or len(selfc) != 1:
                raise RuntimeError(f"{name}: the reference's paths disagree: {counts}")
            rec["cases"][name] = {"k": c["k"], "count": pair.pop(), "self_count_a": selfc.pop(),
                                  "inputs_sha256": corpus.intersect_hashes(c)}
            print(name, rec["cases"][name]["count"], rec["cases"][name]["self_count_a"])
        rc, out, err = run(cases["x_k25"]["a"], cases["x_k31"]["a"], False)
        rec["mismatch"] = {"pair": ["x_k25/a", "x_k31/a"], "exit": rc, "stdout": out, "stderr": err}
        print("mismatch", rc, err.strip())
    OUT.write_text(json.dumps(rec, indent=1) + "\n")


if __name__ == "__main__":
    main()
