"""The fastibs command line over the B200 scan: the reference's CLI
contract (src/FastIBS.cpp) and, on a GPU, its files byte for byte against the
golden TSVs of the reference's own binary."""
import os
import shutil
import subprocess

import pytest

import corpus

FASTIBS = corpus.REPO / "gpu-ibs_b200" / "bin" / "fastibs"


def run(args, cwd, env=None):
    e = dict(os.environ, **(env or {}))
    return subprocess.run([str(FASTIBS)] + [str(a) for a in args], cwd=cwd, capture_output=True,
                          text=True, env=e)


@pytest.fixture(scope="module")
def c25(build_case):
    return build_case("edge_k25")


def test_version_and_help(tmp_path):
    r = run(["--version"], tmp_path)
    assert r.returncode == 0 and r.stdout.startswith("fastibs (GPU-IBS")
    r = run(["-h"], tmp_path)
    assert r.returncode == 0 and "Usage:" in r.stdout
    r = run([], tmp_path)
    assert r.returncode == 1 and "Usage:" in r.stdout


def test_argument_errors(tmp_path, c25):
    r = run([c25["db"], c25["refs"], tmp_path / "o", "abc"], tmp_path)
    assert r.returncode == 1 and "Invalid <windowSize>" in r.stderr
    r = run([c25["db"], c25["refs"], tmp_path / "o", "5000", "--bogus"], tmp_path)
    assert r.returncode == 1 and "Unknown option" in r.stderr
    r = run([c25["db"], c25["refs"], tmp_path / "o", "5000", "--hash-lf=2"], tmp_path)
    assert r.returncode == 1 and "expected 0.1 .. 0.95" in r.stderr
    r = run([tmp_path / "nodb", c25["refs"], tmp_path / "o", "5000"], tmp_path)
    assert r.returncode == 1 and "KMC database folder not found" in r.stderr
    r = run([str(c25["prefix"]), c25["refs"], tmp_path / "o", "5000"], tmp_path)
    assert r.returncode == 1 and "this is a KMC prefix" in r.stderr
    r = run([c25["db"], c25["refs"], tmp_path / "o", "25"], tmp_path)
    assert r.returncode == 1 and "must be larger than the database's k (25)" in r.stderr
    empty = tmp_path / "norefs"
    empty.mkdir()
    (empty / "notes.txt").write_text("x")
    r = run([c25["db"], empty, tmp_path / "o", "5000"], tmp_path)
    assert r.returncode == 1 and "no reference files" in r.stderr and "Skipping notes.txt" in r.stdout


def test_existing_output_is_skipped(tmp_path, c25):
    out = tmp_path / "o"
    out.mkdir()
    (out / "db_v_test_5000.tsv").write_text("kept\n")
    r = run([c25["db"], c25["refs"], out, "5000"], tmp_path)
    assert r.returncode == 0 and "File already exists, skipping" in r.stdout
    assert (out / "db_v_test_5000.tsv").read_text() == "kept\n"


def test_k_above_64_is_refused_before_any_device_work(tmp_path):
    """33 <= k <= 64 builds wide-key tables; a longer k is refused with the
    reason, from the header alone, as the reference refuses what it cannot
    open (exit status 1)."""
    import numpy as np
    import ibs_b200 as ib
    db = tmp_path / "db"
    db.mkdir()
    ib.kmc_write(str(db / "sample"), np.arange(10, dtype=np.uint64), 10, k=32, p=8)
    pre = (db / "sample.kmc_pre").read_bytes()
    pos = len(pre) - (pre[-8] + 8)  # the header's first field is k
    (db / "sample.kmc_pre").write_bytes(pre[:pos] + (72).to_bytes(4, "little") + pre[pos + 4:])
    refs = tmp_path / "refs"
    refs.mkdir()
    (refs / "x_genome.fasta").write_text(">c\n" + "ACGT" * 100 + "\n")
    r = run([db, refs, tmp_path / "o", "5000"], tmp_path)
    assert r.returncode == 1
    assert "k=72 > 64" in r.stderr


def test_panel_of_different_k_is_refused(tmp_path, build_case):
    """A panel shares one k (src/FastIBS.cpp:155-172): every member's header is
    read first, so k = 25 and k = 41 databases are refused before any device
    work, with the reference's message."""
    a, b = build_case("edge_k25"), build_case("edge_k41")
    db2 = tmp_path / "db2"
    shutil.copytree(b["db"], db2)
    r = run([a["db"], a["refs"], tmp_path / "o", "5000", f"--db={db2}"], tmp_path)
    assert r.returncode == 1
    assert "has k=41 but db has k=25; a panel shares one k" in r.stderr


def test_without_a_device_the_reference_fails_and_is_logged(tmp_path, c25):
    import ibs_b200
    if ibs_b200.device_count() > 0:
        pytest.skip("a device is present")
    r = run([c25["db"], c25["refs"], tmp_path / "o", "5000"], tmp_path)
    assert r.returncode == 1
    assert "no CPU fallback" in (tmp_path / "log.txt").read_text()
    assert not (tmp_path / "o" / "db_v_test_5000.tsv").exists()


@pytest.mark.gpu
@pytest.mark.parametrize("name", corpus.GOLDEN_CASES)
def test_cli_files_match_reference_golden(name, build_case, tmp_path):
    gold = corpus.load_golden(name)
    case = build_case(name)
    for W in case["windows"]:
        out = tmp_path / f"o{W}"
        r = run([case["db"], case["refs"], out, W], tmp_path)
        assert r.returncode == 0, r.stderr
        f = out / gold["tsv_name"][str(W)]
        assert f.read_bytes().decode("latin-1") == gold["tsv"][str(W)]


@pytest.mark.gpu
@pytest.mark.parametrize("resident", [0, 1])
def test_cli_panel_equals_single_runs(resident, build_case, tmp_path):
    a, b = build_case("edge_k25"), build_case("edge_k25_kmc1")
    # a panel of the two databases (folders named db and db2) on edge_k25's reference
    db2 = tmp_path / "db2"
    shutil.copytree(b["db"], db2)
    out = tmp_path / "panel"
    args = [a["db"], a["refs"], out, 5000, f"--db={db2}"] + ([f"--resident={resident}"] if resident else [])
    r = run(args, tmp_path)
    assert r.returncode == 0, r.stderr
    assert ("2 rounds" if resident == 1 else "1 round") in r.stdout
    single = tmp_path / "single"
    assert run([db2, a["refs"], single, 5000], tmp_path).returncode == 0
    gold = corpus.load_golden("edge_k25")
    assert (out / "db_v_test_5000.tsv").read_bytes().decode("latin-1") == gold["tsv"]["5000"]
    assert (out / "db2_v_test_5000.tsv").read_bytes() == (single / "db2_v_test_5000.tsv").read_bytes()
