"""KDBIntersect (the intersection size of two KMC databases): the oracle
against the counts of the reference's own KDBIntersect (tests/golden/
intersect.json, made by tests/golden/make_intersect_golden.py), then the
device count (ibs_count_present_kmc) and the KDBIntersect CLI against both."""
import json
import subprocess

import numpy as np
import pytest

import corpus
import oracle as orc

GOLD = json.loads((corpus.GOLDEN / "intersect.json").read_text())
CLI = corpus.REPO / "gpu-ibs_b200" / "bin" / "KDBIntersect"


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    root = tmp_path_factory.mktemp("intersect")
    out = {n: corpus.build_intersect_case(n, root) for n in corpus.INTERSECT_CASES}
    for n, c in out.items():
        assert corpus.intersect_hashes(c) == GOLD["cases"][n]["inputs_sha256"], n
    return out


@pytest.mark.parametrize("name", list(corpus.INTERSECT_CASES))
def test_oracle_matches_reference_counts(cases, name):
    c = cases[name]
    if c["k"] > 32:
        a = set(zip(*(x.tolist() for x in orc.Index(str(c["prefix_a"])).list_codes128())))
        b = set(zip(*(x.tolist() for x in orc.Index(str(c["prefix_b"])).list_codes128())))
        assert len(a & b) == GOLD["cases"][name]["count"]
        assert len(a) == GOLD["cases"][name]["self_count_a"]
        return
    a = orc.Index(str(c["prefix_a"])).list_codes()
    b = orc.Index(str(c["prefix_b"])).list_codes()
    assert len(np.intersect1d(a, b)) == GOLD["cases"][name]["count"]
    assert len(np.unique(a)) == GOLD["cases"][name]["self_count_a"]


def test_cli_usage_without_a_device():
    assert CLI.exists()
    r = subprocess.run([str(CLI)], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stdout
    r = subprocess.run([str(CLI), "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    r = subprocess.run([str(CLI), "/nonexistent/a", "/nonexistent/b"], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("Error: KMC database folder not found")


def test_cli_k_mismatch_is_the_reference_error(cases):
    r = subprocess.run([str(CLI), str(cases["x_k25"]["a"]), str(cases["x_k31"]["a"])],
                       capture_output=True, text=True)
    assert r.returncode == GOLD["mismatch"]["exit"] == 1
    assert r.stdout == GOLD["mismatch"]["stdout"]
    assert r.stderr == GOLD["mismatch"]["stderr"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(corpus.INTERSECT_CASES))
def test_device_count_matches_reference(cases, name):
    import ibs_b200 as ib
    c = cases[name]
    want = GOLD["cases"][name]
    # k > 32: one layout, the wide-key table
    formats = [0] if c["k"] > 32 else [0, 1, 2] + ([4] if 16 <= c["k"] <= 27 else []) + (
        [6] if 16 <= c["k"] <= 31 else [])
    for fmt in formats:
        if fmt == 1 and c["k"] > 25:
            continue  # B8x32 needs 2^(2k-31) buckets
        for big, small in (("b", "a"), ("a", "b")):
            t = ib.Table.open(str(c["prefix_" + big]), force_format=fmt)
            assert t.count_present_kmc(str(c["prefix_" + small])) == want["count"], (name, fmt, big)
            t.close()
        t = ib.Table.open(str(c["prefix_a"]), force_format=fmt)
        assert t.count_present_kmc(str(c["prefix_a"])) == want["self_count_a"]
        if c["k"] > 32:
            lo, hi = orc.Index(str(c["prefix_b"])).list_codes128()
            assert int(t.probe128(lo, hi).sum()) == want["count"]
        else:
            codes = orc.Index(str(c["prefix_b"])).list_codes()
            assert t.count_present(codes) == want["count"]
        t.close()


@pytest.mark.gpu
def test_device_count_rejects_k_mismatch(cases):
    import ibs_b200 as ib
    t = ib.Table.open(str(cases["x_k25"]["prefix_a"]))
    with pytest.raises(ib.IbsError) as e:
        t.count_present_kmc(str(cases["x_k31"]["prefix_a"]))
    assert e.value.status == 1
    t.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(corpus.INTERSECT_CASES))
def test_cli_prints_the_reference_count(cases, name):
    c = cases[name]
    for a, b in ((c["a"], c["b"]), (c["b"], str(c["a"]) + "/")):
        r = subprocess.run([str(CLI), str(a), str(b)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert r.stdout == f"{GOLD['cases'][name]['count']}\n"
