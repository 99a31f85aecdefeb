"""libibs.so / libibs_tools.so on the CPU: they load, export every symbol
their headers declare, and the host-side calls (windowing, packing, KMC
parsing errors) behave; no kernel runs here."""
import ctypes
import re

import numpy as np
import pytest

import corpus
import ibs_b200 as ib
import oracle as orc

REPO = corpus.REPO


def declared(header: str) -> set[str]:
    text = (REPO / "include" / header).read_text()
    return set(re.findall(r"\b(ibs_[a-z0-9_]+)\s*\(", text))


@pytest.mark.parametrize("header,lib", [("ibs.h", "libibs.so"), ("ibs_tools.h", "libibs_tools.so")])
def test_exports_every_declared_symbol(header, lib):
    so = ctypes.CDLL(str(REPO / "gpu-ibs_b200" / "lib" / lib))
    names = declared(header)
    assert names, header
    missing = [n for n in sorted(names) if not hasattr(so, n)]
    assert not missing, missing


def test_window_count_and_bounds_match_reference_rule():
    lens = np.array([0, 1, 24, 25, 26, 99_999, 100_000, 123_457], dtype=np.uint64)
    for W, k in ((50_000, 25), (5_000, 31), (100, 15), (33, 32)):
        n = ib.window_count(lens, W, k)
        assert n == sum(orc.window_count(int(x), W, k) for x in lens)
        rows = ib.window_bounds(lens, W, k)
        r = 0
        for ln in lens:
            for j in range(0, int(ln), W - k):
                assert rows[r]["start"] == j and rows[r]["end"] == min(j + W, int(ln))
                r += 1
    assert ib.window_count(lens, 25, 25) == 0


def test_contigs_beyond_32_bit_coordinates_are_refused():
    # rows carry int32 coordinates (the reference's Window::start / end are
    # int): a contig of 2^31 bases would wrap them, so it is refused; one of
    # 2^31 - 1 bases still fits
    edge = np.array([1000, 2**31 - 1], dtype=np.uint64)
    rows = ib.window_bounds(edge, 50_000, 25)
    assert rows[-1]["end"] == 2**31 - 1 and rows[-1]["start"] > 0
    with pytest.raises(ib.IbsError) as e:
        ib.window_bounds(np.array([1000, 2**31], dtype=np.uint64), 50_000, 25)
    assert e.value.status == 1  # IBS_ERR_ARG
    assert "contig 1" in str(e.value) and "32-bit" in str(e.value)


def _pack_np(seqs):
    """Independent restatement of the packed layout of include/ibs.h."""
    lens = [len(s) for s in seqs]
    off, b = [], 0
    for n in lens:
        off.append(b)
        b += (n + 63) // 64 * 64
    seq = np.zeros(b // 32 + 1, np.uint64)
    mask = np.zeros(b // 64 + 1, np.uint64)
    lut = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3, ord("a"): 0, ord("c"): 1, ord("g"): 2,
           ord("t"): 3}
    for s, o in zip(seqs, off):
        for i, ch in enumerate(s):
            g = o + i
            c = lut.get(ch)
            if c is None:
                mask[g // 64] |= np.uint64(1) << np.uint64(g % 64)
                c = 0
            seq[g // 32] |= np.uint64(c) << np.uint64(2 * (g % 32))
    return seq, mask


def test_pack_ascii_layout():
    rng = np.random.default_rng(3)
    seqs = [bytes(np.frombuffer(b"ACGTacgtNnRY\r", np.uint8)[rng.integers(0, 13, n)])
            for n in (1, 63, 64, 65, 1000, 0, 37)]
    seq, mask, lens = ib.pack_ascii(seqs, threads=3)
    s2, m2 = _pack_np(seqs)
    assert np.array_equal(seq, s2) and np.array_equal(mask, m2)


def test_synthetic_reference_packs_like_its_ascii():
    spec = ib.RefSpec(seed=11, lens=[1000, 70, 5000], n_frac=0.02, n_run=(5, 40), lower_frac=0.1,
                      lower_run=(3, 30))
    seq, mask = spec.reference_host()
    ascii_ = [spec.contig_ascii(c) for c in range(3)]
    s2, m2, _ = ib.pack_ascii(ascii_)
    assert np.array_equal(seq, s2) and np.array_equal(mask, m2)


def test_open_errors_are_reported_without_a_device(tmp_path):
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(tmp_path / "missing"))
    assert e.value.status == 2  # IBS_ERR_IO
    (tmp_path / "bad.kmc_pre").write_bytes(b"XXXX" + b"\0" * 100 + b"XXXX")
    (tmp_path / "bad.kmc_suf").write_bytes(b"KMCSKMCS")
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(tmp_path / "bad"))
    assert e.value.status == 3  # IBS_ERR_FORMAT


def test_open_rejects_k_above_64(tmp_path):
    codes = np.arange(10, dtype=np.uint64)
    ib.kmc_write(str(tmp_path / "s"), codes, 10, k=32, p=8)
    pre = (tmp_path / "s.kmc_pre").read_bytes()
    # patch the header's k (first field of the 64-byte header block) to 72:
    # 33 <= k <= 64 builds a wide-key table, anything longer is refused
    hoff = pre[-8]
    pos = len(pre) - (hoff + 8)
    patched = pre[:pos] + (72).to_bytes(4, "little") + pre[pos + 4:]
    (tmp_path / "s.kmc_pre").write_bytes(patched)
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(tmp_path / "s"))
    assert e.value.status == 6  # IBS_ERR_UNSUPPORTED


def test_no_device_means_no_fallback(build_case):
    if ib.device_count() > 0:
        pytest.skip("a device is present")
    case = build_case("edge_k25")
    with pytest.raises(ib.IbsError) as e:
        ib.Table.open(str(case["prefix"]))
    assert e.value.status == 4  # IBS_ERR_CUDA


def test_kmc_writer_roundtrip_all_layouts(tmp_path):
    rng = np.random.default_rng(9)
    for k, p, ver, cs in ((25, 5, 0x200, 1), (25, 9, 0x200, 4), (31, 7, 0x200, 2), (32, 4, 0x200, 0),
                          (15, 3, 0, 1), (4, 0, 0, 1)):
        codes = corpus.random_codes(rng, 5000, k)
        codes = np.concatenate([codes, codes[:100]])  # duplicates are merged
        pre = tmp_path / f"db_{k}_{p}_{ver}"
        n = ib.kmc_write(str(pre), codes, len(codes), k=k, p=p, version=ver, counter_size=cs,
                         n_bins=16, min_count=2 if cs else 0, max_count=255)
        uniq = np.unique(codes)
        assert n == len(uniq)
        ix = orc.Index(str(pre))
        assert (ix.k, ix.p, ix.total) == (k, p, len(uniq))
        assert np.array_equal(np.sort(ix.list_codes()), uniq)
        miss = corpus.random_codes(rng, 2000, k)
        assert np.array_equal(ix.probe(miss).astype(bool), np.isin(miss, uniq))


def test_sort_unique_host():
    rng = np.random.default_rng(1)
    x = rng.integers(0, 1000, 200_000).astype(np.uint64)
    assert np.array_equal(ib.sort_unique_host(x.copy(), threads=4), np.unique(x))


def test_library_defaults_are_the_committed_tuning():
    import json
    import ibs_b200 as ib
    best = json.loads((ib.PKG_DIR / "tuning" / "b200.json").read_text())["best"]
    t = ib.get_tuning().as_dict()
    for key in ("span_len", "blocks_in_flight", "block_threads", "ctas_per_sm", "keys_per_bucket",
                "table_format"):
        assert t[key] == best[key], key
    assert best["rows_equal"]
    res = json.loads((ib.PKG_DIR / "tuning" / "b200.json").read_text())
    pb = res["panel_best"]
    for key in ("panel_span_len", "panel_ctas_per_sm", "panel_keys_per_bucket", "panel_blocks_in_flight",
                "panel_pass_mb"):
        assert t[key] == pb[key], key
    assert res["panel"]["all_rows_equal"]


def test_python_structs_match_the_c_header(tmp_path):
    """ctypes mirrors of the header's structs: same size and field offsets
    as the C compiler lays them out."""
    import subprocess
    structs = {"ibs_tuning": ib.Tuning, "ibs_server_opts": ib.ServerOpts, "ibs_server_stats": ib.ServerStats,
               "ibs_table_opts": ib.TableOpts, "ibs_table_info": ib.TableInfo,
               "ibs_request_result": ib.RequestResult}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ibs.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "sizes.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(REPO / "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out if ln}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
