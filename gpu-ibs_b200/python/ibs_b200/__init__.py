"""ctypes binding of the B200 fastibs scan library (libibs.so) and its tools
library (libibs_tools.so), for tests and benchmarks.

The scan itself runs only on the GPU through libibs.so; there is no Python or
CPU implementation behind these calls. Loading fails loudly when the built
libraries are missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parents[2]  # gpu-ibs_b200/
LIB_DIR = PKG_DIR / "lib"

IBS_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "ERR_ARG", 2: "ERR_IO", 3: "ERR_FORMAT", 4: "ERR_CUDA", 5: "ERR_NOMEM",
    6: "ERR_UNSUPPORTED", 7: "ERR_CAPACITY", 8: "ERR_TIMEOUT", 9: "ERR_STATE",
}

WINDOW_DTYPE = np.dtype([("start", "<i4"), ("end", "<i4"), ("total_kmers", "<i4"),
                         ("observed_kmers", "<i4"), ("variations", "<i4"),
                         ("kmer_distance", "<i4")])


class IbsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _load(name: str) -> C.CDLL:
    path = LIB_DIR / name
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `make -C {PKG_DIR}` "
                          "(the scan has no fallback without its CUDA library)")
    return C.CDLL(str(path))


_lib = _load("libibs.so")
_tools = _load("libibs_tools.so")

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
vp = C.c_void_p


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("memory_budget", C.c_uint64), ("max_spans_per_launch", C.c_uint32),
                ("min_spans_per_request", C.c_uint32), ("one_request_per_launch", C.c_uint32),
                ("table_format", C.c_uint32), ("keys_per_bucket", C.c_double),
                ("iteration_launches", C.c_uint32), ("idle_exit_us", C.c_uint32)]


class RequestResult(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("sample", C.c_uint32), ("contig", C.c_uint32),
                ("first_window", C.c_uint64), ("n_windows", C.c_uint64), ("status", C.c_int),
                ("submit_time", C.c_double), ("done_time", C.c_double), ("rows", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "launches", "spans", "probes", "reloads",
                                          "reload_bytes", "evictions", "resident_bytes", "resident_tables")] + \
               [(n, C.c_double) for n in ("busy_seconds", "latency_p50", "latency_p99", "latency_max")] + \
               [(n, C.c_uint64) for n in ("failed", "queued", "running", "scanned", "sample_probes",
                                          "persistent_launches", "idle_exits", "wait_timeouts", "replays",
                                          "lookup_failures", "fold_giveups")]


class Tuning(C.Structure):
    _fields_ = [("span_len", C.c_uint32), ("blocks_in_flight", C.c_uint32), ("block_threads", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("keys_per_bucket", C.c_double), ("table_format", C.c_uint32),
                ("panel_pass_mb", C.c_uint32), ("panel_span_len", C.c_uint32), ("panel_ctas_per_sm", C.c_uint32),
                ("panel_keys_per_bucket", C.c_double), ("panel_blocks_in_flight", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


class TableOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("keys_per_bucket", C.c_double),
                ("force_format", C.c_uint32), ("reserved", C.c_uint32 * 5)]


class TableInfo(C.Structure):
    _fields_ = [("k", C.c_uint32), ("format", C.c_uint32), ("fp_bits", C.c_uint32),
                ("reserved0", C.c_uint32), ("n_keys", C.c_uint64), ("n_buckets", C.c_uint64),
                ("stash_keys", C.c_uint64), ("stash_buckets", C.c_uint64),
                ("device_bytes", C.c_uint64), ("build_seconds", C.c_double)]


class SynthRefSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_contigs", C.c_uint32), ("reserved0", C.c_uint32),
                ("lens", u64p), ("n_frac", C.c_double), ("n_run_min", C.c_uint32),
                ("n_run_max", C.c_uint32), ("lower_frac", C.c_double),
                ("lower_run_min", C.c_uint32), ("lower_run_max", C.c_uint32)]


class SynthSampleSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("k", C.c_uint32), ("n_classes", C.c_uint32),
                ("block_len", C.c_uint64), ("class_rate", C.c_double * 4),
                ("class_prob", C.c_double * 4), ("present_frac", C.c_double),
                ("random_frac", C.c_double), ("n_intro", C.c_uint32), ("reserved0", C.c_uint32),
                ("intro_contig", u32p), ("intro_start", u64p), ("intro_len", u64p),
                ("intro_rate", C.c_double)]


class KmcSpec(C.Structure):
    _fields_ = [("k", C.c_uint32), ("p", C.c_uint32), ("sig_len", C.c_uint32),
                ("n_bins", C.c_uint32), ("counter_size", C.c_uint32), ("version", C.c_uint32),
                ("min_count", C.c_uint32), ("max_count", C.c_uint32), ("count_seed", C.c_uint64)]


def _sig(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_ibs_open = _sig(_lib, "ibs_open", C.c_int, [C.c_char_p, C.POINTER(TableOpts), C.POINTER(vp)])
_ibs_from_codes = _sig(_lib, "ibs_table_from_codes", C.c_int,
                       [vp, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(TableOpts), C.POINTER(vp)])
_ibs_info = _sig(_lib, "ibs_table_info_get", C.c_int, [vp, C.POINTER(TableInfo)])
_ibs_probe = _sig(_lib, "ibs_probe", C.c_int, [vp, vp, C.c_uint64, vp])
_ibs_from_codes128 = _sig(_lib, "ibs_table_from_codes128", C.c_int,
                          [vp, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(TableOpts), C.POINTER(vp)])
_ibs_probe128 = _sig(_lib, "ibs_probe128", C.c_int, [vp, vp, C.c_uint64, vp])
_ibs_close = _sig(_lib, "ibs_close", None, [vp])
_ibs_count_present = _sig(_lib, "ibs_count_present", C.c_int, [vp, vp, C.c_uint64, C.c_int, u64p])
_ibs_count_present_kmc = _sig(_lib, "ibs_count_present_kmc", C.c_int, [vp, C.c_char_p, u64p])
_ibs_packed_words = _sig(_lib, "ibs_packed_words", None, [vp, C.c_uint32, u64p, u64p])
_ibs_pack_ascii = _sig(_lib, "ibs_pack_ascii", C.c_int,
                       [C.POINTER(C.c_char_p), vp, C.c_uint32, vp, vp, C.c_int])
_ibs_ref_create = _sig(_lib, "ibs_reference_create", C.c_int,
                       [vp, vp, vp, C.c_uint32, C.c_int, C.POINTER(vp)])
_ibs_ref_create_dev = _sig(_lib, "ibs_reference_create_device", C.c_int,
                           [vp, vp, vp, C.c_uint32, C.c_int, C.POINTER(vp)])
_ibs_ref_free = _sig(_lib, "ibs_reference_free", None, [vp])
_ibs_ref_from_fasta = _sig(_lib, "ibs_reference_from_fasta", C.c_int, [C.c_char_p, C.c_uint64, C.c_int, C.POINTER(vp)])
_ibs_ref_ncontigs = _sig(_lib, "ibs_reference_contig_count", C.c_uint32, [vp])
_ibs_ref_contig = _sig(_lib, "ibs_reference_contig", C.c_int, [vp, C.c_uint32, u64p, C.POINTER(C.c_char_p)])
_ibs_ref_copy = _sig(_lib, "ibs_reference_copy_packed", C.c_int, [vp, vp, vp])
_ibs_map_cov = _sig(_lib, "ibs_map_coverage", C.c_int, [vp, vp, vp, C.c_uint64])
_ibs_map_text = _sig(_lib, "ibs_map_text", C.c_int, [vp, vp, vp, C.POINTER(C.c_void_p), u64p])
_ibs_map_text_free = _sig(_lib, "ibs_map_text_free", None, [vp])
_ibs_window_count = _sig(_lib, "ibs_window_count", C.c_uint64, [vp, C.c_uint32, C.c_uint32, C.c_uint32])
_ibs_window_bounds = _sig(_lib, "ibs_window_bounds", C.c_int,
                          [vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint64])
_ibs_scan = _sig(_lib, "ibs_scan", C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint64])
_ibs_scan_async = _sig(_lib, "ibs_scan_async", C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint64, vp])
_ibs_scan_packed = _sig(_lib, "ibs_scan_packed", C.c_int,
                        [vp, vp, vp, vp, C.c_uint32, C.c_uint32, vp, C.c_uint64])
_ibs_scan_panel = _sig(_lib, "ibs_scan_panel", C.c_int,
                       [C.POINTER(vp), C.c_uint32, vp, C.c_uint32, vp, C.c_uint64])
_ibs_scan_noalloc = _sig(_lib, "ibs_scan_noalloc", C.c_int,
                         [vp, vp, vp, vp, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp])
_ibs_pt_create = _sig(_lib, "ibs_panel_table_create", C.c_int,
                      [C.c_uint32, C.c_uint64, C.POINTER(TableOpts), C.POINTER(vp)])
_ibs_pt_add_kmc = _sig(_lib, "ibs_panel_table_add_kmc", C.c_int, [vp, C.c_char_p])
_ibs_pt_add_codes = _sig(_lib, "ibs_panel_table_add_codes", C.c_int, [vp, vp, C.c_uint64, C.c_int])
_ibs_pt_info = _sig(_lib, "ibs_panel_table_info_get", C.c_int, [vp, C.POINTER(TableInfo), u32p])
_ibs_pt_probe = _sig(_lib, "ibs_panel_table_probe", C.c_int, [vp, vp, C.c_uint64, vp])
_ibs_pt_scan = _sig(_lib, "ibs_panel_table_scan", C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint64])
_ibs_pt_scan_async = _sig(_lib, "ibs_panel_table_scan_async", C.c_int,
                          [vp, vp, C.c_uint32, vp, C.c_uint64, vp])
_ibs_pt_close = _sig(_lib, "ibs_panel_table_close", None, [vp])
_ibs_table_bytes_for = _sig(_lib, "ibs_table_bytes_for", C.c_uint64, [C.c_uint64, C.c_uint32, C.POINTER(TableOpts)])
_ibs_device_memory = _sig(_lib, "ibs_device_memory", C.c_int, [C.c_int, u64p, u64p])
_ibs_srv_create = _sig(_lib, "ibs_server_create", C.c_int,
                       [vp, C.c_uint32, C.c_uint32, C.POINTER(ServerOpts), C.POINTER(vp)])
_ibs_srv_add_kmc = _sig(_lib, "ibs_server_add_sample_kmc", C.c_int, [vp, C.c_char_p, u32p])
_ibs_srv_add_codes = _sig(_lib, "ibs_server_add_sample_codes", C.c_int, [vp, vp, C.c_uint64, C.c_int, u32p])
_ibs_srv_add_panel = _sig(_lib, "ibs_server_add_panel", C.c_int, [vp, vp, C.c_int, u32p])
_ibs_srv_submit = _sig(_lib, "ibs_server_submit", C.c_int,
                       [vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, u64p])
_ibs_srv_poll = _sig(_lib, "ibs_server_poll", C.c_int,
                     [vp, C.POINTER(RequestResult), C.c_uint32, u32p, C.c_int])
_ibs_srv_release = _sig(_lib, "ibs_server_release", None, [vp, C.POINTER(RequestResult)])
_ibs_srv_stats = _sig(_lib, "ibs_server_stats_get", C.c_int, [vp, C.POINTER(ServerStats)])
_ibs_srv_now = _sig(_lib, "ibs_server_now", C.c_double, [vp])
_ibs_srv_close = _sig(_lib, "ibs_server_close", None, [vp])
_ibs_set_tuning = _sig(_lib, "ibs_set_tuning", C.c_int, [C.POINTER(Tuning)])
_ibs_get_tuning = _sig(_lib, "ibs_get_tuning", None, [C.POINTER(Tuning)])
_ibs_last_error = _sig(_lib, "ibs_last_error", C.c_char_p, [])
_ibs_device_count = _sig(_lib, "ibs_device_count", C.c_int, [])
_ibs_launch_count = _sig(_lib, "ibs_launch_count", C.c_uint64, [])

_t_n_runs = _sig(_tools, "ibs_synth_n_runs", C.c_uint64,
                 [C.POINTER(SynthRefSpec), vp, vp, vp, C.c_uint64])
_t_reference = _sig(_tools, "ibs_synth_reference", C.c_int, [C.POINTER(SynthRefSpec), vp, vp, C.c_int])
_t_contig_ascii = _sig(_tools, "ibs_synth_contig_ascii", C.c_int,
                       [C.POINTER(SynthRefSpec), C.c_uint32, vp])
_t_write_fasta = _sig(_tools, "ibs_synth_write_fasta", C.c_int,
                      [C.POINTER(SynthRefSpec), C.c_char_p, C.POINTER(C.c_char_p), C.c_uint32])
_t_sample_codes = _sig(_tools, "ibs_synth_sample_codes", C.c_int,
                       [C.POINTER(SynthRefSpec), C.POINTER(SynthSampleSpec), vp, vp, C.c_int, vp,
                        C.c_uint64, u64p])
_t_kmc_write128 = _sig(_tools, "ibs_kmc_write128", C.c_int, [C.c_char_p, C.POINTER(KmcSpec), vp, C.c_uint64, u64p])
_t_kmc_write = _sig(_tools, "ibs_kmc_write", C.c_int,
                    [C.c_char_p, C.POINTER(KmcSpec), vp, C.c_uint64, C.c_int, u64p])
_t_sort_unique = _sig(_tools, "ibs_sort_unique_host", C.c_uint64, [vp, C.c_uint64, C.c_int])
_t_last_error = _sig(_tools, "ibs_tools_last_error", C.c_char_p, [])
_t_sector_rate = _sig(_tools, "ibs_random_sector_rate", C.c_int, [C.c_uint64, C.POINTER(C.c_double)])


def _check(status: int, tools: bool = False):
    if status != IBS_OK:
        msg = (_t_last_error() if tools else _ibs_last_error()) or b""
        raise IbsError(status, msg.decode(errors="replace"))


def _ptr(a) -> int:
    """Address of a numpy array, a torch tensor, or an int device pointer."""
    if a is None:
        return 0
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(type(a))


def set_tuning(t: Tuning):
    _check(_ibs_set_tuning(C.byref(t)))


def get_tuning() -> Tuning:
    t = Tuning()
    _ibs_get_tuning(C.byref(t))
    return t


def device_count() -> int:
    return _ibs_device_count()


def launch_count() -> int:
    return _ibs_launch_count()


def library_paths() -> list[str]:
    return [str(LIB_DIR / "libibs.so"), str(LIB_DIR / "libibs_tools.so")]


# ---------------------------------------------------------------------------
# tables
# ---------------------------------------------------------------------------
class Table:
    """One sample's device-resident k-mer table (ibs_table)."""

    def __init__(self, handle: int):
        self._h = handle

    @classmethod
    def open(cls, kmc_prefix: str, device: int = 0, keys_per_bucket: float = 0.0,
             force_format: int = 0) -> "Table":
        opts = TableOpts(device, keys_per_bucket, force_format)
        h = vp()
        _check(_ibs_open(str(kmc_prefix).encode(), C.byref(opts), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_codes(cls, codes, n: int, k: int, on_device: bool, device: int = 0,
                   keys_per_bucket: float = 0.0, force_format: int = 0) -> "Table":
        opts = TableOpts(device, keys_per_bucket, force_format)
        h = vp()
        _check(_ibs_from_codes(_ptr(codes), n, k, int(on_device), C.byref(opts), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_codes128(cls, lo, hi, k: int, device: int = 0, keys_per_bucket: float = 0.0) -> "Table":
        """A wide-key table (33 <= k <= 64) from canonical codes given as their
        low and high 64-bit words (host arrays)."""
        codes = pairs128(lo, hi)
        opts = TableOpts(device, keys_per_bucket, 0)
        h = vp()
        _check(_ibs_from_codes128(_ptr(codes), len(codes) // 2, k, 0, C.byref(opts), C.byref(h)))
        return cls(h.value)

    @property
    def handle(self) -> int:
        return self._h

    def info(self) -> TableInfo:
        i = TableInfo()
        _check(_ibs_info(self._h, C.byref(i)))
        return i

    def probe128(self, lo, hi) -> np.ndarray:
        """Membership of wide codes (low / high words) in a wide-key table."""
        codes = pairs128(lo, hi)
        hits = np.zeros(len(codes) // 2, dtype=np.uint8)
        _check(_ibs_probe128(self._h, _ptr(codes), len(codes) // 2, _ptr(hits)))
        return hits

    def count_present(self, codes, n: int | None = None, on_device: bool = False) -> int:
        """How many of the codes the table holds (ibs_count_present)."""
        if not on_device:
            codes = np.ascontiguousarray(codes, dtype=np.uint64)
            n = len(codes)
        c = C.c_uint64()
        _check(_ibs_count_present(self._h, _ptr(codes), n, int(on_device), C.byref(c)))
        return c.value

    def count_present_kmc(self, prefix: str) -> int:
        """Size of the intersection with a KMC database's k-mers (ibs_count_present_kmc)."""
        c = C.c_uint64()
        _check(_ibs_count_present_kmc(self._h, str(prefix).encode(), C.byref(c)))
        return c.value

    def probe(self, codes: np.ndarray) -> np.ndarray:
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        hits = np.zeros(len(codes), dtype=np.uint8)
        _check(_ibs_probe(self._h, _ptr(codes), len(codes), _ptr(hits)))
        return hits

    def close(self):
        if self._h:
            _ibs_close(self._h)
            self._h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PanelTable:
    """A joint table over up to 16 samples (ibs_panel_table)."""

    MAX_SAMPLES = 16

    def __init__(self, k: int, expected_keys: int, device: int = 0, keys_per_bucket: float = 0.0,
                 force_format: int = 0):
        """force_format: 0 = by size (minimizer lines for 16 <= k <= 27 when large
        enough), 3 = hash sectors, 7 = minimizer lines."""
        opts = TableOpts(device, keys_per_bucket, force_format)
        h = vp()
        _check(_ibs_pt_create(k, expected_keys, C.byref(opts), C.byref(h)))
        self._h = h.value

    @property
    def handle(self) -> int:
        return self._h

    def add_kmc(self, prefix: str):
        _check(_ibs_pt_add_kmc(self._h, str(prefix).encode()))

    def add_codes(self, codes, n: int, on_device: bool):
        _check(_ibs_pt_add_codes(self._h, _ptr(codes), n, int(on_device)))

    def info(self):
        i = TableInfo()
        ns = C.c_uint32()
        _check(_ibs_pt_info(self._h, C.byref(i), C.byref(ns)))
        return i, ns.value

    def probe(self, codes) -> np.ndarray:
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        masks = np.zeros(len(codes), dtype=np.uint32)
        _check(_ibs_pt_probe(self._h, _ptr(codes), len(codes), _ptr(masks)))
        return masks

    def scan(self, ref: "Reference", W: int) -> np.ndarray:
        k = self.info()[0].k
        ns = self.info()[1]
        n = window_count(ref.lens, W, k)
        rows = np.zeros(max(n * ns, 1), dtype=WINDOW_DTYPE)
        _check(_ibs_pt_scan(self._h, ref.handle, W, _ptr(rows), n * ns))
        return rows[: n * ns].reshape(ns, n)

    def scan_async(self, ref: "Reference", W: int, rows_dev, cap: int, stream: int = 0):
        _check(_ibs_pt_scan_async(self._h, ref.handle, W, _ptr(rows_dev), cap, stream))

    def close(self):
        if self._h:
            _ibs_pt_close(self._h)
            self._h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def table_bytes_for(n_keys: int, k: int, force_format: int = 0, keys_per_bucket: float = 0.0) -> int:
    if not force_format and not keys_per_bucket:
        return _ibs_table_bytes_for(n_keys, k, None)
    opts = TableOpts(0, keys_per_bucket, force_format)
    return _ibs_table_bytes_for(n_keys, k, C.byref(opts))


def device_memory(device: int = 0) -> tuple[int, int]:
    f, t = C.c_uint64(), C.c_uint64()
    _check(_ibs_device_memory(device, C.byref(f), C.byref(t)))
    return f.value, t.value


# ---------------------------------------------------------------------------
# references
# ---------------------------------------------------------------------------
def packed_words(lens) -> tuple[int, int]:
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    sw, mw = C.c_uint64(), C.c_uint64()
    _ibs_packed_words(_ptr(lens), len(lens), C.byref(sw), C.byref(mw))
    return sw.value, mw.value


def pack_ascii(seqs: list[bytes], threads: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    lens = np.array([len(s) for s in seqs], dtype=np.uint64)
    sw, mw = packed_words(lens)
    seq = np.zeros(sw, dtype=np.uint64)
    mask = np.zeros(mw, dtype=np.uint64)
    arr = (C.c_char_p * max(1, len(seqs)))(*seqs)
    _check(_ibs_pack_ascii(arr, _ptr(lens), len(seqs), _ptr(seq), _ptr(mask), threads))
    return seq, mask, lens


class Reference:
    """A device-resident packed reference (ibs_reference)."""

    def __init__(self, seq2bit, nmask, lens, device: int = 0, on_device: bool = False):
        self.lens = np.ascontiguousarray(lens, dtype=np.uint64)
        h = vp()
        fn = _ibs_ref_create_dev if on_device else _ibs_ref_create
        _check(fn(_ptr(seq2bit), _ptr(nmask), _ptr(self.lens), len(self.lens), device, C.byref(h)))
        self._h = h.value

    @classmethod
    def from_fasta(cls, text: bytes, device: int = 0) -> "Reference":
        """Parses and packs FASTA text on the device (ibs_reference_from_fasta);
        `ids` and `lens` are its contigs."""
        h = vp()
        _check(_ibs_ref_from_fasta(text, len(text), device, C.byref(h)))
        r = cls.__new__(cls)
        r._h = h.value
        n = _ibs_ref_ncontigs(r._h)
        lens, ids = np.zeros(n, dtype=np.uint64), []
        for i in range(n):
            ln, idp = C.c_uint64(), C.c_char_p()
            _check(_ibs_ref_contig(r._h, i, C.byref(ln), C.byref(idp)))
            lens[i] = ln.value
            ids.append(idp.value)
        r.lens, r.ids = lens, ids
        return r

    def copy_packed(self):
        """The packed (seq2bit, nmask) arrays back on the host."""
        sw, mw = packed_words(self.lens)
        seq, mask = np.zeros(sw, np.uint64), np.zeros(mw, np.uint64)
        _check(_ibs_ref_copy(self._h, _ptr(seq), _ptr(mask)))
        return seq, mask

    @property
    def handle(self) -> int:
        return self._h

    def free(self):
        if self._h:
            _ibs_ref_free(self._h)
            self._h = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def map_coverage(table: "Table", ref: Reference) -> np.ndarray:
    """Per-base k-mer coverage of every contig, concatenated (ibs_map_coverage)."""
    n = int(np.sum(ref.lens))
    cov = np.zeros(max(n, 1), dtype=np.uint8)
    _check(_ibs_map_cov(table.handle, ref.handle, _ptr(cov), n))
    return cov[:n]


def map_text(table: "Table", ref: Reference, ids: list[bytes] | None = None) -> bytes:
    """The mapper's output text (ibs_map_text)."""
    arr = (C.c_char_p * len(ids))(*ids) if ids is not None else None
    p, n = C.c_void_p(), C.c_uint64()
    _check(_ibs_map_text(table.handle, ref.handle, arr, C.byref(p), C.byref(n)))
    try:
        return C.string_at(p.value, n.value) if n.value else b""
    finally:
        _ibs_map_text_free(p.value)


def window_count(lens, W: int, k: int) -> int:
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    return _ibs_window_count(_ptr(lens), len(lens), W, k)


def window_bounds(lens, W: int, k: int) -> np.ndarray:
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    n = window_count(lens, W, k)
    rows = np.zeros(n, dtype=WINDOW_DTYPE)
    _check(_ibs_window_bounds(_ptr(lens), len(lens), W, k, _ptr(rows), n))
    return rows


def scan(table: Table, ref: Reference, W: int) -> np.ndarray:
    n = window_count(ref.lens, W, table.info().k)
    rows = np.zeros(max(n, 1), dtype=WINDOW_DTYPE)
    _check(_ibs_scan(table.handle, ref.handle, W, _ptr(rows), n))
    return rows[:n]


def scan_async(table: Table, ref: Reference, W: int, rows_dev, cap: int, stream: int = 0):
    _check(_ibs_scan_async(table.handle, ref.handle, W, _ptr(rows_dev), cap, stream))


def scan_packed(table: Table, seq2bit, nmask, lens, W: int, rows=None) -> np.ndarray:
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    n = window_count(lens, W, table.info().k)
    if rows is None:
        rows = np.zeros(max(n, 1), dtype=WINDOW_DTYPE)
    _check(_ibs_scan_packed(table.handle, _ptr(seq2bit), _ptr(nmask), _ptr(lens), len(lens), W,
                            _ptr(rows), n))
    return rows[:n] if isinstance(rows, np.ndarray) else rows


def scan_noalloc(table: Table, seq2bit_dev, nmask_dev, lens, W: int, rows_dev, cap: int,
                 stream: int = 0):
    """ibs_scan_noalloc: the scan with its scratch in the library's fixed
    device array (no allocation); every pointer but lens is device memory."""
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    _check(_ibs_scan_noalloc(table.handle, _ptr(seq2bit_dev), _ptr(nmask_dev), _ptr(lens), len(lens), W,
                             _ptr(rows_dev), cap, stream))


def scan_panel(tables: list[Table], ref: Reference, W: int) -> np.ndarray:
    k = tables[0].info().k
    n = window_count(ref.lens, W, k)
    rows = np.zeros(max(n * len(tables), 1), dtype=WINDOW_DTYPE)
    arr = (vp * len(tables))(*[t.handle for t in tables])
    _check(_ibs_scan_panel(arr, len(tables), ref.handle, W, _ptr(rows), n * len(tables)))
    return rows[: n * len(tables)].reshape(len(tables), n)


# ---------------------------------------------------------------------------
# synthetic inputs and the KMC writer (libibs_tools.so)
# ---------------------------------------------------------------------------
class RefSpec:
    def __init__(self, seed: int, lens, n_frac=0.0, n_run=(50, 500), lower_frac=0.0,
                 lower_run=(20, 200), names=None):
        self.lens = np.ascontiguousarray(lens, dtype=np.uint64)
        self.names = list(names) if names else [f"chr{i + 1}" for i in range(len(self.lens))]
        self.c = SynthRefSpec(seed, len(self.lens), 0, self.lens.ctypes.data_as(u64p), n_frac,
                              n_run[0], n_run[1], lower_frac, lower_run[0], lower_run[1])

    def packed_words(self):
        return packed_words(self.lens)

    def reference_host(self):
        sw, mw = self.packed_words()
        seq = np.zeros(sw, dtype=np.uint64)
        mask = np.zeros(mw, dtype=np.uint64)
        _check(_t_reference(C.byref(self.c), _ptr(seq), _ptr(mask), 0), tools=True)
        return seq, mask

    def reference_device(self, seq_dev, mask_dev):
        _check(_t_reference(C.byref(self.c), _ptr(seq_dev), _ptr(mask_dev), 1), tools=True)

    def contig_ascii(self, c: int) -> bytes:
        buf = C.create_string_buffer(int(self.lens[c]) + 1)
        _check(_t_contig_ascii(C.byref(self.c), c, C.addressof(buf)), tools=True)
        return buf.raw[: int(self.lens[c])]

    def write_fasta(self, path: str, width: int = 80):
        names = (C.c_char_p * len(self.names))(*[n.encode() for n in self.names])
        _check(_t_write_fasta(C.byref(self.c), str(path).encode(), names, width), tools=True)

    def n_runs(self):
        n = _t_n_runs(C.byref(self.c), None, None, None, 0)
        c = np.zeros(n, np.uint32)
        s = np.zeros(n, np.uint64)
        ln = np.zeros(n, np.uint64)
        _t_n_runs(C.byref(self.c), _ptr(c), _ptr(s), _ptr(ln), n)
        return c, s, ln


class SampleSpec:
    def __init__(self, seed: int, k: int, class_rate=(0.01,), class_prob=(1.0,),
                 block_len=1 << 20, present_frac=1.0, random_frac=0.0, intro=(), intro_rate=0.0001):
        rates = list(class_rate) + [0.0] * (4 - len(class_rate))
        probs = list(class_prob) + [0.0] * (4 - len(class_prob))
        self._ic = np.array([i[0] for i in intro] or [0], dtype=np.uint32)
        self._is = np.array([i[1] for i in intro] or [0], dtype=np.uint64)
        self._il = np.array([i[2] for i in intro] or [0], dtype=np.uint64)
        self.k = k
        self.c = SynthSampleSpec(seed, k, len(class_rate), block_len, (C.c_double * 4)(*rates),
                                 (C.c_double * 4)(*probs), present_frac, random_frac, len(intro), 0,
                                 self._ic.ctypes.data_as(u32p), self._is.ctypes.data_as(u64p),
                                 self._il.ctypes.data_as(u64p), intro_rate)

    def codes_host(self, ref: RefSpec, seq, mask) -> np.ndarray:
        n = C.c_uint64()
        _check(_t_sample_codes(C.byref(ref.c), C.byref(self.c), _ptr(seq), _ptr(mask), 0, None, 0,
                               C.byref(n)), tools=True)
        out = np.zeros(max(n.value, 1), dtype=np.uint64)
        _check(_t_sample_codes(C.byref(ref.c), C.byref(self.c), _ptr(seq), _ptr(mask), 0, _ptr(out),
                               n.value, C.byref(n)), tools=True)
        return out[: n.value]

    def codes_device_bound(self, ref: RefSpec, seq_dev, mask_dev) -> int:
        n = C.c_uint64()
        _check(_t_sample_codes(C.byref(ref.c), C.byref(self.c), _ptr(seq_dev), _ptr(mask_dev), 1, None,
                               0, C.byref(n)), tools=True)
        return n.value

    def codes_device(self, ref: RefSpec, seq_dev, mask_dev, out_dev, cap: int) -> int:
        n = C.c_uint64()
        _check(_t_sample_codes(C.byref(ref.c), C.byref(self.c), _ptr(seq_dev), _ptr(mask_dev), 1,
                               _ptr(out_dev), cap, C.byref(n)), tools=True)
        return n.value


def kmc_write(prefix: str, codes, n: int, k: int, p: int, sig_len: int = 9, n_bins: int = 512,
              counter_size: int = 1, version: int = 0x200, min_count: int = 2, max_count: int = 255,
              count_seed: int = 7, on_device: bool = False) -> int:
    spec = KmcSpec(k, p, sig_len, n_bins, counter_size, version, min_count, max_count, count_seed)
    out = C.c_uint64()
    _check(_t_kmc_write(str(prefix).encode(), C.byref(spec), _ptr(codes), n, int(on_device),
                        C.byref(out)), tools=True)
    return out.value


def pairs128(lo, hi) -> np.ndarray:
    """Low / high word arrays -> the interleaved {lo, hi} layout of ibs_code128."""
    lo = np.ascontiguousarray(lo, dtype=np.uint64)
    hi = np.ascontiguousarray(hi, dtype=np.uint64)
    if lo.shape != hi.shape:
        raise ValueError("lo and hi differ in length")
    out = np.empty(2 * len(lo), dtype=np.uint64)
    out[0::2] = lo
    out[1::2] = hi
    return out


def kmc_write128(prefix: str, lo, hi, k: int, p: int, sig_len: int = 9, n_bins: int = 512,
                 counter_size: int = 1, version: int = 0x200, min_count: int = 2, max_count: int = 255,
                 count_seed: int = 7) -> int:
    """KMC 3 database of 33 <= k <= 64 k-mers given as low / high words (host)."""
    spec = KmcSpec(k, p, sig_len, n_bins, counter_size, version, min_count, max_count, count_seed)
    codes = pairs128(lo, hi)
    out = C.c_uint64()
    _check(_t_kmc_write128(str(prefix).encode(), C.byref(spec), _ptr(codes), len(codes) // 2, C.byref(out)),
           tools=True)
    return out.value


def sort_unique_host(codes: np.ndarray, threads: int = 0) -> np.ndarray:
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    n = _t_sort_unique(_ptr(codes), len(codes), threads)
    return codes[:n]


def random_sector_rate(nbytes: int) -> float:
    """Random 32-byte sector reads per second over a device buffer of nbytes."""
    r = C.c_double()
    _check(_t_sector_rate(nbytes, C.byref(r)), tools=True)
    return r.value


class Server:
    """The serving loop (ibs_server): requests of (sample, contig, window range)."""

    def __init__(self, ref: Reference, W: int, k: int, memory_budget: int = 0, max_spans_per_launch: int = 0,
                 min_spans_per_request: int = 0, device: int = 0, one_request_per_launch: bool = False,
                 table_format: int = 0, keys_per_bucket: float = 0.0, iteration_launches: bool = False,
                 idle_exit_us: int = 0):
        self.ref = ref
        opts = ServerOpts(device, memory_budget, max_spans_per_launch, min_spans_per_request,
                          int(one_request_per_launch), table_format, keys_per_bucket, int(iteration_launches),
                          idle_exit_us)
        h = vp()
        _check(_ibs_srv_create(ref.handle, W, k, C.byref(opts), C.byref(h)))
        self._h = h.value

    def add_codes(self, codes, n: int, on_device: bool) -> int:
        i = C.c_uint32()
        _check(_ibs_srv_add_codes(self._h, _ptr(codes), n, int(on_device), C.byref(i)))
        return i.value

    def add_kmc(self, prefix: str) -> int:
        i = C.c_uint32()
        _check(_ibs_srv_add_kmc(self._h, str(prefix).encode(), C.byref(i)))
        return i.value

    def add_panel(self, panel: "PanelTable", release: bool = False) -> list[int]:
        """Registers every sample of a joint panel table; returns their ids.
        With release=True the panel's device table is freed first (the panel
        then only accepts close())."""
        ns = panel.info()[1]
        i = C.c_uint32()
        _check(_ibs_srv_add_panel(self._h, panel._h, int(release), C.byref(i)))
        return list(range(i.value, i.value + ns))

    def submit(self, sample: int, contig: int, first_window: int = 0, n_windows: int = 0) -> int:
        rid = C.c_uint64()
        _check(_ibs_srv_submit(self._h, sample, contig, first_window, n_windows, C.byref(rid)))
        return rid.value

    def poll(self, max_results: int = 64, timeout_ms: int = 0) -> list[dict]:
        buf = (RequestResult * max_results)()
        n = C.c_uint32()
        if timeout_ms < 0:  # wait in bounded slices so that Python signals are still handled
            while True:
                _check(_ibs_srv_poll(self._h, buf, max_results, C.byref(n), 1000))
                if n.value:
                    break
        else:
            _check(_ibs_srv_poll(self._h, buf, max_results, C.byref(n), timeout_ms))
        out = []
        for i in range(n.value):
            r = buf[i]
            rows = np.ctypeslib.as_array(C.cast(r.rows, C.POINTER(C.c_int32)),
                                         shape=(max(int(r.n_windows), 1) * 6,)).copy().view(WINDOW_DTYPE)
            out.append(dict(request_id=r.request_id, sample=r.sample, contig=r.contig,
                            first_window=r.first_window, n_windows=r.n_windows, status=r.status,
                            submit_time=r.submit_time, done_time=r.done_time,
                            rows=rows[: int(r.n_windows)]))
            _ibs_srv_release(self._h, C.byref(buf[i]))
        return out

    def stats(self) -> dict:
        st = ServerStats()
        _check(_ibs_srv_stats(self._h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in ServerStats._fields_}

    def now(self) -> float:
        return _ibs_srv_now(self._h)

    def close(self):
        if self._h:
            _ibs_srv_close(self._h)
            self._h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
