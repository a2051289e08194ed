"""ctypes declarations of the libspk C ABI (include/spk.h)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB = None

SPK_F_EDGES = 0x1
SPK_F_REF_SOLID = 0x2
SPK_F_KEEP_BLOOM = 0x4
SPK_F_GATED = 0x8
SPK_F_DIRECT = 0x10
SPK_F_CORRECT = 0x20
SPK_F_KEEP_TABLE = 0x40
SPK_NOALLOC_MAX_KEYS = 65536
SPK_SCHEDULE_GATED = 0
SPK_SCHEDULE_FUSED = 1
SPK_SCHEDULE_COUNT_FIRST = 2
SPK_SCHEDULE_PARTITIONED = 3

STATUS = {
    0: "SPK_OK", 1: "SPK_E_INVALID_ARG", 2: "SPK_E_INVALID_K", 3: "SPK_E_OOM",
    4: "SPK_E_TABLE_FULL", 5: "SPK_E_TIMEOUT", 6: "SPK_E_CUDA", 7: "SPK_E_NO_DEVICE",
    8: "SPK_E_ADMISSION", 9: "SPK_E_NOT_READY", 10: "SPK_E_NOT_FOUND",
}

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p


class SpkError(RuntimeError):
    """A libspk call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.name = STATUS.get(code, str(code))
        super().__init__(f"{self.name}: {message}")


class CountOpts(C.Structure):
    _fields_ = [("bloom_bits", C.c_uint64), ("min_count", C.c_uint32),
                ("list_min_count", C.c_uint32), ("min_coverage", C.c_double),
                ("flags", C.c_uint32), ("table_log2", C.c_uint32),
                ("prior_seqs", C.c_void_p), ("prior_offsets", C.c_void_p),
                ("prior_lengths", C.c_void_p), ("n_prior", C.c_uint64),
                ("span_groups_log2", C.c_uint32), ("reserved", C.c_uint32),
                ("solid_keys_out", C.c_void_p), ("solid_counts_out", C.c_void_p),
                ("solid_capacity", C.c_uint64)]


class ResultInfo(C.Structure):
    _fields_ = [("k", C.c_uint32), ("cutoff", C.c_uint32), ("occurrences", C.c_uint64),
                ("admitted_occurrences", C.c_uint64), ("n_table", C.c_uint64),
                ("n_list", C.c_uint64), ("n_solid", C.c_uint64), ("n_edges", C.c_uint64),
                ("n_singletons", C.c_uint64), ("bloom_size_bits", C.c_uint64),
                ("seen_popcount", C.c_uint64), ("twice_popcount", C.c_uint64),
                ("table_capacity", C.c_uint64), ("table_regrows", C.c_uint32),
                ("kernel_launches", C.c_uint32), ("ms_bloom", C.c_float), ("ms_count", C.c_float),
                ("ms_finish", C.c_float), ("ms_sort", C.c_float), ("ms_edges", C.c_float),
                ("ms_total", C.c_float), ("ms_bloom_kernel", C.c_float),
                ("ms_count_kernel", C.c_float), ("schedule", C.c_uint32),
                ("part_rescatters", C.c_uint32), ("n_distinct", C.c_uint64),
                ("ms_scatter_kernel", C.c_float), ("ms_unitigs", C.c_float),
                ("ms_unitigs_host", C.c_float), ("unitig_launches", C.c_uint32),
                ("n_unitigs", C.c_uint64), ("n_corrected_reads", C.c_uint64),
                ("ms_correct", C.c_float), ("part_passes", C.c_uint32),
                ("span_groups", C.c_uint32), ("ms_coarse_kernel", C.c_float),
                ("solid_copied", C.c_uint32), ("reserved2", C.c_uint32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class TableView(C.Structure):
    _fields_ = [("slots", C.c_void_p), ("capacity", C.c_uint64), ("key_limbs", C.c_uint32),
                ("slot_bytes", C.c_uint32), ("k", C.c_uint32), ("cutoff", C.c_uint32),
                ("log2span", C.c_uint32), ("reserved", C.c_uint32)]


class JobC(C.Structure):
    _fields_ = [("data", C.c_void_p), ("data_len", C.c_size_t), ("offsets", C.c_void_p),
                ("lengths", C.c_void_p), ("n_reads", C.c_size_t), ("ks", C.c_void_p),
                ("n_k", C.c_int), ("opts", CountOpts)]


# (name, restype, argtypes)
_SIGS = [
    ("spk_last_error", C.c_char_p, []),
    ("spk_version", C.c_int, []),
    ("spk_validate_k", C.c_int, [C.c_uint32]),
    ("spk_ctx_create", C.c_int, [C.c_int, C.POINTER(vp)]),
    ("spk_ctx_destroy", C.c_int, [vp]),
    ("spk_ctx_memory", C.c_int, [vp, u64p, u64p]),
    ("spk_ctx_set_stream", C.c_int, [vp, vp]),
    ("spk_bloom_create", C.c_int, [vp, C.c_uint64, C.POINTER(vp)]),
    ("spk_bloom_destroy", C.c_int, [vp]),
    ("spk_bloom_size_bits", C.c_uint64, [vp]),
    ("spk_bloom_memory_usage_bytes", C.c_uint64, [vp]),
    ("spk_bloom_insert_u64", C.c_int, [vp, u64p, C.c_size_t, u8p]),
    ("spk_bloom_insert_k256", C.c_int, [vp, u64p, C.c_size_t, u8p]),
    ("spk_bloom_is_solid_u64", C.c_int, [vp, u64p, C.c_size_t, u8p]),
    ("spk_bloom_is_solid_k256", C.c_int, [vp, u64p, C.c_size_t, u8p]),
    ("spk_bloom_download", C.c_int, [vp, u64p, u64p]),
    ("spk_bloom_insert_k256_noalloc", C.c_int, [vp, vp, C.c_uint64, vp, C.c_size_t, vp, vp]),
    ("spk_bloom_correct_reads", C.c_int, [vp, C.c_uint32, vp, C.c_size_t, vp, vp, C.c_size_t, vp, vp,
                                          u64p]),
    ("spk_bloom_correct_reads_device", C.c_int, [vp, C.c_uint32, vp, C.c_size_t, vp, vp, C.c_size_t, vp,
                                                 vp, u64p]),
    ("spk_ingest", C.c_int, [vp, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.POINTER(vp)]),
    ("spk_packed_info", C.c_int, [vp, u64p, u64p, u64p, u64p, u64p]),
    ("spk_packed_stats", C.c_int, [vp, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    ("spk_packed_download", C.c_int, [vp, vp, vp, vp, vp, vp]),
    ("spk_packed_device", C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    ("spk_packed_free", C.c_int, [vp]),
    ("spk_count_opts_default", None, [C.POINTER(CountOpts)]),
    ("spk_count", C.c_int, [vp, vp, C.c_size_t, vp, vp, C.c_size_t, u32p, C.c_int,
                            C.POINTER(CountOpts), C.POINTER(vp)]),
    ("spk_count_device", C.c_int, [vp, vp, C.c_size_t, vp, vp, C.c_size_t, u32p, C.c_int,
                                   C.POINTER(CountOpts), C.POINTER(vp)]),
    ("spk_result_count", C.c_int, [vp, C.POINTER(C.c_int)]),
    ("spk_result_info_get", C.c_int, [vp, C.c_int, C.POINTER(ResultInfo)]),
    ("spk_result_solid", C.c_int, [vp, C.c_int, u64p, u32p, C.POINTER(C.c_size_t)]),
    ("spk_result_kmers", C.c_int, [vp, C.c_int, C.c_uint32, u64p, u32p, C.POINTER(C.c_size_t)]),
    ("spk_result_edges", C.c_int, [vp, C.c_int, u64p, C.POINTER(C.c_size_t)]),
    ("spk_result_bloom", C.c_int, [vp, C.c_int, u64p, u64p, u64p]),
    ("spk_result_table_view", C.c_int, [vp, C.c_int, C.POINTER(TableView)]),
    ("spk_result_unitigs", C.c_int, [vp, C.c_int, C.c_char_p, u64p, u64p, C.POINTER(C.c_double), u64p,
                                     u64p]),
    ("spk_result_free", C.c_int, [vp]),
    ("spk_count_batch", C.c_int, [vp, C.POINTER(JobC), C.c_int, C.POINTER(vp)]),
    ("spk_batch_start", C.c_int, [vp, C.POINTER(JobC), C.c_int, C.POINTER(vp)]),
    ("spk_batch_next", C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(vp)]),
    ("spk_batch_end", C.c_int, [vp]),
    ("spk_serve_start", C.c_int, [vp, C.c_uint64, C.c_int]),
    ("spk_serve_stop", C.c_int, [vp]),
    ("spk_job_hbm_estimate", C.c_int, [C.POINTER(JobC), u64p]),
    ("spk_submit", C.c_int, [vp, C.POINTER(JobC), u64p]),
    ("spk_poll", C.c_int, [vp, C.c_uint64, C.POINTER(C.c_int)]),
    ("spk_wait", C.c_int, [vp, C.c_uint64, C.c_int, C.POINTER(vp), C.POINTER(C.c_double)]),
    ("spk_diag_stuck_claim", C.c_int, [vp, C.c_uint32]),
]

EXPORTED = [s[0] for s in _SIGS]


def lib_path() -> str:
    """The in-tree libspk.so, or the build named by $SPK_LIBRARY (for example a
    build with other values of the launch-shape macros)."""
    return os.environ.get("SPK_LIBRARY") or os.path.join(_PKG_ROOT, "libspk.so")


def build(quiet: bool = True) -> str:
    """Compile libspk.so for sm_100a with the package Makefile (nvcc; no GPU needed)."""
    cmd = ["make", "-j8", "-C", _PKG_ROOT]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return lib_path()


def lib():
    """Load libspk.so; raises SpkError if it is missing (there is no fallback)."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise SpkError(7, f"{path} is not built (run `make -C {_PKG_ROOT}`)")
        L = C.CDLL(path)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def last_error() -> str:
    return lib().spk_last_error().decode(errors="replace")


def check(rc: int):
    if rc:
        raise SpkError(rc, last_error())


def validate_k(k: int) -> None:
    """The CLI's k rule (src/main.rs:11-30): raises SpkError(SPK_E_INVALID_K) if k is rejected."""
    check(lib().spk_validate_k(k))
