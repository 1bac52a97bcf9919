"""ctypes binding of librbsc.so (include/rbsc.h).

The library is loaded from this package directory only; there is no fallback:
if it is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librbsc.so")
CLI_PATH = os.path.join(PKG, "rbsc")

RBSC_OK = 0
STATUS_NAMES = {
    0: "RBSC_OK",
    -1: "RBSC_ERR_INVALID",
    -2: "RBSC_ERR_CUDA",
    -3: "RBSC_ERR_OOM",
    -4: "RBSC_ERR_NOT_CONVERGED",
    -5: "RBSC_ERR_DEVICE",
    -6: "RBSC_ERR_PARSE",
    -7: "RBSC_ERR_TOO_LARGE",
    -8: "RBSC_ERR_BUSY",
    1: "RBSC_PENDING",
}
RBSC_PENDING = 1

RELABEL_HASH = 0
RELABEL_SORT = 1

# every symbol include/rbsc.h declares (checked by the CPU test suite)
EXPORTED = [
    "rbsc_abi_version", "rbsc_opts_default", "rbsc_ctx_create", "rbsc_ctx_destroy", "rbsc_last_error",
    "rbsc_ctx_set_opts", "rbsc_refine", "rbsc_graph_upload", "rbsc_graph_from_device", "rbsc_graph_free",
    "rbsc_graph_info", "rbsc_graph_device_csr", "rbsc_graph_refine", "rbsc_graph_refine_device",
    "rbsc_graph_degree_colors", "rbsc_parse_arcs", "rbsc_host_graph_free", "rbsc_gen_rmat_device",
    "rbsc_gen_rmat_host", "rbsc_graph_profile", "rbsc_refine_noalloc", "rbsc_ctx_trim",
    "rbsc_gen_wl_batch", "rbsc_graph_batch_free", "rbsc_batch_refine", "rbsc_graph_batch_refine",
    "rbsc_gen_er_host", "rbsc_gen_lift_host", "rbsc_refine_edge_batches", "rbsc_graph_upload_streamed",
    "rbsc_gen_rmat_pinned", "rbsc_host_graph_free_pinned", "rbsc_tune_space_default", "rbsc_graph_autotune",
    "rbsc_bv_load", "rbsc_csr_save", "rbsc_csr_load", "rbsc_refine_f64",
    "rbsc_serve_opts_default", "rbsc_serve_footprint", "rbsc_serve_create", "rbsc_serve_destroy",
    "rbsc_serve_last_error", "rbsc_serve_submit", "rbsc_serve_poll", "rbsc_serve_wait", "rbsc_serve_stats_get",
]

NOALLOC_MAX_NODES = 16384
NOALLOC_MAX_ARCS = 1 << 24


class Opts(ctypes.Structure):
    _fields_ = [
        ("relabel", ctypes.c_int32),
        ("verify", ctypes.c_int32),
        ("max_rounds", ctypes.c_uint32),
        ("use_graph", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("test_hash_bits", ctypes.c_int32),
        ("no_persist", ctypes.c_int32),
        ("persist_log2", ctypes.c_int32),
        ("grid_per_sm", ctypes.c_int32),
        ("sig_kernel", ctypes.c_int32),
        ("hot_log2", ctypes.c_int32),
        ("persist_bps", ctypes.c_int32),
        ("persist_sig", ctypes.c_int32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("rounds", ctypes.c_uint32),
        ("blocks", ctypes.c_uint32),
        ("done", ctypes.c_uint32),
        ("verified", ctypes.c_uint32),
        ("repairs", ctypes.c_uint32),
        ("initial_blocks", ctypes.c_uint32),
        ("time_s", ctypes.c_double),
        ("device_ms", ctypes.c_double),
        ("verify_ms", ctypes.c_double),
        ("h2d_ms", ctypes.c_double),
        ("d2h_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
        ("round_blocks", ctypes.c_uint32 * 64),
        ("kernel_launches", ctypes.c_uint64),
        ("init_ms", ctypes.c_double),
        ("loop_ms", ctypes.c_double),
        ("first_signature_ms", ctypes.c_double),
        ("first_signature_arcs", ctypes.c_uint64),
        ("streamed_bytes", ctypes.c_uint64),
        ("streamed_passes", ctypes.c_uint32),
        ("first_signature_hot", ctypes.c_uint32),
    ]


class KernelTimes(ctypes.Structure):
    _fields_ = [
        ("passes", ctypes.c_uint32),
        ("signature_ms", ctypes.c_double),
        ("insert_ms", ctypes.c_double),
        ("relabel_ms", ctypes.c_double),
        ("other_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("init_ms", ctypes.c_double),
        ("setup_ms", ctypes.c_double),
        ("pass_ms", (ctypes.c_float * 4) * 32),
        ("pass_arcs", ctypes.c_uint64 * 32),
        ("pass_nodes", ctypes.c_uint32 * 32),
        ("persist_ms", ctypes.c_double),
        ("persist_passes", ctypes.c_uint32),
    ]


class Csr(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32),
        ("m", ctypes.c_uint64),
        ("offsets", ctypes.c_void_p),
        ("offset_bytes", ctypes.c_int32),
        ("indices", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
    ]


class NoallocResult(ctypes.Structure):
    _fields_ = [
        ("blocks", ctypes.c_uint32),
        ("rounds", ctypes.c_uint32),
        ("repairs", ctypes.c_uint32),
        ("status", ctypes.c_int32),
    ]


class HostGraph(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32),
        ("m", ctypes.c_uint64),
        ("offsets", ctypes.POINTER(ctypes.c_uint64)),
        ("indices", ctypes.POINTER(ctypes.c_uint32)),
        ("weights", ctypes.POINTER(ctypes.c_uint64)),
    ]


class GraphBatch(ctypes.Structure):
    _fields_ = [
        ("num_graphs", ctypes.c_uint32),
        ("graph_nodes", ctypes.POINTER(ctypes.c_uint64)),
        ("labels", ctypes.POINTER(ctypes.c_uint32)),
        ("csr", HostGraph),
    ]


class BatchResult(ctypes.Structure):
    _fields_ = [
        ("colors", ctypes.c_void_p),
        ("local", ctypes.c_void_p),
        ("blocks", ctypes.c_void_p),
        ("fingerprint", ctypes.c_void_p),
        ("hist_offsets", ctypes.c_void_p),
        ("hist_colors", ctypes.c_void_p),
        ("hist_counts", ctypes.c_void_p),
    ]


TUNE_MAX = 8


class TuneSpace(ctypes.Structure):
    _fields_ = [
        ("persist_log2", ctypes.c_int32 * TUNE_MAX),
        ("n_persist", ctypes.c_uint32),
        ("grid_per_sm", ctypes.c_int32 * TUNE_MAX),
        ("n_grid", ctypes.c_uint32),
        ("relabel", ctypes.c_int32 * TUNE_MAX),
        ("n_relabel", ctypes.c_uint32),
        ("use_graph", ctypes.c_int32 * TUNE_MAX),
        ("n_use_graph", ctypes.c_uint32),
        ("sig_kernel", ctypes.c_int32 * TUNE_MAX),
        ("n_sig_kernel", ctypes.c_uint32),
        ("reps", ctypes.c_uint32),
    ]


class TuneReport(ctypes.Structure):
    _fields_ = [
        ("candidates", ctypes.c_uint32),
        ("failed", ctypes.c_uint32),
        ("best_ms", ctypes.c_double),
        ("default_ms", ctypes.c_double),
        ("ms", ctypes.c_double * 64),
        ("opts", Opts * 64),
    ]


class BvStats(ctypes.Structure):
    _fields_ = [
        ("copied_arcs", ctypes.c_uint64),
        ("interval_arcs", ctypes.c_uint64),
        ("residual_arcs", ctypes.c_uint64),
        ("bits", ctypes.c_uint64),
        ("offsets_checked", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
    ]


class EdgeBatchInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_uint32),
        ("last_batches", ctypes.c_uint32),
        ("batches_total", ctypes.c_uint64),
        ("local_refinements", ctypes.c_uint64),
        ("last_arcs", ctypes.c_uint64),
    ]


class ServeOpts(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("slots", ctypes.c_uint32),
        ("hbm_budget", ctypes.c_uint64),
        ("pack_max_arcs", ctypes.c_uint64),
        ("pack_max_graphs", ctypes.c_uint32),
        ("pack_arc_budget", ctypes.c_uint64),
        ("queue_cap", ctypes.c_uint32),
        ("opts", Opts),
        ("dry_run", ctypes.c_int32),
        ("dry_run_ns_per_arc", ctypes.c_uint32),
    ]


class ServeResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("blocks", ctypes.c_uint32),
        ("rounds", ctypes.c_uint32),
        ("packed", ctypes.c_uint32),
        ("slot", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("footprint", ctypes.c_uint64),
        ("queue_ms", ctypes.c_double),
        ("service_ms", ctypes.c_double),
        ("latency_ms", ctypes.c_double),
        ("error", ctypes.c_char * 128),
    ]


class ServeStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("completed", ctypes.c_uint64),
        ("failed", ctypes.c_uint64),
        ("rejected", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("packed_jobs", ctypes.c_uint64),
        ("queued", ctypes.c_uint64),
        ("running", ctypes.c_uint64),
        ("reserved", ctypes.c_uint64),
        ("peak_reserved", ctypes.c_uint64),
        ("peak_busy_slots", ctypes.c_uint32),
        ("slots", ctypes.c_uint32),
        ("hbm_budget", ctypes.c_uint64),
    ]


_lib = None


def load():
    """Loads librbsc.so from the package directory (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"librbsc.so not built ({LIB_PATH}); run `python -m rbsc_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    lib.rbsc_abi_version.restype = ctypes.c_int32
    lib.rbsc_opts_default.argtypes = [P(Opts)]
    lib.rbsc_ctx_create.argtypes = [ctypes.c_int32, P(Opts)]
    lib.rbsc_ctx_create.restype = vp
    lib.rbsc_ctx_destroy.argtypes = [vp]
    lib.rbsc_ctx_trim.argtypes = [vp]
    lib.rbsc_ctx_trim.restype = None
    lib.rbsc_last_error.argtypes = [vp]
    lib.rbsc_last_error.restype = ctypes.c_char_p
    lib.rbsc_ctx_set_opts.argtypes = [vp, P(Opts)]
    lib.rbsc_refine.argtypes = [vp, P(Csr), vp, vp, P(Stats)]
    lib.rbsc_graph_upload.argtypes = [vp, P(Csr), P(vp)]
    lib.rbsc_graph_upload_streamed.argtypes = [vp, P(Csr), ctypes.c_uint64, ctypes.c_uint64, P(vp)]
    lib.rbsc_graph_from_device.argtypes = [vp, P(Csr), P(vp)]
    lib.rbsc_graph_free.argtypes = [vp]
    lib.rbsc_graph_info.argtypes = [vp, P(ctypes.c_uint32), P(ctypes.c_uint64)]
    lib.rbsc_graph_device_csr.argtypes = [vp, P(vp), P(vp)]
    lib.rbsc_graph_refine.argtypes = [vp, vp, vp, vp, P(Stats)]
    lib.rbsc_graph_refine_device.argtypes = [vp, vp, vp, vp, P(Stats)]
    lib.rbsc_graph_degree_colors.argtypes = [vp, vp, vp]
    lib.rbsc_graph_profile.argtypes = [vp, vp, vp, P(KernelTimes), P(Stats)]
    lib.rbsc_refine_noalloc.argtypes = [P(Csr), vp, vp, vp, P(Opts), vp]
    lib.rbsc_parse_arcs.argtypes = [ctypes.c_char_p, ctypes.c_size_t, P(HostGraph)]
    lib.rbsc_host_graph_free.argtypes = [P(HostGraph)]
    lib.rbsc_gen_wl_batch.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                      ctypes.c_int32, P(GraphBatch)]
    lib.rbsc_graph_batch_free.argtypes = [P(GraphBatch)]
    lib.rbsc_graph_batch_free.restype = None
    lib.rbsc_batch_refine.argtypes = [vp, P(Csr), vp, ctypes.c_uint32, vp, P(BatchResult), P(Stats)]
    lib.rbsc_graph_batch_refine.argtypes = [vp, vp, vp, ctypes.c_uint32, vp, P(BatchResult), P(Stats)]
    lib.rbsc_gen_rmat_device.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_uint64, P(vp)]
    lib.rbsc_gen_rmat_host.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_uint64, ctypes.c_int32, P(HostGraph)]
    lib.rbsc_csr_save.argtypes = [ctypes.c_char_p, P(Csr)]
    lib.rbsc_csr_load.argtypes = [ctypes.c_char_p, P(HostGraph)]
    lib.rbsc_bv_load.argtypes = [ctypes.c_char_p, P(HostGraph), P(BvStats)]
    lib.rbsc_tune_space_default.argtypes = [P(TuneSpace)]
    lib.rbsc_tune_space_default.restype = None
    lib.rbsc_graph_autotune.argtypes = [vp, vp, vp, P(TuneSpace), P(Opts), P(TuneReport)]
    lib.rbsc_gen_rmat_pinned.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_uint64, P(HostGraph)]
    lib.rbsc_host_graph_free_pinned.argtypes = [P(HostGraph)]
    lib.rbsc_host_graph_free_pinned.restype = None
    lib.rbsc_gen_er_host.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, ctypes.c_int32, P(HostGraph)]
    lib.rbsc_gen_lift_host.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_uint32, ctypes.c_uint64,
                                       ctypes.c_int32, P(HostGraph)]
    lib.rbsc_refine_edge_batches.argtypes = [vp, P(Csr), ctypes.c_uint64, ctypes.c_int32, vp, P(Stats), P(EdgeBatchInfo)]
    lib.rbsc_refine_f64.argtypes = [vp, P(Csr), vp, vp, vp, P(Stats)]
    lib.rbsc_serve_opts_default.argtypes = [P(ServeOpts)]
    lib.rbsc_serve_opts_default.restype = None
    lib.rbsc_serve_footprint.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32]
    lib.rbsc_serve_footprint.restype = ctypes.c_uint64
    lib.rbsc_serve_create.argtypes = [P(ServeOpts), P(vp)]
    lib.rbsc_serve_destroy.argtypes = [vp]
    lib.rbsc_serve_destroy.restype = None
    lib.rbsc_serve_last_error.argtypes = [vp]
    lib.rbsc_serve_last_error.restype = ctypes.c_char_p
    lib.rbsc_serve_submit.argtypes = [vp, P(Csr), vp, vp, P(ctypes.c_uint64)]
    lib.rbsc_serve_poll.argtypes = [vp, ctypes.c_uint64, P(ServeResult)]
    lib.rbsc_serve_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_int64, P(ServeResult)]
    lib.rbsc_serve_stats_get.argtypes = [vp, P(ServeStats)]
    for name in EXPORTED:
        if name not in ("rbsc_serve_opts_default", "rbsc_host_graph_free_pinned", "rbsc_tune_space_default", "rbsc_serve_footprint", "rbsc_serve_destroy",
                        "rbsc_serve_last_error","rbsc_abi_version", "rbsc_opts_default", "rbsc_ctx_create", "rbsc_ctx_destroy", "rbsc_ctx_trim",
                        "rbsc_graph_batch_free",
                        "rbsc_last_error", "rbsc_graph_free", "rbsc_host_graph_free"):
            getattr(lib, name).restype = ctypes.c_int32
    _lib = lib
    return lib


class RbscError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
