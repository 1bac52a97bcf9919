"""rbsc_b200 -- B200 (sm_100a) colour refinement with rbsc's surface.

Computes the coarsest backward-equivalence (lumpable) partition of a weighted
directed graph -- 1-WL colour refinement over successor multisets -- the path
that src/rbsc/rbsc.cu implements with CUB in the reference.

Host mirror of the reference's interface.  The reference is a process
(``<arcs-cuda text> | rbsc [edge_batch_size] [gpus]`` printing ``time``,
``done`` and ``nodes``, src/rbsc/rbsc.cu:182-497); this module exposes the
same path as calls over the C ABI of include/rbsc.h:

* :func:`run` -- text in, ``(time, done, nodes)`` out, like one reference run;
* :class:`Context` / :class:`Graph` -- resident graphs, repeated refinements,
  labels and statistics;
* :func:`parse_arcs`, :func:`gen_rmat_host` -- input formats and workloads.

Every call goes through librbsc.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import RELABEL_HASH, RELABEL_SORT, RbscError

__all__ = ["Context", "Graph", "Result", "RbscError", "run", "parse_arcs", "gen_rmat_host",
           "RELABEL_HASH", "RELABEL_SORT", "degree_bucket_colors", "gen_wl_batch", "BatchResult",
           "batch_buffers", "gen_er_host", "gen_lift_host", "Server", "ServeResult", "serve_footprint"]

RMAT_ABC = (0.57, 0.19, 0.19)


@dataclass
class Result:
    """One refinement: canonical labels (smallest node id of each block) and
    the counters the reference prints (``nodes`` = blocks, ``done``) plus the
    round count and timings."""
    labels: np.ndarray | None
    blocks: int
    rounds: int
    done: int
    verified: int
    repairs: int
    initial_blocks: int
    time_s: float
    device_ms: float
    verify_ms: float
    h2d_ms: float
    d2h_ms: float
    h2d_bytes: int
    d2h_bytes: int
    round_blocks: list = field(default_factory=list)
    kernel_launches: int = 0
    init_ms: float = 0.0
    loop_ms: float = 0.0
    first_signature_ms: float = 0.0
    first_signature_arcs: int = 0
    streamed_bytes: int = 0
    streamed_passes: int = 0
    first_signature_hot: int = 0


def _result(st: _lib.Stats, labels) -> Result:
    rb = [int(st.round_blocks[i]) for i in range(min(64, st.rounds + 1))]
    return Result(labels, int(st.blocks), int(st.rounds), int(st.done), int(st.verified), int(st.repairs),
                  int(st.initial_blocks), float(st.time_s), float(st.device_ms), float(st.verify_ms),
                  float(st.h2d_ms), float(st.d2h_ms), int(st.h2d_bytes), int(st.d2h_bytes), rb,
                  int(st.kernel_launches), float(st.init_ms), float(st.loop_ms), float(st.first_signature_ms),
                  int(st.first_signature_arcs), int(st.streamed_bytes), int(st.streamed_passes),
                  int(st.first_signature_hot))


def _check(lib, status: int, ctx=None):
    if status != _lib.RBSC_OK:
        msg = lib.rbsc_last_error(ctx)
        raise RbscError(status, msg.decode() if msg else "")


def _csr(off, idx, wt):
    off = np.ascontiguousarray(off)
    if off.dtype not in (np.uint64, np.int64, np.uint32, np.int32):
        off = off.astype(np.uint64)
    ob = off.dtype.itemsize
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    wt = None if wt is None else np.ascontiguousarray(wt, dtype=np.uint64)
    n = len(off) - 1
    m = int(off[-1]) if n >= 0 else 0
    c = _lib.Csr()
    c.n = n
    c.m = m
    c.offsets = off.ctypes.data
    c.offset_bytes = ob
    c.indices = idx.ctypes.data if idx.size else None
    c.weights = wt.ctypes.data if (wt is not None and wt.size) else None
    return c, (off, idx, wt)


class Context:
    """A device context (one CUDA device, one stream).  Options mirror
    ``rbsc_opts`` of include/rbsc.h."""

    def __init__(self, device: int = 0, relabel: int = RELABEL_HASH, verify: bool = True, max_rounds: int = 0,
                 use_graph: bool = True, seed: int = 0x5EED5EED12345678, test_hash_bits: int = 0,
                 persistent: bool = True, persist_log2: int = 0, grid_per_sm: int = 0, sig_kernel: int = 0,
                 hot_log2: int = 0, persist_bps: int = 0, persist_sig: int = 0):
        self._lib = _lib.load()
        o = _lib.Opts()
        self._lib.rbsc_opts_default(ctypes.byref(o))
        o.relabel = relabel
        o.verify = 1 if verify else 0
        o.max_rounds = max_rounds
        o.use_graph = 1 if use_graph else 0
        o.seed = seed
        o.test_hash_bits = test_hash_bits
        o.no_persist = 0 if persistent else 1
        o.persist_log2 = persist_log2
        o.grid_per_sm = grid_per_sm
        o.sig_kernel = sig_kernel
        o.hot_log2 = hot_log2
        o.persist_bps = persist_bps
        o.persist_sig = persist_sig
        self._opts = o
        h = self._lib.rbsc_ctx_create(device, ctypes.byref(o))
        if not h:
            raise RbscError(-2, self._lib.rbsc_last_error(None).decode())
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rbsc_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trim(self):
        """Gives the cached device / pinned buffers back to CUDA (rbsc_ctx_trim)."""
        self._lib.rbsc_ctx_trim(self._h)

    def set_opts(self, **kw):
        for k, v in kw.items():
            if k == "verify" or k == "use_graph":
                v = 1 if v else 0
            if k == "persistent":
                k, v = "no_persist", 0 if v else 1
            setattr(self._opts, k, v)
        _check(self._lib, self._lib.rbsc_ctx_set_opts(self._h, ctypes.byref(self._opts)), self._h)

    def refine(self, off, idx, wt=None, init=None, labels: bool = True, out=None) -> Result:
        """One-shot refinement of a host CSR (rbsc_refine).  `out`: optional
        preallocated uint32 array (e.g. in pinned memory) for the labels."""
        c, keep = _csr(off, idx, wt)
        init_a = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
        if out is not None:
            assert out.dtype == np.uint32 and out.flags.c_contiguous and out.size >= c.n
        elif labels:
            out = np.zeros(max(c.n, 1), dtype=np.uint32)
        st = _lib.Stats()
        _check(self._lib, self._lib.rbsc_refine(self._h, ctypes.byref(c),
                                                None if init_a is None else init_a.ctypes.data,
                                                None if out is None else out.ctypes.data, ctypes.byref(st)), self._h)
        return _result(st, None if out is None else out[: c.n])

    def refine_edge_batches(self, off, idx, wt=None, edge_batch_size: int = 0, aggressive: bool = False,
                            labels: bool = True):
        """The reference's edge-batch (quotient) mode (rbsc_refine_edge_batches):
        returns (Result, info dict).  Result.blocks / .done are the reference
        program's "nodes" / "done" lines for this edge_batch_size."""
        c, keep = _csr(off, idx, wt)
        out = np.zeros(max(c.n, 1), dtype=np.uint32) if labels else None
        st = _lib.Stats()
        info = _lib.EdgeBatchInfo()
        _check(self._lib, self._lib.rbsc_refine_edge_batches(self._h, ctypes.byref(c), edge_batch_size,
                                                             1 if aggressive else 0,
                                                             None if out is None else out.ctypes.data,
                                                             ctypes.byref(st), ctypes.byref(info)), self._h)
        return (_result(st, None if out is None else out[: c.n]),
                {k: int(getattr(info, k)) for k, _ in _lib.EdgeBatchInfo._fields_})

    def refine_f64(self, off, idx, wt, init=None, labels: bool = True) -> Result:
        """Lumping with double weights (rbsc_refine_f64): the rounded-to-float
        sums into every block decide, as in Valmari's minimiser built with
        MDP_weight_is_double."""
        c, keep = _csr(off, idx, None)
        w = np.ascontiguousarray(wt, dtype=np.float64)
        if w.size < c.m:
            raise ValueError("rbsc_refine_f64: fewer weights than arcs")
        init_a = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
        out = np.zeros(max(c.n, 1), dtype=np.uint32) if labels or c.n else None
        st = _lib.Stats()
        _check(self._lib, self._lib.rbsc_refine_f64(self._h, ctypes.byref(c), w.ctypes.data if w.size else None,
                                                    None if init_a is None else init_a.ctypes.data,
                                                    out.ctypes.data, ctypes.byref(st)), self._h)
        return _result(st, out[: c.n] if labels else None)

    def batch_refine(self, off, idx, graph_nodes, init=None, out=None) -> BatchResult:
        """One-shot refinement of a batch of graphs side by side
        (rbsc_batch_refine).  `out`: optional arrays from batch_buffers."""
        c, keep = _csr(off, idx, None)
        return _batch_call(lambda *a: _check(self._lib, self._lib.rbsc_batch_refine(self._h, ctypes.byref(c), *a), self._h),
                           int(c.n), graph_nodes, init, out)

    def upload(self, off, idx, wt=None) -> "Graph":
        c, keep = _csr(off, idx, wt)
        h = ctypes.c_void_p()
        _check(self._lib, self._lib.rbsc_graph_upload(self._h, ctypes.byref(c), ctypes.byref(h)), self._h)
        return Graph(self, h)

    def upload_streamed(self, off, idx, wt=None, batch_arcs: int = 0, resident_arcs: int = 0) -> "Graph":
        """A resident graph whose arcs stay in host memory and are streamed to
        the device in batches of batch_arcs arcs during the signature passes
        (rbsc_graph_upload_streamed).  The arrays are kept alive by the
        returned Graph."""
        c, keep = _csr(off, idx, wt)
        h = ctypes.c_void_p()
        _check(self._lib, self._lib.rbsc_graph_upload_streamed(self._h, ctypes.byref(c), batch_arcs, resident_arcs,
                                                               ctypes.byref(h)), self._h)
        g = Graph(self, h)
        g._keep = keep
        return g

    def gen_rmat_pinned(self, scale: int, edge_factor: int, a=RMAT_ABC[0], b=RMAT_ABC[1], c=RMAT_ABC[2],
                        seed: int = 1) -> "PinnedGraph":
        """R-MAT generated on the device in source buckets into page-locked host
        memory (rbsc_gen_rmat_pinned): the same arcs as gen_rmat_host."""
        hg = _lib.HostGraph()
        _check(self._lib, self._lib.rbsc_gen_rmat_pinned(self._h, scale, edge_factor, a, b, c, seed, ctypes.byref(hg)),
               self._h)
        return PinnedGraph(self._lib, hg)

    def from_device(self, n: int, m: int, d_off: int, d_idx: int, d_wt: int | None = None,
                    offset_bytes: int = 8) -> "Graph":
        c = _lib.Csr()
        c.n, c.m, c.offsets, c.offset_bytes, c.indices, c.weights = n, m, d_off, offset_bytes, d_idx, d_wt
        h = ctypes.c_void_p()
        _check(self._lib, self._lib.rbsc_graph_from_device(self._h, ctypes.byref(c), ctypes.byref(h)), self._h)
        return Graph(self, h)

    def gen_rmat(self, scale: int, edge_factor: int, a=RMAT_ABC[0], b=RMAT_ABC[1], c=RMAT_ABC[2],
                 seed: int = 1) -> "Graph":
        """R-MAT graph generated directly in device memory."""
        h = ctypes.c_void_p()
        _check(self._lib, self._lib.rbsc_gen_rmat_device(self._h, scale, edge_factor, a, b, c, seed,
                                                         ctypes.byref(h)), self._h)
        return Graph(self, h)


class Graph:
    """A graph resident in device memory (rbsc_graph)."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._h = handle
        n = ctypes.c_uint32()
        m = ctypes.c_uint64()
        ctx._lib.rbsc_graph_info(handle, ctypes.byref(n), ctypes.byref(m))
        self.n = int(n.value)
        self.m = int(m.value)

    def free(self):
        if getattr(self, "_h", None):
            self.ctx._lib.rbsc_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def refine(self, init=None, labels: bool = True) -> Result:
        lib = self.ctx._lib
        init_a = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
        out = np.zeros(max(self.n, 1), dtype=np.uint32) if labels else None
        st = _lib.Stats()
        _check(lib, lib.rbsc_graph_refine(self.ctx._h, self._h, None if init_a is None else init_a.ctypes.data,
                                          None if out is None else out.ctypes.data, ctypes.byref(st)), self.ctx._h)
        return _result(st, None if out is None else out[: self.n])

    def batch_refine(self, graph_nodes, init=None, out=None) -> BatchResult:
        """This resident graph holds a batch of graphs side by side
        (rbsc_graph_batch_refine).  `out`: optional arrays from batch_buffers."""
        lib = self.ctx._lib
        return _batch_call(lambda *a: _check(lib, lib.rbsc_graph_batch_refine(self.ctx._h, self._h, *a), self.ctx._h),
                           self.n, graph_nodes, init, out)

    def refine_device(self, d_init: int | None = None, d_out: int | None = None) -> Result:
        """Refinement with device-resident initial colours / labels (raw
        device addresses, e.g. ``tensor.data_ptr()``)."""
        lib = self.ctx._lib
        st = _lib.Stats()
        _check(lib, lib.rbsc_graph_refine_device(self.ctx._h, self._h, d_init, d_out, ctypes.byref(st)), self.ctx._h)
        return _result(st, None)

    def profile(self, d_init: int | None = None):
        """Refinement with CUDA events around every kernel (rbsc_graph_profile):
        returns (per-kernel times dict, Result)."""
        lib = self.ctx._lib
        kt = _lib.KernelTimes()
        st = _lib.Stats()
        _check(lib, lib.rbsc_graph_profile(self.ctx._h, self._h, d_init, ctypes.byref(kt), ctypes.byref(st)),
               self.ctx._h)
        times = {k: getattr(kt, k) for k, _ in _lib.KernelTimes._fields_
                 if k not in ("pass_ms", "pass_arcs", "pass_nodes")}
        np_ = min(32, kt.passes)
        times["per_pass"] = [dict(signature_ms=kt.pass_ms[i][0], insert_ms=kt.pass_ms[i][1],
                                  relabel_ms=kt.pass_ms[i][2], other_ms=kt.pass_ms[i][3],
                                  arcs=int(kt.pass_arcs[i]), nodes=int(kt.pass_nodes[i])) for i in range(np_)]
        return times, _result(st, None)

    def degree_colors_device(self, d_out: int):
        lib = self.ctx._lib
        _check(lib, lib.rbsc_graph_degree_colors(self.ctx._h, self._h, d_out), self.ctx._h)

    def autotune(self, d_init: int | None = None, persist_log2=None, grid_per_sm=None, relabel=None, use_graph=None,
                 sig_kernel=None, reps: int = 3, apply: bool = True) -> dict:
        """Times refinements of this graph under combinations of the pass
        kernels' knobs (rbsc_graph_autotune) and, with apply, sets the fastest
        on the context.  Lists left at None take the library's default search
        space.  Returns the chosen knobs, the default and best times and every
        candidate's time."""
        lib = self.ctx._lib
        sp = _lib.TuneSpace()
        lib.rbsc_tune_space_default(ctypes.byref(sp))
        for name, vals, cnt in (("persist_log2", persist_log2, "n_persist"), ("grid_per_sm", grid_per_sm, "n_grid"),
                                ("relabel", relabel, "n_relabel"), ("use_graph", use_graph, "n_use_graph"),
                                ("sig_kernel", sig_kernel, "n_sig_kernel")):
            if vals is not None:
                arr = getattr(sp, name)
                for i, v in enumerate(vals[: _lib.TUNE_MAX]):
                    arr[i] = int(v)
                setattr(sp, cnt, min(len(vals), _lib.TUNE_MAX))
        sp.reps = reps
        best = _lib.Opts()
        rep = _lib.TuneReport()
        _check(lib, lib.rbsc_graph_autotune(self.ctx._h, self._h, d_init, ctypes.byref(sp), ctypes.byref(best),
                                            ctypes.byref(rep)), self.ctx._h)
        knobs = ("persist_log2", "grid_per_sm", "relabel", "use_graph", "no_persist", "sig_kernel")
        if apply:
            for k in knobs:
                setattr(self.ctx._opts, k, getattr(best, k))
            _check(lib, lib.rbsc_ctx_set_opts(self.ctx._h, ctypes.byref(self.ctx._opts)), self.ctx._h)
        n = min(int(rep.candidates), 64)
        return {"best": {k: int(getattr(best, k)) for k in knobs}, "best_ms": float(rep.best_ms),
                "default_ms": float(rep.default_ms), "candidates": int(rep.candidates), "failed": int(rep.failed),
                "table": [dict({k: int(getattr(rep.opts[i], k)) for k in knobs}, ms=float(rep.ms[i])) for i in range(n)]}

    def device_csr(self):
        lib = self.ctx._lib
        o = ctypes.c_void_p()
        i = ctypes.c_void_p()
        _check(lib, lib.rbsc_graph_device_csr(self._h, ctypes.byref(o), ctypes.byref(i)), self.ctx._h)
        return o.value, i.value


class PinnedGraph:
    """A host CSR in page-locked memory owned by the library; `off` and `idx`
    are numpy views of it (valid until free())."""

    def __init__(self, lib, hg):
        self._lib, self._hg = lib, hg
        self.n, self.m = int(hg.n), int(hg.m)
        self.off = np.ctypeslib.as_array(hg.offsets, shape=(self.n + 1,))
        self.idx = np.ctypeslib.as_array(hg.indices, shape=(max(self.m, 1),))[: self.m]

    def free(self):
        if getattr(self, "_hg", None) is not None:
            self.off = self.idx = None
            self._lib.rbsc_host_graph_free_pinned(ctypes.byref(self._hg))
            self._hg = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _host_graph_to_numpy(lib, hg: _lib.HostGraph):
    n, m = int(hg.n), int(hg.m)
    off = np.ctypeslib.as_array(hg.offsets, shape=(n + 1,)).copy()
    idx = np.ctypeslib.as_array(hg.indices, shape=(max(m, 1),))[:m].copy() if m else np.zeros(0, np.uint32)
    wt = None
    if bool(hg.weights):
        wt = np.ctypeslib.as_array(hg.weights, shape=(max(m, 1),))[:m].copy()
    lib.rbsc_host_graph_free(ctypes.byref(hg))
    return off, idx, wt


def parse_arcs(text: bytes):
    """arcs-cuda text -> (offsets uint64, indices uint32, weights uint64 | None)."""
    lib = _lib.load()
    hg = _lib.HostGraph()
    st = lib.rbsc_parse_arcs(text, len(text), ctypes.byref(hg))
    _check(lib, st, None)
    return _host_graph_to_numpy(lib, hg)


def save_csr(path: str, off, idx, wt=None) -> None:
    """Binary CSR cache file (rbsc_csr_save)."""
    lib = _lib.load()
    c, keep = _csr(np.ascontiguousarray(off, dtype=np.uint64), idx, wt)
    _check(lib, lib.rbsc_csr_save(path.encode(), ctypes.byref(c)), None)


def load_csr(path: str):
    """(offsets, indices, weights | None) from a binary CSR cache file (rbsc_csr_load)."""
    lib = _lib.load()
    hg = _lib.HostGraph()
    _check(lib, lib.rbsc_csr_load(path.encode(), ctypes.byref(hg)), None)
    return _host_graph_to_numpy(lib, hg)


def load_bvgraph(basename: str):
    """A BV-compressed (WebGraph / LAW) graph: (offsets uint64, indices uint32,
    stats dict) -- rbsc_bv_load."""
    lib = _lib.load()
    hg = _lib.HostGraph()
    st = _lib.BvStats()
    _check(lib, lib.rbsc_bv_load(basename.encode(), ctypes.byref(hg), ctypes.byref(st)), None)
    off, idx, _ = _host_graph_to_numpy(lib, hg)
    return off, idx, {k: int(getattr(st, k)) for k, _ in _lib.BvStats._fields_ if k != "pad"}


def gen_rmat_host(scale: int, edge_factor: int, a=RMAT_ABC[0], b=RMAT_ABC[1], c=RMAT_ABC[2], seed: int = 1,
                  threads: int = 0):
    """The device generator's graph, built on the host: (offsets, indices)."""
    lib = _lib.load()
    hg = _lib.HostGraph()
    _check(lib, lib.rbsc_gen_rmat_host(scale, edge_factor, a, b, c, seed, threads, ctypes.byref(hg)), None)
    off, idx, _ = _host_graph_to_numpy(lib, hg)
    return off, idx


def gen_wl_batch(num_graphs: int, nmin: int = 10, nmax: int = 500, num_labels: int = 8, seed: int = 1,
                 threads: int = 0):
    """The small-graph batch (rbsc_gen_wl_batch): (offsets uint64, indices
    uint32, graph_nodes uint64[num_graphs+1], labels uint32) of the graphs side
    by side over global node ids."""
    lib = _lib.load()
    b = _lib.GraphBatch()
    _check(lib, lib.rbsc_gen_wl_batch(num_graphs, nmin, nmax, num_labels, seed, threads, ctypes.byref(b)), None)
    try:
        n, m, G = int(b.csr.n), int(b.csr.m), int(b.num_graphs)
        off = np.ctypeslib.as_array(b.csr.offsets, shape=(n + 1,)).copy()
        idx = np.ctypeslib.as_array(b.csr.indices, shape=(max(m, 1),))[:m].copy()
        gn = np.ctypeslib.as_array(b.graph_nodes, shape=(G + 1,)).copy()
        labels = np.ctypeslib.as_array(b.labels, shape=(max(n, 1),))[:n].copy()
    finally:
        lib.rbsc_graph_batch_free(ctypes.byref(b))
    return off, idx, gn, labels


def gen_er_host(n: int, mean_degree: float, seed: int = 1, threads: int = 0):
    """Directed Erdos-Renyi G(n, mean_degree / (n-1)) without self-loops
    (rbsc_gen_er_host): (offsets uint64, indices uint32)."""
    lib = _lib.load()
    hg = _lib.HostGraph()
    _check(lib, lib.rbsc_gen_er_host(n, float(mean_degree), seed, threads, ctypes.byref(hg)), None)
    off, idx, _ = _host_graph_to_numpy(lib, hg)
    return off, idx


def gen_lift_host(base_n: int, mean_degree: float, lift: int, seed: int = 1, threads: int = 0):
    """Random lift of a directed Erdos-Renyi base graph (rbsc_gen_lift_host):
    (offsets uint64, indices uint32) of base_n * lift nodes."""
    lib = _lib.load()
    hg = _lib.HostGraph()
    _check(lib, lib.rbsc_gen_lift_host(base_n, float(mean_degree), lift, seed, threads, ctypes.byref(hg)), None)
    off, idx, _ = _host_graph_to_numpy(lib, hg)
    return off, idx


@dataclass
class BatchResult:
    """Per-graph results of a batch refinement (rbsc_batch_result)."""
    colors: np.ndarray        # shared colour of every node (smallest global node id of its class)
    local: np.ndarray         # smallest local node id of each node's block in its own graph
    blocks: np.ndarray        # blocks per graph
    fingerprint: np.ndarray   # 64-bit digest of each graph's colour histogram
    hist_offsets: np.ndarray  # histogram entries of each graph
    hist_colors: np.ndarray
    hist_counts: np.ndarray
    stats: Result

    def histogram(self, g: int):
        a, b = int(self.hist_offsets[g]), int(self.hist_offsets[g + 1])
        return self.hist_colors[a:b], self.hist_counts[a:b]


_BATCH_FIELDS = (("colors", "n", np.uint32), ("local", "n", np.uint32), ("blocks", "G", np.uint32),
                 ("fingerprint", "G", np.uint64), ("hist_offsets", "G1", np.uint64), ("hist_colors", "n", np.uint32),
                 ("hist_counts", "n", np.uint32))


def batch_buffers(n: int, num_graphs: int, alloc=np.empty) -> dict:
    """Output arrays for a batch refinement of n nodes in num_graphs graphs;
    `alloc(shape, dtype)` may return pinned memory (e.g. a view of a pinned
    torch tensor) for faster copies."""
    size = {"n": max(n, 1), "G": max(num_graphs, 1), "G1": num_graphs + 1}
    return {k: alloc(size[s], dt) for k, s, dt in _BATCH_FIELDS}


def _batch_call(fn, n: int, graph_nodes, init, out=None):
    gn = np.ascontiguousarray(graph_nodes, dtype=np.uint64)
    G = len(gn) - 1
    init_a = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
    arrs = out if out is not None else batch_buffers(n, G)
    for k, s, dt in _BATCH_FIELDS:
        need = {"n": n, "G": G, "G1": G + 1}[s]
        a = arrs[k]
        assert a.dtype == dt and a.flags.c_contiguous and a.size >= need, k
    out = _lib.BatchResult(*(arrs[k].ctypes.data for k in ("colors", "local", "blocks", "fingerprint", "hist_offsets",
                                                            "hist_colors", "hist_counts")))
    st = _lib.Stats()
    fn(gn.ctypes.data, G, None if init_a is None else init_a.ctypes.data, ctypes.byref(out), ctypes.byref(st))
    H = int(arrs["hist_offsets"][G])
    return BatchResult(arrs["colors"][:n], arrs["local"][:n], arrs["blocks"][:G], arrs["fingerprint"][:G],
                       arrs["hist_offsets"], arrs["hist_colors"][:H], arrs["hist_counts"][:H], _result(st, None))


@dataclass
class ServeResult:
    """The result of one served job (rbsc_serve_result)."""
    labels: np.ndarray | None
    status: int
    blocks: int
    rounds: int
    packed: int          # jobs in the batch it ran in (1 = alone)
    slot: int
    footprint: int
    queue_ms: float
    service_ms: float
    latency_ms: float
    error: str


def serve_footprint(n: int, m: int, weighted: bool = False, graphs: int = 1) -> int:
    """Device bytes a server reserves for a refinement (rbsc_serve_footprint)."""
    return int(_lib.load().rbsc_serve_footprint(n, m, 1 if weighted else 0, graphs))


class Server:
    """Refinement service with continuous batching (rbsc_serve_*): `slots`
    executors on one device, admission by device footprint within
    `hbm_budget`, small jobs packed into one batch refinement.  The arrays of
    a submitted job are kept alive here until its result is collected."""

    def __init__(self, device: int = 0, slots: int = 2, hbm_budget: int = 0, pack_max_arcs: int = 0,
                 pack_max_graphs: int = 0, pack_arc_budget: int = 0, queue_cap: int = 0, verify: bool = True,
                 seed: int | None = None, dry_run_ns_per_arc: int | None = None):
        self._lib = _lib.load()
        o = _lib.ServeOpts()
        self._lib.rbsc_serve_opts_default(ctypes.byref(o))
        o.device, o.slots, o.hbm_budget = device, slots, hbm_budget
        o.pack_max_arcs, o.pack_max_graphs, o.pack_arc_budget, o.queue_cap = (pack_max_arcs, pack_max_graphs,
                                                                              pack_arc_budget, queue_cap)
        o.opts.verify = 1 if verify else 0
        if seed is not None:
            o.opts.seed = seed
        if dry_run_ns_per_arc is not None:
            o.dry_run, o.dry_run_ns_per_arc = 1, dry_run_ns_per_arc
        h = ctypes.c_void_p()
        st = self._lib.rbsc_serve_create(ctypes.byref(o), ctypes.byref(h))
        if st != _lib.RBSC_OK:
            raise RbscError(st, self._lib.rbsc_serve_last_error(None).decode())
        self._h = h
        self._keep = {}

    def _fail(self, st):
        raise RbscError(st, self._lib.rbsc_serve_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rbsc_serve_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, off, idx, wt=None, init=None, labels: bool = True) -> int:
        """Queues a job; returns its id.  Raises RbscError with RBSC_ERR_BUSY
        (-8) when the queue is full and RBSC_ERR_TOO_LARGE (-7) when the job
        exceeds the budget."""
        c, keep = _csr(off, idx, wt)
        init_a = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
        out = np.zeros(max(c.n, 1), dtype=np.uint32) if labels else None
        jid = ctypes.c_uint64()
        st = self._lib.rbsc_serve_submit(self._h, ctypes.byref(c), None if init_a is None else init_a.ctypes.data,
                                         None if out is None else out.ctypes.data, ctypes.byref(jid))
        if st != _lib.RBSC_OK:
            self._fail(st)
        self._keep[jid.value] = (c, keep, init_a, out)
        return int(jid.value)

    def _collect(self, jid: int, r: _lib.ServeResult) -> ServeResult:
        c, _, _, out = self._keep.pop(jid)
        return ServeResult(None if out is None else out[: c.n], int(r.status), int(r.blocks), int(r.rounds),
                           int(r.packed), int(r.slot), int(r.footprint), float(r.queue_ms), float(r.service_ms),
                           float(r.latency_ms), r.error.decode(errors="replace"))

    def poll(self, jid: int) -> ServeResult | None:
        r = _lib.ServeResult()
        st = self._lib.rbsc_serve_poll(self._h, jid, ctypes.byref(r))
        if st == _lib.RBSC_PENDING:
            return None
        if st != _lib.RBSC_OK:
            self._fail(st)
        return self._collect(jid, r)

    def wait(self, jid: int, timeout_ms: int = -1) -> ServeResult | None:
        r = _lib.ServeResult()
        st = self._lib.rbsc_serve_wait(self._h, jid, timeout_ms, ctypes.byref(r))
        if st == _lib.RBSC_PENDING:
            return None
        if st != _lib.RBSC_OK:
            self._fail(st)
        return self._collect(jid, r)

    def stats(self) -> dict:
        s = _lib.ServeStats()
        st = self._lib.rbsc_serve_stats_get(self._h, ctypes.byref(s))
        if st != _lib.RBSC_OK:
            self._fail(st)
        return {k: int(getattr(s, k)) for k, _ in _lib.ServeStats._fields_}


def degree_bucket_colors(off) -> np.ndarray:
    """floor(log2(out_degree + 1)) as uint32 (the initial colours of the R-MAT-24 workload)."""
    x = np.diff(np.asarray(off, dtype=np.int64)) + 1
    out = np.zeros(x.shape, dtype=np.uint32)
    for sh in (32, 16, 8, 4, 2, 1):
        big = x >= (1 << sh)
        out[big] += sh
        x = np.where(big, x >> sh, x)
    return out


def run(text: bytes, edge_batch_size: int | None = None, gpus: int = 1, device: int = 0):
    """One reference-style run: arcs-cuda text -> (time_s, done, nodes), the
    three values rbsc.cu:492-494 prints."""
    off, idx, wt = parse_arcs(text)
    with Context(device) as ctx:
        r = ctx.refine(off, idx, wt, labels=False)
    return r.time_s, r.done, r.blocks
