"""Python front end of the oracle -- TEST INFRASTRUCTURE ONLY.

The checker that the CUDA product path is compared against.  Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this module; the product (``rbsc_b200``, ``librbsc.so``, the ``rbsc`` CLI)
never does.

Two kinds of oracle are reachable from here:

* ``refine_exact`` / ``refine_rsc``: the C restatement in ``oracle.c``
  (built into ``liboracle.so``);
* ``run_ref_rsc`` / ``run_ref_valmari``: the reference programs themselves,
  compiled unmodified from their sources into ``oracle/_ref/`` by
  ``oracle/Makefile`` (``src/rsc/rsc.cpp`` and ``src/part_ref``).

All labels returned are canonical: each node carries the smallest node id of
its block.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_RSC = os.path.join(REF_DIR, "ref_rsc")
REF_VALMARI = os.path.join(REF_DIR, "ref_valmari")
REF_VALMARI_F64 = os.path.join(REF_DIR, "ref_valmari_f64")
REF_RBSC = os.path.join(REF_DIR, "ref_rbsc")
# decoded copy of the reference's vendored LAW sample (webgraph-rs/data/cnr-2000),
# made in this container by prepare_law() and carried with the tree
LAW_CNR2000 = os.path.join(REF_DIR, "cnr-2000.npz")


def reference_tree() -> str | None:
    """The reference checkout used to build oracle/_ref and the fixtures:
    $RBSC_REFERENCE, else the location oracle/Makefile names; None when that
    directory does not exist on this machine."""
    ref = os.environ.get("RBSC_REFERENCE")
    if not ref:
        try:
            ref = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True,
                                 timeout=30).stdout.strip()
        except (OSError, subprocess.SubprocessError):
            ref = None
    return ref if ref and os.path.isdir(ref) else None


def prepare_law(ref: str | None) -> str | None:
    """Decodes the reference's cnr-2000 BV graph (webgraph-rs/data) into
    LAW_CNR2000, once; returns the path or None when the reference tree is
    absent and no copy was made before."""
    if os.path.exists(LAW_CNR2000):
        return LAW_CNR2000
    base = None if not ref else os.path.join(ref, "webgraph-rs", "data", "cnr-2000")
    if not base or not os.path.exists(base + ".graph"):
        return None
    import rbsc_b200 as R
    off, idx, _ = R.load_bvgraph(base)
    os.makedirs(REF_DIR, exist_ok=True)
    np.savez(LAW_CNR2000, off=off, idx=idx)
    return LAW_CNR2000


def load_law():
    """(off, idx) of the decoded cnr-2000, or None."""
    if not os.path.exists(LAW_CNR2000):
        return None
    z = np.load(LAW_CNR2000)
    return z["off"], z["idx"]

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)


def build(ref: str | None = None) -> None:
    """Run oracle/Makefile (liboracle.so, and oracle/_ref when the reference
    tree is present)."""
    cmd = ["make", "-s", "-C", HERE]
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.orc_refine_exact.argtypes = [ctypes.c_uint32, _u64p, _u32p, _u64p, _u32p, _u32p,
                                         _u32p, _u32p, _u32p, ctypes.c_uint32]
        lib.orc_refine_exact.restype = ctypes.c_int
        lib.orc_refine_rsc.argtypes = [ctypes.c_uint32, _u64p, _u32p, _u64p, _u32p, _u32p,
                                       _u32p, _u32p, _u32p, ctypes.c_uint32]
        lib.orc_refine_rsc.restype = ctypes.c_int
        lib.orc_refine_rsc_mt.argtypes = [ctypes.c_uint32, _u64p, _u32p, _u64p, _u32p, _u32p,
                                          _u32p, _u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32]
        lib.orc_refine_rsc_mt.restype = ctypes.c_int
        lib.orc_canonicalize.argtypes = [ctypes.c_uint32, _u32p, _u32p]
        lib.orc_canonicalize.restype = ctypes.c_uint32
        lib.orc_rsc_randomize.argtypes = [ctypes.c_uint64]
        lib.orc_rsc_randomize.restype = ctypes.c_uint64
        lib.orc_write_arcs.argtypes = [ctypes.c_char_p, ctypes.c_uint32, _u64p, _u32p, _u64p]
        lib.orc_write_arcs.restype = ctypes.c_int
        lib.orc_refine_edge_batches.argtypes = [ctypes.c_uint32, _u64p, _u32p, _u64p, ctypes.c_uint64, ctypes.c_int,
                                                _u32p, _u32p, _u32p, _u32p]
        lib.orc_refine_edge_batches.restype = ctypes.c_int
        lib.orc_gen_rmat.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_u64p),
                                     ctypes.POINTER(_u32p), ctypes.POINTER(ctypes.c_uint64)]
        lib.orc_gen_rmat.restype = ctypes.c_int
        lib.orc_free.argtypes = [ctypes.c_void_p]
        lib.orc_free.restype = None
        lib.orc_write_mdp.argtypes = [ctypes.c_char_p, ctypes.c_uint32, _u64p, _u32p, _u64p, _u32p]
        lib.orc_write_mdp.restype = ctypes.c_int
        lib.orc_refine_f64.argtypes = [ctypes.c_uint32, _u64p, _u32p, _f64p, _u32p, _u32p,
                                       _u32p, _u32p, _u32p, ctypes.c_uint32]
        lib.orc_refine_f64.restype = ctypes.c_int
        lib.orc_reader_decimal.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        lib.orc_reader_decimal.restype = ctypes.c_size_t
        _lib = lib
    return _lib


def _p32(a):
    return None if a is None else a.ctypes.data_as(_u32p)


def _p64(a):
    return None if a is None else a.ctypes.data_as(_u64p)


@dataclass
class OracleResult:
    labels: np.ndarray      # canonical labels (min node id per block), uint32
    blocks: int
    rounds: int             # rounds, GPU convention
    rounds_cpu: int | None = None
    round_blocks: list | None = None
    status: int = 0


def _csr(off, idx, wt):
    off = np.ascontiguousarray(off, dtype=np.uint64)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    if idx.size == 0:
        idx = np.zeros(1, dtype=np.uint32)
    wt = None if wt is None else np.ascontiguousarray(wt, dtype=np.uint64)
    if wt is not None and wt.size == 0:
        wt = np.zeros(1, dtype=np.uint64)
    return off, idx, wt


def refine_exact(off, idx, wt=None, init=None, max_rounds: int | None = None) -> OracleResult:
    """Exact coarsest stable refinement (oracle.c: orc_refine_exact)."""
    lib = _load()
    n = len(off) - 1
    off, idx, wt = _csr(off, idx, wt)
    init = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
    if max_rounds is None:
        max_rounds = n + 2
    labels = np.zeros(max(n, 1), dtype=np.uint32)
    rounds = ctypes.c_uint32()
    blocks = ctypes.c_uint32()
    rb = np.zeros(max_rounds + 1, dtype=np.uint32)
    st = lib.orc_refine_exact(n, _p64(off), _p32(idx), _p64(wt), _p32(init), _p32(labels),
                              ctypes.byref(rounds), ctypes.byref(blocks), _p32(rb), max_rounds)
    return OracleResult(labels[:n].copy(), blocks.value, rounds.value, None,
                        [int(x) for x in rb[: rounds.value + 1]], st)


def refine_f64(off, idx, wt, init=None, max_rounds: int | None = None) -> OracleResult:
    """Exact coarsest stable refinement with double weights, sums into a block
    rounded to float (oracle.c: orc_refine_f64)."""
    lib = _load()
    n = len(off) - 1
    off, idx, _ = _csr(off, idx, None)
    w = np.ascontiguousarray(wt, dtype=np.float64)
    if w.size == 0:
        w = np.zeros(1, dtype=np.float64)
    init = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
    if max_rounds is None:
        max_rounds = n + 2
    labels = np.zeros(max(n, 1), dtype=np.uint32)
    rounds = ctypes.c_uint32()
    blocks = ctypes.c_uint32()
    rb = np.zeros(max_rounds + 1, dtype=np.uint32)
    st = lib.orc_refine_f64(n, _p64(off), _p32(idx), w.ctypes.data_as(_f64p), _p32(init), _p32(labels),
                            ctypes.byref(rounds), ctypes.byref(blocks), _p32(rb), max_rounds)
    return OracleResult(labels[:n].copy(), blocks.value, rounds.value, None,
                        [int(x) for x in rb[: rounds.value + 1]], st)


def reader_decimals(texts) -> np.ndarray:
    """Doubles of decimal weight strings as the minimiser's reader computes
    them (src/part_ref/reader.cc:110-147, restated in oracle.c:
    orc_reader_decimal)."""
    lib = _load()
    out = np.zeros(len(texts), dtype=np.float64)
    v = ctypes.c_double()
    for i, t in enumerate(texts):
        if lib.orc_reader_decimal(t.encode(), ctypes.byref(v)) != len(t):
            raise ValueError(f"not a decimal: {t!r}")
        out[i] = v.value
    return out


def mdp_text_f64(off, idx, wt_text, init=None) -> bytes:
    """Valmari MDP text with decimal weights (the strings themselves, which
    the double-weight minimiser parses; no merging of parallel arcs)."""
    off = np.asarray(off, dtype=np.uint64)
    idx = np.asarray(idx, dtype=np.uint32)
    n = len(off) - 1
    m = int(off[-1])
    if m > n * n:
        raise ValueError("more transitions than states squared: the reader refuses them")
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64)))
    blocks = []
    if init is not None:
        init = np.asarray(init, dtype=np.uint32)
        for c in sorted(set(init.tolist()))[1:]:
            blocks.append(" ".join(map(str, (np.nonzero(init == c)[0] + 1).tolist())) + " 0")
    out = [f"{n} 0 0 {m} {1 + len(blocks)}\n"]
    if m:
        out.append("\n".join(f"{a + 1} {w} {c + 1}" for a, w, c in zip(src.tolist(), wt_text, idx[:m].tolist())))
        out.append("\n")
    if blocks:
        out.append("\n".join(blocks) + "\n")
    return "".join(out).encode()


def run_ref_valmari_f64(off, idx, wt_text, init=None, timeout: float = 600.0) -> OracleResult:
    """Valmari's minimiser built with double weights (src/part_ref, unmodified,
    MDP_weight_is_double) on a graph whose weights are decimal strings."""
    if not os.path.exists(REF_VALMARI_F64):
        raise FileNotFoundError(REF_VALMARI_F64)
    txt = subprocess.run([REF_VALMARI_F64], input=mdp_text_f64(off, idx, wt_text, init), capture_output=True,
                         timeout=timeout, check=True).stdout.decode()
    t, done, nodes, rounds, labels = _parse_ref_output(txt)
    n = len(off) - 1
    lab = _canon_u64(labels) if n else np.zeros(0, dtype=np.uint32)
    res = OracleResult(lab, nodes, -1, None)
    res.time_s = t
    return res


@dataclass
class EdgeBatchResult:
    labels: np.ndarray      # canonical labels of the final partition
    blocks: int             # the reference's "nodes" line (new_node_n)
    done: int               # 1 iff the last iteration had one batch
    iterations: int


def refine_edge_batches(off, idx, wt=None, batch: int = 0, aggressive: bool = False) -> EdgeBatchResult:
    """The reference GPU program's edge-batch (quotient) mode, restated with
    exact local refinements (oracle.c: orc_refine_edge_batches)."""
    lib = _load()
    n = len(off) - 1
    off, idx, wt = _csr(off, idx, wt)
    labels = np.zeros(max(n, 1), dtype=np.uint32)
    bl, dn, it = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    lib.orc_refine_edge_batches(n, _p64(off), _p32(idx), _p64(wt), batch, 1 if aggressive else 0, _p32(labels),
                                ctypes.byref(bl), ctypes.byref(dn), ctypes.byref(it))
    return EdgeBatchResult(labels[:n].copy(), bl.value, dn.value, it.value)


def refine_rsc(off, idx, wt=None, init=None, max_rounds: int | None = None, threads: int | None = None) -> OracleResult:
    """The reference CPU loop restated (oracle.c: orc_refine_rsc); with
    `threads`, the multi-threaded restatement (orc_refine_rsc_mt: the same
    ranks and results, for graphs of billions of arcs)."""
    lib = _load()
    n = len(off) - 1
    off, idx, wt = _csr(off, idx, wt)
    init = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
    if max_rounds is None:
        max_rounds = min(n + 2, 0xFFFFFFFF)
    labels = np.zeros(max(n, 1), dtype=np.uint32)
    rg, rc, bl = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    if threads:
        st = lib.orc_refine_rsc_mt(n, _p64(off), _p32(idx), _p64(wt), _p32(init), _p32(labels),
                                   ctypes.byref(rg), ctypes.byref(rc), ctypes.byref(bl), max_rounds, int(threads))
    else:
        st = lib.orc_refine_rsc(n, _p64(off), _p32(idx), _p64(wt), _p32(init), _p32(labels),
                                ctypes.byref(rg), ctypes.byref(rc), ctypes.byref(bl), max_rounds)
    return OracleResult(labels[:n].copy(), bl.value, rg.value, rc.value, None, st)


def canonicalize(labels) -> tuple[np.ndarray, int]:
    lib = _load()
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    out = np.zeros(max(lab.size, 1), dtype=np.uint32)
    b = lib.orc_canonicalize(lab.size, _p32(lab if lab.size else out), _p32(out))
    return out[: lab.size].copy(), int(b)


def rsc_randomize(x: int) -> int:
    return int(_load().orc_rsc_randomize(x))


# ---------------------------------------------------------------------------
# text formats of the reference
# ---------------------------------------------------------------------------

def arcs_cuda_text(off, idx, wt=None) -> bytes:
    """arcs-cuda text (webgraph-rs cli/src/to/arcscuda.rs:61-66):
    "N\\nM\\n" then one "u wt v" line per arc, grouped by u."""
    off = np.asarray(off, dtype=np.uint64)
    idx = np.asarray(idx, dtype=np.uint32)
    n = len(off) - 1
    m = int(off[-1]) if n >= 0 else 0
    deg = np.diff(off.astype(np.int64))
    src = np.repeat(np.arange(n, dtype=np.int64), deg)
    w = np.ones(m, dtype=np.uint64) if wt is None else np.asarray(wt, dtype=np.uint64)
    lines = [f"{n}\n{m}\n"]
    if m:
        lines.append("\n".join(f"{a} {b} {c}" for a, b, c in zip(src.tolist(), w.tolist(), idx[:m].tolist())))
        lines.append("\n")
    return "".join(lines).encode()


def mdp_text(off, idx, wt=None, init=None, merge: bool = False) -> bytes:
    """Valmari MDP text (src/part_ref/MDP_read.cc:51-63), the conversion that
    valmari-adapter:9-16 performs, extended with <blocks> for initial colours.
    merge: parallel arcs become one transition carrying their summed weight
    (the same weight sum into every block, so the same lumping); the reader
    refuses more transitions than states squared."""
    off = np.asarray(off, dtype=np.uint64)
    idx = np.asarray(idx, dtype=np.uint32)
    n = len(off) - 1
    m = int(off[-1])
    deg = np.diff(off.astype(np.int64))
    src = np.repeat(np.arange(n, dtype=np.int64), deg)
    w = np.ones(m, dtype=np.uint64) if wt is None else np.asarray(wt, dtype=np.uint64)[:m]
    if merge and m:
        key = src * n + idx[:m].astype(np.int64)
        uk, inv = np.unique(key, return_inverse=True)
        wsum = np.zeros(len(uk), dtype=np.uint64)
        np.add.at(wsum, inv, w)  # exact (modulo 2^64)
        w = wsum
        src, idx = uk // n, (uk % n).astype(np.uint32)
        m = len(uk)
    blocks = []
    if init is not None:
        init = np.asarray(init, dtype=np.uint32)
        colours = sorted(set(init.tolist()))
        # block 1 = the remaining states (MDP_read.cc:58-59): the first colour
        for c in colours[1:]:
            members = (np.nonzero(init == c)[0] + 1).tolist()
            blocks.append(" ".join(map(str, members)) + " 0")
    nb = 1 + len(blocks)
    out = [f"{n} 0 0 {m} {nb}\n"]
    if m:
        out.append("\n".join(f"{a + 1} {b} {c + 1}" for a, b, c in zip(src.tolist(), w.tolist(), idx[:m].tolist())))
        out.append("\n")
    if blocks:
        out.append("\n".join(blocks) + "\n")
    return "".join(out).encode()


def write_arcs_file(path: str, off, idx, wt=None) -> None:
    """arcs-cuda text of a CSR, written by C (fast enough for 1e8 arcs)."""
    off, idx, wt = _csr(off, idx, wt)
    n = len(off) - 1
    if _load().orc_write_arcs(path.encode(), n, _p64(off), _p32(idx), _p64(wt)) != 0:
        raise OSError(f"cannot write {path}")


def gen_rmat(scale: int, edge_factor: int, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
             threads: int | None = None):
    """R-MAT CSR (offsets uint64, heads uint32) by oracle.c: orc_gen_rmat, the
    same graph as the product's generator, without loading the product."""
    lib = _load()
    po, pi, m = _u64p(), _u32p(), ctypes.c_uint64()
    st = lib.orc_gen_rmat(scale, edge_factor, a, b, c, seed, int(threads or os.cpu_count() or 1),
                          ctypes.byref(po), ctypes.byref(pi), ctypes.byref(m))
    if st != 0:
        raise MemoryError(f"orc_gen_rmat failed ({st})")
    n = 1 << scale
    try:
        off = np.ctypeslib.as_array(po, shape=(n + 1,)).copy()
        idx = np.ctypeslib.as_array(pi, shape=(max(m.value, 1),))[: m.value].copy()
    finally:
        lib.orc_free(ctypes.cast(po, ctypes.c_void_p))
        lib.orc_free(ctypes.cast(pi, ctypes.c_void_p))
    return off, idx


def write_mdp_file(path: str, off, idx, wt=None, init=None) -> None:
    """Valmari MDP text of a CSR with initial colours as <blocks>, written by C
    (oracle.c: orc_write_mdp; the same text as mdp_text without merging)."""
    off, idx, wt = _csr(off, idx, wt)
    n = len(off) - 1
    init = None if init is None else np.ascontiguousarray(init, dtype=np.uint32)
    if _load().orc_write_mdp(path.encode(), n, _p64(off), _p32(idx), _p64(wt), _p32(init)) != 0:
        raise OSError(f"cannot write {path}")


def run_ref_rsc_file(path: str, timeout: float = 3600.0):
    """Runs the reference rsc on an arcs-cuda file; returns (internal refinement
    time in s, blocks, rounds in rsc's own convention, wall time in s)."""
    import time
    t0 = time.perf_counter()
    with open(path, "rb") as f:
        txt = subprocess.run([REF_RSC], stdin=f, capture_output=True, timeout=timeout, check=True).stdout.decode()
    wall = time.perf_counter() - t0
    lines = txt.split("\n")
    rounds = None
    for ln in lines[3:]:
        if ln.startswith("rounds "):
            rounds = int(ln.split()[1])
            break
    return float(lines[0]), int(lines[2]), rounds, wall


def _parse_ref_output(txt: str):
    lines = txt.strip().split("\n")
    t = float(lines[0])
    done = int(lines[1])
    nodes = int(lines[2])
    rounds = None
    labels = None
    for ln in lines[3:]:
        if ln.startswith("rounds "):
            rounds = int(ln.split()[1])
        elif ln.startswith("labels"):
            labels = np.array([int(x) for x in ln.split()[1:]], dtype=np.uint64)
    return t, done, nodes, rounds, labels


def _canon_u64(labels: np.ndarray) -> np.ndarray:
    _, inv = np.unique(labels, return_inverse=True)
    out, _ = canonicalize(inv.astype(np.uint32))
    return out


def run_ref_rsc(off, idx, wt=None, timeout: float = 600.0) -> OracleResult:
    """Run the reference rsc (src/rsc/rsc.cpp, unmodified) on a graph.
    Uniform initial colours only: rsc.cpp:118-121 fixes w = 1."""
    if not os.path.exists(REF_RSC):
        raise FileNotFoundError(REF_RSC)
    txt = subprocess.run([REF_RSC], input=arcs_cuda_text(off, idx, wt), capture_output=True,
                         timeout=timeout, check=True).stdout.decode()
    t, done, nodes, rounds, labels = _parse_ref_output(txt)
    n = len(off) - 1
    lab = _canon_u64(labels) if n else np.zeros(0, dtype=np.uint32)
    res = OracleResult(lab, nodes, rounds_gpu_from_cpu(rounds, nodes, n), rounds)
    res.time_s = t
    return res


def rounds_gpu_from_cpu(rounds_cpu: int, blocks: int, n: int) -> int:
    """rsc.cpp starts its block count at N (rsc.cpp:108-109); the GPU program
    starts at 1 (rbsc.cu:339).  They differ only when the first pass already
    yields N blocks (rsc stops one pass earlier) or a single block (rsc runs
    one pass more)."""
    if rounds_cpu == 1 and blocks == n and n != 1:
        return 2
    if rounds_cpu == 2 and blocks == 1 and n != 1:
        return 1
    return rounds_cpu


def run_ref_valmari(off, idx, wt=None, init=None, timeout: float = 600.0) -> OracleResult:
    """Run Valmari's minimiser (src/part_ref, unmodified) on a graph; initial
    colours go in as MDP <blocks>."""
    if not os.path.exists(REF_VALMARI):
        raise FileNotFoundError(REF_VALMARI)
    n = len(off) - 1
    merge = int(off[-1]) > n * n  # more arcs than the reader takes: merge parallel ones
    txt = subprocess.run([REF_VALMARI], input=mdp_text(off, idx, wt, init, merge=merge), capture_output=True,
                         timeout=timeout, check=True).stdout.decode()
    t, done, nodes, rounds, labels = _parse_ref_output(txt)
    n = len(off) - 1
    lab = _canon_u64(labels) if n else np.zeros(0, dtype=np.uint32)
    res = OracleResult(lab, nodes, -1, None)
    res.time_s = t
    return res
