"""bench.py -- colour refinement of R-MAT-24 on B200: edge-rounds/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the plain-refinement-at-scale configuration): directed R-MAT scale
24, edge factor 16, (a, b, c) = (0.57, 0.19, 0.19), duplicates and self-loops
removed, CSR with int64 offsets and int32 heads, initial colours
floor(log2(out_degree + 1)), refined to the fixpoint.  Synthetic and seeded:
the reference's own suite (LAW web graphs) is not available.

One step = one refinement of the resident graph from its initial colours to
the verified fixpoint (time-to-fixpoint).  metric = arcs x rounds / time.
The inputs (1 GB of heads, 134 MB of offsets) are larger than the 126 MB L2,
so no flush is needed between steps.

Multi-GPU: the path does not shard here (one graph, one GPU); N ranks run N
independent replicas, `value` is the sum over ranks of arcs x rounds divided
by the slowest rank's time.

--impl reference: the reference's own CPU program (src/rsc/rsc.cpp, compiled
unmodified into oracle/_ref/ref_rsc) on the same R-MAT-24 graph, built by the
oracle's generator (nothing of this package is loaded); one step = one rsc
round over the whole graph, timed between rsc's per-round sorts, after a single
parse of its input; rank 0 only.

Beside the line: `cpu_baseline` (the same program, a bounded sample of rounds
of the same graph, plus the oracle's rsc restatement on every host core) and
`reference_gpu_program` (src/rbsc/rbsc.cu, unmodified, one batch, on the same
graph: its own timer and block count).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge-rounds/s (R-MAT-24 colour refinement to the verified fixpoint)"
UNIT = "edge-rounds/s"


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(values, dist):
    """Element-wise maximum of every rank's values (the slowest rank's times);
    the values themselves with one rank.  NCCL reduces on the GPU, gloo on the
    host."""
    vals = [float(v) for v in values]
    if dist is None:
        return vals
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_value(world: int, arcs: int, rounds: int, steps: int, slowest_ms: float) -> float:
    """Whole-job edge-rounds/s of N replicas: every rank refines its own copy
    of the graph `steps` times; the job takes the slowest rank's time."""
    return world * arcs * rounds * steps / (slowest_ms / 1000.0)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def signature_traffic_per_arc(kernel: str = "k_signature"):
    """DRAM bytes per arc of the first-pass signature kernel from its committed
    ncu summary (profiles/<kernel>_rmat24.md, line 'traffic_bytes_per_arc: X'),
    or None."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_rmat24.md")
    try:
        for ln in open(p):
            if ln.startswith("traffic_bytes_per_arc:"):
                return float(ln.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.25)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.f.read().splitlines():
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def ref_rsc_round_samples(off, idx, samples: int, timeout: float = 1800.0):
    """The reference rsc (oracle/_ref/ref_rsc: src/rsc/rsc.cpp compiled
    unmodified) on one graph: the arcs-cuda text goes through a pipe, rsc's
    input is parsed once, and refinements run in forked children until they
    have reported `samples` round times (the time between successive entries
    of the per-round sort of rsc.cpp:130, one complete round each).  Returns
    {"round_s": [...], "runs": [{time_s, rounds, blocks}, ...]} where time_s is
    rsc's own refinement timer (rsc.cpp:116-147) of each full run."""
    import threading
    from oracle import oracle
    rfd, wfd = os.pipe()
    proc = subprocess.Popen([oracle.REF_RSC, "--round-samples", str(int(samples)), "--no-labels"], stdin=rfd,
                            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL)
    os.close(rfd)
    err = []

    def feed():
        try:
            oracle.write_arcs_file(f"/dev/fd/{wfd}", off, idx)
        except Exception as e:  # reported below
            err.append(e)
        finally:
            os.close(wfd)

    th = threading.Thread(target=feed)
    th.start()
    out, _ = proc.communicate(timeout=timeout)
    th.join()
    if err or proc.returncode != 0:
        raise RuntimeError(f"ref_rsc failed (rc {proc.returncode}): {err}")
    lines = out.decode().split("\n")
    runs, rs = [], []
    i = 0
    while i + 4 < len(lines) and lines[i + 3].startswith("rounds "):
        runs.append({"time_s": float(lines[i]), "blocks": int(lines[i + 2]), "rounds": int(lines[i + 3].split()[1])})
        rs.extend(float(x) for x in lines[i + 4].split()[1:])
        i += 5
    return {"round_s": rs, "runs": runs}


def cpu_baseline_reference(off, idx, samples: int = 4):
    """cpu_baseline of the bench line: the reference rsc on the workload's own
    graph (R-MAT-24), a bounded sample of `samples` rounds (about 10 s of
    refinement), single-threaded as rsc is; beside it the oracle's restatement
    of rsc on every host core (orc_refine_rsc_mt) over the full refinement of
    the same graph.  Falls back to the restatement alone when the reference
    binary was not built."""
    from oracle import oracle
    m = len(idx)
    sample = (f"{samples} rounds of rsc on the workload's own graph (R-MAT-24, {m} arcs); rsc.cpp:118-121 fixes "
              "uniform initial colours (the degree classes come out of its first round; same final partition); "
              "round time = interval between successive per-round sorts (rsc.cpp:130) in one refinement")

    def port_all_cores():
        try:
            thr = os.cpu_count() or 1
            t0 = time.perf_counter()
            r = oracle.refine_rsc(off, idx, threads=thr)
            t = time.perf_counter() - t0
            return {"value": m * r.rounds_cpu / t, "unit": UNIT, "cores": thr, "kind": "port", "time_s": t,
                    "rounds": r.rounds_cpu, "blocks": r.blocks,
                    "note": "orc_refine_rsc_mt: the same ranks as rsc, on pthreads; wall time of the call, refinement only"}
        except Exception as e:  # an informational figure: never fails the bench
            return {"unavailable": str(e)[:200]}

    if os.path.exists(oracle.REF_RSC):
        r = ref_rsc_round_samples(off, idx, samples)
        ts = r["round_s"][:samples]
        own = r["runs"][0]
        return {"value": m * len(ts) / sum(ts), "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample,
                "round_s": ts, "rsc_own_timer": {"time_s": own["time_s"], "rounds": own["rounds"],
                                                 "blocks": own["blocks"],
                                                 "edge_rounds_per_s": m * own["rounds"] / own["time_s"]},
                "host_cores": os.cpu_count(), "port_all_cores": port_all_cores()}
    pa = port_all_cores()
    return {"value": pa.get("value"), "unit": UNIT, "cores": pa.get("cores"), "kind": "port",
            "sample": "the oracle's rsc restatement, full refinement of the workload's graph", "host_cores": os.cpu_count()}


def reference_gpu_program(off, idx, blocks: int, timeout: float = 900.0):
    """The reference GPU program (src/rbsc/rbsc.cu, unmodified, its stdin served
    from memory: oracle/_ref/ref_rbsc_fast) on the workload's graph, one batch
    (edge_batch_size = M), uniform initial colours as it takes them.  Its own
    timer (rbsc.cu:272, 489-494) covers the H2D copies and the round loop; its
    "nodes" line must equal the blocks found here.  Informational."""
    import threading
    from oracle import oracle
    exe = os.path.join(oracle.REF_DIR, "ref_rbsc_fast")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_rbsc_fast was not built (reference tree absent at build time)"}
    rfd, wfd = os.pipe()
    t0 = time.perf_counter()
    proc = subprocess.Popen([exe, str(len(idx))], stdin=rfd, stdout=subprocess.PIPE, stderr=subprocess.PIPE)
    os.close(rfd)

    def feed():
        try:
            oracle.write_arcs_file(f"/dev/fd/{wfd}", off, idx)
        finally:
            os.close(wfd)

    th = threading.Thread(target=feed)
    th.start()
    try:
        out, errb = proc.communicate(timeout=timeout)
    except subprocess.TimeoutExpired:
        proc.kill()
        proc.communicate()
        th.join()
        return {"unavailable": f"no result within {timeout:.0f} s"}
    th.join()
    wall = time.perf_counter() - t0
    lines = out.decode().split("\n")
    if proc.returncode != 0 or len(lines) < 3:
        return {"unavailable": f"rc {proc.returncode}: {(out + errb).decode()[-200:]}"}
    t, done, nodes = float(lines[0]), int(lines[1]), int(lines[2])
    return {"program": "src/rbsc/rbsc.cu (unmodified), edge_batch_size = M, one GPU", "time_s": t, "done": done,
            "nodes": nodes, "same_block_count": nodes == blocks, "wall_s_with_parse": wall,
            "note": "its own timer: from after setup to the end of refinement, H2D of the arcs included"}


def config(n=None, m=None, scale=24, ef=16):
    return {"workload": f"rmat{scale}_ef{ef}", "model": "none (graph refinement)", "scale": scale, "edge_factor": ef,
            "rmat_abc": [0.57, 0.19, 0.19], "nodes": n, "arcs": m,
            "initial_colors": "floor(log2(out_degree+1))", "offsets": "int64", "indices": "int32",
            "l2": "no flush: inputs larger than L2 (heads 4 B/arc)", "parallelism": "replicas",
            "global_batch": 1, "seq_len": None}


def run_reference(args, rank, world):
    """The reference arm: rsc (src/rsc/rsc.cpp, unmodified) on the same
    workload graph, generated by the oracle (oracle.c: orc_gen_rmat, the same
    arcs as the product's generator) so that nothing of the product is
    loaded.  One step = one rsc round over the whole graph (rsc processes every
    arc and node in every round); W + K round samples from refinements forked
    after a single parse.  Rank 0 only."""
    if rank != 0:
        return 0
    from oracle import oracle
    if not os.path.exists(oracle.REF_RSC):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_rsc was not built (reference tree absent at build time)"}))
        return 0
    t0 = time.perf_counter()
    off, idx = oracle.gen_rmat(args.scale, args.ef, seed=args.seed)
    n, m = len(off) - 1, len(idx)
    gen_s = time.perf_counter() - t0
    r = ref_rsc_round_samples(off, idx, args.warmup + args.steps)
    rs = r["round_s"]
    timed = rs[args.warmup: args.warmup + args.steps]
    tot = sum(timed)
    value = m * len(timed) / tot
    own_t = sum(x["time_s"] for x in r["runs"])
    own_er = sum(m * x["rounds"] for x in r["runs"])
    sample = (f"one step = one rsc round over the whole R-MAT scale {args.scale} graph ({m} arcs, {n} nodes; "
              "rsc touches every arc and node every round); round time = interval between successive per-round "
              "sorts (rsc.cpp:130); rsc.cpp:118-121 fixes uniform initial colours (the degree classes come out of "
              "its first round; same final partition)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": len(timed), "warmup": args.warmup, "ms_per_step": 1000.0 * tot / len(timed),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config(n, m, args.scale, args.ef),
            "rounds": r["runs"][0]["rounds"], "blocks": r["runs"][0]["blocks"],
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample,
                             "host_cores": os.cpu_count()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "rsc_own_timer": {"runs": r["runs"], "edge_rounds_per_s": own_er / own_t},
            "generation_s": gen_s, "gpu_launches": 0,
            "program": "oracle/_ref/ref_rsc: src/rsc/rsc.cpp compiled unmodified (-O2), single-threaded"}
    print(json.dumps(line))
    return 0


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import rbsc_b200 as R

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    ctx = R.Context(local_rank, relabel=R.RELABEL_SORT if args.relabel == "sort" else R.RELABEL_HASH,
                    persistent=not args.no_persist)
    g = ctx.gen_rmat(args.scale, args.ef, seed=args.seed)
    n, m = g.n, g.m
    d_init = torch.empty(n, dtype=torch.int32, device="cuda")
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    g.degree_colors_device(d_init.data_ptr())
    torch.cuda.synchronize()

    if args.profile_refine:
        # one refinement with every kernel a separate launch (the host-driven
        # loop with CUDA events around each kernel): the form the ncu
        # summaries under profiles/ are taken from
        g.refine_device(d_init.data_ptr(), d_out.data_ptr())
        times, pr = g.profile(d_init.data_ptr())
        if rank == 0:
            print(json.dumps({"profile_refine": config(n, m, args.scale, args.ef), "rounds": pr.rounds,
                              "device_ms": pr.device_ms, "round_blocks": list(pr.round_blocks),
                              "times": times}))
        g.free()
        ctx.close()
        return 0

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        r = g.refine_device(d_init.data_ptr(), d_out.data_ptr())
    # the pass kernels' knobs chosen by the library's autotuner on this graph
    # (before the timed region; every candidate checked for the same result)
    tune = None
    if not args.no_autotune:
        tune = g.autotune(d_init.data_ptr())
        tune = {k: v for k, v in tune.items() if k != "table"}
        for _ in range(args.warmup):
            g.refine_device(d_init.data_ptr(), d_out.data_ptr())
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local_rank)
    clocks.start()
    t0 = time.perf_counter()
    results = []
    for _ in range(args.steps):
        results.append(g.refine_device(d_init.data_ptr(), d_out.data_ptr()))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier()
    clk = clocks.stop()
    dev_ms = sum(r.device_ms for r in results)
    rounds = results[0].rounds
    assert all(r.rounds == rounds and r.blocks == results[0].blocks and r.verified == 1 for r in results)
    launches = sum(r.kernel_launches for r in results)
    dev_ms = max_over_ranks([dev_ms], dist)[0]
    value = replica_value(world, m, rounds, args.steps, dev_ms)

    # per-kernel times: one refinement with CUDA events around every launch
    # (host-driven loop, same kernels and work as the timed graph-driven loop)
    times, pr = g.profile(d_init.data_ptr())
    per_pass = times.pop("per_pass")
    peak, peak_kind = measured_peaks()
    ob = 8
    # The dominant kernel is k_signature, and its largest launch is the first
    # pass (every arc).  Algorithmic bytes of a launch over `arcs` arcs: 4 B of
    # head + 4 B of gathered colour per arc, ob B of offsets + 8 B of
    # signature per node.  Its duration is taken live in the timed steps
    # (CUDA events around that launch on the library's stream); the later
    # passes' signature launches come from the host-driven profile above.
    p1 = per_pass[0]
    sig_ms_live = [r.first_signature_ms for r in results if r.first_signature_ms > 0]
    arcs1 = results[0].first_signature_arcs or p1["arcs"]
    sig_ms1 = statistics.median(sig_ms_live) if sig_ms_live else p1["signature_ms"]
    sig_bytes_p1 = 8 * arcs1 + n * (ob + 8)
    sig_bytes_all = sum(8 * p["arcs"] for p in per_pass) + len(per_pass) * n * (ob + 8)
    sig_ms_all = sum(p["signature_ms"] for p in per_pass)
    hot = results[0].first_signature_hot
    # the hot first pass by tensor copies (the default, sig_kernel 0 or 4) or
    # by 16-byte loads (sig_kernel 3), as the options in effect choose
    sigk = (tune or {}).get("best", {}).get("sig_kernel", 0)
    kname = ("k_signature_hot_tma" if sigk in (0, 4) else "k_signature_hot") if hot else "k_signature"
    tpa = signature_traffic_per_arc(kname)
    round_bytes = 8 * m + n * (ob + 28)
    ach = sig_bytes_p1 / (sig_ms1 / 1e3) / 1e9
    kdesc = (f"{kname} (first pass: every arc; the class ranks of the {hot} most pointed-to nodes "
             "read from shared memory" + ("; each warp's tile of heads brought into shared memory by the tensor "
                                          "memory accelerator)" if kname == "k_signature_hot_tma" else ")")
             if hot else f"{kname} (first pass: every arc)")
    roofline = {"bound": "hbm", "kernel": kdesc,
                "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                "traffic": None if tpa is None else tpa * arcs1,
                "algorithmic_bytes_per_launch": sig_bytes_p1, "arcs_per_launch": arcs1, "launch_ms": sig_ms1,
                "duration_source": "CUDA events in the timed steps" if sig_ms_live else "host-driven profile",
                "all_signature_launches": {"launches": len(per_pass), "ms": sig_ms_all,
                                           "algorithmic_bytes": sig_bytes_all,
                                           "achieved_gbs": sig_bytes_all / (sig_ms_all / 1e3) / 1e9,
                                           "frac": sig_bytes_all / (sig_ms_all / 1e3) / 1e9 / peak},
                "round_formula": {"bytes_per_round": round_bytes, "ms_per_round": dev_ms / args.steps / rounds,
                                  "frac": round_bytes / (dev_ms / args.steps / rounds / 1e3) / 1e9 / peak,
                                  "note": "8*M + N*(ob+28) per round as if every arc and node were processed every round"},
                "per_pass": per_pass, "init_ms": times["init_ms"], "setup_ms": times["setup_ms"],
                "persistent": {"passes": times["persist_passes"], "ms": times["persist_ms"],
                               "note": "passes after the hand-off run inside one cooperative k_refine_persistent launch"}}

    # end to end through the C ABI with host buffers (pinned), copies inside the timed region
    d_off, d_idx = g.device_csr()
    off_h = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    idx_h = torch.empty(m, dtype=torch.int32, pin_memory=True)
    init_h = torch.empty(n, dtype=torch.int32, pin_memory=True)
    out_h = torch.empty(n, dtype=torch.int32, pin_memory=True)

    class _Arr:
        def __init__(self, p, cnt, ts):
            self.__cuda_array_interface__ = {"shape": (cnt,), "typestr": ts, "data": (p, False), "version": 3}

    off_h.copy_(torch.as_tensor(_Arr(d_off, n + 1, "<i8"), device="cuda"))
    idx_h.copy_(torch.as_tensor(_Arr(d_idx, m, "<i4"), device="cuda"))
    init_h.copy_(d_init)
    torch.cuda.synchronize()
    off_np = off_h.numpy().view(np.uint64)
    idx_np = idx_h.numpy().view(np.uint32)
    init_np = init_h.numpy().view(np.uint32)
    out_np = out_h.numpy().view(np.uint32)
    e2e_res = []
    ctx.refine(off_np, idx_np, init=init_np, out=out_np)  # warm-up
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_res.append(ctx.refine(off_np, idx_np, init=init_np, out=out_np))
    e2e_wall = time.perf_counter() - t0
    e2e_s = sum(r.time_s for r in e2e_res)
    e2e_s = max_over_ranks([e2e_s], dist)[0]
    assert all(r.rounds == rounds and r.blocks == results[0].blocks for r in e2e_res)
    assert np.array_equal(out_np, d_out.cpu().numpy().view(np.uint32))
    e2e = {"value": world * m * rounds * args.e2e_steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(e2e_res[0].h2d_bytes), "d2h_bytes_per_step": int(e2e_res[0].d2h_bytes),
           "ms_per_step": 1000.0 * e2e_s / args.e2e_steps, "steps": args.e2e_steps,
           "h2d_ms": e2e_res[-1].h2d_ms, "d2h_ms": e2e_res[-1].d2h_ms,
           "path": "rbsc_refine (C ABI): pinned host CSR + colours in, labels out"}

    batched = None if args.batch_graphs <= 0 else run_batched(args, ctx, world, dist)
    # the served, LAW and streamed sections describe one GPU (the streamed one
    # alone pins 36 GB of host memory): they run at N = 1 only.  The main
    # context's cached buffers go back to CUDA first: the server sizes its
    # budget and its slots' buffer caches from the free device memory
    single = world == 1
    ctx.trim()
    served = None if args.serve_requests <= 0 or not single else run_served(args, world, dist, local_rank)
    law = None if args.law_steps <= 0 or not single else run_law(args, local_rank)
    streamed = None if args.stream_scale <= 0 or not single else run_streamed(args, ctx, local_rank)
    lump_f64 = None if args.f64_scale <= 0 or not single else run_lump_f64(args, ctx)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_reference(off_np, idx_np)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        ref_gpu = reference_gpu_program(off_np, idx_np, results[0].blocks)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": config(n, m, args.scale, args.ef), "rounds": rounds, "time_to_fixpoint_ms": dev_ms / args.steps,
                "blocks": results[0].blocks, "verify_ms": results[0].verify_ms,
                "phase_ms": {"init": results[-1].init_ms, "loop": results[-1].loop_ms, "verify": results[-1].verify_ms},
                "wall_ms_per_step": 1000.0 * wall / args.steps, "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": launches, "clocks": clk, "relabel": args.relabel, "autotune": tune, "batched": batched,
                "served": served, "law_cnr2000": law, "streamed": streamed, "lump_f64": lump_f64,
                "reference_gpu_program": ref_gpu}
        print(json.dumps(line))
    g.free()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _pinned(n, dtype):
    import torch
    tdt = {np.uint32: torch.int32, np.uint64: torch.int64}[dtype]
    return torch.empty(max(int(n), 1), dtype=tdt, pin_memory=True).numpy().view(dtype)


def _pinned_copy(a):
    out = _pinned(a.size, a.dtype.type)
    out[: a.size] = a
    return out[: a.size]


def run_batched(args, ctx, world, dist):
    """Small-graph batch: graphs/s of one batch refinement (all graphs side by
    side in one resident graph, one shared colour namespace) against one
    refinement call per graph, on the same GPU.  Inputs generated off the
    clock; both paths take host buffers and return host results."""
    import torch
    import rbsc_b200 as R
    G = args.batch_graphs
    off, idx, gn, lab = R.gen_wl_batch(G, 10, 500, 8, seed=args.seed)
    n, m = len(off) - 1, len(idx)
    off_p, idx_p, lab_p = _pinned_copy(off), _pinned_copy(idx), _pinned_copy(lab)
    bufs = R.batch_buffers(n, G, alloc=lambda k, dt: _pinned(k, dt))
    rg = ctx.upload(off_p, idx_p)
    tune = None
    if not args.no_autotune:
        d_lab = torch.from_numpy(lab.view(np.int32)).cuda()
        tune = rg.autotune(d_lab.data_ptr())
        tune = {k: v for k, v in tune.items() if k != "table"}
    for _ in range(2):
        rg.batch_refine(gn, lab_p, out=bufs)
    res_t, res_dev = [], []
    for _ in range(args.batch_steps):
        t0 = time.perf_counter()
        b = rg.batch_refine(gn, lab_p, out=bufs)
        res_t.append(time.perf_counter() - t0)
        res_dev.append(b.stats.device_ms)
    rg.free()
    ctx.batch_refine(off_p, idx_p, gn, lab_p, out=bufs)
    one_t = []
    for _ in range(args.batch_steps):
        t0 = time.perf_counter()
        b = ctx.batch_refine(off_p, idx_p, gn, lab_p, out=bufs)
        one_t.append(time.perf_counter() - t0)
    # one refinement call per graph, on the first `sample` graphs
    S = min(args.batch_sample, G)
    subs = []
    for k in range(S):
        a, e = int(gn[k]), int(gn[k + 1])
        o = off[a: e + 1].astype(np.int64)
        subs.append(((o - o[0]).astype(np.uint64), (idx[o[0]: o[-1]].astype(np.int64) - a).astype(np.uint32), lab[a:e]))
    for o, ix, l in subs[:20]:
        ctx.refine(o, ix, init=l)
    t0 = time.perf_counter()
    per = [ctx.refine(o, ix, init=l) for o, ix, l in subs]
    per_t = time.perf_counter() - t0
    for k, r1 in enumerate(per):  # each graph's partition = its part of the batch result
        assert np.array_equal(r1.labels, b.local[int(gn[k]): int(gn[k + 1])])
    gs = [ctx.upload(o, ix) for o, ix, _ in subs]
    for gg, (_, _, l) in zip(gs, subs):  # buffers and captured loop in place
        gg.refine(l)
    t0 = time.perf_counter()
    for gg, (_, _, l) in zip(gs, subs):
        gg.refine(l)
    per_res_t = time.perf_counter() - t0
    for gg in gs:
        gg.free()
    ts = max_over_ranks([float(np.median(one_t)), float(np.median(res_t)), per_t, per_res_t], dist)
    one_s, res_s, per_t, per_res_t = ts
    return {"workload": f"{G} graphs: n ~ U[10, 500]; even: Erdos-Renyi p = 4/(n-1), odd: random 3-regular; "
                        "symmetric arcs; labels U{1..8}",
            "graphs": G * world, "nodes": n, "arcs": m, "rounds": b.stats.rounds, "blocks": b.stats.blocks,
            "graphs_per_s": G * world / one_s, "ms": 1000.0 * one_s,
            "resident_graphs_per_s": G * world / res_s, "resident_ms": 1000.0 * res_s,
            "device_ms": float(np.median(res_dev)),
            "per_launch_graphs_per_s": S * world / per_t, "per_launch_resident_graphs_per_s": S * world / per_res_t,
            "per_launch_sample": S, "autotune": tune,
            "speedup": (G / one_s) / (S / per_t), "speedup_resident": (G / res_s) / (S / per_res_t),
            "paths": {"batched": "rbsc_batch_refine: host CSR + labels in (pinned), colours, local labels, "
                                 "histograms, fingerprints out",
                      "batched_resident": "rbsc_graph_batch_refine on the uploaded batch",
                      "per_launch": "rbsc_refine per graph: host CSR + labels in, labels out",
                      "per_launch_resident": "rbsc_graph_refine per uploaded graph (each refined once before)"}}


def served_pool(args):
    """Distinct graphs of the served mix, generated on the host off the clock:
    arcs log-uniform in [1e3, 5e7], kinds in turn a random lift (x32 of an
    Erdos-Renyi base of mean degree 8), R-MAT (a, b, c as the main workload,
    edge factor about 16) and Erdos-Renyi (mean degree 8); int32 heads."""
    import rbsc_b200 as R
    rng = np.random.default_rng(args.seed + 77)
    pool = []
    for k in range(args.serve_pool):
        e = float(np.exp(rng.uniform(np.log(1e3), np.log(5e7))))
        seed = args.seed * 1000 + k
        if k % 3 == 0:
            off, idx = R.gen_lift_host(max(2, int(round(e / (8 * 32)))), 8.0, 32, seed=seed)
            kind = "lift"
        elif k % 3 == 1:
            scale = max(4, int(round(np.log2(e / 16))))
            off, idx = R.gen_rmat_host(scale, max(1, int(round(e / 2 ** scale))), seed=seed)
            kind = "rmat"
        else:
            off, idx = R.gen_er_host(max(2, int(e / 8)), 8.0, seed=seed)
            kind = "er"
        pool.append((kind, _pinned_copy(off), _pinned_copy(idx)))
    return pool


def served_breakdown(ctx, pool, pick):
    """Where a one-graph-per-call refinement of the served mix spends its time,
    per request of the stream (pool graphs weighted by how often they are
    drawn): wall time of the call, device time of the refinement (events
    around it: kernels and the gaps between them), host-link copies (bytes and
    time), the rest on the host.  Every request's graph must cross the host
    link, so no server on one GPU fed from host memory can beat
    bytes / (measured copy bandwidth) per request: that floor bounds the
    served throughput and its speed-up over one call per graph."""
    import numpy as np
    import torch
    hbuf = torch.empty(1 << 28, dtype=torch.int32, pin_memory=True)
    dbuf = torch.empty(1 << 28, dtype=torch.int32, device="cuda")
    bw = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dbuf.copy_(hbuf, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        bw.append(4.0 * (1 << 28) / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del hbuf, dbuf
    link = max(bw)
    rows = {}
    for k in sorted(set(pick.tolist())):
        _, off, idx = pool[k]
        ctx.refine(off, idx)
        ts = [ctx.refine(off, idx) for _ in range(3)]
        r = min(ts, key=lambda x: x.time_s)
        rows[k] = (1e3 * r.time_s, r.device_ms, r.h2d_ms, r.d2h_ms, r.h2d_bytes + r.d2h_bytes)
    w = np.array([rows[int(k)] for k in pick])
    wall, dev, h2d, d2h, nbytes = (float(x) for x in w.mean(axis=0))
    link_ms = nbytes / (link * 1e9) * 1e3
    out = {"per_request_mean": {"wall_ms": wall, "device_ms": dev, "h2d_ms": h2d, "d2h_ms": d2h,
                                "host_ms": max(0.0, wall - dev - h2d - d2h), "bytes": nbytes},
           "host_link_gbs_measured": link,
           "host_link_floor_ms_per_request": link_ms,
           "bound_graphs_per_s": 1e3 / link_ms,
           "one_per_call_graphs_per_s": 1e3 / wall,
           "note": "the bound is the host link alone (every request's arrays cross it once); device_ms of one call "
                   "per graph is context only: packing small graphs into one batch refinement lowers the device "
                   "time per graph"}
    out["bound_speedup_vs_one_per_call"] = out["bound_graphs_per_s"] / out["one_per_call_graphs_per_s"]
    return out


def run_served(args, world, dist, local_rank):
    """Served refinement (the served-stream configuration): a Poisson stream of
    requests drawn from a pool of seeded graphs, through a server with
    continuous batching (several slots whose work overlaps on the GPU,
    admission by device footprint, small jobs packed into one batch
    refinement) against the same stream through a server with one slot and no
    packing (one graph per launch, in arrival order).  Latency = submit to
    labels in host memory; every partition is checked against a refinement
    of the same graph alone."""
    import torch
    import rbsc_b200 as R
    pool = served_pool(args)
    rng = np.random.default_rng(args.seed + 99)
    N = args.serve_requests
    pick = rng.integers(0, len(pool), size=N)
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, size=N))
    ref = {}
    with R.Context(local_rank) as c:
        for k in sorted(set(pick.tolist())):
            _, off, idx = pool[k]
            ref[k] = c.refine(off, idx)
        breakdown = served_breakdown(c, pool, pick)

    def start(slots, pack):
        kw = dict(slots=slots) if pack else dict(slots=slots, pack_max_graphs=1)
        srv = R.Server(local_rank, **kw)
        for _ in range(2 * slots):   # every slot's buffer pool warmed on every pool graph
            ids = [srv.submit(off, idx) for _, off, idx in pool]
            for j in ids:
                srv.wait(j)
        return srv

    def run(srv, poisson):
        st0 = srv.stats()
        ids = []
        t0 = time.perf_counter()
        for i in range(N):
            if poisson:
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            _, off, idx = pool[pick[i]]
            ids.append(srv.submit(off, idx))
        res = [srv.wait(j) for j in ids]
        span = time.perf_counter() - t0
        st = srv.stats()
        for i, r in enumerate(res):
            a = ref[int(pick[i])]
            assert r.status == 0 and r.blocks == a.blocks and np.array_equal(r.labels, a.labels), r.error
        lat = np.array([r.latency_ms for r in res])
        q = np.array([r.queue_ms for r in res])
        sv = np.array([r.service_ms for r in res])
        dec = np.array_split(lat, 10)
        return {"graphs_per_s": N / span, "span_s": span, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "queue_ms_mean": float(q.mean()), "service_ms_mean": float(sv.mean()),
                "service_ms_p50": float(np.percentile(sv, 50)), "service_ms_p99": float(np.percentile(sv, 99)),
                "latency_mean_by_arrival_decile_ms": [float(d.mean()) for d in dec],
                "packed_jobs": st["packed_jobs"] - st0["packed_jobs"], "executions": st["batches"] - st0["batches"],
                "peak_busy_slots": st["peak_busy_slots"], "peak_reserved_bytes": st["peak_reserved"]}

    with start(args.serve_slots, True) as srv:
        served, served_sat = run(srv, True), run(srv, False)
    with start(1, False) as srv:
        serial, serial_sat = run(srv, True), run(srv, False)
    out = {"workload": f"Poisson stream at {args.serve_rate:g} req/s, {N} requests drawn uniformly from "
                       f"{len(pool)} seeded graphs: arcs log-uniform in [1e3, 5e7], kinds in turn random lift x32 / "
                       f"R-MAT / Erdos-Renyi, uniform initial colours",
           "requests": N, "pool_arcs": [int(len(p[2])) for p in pool],
           "served": served, "serial": serial, "served_saturated": served_sat, "serial_saturated": serial_sat,
           "slots": args.serve_slots, "bit_exact": True,
           "paths": {"served": "rbsc_serve_submit / rbsc_serve_wait: several slots, packing, footprint admission",
                     "serial": "the same server with one slot and no packing: one rbsc_refine per request in order"}}
    out["saturated_speedup"] = out["served_saturated"]["graphs_per_s"] / out["serial_saturated"]["graphs_per_s"]
    out["breakdown"] = breakdown
    return out


def run_law(args, local_rank):
    """The reference's own LAW sample, cnr-2000 (325,557 nodes, 3,216,152 arcs,
    173 rounds), decoded from its BV files by rbsc_bv_load at build time
    (oracle/_ref/cnr-2000.npz; absent -> section skipped).  Uniform initial
    colours, as the reference programs run it.  Resident refinement (device
    time) and the one-shot call from page-locked host arrays; the partition is
    checked against the reference programs' (tests/golden/law_cnr2000.json),
    whose recorded reference-GPU-program time on a B200 is quoted beside.
    A context of its own with the library's default knobs: the main context
    carries the knobs that the autotuner chose for the batch of small graphs
    (with its hand-off limit of 2^18 arcs, cnr-2000's passes stayed in the
    pass loop longer instead of the persistent kernel: 15.5 ms instead of 7.2
    in one run)."""
    import rbsc_b200 as R
    from oracle import oracle  # the decoded graph only; nothing under oracle/ runs here
    g0 = oracle.load_law()
    if g0 is None:
        return None
    with R.Context(local_rank) as ctx:
        return _run_law(args, ctx, g0)


def _run_law(args, ctx, g0):
    import hashlib
    fx = json.load(open(os.path.join(ROOT, "tests", "golden", "law_cnr2000.json")))
    off, idx = _pinned_copy(g0[0]), _pinned_copy(g0[1])
    m = len(idx)
    g = ctx.upload(off, idx)
    for _ in range(3):
        g.refine_device()
    res = [g.refine_device() for _ in range(args.law_steps)]
    g.free()
    out_p = _pinned(len(off) - 1, np.uint32)
    ctx.refine(off, idx, out=out_p)
    one = [ctx.refine(off, idx, out=out_p) for _ in range(args.law_steps)]
    lab = out_p[: len(off) - 1]
    ok = (one[-1].blocks == fx["blocks"] and one[-1].rounds == fx["rounds"]
          and hashlib.sha256(np.ascontiguousarray(lab).tobytes()).hexdigest() == fx["labels_sha256"])
    assert ok, "cnr-2000 partition differs from the reference programs'"
    dev = statistics.median([r.device_ms for r in res])
    e2e = statistics.median([r.time_s for r in one]) * 1e3
    ref_gpu = next((r["time_s"] for r in fx.get("ref_rbsc", {}).get("runs", []) if r["batch"] >= m), None)
    return {"workload": "cnr-2000 (LAW; the reference's webgraph-rs/data sample), uniform initial colours",
            "nodes": len(off) - 1, "arcs": m, "rounds": res[0].rounds, "blocks": res[0].blocks,
            "ms_to_fixpoint": dev, "edge_rounds_per_s": m * res[0].rounds / (dev / 1e3),
            "e2e_ms": e2e, "e2e_edge_rounds_per_s": m * res[0].rounds / (e2e / 1e3),
            "same_partition_as_reference_programs": ok,
            "reference_gpu_program_ms_recorded": None if ref_gpu is None else 1e3 * ref_gpu,
            "reference_note": "reference GPU program time: its own timer (H2D + refinement), one batch, recorded on a "
                              "B200 by tests/golden/make_law_golden.py --gpu; compare with e2e_ms"}


def run_lump_f64(args, ctx):
    """Lumping with double weights (rbsc_refine_f64): R-MAT scale
    args.f64_scale, edge factor 16, every arc weighted k/2 with k uniform in
    0..8 (decimal texts "0.0" .. "4.0" in the minimiser's MDP text; its reader
    turns every one of them into exactly k/2).  One-shot calls from host
    arrays (device time and wall time of the call).  cpu_baseline: Valmari's
    minimiser built with double weights (oracle/_ref/ref_valmari_f64, compiled
    unmodified from the reference's src/part_ref), single-threaded, its own
    timer around minimize(); its partition must equal ours."""
    import numpy as np
    import rbsc_b200 as R
    off, idx = R.gen_rmat_host(args.f64_scale, 16, seed=args.seed)
    n, m = len(off) - 1, len(idx)
    rng = np.random.default_rng(args.seed)
    k = rng.integers(0, 9, m)
    w = k / 2.0
    ctx.refine_f64(off, idx, w)
    res = [ctx.refine_f64(off, idx, w) for _ in range(args.f64_steps)]
    r0 = res[0]
    assert all(r.blocks == r0.blocks and r.rounds == r0.rounds and r.verified == 1 for r in res)
    dev = statistics.median([r.device_ms for r in res])
    wall = statistics.median([r.time_s for r in res]) * 1e3
    out = {"workload": f"rmat{args.f64_scale}_ef16, weights k/2 (k uniform 0..8), uniform initial colours",
           "nodes": n, "arcs": m, "rounds": r0.rounds, "blocks": r0.blocks, "device_ms": dev, "call_ms": wall,
           "edge_rounds_per_s": m * r0.rounds / (dev / 1e3), "gpu_launches_per_call": int(r0.kernel_launches),
           "h2d_bytes": int(r0.h2d_bytes), "d2h_bytes": int(r0.d2h_bytes), "cpu_baseline": None}
    if args.no_cpu_baseline:
        return out
    import subprocess
    from oracle import oracle  # the reference program, as the checker and CPU baseline
    if not os.path.exists(oracle.REF_VALMARI_F64):
        out["cpu_baseline"] = {"unavailable": "oracle/_ref/ref_valmari_f64 not built"}
        return out
    texts = [f"{x / 2:.1f}" for x in range(9)]
    lines = [f"{n} 0 0 {m} 1\n"]
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64))) + 1
    tk = np.array(texts)[k]
    lines.append("\n".join(f"{a} {t} {b}" for a, t, b in zip(src.tolist(), tk.tolist(), (idx.astype(np.int64) + 1).tolist())))
    lines.append("\n")
    t0 = time.perf_counter()
    txt = subprocess.run([oracle.REF_VALMARI_F64], input="".join(lines).encode(), capture_output=True, check=True,
                         timeout=1800).stdout.decode().split("\n")
    wall_ref = time.perf_counter() - t0
    lab = np.array(txt[3].split()[1:], dtype=np.int64)
    # canonical labels of the minimiser's block numbers: smallest state id
    first = {}
    canon = np.empty(n, dtype=np.uint32)
    for i, b in enumerate(lab.tolist()):
        canon[i] = first.setdefault(b, i)
    out_lab = ctx.refine_f64(off, idx, w).labels
    out["cpu_baseline"] = {"kind": "reference", "program": "Valmari minimiser, MDP_weight_is_double (src/part_ref)",
                           "cores": 1, "minimize_s": float(txt[0]), "wall_s_with_parse": wall_ref,
                           "blocks": int(txt[2]), "same_partition": bool(np.array_equal(canon, out_lab)),
                           "speedup_device": float(txt[0]) * 1e3 / dev, "speedup_call": float(txt[0]) * 1e3 / wall}
    assert out["cpu_baseline"]["same_partition"], "double-weight lumping differs from the reference minimiser"
    return out


def run_streamed(args, ctx, local_rank):
    """Arcs in host memory (the out-of-HBM configuration): R-MAT scale
    args.stream_scale, edge factor args.stream_ef, generated on the device in
    source buckets into page-locked host memory; int64 offsets, int32 heads,
    degree-bucket initial colours.  Each signature pass over the full arc set
    streams it in batches of a quarter of the arcs through two device buffers,
    the copy of the next batch beside the signature kernel of the current one.
    The same graph refined from device memory gives the parity check (labels
    equal) and the in-HBM time beside it."""
    import torch
    t0 = time.perf_counter()
    pg = ctx.gen_rmat_pinned(args.stream_scale, args.stream_ef, seed=args.seed)
    gen_s = time.perf_counter() - t0
    n, m = pg.n, pg.m
    # host-link reference: one page-locked 4 GiB host->device copy, best of 3
    hbuf = torch.empty(1 << 30, dtype=torch.int32, pin_memory=True)
    dbuf = torch.empty(1 << 30, dtype=torch.int32, device="cuda")
    h2d = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dbuf.copy_(hbuf, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        h2d.append(4.0 * (1 << 30) / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del hbuf, dbuf
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    g = ctx.upload_streamed(pg.off, pg.idx)
    up_s = time.perf_counter() - t0
    d_init = torch.empty(n, dtype=torch.int32, device="cuda")
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    g.degree_colors_device(d_init.data_ptr())
    torch.cuda.synchronize()
    for _ in range(1):
        g.refine_device(d_init.data_ptr(), d_out.data_ptr())
    res = [g.refine_device(d_init.data_ptr(), d_out.data_ptr()) for _ in range(args.stream_steps)]
    times, pr = g.profile(d_init.data_ptr())
    labels_stream = d_out.cpu()
    g.free()
    ctx.trim()
    ms = [r.device_ms for r in res]
    rounds = res[0].rounds
    p1 = times["per_pass"][0]
    # the same graph from device memory
    t0 = time.perf_counter()
    g2 = ctx.upload(pg.off, pg.idx)
    up2_s = time.perf_counter() - t0
    g2.refine_device(d_init.data_ptr(), d_out.data_ptr())
    res2 = [g2.refine_device(d_init.data_ptr(), d_out.data_ptr()) for _ in range(args.stream_steps)]
    same = bool(torch.equal(labels_stream, d_out.cpu())) and res2[0].blocks == res[0].blocks and res2[0].rounds == rounds
    assert same, "streamed and in-HBM refinements differ"
    g2.free()
    pg.free()
    ctx.trim()
    med = statistics.median(ms)
    sig1 = p1["signature_ms"]
    return {"workload": f"R-MAT scale {args.stream_scale}, edge factor {args.stream_ef} (a, b, c = 0.57, 0.19, 0.19), "
                        "duplicates and self-loops removed; int64 offsets, int32 heads in page-locked host memory; "
                        "initial colours floor(log2(out_degree+1)); batches of 25% of the arcs per streamed pass",
            "nodes": n, "arcs": m, "rounds": rounds, "blocks": res[0].blocks,
            "edge_rounds_per_s": m * rounds / (med / 1e3), "ms_to_fixpoint": med, "ms_all": ms,
            "streamed_passes": res[0].streamed_passes, "streamed_bytes": res[0].streamed_bytes,
            "first_pass_signature_ms": sig1, "first_pass_arcs": p1["arcs"],
            "first_pass_h2d_gbs": 4.0 * p1["arcs"] / (sig1 / 1e3) / 1e9,
            "h2d_copy_gbs_measured": max(h2d),
            "host_link_frac": (4.0 * p1["arcs"] / (sig1 / 1e3) / 1e9) / max(h2d),
            "per_pass": times["per_pass"][:6], "verify_ms": res[0].verify_ms,
            "in_hbm": {"ms_to_fixpoint": statistics.median([r.device_ms for r in res2]),
                       "upload_s": up2_s, "same_partition": same},
            "generation_s": gen_s, "upload_streamed_s": up_s,
            "path": "rbsc_graph_upload_streamed + rbsc_graph_refine_device; parity against rbsc_graph_upload of the "
                    "same arrays (labels, blocks, rounds equal)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--relabel", choices=["hash", "sort"], default="hash")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference GPU program (src/rbsc/rbsc.cu) on the same graph")
    ap.add_argument("--batch-graphs", type=int, default=100000, help="small-graph batch size (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--batch-sample", type=int, default=1000, help="graphs refined one call each")
    ap.add_argument("--serve-requests", type=int, default=600, help="served stream length (0: skip)")
    ap.add_argument("--law-steps", type=int, default=5, help="refinements of the LAW sample cnr-2000 (0: skip)")
    ap.add_argument("--stream-scale", type=int, default=28, help="R-MAT scale of the streamed graph (0: skip)")
    ap.add_argument("--stream-ef", type=int, default=32)
    ap.add_argument("--stream-steps", type=int, default=2)
    ap.add_argument("--f64-scale", type=int, default=20, help="R-MAT scale of the double-weight lumping (0: skip)")
    ap.add_argument("--f64-steps", type=int, default=3)
    ap.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-pool", type=int, default=48, help="distinct graphs the requests draw from")
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default pass-kernel knobs")
    ap.add_argument("--no-persist", action="store_true",
                    help="every pass as separate launches (no persistent kernel for small active sets)")
    ap.add_argument("--profile-f64", action="store_true",
                    help="only the double-weight lumping: one warm-up and one profiled call, for ncu")
    ap.add_argument("--profile-refine", action="store_true",
                    help="only one host-driven refinement (every kernel its own launch), for ncu")
    args = ap.parse_args()
    rank, world, local_rank = env_rank()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.profile_f64:
        # the double-weight lumping alone (one warm-up call, one profiled
        # call), for the ncu launch list under profiles/
        import numpy as np
        import rbsc_b200 as R
        off, idx = R.gen_rmat_host(args.f64_scale, 16, seed=args.seed)
        w = np.random.default_rng(args.seed).integers(0, 9, len(idx)) / 2.0
        with R.Context(local_rank) as ctx:
            ctx.refine_f64(off, idx, w)
            r = ctx.refine_f64(off, idx, w)
        print(json.dumps({"profile_f64": f"rmat{args.f64_scale}_ef16", "rounds": r.rounds, "blocks": r.blocks,
                          "device_ms": r.device_ms, "gpu_launches": int(r.kernel_launches)}))
        return 0
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
