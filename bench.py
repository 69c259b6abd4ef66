"""Exact-BC TEPS benchmark of the B200 engine (one JSON line on rank 0).

Workload (N=1): R-MAT scale 20, edge factor 16, (a,b,c,d) = (0.57,0.19,0.19,
0.05), seed 2, plus pendant trees on 10% of the vertices (Geometric sizes,
mean 4); 4096 sources drawn uniformly without replacement with seed 2;
pendant-tree pruning on (--prune degree1: one layer, as bc2d -H 1); FP64
delta/bc, uint64 sigma.  Seeded synthetic input:
no public dataset is involved.

A step = one exact-BC pass over the step's sources (one kernel launch of the
engine), preceded (untimed) by a reset of the bc accumulator and an L2 flush
(a 512 MiB device write, larger than the 126 MB L2).  With N ranks (one per
GPU; `--gpus N` starts them itself through torch.distributed.run when no
launcher did) every rank takes its own block of 4096 sources (weak scaling)
and the step ends with the path's one exchange: the FP64 bc partials
all-gathered over NCCL and added in rank order (bit-reproducible).

  value  TEPS = sum over all ranks' sources of the undirected edge count of
         the source's component / max-over-ranks device time (CUDA events on
         the launching stream), graph and sources resident in HBM.
  e2e    the same metric through the C ABI with host buffers: per step
         bcg_graph_create (pinned host CSR -> device, pruning, tiles),
         bcg_run (host source list), [all-reduce], bcg_get_bc (device -> host).
  roofline  algorithmic bytes of the sweep kernel = sum over sources of
         16*m_comp + 56*n_comp + 8 (int32 ids, uint64 sigma, FP64 delta/bc),
         divided by its CUDA-event time; peak = MEASURED_PEAKS.json hbm_gbs.
  cpu_baseline  the oracle (CPU Brandes restatement, all host threads) on a
         bounded sample of the same workload's sources, rank 0 at N=1.
--impl reference: the reference program has no CPU Brandes; its path is timed
through the oracle port on the host cores (all threads), each step a bounded
sample of the same sources, on the same graph rebuilt by oracle/graphgen.py
(no product library is loaded by that arm).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ck-bc_b200"))

WORKLOAD = "rmat20_ef16_pendant10_4096src"
SPEC = "rmat:scale=20,ef=16,a=0.57,b=0.19,c=0.19,seed=2,pendant_frac=0.1,pendant_mean=4"
SRC_SEED = 2
NSRC = 4096
METRIC = "exact-BC TEPS (sources*edges/s)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        busy = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_source(prune: str, kernel: str):
    """DRAM bytes per root of the sweep kernel from the committed ncu summary
    of the same pruning mode (profiles/sweep_traffic.json), if it was captured
    from the same kernel instantiation; else None and the reason."""
    p = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d.get(prune)
        if e is None:
            return None, ""
        if e.get("kernel") != kernel:
            return None, (f"no ncu capture of {kernel} in this pruning mode (the committed one is of "
                          f"{e.get('kernel')}, an earlier build)")
        return float(e["dram_bytes_per_source"]), e.get("note", "")
    except Exception:
        return None, ""


def rank_sources(sampler, n, per_rank, rank, world):
    """This rank's block of the workload's sources: per_rank * world distinct
    sources drawn with the workload's seed, cut into contiguous blocks in rank
    order (weak scaling: every rank runs per_rank sources)."""
    sys.path.insert(0, os.path.join(ROOT, "ck-bc_b200"))
    import shard

    return shard.shard_sources(sampler(n, per_rank * world, SRC_SEED), rank, world)


def combine_bc(bc_t):
    """The step's one exchange: every rank's FP64 bc partial summed in rank
    order (all-gather, then a fixed-order add), so the result is the same
    bits on every run and every rank."""
    import shard

    return shard.reduce_bc(bc_t, deterministic=True)


def relaunch(args):
    """--gpus N > 1 without a launcher: start N ranks of this script with
    torch.distributed.run (one per GPU, rendezvous on 127.0.0.1) and return
    its exit code; rank 0 prints the JSON line."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    log(f"starting {args.gpus} ranks: {' '.join(cmd[4:])}")
    return subprocess.call(cmd)


def cpu_baseline(offs, adj, sources, budget_s=15.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle

    nt = oracle.max_threads()
    done = 0
    edges = 0
    t0 = time.perf_counter()
    chunk = max(nt, 1)
    while done < len(sources) and time.perf_counter() - t0 < budget_s:
        s = sources[done:done + chunk]
        _, st = oracle.bc(offs, adj, s, nthreads=nt)
        edges += st["teps_edges"]
        done += len(s)
    el = time.perf_counter() - t0
    out = {"value": edges / el if el > 0 else None, "unit": "TEPS", "cores": nt, "kind": "port",
           "sample": f"first {done} of the {len(sources)} workload sources, oracle/brandes.c FP64 Brandes on the "
                     f"unpruned graph (no pendant folding), {nt} OpenMP threads, {el:.1f} s"}
    # the same sources with pendant trees folded, as the GPU arm computes them
    # (oracle/trees_ref.cpp); the one-off peeling is charged pro rata to the
    # sample's share of the workload's sources
    t1 = time.perf_counter()
    _, tst = oracle.bc_trees(offs, adj, sources[:done], nthreads=nt)
    el2 = time.perf_counter() - t1
    charged = el2 - tst["peel_seconds"] * (1.0 - done / len(sources))
    out["pruned"] = {"value": tst["teps_edges"] / charged if charged > 0 else None, "unit": "TEPS", "cores": nt,
                     "sample": f"the same {done} sources, oracle/trees_ref.cpp: pendant trees folded, reach-weighted "
                               f"FP64 Brandes from {tst['roots']} anchors, closed-form tree terms; {el2:.1f} s, of "
                               f"which peeling {tst['peel_seconds']:.2f} s is charged for {done}/{len(sources)}"}
    return out


def run_reference(args, rank, world):
    """--impl reference: the reference path's CPU restatement, all host threads.
    The graph and sources come from oracle/graphgen.py (the seeded generators
    restated in numpy, bit-identical to the library's), so this arm loads
    only oracle/ code."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import graphgen
    import oracle

    t_gen = time.perf_counter()
    offs, adj = graphgen.generate(args.graph)
    n = len(offs) - 1
    srcs = rank_sources(graphgen.sample_sources, n, args.sources, 0, 1)
    log(f"[reference] graph n={n} nnz={len(adj)} generated in {time.perf_counter() - t_gen:.1f}s (numpy)")
    nt = oracle.max_threads()
    per_step = max(nt, 1)
    times, edges = [], []
    pos = 0
    for i in range(args.warmup + args.steps):
        s = srcs[pos:pos + per_step]
        pos = (pos + per_step) % (len(srcs) - per_step)
        t0 = time.perf_counter()
        _, st = oracle.bc(offs, adj, s, nthreads=nt)
        el = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(el)
            edges.append(st["teps_edges"])
    tot_t = sum(times)
    val = sum(edges) / tot_t if tot_t > 0 else None
    out = {"metric": METRIC, "value": val, "unit": "TEPS", "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / max(1, len(times)),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "graph": args.graph, "n": n, "m": len(adj) // 2,
                      "sources_per_gpu": args.sources, "source_seed": SRC_SEED, "pruning": "none",
                      "sample_per_step": per_step},
           "cpu_baseline": {"value": val, "unit": "TEPS", "cores": nt, "kind": "port",
                            "sample": f"{per_step} sources per step of the workload's {args.sources}, "
                                      f"oracle/brandes.c FP64 Brandes on the unpruned graph (no pendant "
                                      f"folding; the reference has no CPU Brandes), {nt} OpenMP threads"},
           "e2e": {"value": val, "unit": "TEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def run_batched(args, rank, world):
    """Batched form (all-sources exact BC of every graph) against the plain
    per-graph loop (bcg_graph_create + bcg_run over all vertices + bcg_get_bc
    + bcg_graph_destroy for each graph).  Graphs: the front of the seeded
    2000-graph set (ck-bc_b200/workloads.py), optionally capped by scale.  One
    GPU (replicas only: with N ranks every rank runs the same set)."""
    import numpy as np
    import torch

    import bcg
    import workloads

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs = [s for s in workloads.batched_specs()[:args.graphs] if workloads.spec_scale_ef(s)[0] <= args.max_scale]
    t_gen = time.perf_counter()
    graphs = [bcg.generate(s) for s in specs]
    log(f"{len(graphs)} graphs generated in {time.perf_counter() - t_gen:.1f}s")
    # plain loop (one warm-up graph first)
    with bcg.Graph(*graphs[0]) as G:
        G.run(np.arange(len(graphs[0][0]) - 1, dtype=np.uint32))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_edges, plain_kernel_ms = 0, 0.0
    for offs, adj in graphs:
        with bcg.Graph(offs, adj) as G:
            st = G.run(np.arange(len(offs) - 1, dtype=np.uint32))
            G.bc()
        plain_edges += st.teps_edges
        plain_kernel_ms += st.kernel_ms
    plain_s = time.perf_counter() - t0
    # batched: resident union, autotuned, captured launch replayed every step
    t0 = time.perf_counter()
    B = bcg.Batch(graphs)
    create_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tune = B.autotune()
    tune_s = time.perf_counter() - t0
    for _ in range(max(1, args.warmup)):
        B.run()
        B.reset()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    kern, wall, edges = [], [], 0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = B.run()
        for i in range(len(graphs)):
            B.bc(i)
        wall.append(time.perf_counter() - t0)
        kern.append(st.kernel_ms)
        edges = st.teps_edges
        B.reset()
    clk = clocks.stop()
    info = B.info()
    B.close()
    assert edges == plain_edges, (edges, plain_edges)
    k_s = sum(kern) / len(kern) / 1e3
    w_s = sum(wall) / len(wall)
    out = {"metric": "batched exact-BC TEPS (all sources of every graph)", "value": edges / k_s, "unit": "TEPS",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * k_s,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "impl": "bcg-batched",
           "config": {"workload": "batched_2000_seed4_prefix", "graphs": len(graphs), "first": args.graphs,
                      "max_scale": args.max_scale, "edges_per_step": edges, "width": info["width"],
                      "tile": [info["tile_vertices"], info["tile_entries"]], "captured": info["captured"],
                      "packed_batches": info["nbatch"]},
           "graphs_per_s": len(graphs) / w_s,
           "e2e": {"value": edges / w_s, "unit": "TEPS", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": int(8 * sum(len(o) - 1 for o, _ in graphs)),
                   "path": "bcg_batch_run (resident union) + bcg_batch_get_bc per graph"},
           "plain_loop": {"TEPS_wall": plain_edges / plain_s, "TEPS_kernel": plain_edges / (plain_kernel_ms / 1e3),
                          "graphs_per_s": len(graphs) / plain_s, "wall_s": plain_s,
                          "path": "per graph: bcg_graph_create + bcg_run(all) + bcg_get_bc + destroy"},
           "speedup_vs_plain": {"kernel": (plain_kernel_ms / 1e3) / k_s, "wall": plain_s / w_s},
           "setup_s": {"create": create_s, "autotune": tune_s, "choice": list(tune)},
           "clocks": clk, "gpu_launches": 1}
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def run_serve(args, rank, world):
    """Serving form against the plain per-request loop on the front of the
    seeded request stream (ck-bc_b200/workloads.py: pool of 64 R-MAT graphs,
    Poisson arrivals, exact or k-source requests).  Exact requests on graphs
    above --exact-max-scale are left out of both arms and counted.  Plain
    loop: the pool resident as one bcg_graph per graph, each request in
    arrival order as bcg_reset_bc + bcg_run(sources) + bcg_get_bc; its Poisson
    latencies replay the measured service times through a FIFO queue.
    Served: bcg_server (HBM budget 150 GB), a client thread submitting while
    the serving thread steps; throughput with every request arriving at once,
    latency from a real-time replay of Poisson arrivals at half the served
    throughput.  One GPU (replicas only)."""
    import numpy as np
    import torch

    import bcg
    import workloads

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs = workloads.serving_pool()
    t_gen = time.perf_counter()
    pool = [bcg.generate(s) for s in specs]
    sizes = [len(o) - 1 for o, _ in pool]
    log(f"pool of {len(pool)} graphs generated in {time.perf_counter() - t_gen:.1f}s, "
        f"{sum(sizes)} vertices, {sum(len(a) for _, a in pool)} entries")
    scale = [workloads.spec_scale_ef(s)[0] for s in specs]
    stream = workloads.serving_stream(sizes)
    reqs, left_out = [], 0
    for t, g, src in stream:
        if len(reqs) >= args.requests:
            break
        if src is None and scale[g] > args.exact_max_scale:
            left_out += 1
            continue
        reqs.append((g, src))
    n_exact = sum(1 for _, s in reqs if s is None)

    # ---- plain loop
    handles = [bcg.Graph(o, a) for o, a in pool]
    with bcg.Graph(*pool[0]) as G:
        G.run(np.arange(min(64, sizes[0]), dtype=np.uint32))
    torch.cuda.synchronize()
    service = []
    plain_res = []
    t0 = time.perf_counter()
    for g, src in reqs:
        ts = time.perf_counter()
        H = handles[g]
        H.reset()
        H.run(np.arange(sizes[g], dtype=np.uint32) if src is None else src)
        plain_res.append(H.bc())
        service.append(time.perf_counter() - ts)
    plain_s = time.perf_counter() - t0
    for H in handles:
        H.close()
    plain_rps = len(reqs) / plain_s

    budget = 150 * 10**9

    def serve(arrivals):
        """Requests are submitted by a client thread at their arrival times
        while this thread keeps the server stepping (bcg_server_step never
        waits for the GPU, so arrivals are admitted while waves run)."""
        done_at = {}
        S = bcg.Server(pool, budget, args.wave_batches)
        ids = [None] * len(reqs)
        results = {}
        t_start = time.perf_counter()

        def client():
            for i, (g, src) in enumerate(reqs):
                delay = arrivals[i] - (time.perf_counter() - t_start)
                if delay > 0:
                    time.sleep(delay)
                ids[i] = S.submit(g, src)

        th = threading.Thread(target=client)
        th.start()
        while len(done_at) < len(reqs):
            got = S.step()
            for rid in got:
                done_at[rid] = time.perf_counter() - t_start
                results[rid] = S.result(rid)
            if not got:
                time.sleep(0.0002)
        th.join()
        info = S.info()
        S.close()
        lat = [done_at[ids[i]] - arrivals[i] for i in range(len(reqs))]
        span = max(done_at.values())
        return lat, span, info, [results[ids[i]] for i in range(len(reqs))]

    lat_sat, span_sat, info_sat, served_res = serve([0.0] * len(reqs))
    served_rps = len(reqs) / span_sat
    # results agree with the plain loop
    worst = 0.0
    for a, b in zip(served_res, plain_res):
        worst = max(worst, float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0))) if len(a) else 0.0)
    rate = 0.5 * served_rps
    arr = np.cumsum(np.random.Generator(np.random.PCG64(5)).exponential(1.0 / rate, size=len(reqs)))
    arr = [float(x) for x in arr]
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    lat, span, info, _ = serve(arr)
    clk = clocks.stop()
    # the plain loop at the same arrivals: FIFO replay of its service times
    free, plat = 0.0, []
    for a, sv in zip(arr, service):
        start = max(a, free)
        free = start + sv
        plat.append(free - a)

    def pct(x, q):
        return float(np.percentile(np.asarray(x), q))

    out = {"metric": "served BC requests/s (exact and k-source, seeded Poisson stream)", "value": served_rps,
           "unit": "req/s", "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * span_sat,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "impl": "bcg-served",
           "config": {"workload": "serving_pool64_stream_seed5_prefix", "requests": len(reqs), "exact": n_exact,
                      "k_source": len(reqs) - n_exact, "exact_left_out_above_scale": args.exact_max_scale,
                      "exact_left_out": left_out, "wave_batches": args.wave_batches, "hbm_budget_bytes": budget,
                      "resident_bytes": info["resident_bytes"], "pool_vertices": sum(sizes)},
           "plain_loop": {"req_per_s": plain_rps, "wall_s": plain_s,
                          "p50_s": pct(plat, 50), "p99_s": pct(plat, 99),
                          "path": "resident bcg_graph per graph; per request bcg_reset_bc + bcg_run + bcg_get_bc"},
           "speedup_vs_plain": served_rps / plain_rps,
           "latency": {"arrival_rate_per_s": rate, "p50_s": pct(lat, 50), "p99_s": pct(lat, 99),
                       "makespan_s": span, "waves": info["waves"]},
           "saturated": {"makespan_s": span_sat, "p50_s": pct(lat_sat, 50), "p99_s": pct(lat_sat, 99),
                         "waves": info_sat["waves"]},
           "max_rel_diff_vs_plain": worst, "clocks": clk, "gpu_launches": info_sat["waves"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def run_grid(args, rank, world):
    """High-diameter workload: 2048 x 2048 grid, each edge dropped with
    probability 0.05 (seed 3), largest component kept; 256 sources (seed 3),
    pendant-tree pruning (--prune degree1: one layer).  Path counts reach about 2^4000, so the run switches to
    extended-range counts (bcg_stats.extended_sigma).  value: TEPS over the
    device time of the run; cpu_baseline: the oracle's __float128 restatement
    on a bounded sample of the sources.  One GPU (replicas only)."""
    import numpy as np
    import torch

    import bcg

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    spec = "grid:w=2048,h=2048,drop=0.05,seed=3"
    offs, adj = bcg.generate(spec)
    n = len(offs) - 1
    src = bcg.sample_sources(n, 256, 3)
    pflag = bcg.PRUNE_TREES if args.prune == "trees" else bcg.PRUNE_DEGREE1
    g = bcg.Graph(offs, adj, pflag)
    g.set_sigma_mode(bcg.SIGMA_EXTENDED)  # the counts do not fit uint64; no aborted exact attempt is timed
    if args.width:
        g.set_batch_width(args.width)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(1, args.warmup)):
        g.reset()
        g.run(src)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    ms, st = [], None
    for _ in range(args.steps):
        g.reset()
        flush.zero_()
        torch.cuda.synchronize()
        st = g.run(src)
        ms.append(st.kernel_ms)
    clk = clocks.stop()
    g.close()
    kern_s = sum(ms) / len(ms) / 1e3
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with bcg.Graph(offs, adj, pflag) as ge:
        ste = ge.run(src)
        ge.bc()
    e2e_s = time.perf_counter() - t0
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        k = max(1, oracle.max_threads())
        t0 = time.perf_counter()
        _, ost = oracle.bc_q(offs, adj, src[:k], nthreads=k)
        dt = time.perf_counter() - t0
        cpu = {"value": ost["teps_edges"] / dt, "unit": "TEPS", "cores": k, "kind": "port",
               "sample": f"first {k} of the 256 sources, oracle/brandes.c __float128 Brandes, {k} threads, {dt:.1f} s"}
    alg = 16.0 * st.teps_edges + 56.0 * st.comp_vertices + 8.0 * st.roots
    peak, peak_kind = measured_peak()
    out = {"metric": "exact-BC TEPS (sources*edges/s), high-diameter grid", "value": st.teps_edges / kern_s,
           "unit": "TEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * kern_s,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "ext64", "data": "synthetic",
           "impl": "bcg-grid",
           "config": {"workload": "grid2048_drop5_256src", "graph": spec, "n": n, "m": len(adj) // 2,
                      "sources": 256, "source_seed": 3, "pruning": "pendant trees" if args.prune == "trees" else "degree-1",
                      "sigma": "extended (set explicitly)", "extended_sigma": int(st.extended_sigma),
                      "max_depth": int(st.max_depth),
                      "batch_width": int(st.batch_width),
                      "l2": "512 MiB flush write between steps (untimed)"},
           "roofline": {"bound": "hbm", "achieved": alg / kern_s / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / kern_s / 1e9 / peak, "peak_kind": peak_kind, "traffic": None},
           "e2e": {"value": ste.teps_edges / e2e_s, "unit": "TEPS", "h2d_bytes_per_step": int(4 * (n + 1 + len(adj))),
                   "d2h_bytes_per_step": int(8 * n)},
           "cpu_baseline": cpu, "clocks": clk, "gpu_launches": 1}
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bcg", choices=["bcg", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=0, help="e2e steps (default: min(steps, 3))")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sources", type=int, default=NSRC, help="sources per GPU (profiling runs use fewer)")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "serve", "grid"],
                    help="batched: the batched form on a prefix of the seeded 2000-graph set")
    ap.add_argument("--graphs", type=int, default=120, help="batched form: graphs taken from the set's front")
    ap.add_argument("--max-scale", type=int, default=16, help="batched form: keep graphs up to this scale")
    ap.add_argument("--requests", type=int, default=200, help="serving form: requests taken from the stream's front")
    ap.add_argument("--exact-max-scale", type=int, default=16,
                    help="serving form: exact requests on larger graphs are left out (hours each)")
    ap.add_argument("--wave-batches", type=int, default=64, help="serving form: batches per graph per wave")
    ap.add_argument("--width", type=int, default=0, help="sources per batch, 1, 3 or 6 (0: automatic)")
    ap.add_argument("--prune", default="trees", choices=["degree1", "trees"],
                    help="plain/grid forms: whole pendant trees (default) or one layer of degree-1 vertices "
                         "(as bc2d -H 1)")
    ap.add_argument("--graph", default=SPEC, help="plain form: generator spec (default: the workload's graph)")
    args = ap.parse_args()

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.form == "batched":
        return run_batched(args, rank, world)
    if args.form == "serve":
        return run_serve(args, rank, world)
    if args.form == "grid":
        return run_grid(args, rank, world)

    import numpy as np
    import torch

    import bcg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    t_gen = time.perf_counter()
    offs, adj = bcg.generate(args.graph)
    n = len(offs) - 1
    ns = args.sources
    srcs = rank_sources(bcg.sample_sources, n, ns, rank, world)
    log(f"[rank {rank}] graph n={n} nnz={len(adj)} generated in {time.perf_counter() - t_gen:.1f}s")

    pflag = bcg.PRUNE_TREES if args.prune == "trees" else bcg.PRUNE_DEGREE1
    g = bcg.Graph(offs, adj, pflag)
    if args.width:
        g.set_batch_width(args.width)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    bc_t = torch.as_tensor(bcg.DeviceArray(g.bc_device_ptr(), n), device="cuda")
    stream = torch.cuda.current_stream()

    def one_step():
        g.reset()
        flush.zero_()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        st = g.run(srcs)
        if dist is not None:
            combine_bc(bc_t)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1), st

    for _ in range(args.warmup):
        one_step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, kern_ms, edges, cverts, ran, s_edges, s_verts, roots = [], [], 0, 0, 0, 0, 0, 0
    launches = 0  # this library's kernels (bcg_stats.launches): the sweep, the source gather, the tree terms
    for _ in range(args.steps):
        ms, st = one_step()
        launches += st.launches
        step_ms.append(ms)
        kern_ms.append(st.kernel_ms)
        edges += st.teps_edges
        cverts += st.comp_vertices
        ran += st.sources - st.skipped
        s_edges += st.search_edges
        s_verts += st.visited
        roots += st.roots
    clk = clocks.stop()
    barrier()
    tot_ms = sum(step_ms)
    tot_edges = edges
    if dist is not None:
        t = torch.tensor([tot_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
        e = torch.tensor([tot_edges], dtype=torch.float64, device="cuda")
        dist.all_reduce(e)
        tot_edges = float(e.item())
    value = tot_edges / (tot_ms / 1e3)

    # ---- roofline of the sweep kernel (this rank)
    peak, peak_kind = measured_peak()
    alg_bytes = 16.0 * edges + 56.0 * cverts + 8.0 * ran
    kern_s = sum(kern_ms) / 1e3
    achieved = alg_bytes / kern_s / 1e9
    tps, tnote = traffic_per_source(args.prune, f"bcg::bc_sweep_kernel<{int(st.batch_width)}, "
                                                f"{'true' if st.extended_sigma else 'false'}>")
    traffic = tps * (ran / args.steps) if tps is not None else None
    # the same bytes per search over the graph the kernel actually walks (the
    # pruned graph, one search per root however many sources it stands for)
    s_bytes = 16.0 * s_edges + 56.0 * s_verts + 8.0 * roots
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": alg_bytes / args.steps, "kernel_ms_per_launch": 1e3 * kern_s / args.steps,
                "searched": {"achieved": s_bytes / kern_s / 1e9, "frac": s_bytes / kern_s / 1e9 / peak,
                             "bytes_per_launch": s_bytes / args.steps,
                             "note": "16 B per searched edge + 56 B per searched vertex + 8 B per root, over the "
                                     "pruned graph each root's search walks"}}
    if tnote:
        roofline["traffic_note"] = tnote

    # ---- e2e through the C ABI with host buffers
    e2e_steps = args.e2e_steps or min(args.steps, 3)
    h_offs = torch.from_numpy(offs).pin_memory().numpy()
    h_adj = torch.from_numpy(adj).pin_memory().numpy()
    h_bc = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    barrier()
    e2e_ms, e2e_edges = [], 0
    for _ in range(e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ge = bcg.Graph(h_offs, h_adj, pflag)
        if args.width:
            ge.set_batch_width(args.width)
        t1 = time.perf_counter()
        st = ge.run(srcs)
        if dist is not None:
            bt = torch.as_tensor(bcg.DeviceArray(ge.bc_device_ptr(), n), device="cuda")
            combine_bc(bt)
        t2 = time.perf_counter()
        bcg.lib().bcg_get_bc(ge.h, h_bc.ctypes.data_as(bcg._f64p))
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        e2e_ms.append(1e3 * (t3 - t0))
        ge.close()  # releasing the graph is not part of the user's step
        t4 = time.perf_counter()
        log(f"[rank {rank}] e2e step: create {t1 - t0:.3f} s, run {t2 - t1:.3f} s (kernel {st.kernel_ms / 1e3:.3f} s), "
            f"read {t3 - t2:.3f} s; destroy (untimed) {t4 - t3:.3f} s")
        e2e_edges += st.teps_edges
    e2e_tot = sum(e2e_ms)
    if dist is not None:
        t = torch.tensor([e2e_tot, float(e2e_edges)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t[1:2])
        tm = t[0:1].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        e2e_tot, e2e_edges = float(tm.item()), float(t[1].item())
    e2e = {"value": e2e_edges / (e2e_tot / 1e3), "unit": "TEPS",
           "h2d_bytes_per_step": int(4 * (n + 1) + 4 * len(adj) + 4 * len(srcs)),
           "d2h_bytes_per_step": int(8 * n), "steps": e2e_steps,
           "path": "bcg_graph_create(host CSR) + bcg_run(host sources) + bcg_get_bc(host)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(offs, adj, srcs)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "TEPS", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": WORKLOAD, "graph": args.graph, "n": n, "m": len(adj) // 2,
                          "sources_per_gpu": ns, "source_seed": SRC_SEED,
                          "pruning": "pendant trees" if args.prune == "trees" else "degree-1",
                          "sources_skipped_per_step": int(st.skipped), "batch_width": int(st.batch_width),
                          "parallelism": f"source-sharded x{world}, bc summed in rank order" if world > 1
                          else "1 GPU",
                          "l2": "512 MiB flush write between steps (untimed); graph + state exceed L2"},
               "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clk,
               "gpu_launches": int(launches)}
        print(json.dumps(out), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
