#!/usr/bin/env python
"""Benchmark of the B200 race-free graph suite (the driver's contract).

Default workload (one "step"): the full plain suite on R-MAT scale 22
(2^22 vertices, edge factor 16, a=.57 b=.19 c=.19, seed 2): CC, MIS, GC and
MST (int32 weights uniform in [1, 2^20), seed 3, symmetric per pair) on the
symmetrised, duplicate- and self-loop-free graph, and SCC on the directed
graph of the same parameters.  Metric: edges/s = sum of each solve's
g.edges / sum of solve times, as the reference computes edges/s
(ECL-CC-atomic.cu:314-316): inputs resident on the device, kernel time only.
L2 (126 MB) is flushed by a 256 MiB write before every solve.  The line also
carries the end-to-end rate through the C ABI (host CSR in, results out),
the dominant kernel's roofline, GC's latency roofline (critical path x the
measured hop cost), a CPU baseline on the same graphs and, on one GPU, the
other four configs measured after the headline (`other_configs`: the grid
CC, APSP n=8192, the batched 4096-graph mix, the served Poisson stream),
each with its own clocks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload suite|grid|apsp|batch|serve] [--scale S]
                  [--no-other-configs] [--no-cpu-baseline]

--impl reference times the reference's own CPU routines (cpuMST; the C
restatement where the reference has no CPU solver) on the same graphs, built
by the restated generators under oracle/ without loading the product, plus
the reference's race-free CUDA build on them (`reference_gpu`).

Multi-GPU: replicas only -- every rank solves its own copy of the workload, no
collective on the data path; value = edges of all ranks / max time over ranks.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ecl-suite_b200"))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}
CODES_SYM = ["cc", "mis", "gc", "mst"]


# ---------------------------------------------------------------- ranks
# One process per GPU (torchrun); every rank runs the same steps and the same
# collectives in the same order.  A rate is the units ALL ranks processed
# divided by the slowest rank's device time.


def rank_barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    """Largest x over all ranks (the identity on one rank)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_per_rank, world, max_seconds):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units, timed by the slowest rank."""
    return world * units_per_rank / max_seconds


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["suite", "grid", "apsp", "batch", "serve"], default="suite")
    p.add_argument("--serve-graphs", type=int, default=16)
    p.add_argument("--batch-count", type=int, default=4096)
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false",
                   help="skip the CPU baseline leg of our arm")
    p.add_argument("--no-other-configs", dest="other_configs", action="store_false",
                   help="suite only: skip the grid, APSP, batched and served configs measured after it")
    return p.parse_args(argv)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        d["source"] = "measured"
        return d
    except Exception:
        return dict(PEAKS_FALLBACK)


# ---------------------------------------------------------------- clocks


class Clocks:
    """SM clock and clock-event reasons sampled DURING the timed region.

    An NVML thread samples every 10 ms (the suite's timed region is ~70 ms, too
    short for nvidia-smi's start-up and 200 ms period), with one sample at
    start(); the device is matched to the CUDA device by UUID.  Falls back to
    nvidia-smi sampling when NVML is unavailable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.stop_evt = None
        self.thread = None
        self.p = None
        self.nv = None
        try:
            import pynvml as nv
            import torch

            nv.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            handle = None
            for i in range(nv.nvmlDeviceGetCount()):
                h = nv.nvmlDeviceGetHandleByIndex(i)
                u = nv.nvmlDeviceGetUUID(h)
                u = u.decode() if isinstance(u, bytes) else u
                if u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                    handle = h
            if handle is None:
                handle = nv.nvmlDeviceGetHandleByIndex(index)
            self.nv, self.h = nv, handle
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(handle, nv.NVML_CLOCK_SM))
            self.bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                         nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        except Exception:
            self.nv = None

    def _sample(self):
        nv, h = self.nv, self.h
        mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((mhz, [n for n, b in zip(self.NAMES, self.bits) if r & b]))

    def _run(self):
        while not self.stop_evt.wait(0.01):
            try:
                self._sample()
            except Exception:
                return

    def start(self):
        if self.nv is not None:
            import threading

            self._sample()
            self.stop_evt = threading.Event()
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
            return
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.nv is not None:
            self.stop_evt.set()
            self.thread.join(timeout=5)
            sm = sorted(m for m, _ in self.samples)
            reasons = sorted({n for _, rs in self.samples for n in rs})
            return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "nvml, 10 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------- workloads


def make_suite_graphs(gen, scale):
    """The suite's graphs from `gen`: the product library in our arm, the
    oracle's restated generators (same bytes) in the reference arm."""
    sym = gen.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=2, symmetrise=True, weight_seed=3, weight_max=1 << 20)
    dirg = gen.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=2, symmetrise=False)
    return sym, dirg


# Algorithmic (compulsory) bytes of each kernel phase, per launch: the bytes
# the phase must move at minimum (CSR read once, per-vertex state read or
# written once).  n = vertices, m = CSR entries.
def phase_bytes(code, phase, n, m):
    csr = 4 * (n + 1) + 4 * m
    table = {
        ("cc", 0): 4 * (n + 1) + 4 * n,            # init: nindex + first entries, parent write
        ("cc", 1): csr + 4 * n,                    # hook: CSR + parent
        ("cc", 2): 4 * m // 8,                     # chunks: hub entries (upper bound share)
        ("cc", 3): 8 * n,                          # flatten: parent read + write
        # symmetric path: 2 sampled entries per vertex, compressions, giant-membership bytes
        ("cc_sym", 0): 4 * (n + 1) + 8 * n + 4 * n + 16 * n + n,
        ("cc_sym", 1): 4 * (n + 1) + n,            # rest: rows + membership (giant rows skipped)
        ("cc_sym", 2): 4 * m // 8,
        ("cc_sym", 3): 8 * n,
        ("mis", 0): 4 * (n + 1) + n,
        ("mis", 1): csr + n,
        ("mis", 2): 2 * n,
        # keys + init: rows read for the keys (4n), keys + ids written (12n), CSR read once, the
        # higher-priority half of nl2 and the counts written
        ("gc", 0): csr + 16 * n + 4 * (m // 2) + 4 * n,
        # radix passes over (8 B key, 4 B value), read + write; 32 hash bits + the bits of m
        ("gc", 1): -(-(32 + max(1, m.bit_length())) // 8) * 24 * n,
        ("gc", 2): None,                           # core: latency-bound, no byte model (its entries are booked to pull)
        ("gc", 3): 4 * (n + 1) + 4 * (m // 2) + 12 * n,  # pull: higher-priority half read once, order, colours
        ("mst", 0): 16 * n,
        ("mst", 1): 4 * (n + 1) + 8 * m,           # light scan: CSR + weights
        ("mst", 2): 16 * n,
        ("mst", 3): 4 * (n + 1) + 8 * m + 4 * n,   # heavy scan: CSR + weights + roots
        ("mst", 4): 16 * n,
        ("scc", 0): csr + 4 * n + 8 * m,           # mark: CSR read, flags, the 8-byte edge list written
        ("scc", 1): 8 * m + 12 * n,                # solve: one sweep of the edge list, io words and labels
    }
    return table[(code, phase)] if (code, phase) in table else csr


PHASE_NAMES = {
    "cc": ["cc_init", "cc_hook", "cc_chunks", "cc_flatten"],
    "cc_sym": ["cc_init+sample+giant", "cc_rest", "cc_rest_chunks", "cc_flatten"],
    "mis": ["mis_init", "mis_run", "mis_emit"],
    "gc": ["gc_keys+init+chunks", "radix_sort", "gc_core", "gc_pull"],
    "mst": ["mst_init+threshold", "mst_scan<light>+chunks", "mst_boruvka(light)", "mst_scan<heavy>+chunks",
            "mst_boruvka(heavy)"],
    "scc": ["scc_mark+chunks", "scc_solve"],
    "apsp": ["apsp_fill+edges", "apsp_panels+update"],
}


def phase_code(code, g):
    """Phase table of a solve: symmetric graphs take CC's sampling path."""
    return "cc_sym" if code == "cc" and getattr(g, "symmetric", False) else code


# ---------------------------------------------------------------- our arm


def bench_batch(args, rank, world, local_rank):
    """Batched config: 4096 graphs (n log-uniform in [1k, 200k], seed 5;
    ER d=8 / grid / R-MAT ef=8; weights in [1, 2^16)), CC+MIS+MST per graph.
    value = graphs/s of the batched engine (one CUDA-graph replay per step);
    plain_graphs_per_s = the same solves one graph per call (ecl_cc, ecl_mis,
    ecl_mst on device-resident graphs, preallocated workspace)."""
    import numpy as np
    import torch

    import ecl_b200 as ecl

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    b = ecl.Batch()
    b.add_mix(args.batch_count, n_min=1000, n_max=200000, seed=5, weight_max=1 << 16)
    gen_s = time.perf_counter() - t0
    codes = ecl.BATCH_CC | ecl.BATCH_MIS | ecl.BATCH_MST
    t0 = time.perf_counter()
    b.build(codes, stream=stream.cuda_stream)
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tuned = b.tune(trials=1)
    tune_s = time.perf_counter() - t0
    G = b.graphs
    sizes = [b.graph(i) for i in range(G)]
    tot_n = sum(g.nodes for g in sizes)
    tot_m = sum(g.edges for g in sizes)
    for _ in range(args.warmup):
        b.run()
    rank_barrier(world)
    clk = Clocks(local_rank)
    clk.start()
    l0 = ecl.kernel_launches()
    ms = 0.0
    replay = True
    for _ in range(args.steps):
        t, r = b.run()
        ms += t
        replay = replay and r
    launches = ecl.kernel_launches() - l0
    rank_barrier(world)
    clocks = clk.stop()
    ms = max_over_ranks(ms, world)
    value = job_rate(G * args.steps, world, ms / 1e3)

    # one graph per call, same solves, device-resident inputs
    dgs = [g.to_device(dev) for g in sizes]
    for dg in dgs:
        dg.symmetric = True
    wsb = max(ecl.workspace_bytes(c, g.nodes, g.edges) for g in sizes for c in (ecl.CC, ecl.MIS, ecl.MST))
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    maxn = max(g.nodes for g in sizes)
    maxm = max(g.edges for g in sizes)
    o_cc = torch.empty(maxn, dtype=torch.int32, device=dev)
    o_mis = torch.empty(maxn, dtype=torch.uint8, device=dev)
    o_mst = torch.empty(maxm, dtype=torch.uint8, device=dev)
    sh = stream.cuda_stream

    def plain(dg):
        ecl.cc(dg, out=o_cc, opts=ecl._opts(stream=sh, workspace=ws))
        ecl.mis(dg, out=o_mis, opts=ecl._opts(stream=sh, workspace=ws))
        ecl.mst(dg, out=o_mst, opts=ecl._opts(stream=sh, workspace=ws))

    for dg in dgs[:16]:
        plain(dg)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for dg in dgs:
        plain(dg)
    ev1.record(stream)
    ev1.synchronize()
    plain_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    plain_gps = job_rate(G, world, plain_ms / 1e3)
    line = {
        "metric": "graphs/s (batched CC+MIS+MST over the 4096-graph mix; one CUDA-graph replay per step)",
        "value": value, "unit": "graphs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded mix generator, seed 5)",
        "config": {"workload": f"batch{G}: ER(d=8)/grid/R-MAT(ef=8), n log-uniform [1k,200k], weights [1,2^16)",
                   "graphs": G, "vertices": tot_n, "csr_entries": tot_m, "superbatches": b.superbatches,
                   "codes": "CC+MIS+MST", "parallelism": f"replicas x{world}"},
        "plain_graphs_per_s": plain_gps, "plain_ms": plain_ms, "speedup_vs_plain": value / plain_gps,
        "edges_per_s": 3 * tot_m * args.steps / (ms / 1e3),
        "cuda_graph_replay": replay, "tuned": tuned.as_dict(), "tune_points": b.tune_points,
        "setup_s": {"generate": round(gen_s, 2), "build_upload": round(build_s, 2), "tune": round(tune_s, 2)},
        "gpu_launches": int(launches), "clocks": clocks,
    }
    del dgs, ws, o_cc, o_mis, o_mst
    b.close()
    return line


def bench_serve(args, rank, world, local_rank):
    """Served config: Poisson arrivals (seed 6) of CC/MIS/GC/MST/SCC requests
    on a pool of resident seeded graphs (R-MAT or grid, n log-uniform in
    [10k, 8M], edge factor 8-16, weights uniform in [1, 2^20)), admitted
    against a 160 GB HBM budget; rates swept 10 - 10k req/s.  value =
    graphs/s at the highest rate; p50/p99 latency per rate."""
    import math

    import numpy as np
    import torch

    import ecl_b200 as ecl

    torch.cuda.set_device(local_rank)
    rng = np.random.default_rng(6)
    srv = ecl.Server(slots=8, hbm_budget_bytes=160 * 10**9)
    t0 = time.perf_counter()
    pool = []
    for k in range(args.serve_graphs):
        n = int(math.exp(rng.uniform(math.log(1e4), math.log(8e6))))
        ef = int(rng.integers(8, 17))
        if rng.random() < 0.5:
            g = ecl.gen_rmat(max(1, round(math.log2(n))), ef, seed=600 + k, weight_seed=700 + k, weight_max=1 << 20)
            kind = "rmat"
        else:
            r = max(1, int(math.sqrt(n)))
            g = ecl.gen_grid(r, max(1, n // r), 0.0, seed=600 + k, weight_seed=700 + k, weight_max=1 << 20)
            kind = "grid"
        g.symmetric = True
        pool.append((srv.add_graph(g), g.nodes, g.edges, kind))
        print(f"serve: graph {k} {kind} n={g.nodes} m={g.edges}", file=sys.stderr, flush=True)
    setup_s = time.perf_counter() - t0
    codes = [ecl.CC, ecl.MIS, ecl.GC, ecl.MST, ecl.SCC]
    names = {ecl.CC: "cc", ecl.MIS: "mis", ecl.GC: "gc", ecl.MST: "mst", ecl.SCC: "scc"}
    sweep = []
    l0 = ecl.kernel_launches()
    # warm-up: a burst of every code on every resident graph at t = 0, so the
    # slots run concurrently and the stream-ordered memory pool grows to its
    # concurrent working size before any timed request (growing it later
    # costs a stall that every in-flight request sees)
    srv.run([(c, p[0], 0.0, None) for c in codes for p in pool])
    srv.run([(c, p[0], 0.0, None) for p in sorted(pool, key=lambda p: -p[2])[:8] for c in codes])
    clk = Clocks(local_rank)
    clk.start()
    for rate in (10, 100, 1000, 10000):
        count = int(min(400, max(40, rate * 3)))
        t = 0.0
        reqs = []
        for _ in range(count):
            t += rng.exponential(1.0 / rate)
            c = codes[int(rng.integers(0, 5))]
            gid = pool[int(rng.integers(0, len(pool)))][0]
            reqs.append((c, gid, t, None))
        print(f"serve: rate {rate} req/s, {count} requests", file=sys.stderr, flush=True)
        rank_barrier(world)
        rc, arr, st = srv.run(reqs)
        print(f"serve: rate {rate} done rc={rc} p50={st.p50_s*1e3:.2f} ms p99={st.p99_s*1e3:.2f} ms "
              f"{st.graphs_per_s:.1f} graphs/s", file=sys.stderr, flush=True)
        per = {}
        for c in codes:
            lat = sorted(arr[k].latency_s for k in range(count) if arr[k].code == c and arr[k].status == 0)
            if lat:
                per[names[c]] = {"p50_ms": 1e3 * lat[len(lat) // 2], "p99_ms": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                                 "n": len(lat)}
        # every rank serves its own stream: completions add up over the
        # slowest rank's makespan; latency quantiles are the worst rank's
        done = sum_over_ranks(st.completed, world)
        makespan = max_over_ranks(st.makespan_s, world)
        sweep.append({"rate_req_s": rate * world, "requests": count * world, "completed": int(done),
                      "failed": int(sum_over_ranks(st.failed, world)),
                      "graphs_per_s": done / makespan if makespan > 0 else 0.0,
                      "p50_ms": 1e3 * max_over_ranks(st.p50_s, world), "p99_ms": 1e3 * max_over_ranks(st.p99_s, world),
                      "mean_ms": 1e3 * st.mean_s, "max_in_flight": st.max_in_flight,
                      "peak_gb": st.peak_bytes / 1e9, "per_code": per, "rc": rc})
    clocks = clk.stop()
    top = sweep[-1]
    line = {
        "metric": "graphs/s and p50/p99 latency of a served Poisson request stream (CC/MIS/GC/MST/SCC)",
        "value": top["graphs_per_s"], "unit": "graphs/s", "n_gpus": world, "steps": len(sweep), "warmup": 1,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT / grid pool, seed 6)",
        "config": {"workload": f"serve: {len(pool)} resident graphs, n log-uniform [10k, 8M], ef 8-16, "
                               f"budget 160 GB, 8 slots", "graphs": [{"n": p[1], "m": p[2], "kind": p[3]} for p in pool],
                   "resident_gb": sum(4 * (p[1] + 1) + 8 * p[2] for p in pool) / 1e9, "parallelism": f"replicas x{world}"},
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"], "sweep": sweep, "setup_s": round(setup_s, 2),
        "gpu_launches": int(ecl.kernel_launches() - l0), "clocks": clocks,
    }
    srv.close()
    return line


def bench_plain(args, rank, world, local_rank):
    import numpy as np
    import torch

    import ecl_b200 as ecl

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    if args.workload == "suite":
        sym, dirg = make_suite_graphs(ecl, args.scale)
        jobs = [(c, sym) for c in CODES_SYM] + [("scc", dirg)]
        wl_name = suite_name(args.scale, sym, dirg)
    elif args.workload == "grid":
        g = grid_graph(ecl)
        jobs = [("cc", g)]
        wl_name = grid_name(g)
    else:
        g = apsp_graph(ecl)
        jobs = [("apsp", g)]
        wl_name = apsp_name(g)

    dgs = {}
    for code, g in jobs:
        if id(g) not in dgs:
            dgs[id(g)] = g.to_device(dev)
    wsb = max(ecl.workspace_bytes(getattr(ecl, code.upper()), g.nodes, g.edges) for code, g in jobs)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    outs = {}
    for code, g in jobs:
        if code == "mst":
            outs[code] = torch.empty(max(g.edges, 1), dtype=torch.uint8, device=dev)
        elif code == "mis":
            outs[code] = torch.empty(g.nodes, dtype=torch.uint8, device=dev)
        elif code == "apsp":
            outs[code] = torch.empty((g.nodes, g.nodes), dtype=torch.int32, device=dev)
        else:
            outs[code] = torch.empty(g.nodes, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def solve(code, g, detail):
        o = ecl._opts(stream=sh, workspace=ws, detail=detail)
        dg = dgs[id(g)]
        fn = getattr(ecl, code)
        if code == "apsp":
            fn(dg, out=outs[code], opts=o)
        else:
            fn(dg, out=outs[code], opts=o)
        return o

    per_code_ms = {c: 0.0 for c, _ in jobs}
    per_code_rounds = {}
    phase_tot = {}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def step(timed):
        tot = 0.0
        for code, g in jobs:
            flush.fill_(1)
            ev0.record(stream)
            o = solve(code, g, detail=timed)
            ev1.record(stream)
            ev1.synchronize()
            ms = ev0.elapsed_time(ev1)
            if timed:
                per_code_ms[code] += ms
                per_code_rounds[code] = int(o.rounds)
                for i in range(o.nphases):
                    key = (phase_code(code, g), i)
                    phase_tot[key] = phase_tot.get(key, 0.0) + o.phase_ms[i]
            tot += ms
        return tot

    for _ in range(args.warmup):
        step(False)
    rank_barrier(world)
    torch.cuda.synchronize()
    clk = Clocks(local_rank)
    clk.start()
    l0 = ecl.kernel_launches()
    total_ms = 0.0
    for _ in range(args.steps):
        total_ms += step(True)
    launches = ecl.kernel_launches() - l0
    torch.cuda.synchronize()
    rank_barrier(world)
    clocks = clk.stop()

    is_apsp = jobs[0][0] == "apsp"
    # units of one step: CSR entries (edges/s, as the reference prints), or
    # n^3 relaxations for APSP (updates/s)
    units_step = float(jobs[0][1].nodes) ** 3 if is_apsp else sum(g.edges for _, g in jobs)
    unit = "updates/s" if is_apsp else "edges/s"
    total_ms = max_over_ranks(total_ms, world)
    value = job_rate(units_step * args.steps, world, total_ms / 1e3)
    ms_per_step = total_ms / args.steps

    # dominant kernel phase and its roofline
    # the dominant phase among those with a byte model
    modelled = {k: v for k, v in phase_tot.items() if k[0] == "apsp" or phase_bytes(k[0], k[1], 1, 1) is not None}
    dom = max(modelled.items(), key=lambda kv: kv[1]) if modelled else None
    pk = peaks()
    roof = None
    if dom is not None and jobs[0][0] != "apsp":
        (code, idx), tot = dom
        g = {phase_code(c, gg): gg for c, gg in jobs}[code]
        avg_ms = tot / args.steps
        byts = phase_bytes(code, idx, g.nodes, g.edges)
        ach = byts / (avg_ms / 1e3) / 1e9
        traffic = None
        try:
            with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
                traffic = json.load(f).get(PHASE_NAMES[code][idx])
        except Exception:
            pass
        roof = {"bound": "hbm", "kernel": PHASE_NAMES[code][idx], "achieved": round(ach, 1),
                "peak": pk.get("hbm_gbs"), "unit": "GB/s", "frac": round(ach / pk.get("hbm_gbs", 1), 4),
                "traffic": traffic, "algorithmic_bytes": byts, "avg_ms": round(avg_ms, 4),
                "share": round(tot / sum(phase_tot.values()), 3), "peak_source": pk.get("source")}
    elif dom is not None:
        n = jobs[0][1].nodes
        N = (n + 127) // 128 * 128
        avg_ms = per_code_ms["apsp"] / args.steps
        ops = 2.0 * float(N) ** 3  # one add + one min per update of the padded N x N closure
        peak_dpx = ecl.minplus_peak(0) / 1e12
        peak_sep = ecl.minplus_peak(1) / 1e12
        ach = ops / (avg_ms / 1e3) / 1e12
        roof = {"bound": "int32", "kernel": "apsp_panels+apsp_update", "achieved": round(ach, 3),
                "peak": round(peak_dpx, 3), "unit": "Tops/s", "frac": round(ach / peak_dpx, 4), "traffic": None,
                "avg_ms": round(avg_ms, 3), "peak_source": "measured in this run: ecl_minplus_peak(0), DPX add-min "
                "throughput over a full wave (MEASURED_PEAKS.json has no integer peak)",
                "peak_add_then_min": round(peak_sep, 3),
                "note": "2 integer ops (add + min) per update of the padded N^3 closure, N = ceil(n/128)*128"}

    # GC's colouring is bound by its dependency chain, not by bytes: the
    # latency roofline is the longest chain of the input (hops inside the
    # shared-memory core and after it) times the measured cost of one hop
    # there, against the measured gc_core + gc_pull time
    gc_latency = None
    if args.workload == "suite" and ("gc", 3) in phase_tot:
        hop = {"l2_backoff": ecl.hop_latency(0), "l2_spin": ecl.hop_latency(1), "smem": ecl.hop_latency(2)}
        tune = ecl.get_tune()
        hops, hops_core, path_ns = ecl.gc_critical_path(sym, tune.gc_core_ranks, hop["smem"], hop["l2_backoff"])
        got_ms = (phase_tot[("gc", 2)] + phase_tot[("gc", 3)]) / args.steps
        gc_latency = {"kernels": "gc_core+gc_pull", "hops": hops, "hops_in_core": hops_core,
                      "hop_ns": {k: round(v, 1) for k, v in hop.items()}, "bound_ms": round(path_ns / 1e6, 4),
                      "achieved_ms": round(got_ms, 4), "frac": round(path_ns / 1e6 / got_ms, 4),
                      "model": "longest chain of higher-priority dependencies; a hop into the core costs the "
                               "shared-memory hop, any other the L2 hop with the pull's back-off polling"}
        if roof is not None and roof.get("kernel") == "gc_pull":
            roof["latency"] = gc_latency

    # The CSR scans stream the column indices once and load one L2-resident
    # per-vertex word per entry; their bound is the measured rate of exactly
    # that on the graph's own indices (ecl_gather_peak), not HBM bandwidth.
    scan_roof = None
    if args.workload == "suite":
        scans = [(("gc", 0), "read-only"), (("mst", 1), "read-only"), (("mst", 3), "atomic"),
                 (("scc", 0), "atomic")]
        graph_of = {phase_code(c, gg): gg for c, gg in jobs}
        peak_cache = {}
        scan_roof = {}
        for (code, idx), kind in scans:
            if (code, idx) not in phase_tot:
                continue
            g = graph_of[code]
            key = (id(g), kind)
            if key not in peak_cache:
                peak_cache[key] = ecl.gather_peak(dgs[id(g)].nlist, g.nodes, 0 if kind == "read-only" else 1)
            avg_ms = phase_tot[(code, idx)] / args.steps
            ach = g.edges / (avg_ms / 1e3)
            scan_roof[PHASE_NAMES[code][idx]] = {
                "entries": g.edges, "avg_ms": round(avg_ms, 4), "achieved_g_entries_s": round(ach / 1e9, 2),
                "peak_g_entries_s": round(peak_cache[key] / 1e9, 2), "frac": round(ach / peak_cache[key], 3),
                "loads": kind}

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        hosts = {}

        def pinned(a):
            t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
            return t.numpy(), t

        keep = []
        for code, g in jobs:
            if id(g) in hosts:
                continue
            ni, t1 = pinned(g.nindex)
            nl, t2 = pinned(g.nlist)
            ew = None
            if g.eweight is not None:
                ew, t3 = pinned(g.eweight)
                keep.append(t3)
            keep += [t1, t2]
            hosts[id(g)] = ecl.Graph(ni, nl, ew, g.symmetric)
        houts = {}
        for code, g in jobs:
            if code == "apsp":
                t = torch.empty((g.nodes, g.nodes), dtype=torch.int32).pin_memory()
            elif code in ("mst",):
                t = torch.empty(max(g.edges, 1), dtype=torch.uint8).pin_memory()
            elif code == "mis":
                t = torch.empty(g.nodes, dtype=torch.uint8).pin_memory()
            else:
                t = torch.empty(g.nodes, dtype=torch.int32).pin_memory()
            keep.append(t)
            houts[code] = t.numpy()
        h2d = d2h = 0
        for code, g in jobs:
            h2d += 4 * (g.nodes + 1) + 4 * g.edges + (4 * g.edges if code in ("mst", "apsp") else 0)
            d2h += houts[code].nbytes if code != "mst" else g.edges
        e_ms = 0.0
        for it in range(args.e2e_steps + 1):
            torch.cuda.synchronize()
            ev0.record(stream)
            for code, g in jobs:
                o = ecl._opts(stream=sh)
                fn = getattr(ecl, code)
                fn(hosts[id(g)], out=houts[code], opts=o)
            ev1.record(stream)
            ev1.synchronize()
            if it > 0:  # first call warms the stream-ordered allocator
                e_ms += ev0.elapsed_time(ev1)
        e_ms = max_over_ranks(e_ms, world)
        e2e = {"value": job_rate(units_step * args.e2e_steps, world, e_ms / 1e3), "unit": unit,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
               "ms_per_step": e_ms / args.e2e_steps}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        if args.workload == "suite":
            cpu = cpu_baseline(sym, dirg)
        elif args.workload == "grid":
            cpu = cpu_baseline_grid(g)
        else:
            cpu = cpu_baseline_apsp()

    per_code = {c: {"edges": g.edges, "ms": per_code_ms[c] / args.steps,
                    "edges_per_s": g.edges / (per_code_ms[c] / args.steps / 1e3),
                    "rounds": per_code_rounds.get(c)} for c, g in jobs}
    phases = {f"{PHASE_NAMES[c][i]}": round(v / args.steps, 4) for (c, i), v in sorted(phase_tot.items())}
    metric = ("updates/s (n^3 / compute time of the blocked Floyd-Warshall closure; inputs resident)" if is_apsp else
              "edges/s (sum of g.edges over the suite's solves / sum of solve times; kernel time, inputs resident)")
    line = {
        "metric": metric,
        "value": value, "unit": unit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded generators: R-MAT / grid / Erdos-Renyi)",
        "config": {"workload": wl_name, "l2": L2_NOTE}, "parallelism": f"replicas x{world}",
        "per_code": per_code, "phase_ms": phases, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clocks,
    }
    if gc_latency is not None:
        line["gc_latency_roofline"] = gc_latency
    if scan_roof:
        line["scan_gather_roofline"] = scan_roof
    del dgs, ws, outs, flush
    return line


def other_configs(args, local_rank):
    """The other four configs, measured after the headline suite on the same
    GPU (1 GPU only): the 1024x1024 grid CC, APSP on ER n=8192, the batched
    4096-graph mix and the served Poisson stream.  Each has its own clocks;
    none is inside the headline's timed region."""
    import torch

    out = {}
    plan = [("grid", dict(workload="grid", steps=args.steps, warmup=args.warmup, e2e_steps=args.e2e_steps)),
            ("apsp", dict(workload="apsp", steps=min(args.steps, 5), warmup=min(args.warmup, 3),
                          e2e_steps=min(args.e2e_steps, 1))),
            ("batch", dict(workload="batch", steps=min(args.steps, 5), warmup=min(args.warmup, 3))),
            ("serve", dict(workload="serve"))]
    for name, over in plan:
        sub = argparse.Namespace(**vars(args))
        for k, v in over.items():
            setattr(sub, k, v)
        t0 = time.perf_counter()
        try:
            if name == "batch":
                r = bench_batch(sub, 0, 1, local_rank)
            elif name == "serve":
                r = bench_serve(sub, 0, 1, local_rank)
            else:
                r = bench_plain(sub, 0, 1, local_rank)
        except Exception as ex:  # reported in the line; the headline stands on its own
            r = {"error": f"{type(ex).__name__}: {ex}"}
        r["wall_s"] = round(time.perf_counter() - t0, 1)
        out[name] = r
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        print(f"bench: {name} done in {r['wall_s']} s", file=sys.stderr, flush=True)
    return out


# ---------------------------------------------------------------- CPU baseline / reference arm
#
# Both use the checker code under oracle/ only: the reference's own CPU
# routines and CUDA build compiled from its sources (oracle/_ref), the C
# restatement (oracle/_build) for the codes the reference has no CPU solver
# for, and the restated generators, so the reference arm never loads the
# product library.


def _orc():
    p = os.path.join(ROOT, "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)
    import oracle

    return oracle


def _ref():
    p = os.path.join(ROOT, "oracle", "_ref", "libeclref.so")
    if not os.path.exists(p):
        return None
    r = C.CDLL(p)
    r.eclref_mst_cpu.restype = C.c_double
    r.eclref_mst_gpu.restype = C.c_double
    r.eclref_apsp_gpu.restype = C.c_double
    r.eclref_apsp_cpu.restype = C.c_double
    r.eclref_cc_device.restype = C.c_float
    r.eclref_mis_device.restype = C.c_float
    r.eclref_gc_device.restype = C.c_float
    r.eclref_gc_scratch_bytes.restype = C.c_size_t
    r.eclref_scc_device.restype = C.c_float
    r.eclref_scc_scratch_bytes.restype = C.c_size_t
    return r


# CPU leg per code.  CC, MIS, GC and SCC have no CPU solver in the reference:
# each is run both as the serial C oracle and as its OpenMP rendering
# (oracle/omp_baseline.c, all host threads) once, and the faster of the two on
# this machine is the baseline.  MST is the reference's own serial cpuMST
# (ECL-MST_10-atomic.cu:112) when oracle/_ref is built.
_CPU_PICK = {}
SUITE_LEGS = ("cc", "mis", "gc", "mst", "scc")


def cpu_leg(orc, code, g):
    """Runs the chosen CPU leg of `code` on g; returns (seconds, kind, cores)."""
    key = (code, g.nodes, g.edges)
    if key not in _CPU_PICK:
        times = {}
        for name in (code, "omp_" + code):
            t0 = time.perf_counter()
            getattr(orc, name)(g)
            times[name] = time.perf_counter() - t0
        _CPU_PICK[key] = min(times, key=times.get)
    name = _CPU_PICK[key]
    t0 = time.perf_counter()
    getattr(orc, name)(g)
    dt = time.perf_counter() - t0
    if name.startswith("omp_"):
        return dt, "port (OpenMP)", orc.omp_threads()
    return dt, "port (serial)", 1


def suite_leg(orc, ref, code, sym, dirg):
    """One code of the CPU suite: returns (edges, seconds, kind, cores)."""
    import numpy as np

    if code == "scc":
        dt, kind, cores = cpu_leg(orc, "scc", dirg)
        return dirg.edges, dt, kind, cores
    if code != "mst":
        dt, kind, cores = cpu_leg(orc, code, sym)
        return sym.edges, dt, kind, cores
    out = np.zeros(max(sym.edges, 1), np.uint8)
    t0 = time.perf_counter()
    if ref is not None:
        P = lambda a: C.c_void_p(a.ctypes.data)
        ref.eclref_mst_cpu(sym.nodes, sym.edges, P(sym.nindex), P(sym.nlist), P(sym.eweight), P(out))
        kind = "reference"
    else:
        orc.mst(sym)
        kind = "port (serial)"
    return sym.edges, time.perf_counter() - t0, kind, 1


def overall_kind(kinds):
    """'reference' or 'port' when every code agrees, else 'mixed' (the
    per-code kinds are reported beside it)."""
    ks = {("reference" if k == "reference" else "port") for k in kinds.values()}
    return ks.pop() if len(ks) == 1 else "mixed"


def suite_rate(times, edges):
    """Suite edges/s from per-code mean times: sum of one pass's edges over the
    sum of the codes' mean solve times."""
    codes = [c for c in SUITE_LEGS if times.get(c)]
    t = sum(sum(times[c]) / len(times[c]) for c in codes)
    return sum(edges[c] for c in codes) / t


def cpu_baseline(sym, dirg):
    """One pass of the CPU suite on the bench's own R-MAT graphs."""
    orc, ref = _orc(), _ref()
    kinds, cores, times, edges = {}, {}, {}, {}
    for code in SUITE_LEGS:
        edges[code], dt, kinds[code], cores[code] = suite_leg(orc, ref, code, sym, dirg)
        times[code] = [dt]
    tot = sum(t[0] for t in times.values())
    return {"value": suite_rate(times, edges), "unit": "edges/s", "cores": max(cores.values()),
            "kind": overall_kind(kinds),
            "sample": f"one pass of the suite on the same graphs: MST by the reference's own serial cpuMST, "
                      f"CC/MIS/GC/SCC (no CPU solver in the reference) by the faster of the serial C oracle and "
                      f"its OpenMP rendering ({orc.omp_threads()} threads) on this host; {tot:.1f} s",
            "per_code_kind": kinds, "per_code_cores": cores,
            "per_code_s": {c: round(times[c][0], 3) for c in SUITE_LEGS}}


def grid_graph(gen):
    return gen.gen_grid(1024, 1024, 0.05, seed=1)


def apsp_graph(gen, n=8192):
    # ER with the same expected degree as n=8192, p=0.001 (about 8.2)
    return gen.gen_er(n, 0.001 * 8192 / n, seed=4, weight_seed=5, weight_min=1, weight_max=1000)


def suite_name(scale, sym, dirg):
    return (f"rmat{scale}-suite: CC+MIS+GC+MST on symmetrised R-MAT-{scale} "
            f"(n={sym.nodes}, m={sym.edges}), SCC on directed R-MAT-{scale} (m={dirg.edges})")


def grid_name(g):
    return f"grid1024-cc: CC on 1024x1024 grid, 5% deleted (n={g.nodes}, m={g.edges})"


def apsp_name(g):
    return f"er8192-apsp: blocked FW on ER n=8192 p=0.001 (m={g.edges})"


# the timed region of either arm runs on inputs larger than L2 (the suite) or
# after a flush; the CPU arm's inputs exceed every host cache
L2_NOTE = "256 MiB write (> 126 MB L2) before every GPU solve; CPU legs run on the same host arrays"


def cpu_grid_once(g, orc):
    dt, kind, cores = cpu_leg(orc, "cc", g)
    return g.edges, dt, cores


def cpu_baseline_grid(g):
    orc = _orc()
    e, t, cores = 0, 0.0, 1
    while t < 2.0:
        de, dt, cores = cpu_grid_once(g, orc)
        e, t = e + de, t + dt
    return {"value": e / t, "unit": "edges/s", "cores": cores, "kind": "port",
            "sample": f"the full 1024x1024 grid, the faster of the serial C oracle CC and its OpenMP rendering "
                      f"(used: {cores} thread(s); the reference has no CPU CC solver), {t:.1f} s"}


APSP_CPU_N = 2048  # sample size for the serial O(n^3) CPU closure


def cpu_apsp_once(g, orc, ref):
    """One serial closure on the host: the reference's own FW_cpu
    (ECL-APSP-atomic.cu:533) when oracle/_ref is built, else the C oracle."""
    import numpy as np

    if ref is not None:
        out = np.zeros((g.nodes, g.nodes), np.int32)
        P = lambda a: C.c_void_p(a.ctypes.data)
        t0 = time.perf_counter()
        ref.eclref_apsp_cpu(g.nodes, g.edges, P(g.nindex), P(g.nlist), P(g.eweight), P(out))
        return float(g.nodes) ** 3, time.perf_counter() - t0, "reference"
    t0 = time.perf_counter()
    orc.apsp(g)
    return float(g.nodes) ** 3, time.perf_counter() - t0, "port"


def cpu_baseline_apsp():
    orc = _orc()
    g = apsp_graph(orc, APSP_CPU_N)
    u, t, kind = cpu_apsp_once(g, orc, _ref())
    return {"value": u / t, "unit": "updates/s", "cores": 1, "kind": kind,
            "sample": f"one serial closure on an ER graph with n={APSP_CPU_N} (same expected degree and weights), "
                      f"{'reference FW_cpu' if kind == 'reference' else 'C oracle'}, {t:.1f} s"}


def reference_gpu_grid(g):
    import torch

    ref = _ref()
    if ref is None or not torch.cuda.is_available():
        return None
    P = lambda t: C.c_void_p(t.data_ptr())
    ni, nl = torch.from_numpy(g.nindex).cuda(), torch.from_numpy(g.nlist).cuda()
    st = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    wl = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
    ms = min(ref.eclref_cc_device(g.nodes, P(ni), P(nl), P(st), P(wl)) for _ in range(5))
    return {"value": g.edges / (ms / 1e3), "unit": "edges/s", "per_code": {"cc": {"ms": ms}},
            "note": "reference race-free CUDA build (nvcc -O3 sm_100a), same graph, its own timed region"}


def reference_gpu_apsp(g):
    import numpy as np
    import torch

    ref = _ref()
    if ref is None or not torch.cuda.is_available():
        return None
    upper = (g.nodes + 63) // 64 * 64
    out = np.zeros((upper, upper), np.int32)
    Q = lambda a: C.c_void_p(a.ctypes.data)
    ms = min(ref.eclref_apsp_gpu(g.nodes, g.edges, Q(g.nindex), Q(g.nlist), Q(g.eweight), Q(out)) for _ in range(2))
    return {"value": float(g.nodes) ** 3 / (ms / 1e3), "unit": "updates/s", "per_code": {"apsp": {"ms": ms}},
            "note": "reference FW_gpu_64 (nvcc -O3 sm_100a), same graph, its printed compute time"}


def reference_gpu(sym, dirg):
    """The reference's race-free CUDA build (oracle/_ref) on the same graphs:
    kernel time as each reference driver times it."""
    import numpy as np
    import torch

    ref = _ref()
    if ref is None or not torch.cuda.is_available():
        return None
    P = lambda t: C.c_void_p(t.data_ptr())
    ni, nl = torch.from_numpy(sym.nindex).cuda(), torch.from_numpy(sym.nlist).cuda()
    res = {}
    st = torch.empty(sym.nodes, dtype=torch.int32, device="cuda")
    wl = torch.empty(sym.nodes, dtype=torch.int32, device="cuda")
    res["cc"] = min(ref.eclref_cc_device(sym.nodes, P(ni), P(nl), P(st), P(wl)) for _ in range(3))
    st8 = torch.empty((sym.nodes + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    res["mis"] = min(ref.eclref_mis_device(sym.nodes, sym.edges, P(ni), P(nl), P(st8)) for _ in range(3))
    scr = torch.empty(ref.eclref_gc_scratch_bytes(sym.nodes, sym.edges) // 4 + 1, dtype=torch.int32, device="cuda")
    res["gc"] = min(ref.eclref_gc_device(sym.nodes, sym.edges, P(ni), P(nl), P(st), P(scr)) for _ in range(3))
    del scr
    inm = np.zeros(sym.edges, np.uint8)
    Q = lambda a: C.c_void_p(a.ctypes.data)
    res["mst"] = min(ref.eclref_mst_gpu(sym.nodes, sym.edges, Q(sym.nindex), Q(sym.nlist), Q(sym.eweight), Q(inm))
                     for _ in range(2))
    del ni, nl, st, wl, st8
    di, dl = torch.from_numpy(dirg.nindex).cuda(), torch.from_numpy(dirg.nlist).cuda()
    scr = torch.empty(ref.eclref_scc_scratch_bytes(dirg.nodes, dirg.edges) // 8 + 2, dtype=torch.int64, device="cuda")
    res["scc"] = min(ref.eclref_scc_device(dirg.nodes, dirg.edges, P(di), P(dl), None, P(scr)) for _ in range(2))
    del di, dl, scr
    torch.cuda.empty_cache()
    edges = {"cc": sym.edges, "mis": sym.edges, "gc": sym.edges, "mst": sym.edges, "scc": dirg.edges}
    tot_e = sum(edges.values())
    tot_ms = sum(res.values())
    return {"value": tot_e / (tot_ms / 1e3), "unit": "edges/s",
            "per_code": {c: {"ms": res[c], "edges_per_s": edges[c] / (res[c] / 1e3)} for c in res},
            "note": "reference race-free CUDA build (nvcc -O3 sm_100a), same graphs, its own timed regions"}


def _reference_line(args, metric, value, unit, ms_per_step, wl, cpu, gpu, world):
    return {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generators: R-MAT / grid / Erdos-Renyi)",
        "config": {"workload": wl, "l2": L2_NOTE}, "parallelism": "host cores (rank 0 only)",
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": gpu,
    }


SUITE_METRIC = "edges/s (sum of g.edges over the suite's solves / sum of solve times; kernel time, inputs resident)"
APSP_METRIC = "updates/s (n^3 / compute time of the blocked Floyd-Warshall closure; inputs resident)"


def reference_small(args, workload, world):
    """Reference arm of the grid and APSP workloads."""
    orc, ref = _orc(), _ref()
    if workload == "grid":
        g = grid_graph(orc)
        for _ in range(args.warmup):
            cpu_grid_once(g, orc)
        u, t, gcores = 0.0, 0.0, 1
        for _ in range(args.steps):
            du, dt, gcores = cpu_grid_once(g, orc)
            u, t = u + du, t + dt
        kind, unit, cores = "port", "edges/s", gcores
        sample = (f"the full 1024x1024 grid, the faster of the serial oracle CC and its OpenMP rendering "
                  f"({gcores} thread(s)); the reference has no CPU CC solver")
        wl, metric = grid_name(g), SUITE_METRIC
        try:
            gpu = reference_gpu_grid(g)
        except Exception as ex:
            gpu = {"error": str(ex)}
    else:
        full = apsp_graph(orc)
        g = apsp_graph(orc, APSP_CPU_N)
        u, t, kind = 0.0, 0.0, "port"
        for _ in range(args.steps):  # no warm-up: each closure takes seconds
            du, dt, kind = cpu_apsp_once(g, orc, ref)
            u, t = u + du, t + dt
        unit, cores = "updates/s", 1
        sample = (f"serial closure on ER n={APSP_CPU_N}, same expected degree and weights "
                  f"({'reference FW_cpu' if kind == 'reference' else 'C oracle'}); one closure per step")
        wl, metric = apsp_name(full), APSP_METRIC
        try:
            gpu = reference_gpu_apsp(full)
        except Exception as ex:
            gpu = {"error": str(ex)}
    value = u / t
    cpu = {"value": value, "unit": unit, "cores": cores, "kind": kind, "sample": sample}
    return _reference_line(args, metric, value, unit, 1e3 * t / args.steps, wl, cpu, gpu, world)


def reference_suite(args, world):
    """Reference arm of the R-MAT suite, on the same R-MAT-22 graphs as our
    arm.  A step is a bounded sample of the suite: ONE code, round robin over
    CC, MIS, GC, MST, SCC, so that K steps cover every code about K/5 times
    (with fewer than 5 steps every step runs the whole suite).  value = one
    pass's edges over the sum of each code's mean time, the suite metric."""
    orc, ref = _orc(), _ref()
    sym, dirg = make_suite_graphs(orc, args.scale)
    whole = args.steps < len(SUITE_LEGS)

    def step(i, times, kinds, cores, edges):
        t = 0.0
        for code in (SUITE_LEGS if whole else (SUITE_LEGS[i % len(SUITE_LEGS)],)):
            edges[code], dt, kinds[code], cores[code] = suite_leg(orc, ref, code, sym, dirg)
            times.setdefault(code, []).append(dt)
            t += dt
        return t

    for i in range(args.warmup):
        step(i, {}, {}, {}, {})
    times, kinds, cores, edges = {}, {}, {}, {}
    t_tot = sum(step(i, times, kinds, cores, edges) for i in range(args.steps))
    value = suite_rate(times, edges)
    cpu = {"value": value, "unit": "edges/s", "cores": max(cores.values()), "kind": overall_kind(kinds),
           "sample": "the suite on the same R-MAT-22 graphs, one code per step round robin: MST by the reference's "
                     "own serial cpuMST; CC/MIS/GC/SCC (no CPU solver in the reference) by the faster of the serial "
                     f"C oracle and its OpenMP rendering ({orc.omp_threads()} threads) on this host",
           "per_code_kind": kinds, "per_code_cores": cores,
           "per_code_mean_s": {c: round(sum(v) / len(v), 3) for c, v in times.items()}}
    try:
        gpu = reference_gpu(sym, dirg)
    except Exception as ex:  # reported, not fatal: the CPU arm is the reference arm
        gpu = {"error": str(ex)}
    return _reference_line(args, SUITE_METRIC, value, "edges/s", 1e3 * t_tot / args.steps,
                           suite_name(args.scale, sym, dirg), cpu, gpu, world)


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload in ("batch", "serve"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched or served mode: each "
                          "ECL code is a standalone executable that solves one graph per process"}), flush=True)
        return
    if args.workload == "suite":
        line = reference_suite(args, world)
        if world == 1 and args.other_configs:
            sub = argparse.Namespace(**vars(args))
            sub.steps, sub.warmup = min(args.steps, 5), min(args.warmup, 1)
            line["other_configs"] = {w: reference_small(sub, w, world) for w in ("grid", "apsp")}
    else:
        line = reference_small(args, args.workload, world)
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    if args.workload == "batch":
        line = bench_batch(args, rank, world, local_rank)
    elif args.workload == "serve":
        line = bench_serve(args, rank, world, local_rank)
    else:
        line = bench_plain(args, rank, world, local_rank)
        # the other configs on one GPU only: a scaling run times the suite
        if args.workload == "suite" and world == 1 and args.other_configs:
            line["other_configs"] = other_configs(args, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import datetime

    import torch

    if world > 1:
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
