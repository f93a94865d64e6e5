"""Benchmark: exact subgraph counting throughput (matches/s) on B200.

Headline workload ("plain, mid"): R-MAT scale 20, edge factor 3,
(a, b, c) = (0.57, 0.19, 0.19), seed 7 (loops and duplicates removed, int32
CSR with both directions); one step = device build of the graph from the
resident CSR, then exact counts of the 4-clique and the diamond (sgm), each
including its peel and priority relabelling.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--extras c1,c3,c4,c5] [--workload c1|c2|c3|c4|c5]

value: total matches counted per second with the CSR resident in HBM (device
time over K steps, CUDA events on the library's stream, L2 flushed between
steps). e2e: the same through the public API from pinned host buffers,
host->device copy of the CSR and the count read-back inside the timed region.
Under torchrun each rank builds the graph and counts the roots whose input id
% N == rank (beep_count_shard), and one NCCL all-reduce per step sums the
counts; times are the max over ranks.

The same JSON line carries the other workloads under extra keys: "c1" (ER
triangle, sgc), "c3" (R-MAT scale 22 edge factor 28, 5-clique + 4-wheel, one
timed step), "c4" (batched: Chung-Lu graphs x the 15 central 4-5-vertex
patterns, one CUDA-graph replay against the per-pair loop) and "c5" (served:
a Poisson request stream, p50/p99 latency, against running the requests one
after another).

The reference arm (--impl reference) runs the reference's own binary
(oracle/_ref/beep_ref, src/main.cu built for sm_100a) on the same C2 and C1
inputs, written by the numpy generators in oracle/synth.py: that process
never loads this library.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "matches/sec on 1 B200 (exact counts), batched/served vs plain; p50/p99 latency"
UNIT = "matches/s"
L2_NOTE = "cold: L2 flushed (256 MB write) before every step; the reference starts a process per pattern"

WORKLOADS = {
    "c2": {"desc": "plain-mid: R-MAT s20 ef3 seed 7; 4-clique + diamond (sgm)",
           "graph": ("rmat", (20, 3, 0.57, 0.19, 0.19, 7)), "patterns": ["k4", "diamond"], "mode": "sgm"},
    "c3": {"desc": "plain-large: R-MAT s22 ef28 seed 11; 5-clique + 4-wheel (sgm)",
           "graph": ("rmat", (22, 28, 0.57, 0.19, 0.19, 11)), "patterns": ["k5", "w5"], "mode": "sgm"},
    "c1": {"desc": "plain-small: ER G(4096, 0.004) seed 1; triangle (sgc)",
           "graph": ("er", (4096, 0.004, 1)), "patterns": ["triangle"], "mode": "sgc"},
    "c4": {"desc": "batched: Chung-Lu graphs (exponent 2.1, seed 13) x the 15 central 4-5-vertex patterns (sgm)"},
    "c5": {"desc": "served: Poisson requests (seed 17) over resident Chung-Lu graphs (exponent 2.1)"},
}


# Why the reference arm does not run the large workload: its neighbourhood
# bitmap buffer is grid x maxdeg x ceil(maxdeg / 32) words, one cudaMalloc
# (subgraph_matching.cuh:1185-1191); at the large workload's maximum degree
# that is terabytes. The recorded attempt is in tests/golden/reference_counts.json.
REFERENCE_C3 = ("the reference's per-block bitmap buffer (grid x maxdeg x ceil(maxdeg/32) u32, "
                "subgraph_matching.cuh:1185-1191) does not fit one B200 at max degree ~240K; see "
                "tests/golden/reference_counts.json")


def patterns_module():
    """beep_b200/patterns.py loaded by path (plain Python: edge lists of the
    named queries), so the reference arm does not import the library."""
    spec = importlib.util.spec_from_file_location("beep_patterns", os.path.join(ROOT, "beep_b200", "patterns.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_config(wl: dict, n: int, m: int) -> dict:
    """The config object both arms print for a plain workload."""
    return {"workload": wl["desc"], "n": int(n), "m_directed": int(m), "patterns": list(wl["patterns"]),
            "mode": wl["mode"], "l2": L2_NOTE}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def profiled_traffic() -> dict:
    """Per-launch DRAM bytes (read + write) of kernels captured with ncu, as
    recorded in the summaries under profiles/ (lines
    'traffic_bytes_per_launch[<kernel>]: <bytes>', each with the file it came
    from). ncu cannot run inside this process, so the figure is the one of the
    committed capture, not of this run."""
    import glob
    import re

    out = {}
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for m in re.finditer(r"traffic_bytes_per_launch\[(\w+)\]:\s*([0-9.eE+]+)", f.read()):
                out[m.group(1)] = (float(m.group(2)), os.path.relpath(path, ROOT))
    return out


def note(msg: str) -> None:
    """Progress on stderr (the JSON line stays alone on stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def gen_graph(kind, args):
    import beep_b200 as B

    return {"rmat": B.gen_rmat, "er": B.gen_erdos_renyi, "cl": B.gen_chung_lu}[kind](*args)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 500 ms (each query
    takes driver time; a timed region of one to two seconds still gets two or
    more samples)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "500"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's own start-up takes driver time: let it finish (first
        # sample printed) before the timed region begins
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
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
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# ranks
# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def _coll_device():
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float, world: int) -> float:
    """Largest value over the ranks (device times are reported as the max)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_coll_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_counts_over_ranks(xs: list[int], world: int) -> list[int]:
    """Element-wise sum of exact counts over the ranks: one int64 all-reduce."""
    if world == 1:
        return [int(x) for x in xs]
    import torch
    import torch.distributed as dist

    t = torch.tensor([int(x) for x in xs], dtype=torch.int64, device=_coll_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [int(v) for v in t.tolist()]


def sum_over_ranks(x: int, world: int) -> int:
    return sum_counts_over_ranks([x], world)[0]


def sharded_counts(count_shard, patterns: list, world: int, rank: int) -> list[int]:
    """Counts of every pattern with the roots sharded over the ranks: this
    rank counts the roots whose input vertex id % world == rank
    (count_shard(pattern, shard, nshards)); roots are independent, so one
    all-reduce of the per-pattern counts gives the full counts on every rank."""
    local = [count_shard(p, rank, world) for p in patterns]
    return sum_counts_over_ranks(local, world)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (OpenMP port of the reference algorithm) on the
# host cores, on the same workload
# ---------------------------------------------------------------------------
def cpu_baseline(rp, col, wl, budget_s: float = 20.0) -> dict:
    from oracle import pyoracle as O

    P = patterns_module()
    threads = os.cpu_count() or 1
    sgc = wl["mode"] == "sgc"
    t0 = time.perf_counter()
    total = 0
    for name in wl["patterns"]:
        total += O.count(rp, col, P.NAMED[name], sgc=sgc, threads=threads)["count"]
    dt = time.perf_counter() - t0
    runs = 1
    # repeat the full workload while it stays inside the time budget
    while dt / runs * (runs + 1) < budget_s and runs < 5:
        for name in wl["patterns"]:
            O.count(rp, col, P.NAMED[name], sgc=sgc, threads=threads)
        runs += 1
        dt = time.perf_counter() - t0
    return {"value": total * runs / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"full workload ({' + '.join(wl['patterns'])}, all roots) x{runs}, {dt:.1f} s, "
                      f"OpenMP oracle on {threads} host threads"}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference_binary(binary, bel, mtx, mode, timeout):
    r = subprocess.run([binary, "-g", bel, "-t", mtx, "-m", mode, "-d", "0"], capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference exited {r.returncode}: {r.stderr[-400:]}")
    out = r.stdout
    import re

    cnt = re.search(r"Counter = (\d+)", out)
    prep = re.search(r"Preprocessing TIME: ([0-9.eE+-]+) ms", out)
    fin = re.search(r"final count time ([0-9.eE+-]+) s", out)
    xfer = re.search(r"Transfer Time: ([0-9.eE+-]+) s", out)
    if not cnt or not fin:
        raise RuntimeError("reference output lacks the Counter / final count time lines")
    t = float(fin.group(1)) + (float(prep.group(1)) / 1e3 if prep else 0.0) + (float(xfer.group(1)) if xfer else 0.0)
    return int(cnt.group(1)), t


def synth_graph(kind, args):
    from oracle import synth as S

    return {"rmat": S.rmat, "er": S.erdos_renyi, "cl": S.chung_lu}[kind](*args)


def reference_workload(args, wl, binary, budget_s) -> dict:
    """The reference binary on one plain workload: one process per pattern per
    step, each timed by its own Transfer + Preprocessing + final count lines
    (file parsing excluded); median over the steps that fit the budget."""
    from oracle import synth as S

    P = patterns_module()
    rp, col = synth_graph(*wl["graph"])
    out = {"config": workload_config(wl, len(rp) - 1, len(col))}
    with tempfile.TemporaryDirectory() as td:
        bel = os.path.join(td, "g.bel")
        S.write_bel(bel, rp, col)
        mtxs = {}
        for name in wl["patterns"]:
            mtxs[name] = os.path.join(td, f"{name}.mtx")
            S.write_mtx(mtxs[name], P.NAMED[name])
        # one untimed run per pattern (process start, module load, file cache)
        if args.warmup > 0:
            for name in wl["patterns"]:
                run_reference_binary(binary, bel, mtxs[name], wl["mode"], args.reference_timeout)
        times, counts = [], None
        t_start = time.time()
        for _ in range(args.steps):
            if times and time.time() - t_start > budget_s:
                break  # bounded: each step is a full process run per pattern
            tot_t, cs = 0.0, []
            for name in wl["patterns"]:
                c, t = run_reference_binary(binary, bel, mtxs[name], wl["mode"], args.reference_timeout)
                cs.append(c)
                tot_t += t
            counts = cs
            times.append(tot_t)
    med = statistics.median(times)
    out.update({"value": sum(counts) / med, "unit": UNIT, "ms_per_step": med * 1e3,
                "counts": dict(zip(wl["patterns"], counts)), "steps_run": len(times)})
    return out


def reference_arm(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return  # one reference process on rank 0; the others exit without work
    binary = os.path.join(ROOT, "oracle", "_ref", "beep_ref")
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic"}
    if os.path.exists(binary) and not args.reference_port:
        try:
            r = reference_workload(args, wl, binary, args.reference_budget)
            line.update({"value": r["value"], "ms_per_step": r["ms_per_step"], "config": r["config"],
                         "counts": r["counts"], "steps_run": r["steps_run"],
                         "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                          "sample": "the reference's own sgm/sgc (src/main.cu built for sm_100a by "
                                                    "oracle/refbuild.py) run on the B200 from one host thread; "
                                                    "time per step = its Transfer + Preprocessing + final count "
                                                    "lines for each pattern (file parsing excluded); median of "
                                                    f"{r['steps_run']} steps"},
                         "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                 "d2h_bytes_per_step": 0},
                         "inputs": "written by oracle/synth.py (numpy); this process loads no library of this "
                                   "repository"})
            if args.workload == "c2" and "c1" in args.extras_list:
                try:
                    c1 = reference_workload(args, WORKLOADS["c1"], binary, args.reference_budget / 3)
                    line["c1"] = c1
                except (RuntimeError, subprocess.TimeoutExpired) as e:
                    line["c1"] = {"error": str(e)[:300]}
            print(json.dumps(line), flush=True)
            return
        except (RuntimeError, subprocess.TimeoutExpired) as e:
            line["reference_binary_error"] = str(e)[:300]
    # the CPU port of the reference algorithm
    rp, col = synth_graph(*wl["graph"])
    cb = cpu_baseline(rp, col, wl, budget_s=30.0)
    line.update({"value": cb["value"], "ms_per_step": None, "config": workload_config(wl, len(rp) - 1, len(col)),
                 "cpu_baseline": cb,
                 "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# plain workloads (our arm)
# ---------------------------------------------------------------------------
def plain_workload(args, wl, world, rank, local, steps, warmup, with_serial=True, with_cpu=True,
                   with_e2e=True) -> dict:
    """One plain workload timed as the module docstring describes. Returns
    the fields of its JSON object."""
    import torch

    import beep_b200 as B
    from beep_b200 import patterns as P

    rp, col = gen_graph(*wl["graph"])
    n, m = len(rp) - 1, len(col)
    note(f"{wl['desc']}: n={n} m={m}")
    mode = B.SGC if wl["mode"] == "sgc" else B.SGM
    stream = torch.cuda.Stream()
    ctx = B.Context(local, cuda_stream=stream.cuda_stream)
    queries = [B.Query.from_edges(P.NAMED[p]) for p in wl["patterns"]]
    d_rp = torch.from_numpy(rp).cuda()
    d_col = torch.from_numpy(col).cuda()
    h_rp = torch.from_numpy(rp).pin_memory()
    h_col = torch.from_numpy(col).pin_memory()
    h_rp_np, h_col_np = h_rp.numpy(), h_col.numpy()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    torch.cuda.synchronize()

    def step(host: bool, options: int = 0):
        if host:
            g = B.Graph.from_csr(ctx, h_rp_np, h_col_np)
        else:
            g = B.Graph.from_device_csr(ctx, n, m, d_rp.data_ptr(), d_col.data_ptr())
        sts = []
        if world > 1:
            # roots sharded over the ranks, one all-reduce of the counts
            def count_shard(q, shard, nshards):
                c, st = B.count_shard(g, q, shard, nshards, mode, options, ctx=ctx, stats=True)
                sts.append(st)
                return c

            counts = sharded_counts(count_shard, queries, world, rank)
        elif args.step_api == "batch":
            # one planned call over every pattern: the views of all patterns
            # are built, then all their count kernels run together
            b = B.Batch(ctx)
            for q in queries:
                b.add(g, q, mode)
            counts, st = b.run(options | B.OPT_NO_GRAPH, stats=True)
            b.close()
            sts = [st]
        else:
            counts = []
            for q in queries:
                c, st = B.count(g, q, mode, options, ctx=ctx, stats=True)
                counts.append(c)
                sts.append(st)
        g.close()
        return counts, sts

    def timed(host: bool, k: int, options: int = 0):
        for _ in range(warmup):
            step(host, options)
        torch.cuda.synchronize()
        barrier(world)
        launches0 = ctx.kernel_launches()
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            stream.synchronize()
            e0.record(stream)
            total, allst, counts = 0, [], None
            for _ in range(k):
                flush.fill_(1)
                counts, sts = step(host, options)
                total += sum(counts)
                allst.append(sts)
            e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1)
        return total, ms, allst, ctx.kernel_launches() - launches0, counts

    clk = ClockSampler(local)
    clk.start()
    total, ms, allst, launches, counts = timed(False, steps)
    clocks = clk.stop()
    ms = max_over_ranks(ms, world)
    ms_step = ms / steps
    per_step = total // steps
    value = per_step / (ms_step / 1e3)

    e_total, e_ms = 0, 0.0
    if with_e2e:
        e_total, e_ms, _, _, _ = timed(True, steps)
        e_ms = max_over_ranks(e_ms, world)
    e2e_value = (e_total // steps) / (e_ms / steps / 1e3) if with_e2e else None

    # host->device copy of one step's inputs alone (pinned buffers, same stream), to explain e2e - value
    with torch.cuda.stream(stream):
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(3):
            d_rp.copy_(h_rp, non_blocking=True)
            d_col.copy_(h_col, non_blocking=True)
        c1.record(stream)
    c1.synchronize()
    h2d_ms = c0.elapsed_time(c1) / 3

    out = {"value": value, "unit": UNIT, "ms_per_step": ms_step, "steps": steps, "warmup": warmup,
           "config": workload_config(wl, n, m), "counts": dict(zip(wl["patterns"], counts)),
           "matches_per_step": per_step,
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(4 * (n + 1) + 4 * m),
                   "d2h_bytes_per_step": 16 * len(queries), "ms_per_step": e_ms / steps if with_e2e else None,
                   "h2d_copy_ms": h2d_ms},
           "gpu_launches": int(launches), "clocks": clocks,
           "step": "device CSR build + per-pattern peel/relabel + count" +
                   (f", roots sharded over {world} ranks (beep_count_shard) + one NCCL all-reduce of the counts"
                    if world > 1 else
                    (", all patterns in one batched call (beep_batch, no CUDA graph)" if args.step_api == "batch"
                     else ", one beep_count per pattern"))}
    if with_serial and world == 1:
        out.update(serial_phases(B, step, timed, steps))
    if with_cpu and rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(rp, col, wl)
    ctx.close()
    return out


def serial_phases(B, step, timed, steps) -> dict:
    """Per-kernel times. In the timed steps the kernel tiers overlap on side
    streams, so an event pair around one kernel measures the overlap, not the
    kernel. These steps run the same work with the tiers one after another
    (BEEP_OPT_SERIAL_TIERS) and an event pair around every launch, so each
    kernel's time is its own and the shares compare with the ncu launch list."""
    ser_steps = max(1, min(steps, 10))
    _, _, allst, _, _ = timed(False, ser_steps, B.OPT_TIMING | B.OPT_SERIAL_TIERS)
    # adjacency bytes per tier, from one untimed pass (identical every step)
    _, byte_sts = step(False, B.OPT_ALG_BYTES)
    for sts in allst:
        for st, bst in zip(sts, byte_sts):
            for k in ("small_bytes", "medium_bytes", "large_bytes", "adjacency_bytes", "alg_small_bytes",
                      "alg_medium_bytes", "alg_large_bytes"):
                st[k] = bst[k]
    # dominant kernel of the counting phase: its algorithmic bytes (4 * (deg r
    # + sum of the neighbours' degrees) per searched root, on the input CSR)
    # and the adjacency bytes it actually has to read (its own model)
    tiers = {"small": ("small_ms", "alg_small_bytes", "small_bytes", "small_launches", "k_small"),
             "medium": ("medium_ms", "alg_medium_bytes", "medium_bytes", "medium_launches", "k_medium"),
             "large_dfs": ("large_dfs_ms", "alg_large_bytes", "large_bytes", "large_dfs_launches", "k_large_dfs"),
             "large_rows": ("large_encode_ms", "alg_large_bytes", "large_bytes", "large_encode_launches",
                            "k_large_rows")}
    agg = {k: [0.0, 0, 0, 0] for k in tiers}
    prep_ms = count_ms = 0.0
    for sts in allst:
        for st in sts:
            prep_ms += st["prep_ms"]
            count_ms += st["count_ms"]
            for k, (tk, ak, bk, lk, _) in tiers.items():
                agg[k][0] += st[tk]
                agg[k][1] += st[ak]
                agg[k][2] += st[bk]
                agg[k][3] += st[lk]
    dom = max(agg, key=lambda k: agg[k][0])
    dom_ms, dom_bytes, dom_read, dom_launches = agg[dom]
    peak, peak_kind = peaks()
    achieved = (dom_bytes / max(dom_launches, 1)) / ((dom_ms / max(dom_launches, 1)) / 1e3) / 1e9 if dom_ms else 0.0
    traffic = profiled_traffic().get(tiers[dom][4])
    return {
        "phases_ms_per_step": {"prep": prep_ms / ser_steps, "count": count_ms / ser_steps,
                               **{k: v[0] / ser_steps for k, v in agg.items()},
                               "note": f"{ser_steps} extra steps with the kernel tiers serialised and timed per "
                                       "launch"},
        "roofline": {"bound": "hbm", "kernel": tiers[dom][4], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": traffic[0] if traffic else None,
                     "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one {tiers[dom][4]} "
                                        f"launch on this workload, recorded in {traffic[1]} (not measured in this "
                                        "run)") if traffic else None,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                     else "fallback 6650 GB/s",
                     "bytes_per_launch": dom_bytes / max(dom_launches, 1),
                     "bytes_def": "algorithmic: 4*(deg r + sum of deg v over N(r)) per searched root, input CSR",
                     "read_model_bytes_per_launch": dom_read / max(dom_launches, 1),
                     "ms_per_launch": dom_ms / max(dom_launches, 1),
                     "timing": "per-launch CUDA events in steps with the kernel tiers serialised"},
    }


# ---------------------------------------------------------------------------
# batched and served forms
# ---------------------------------------------------------------------------
def c4_graph_specs(n_graphs, lo_scale, hi_scale, dmin, dmax, seed=13):
    import numpy as np

    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_graphs):
        n = int(round(2 ** rng.uniform(lo_scale, hi_scale)))
        d = float(rng.uniform(dmin, dmax))
        specs.append((n, d, 2.1, seed * 1000 + i))
    return specs


def pattern_label(edges, index) -> str:
    """'<index>:<name>' for a query edge list: its name among the named
    patterns when it is one of them, else its vertex and edge counts."""
    from beep_b200 import patterns as P

    n = max(max(a, b) for a, b in edges) + 1
    und = sorted({(min(a, b), max(a, b)) for a, b in edges})
    canon = P._canon(n, und)
    for name, q in P.NAMED.items():
        qn = max(max(a, b) for a, b in q) + 1
        if qn == n and P._canon(qn, sorted({(min(a, b), max(a, b)) for a, b in q})) == canon:
            return f"{index}:{name}"
    return f"{index}:{n}v{len(und)}e"


def bench_batched(args) -> dict:
    import torch

    import beep_b200 as B
    from beep_b200 import patterns as P

    specs = c4_graph_specs(args.c4_graphs, 10, args.c4_max_scale, 8, args.c4_max_degree)
    stream = torch.cuda.Stream()
    ctx = B.Context(0, cuda_stream=stream.cuda_stream)
    t0 = time.perf_counter()
    host = [B.gen_chung_lu(*sp) for sp in specs]
    gen_s = time.perf_counter() - t0
    graphs = [B.Graph.from_csr(ctx, rp, col) for rp, col in host]
    note(f"c4: {len(graphs)} graphs generated in {gen_s:.1f} s, {sum(len(c) for _, c in host)} directed edges")
    qedges = P.central_patterns(4) + P.central_patterns(5)
    pats = [B.Query.from_edges(q) for q in qedges]
    pairs = [(gi, qi) for gi in range(len(graphs)) for qi in range(len(pats))]

    def plain(gi, qi):
        try:
            return B.count(graphs[gi], pats[qi])
        except B.BeepError as e:
            if e.status != B.ERR_OVERFLOW:
                raise
            return B.COUNT_OVERFLOW

    # the batch first: planning builds every graph's views (cached on the
    # graphs), classifies the roots and captures the launches
    batch = B.Batch(ctx)
    for gi, qi in pairs:
        batch.add(graphs[gi], pats[qi])
    tuned = None
    if args.c4_autotune:
        t0 = time.perf_counter()
        # tier limits and donation threshold by measurement (or from the tuning
        # cache file), before the timed replays
        tuned = batch.autotune(cache=args.c4_tune_cache,
                               key=f"c4:{args.c4_graphs}:{args.c4_max_scale}:{args.c4_max_degree}")
        tuned["seconds"] = time.perf_counter() - t0
        note(f"c4: autotune {tuned['seconds']:.1f} s")
    t0 = time.perf_counter()
    first = batch.run()  # plans and captures
    plan_s = time.perf_counter() - t0
    note(f"c4: plan (views included) + capture + first replay {plan_s:.1f} s")
    # plain loop: one count per pair, views resident
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_counts = []
    by_pattern = [0.0] * len(pats)  # per-pair loop seconds per pattern: where the GPU time goes
    for gi, qi in pairs:
        t1 = time.perf_counter()
        plain_counts.append(plain(gi, qi))
        by_pattern[qi] += time.perf_counter() - t1
    plain_s = time.perf_counter() - t0
    note(f"c4: per-pair loop {plain_s:.1f} s")
    clocks = ClockSampler(0)
    clocks.start()
    for _ in range(args.warmup):
        batch.run()
    times, host_times = [], []
    got = first
    for _ in range(args.steps):
        # device time of one replay on the library's stream (CUDA events), and
        # the host time of the call around it
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        got = batch.run()
        e1.record(stream)
        e1.synchronize()
        host_times.append(time.perf_counter() - t0)
        times.append(e0.elapsed_time(e1) / 1e3)
    clk = clocks.stop()
    assert got == first and got == plain_counts, "batched counts differ from the plain loop"
    over = [i for i, c in enumerate(got) if c == B.COUNT_OVERFLOW]
    total = sum(c for c in got if c != B.COUNT_OVERFLOW)
    step_s = statistics.median(times)
    host_s = statistics.median(host_times)
    out = {"form": "batched", "value": total / step_s, "unit": UNIT, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": step_s * 1e3, "host_ms_per_step": host_s * 1e3, "clocks": clk,
           "config": {"workload": WORKLOADS["c4"]["desc"], "graphs": len(graphs), "patterns": len(pats),
                      "pairs": len(pairs), "n_log2_range": [10, args.c4_max_scale],
                      "avg_degree_range": [8, args.c4_max_degree],
                      "edges_directed": int(sum(len(c) for _, c in host)),
                      "step": "one replay of the captured CUDA graph over every pair (views resident)"},
           "matches_per_step": int(total),
           "overflow_pairs": [{"graph": pairs[i][0], "graph_spec": list(specs[pairs[i][0]][:2]),
                               "pattern": pairs[i][1]} for i in over],
           "plain_loop": {"value": total / plain_s, "ms": plain_s * 1e3,
                          "what": "beep_count per pair, same pairs, views resident, host wall time",
                          "s_by_pattern": {pattern_label(qedges[qi], qi): round(by_pattern[qi], 3) for qi in
                                           sorted(range(len(pats)), key=lambda q: -by_pattern[q])}},
           "speedup_vs_plain_loop": plain_s / host_s,
           "speedup_note": "both sides host wall time of the calls (the replay's device time is ms_per_step)",
           "plan_and_capture_ms": plan_s * 1e3, "autotuned_tiers": tuned, "generate_s": gen_s}
    batch.close()
    for g in graphs:
        g.close()
    ctx.close()
    return out


def bench_served(args) -> dict:
    import numpy as np
    import torch

    import beep_b200 as B
    from beep_b200 import patterns as P

    rng = np.random.default_rng(17)
    ctx = B.Context(0)
    graphs, host = [], []
    for i in range(args.c5_graphs):
        m_und = 10 ** rng.uniform(4, args.c5_max_log10_edges)
        n = max(64, int(2 * m_und / 16))
        rp, col = B.gen_chung_lu(n, 16.0, 2.1, 17000 + i)
        host.append((rp, col))
        graphs.append(B.Graph.from_csr(ctx, rp, col))
    note(f"c5: {len(graphs)} graphs, {sum(len(c) for _, c in host)} directed edges")
    names = ["triangle", "diamond", "k4", "tailed_triangle", "w5", "k5"]
    queries = {nm: B.Query.from_edges(P.NAMED[nm]) for nm in names}
    n_req = int(args.c5_rate * args.c5_seconds)
    gaps = rng.exponential(1.0 / args.c5_rate, size=n_req)
    arrivals = np.cumsum(gaps)
    reqs = [(int(rng.integers(0, len(graphs))), names[int(rng.integers(0, len(names)))],
             args.c5_k if rng.random() < 0.2 else 0) for _ in range(n_req)]
    # serial plain execution of the same requests (views warmed first)
    for g in graphs:
        for nm in names:
            B.count(g, queries[nm])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    serial = []
    by_kind = {}  # serial seconds per (pattern, count or first-k) kind: where the GPU time goes
    for gi, nm, k in reqs:
        t1 = time.perf_counter()
        if k:
            _, tot = B.enumerate_matches(graphs[gi], queries[nm], k)
            serial.append(tot)
        else:
            serial.append(B.count(graphs[gi], queries[nm]))
        kind = f"{nm}/{'first-k' if k else 'count'}"
        by_kind[kind] = by_kind.get(kind, 0.0) + time.perf_counter() - t1
    serial_s = time.perf_counter() - t0
    note(f"c5: serial run of {n_req} requests {serial_s:.1f} s")
    srv = B.Server(ctx, max_batch=args.c5_max_batch, streams=args.c5_streams)
    gids = [srv.add_graph(g) for g in graphs]
    start = time.perf_counter()
    rids = []
    for (gi, nm, k), at in zip(reqs, arrivals):
        now = time.perf_counter() - start
        if at > now:
            time.sleep(at - now)
        rids.append((srv.submit(gids[gi], queries[nm], B.SGM, k), k))
    served = [srv.wait(rid, k)["count"] for rid, k in rids]
    st = srv.stats()
    assert served == serial, "served counts differ from the serial run"
    total = sum(served)
    out = {"form": "served", "value": total / st["span_s"], "unit": UNIT,
           "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
           "config": {"workload": WORKLOADS["c5"]["desc"], "graphs": len(graphs),
                      "log10_undirected_edges_range": [4, args.c5_max_log10_edges], "avg_degree": 16,
                      "rate_per_s": args.c5_rate, "requests": n_req, "enumerate_fraction": 0.2,
                      "enumerate_k": args.c5_k, "patterns": names, "max_batch": args.c5_max_batch,
                      "streams": args.c5_streams,
                      "edges_directed": int(sum(len(c) for _, c in host))},
           "matches": int(total),
           "serial_plain": {"value": total / serial_s, "s": serial_s,
                            "s_by_kind": {k: round(v, 3) for k, v in sorted(by_kind.items(), key=lambda x: -x[1])}},
           "speedup_vs_serial_plain": (total / st["span_s"]) / (total / serial_s),
           "batches": st["batches"], "largest_batch": st["max_batch"], "span_s": st["span_s"],
           "offered_span_s": float(arrivals[-1]) if n_req else 0.0}
    srv.close()
    for g in graphs:
        g.close()
    ctx.close()
    return out


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--extras", default="c1,c3,c4,c5",
                    help="with the c2 workload on one GPU: other workloads reported under extra keys ('' for none)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--step-api", choices=["batch", "plain"], default="batch",
                    help="count the step's patterns with one batched call or one beep_count per pattern")
    ap.add_argument("--reference-port", action="store_true", help="reference arm: use the CPU port")
    ap.add_argument("--reference-timeout", type=float, default=300.0)
    ap.add_argument("--reference-budget", type=float, default=150.0,
                    help="reference arm: stop starting new steps after this many seconds")
    ap.add_argument("--c3-steps", type=int, default=1)
    ap.add_argument("--c4-graphs", type=int, default=256)
    ap.add_argument("--c4-max-scale", type=float, default=18.0)
    ap.add_argument("--c4-max-degree", type=float, default=64.0)
    ap.add_argument("--c4-autotune", action="store_true",
                    help="batched: pick the tier limits and donation threshold by measurement before the replays")
    ap.add_argument("--c4-no-autotune", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--c4-steps", type=int, default=2)
    ap.add_argument("--c4-tune-cache", default=None,
                    help="JSON file of autotuned tier limits per batched workload (read if present, else written)")
    ap.add_argument("--c5-graphs", type=int, default=32)
    ap.add_argument("--c5-max-log10-edges", type=float, default=7.0)
    ap.add_argument("--c5-rate", type=float, default=2000.0)
    ap.add_argument("--c5-seconds", type=float, default=2.0)
    ap.add_argument("--c5-k", type=int, default=10000)
    ap.add_argument("--c5-max-batch", type=int, default=64)
    ap.add_argument("--c5-streams", type=int, default=4)
    args = ap.parse_args()
    args.extras_list = [x for x in args.extras.split(",") if x]
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        if args.workload == "c3":
            print(json.dumps({"impl": "reference", "unavailable": REFERENCE_C3}))
            return
        if args.workload not in ("c1", "c2"):
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched or served form "
                                                                  "(one SG_Match per query and graph)"}))
            return
        reference_arm(args, wl)
        return

    base = {"metric": METRIC, "impl": "ours", "higher_is_better": True, "vs_baseline": None, "dtype": "u32",
            "data": "synthetic"}
    if args.workload == "c4":
        c4args = argparse.Namespace(**{**vars(args), "steps": args.steps, "warmup": args.warmup})
        print(json.dumps({**base, "n_gpus": 1, "scaling": "strong", **bench_batched(c4args)}), flush=True)
        return
    if args.workload == "c5":
        print(json.dumps({**base, "n_gpus": 1, "scaling": "strong", **bench_served(args)}), flush=True)
        return

    world, rank, local = dist_setup()
    import torch

    torch.cuda.set_device(local)
    res = plain_workload(args, wl, world, rank, local, args.steps, args.warmup)
    line = {**base, "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "scaling": "strong",
            "sharding": f"roots by input id % {world} (beep_count_shard), one NCCL all-reduce per step"
            if world > 1 else "one GPU", **res}
    if world == 1 and args.workload == "c2":
        # the other workloads, each under its own key, each in its own guard
        for key in args.extras_list:
            t0 = time.perf_counter()
            try:
                if key in ("c1", "c3"):
                    k_steps = args.steps if key == "c1" else args.c3_steps
                    k_warm = args.warmup if key == "c1" else 0
                    r = plain_workload(args, WORKLOADS[key], 1, 0, 0, k_steps, k_warm, with_serial=(key == "c1"),
                                       with_cpu=(key == "c1"), with_e2e=(key == "c1"))
                elif key == "c4":
                    # the replay right after the capture is the warm-up of these timed replays
                    r = bench_batched(argparse.Namespace(**{**vars(args), "steps": args.c4_steps, "warmup": 0}))
                elif key == "c5":
                    r = bench_served(args)
                else:
                    continue
            except Exception as e:  # a failed extra must not lose the headline line
                r = {"error": f"{type(e).__name__}: {str(e)[:400]}"}
            r["wall_s"] = time.perf_counter() - t0
            line[key] = r
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
