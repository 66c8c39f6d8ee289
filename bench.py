"""Benchmark: RRR sets/s of full IMM runs on one or more B200s.

Default workload (N=1): plain IMM under the IC model on a directed R-MAT graph
with 2^24 vertices and 32*2^24 edge draws (a,b,c,d = .57,.19,.19,.05, seed 0,
self-loops and duplicates removed: m = 520 761 423), weighted-cascade
probabilities p = 1/in-degree(dst), k=100, epsilon=0.13, seeds chosen with the
reference CPU heap's tie-break.  Other workloads: --workload lt20 (R-MAT 2^20,
16*2^20 draws, LT in-weights U(0,1) normalised per destination, k=50,
epsilon=0.3), ic14 (R-MAT 2^14, 2^18 draws, IC p ~ U(0,0.1), k=20,
epsilon=0.5), ic24_samplers (each IC sampler on one fixed set range of the
2^24 graph), b1 (batching), s1 (serving), spread (forward Monte Carlo).

One step = one complete IMM (martingale theta estimation + final sampling +
final greedy selection) from an empty RRR pool, with a fresh sampler seed each
step, the graph already resident in HBM.  The K timed steps are split between
--clients concurrent client threads (3 on the 2^24 IC workload, 4 on the
2^20 LT one, else 1), each with its own context,
graph copy and pool, so that one query's sampling fills the GPU while
another's reference-heap selection waits on the host.  value = RRR sets
generated per second, summed over ranks, over the max-over-ranks device time
of the K timed steps; one_client = the same IMMs one after another.  e2e = the same metric through the public API with the graph uploaded
from pinned host memory and the seeds read back every step, from the
workload's concurrent clients (at least two, one context each) so that a
step's upload overlaps other steps' IMMs; e2e.serial is one client doing
both in turn.

Multi-GPU: the path does not shard across GPUs in this build ("replicas
only"): each rank runs its own independent IMM query (its own seeds), and
`value` aggregates the ranks' sets -- weak scaling, no collective on the data
path.

--impl reference runs the reference's own CPU implementation (built from its
sources into oracle/_ref/ by oracle/ref.mk) on rank 0 only, on the same graph
written in the reference's binary format by the oracle's generator (the
process never loads this package's library):
  IC: the imm tool's `-p --rrsets N` sampling path (GenerateRRRSets over an
      ICStreamingGenerator on every host thread), N sized so a step takes a
      few seconds: sets/s of sampling alone, an upper bound of the reference's
      full-IMM rate (its selection time is left out).
  LT: the sequential imm (`-p` runs IC coin flips on its CPU workers,
      include/ripples/batched_add_rrrset.h:231-245), full IMM runs, 1 core.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # clients: concurrent IMM clients of the timed region (a query's
    # reference-heap selection waits on the host while another's sampling and
    # picks use the GPU): 3 on the 2^24 IC graph (1, 2, 3, 4 clients: 5.5,
    # 6.6, 7.2, 6.7 M sets/s), 12 on LT (1 to 4: 2.8, 5.0, 7.0, 7.9 M sets/s;
    # 6: 11.3-11.8 M; 8: 13.3 M; 10: 13.2 M; 12: 13.1-14.9 M, on 16 host
    # threads).
    "ic24": dict(name="imm_ic_rmat24_deg32_wc_k100_eps0.13", scale=24, draws=32 << 24,
                 model="IC", k=100, eps=0.13, weights="wc", clients=3),
    "lt20": dict(name="imm_lt_rmat20_deg16_k50_eps0.3", scale=20, draws=16 << 20, model="LT",
                 k=50, eps=0.3, weights="lt_normalized", clients=12),
    "ic14": dict(name="imm_ic_rmat14_2^18_k20_eps0.5", scale=14, draws=1 << 18, model="IC",
                 k=20, eps=0.5, weights="uniform_0_0.1"),
    # 64 IMM instances over 16 graphs (ER + R-MAT, 2^12..2^22 vertices, average
    # degree 4..64; half IC p ~ U(0,0.05), half LT normalised), k ~ U[10,200],
    # eps ~ U[0.1,0.5], generator seed 2: batched (one continuous batch, one
    # sampling launch per round) against one plain IMM at a time
    "b1": dict(name="batch_64_imm_16_graphs", kind="batch"),
    # request loop: resident R-MAT graphs 2^18..2^24 (degree 16) with IC
    # p ~ U(0,0.1) and LT normalised weights, Poisson arrivals at 200 req/s
    # (seed 3), k log-uniform in [5,500], eps in {0.5,0.3,0.13}, IC/LT 50/50
    "s1": dict(name="serve_rmat18-24_poisson200", kind="serve"),
    # R-MAT 2^24, 32*2^24 draws, weighted cascade p = 1/indeg, k=100,
    # eps=0.13: full IMM with the autotuned sampler, plus each sampler
    # (one set per warp, fused 64/128/256 colours) on the same fixed set range
    "ic24_samplers": dict(name="samplers_ic_rmat24_deg32_wc", kind="p3", scale=24,
                          draws=32 << 24, model="IC", k=100, eps=0.13, weights="wc",
                          sets=1 << 18),
    # the serving workload's 2^24 IC graph (degree 16, p ~ U(0, 0.1)): a
    # supercritical reverse BFS, sets large and overlapping
    "ic24u_samplers": dict(name="samplers_ic_rmat24_deg16_u0.1", kind="p3", scale=24,
                           draws=16 << 24, model="IC", k=100, eps=0.13,
                           weights="uniform_0_0.1", sets=1 << 12),
    # forward Monte Carlo spread (rip_spread_ic) of the 50 vertices of largest
    # out-degree on R-MAT 2^20 (16*2^20 draws, IC p ~ U(0,0.1)), 20000
    # replicas a step; the reference's own simulator timed beside it
    # one IMM per step with its sets split across the ranks (and --shards
    # pools per rank), counts combined across them at every pick; lowest-id
    # picks, so each step's answer is the single-pool one (strong scaling)
    "ic24_sharded": dict(name="imm_sharded_ic_rmat24_deg32_wc_k100_eps0.13", kind="sharded",
                         scale=24, draws=32 << 24, model="IC", k=100, eps=0.13, weights="wc"),
    "spread": dict(name="spread_ic_rmat20_deg16_k50", kind="spread", scale=20,
                   draws=16 << 20, model="IC", weights="uniform_0_0.1", k=50,
                   replicas=20000),
}
METRIC = "RRR sets/s (full IMM)"


RMAT_ABC = (0.57, 0.19, 0.19)


def workload_config(w, n, m):
    """The `config` object of both arms' lines (identical by construction)."""
    return {"workload": w["name"], "model": w["model"], "k": w["k"], "epsilon": w["eps"],
            "n": n, "m": m, "weights": w["weights"],
            "graph": "R-MAT 2^%d, %d draws, a,b,c = %s, seed 0, no self-loops or duplicates"
                     % (w["scale"], w["draws"], ",".join(str(x) for x in RMAT_ABC)),
            "l2": l2_note(8 * m + 4 * (n + 1))}


def l2_note(graph_bytes):
    """How the timed steps stand to the 126 MB L2 (no flush between steps)."""
    mb = graph_bytes / 1e6
    if mb > 126:
        return "no flush: the graph alone (%.0f MB) exceeds the 126 MB L2" % mb
    return "no flush: the graph (%.1f MB) fits in the 126 MB L2, steps run L2-warm" % mb


def build_graph(w):
    import ripples_b200 as rb
    g = rb.HostGraph.rmat(w["scale"], w["draws"], *RMAT_ABC, seed=0)
    if w["weights"] == "lt_normalized":
        return g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=1)
    if w["weights"] == "wc":
        return g.with_weights(rb.WEIGHTS_WC)
    return g.with_weights(rb.WEIGHTS_UNIFORM, seed=1, lo=0.0, hi=0.1)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
             "--format=csv,noheader,nounits", "-lms", "100"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl"
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return world, rank, local


def _reduce(x, world, op_name):
    """One float reduced over the ranks (NCCL on GPUs, gloo on CPU)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def allreduce_max(x, world):
    return _reduce(x, world, "MAX")


def allreduce_sum(x, world):
    return _reduce(x, world, "SUM")


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def replica_seed(rank, step):
    """Sampler seed of a replica's step: ranks run independent IMM queries."""
    return 1000003 * (rank + 1) + step


def aggregate(sets, elapsed_ms, world):
    """Whole-job throughput of the replicas: every rank's sets over the
    slowest rank's device time."""
    t_max = allreduce_max(elapsed_ms, world)
    return allreduce_sum(sets, world) / (t_max / 1e3), t_max


def run_reference_imm(bin_path, w, threads, parallel, timeout_s):
    """One run of the reference imm tool; returns (sets, total_ms, record)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "imm")
    out = tempfile.mktemp(suffix=".json")
    cmd = [exe, "-i", bin_path, "--reload-binary", "-d", w["model"], "-k", str(w["k"]),
           "-e", str(w["eps"]), "-o", out]
    if parallel:
        cmd.append("-p")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    subprocess.run(cmd, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   timeout=timeout_s, check=True)
    with open(out) as fh:
        rec = json.load(fh)[0]
    os.unlink(out)
    sets = max(int(rec["Theta"]), int(sum(rec["ThetaPrimeDeltas"])))
    return sets, float(rec["Total"]), rec


def oracle_graph(w):
    """The workload's graph drawn by the oracle's generator (tests pin it equal
    to the library's host builder), so the reference arm never loads this
    package's library.  Returns (n, index, src, weights)."""
    from oracle import oracle as O
    kind, lo, hi = {"wc": ("wc", 0.0, 0.0), "lt_normalized": ("lt_normalized", 0.0, 0.0),
                    "uniform_0_0.1": ("uniform", 0.0, 0.1)}[w["weights"]]
    return O.rmat_graph(w["scale"], w["draws"], *RMAT_ABC, seed=0, weights=kind, weight_seed=1,
                        lo=lo, hi=hi)


def reference_sampling(path, steps, warmup, target_s):
    """The reference's `imm -p -d IC --rrsets N` sampling path (tools/imm.cc:
    224-262: GenerateRRRSets over an ICStreamingGenerator with one CPU worker
    per host thread) through the harness built from its sources, the graph
    loaded once.  N is a multiple of 64 sets per thread sized so one call takes
    about target_s.  Returns (N, [ms of each timed call], threads)."""
    import ctypes
    from oracle import oracle as O
    R = O.reference()
    threads = os.cpu_count() or 1
    g = R.ref_graph_load(path.encode())
    try:
        unit = 64 * threads
        ne = ctypes.c_uint64()
        ms = R.ref_generate_parallel(g, unit, 0, ctypes.byref(ne))  # sizing call
        N = max(unit, int(target_s * 1e3 / max(ms, 1e-3)) * unit)
        for i in range(warmup):
            R.ref_generate_parallel(g, N, 1 + i, ctypes.byref(ne))
        times = [R.ref_generate_parallel(g, N, 1000 + i, ctypes.byref(ne)) for i in range(steps)]
    finally:
        R.ref_graph_free(g)
    return N, times, threads


def reference_arm(args, w, world, rank):
    if rank != 0:
        return 0
    from oracle import oracle as O
    exe = os.path.join(ROOT, "oracle", "_ref", "imm")
    if not os.path.exists(exe) or O.reference() is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref not built (make -f oracle/ref.mk needs the "
                          "reference sources)"}))
        return 0
    n, index, src, wts = oracle_graph(w)
    m = len(src)
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "graph.bin")
    O.write_binary(path, n, index, src, wts)
    del index, src, wts
    config = workload_config(w, n, m)
    if w["model"] == "IC":
        # a step: one bounded GenerateRRRSets call, the whole run a few minutes
        per_step = min(5.0, max(1.0, 150.0 / max(1, args.steps + args.warmup)))
        N, times, threads = reference_sampling(path, args.steps, args.warmup, per_step)
        tot_sets, tot_ms = N * len(times), sum(times)
        path_note = ("imm -p --rrsets %d (GenerateRRRSets, ICStreamingGenerator, %d CPU "
                     "workers): sampling only, theta-capped" % (N, threads))
        sample = (f"{args.steps} calls of the reference's parallel GenerateRRRSets, {N} sets "
                  f"each, on all {threads} host threads (graph loaded once)")
    else:
        # The reference's LT sampler is only correct on its sequential path:
        # the parallel CPU workers run IC coin flips whatever the model
        # (include/ripples/batched_add_rrrset.h:231-245).
        threads = 1
        for _ in range(args.warmup):
            run_reference_imm(path, w, threads, False, 600)
        tot_sets, tot_ms = 0, 0.0
        for _ in range(args.steps):
            s_, ms, rec = run_reference_imm(path, w, threads, False, 600)
            tot_sets += s_
            tot_ms += ms
        path_note = "imm (sequential), full IMM runs"
        sample = f"{args.steps} full IMM runs of the workload, sequential imm"
    shutil.rmtree(tmp, ignore_errors=True)
    value = tot_sets / (tot_ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sets/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic R-MAT (seed 0) from the oracle's generator, written in the "
                    "reference binary format",
            "config": config, "reference_path": path_note,
            "cpu_baseline": {"value": value, "unit": "sets/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "sets/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def reference_arm_other(args, w, world, rank):
    """The reference arm of the non-default workloads.  spread: the replica
    loop of the reference's simulator tool (tools/simulator.cc:139-149 over
    ripples::simulate, built from its sources) on all host cores, replicas of
    the same seeds on the same forward graph.
    batch / serve: the reference has no batching or serving path, and p3 (one
    IMM on a 2^24-vertex, 521 M-edge graph) runs for hours on host cores: those
    print an unavailable line."""
    if rank != 0:
        return 0
    kind = w["kind"]
    if kind != "spread":
        why = {"batch": "the reference runs one IMM instance per process (no batching path)",
               "serve": "the reference has no request loop (no serving path)",
               "p3": "this workload compares the library's samplers with one another; the "
                     "reference arm of the 2^24 graph is --workload ic24",
               "sharded": "the reference's sharded IMM is its MPI build (mpi/imm.h), and "
                          "this image has no MPI"}[kind]
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    R = O.reference()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref not built (make -f oracle/ref.mk needs the reference "
                          "sources)"}))
        return 0
    import numpy as np
    g = build_graph(w)
    f = g.forward()
    outdeg = np.diff(f.index).astype(np.int64)
    seeds = np.lexsort((np.arange(g.n), -outdeg))[: w["k"]].astype(np.uint32)
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "fwd.bin")
    g.write_binary(path, backward=False)
    cores = os.cpu_count() or 1
    reps = max(cores * 8, 64)  # a bounded sample: a few seconds of all cores

    def run(r):
        t0 = time.perf_counter()
        mean = R.ref_simulate_parallel(path.encode(), 0 if w["model"] == "IC" else 1,
                                       seeds.ctypes.data, len(seeds), r)
        return time.perf_counter() - t0, mean

    for _ in range(args.warmup):
        run(cores)
    tot_s, means = 0.0, []
    for _ in range(args.steps):
        dt, m = run(reps)
        tot_s += dt
        means.append(m)
    value = reps * args.steps / tot_s
    shutil.rmtree(tmp, ignore_errors=True)
    print(json.dumps({
        "impl": "reference", "metric": "IC spread replicas/s (forward Monte Carlo)",
        "value": value, "unit": "replicas/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
        "higher_is_better": True, "scaling": "replicas only", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic R-MAT graph (seed 0) and weights (seed 1), forward "
                                "binary format",
        "config": {"workload": w["name"], "n": g.n, "m": g.m, "k": w["k"],
                   "replicas_per_step": reps,
                   "reference_path": "simulator's OpenMP replica loop"},
        "mean_spread": float(np.mean(means)),
        "cpu_baseline": {"value": value, "unit": "replicas/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"{args.steps} runs of the simulator's replica loop, "
                                   f"{reps} replicas each, graph load included"},
        "e2e": {"value": value, "unit": "replicas/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))
    return 0


def cpu_baseline(w, g, budget_s=10.0):
    """The reference's own CPU path on this box's host cores, a bounded sample:
    IC -- its parallel sampler (the imm tool's -p --rrsets path) on every host
    thread, about budget_s of work; LT -- one full sequential imm run."""
    from oracle import oracle as O
    exe = os.path.join(ROOT, "oracle", "_ref", "imm")
    if not os.path.exists(exe) or O.reference() is None:
        return None
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "graph.bin")
    g.write_binary(path, backward=True)
    try:
        if w["model"] == "IC":
            N, times, threads = reference_sampling(path, 1, 0, budget_s)
            return {"value": N / (times[0] / 1e3), "unit": "sets/s", "cores": threads,
                    "kind": "reference",
                    "sample": f"{N} sets ({times[0]:.0f} ms) of the reference's parallel "
                              f"GenerateRRRSets (imm -p --rrsets path) on {threads} threads: "
                              f"sampling only"}
        s_, ms, rec = run_reference_imm(path, w, 1, False, max(60, budget_s * 12))
        return {"value": s_ / (ms / 1e3), "unit": "sets/s", "cores": 1, "kind": "reference",
                "sample": f"one full IMM run ({s_} sets, {ms:.0f} ms) with the reference's "
                          f"sequential imm built from its sources"}
    except (subprocess.TimeoutExpired, subprocess.CalledProcessError) as e:
        return {"value": None, "unit": "sets/s", "cores": None, "kind": "reference",
                "sample": f"failed: {type(e).__name__}"}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--clients", type=int, default=0,
                    help="IMM workloads: concurrent client threads of the timed region, "
                         "each with its own context, graph and pool (the K steps are "
                         "split between them); 0 = the workload's default (3 for the "
                         "2^24 IC IMM, 4 for the 2^20 LT one, 1 otherwise)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ic24", choices=sorted(WORKLOADS))
    ap.add_argument("--shards", type=int, default=1,
                    help="ic24_sharded: pools (shards) per process")
    ap.add_argument("--exchange", default="auto", choices=["auto", "sparse", "dense"],
                    help="ic24_sharded: per-pick exchange (decrement lists or whole counts)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-scales", default="18,20,22,24",
                    help="s1: R-MAT scales of the resident graphs")
    ap.add_argument("--serve-queries", type=int, default=64)
    ap.add_argument("--serve-tiebreak", default="lowest_id", choices=["lowest_id", "ref_heap"],
                    help="s1: tie-break of every query, served and plain")
    ap.add_argument("--serve-eps", default="0.5,0.3,0.13")
    ap.add_argument("--serve-max-active", type=int, default=32)
    ap.add_argument("--serve-deadline", type=float, default=600.0,
                    help="s1: seconds after which unfinished queries count as failed")
    ap.add_argument("--baseline-seconds", type=float, default=60.0)
    ap.add_argument("--case-scale", type=int, default=0,
                    help="profiling case of the p3 workload: R-MAT scale (default 24)")
    ap.add_argument("--sampler-case", type=int, default=0,
                    help="profiling case: one sampler launch of this many sets on the "
                         "workload's graph (after a 1024-set pilot launch); prints its "
                         "algorithmic bytes")
    ap.add_argument("--imm-case", action="store_true",
                    help="profiling case: one IMM of the workload (IC graphs autotuned), "
                         "after two warm-up IMMs, alone between cudaProfilerStart and "
                         "cudaProfilerStop (ncu --profile-from-start off)")
    ap.add_argument("--spread-case", type=int, default=0,
                    help="profiling case of the spread workload: one rip_spread_ic call "
                         "of this many replicas after a warm-up call, alone in a "
                         "profiler range")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    world, rank, local = dist_setup()
    if args.impl == "reference" and w.get("kind") in ("batch", "serve", "p3", "spread", "sharded"):
        rc = reference_arm_other(args, w, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc
    if args.sampler_case:
        return run_sampler_case(args, w, local)
    if args.imm_case:
        return run_imm_case(args, w, local)
    if args.spread_case:
        return run_spread_case(args, w, local)
    if w.get("kind") == "batch":
        return run_batch(args, w, world, rank, local)
    if w.get("kind") == "serve":
        return run_serve(args, w, world, rank, local)
    if w.get("kind") == "p3":
        return run_p3(args, w, world, rank, local)
    if w.get("kind") == "spread":
        return run_spread(args, w, world, rank, local)
    if w.get("kind") == "sharded":
        return run_sharded(args, w, world, rank, local)
    if args.impl == "reference":
        rc = reference_arm(args, w, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import numpy as np
    import torch
    import ripples_b200 as rb
    import ctypes

    torch.cuda.set_device(local)
    g = build_graph(w)
    ctx = rb.Context(local)
    sp = ctypes.c_void_p()
    rb._lib.check(rb._lib.lib.rip_ctx_stream(ctx.h, ctypes.byref(sp)), "rip_ctx_stream")
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local))
    dg = rb.DeviceGraph(ctx, g, w["model"])
    tune = dg.autotune(seed=1, pilot=32768) if w["model"] == "IC" else None  # setup, untimed
    pool = rb.Pool(dg)
    seed_base = replica_seed(rank, 0)

    def one_step(step):
        pool.clear()
        seeds, rec = pool.imm(w["k"], w["eps"], 1.0, seed=seed_base + step)
        return rec

    for i in range(args.warmup):
        one_step(-1 - i)
    # Further clients: a context, graph and pool each (same host graph, tuned
    # the same way), so that one query's sampling runs while another's
    # selection waits on the host, as concurrent queries would.
    n_clients = args.clients if args.clients > 0 else w.get("clients", 1)
    extra = []
    for j in range(1, n_clients):
        cx = rb.Context(local)
        dgx = rb.DeviceGraph(cx, g, w["model"])
        if w["model"] == "IC":
            dgx.autotune(seed=1, pilot=32768)
        px = rb.Pool(dgx)
        for i in range(args.warmup):
            px.clear()
            px.imm(w["k"], w["eps"], 1.0, seed=seed_base + 1000 * j - 1 - i)
        extra.append((cx, dgx, px))
    pools = [pool] + [e[2] for e in extra]
    # ---- timed region (device events on the library's stream) --------------
    for px in pools:
        px.clear()
    launches0 = rb._lib.lib.rip_kernel_launches()
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    acc = [dict(sets=0, kern_ms=0.0, kern_n=0, st=np.zeros(8, np.uint64), thetas=[],
                gen_ms=0.0, sel_ms=0.0, sel_prof={}, err=None) for _ in pools]

    def client(j):
        a, px = acc[j], pools[j]
        try:
            for step in range(j, args.steps, n_clients):
                px.clear()
                seeds, rec = px.imm(w["k"], w["eps"], 1.0, seed=seed_base + step)
                a["sets"] += rec.total_sets
                a["thetas"].append(int(rec.theta))
                nr = min(rec.num_rounds, 64)
                a["gen_ms"] += rec.generate_ms + sum(rec.round_generate_ms[i] for i in range(nr))
                a["sel_ms"] += rec.select_ms + sum(rec.round_select_ms[i] for i in range(nr))
                km, kn, _ = px.timing()
                a["kern_ms"] += km
                a["kern_n"] += kn
                a["st"] += px.stats()
                for kk, vv in px.select_profile().items():
                    a["sel_prof"][kk] = a["sel_prof"].get(kk, 0.0) + vv
        except Exception as exc:  # reported after the join
            a["err"] = repr(exc)

    workers = [threading.Thread(target=client, args=(j,)) for j in range(n_clients)]
    for th in workers:
        th.start()
    for th in workers:
        th.join()
    torch.cuda.synchronize()  # every client's stream is done before ev1
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    errs = [a["err"] for a in acc if a["err"]]
    if errs:
        raise RuntimeError("timed clients: " + "; ".join(errs))
    launches = int(rb._lib.lib.rip_kernel_launches() - launches0)
    elapsed_ms = ev0.elapsed_time(ev1)
    total_sets = sum(a["sets"] for a in acc)
    kern_ms = sum(a["kern_ms"] for a in acc)
    kern_n = sum(a["kern_n"] for a in acc)
    st_tot = sum((a["st"] for a in acc), np.zeros(8, np.uint64))
    thetas = [t for a in acc for t in a["thetas"]]
    gen_ms = sum(a["gen_ms"] for a in acc)
    sel_ms = sum(a["sel_ms"] for a in acc)
    sel_prof = {}
    for a in acc:
        for kk, vv in a["sel_prof"].items():
            sel_prof[kk] = sel_prof.get(kk, 0.0) + vv
    value, t_max = aggregate(total_sets, elapsed_ms, world)
    for cx, dgx, px in extra:
        px.close()
        dgx.close()
        cx.close()

    # ---- one client alone (each IMM's own latency) -------------------------
    torch.cuda.synchronize()
    ev4, ev5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    one_steps = max(1, min(args.steps, 5))
    ev4.record(stream)
    one_sets, one_kern_ms, one_kern_n, one_st = 0, 0.0, 0, np.zeros(8, np.uint64)
    for step in range(one_steps):
        pool.clear()
        _, rec = pool.imm(w["k"], w["eps"], 1.0, seed=seed_base + step)
        one_sets += rec.total_sets
        km, kn, _ = pool.timing()
        one_kern_ms += km
        one_kern_n += kn
        one_st += pool.stats()
    ev5.record(stream)
    torch.cuda.synchronize()
    one_ms = allreduce_max(ev4.elapsed_time(ev5), world)
    one_value = allreduce_sum(one_sets, world) / (one_ms / 1e3)

    # ---- the same IMM runs with the reference GPU path's tie-break ---------
    # (lowest vertex id among equal counts, thrust::max_element): every pick
    # stays on the device, one read-back per selection
    torch.cuda.synchronize()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    low_steps = max(1, min(args.steps, 5))
    ev2.record(stream)
    low_sets = 0
    for step in range(low_steps):
        pool.clear()
        _, rec = pool.imm(w["k"], w["eps"], 1.0, seed=seed_base + step,
                          tiebreak=rb.TIE_LOWEST_ID)
        low_sets += rec.total_sets
    ev3.record(stream)
    torch.cuda.synchronize()
    low_ms = allreduce_max(ev2.elapsed_time(ev3), world)
    low_value = allreduce_sum(low_sets, world) / (low_ms / 1e3)
    low_ms_per_step = low_ms / low_steps

    # ---- the IC samplers with and without per-vertex uniform thresholds ----
    # (the same sets either way; untimed by the headline)
    uniform_cmp = None
    if w["model"] == "IC" and dg.uniform_thresholds():
        uniform_cmp = {}
        for label, on in (("on", True), ("off", False)):
            dg.uniform_thresholds(on)
            p2 = rb.Pool(dg)
            p2.sample(1 << 14, seed=77)
            p2.clear()
            torch.cuda.synchronize()
            t_u = time.perf_counter()
            p2.sample(1 << 18, seed=77)
            torch.cuda.synchronize()
            t_u = time.perf_counter() - t_u
            km_u, _, _ = p2.timing()
            st_u = p2.stats()
            uniform_cmp[label] = {"sets_per_s": (1 << 18) / t_u, "kernel_ms": km_u,
                                  "alg_gb_per_s": alg_bytes_of(st_u, on) / (km_u / 1e3) / 1e9}
            p2.close()
        dg.uniform_thresholds(True)

    # ---- e2e through the public API: host graph -> device -> seeds ---------
    pin_idx = torch.from_numpy(g.index).pin_memory()
    pin_src = torch.from_numpy(g.src).pin_memory()
    pin_w = torch.from_numpy(g.weights).pin_memory()
    h2d = pin_idx.numel() * 8 + pin_src.numel() * 4 + pin_w.numel() * 4
    d2h = 4 * w["k"]

    e2e_split = {"upload_ms": 0.0, "imm_ms": 0.0}
    e2e_step_ms = []

    def e2e_step(step):
        t0 = time.perf_counter()
        gen_g = rb.HostGraph(g.n, pin_idx.numpy(), pin_src.numpy(), pin_w.numpy())
        gen = rb.B200RRRGenerator(gen_g, w["model"], seed=seed_base + 7919 + step, ctx=ctx)
        t1 = time.perf_counter()
        CFG = rb.IMMConfiguration(k=w["k"], epsilon=w["eps"], diffusionModel=w["model"])
        rec = rb.IMMExecutionRecord()
        seeds = rb.IMM(gen_g, CFG, 1.0, gen, rec)
        n_sets = rec.TotalSets
        gen.pool.close()
        gen.graph.close()
        t2 = time.perf_counter()
        e2e_split["upload_ms"] += 1e3 * (t1 - t0)
        e2e_split["imm_ms"] += 1e3 * (t2 - t1)
        e2e_step_ms.append(round(1e3 * (t2 - t0), 2))
        return n_sets, seeds

    e2e_steps = max(1, min(args.steps, 5 if g.m > (1 << 28) else 10))
    e2e_step(-1)
    e2e_split.update(upload_ms=0.0, imm_ms=0.0)
    e2e_step_ms.clear()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_sets = 0
    for step in range(e2e_steps):
        s, _ = e2e_step(step)
        e2e_sets += s
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    e2e_serial = allreduce_sum(e2e_sets, world) / (allreduce_max(e2e_ms, world) / 1e3)

    # The same steps from concurrent clients, each with its own context: one
    # more than the timed region's (at any time about one client is copying
    # its graph in rather than running an IMM), so a step's upload crosses
    # the bus while other steps' IMMs run on the GPU, as concurrent queries
    # of a serving client would; four steps a client, so that the pipeline's
    # fill and drain do not dominate.  Every step still copies its graph in
    # and its seeds out.
    n_pipe = n_clients + 1
    pipe_ctx = [rb.Context(local) for _ in range(n_pipe)]
    pipe_sets, pipe_err = [0] * n_pipe, []

    def pipe_worker(j):
        try:
            for step in range(j, e2e_pipe_steps, n_pipe):
                gen_g = rb.HostGraph(g.n, pin_idx.numpy(), pin_src.numpy(), pin_w.numpy())
                gen = rb.B200RRRGenerator(gen_g, w["model"], seed=seed_base + 7919 + step,
                                          ctx=pipe_ctx[j])
                CFG = rb.IMMConfiguration(k=w["k"], epsilon=w["eps"], diffusionModel=w["model"])
                rec = rb.IMMExecutionRecord()
                rb.IMM(gen_g, CFG, 1.0, gen, rec)
                pipe_sets[j] += rec.TotalSets
                gen.pool.close()
                gen.graph.close()
        except Exception as exc:  # reported after the join
            pipe_err.append(repr(exc))

    e2e_pipe_steps = max(e2e_steps, 4 * n_pipe)
    for j in range(n_pipe):  # each context's buffers sized once, untimed
        warm_g = rb.HostGraph(g.n, pin_idx.numpy(), pin_src.numpy(), pin_w.numpy())
        warm = rb.B200RRRGenerator(warm_g, w["model"], seed=seed_base + 7, ctx=pipe_ctx[j])
        rb.IMM(warm_g, rb.IMMConfiguration(k=w["k"], epsilon=w["eps"], diffusionModel=w["model"]),
               1.0, warm, rb.IMMExecutionRecord())
        warm.pool.close()
        warm.graph.close()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    threads = [threading.Thread(target=pipe_worker, args=(j,)) for j in range(n_pipe)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    torch.cuda.synchronize()
    pipe_ms = (time.perf_counter() - t0) * 1e3
    if pipe_err:
        raise RuntimeError("pipelined e2e: " + "; ".join(pipe_err))
    e2e_value = allreduce_sum(sum(pipe_sets), world) / (allreduce_max(pipe_ms, world) / 1e3)
    for cx in pipe_ctx:
        cx.close()

    # ---- roofline of the dominant kernel (the sampler) ----------------------
    # Algorithmic bytes: 8 B per vertex expansion (two u32 CSR offsets), 8 B
    # per in-edge record read (u32 source + u32 threshold), 4 B per pool
    # element written, 8 + 4 B per set (pool offset + length).
    vthr = bool(dg.uniform_thresholds()) if w["model"] == "IC" else False
    alg_bytes = alg_bytes_of(st_tot, vthr)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else None
    # the same kernels with no other query's launches beside them
    one_alg = alg_bytes_of(one_st, vthr)
    one_achieved = one_alg / (one_kern_ms / 1e3) / 1e9 if one_kern_ms > 0 else None
    kernel = ("lt_walk_kernel" if w["model"] == "LT" else
              "ic_fused_kernel" if tune and tune["name"].startswith("fused") else
              "ic_plain_kernel + ic_bigset_kernel (every IC sampler launch)")
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        with open(prof) as fh:
            tr = json.load(fh).get(w["name"])
        if tr and kern_n:
            # DRAM bytes per algorithmic byte from the ncu capture, applied to
            # this run's average launch
            traffic = tr["dram_bytes_per_alg_byte"] * alg_bytes / kern_n

    coin_roofline = None
    if w["model"] == "IC" and kern_ms > 0:
        coin_peak = ctx.coin_rate()
        coins = int(st_tot[5]) / (kern_ms / 1e3)
        coin_roofline = {"bound": "coin arithmetic (Philox4x32-10, integer issue)",
                         "kernel": kernel, "achieved": coins, "peak": coin_peak,
                         "peak_kind": "measured (coin-only kernel, same run)",
                         "unit": "coins/s", "frac": coins / coin_peak if coin_peak else None}
        if one_kern_ms > 0:
            one_coins = int(one_st[5]) / (one_kern_ms / 1e3)
            coin_roofline["one_client"] = {
                "achieved": one_coins, "frac": one_coins / coin_peak if coin_peak else None,
                "note": "the one-client steps: no other query's launches beside the kernel"}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(w, g)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "sets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32",
            "data": "synthetic R-MAT graph (seed 0) and weights (seed 1); fresh sampler seed per step",
            "config": workload_config(w, g.n, g.m),
            "theta": thetas[0] if thetas else None,
            "parallelism": f"replicas x{world}",
            "e2e": {"value": e2e_value, "unit": "sets/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_pipe_steps,
                    "clients": n_pipe,
                    "note": "concurrent client threads (one more than the timed region's), "
                            "one context each: a step's upload overlaps other steps' IMMs",
                    "ms_per_step": pipe_ms / e2e_pipe_steps,
                    "serial": {"value": e2e_serial, "note": "one client: upload, then IMM",
                               "split_ms_per_step": {kk: vv / e2e_steps
                                                     for kk, vv in e2e_split.items()},
                               "step_ms": e2e_step_ms}},
            "roofline": {"bound": "hbm", "kernel": kernel,
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes / max(kern_n, 1),
                         "launches": kern_n, "kernel_ms": kern_ms,
                         "one_client": {"achieved": one_achieved,
                                        "frac": (one_achieved / peak) if one_achieved else None,
                                        "launches": one_kern_n, "kernel_ms": one_kern_ms,
                                        "note": "the one-client steps: no other query's "
                                                "launches beside the kernel"}},
            # sum over sets of the in-degrees of their members (per-set
            # semantics, fused expansions counted per colour) over the
            # sampler kernels' time
            "traversed_edges_per_s": int(st_tot[5]) / (kern_ms / 1e3) if kern_ms > 0 else None,
            # IC samplers draw one coin per in-edge of every member; on
            # uniform-threshold graphs they read almost nothing else, so the
            # ceiling is the coin function's own rate on this GPU, measured
            # here by a coin-only kernel at full occupancy (rip_coin_rate)
            "compute_roofline": coin_roofline,
            "cpu_baseline": base,
            "clocks": clk,
            "gpu_launches": launches,
            "imm_ms_per_step": t_max / args.steps,
            "host_split_ms_per_step": {"generate": gen_ms / args.steps,
                                       "select": sel_ms / args.steps},
            "select_profile_per_step": {kk: vv / args.steps for kk, vv in sel_prof.items()},
            "sets_per_step": total_sets / args.steps,
            "autotune": tune,
            "uniform_thresholds_2^18_sets": uniform_cmp,
            "branching": dg.branching if w["model"] == "IC" else None,
            "tiebreak": "reference CPU heap (CompareHeap lazy max-heap)",
            "clients": n_clients,
            "one_client": {"value": one_value, "unit": "sets/s", "ms_per_step": one_ms / one_steps,
                           "steps": one_steps,
                           "note": "the same IMMs one after another from one client"},
            "lowest_id_tiebreak": {"value": low_value, "unit": "sets/s",
                                   "ms_per_step": low_ms_per_step, "steps": low_steps,
                                   "note": "same IMM runs, reference GPU tie-break "
                                           "(lowest id), picks on the device"},
        }
        print(json.dumps(line))
    pool.close()
    dg.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def alg_bytes_of(st, vthr=False):
    """Algorithmic bytes of the sampler work in a pool's counters: 8 B per
    vertex expansion (two CSR offsets), 8 B per in-edge record read (source +
    threshold), 4 B per stored element, 12 B per stored set (offset + length).
    With per-vertex uniform thresholds (vthr) an expansion also reads its
    vertex's threshold (4 B), the records of uniform in-lists are not read
    (counter 6) and only their live edges' sources are (4 B each, counter 7)."""
    return (8 * int(st[0]) + 8 * (int(st[1]) - int(st[6])) + 4 * int(st[7]) +
            4 * int(st[3]) + 12 * int(st[2]) + (4 * int(st[0]) if vthr else 0))


def run_sampler_case(args, w, local):
    import torch
    import ripples_b200 as rb
    torch.cuda.set_device(local)
    ctx = rb.Context(local)
    if w.get("scale") == 24:
        # the 2^24 graphs, built on the device (smaller with --case-scale, same
        # draws per vertex)
        scale = args.case_scale or w["scale"]
        draws = w["draws"] >> (w["scale"] - scale)
        if w["weights"] == "wc":
            dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_WC, seed=0)
        else:
            dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_UNIFORM,
                                               seed=0, weight_seed=1, lo=0.0, hi=0.1)
    else:
        dg = rb.DeviceGraph(ctx, build_graph(w), w["model"])
    pool = rb.Pool(dg)
    pool.sample(1024, seed=5)
    ctx.sync()
    st0 = pool.stats()
    km0, _, _ = pool.timing()
    pool.sample(args.sampler_case, seed=5)
    ctx.sync()
    st = pool.stats() - st0
    km, _, _ = pool.timing()
    alg = alg_bytes_of(st, w["model"] == "IC" and dg.uniform_thresholds())
    print(json.dumps({"case": w["name"], "n": dg.n, "m": dg.m, "sets": args.sampler_case,
                      "alg_bytes": alg,
                      "kernel_ms": km - km0, "gb_per_s": alg / ((km - km0) / 1e3) / 1e9,
                      "stats": [int(x) for x in st]}))
    pool.close()
    dg.close()
    ctx.close()
    return 0


def case_graph(args, w, ctx):
    """The workload's graph for a profiling case: the 2^24 graphs built on the
    device (smaller with --case-scale, same draws per vertex), others as the
    bench builds them."""
    import ripples_b200 as rb
    if w.get("scale") == 24:
        scale = args.case_scale or w["scale"]
        draws = w["draws"] >> (w["scale"] - scale)
        if w["weights"] == "wc":
            return rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_WC, seed=0)
        return rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_UNIFORM,
                                             seed=0, weight_seed=1, lo=0.0, hi=0.1)
    return rb.DeviceGraph(ctx, build_graph(w), w["model"])


def run_imm_case(args, w, local):
    import torch
    import ripples_b200 as rb
    torch.cuda.set_device(local)
    ctx = rb.Context(local)
    dg = case_graph(args, w, ctx)
    tune = dg.autotune(seed=1, pilot=32768) if w["model"] == "IC" else None
    pool = rb.Pool(dg)
    for s in range(2):
        pool.clear()
        pool.imm(w["k"], w["eps"], 1.0, seed=100 + s)
    pool.clear()
    ctx.sync()
    torch.cuda.profiler.start()
    t0 = time.perf_counter()
    seeds, rec = pool.imm(w["k"], w["eps"], 1.0, seed=7)
    ctx.sync()
    ms = (time.perf_counter() - t0) * 1e3
    torch.cuda.profiler.stop()
    print(json.dumps({"case": w["name"], "imm_ms": ms, "theta": int(rec.theta),
                      "tuned": tune["name"] if tune else None,
                      "select_profile": pool.select_profile()}))
    pool.close()
    dg.close()
    ctx.close()
    return 0


def run_spread_case(args, w, local):
    import numpy as np
    import torch
    import ripples_b200 as rb
    torch.cuda.set_device(local)
    g = build_graph(w)
    f = g.forward()
    ctx = rb.Context(local)
    dg = rb.DeviceGraph(ctx, f, "IC")
    outdeg = np.diff(f.index).astype(np.int64)
    seeds = np.lexsort((np.arange(g.n), -outdeg))[: w["k"]].astype(np.uint32)
    rb.spread_ic(dg, seeds, args.spread_case, seed=1)
    ctx.sync()
    torch.cuda.profiler.start()
    t0 = time.perf_counter()
    mean = rb.spread_ic(dg, seeds, args.spread_case, seed=2)
    ctx.sync()
    ms = (time.perf_counter() - t0) * 1e3
    torch.cuda.profiler.stop()
    print(json.dumps({"case": w["name"], "replicas": args.spread_case, "ms": ms,
                      "mean_spread": float(mean)}))
    dg.close()
    ctx.close()
    return 0


def _pct(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if xs else None


def _not_on_rank0(world, rank, args, w):
    """Batch and serve workloads run on rank 0 only (one GPU each: the path
    does not shard); the other ranks exit without work."""
    return rank != 0


def run_batch(args, w, world, rank, local):
    import numpy as np
    import torch
    import ripples_b200 as rb
    if _not_on_rank0(world, rank, args, w):
        return 0
    torch.cuda.set_device(local)
    rng = np.random.default_rng(2)
    ctx = rb.Context(local)
    graphs = []
    for i in range(16):
        scale = int(rng.integers(12, 23))
        deg = int(rng.choice([4, 8, 16, 32, 64]))
        kind = "er" if i % 2 else "rmat"
        model = "IC" if (i // 2) % 2 == 0 else "LT"
        wk = rb.WEIGHTS_UNIFORM if model == "IC" else rb.WEIGHTS_LT_NORMALIZED
        if kind == "rmat":
            dg = rb.DeviceGraph.rmat_on_device(ctx, scale, deg << scale, model, wk, seed=i,
                                               weight_seed=100 + i, lo=0.0, hi=0.05)
        else:
            dg = rb.DeviceGraph.erdos_renyi_on_device(ctx, 1 << scale, deg << scale, model, wk,
                                                      seed=i, weight_seed=100 + i, lo=0.0,
                                                      hi=0.05)
        graphs.append(dict(dg=dg, scale=scale, deg=deg, kind=kind, model=model, m=dg.m))
    t_tune = time.perf_counter()
    for gd in graphs:
        gd["tuned"] = gd["dg"].autotune(seed=1, pilot=1024)["name"]
    t_tune = time.perf_counter() - t_tune
    inst = []
    for j in range(64):
        gi = int(rng.integers(0, 16))
        inst.append(dict(g=gi, k=int(rng.integers(10, 201)), eps=float(rng.uniform(0.1, 0.5)),
                         seed=10_000 + j))

    server_stats = {}

    def batched(tag):
        """All instances as one continuous batch (what rip_imm_batch runs),
        through the server API so its phase timing can be reported."""
        qs = [rb.Query(graphs[x["g"]]["dg"], x["k"], x["eps"], seed=x["seed"] + tag)
              for x in inst]
        srv = rb.Server(ctx, max_active=len(qs))
        for q in qs:
            srv.submit(q)
        srv.drain()
        server_stats.update(srv.stats())
        srv.close()
        return qs

    def plain(tag, limit_s=None):
        """One instance at a time through rip_imm_pool: a fresh pool and the
        same (autotuned) samplers as the batch, no multi-instance launch, no
        shared rounds.  An instance whose pool does not fit the device fails
        here as it does in the batch."""
        out, t0 = [], time.perf_counter()
        for x in inst:
            p = rb.Pool(graphs[x["g"]]["dg"])
            ti = time.perf_counter()
            try:
                seeds, rec = p.imm(x["k"], x["eps"], seed=x["seed"] + tag,
                                   tiebreak=rb.TIE_LOWEST_ID, sampler=rb.SAMPLER_PLAIN)
                out.append((seeds, rec.total_sets, 1e3 * (time.perf_counter() - ti)))
            except rb.RipError:
                out.append((None, 0, 1e3 * (time.perf_counter() - ti)))
            p.close()
            if limit_s and time.perf_counter() - t0 > limit_s:
                break
        return out

    for i in range(args.warmup):
        batched(1_000_000 * (i + 1))
    launches0 = rb._lib.lib.rip_kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sets = 0
    last = None
    failed = 0
    for s in range(args.steps):
        last = batched(0 if s == 0 else 7 * s)
        sets += sum(q.record.total_sets for q in last if q.status == 0)
        failed += sum(1 for q in last if q.status != 0)
    torch.cuda.synchronize()
    t_b = time.perf_counter() - t0
    clk = clocks.stop()
    launches = int(rb._lib.lib.rip_kernel_launches() - launches0)
    # plain one-instance-at-a-time path on the same instances (step 0 seeds)
    plain(12345, limit_s=5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pl = plain(0)
    torch.cuda.synchronize()
    t_p = time.perf_counter() - t0
    first = batched(0)
    same = all(np.array_equal(a[0], q.seeds) for a, q in zip(pl, first)
               if a[0] is not None and q.status == 0)
    for j, q in enumerate(first):  # per-instance account on stderr
        x, gd, r = inst[j], graphs[inst[j]["g"]], q.record
        nr = min(r.num_rounds, 64)
        gen = r.generate_ms + sum(r.round_generate_ms[i] for i in range(nr))
        sel = r.select_ms + sum(r.round_select_ms[i] for i in range(nr))
        pms = f"{pl[j][2]:.0f}" if j < len(pl) else "-"
        print(f"instance {j} ({gd['scale']} {gd['kind']} deg {gd['deg']} {gd['model']} "
              f"k={x['k']} eps={x['eps']:.2f}): status {q.status} theta {r.theta} "
              f"elements {r.pool_elements} rounds {r.num_rounds} batched {r.total_ms:.0f} ms "
              f"(generate {gen:.0f} select {sel:.0f}) plain {pms} ms", file=sys.stderr)
    p_failed = sum(1 for a in pl if a[0] is None)
    p_sets = sum(x[1] for x in pl)
    line = {"metric": "RRR sets/s (64 batched IMM instances)", "value": sets / t_b,
            "unit": "sets/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_b / args.steps, "higher_is_better": True,
            "scaling": "replicas only", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic ER/R-MAT graphs and weights (generator seed 2)",
            "config": {"workload": w["name"], "instances": 64,
                       "graphs": [{k: v for k, v in g.items() if k != "dg"} for g in graphs],
                       "tiebreak": "lowest id (device picks)"},
            "failed_instances_per_step": failed / max(args.steps, 1),
            "server_last_step": dict(server_stats),
            "autotune_s": t_tune,
            "plain_one_at_a_time": {"value": p_sets / t_p, "unit": "sets/s",
                                    "instances": len(pl), "failed": p_failed,
                                    "seconds": t_p, "imm_per_s": len(pl) / t_p},
            "batched_imm_per_s": 64 * args.steps / t_b,
            "speedup_vs_plain": (sets / t_b) / (p_sets / t_p),
            "same_seeds_as_plain": bool(same),
            "e2e": {"value": sets / t_b, "unit": "sets/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(sum(4 * x["k"] for x in inst)),
                    "note": "queries and seeds cross the host boundary; graphs resident"},
            "clocks": clk, "gpu_launches": launches}
    print(json.dumps(line))
    ctx.close()
    return 0


def run_p3(args, w, world, rank, local):
    """Each IC sampler on one fixed range of sets of a 2^24-vertex R-MAT graph
    (identical sets whatever the sampler): one set per warp with heavy sets
    one CTA each, the same with heavy sets grown by the grid-wide multi-colour
    BFS, and the fused multi-colour BFS at 64/128/256 colours."""
    import numpy as np
    import torch
    import ripples_b200 as rb
    if _not_on_rank0(world, rank, args, w):
        return 0
    torch.cuda.set_device(local)
    ctx = rb.Context(local)
    t0 = time.perf_counter()
    scale = args.case_scale or w["scale"]
    draws = w["draws"] >> (w["scale"] - scale)
    if w["weights"] == "wc":
        dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_WC, seed=0)
    else:
        dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_UNIFORM, seed=0,
                                           weight_seed=1, lo=0.0, hi=0.1)
    t_build = time.perf_counter() - t0
    peak, peak_kind = measured_peaks()
    count = w["sets"]
    samplers = {}
    clocks = ClockSampler(local)
    clocks.start()
    for name, smp, colors, heavy in [("plain, heavy sets one CTA each", rb.SAMPLER_PLAIN, 64, 0),
                                     ("plain, heavy sets grid-wide BFS", rb.SAMPLER_PLAIN, 64, 32),
                                     ("fused64", rb.SAMPLER_FUSED, 64, 32),
                                     ("fused128", rb.SAMPLER_FUSED, 128, 32),
                                     ("fused256", rb.SAMPLER_FUSED, 256, 32)]:
        p = rb.Pool(dg)
        p.configure(colors=colors)
        p.heavy_batch(heavy)
        p.sample(max(256, count // 16), seed=7, sampler=smp)  # warm-up: scratch, pool sizing
        p.clear()
        ctx.sync()
        t1 = time.perf_counter()
        p.sample(count, seed=7, sampler=smp)
        ctx.sync()
        dt = time.perf_counter() - t1
        st = p.stats()
        km, kn, _ = p.timing()
        alg = alg_bytes_of(st, bool(dg.uniform_thresholds()))
        samplers[name] = {"sets_per_s": count / dt, "kernel_ms": km, "launches": kn,
                          "alg_gb_per_s": alg / (km / 1e3) / 1e9 if km else None,
                          "frac_of_hbm": (alg / (km / 1e3) / 1e9) / peak if km else None,
                          "fusion_ratio": (int(st[4]) / int(st[0])) if st[0] else None,
                          "traversed_edges_per_s": int(st[5]) / (km / 1e3) if km else None,
                          "mean_set": int(st[3]) / count}
        p.close()
    clk = clocks.stop()
    plain = samplers["plain, heavy sets one CTA each"]["sets_per_s"]
    line = {"metric": "RRR sets/s (one sampler launch series)", "value": plain,
            "unit": "sets/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "higher_is_better": True, "scaling": "replicas only", "vs_baseline": None,
            "dtype": "u32",
            "data": "synthetic R-MAT graph (seed 0), " + ("weighted cascade" if w["weights"] == "wc"
                                                          else "IC p ~ U(0, 0.1) (seed 1)"),
            "config": {"workload": w["name"], "n": dg.n, "m": dg.m, "sets": count,
                       "branching": dg.branching,
                       "uniform_thresholds": bool(dg.uniform_thresholds())},
            "graph_build_s": t_build, "samplers": samplers,
            "best_vs_plain": {k: v["sets_per_s"] / plain for k, v in samplers.items()},
            "clocks": clk}
    print(json.dumps(line))
    ctx.close()
    return 0


def run_sharded(args, w, world, rank, local):
    """One IMM per step on the 2^24 weighted-cascade graph with its sets split
    across every rank's --shards pools (ripples_b200.sharded): each rank
    samples its id ranges; the counts are summed once per selection (in
    process, then NCCL all_reduce) and after each pick the shards exchange
    their decrement lists (all_gather; --exchange sparse) or sum their whole
    counts again (--exchange dense).  Whole-job sets/s of one IMM (strong scaling), timed on
    the device from a synchronised start to a synchronised end, max over
    ranks; at one GPU the single-pool IMM under the same (lowest-id)
    tie-break is timed beside it."""
    import torch
    import ripples_b200 as rb
    from ripples_b200.sharded import DeviceShard, imm_sharded
    torch.cuda.set_device(local)
    group = None
    if world > 1:
        import torch.distributed as dist
        group = dist.group.WORLD
    ctx = rb.Context(local)
    scale = args.case_scale or w["scale"]
    draws = w["draws"] >> (w["scale"] - scale)
    dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_WC, seed=0)
    shards = [DeviceShard(rb.Pool(dg)) for _ in range(max(1, args.shards))]

    def one(step):
        for s in shards:
            s.pool.clear()
        return imm_sharded(shards, w["k"], w["eps"], 1.0, seed=step, group=group,
                           exchange=args.exchange)

    for i in range(args.warmup):
        one(1000 + i)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    sets = 0
    recs = []
    for i in range(args.steps):
        _, rec = one(i)
        sets += rec["total_sets"]
        recs.append(rec)
    torch.cuda.synchronize()
    ev1.record()
    ev1.synchronize()
    clk = clocks.stop()
    ms = allreduce_max(ev0.elapsed_time(ev1), world)
    single = None
    if world == 1:
        p1 = rb.Pool(dg)
        p1.imm(w["k"], w["eps"], 1.0, seed=1000, tiebreak=rb.TIE_LOWEST_ID)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s1 = 0
        for i in range(args.steps):
            p1.clear()
            _, r1 = p1.imm(w["k"], w["eps"], 1.0, seed=i, tiebreak=rb.TIE_LOWEST_ID)
            s1 += r1.total_sets
        torch.cuda.synchronize()
        single = {"sets_per_s": s1 / (time.perf_counter() - t0),
                  "note": "rip_imm_pool, lowest-id tie-break, same seeds (host clock)"}
        p1.close()
    if rank == 0:
        picks = sum(r["picks"] for r in recs)
        line = {"metric": METRIC, "value": sets / (ms / 1e3), "unit": "sets/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic R-MAT graph (seed 0), weighted cascade",
                "config": {"workload": w["name"], "n": dg.n, "m": dg.m, "k": w["k"],
                           "epsilon": w["eps"], "shards_per_rank": len(shards),
                           "shards": world * len(shards), "tiebreak": "lowest_id",
                           "exchange": recs[0]["exchange"] if recs else args.exchange,
                           "l2": l2_note(8 * dg.m + 4 * (dg.n + 1))},
                "sets_per_step": sets / args.steps,
                "picks_per_step": picks / args.steps,
                "select_ms_per_step": sum(sum(r["round_select_ms"]) + r["select_ms"]
                                          for r in recs) / args.steps,
                "collective_ms_per_step": sum(r["allreduce_ms"] for r in recs) / args.steps,
                "exchanged_per_step": sum(r["exchanged"] for r in recs) / args.steps,
                "single_pool": single, "clocks": clk}
        print(json.dumps(line))
    for s in shards:
        s.pool.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_spread(args, w, world, rank, local):
    import ctypes
    import numpy as np
    import torch
    import ripples_b200 as rb
    if _not_on_rank0(world, rank, args, w):
        return 0
    torch.cuda.set_device(local)
    g = build_graph(w)
    f = g.forward()
    ctx = rb.Context(local)
    sp = ctypes.c_void_p()
    rb._lib.check(rb._lib.lib.rip_ctx_stream(ctx.h, ctypes.byref(sp)), "rip_ctx_stream")
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local))
    dg = rb.DeviceGraph(ctx, f, "IC")
    outdeg = np.diff(f.index).astype(np.int64)
    seeds = np.lexsort((np.arange(g.n), -outdeg))[: w["k"]].astype(np.uint32)
    R = w["replicas"]
    for i in range(args.warmup):
        rb.spread_ic(dg, seeds, R // 10, seed=1000 + i)
    launches0 = rb._lib.lib.rip_kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    means, dev_ms, wall = [], 0.0, 0.0
    for step in range(args.steps):
        t0 = time.perf_counter()
        ev0.record(stream)
        means.append(rb.spread_ic(dg, seeds, R, seed=step))
        ev1.record(stream)
        ev1.synchronize()
        wall += time.perf_counter() - t0
        dev_ms += ev0.elapsed_time(ev1)
    clk = clocks.stop()
    launches = int(rb._lib.lib.rip_kernel_launches() - launches0)
    # algorithmic bytes of one replica: 8 (two offsets) + 8 per out-edge
    # record of every reached vertex.  The oracle reproduces replicas 0..7 of
    # step 0 bit for bit, and their reached vertices' out-edges give the mean.
    from oracle import oracle as O
    thr = O.pack("IC", f.index, f.weights)
    sample_reps = 8
    s_mean, _, s_edges = O.spread_ic(f.n, f.index, f.src, thr, seeds, sample_reps, seed=0,
                                     with_edges=True)
    alg_per_replica = 8.0 * s_mean + 8.0 * s_edges / sample_reps
    mean = float(np.mean(means))
    value = R * args.steps / (dev_ms / 1e3)
    peak, peak_kind = measured_peaks()
    # the reference's simulator (ripples::simulate) on one host core, a
    # bounded sample of replicas
    cpu = None
    if O.reference() is not None:
        tmpd = tempfile.mkdtemp()
        path = os.path.join(tmpd, "fwd.bin")
        g.write_binary(path, backward=False)
        reps_cpu = 20
        t0 = time.perf_counter()
        ref_mean = O.reference().ref_simulate(path.encode(), 0, seeds.ctypes.data, len(seeds),
                                              reps_cpu, 0)
        t_cpu = time.perf_counter() - t0
        shutil.rmtree(tmpd, ignore_errors=True)
        cpu = {"value": reps_cpu / t_cpu, "unit": "replicas/s", "cores": 1, "kind": "reference",
               "sample": f"{reps_cpu} replicas of ripples::simulate (IC) on the same graph and "
                         f"seeds, {1e3 * t_cpu:.0f} ms; its mean spread {ref_mean:.1f}"}
    line = {"metric": "IC spread replicas/s (forward Monte Carlo)", "value": value,
            "unit": "replicas/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "replicas only", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic R-MAT graph (seed 0) and weights (seed 1), forward CSR",
            "config": {"workload": w["name"], "n": g.n, "m": g.m, "k": w["k"],
                       "replicas_per_step": R,
                       "l2": "graph (130 MB) exceeds L2 (126 MB); per-CTA bitmaps and queues"},
            "mean_spread": mean, "reached_vertices_per_s": mean * value,
            "e2e": {"value": R * args.steps / wall, "unit": "replicas/s",
                    "h2d_bytes_per_step": 4 * len(seeds), "d2h_bytes_per_step": 8,
                    "note": "one rip_spread_ic call per step: seeds in, mean out"},
            "roofline": {"bound": "hbm", "kernel": "ic_spread_kernel",
                         "achieved": alg_per_replica * value / 1e9, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": alg_per_replica * value / 1e9 / peak, "traffic": None,
                         "alg_bytes_per_replica": alg_per_replica,
                         "alg_note": "mean over replicas 0-7 of step 0 (oracle, bit-exact)"},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches}
    print(json.dumps(line))
    dg.close()
    ctx.close()
    return 0


def _progress(t0, msg):
    """Timestamped progress line on stderr (the JSON line stays on stdout)."""
    print(f"[{time.perf_counter() - t0:8.2f}s] {msg}", file=sys.stderr, flush=True)


def run_serve(args, w, world, rank, local):
    import numpy as np
    import torch
    import ripples_b200 as rb
    if _not_on_rank0(world, rank, args, w):
        return 0
    t_run = time.perf_counter()
    torch.cuda.set_device(local)
    ctx = rb.Context(local)
    scales = [int(x) for x in args.serve_scales.split(",") if x]
    eps_choices = [float(x) for x in args.serve_eps.split(",") if x]
    graphs = {}
    t_build = time.perf_counter()
    for sc in scales:
        graphs[(sc, "IC")] = rb.DeviceGraph.rmat_on_device(
            ctx, sc, 16 << sc, "IC", rb.WEIGHTS_UNIFORM, seed=0, weight_seed=1, lo=0.0, hi=0.1)
        graphs[(sc, "LT")] = rb.DeviceGraph.rmat_on_device(
            ctx, sc, 16 << sc, "LT", rb.WEIGHTS_LT_NORMALIZED, seed=0, weight_seed=1)
    t_build = time.perf_counter() - t_build
    _progress(t_run, f"graphs built ({t_build:.1f}s)")
    t_tune = time.perf_counter()
    tuned = {}
    for sc in scales:
        tuned[f"{sc}IC"] = graphs[(sc, "IC")].autotune(seed=3, pilot=512)["name"]
        _progress(t_run, f"autotuned {sc}IC: {tuned[f'{sc}IC']}")
    t_tune = time.perf_counter() - t_tune
    rng = np.random.default_rng(3)
    N = args.serve_queries
    arrivals = np.cumsum(rng.exponential(1.0 / 200.0, size=N))
    arrivals -= arrivals[0]
    spec = []
    for i in range(N):
        sc = scales[int(rng.integers(0, len(scales)))]
        model = "IC" if rng.random() < 0.5 else "LT"
        k = int(round(float(np.exp(rng.uniform(np.log(5), np.log(500))))))
        eps = eps_choices[int(rng.integers(0, len(eps_choices)))]
        spec.append(dict(scale=sc, model=model, k=k, eps=eps))
    used, budget = ctx.memory()
    fp_budget = min(150 << 30, int(0.8 * budget))
    srv = rb.Server(ctx, footprint_budget=fp_budget, max_active=args.serve_max_active)
    tie = rb.TIE_REF_HEAP if args.serve_tiebreak == "ref_heap" else rb.TIE_LOWEST_ID
    qs = [rb.Query(graphs[(s["scale"], s["model"])], s["k"], s["eps"], seed=3, tiebreak=tie)
          for s in spec]
    launches0 = rb._lib.lib.rip_kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    sub_t = [0.0] * N
    ticks = 0
    _progress(t_run, "serving")
    t0 = time.perf_counter()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        while nxt < N and arrivals[nxt] <= now:
            srv.submit(qs[nxt])
            sub_t[nxt] = now
            nxt += 1
        active, queued = srv.pending()
        ticks += 1
        if ticks % 20 == 0:
            done_n = sum(1 for q in qs[:nxt] if q.done)
            _progress(t_run, f"tick {ticks}: submitted {nxt} active {active} queued {queued} "
                             f"done {done_n}")
        if now > args.serve_deadline:
            break
        if active == 0 and queued == 0:
            if nxt >= N:
                break
            time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
            continue
        t_tick = time.perf_counter()
        srv.tick()
        t_tick = time.perf_counter() - t_tick
        if t_tick > 1.0:
            _progress(t_run, f"tick {ticks} took {t_tick:.1f}s (active {active})")
    torch.cuda.synchronize()
    makespan = time.perf_counter() - t0
    clk = clocks.stop()
    for i, q in enumerate(qs):  # per-query account on stderr
        if not q.done:
            continue
        r = q.record
        nr = min(r.num_rounds, 64)
        gen = r.generate_ms + sum(r.round_generate_ms[j] for j in range(nr))
        sel = r.select_ms + sum(r.round_select_ms[j] for j in range(nr))
        s = spec[i]
        _progress(t_run, f"query {i} ({s['scale']} {s['model']} k={s['k']} eps={s['eps']}): "
                         f"status {q.status} theta {r.theta} elements {r.pool_elements} "
                         f"rounds {r.num_rounds} latency {q.latency_ms:.0f} ms "
                         f"queue {q.q.queue_ms:.0f} generate {gen:.0f} select {sel:.0f}")
    launches = int(rb._lib.lib.rip_kernel_launches() - launches0)
    ok = [q for q in qs if q.done and q.status == 0]
    lat = [1e3 * (sub_t[i] - arrivals[i]) + qs[i].latency_ms for i in range(N)
           if qs[i].done and qs[i].status == 0]
    st = srv.stats()
    srv.close()
    # plain path, one query at a time (a fresh pool each, one set per warp,
    # the same tie-break): every query of the same stream, in arrival order,
    # so both arms serve the identical workload
    torch.cuda.synchronize()
    tb = time.perf_counter()
    base, same, base_ok = [], True, 0
    for i in range(N):
        s = spec[i]
        p = rb.Pool(graphs[(s["scale"], s["model"])])
        t1 = time.perf_counter()
        try:
            seeds, rec = p.imm(s["k"], s["eps"], seed=3, tiebreak=tie,
                               sampler=rb.SAMPLER_PLAIN)
            base_ok += 1
            if qs[i].done and qs[i].status == 0:
                same = same and np.array_equal(seeds, qs[i].seeds)
        except rb.RipError:
            pass
        base.append(1e3 * (time.perf_counter() - t1))
        _progress(t_run, f"baseline query {i} ({s['scale']} {s['model']} k={s['k']} "
                         f"eps={s['eps']}): {base[-1]:.0f} ms")
        p.close()
    t_base = time.perf_counter() - tb
    base_qps = base_ok / t_base
    line = {"metric": "IMM queries/s (serving loop)", "value": len(ok) / makespan,
            "unit": "queries/s", "n_gpus": 1, "steps": N, "warmup": 0,
            "ms_per_step": 1e3 * makespan / max(N, 1), "higher_is_better": True,
            "scaling": "replicas only", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic R-MAT graphs (seed 0) and weights (seed 1); query stream seed 3",
            "config": {"workload": w["name"], "scales": scales, "degree": 16,
                       "arrival_rate": 200, "queries": N, "eps": eps_choices,
                       "k": "log-uniform 5..500", "max_active": args.serve_max_active,
                       "footprint_budget_gb": fp_budget / 2**30},
            "latency_ms": {"p50": _pct(lat, 50), "p99": _pct(lat, 99), "max": max(lat) if lat else None},
            "completed": len(ok), "failed": N - len(ok), "makespan_s": makespan,
            "tiebreak": args.serve_tiebreak,
            "plain_one_at_a_time": {"value": base_qps, "unit": "queries/s",
                                    "queries": len(base), "completed": base_ok,
                                    "seconds": t_base,
                                    "service_ms_p50": _pct(base, 50),
                                    "service_ms_p99": _pct(base, 99)},
            "speedup_vs_plain": (len(ok) / makespan) / base_qps if base_qps else None,
            "same_seeds_as_plain": bool(same),
            "server": st, "graph_build_s": t_build, "autotune_s": t_tune,
            "autotuned": tuned,
            "e2e": {"value": len(ok) / makespan, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(np.mean([4 * s["k"] for s in spec])),
                    "note": "queries and seeds cross the host boundary; graphs resident"},
            "clocks": clk, "gpu_launches": launches}
    print(json.dumps(line))
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
