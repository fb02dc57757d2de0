"""Benchmark: exact swap deltas/s of the pairwise sweep at N=18,524.

Workload (the reference-scale pairwise sweep): a synthetic graph pair with
N=18,524 vertices and 5,000,000 directed G1 edges (power-law out-degree,
exponent 2.1; weights 1+Geometric(0.35) with a 1e-3 heavy tail capped at
30,000, so 16-bit storage is exact), G2 = G1 relabelled with 10% of edges
deleted, 10% added and weights jittered; the initial matching is uniform
random.  One step = one full sweep: all 171,567,726 pair deltas, best
partner per vertex, sorted set commit.  The timed region runs on inputs
already resident in HBM (the profit matrix alone is 1.37 GB, far above the
126 MB L2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

--impl reference times the reference's own calculate_swap_delta
(src/graph-alignment-optimized.c:321-408, compiled in place into
oracle/_ref/librefgao.so) under OpenMP on the host cores, row by row as
src/alignment-omp.c:601-622 drives it, on a bounded sample of rows.
Multi-GPU runs are independent replicas (one instance per rank, weak scaling).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "brain-match_b200"))

WORKLOADS = {
    "n18524_e5m": dict(n=18524, e=5_000_000, wmax=30000, tail_prob=1e-3, seed=20261204),
    "n1000_e20k": dict(n=1000, e=20_000, wmax=5000, tail_prob=0.0, seed=20261203),
    # smaller pair for ncu captures (S = 268 MB, still above L2)
    "n8192_e1m": dict(n=8192, e=1_000_000, wmax=30000, tail_prob=1e-3, seed=20261206),
}
OWN_KERNELS_PER_SWEEP = 18  # relabel x5, hub B build, hub GEMM, profit, diagonal, combine, reduce, candidates,
#                             4 L2 prefetches, candidate extents, commit (row work only after a new matching)
# batch sweep, launch sequence: relabel, row work, profit, combine, reduce, candidates, commit
# (+ 21 CUB launches: the row sort and the segmented candidate sort); the persistent schedule is one launch
OWN_KERNELS_PER_BATCH_SWEEP = 7
CUB_KERNELS_PER_SWEEP = 16  # two radix sorts: histogram + exclusive sum + 6 onesweep passes each
# learned sweep: contribution, dynamic features, column stats, normalise, pool, U/V, fused ranking,
# score keys, gather, exact deltas, candidate keys, candidate extents, commit (plus two CUB radix sorts)
OWN_KERNELS_PER_LEARNED_SWEEP = 13
# greedy matching: 2 id conversions, 6 list builds (histogram + scatter), pair keys, last-of-run,
# gather, 4 two-hop counts, 2 feature kernels, positions, the matching kernel (plus CUB sorts/scans)
OWN_KERNELS_PER_GREEDY = 25
# best swap: combine + per-row reduce, pick/commit, corner x2, column permutation, term update (scatter
# and row paths), pS sync
OWN_KERNELS_PER_LOOKUP_SWAP = 9


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples (200 ms) during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[2:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_reference(g, rows_target_s, seed=5, rows=None):
    """Times the reference's calculate_swap_delta under OpenMP on a row sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    R = oracle.RefGAO()
    n = g["n"]
    t0 = time.perf_counter()
    gm = R.graph(g["src1"], g["dst1"], g["w1"])
    gf = R.graph(g["src2"], g["dst2"], g["w2"])
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    m = g["map0"]
    if rows is None:
        probe = rng.choice(np.arange(1, n + 1), 4, replace=False).astype(np.int32)
        t = time.perf_counter()
        R.rows_omp(gm, gf, m, probe, n)
        dt = max(time.perf_counter() - t, 1e-3)
        rows = int(min(2048, max(4, 4 * rows_target_s / dt)))
    sample = rng.choice(np.arange(1, n + 1), rows, replace=False).astype(np.int32)
    t = time.perf_counter()
    cnt, checksum, threads = R.rows_omp(gm, gf, m, sample, n)
    dt = time.perf_counter() - t
    return dict(value=cnt / dt, deltas=cnt, seconds=dt, rows=rows, threads=threads, build_s=build_s,
                R=R, gm=gm, gf=gf, checksum=checksum)


def cpu_racy(g, target_s, seed=6):
    """The reference's racy OpenMP tool (src/graph-alignment-optimized-parallel.c:544-582,
    compiled in place): its parallel loop over partners, with every improving
    swap committed in a critical section followed by a full rescore, for one
    seeded row against a bounded prefix of partners sized to ~target_s seconds,
    from the random start.  Its deltas read a matching other threads change,
    so its moves are not deterministic: it is timed as shipped, beside the
    race-free row loop, and never used as a result."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    RQ = oracle.RefPar()
    n = g["n"]
    gm = RQ.graph(g["src1"], g["dst1"], g["w1"])
    gf = RQ.graph(g["src2"], g["dst2"], g["w2"])
    row = np.array([int(np.random.default_rng(seed).integers(1, n + 1))], np.int32)
    k = min(n, 256)
    t = time.perf_counter()
    RQ.rows(gm, gf, g["map0"].copy(), row, k)
    dt = max(time.perf_counter() - t, 1e-3)
    k = int(min(n, max(k, k * target_s / dt)))
    t = time.perf_counter()
    cnt, commits, threads = RQ.rows(gm, gf, g["map0"].copy(), row, k)
    dt = time.perf_counter() - t
    RQ.free(gm)
    RQ.free(gf)
    return {"value": cnt / dt, "unit": "deltas/s", "cores": threads, "kind": "reference",
            "sample": f"row {int(row[0])} x partners 1..{k} from the random start ({cnt} deltas, {commits} "
                      f"commits with the tool's full rescore each, {dt:.1f} s)",
            "note": "racy: deltas read a matching other threads change, and two commits in one row can "
                    "give one image to two vertices; timed as shipped, not a result"}


def run_reference(args, g, world, rank, pg):
    wl = args.workload
    if rank != 0:
        return
    n = g["n"]
    per_step = max(1.0, 120.0 / max(1, args.steps + args.warmup))
    first = cpu_reference(g, per_step)
    rows = first["rows"]
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_step(first, g, rows, seed=100 + i)
        if i >= args.warmup:
            vals.append(r)
    tot_d = sum(v[0] for v in vals)
    tot_s = sum(v[1] for v in vals)
    value = tot_d / tot_s
    line = {
        "impl": "reference", "metric": "exact swap deltas/s", "value": value, "unit": "deltas/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_s / len(vals), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": wl, "n": n, "e1": int(len(g["src1"])), "e2": int(len(g["src2"])),
                   "step": f"{rows} full rows of pair deltas (bounded sample of one sweep)"},
        "cpu_baseline": {"value": value, "unit": "deltas/s", "cores": first["threads"], "kind": "reference",
                         "sample": f"{rows} seeded rows x {n - 1} partners per step, OpenMP dynamic"},
        "e2e": {"value": value, "unit": "deltas/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_reference_step(ctx, g, rows, seed):
    R, gm, gf = ctx["R"], ctx["gm"], ctx["gf"]
    n = g["n"]
    rng = np.random.default_rng(seed)
    sample = rng.choice(np.arange(1, n + 1), rows, replace=False).astype(np.int32)
    t = time.perf_counter()
    cnt, _, _ = R.rows_omp(gm, gf, g["map0"], sample, n)
    return cnt, time.perf_counter() - t


def run_engine(args, g, world, rank, local, pg):
    import bm
    import torch
    torch.cuda.set_device(local)
    n = g["n"]
    E = bm.Engine.from_pair(g)
    info = E.info()
    E.set_mapping(g["map0"])
    deltas_per_sweep = n * (n - 1) // 2
    for _ in range(args.warmup):
        E.sweep()
    m_start = E.get_mapping()  # the e2e leg replays the timed sweeps from here
    barrier(pg)
    torch.cuda.synchronize()
    stats = []
    with Clocks(local) as clk:
        E.timer_mark(0)
        for _ in range(args.steps):
            stats.append(E.sweep())
        E.timer_mark(1)
        torch.cuda.synchronize()
    barrier(pg)
    ms = E.timer_elapsed(0, 1)
    ms_max = allreduce_max(pg, ms)
    value = world * args.steps * deltas_per_sweep / (ms_max / 1e3)

    # end to end through the C ABI with host buffers: H2D of the matching,
    # sweep, D2H of the matching and the score -- the same sweeps as the timed
    # region, replayed from the same starting matching
    host_map = m_start
    e2e_steps = args.steps
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        E.set_mapping(host_map)
        st = E.sweep()
        host_map = E.get_mapping()
        _ = st["score_after"]
    t1 = time.perf_counter()
    e2e_s = allreduce_max(pg, t1 - t0)
    e2e_value = world * e2e_steps * deltas_per_sweep / e2e_s
    h2d = 2 * (n + 1) * 4
    d2h = (n + 1) * 4 + 8 + 96

    # roofline of the dominant kernel (profit rows), timed live with events
    prof_ms = statistics.mean(s["ms_profit"] for s in stats)
    alg_bytes = 2 * n * n * (info["entry_bits"] // 8)   # W1 and P2 once, per sweep
    peak, peak_kind = peaks()
    achieved = alg_bytes / (prof_ms / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "k_profit_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("bytes_per_launch_full_size")
        except (OSError, ValueError):
            traffic = None
    terms = statistics.mean(s["min_terms"] for s in stats)
    # the engine's own microbenchmark of shared-memory atomic adds at random
    # addresses (the profit kernel's inner operation)
    try:
        red_peak, _ = bm.measure_peaks(n)
    except Exception:
        red_peak = None
    # k_profit against the roof that binds it: one shared-memory atomic add per
    # scattered min term, against the measured red.shared.add rate
    profit_atomics = None
    if red_peak and prof_ms > 0:
        rate = terms / (prof_ms / 1e3)
        profit_atomics = {"terms_per_launch": terms, "achieved_per_s": rate, "peak_per_s": red_peak,
                          "frac": rate / red_peak,
                          "note": "min terms scattered per launch / the launch's event time, against the "
                                  "engine's shared-memory atomic microbenchmark"}

    # descent to convergence from the initial matching, device time: sweeps
    # that rebuild the profit matrix against sweeps that update it from the
    # vertices the previous commit moved (identical moves, checked here)
    descent = None
    if not args.no_descent:
        runs = {}
        for inc in (False, True):
            E.set_mapping(g["map0"])
            tot, upd, sw, per = 0.0, 0, 0, []
            for _ in range(500):
                s = E.sweep(incremental=inc)
                tot += s["ms_total"]
                upd += s["profit_mode"] == 1
                sw += 1
                per.append([s["committed"], s["profit_mode"], round(s["ms_prep"] + s["ms_hub"] + s["ms_profit"], 3),
                            round(s["ms_total"], 3)])
                if s["committed"] == 0:
                    break
            runs[inc] = (tot, upd, sw, s["score_after"], E.get_mapping(), per)
        assert runs[False][3] == runs[True][3] and np.array_equal(runs[False][4], runs[True][4])
        descent = {"sweeps": runs[False][2], "final_score": runs[False][3], "rebuild_ms": runs[False][0],
                   "incremental_ms": runs[True][0], "updated_sweeps": runs[True][1],
                   "per_sweep_incremental": runs[True][5],
                   "per_sweep_fields": ["committed", "profit_mode (0 rebuilt, 1 updated)", "ms making S exact",
                                        "ms sweep"]}

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            try:
                c = cpu_reference(g, args.cpu_seconds)
                cpu = {"value": c["value"], "unit": "deltas/s", "cores": c["threads"], "kind": "reference",
                       "sample": f"{c['rows']} seeded rows x {n - 1} partners ({c['deltas']} deltas, "
                                 f"{c['seconds']:.1f} s), reference calculate_swap_delta under OpenMP"}
                c["R"].free(c["gm"])
                c["R"].free(c["gf"])
                cpu["racy_tool"] = cpu_racy(g, 6.0)
            except OSError as e:
                cpu = {"value": None, "unit": "deltas/s", "cores": 0, "kind": "reference", "sample": str(e)}
        line = {
            "metric": "exact swap deltas/s", "value": value, "unit": "deltas/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": args.workload, "n": n, "e1": int(info["e1"]), "e2": int(info["e2"]),
                       "entry_bits": info["entry_bits"], "step": "full pairwise sweep + set commit",
                       "deltas_per_step": deltas_per_sweep, "l2": "inputs larger than L2",
                       "parallelism": f"replicas{world}"},
            "e2e": {"value": e2e_value, "unit": "deltas/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_profit", "kernel_ms": prof_ms, "alg_bytes": alg_bytes,
                         "min_terms": terms},
            "profit_smem_atomics": profit_atomics,
            "descent": descent,
            "cpu_baseline": cpu,
            "gpu_launches": args.steps * (OWN_KERNELS_PER_SWEEP + CUB_KERNELS_PER_SWEEP),
            "clocks": clk.summary(),
            "sweeps": [{k: s[k] for k in ("score_before", "score_after", "committed", "verified", "candidates",
                                         "ms_prep", "ms_hub", "ms_profit", "ms_combine", "ms_commit",
                                         "ms_total", "min_terms", "commit_entries", "commit_steps",
                                         "commit_carried")} for s in stats],
        }
        print(json.dumps(line), flush=True)
    E.close()


def batch_pairs(seed=20261207, count=64):
    """64 instances, N log-uniform in [500, 8000], E = 20 N, weights as the N=1,000 workload."""
    import bm
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(500), np.log(8000), count)).astype(int)
    return [bm.generate(bm.gen_params(n=int(n), e=20 * int(n), seed=seed + 1 + i)) for i, n in enumerate(ns)]


def run_batch(args, world, rank, local, pg):
    import bm
    import torch
    torch.cuda.set_device(local)
    pairs = batch_pairs(20261207 + 1000 * rank)
    B = bm.Batch(pairs)
    info = B.info()
    B.set_mappings([g["map0"] for g in pairs])
    schedules = None
    if args.batch_schedules:
        # every schedule set directly: sweeps 3-5 from the same random start, device ms per sweep
        schedules = {}
        for sched in ((True, 1024, 64), (True, 1024, 32), (False, 256, 64), (False, 256, 32), (False, 512, 64)):
            B.set_mappings([g["map0"] for g in pairs])
            B.set_schedule(*sched)
            B.sweeps(2)
            _, ms3 = B.sweeps(3)
            name = ("persistent" if sched[0] else "sequence/%d" % sched[1]) + "/tile%d" % sched[2]
            schedules[name] = ms3 / 3
        B.set_mappings([g["map0"] for g in pairs])
    pt, tile = B.autotune()
    persistent = pt == 1024   # the one-launch schedule reports its 1024-thread CTA
    B.sweeps(args.warmup)
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        commits, ms = B.sweeps(args.steps)
        torch.cuda.synchronize()
    barrier(pg)
    ms_max = allreduce_max(pg, ms)
    value = world * args.steps * info["total_pairs"] / (ms_max / 1e3)
    maps = B.get_mappings()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        B.set_mappings(maps)
        B.sweeps(1)
        maps = B.get_mappings()
    e2e_s = allreduce_max(pg, time.perf_counter() - t0)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            try:
                cpu = cpu_batch(pairs, args.cpu_seconds)
            except OSError as e:
                cpu = {"value": None, "unit": "deltas/s", "cores": 0, "kind": "reference", "sample": str(e)}
        h2d = sum(2 * (g["n"] + 1) * 4 for g in pairs)
        line = {
            "metric": "exact swap deltas/s (batched instances)", "value": value, "unit": "deltas/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "batch64", "instances": info["count"], "max_n": info["max_n"],
                       "pairs_per_step": info["total_pairs"], "edges": "20 N per instance",
                       "autotuned": {"profit_threads": pt, "combine_tile": tile,
                                     "schedule": "one persistent launch" if persistent else "launch sequence"},
                       "step": "one sweep of every instance (CUDA graph replay)", "parallelism": f"replicas{world}"},
            "gpu_launches": args.steps * (1 if persistent else OWN_KERNELS_PER_BATCH_SWEEP),
            "e2e": {"value": world * args.steps * info["total_pairs"] / e2e_s, "unit": "deltas/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d // 2},
            "committed_last_steps": int(commits.sum()),
            "schedules_ms_per_sweep": schedules,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    B.close()


def run_triples(args, world, rank, local, pg):
    """3-cycle rounds on the N=18,524 pair, starting from the pairwise sweep's
    output matching (50 sweeps, untimed): 256 two-hop partners per vertex,
    both rotations of every triple evaluated exactly, best disjoint set
    committed."""
    import bm
    import torch
    torch.cuda.set_device(local)
    p = dict(WORKLOADS["n18524_e5m"])
    p["seed"] += rank
    g = bm.generate(bm.gen_params(**p))
    E = bm.Engine.from_pair(g)
    E.set_mapping(g["map0"])
    for _ in range(args.pre_sweeps):
        if E.sweep()["committed"] == 0:
            break
    start_score = E.score()
    for r in range(args.warmup):
        E.triple_round(partners=256, seed=1000 + r)
    m_timed = E.get_mapping()
    barrier(pg)
    torch.cuda.synchronize()
    stats = []
    with Clocks(local) as clk:
        E.timer_mark(0)
        for r in range(args.steps):
            stats.append(E.triple_round(partners=256, seed=2000 + r))
        E.timer_mark(1)
        torch.cuda.synchronize()
    barrier(pg)
    ms = allreduce_max(pg, E.timer_elapsed(0, 1))
    m_end = E.get_mapping()
    inc_ms = replay_rounds_incremental(
        E, m_timed, args.steps, lambda r, inc: E.triple_round(partners=256, seed=2000 + r, incremental=inc))
    assert np.array_equal(E.get_mapping(), m_end)
    rot = sum(s["rotations"] for s in stats)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            try:
                cpu = cpu_triples(g, m_timed, 2000 + 0, args.cpu_seconds)
            except OSError as e:
                cpu = {"value": None, "unit": "rotations/s", "cores": 0, "kind": "reference", "sample": str(e)}
        line = {
            "metric": "exact 3-cycle rotation deltas/s", "value": world * rot / (ms / 1e3), "unit": "rotations/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "triples_n18524", "partners": 256, "pre_sweeps": args.pre_sweeps,
                       "start_score": start_score, "step": "one 3-cycle round"},
            "incremental": {"ms_per_step": inc_ms, "value": world * rot / (args.steps * inc_ms / 1e3),
                            "note": "the same rounds with the profit matrix updated from the previous "
                                    "round's moves (identical moves, asserted)"},
            "rounds": [{k: s[k] for k in ("triples", "committed", "verified", "score_after", "ms_sample",
                                         "ms_eval", "ms_commit", "ms_total")} for s in stats],
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    E.close()


def cpu_triples(g, m, seed, target_s):
    """The reference's 3-cycle delta: calculate_permutation_delta
    (src/permutation.c:623-696, compiled in place) before and after each
    rotation, under OpenMP over triples, on a seeded sample of the round's
    triples (the same 256-partner two-hop sampling) sized to ~target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    O = oracle.Oracle.from_pair(g)
    RP = oracle.RefPerm()
    n = g["n"]
    gm = RP.graph(g["src1"], g["dst1"], g["w1"])
    gf = RP.graph(g["src2"], g["dst2"], g["w2"])
    bs, cs = O.triple_samples(seed, 256)
    valid = bs > 0
    a = np.repeat(np.arange(1, n + 1, dtype=np.int32), 256).reshape(n, 256)[valid]
    b, c = bs[valid], cs[valid]
    rng = np.random.default_rng(seed)
    k = 32
    idx = rng.choice(len(a), k, replace=False)
    t = time.perf_counter()
    RP.triples_omp(gm, gf, m, a[idx], b[idx], c[idx])
    dt = max(time.perf_counter() - t, 1e-3)
    k = int(min(len(a), max(k, k * target_s / dt)))
    idx = rng.choice(len(a), k, replace=False)
    t = time.perf_counter()
    _, threads = RP.triples_omp(gm, gf, m, a[idx], b[idx], c[idx])
    dt = time.perf_counter() - t
    RP.free(gm)
    RP.free(gf)
    return {"value": 2 * k / dt, "unit": "rotations/s", "cores": threads, "kind": "reference",
            "sample": f"{k} seeded triples of the round ({2 * k} rotations, {dt:.1f} s), reference "
                      "calculate_permutation_delta before/after each rotation under OpenMP"}


def cpu_batch(pairs, target_s, seed=9):
    """The reference's calculate_swap_delta (compiled in place, OpenMP over
    partners as in src/alignment-omp.c:601-622) on seeded rows of four of the
    batch's instances (smallest, largest, two between), each instance's
    share of ~target_s seconds; deltas/s over all of them.  The reference
    sizes every graph by NUM_NODES, so instances are built one at a time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    R = oracle.RefGAO()
    order = np.argsort([g["n"] for g in pairs])
    pick = [order[0], order[len(order) // 3], order[2 * len(order) // 3], order[-1]]
    rng = np.random.default_rng(seed)
    tot_d, tot_s, threads, ns = 0, 0.0, 0, []
    for i in pick:
        g = pairs[int(i)]
        n = int(g["n"])
        gm = R.graph(g["src1"], g["dst1"], g["w1"])
        gf = R.graph(g["src2"], g["dst2"], g["w2"])
        t = time.perf_counter()
        R.rows_omp(gm, gf, g["map0"], rng.choice(np.arange(1, n + 1), 2, replace=False).astype(np.int32), n)
        per_row = max((time.perf_counter() - t) / 2, 1e-4)
        rows = int(min(n, max(2, target_s / 4 / per_row)))
        sample = rng.choice(np.arange(1, n + 1), rows, replace=False).astype(np.int32)
        t = time.perf_counter()
        cnt, _, threads = R.rows_omp(gm, gf, g["map0"], sample, n)
        tot_s += time.perf_counter() - t
        tot_d += cnt
        ns.append((n, rows))
        R.free(gm)
        R.free(gf)
    return {"value": tot_d / tot_s, "unit": "deltas/s", "cores": threads, "kind": "reference",
            "sample": "seeded full rows of 4 instances (n, rows): " + ", ".join(f"({a}, {b})" for a, b in ns) +
                      f"; {tot_d} deltas in {tot_s:.1f} s, reference calculate_swap_delta under OpenMP"}


def run_first_improvement(args, world, rank, local, pg):
    """The N=1,000 / 20,000-edge workload end to end: the reference's
    sequential first-improvement order (src/graph-alignment-optimized.c:
    515-577) from the random start until a pass commits nothing.  Engine:
    bm_first_improvement; CPU: the reference's own loop compiled in place
    (its commit validation and full rescore included).  Both make the same
    moves; the final scores are asserted equal."""
    import bm
    import torch
    torch.cuda.set_device(local)
    p = dict(WORKLOADS["n1000_e20k"])
    p["seed"] += rank
    g = bm.generate(bm.gen_params(**p))
    E = bm.Engine.from_pair(g)
    for _ in range(args.warmup):
        E.set_mapping(g["map0"])
        E.first_improvement(10_000)
    walls, devs = [], []
    barrier(pg)
    with Clocks(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            E.set_mapping(g["map0"])
            E.timer_mark(0)
            commits, passes = E.first_improvement(10_000)
            E.timer_mark(1)
            score = E.score()
            m = E.get_mapping()
            walls.append(time.perf_counter() - t0)
            devs.append(E.timer_elapsed(0, 1) / 1e3)
    barrier(pg)
    dev = allreduce_max(pg, statistics.median(devs))
    wall = allreduce_max(pg, statistics.median(walls))
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            try:
                sys.path.insert(0, os.path.join(ROOT, "oracle"))
                import oracle
                R = oracle.RefGAO()
                gm = R.graph(g["src1"], g["dst1"], g["w1"])
                gf = R.graph(g["src2"], g["dst2"], g["w2"])
                mr = g["map0"].copy()
                t0 = time.perf_counter()
                rscore, rcommits, rpasses = R.first_improvement(gm, gf, mr, g["n"], 10_000)
                rs = time.perf_counter() - t0
                R.free(gm)
                R.free(gf)
                assert rscore == score and np.array_equal(mr, m) and (rcommits, rpasses) == (commits, passes)
                cpu = {"value": rs, "unit": "s", "cores": 1, "kind": "reference",
                       "sample": f"the whole descent: {rcommits} commits over {rpasses} passes, final score "
                                 f"{rscore} (identical matching to the engine's), m1, m2 over 1..n"}
            except OSError as e:
                cpu = {"value": None, "unit": "s", "cores": 0, "kind": "reference", "sample": str(e)}
        line = {
            "metric": "first-improvement descent time to the fixed point", "value": dev, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": "first_improvement_n1000", "n": int(g["n"]), "e1": int(len(g["src1"])),
                       "step": "one sequential first-improvement descent from the random start to a pass "
                               "without a commit"},
            "final_score": score, "commits": commits, "passes": passes,
            "e2e": {"value": wall, "unit": "s", "h2d_bytes_per_step": 4 * (int(g["n"]) + 1),
                    "d2h_bytes_per_step": 4 * (int(g["n"]) + 1) + 8},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    E.close()


def replay_rounds_incremental(E, start, steps, round_fn):
    """The timed rounds replayed from the same matching with the profit matrix
    updated from the previous round's moves instead of rebuilt; the moves must
    be identical.  Returns the device ms per round."""
    import torch
    E.set_mapping(start)
    round_fn(0, True)      # the first round after a new mapping rebuilds: untimed
    E.set_mapping(start)
    torch.cuda.synchronize()
    E.timer_mark(2)
    for r in range(steps):
        round_fn(r, True)
    E.timer_mark(3)
    torch.cuda.synchronize()
    return E.timer_elapsed(2, 3) / steps


def run_greedy(args, world, rank, local, pg):
    """The greedy feature matcher on the N=18,524 pair: one step = one whole
    initial matching (features of both graphs + the sequential matching) from
    host edge arrays to the host matching."""
    import bm
    import torch
    torch.cuda.set_device(local)
    p = dict(WORKLOADS["n18524_e5m"])
    p["seed"] += rank
    g = bm.generate(bm.gen_params(**p))
    for _ in range(args.warmup):
        bm.greedy_match(g)
    barrier(pg)
    torch.cuda.synchronize()
    dev_ms, walls = [], []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            m, st = bm.greedy_match(g)
            walls.append(time.perf_counter() - t0)
            dev_ms.append(st["ms_features"] + st["ms_match"])
        torch.cuda.synchronize()
    barrier(pg)
    dev_s = allreduce_max(pg, sum(dev_ms) / 1e3)
    wall_s = allreduce_max(pg, sum(walls))
    with bm.Engine.from_pair(g) as E:
        E.set_mapping(m)
        greedy_score = E.score()
        E.set_mapping(g["map0"])
        random_score = E.score()
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            t0 = time.perf_counter()
            mo = oracle.greedy_match(g)
            cs = time.perf_counter() - t0
            cpu = {"value": cs, "unit": "s", "cores": os.cpu_count(), "kind": "port",
                   "sample": "one whole matching (the oracle restatement: OpenMP features, scalar matching loop); "
                             "identical to the GPU result: " + str(bool(np.array_equal(mo, m)))}
        line = {
            "metric": "greedy initial matching time", "value": dev_s / args.steps, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int32+f64",
            "data": "synthetic",
            "config": {"workload": "greedy_n18524", "n": int(g["n"]), "e1": int(len(g["src1"])),
                       "e2": int(len(g["src2"])), "step": "features of both graphs + the sequential greedy matching"},
            "e2e": {"value": wall_s / args.steps, "unit": "s",
                    "h2d_bytes_per_step": 4 * 3 * (len(g["src1"]) + len(g["src2"])),
                    "d2h_bytes_per_step": 4 * int(g["n"])},
            "greedy_score": greedy_score, "random_start_score": random_score,
            "gpu_launches": args.steps * OWN_KERNELS_PER_GREEDY,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def run_lookup(args, world, rank, local, pg):
    """Best-swap descent on the exact table (N=18,524 pair, random start):
    one step = one committed swap (combine, pick, swap, table update); the
    table is built before the timed region."""
    import bm
    import torch
    torch.cuda.set_device(local)
    p = dict(WORKLOADS["n18524_e5m"])
    p["seed"] += rank
    g = bm.generate(bm.gen_params(**p))
    E = bm.Engine.from_pair(g)
    E.set_mapping(g["map0"])
    E.lookup_descent(max(args.warmup, 1))
    swaps = 8 * args.steps
    barrier(pg)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        E.timer_mark(0)
        st = E.lookup_descent(swaps)
        E.timer_mark(1)
        torch.cuda.synchronize()
    barrier(pg)
    ms = allreduce_max(pg, E.timer_elapsed(0, 1))
    done = st["swaps"]
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            try:
                c = cpu_reference(g, 8.0)
                # the reference refreshes 4N table entries per swap (update_lookup_and_heap,
                # src/best-swap/score-lookup.c:514-537), each one calculate_swap_delta
                per_swap = 4 * int(g["n"])
                cpu = {"value": c["value"] / per_swap, "unit": "swaps/s", "cores": c["threads"], "kind": "reference",
                       "sample": f"{c['rows']} seeded rows of reference deltas under OpenMP "
                                 f"({c['value']:.3g} deltas/s) / {per_swap} deltas refreshed per swap"}
            except OSError as e:
                cpu = {"value": None, "unit": "swaps/s", "cores": 0, "kind": "reference", "sample": str(e)}
        line = {
            "metric": "exact best swaps/s", "value": world * done / (ms / 1e3), "unit": "swaps/s", "n_gpus": world,
            "steps": done, "warmup": args.warmup, "ms_per_step": ms / max(done, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "lookup_n18524", "n": int(g["n"]),
                       "step": "one exact best swap: pair combine over the table, pick, swap, table update"},
            "score_before": st["score_before"], "score_after": st["score_after"],
            "gpu_launches": done * OWN_KERNELS_PER_LOOKUP_SWAP,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    E.close()


def run_quads(args, world, rank, local, pg):
    """4-set permutation rounds on the N=18,524 pair, from the pairwise
    sweep's output matching (up to 50 sweeps, untimed): 64 connected 4-sets
    (3-step walks) per vertex, all 23 permutations of each evaluated exactly,
    best disjoint set committed."""
    import bm
    import torch
    torch.cuda.set_device(local)
    p = dict(WORKLOADS["n18524_e5m"])
    p["seed"] += rank
    g = bm.generate(bm.gen_params(**p))
    E = bm.Engine.from_pair(g)
    E.set_mapping(g["map0"])
    for _ in range(args.pre_sweeps):
        if E.sweep()["committed"] == 0:
            break
    start_score = E.score()
    for r in range(args.warmup):
        E.quad_round(partners=64, seed=1000 + r)
    m_timed = E.get_mapping()
    barrier(pg)
    torch.cuda.synchronize()
    stats = []
    with Clocks(local) as clk:
        E.timer_mark(0)
        for r in range(args.steps):
            stats.append(E.quad_round(partners=64, seed=2000 + r))
        E.timer_mark(1)
        torch.cuda.synchronize()
    barrier(pg)
    ms = allreduce_max(pg, E.timer_elapsed(0, 1))
    m_end = E.get_mapping()
    inc_ms = replay_rounds_incremental(
        E, m_timed, args.steps, lambda r, inc: E.quad_round(partners=64, seed=2000 + r, incremental=inc))
    assert np.array_equal(E.get_mapping(), m_end)
    perms = sum(s["permutations"] for s in stats)
    if rank == 0:
        line = {
            "metric": "exact 4-set permutation deltas/s", "value": world * perms / (ms / 1e3),
            "unit": "permutations/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": "quads_n18524", "partners": 64, "pre_sweeps": args.pre_sweeps,
                       "start_score": start_score, "step": "one 4-set round (23 permutations per set)"},
            "incremental": {"ms_per_step": inc_ms, "value": world * perms / (args.steps * inc_ms / 1e3),
                            "note": "the same rounds with the profit matrix updated from the previous "
                                    "round's moves (identical moves, asserted)"},
            "rounds": [{k: s[k] for k in ("quads", "committed", "verified", "score_after", "ms_sample",
                                         "ms_eval", "ms_commit", "ms_total")} for s in stats],
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    E.close()


def run_learned(args, world, rank, local, pg):
    """Time to score, learned vs plain, on the N=18,524 pair by default
    (--graph picks another pair; one GPU per replica).  Plain: exhaustive sweeps from the random start until one
    commits nothing; its final score is the target.  Learned: the network
    (trained beforehand on exact deltas that the engine logs along a run from
    another random start; training time reported apart) drives
    bm_learned_run from the same start until the target is reached.  Each
    timed step is one descent of each form; values are medians over steps.
    The untrained network's time to the same target shows what training adds."""
    import bm
    import torch
    torch.cuda.set_device(local)
    p = dict(WORKLOADS[args.graph])
    p["seed"] += rank
    g = bm.generate(bm.gen_params(**p))
    n = g["n"]
    E = bm.Engine.from_pair(g)

    def plain_descent():
        E.set_mapping(g["map0"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sweeps, dev_ms = 0, 0.0
        while True:
            st = E.sweep()
            sweeps += 1
            dev_ms += st["ms_total"]
            if st["committed"] == 0 or sweeps >= 2000:
                break
        score = E.score()
        return time.perf_counter() - t0, dev_ms, sweeps, score

    # training: exact deltas logged along a run from another random start
    rng = np.random.default_rng(1000 + rank)
    start = np.concatenate([[0], rng.permutation(n) + 1]).astype(np.int32)
    net = bm.Mlp(seed=13)
    E.set_mapping(start)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tstats = net.train_from(E, sweeps=args.train_sweeps, extra_partners=64, epochs=1, lr=1e-2, seed=5)
    train_s = time.perf_counter() - t0
    untrained = bm.Mlp(seed=13)
    opts = dict(pool=64, top_fraction=0.02, probe_every=8)

    def learned_descent(model, target, seed, host_io):
        m0 = g["map0"]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E.set_mapping(m0)
        r = model.learned_run(E, max_sweeps=4000, target_score=target, seed=seed, trace=False, **opts)
        if host_io:
            _ = E.get_mapping()
        return time.perf_counter() - t0, r

    for w in range(args.warmup):
        plain_descent()
    target = plain_descent()[3]
    for w in range(args.warmup):
        learned_descent(net, target, 100 + w, True)
    barrier(pg)
    plain_t, learned_t, untrained_t, runs, plain_info = [], [], [], [], []
    with Clocks(local) as clk:
        for k in range(args.steps):
            pt, pdev, psw, pscore = plain_descent()
            plain_t.append(pt)
            plain_info.append((pdev, psw, pscore))
            lt, r = learned_descent(net, pscore, 200 + k, True)
            learned_t.append(lt)
            runs.append(r)
    barrier(pg)
    ut, ur = learned_descent(untrained, target, 300, True)
    # the full learned descent to its own local optimum (no target)
    E.set_mapping(g["map0"])
    t0 = time.perf_counter()
    full = net.learned_run(E, max_sweeps=4000, target_score=0, seed=400, **opts)
    full_s = time.perf_counter() - t0
    T_plain = allreduce_max(pg, statistics.median(plain_t))
    T_learned = allreduce_max(pg, statistics.median(learned_t))
    if rank == 0:
        r0 = runs[len(runs) // 2]
        own_launches = int(statistics.median(r["learned"] * OWN_KERNELS_PER_LEARNED_SWEEP + r["exhaustive"] * OWN_KERNELS_PER_SWEEP
                                             for r in runs))
        line = {
            "metric": "wall seconds to the plain sweep's final score (learned form)", "value": T_learned,
            "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * T_learned, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32 deltas, bf16 network", "data": "synthetic",
            "config": {"workload": "learned_" + args.graph, "n": n, "e1": int(len(g["src1"])),
                       "step": "one descent from the random start to the plain form's final score",
                       "pool": opts["pool"], "top_fraction": opts["top_fraction"],
                       "probe_every": opts["probe_every"], "l2": "inputs larger than L2",
                       "parallelism": f"replicas{world}"},
            "plain": {"seconds": T_plain, "device_ms": plain_info[0][0], "sweeps": plain_info[0][1],
                      "final_score": plain_info[0][2]},
            "learned": {"seconds": T_learned, "ratio_to_plain": T_learned / T_plain, "steps": r0["sweeps"],
                        "learned_sweeps": r0["learned"], "exhaustive_sweeps": r0["exhaustive"],
                        "device_ms": r0["ms_total"], "score": r0["score_after"], "reached": r0["reached"]},
            "learned_to_convergence": {"seconds": full_s, "score": full["score_after"], "steps": full["sweeps"],
                                       "learned_sweeps": full["learned"], "exhaustive_sweeps": full["exhaustive"]},
            "untrained": {"seconds": ut, "ratio_to_plain": ut / T_plain, "steps": ur["sweeps"],
                          "reached": ur["reached"]},
            "training": {"seconds": train_s, "samples": tstats["samples"], "steps": tstats["steps"],
                         "logged_sweeps": args.train_sweeps, "first_epoch_loss": tstats["first_loss"],
                         "last_epoch_loss": tstats["last_loss"], "start": "another random matching"},
            "e2e": {"value": T_learned, "unit": "s", "h2d_bytes_per_step": (n + 1) * 4,
                    "d2h_bytes_per_step": (n + 1) * 4, "note": "set_mapping and get_mapping inside the timed region"},
            "gpu_launches": own_launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    net.close()
    untrained.close()
    E.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="n18524_e5m",
                    choices=sorted(WORKLOADS) + ["batch64", "triples", "quads", "learned", "greedy", "lookup",
                                                 "first_improvement"])
    ap.add_argument("--train-sweeps", type=int, default=40)
    ap.add_argument("--graph", default="n18524_e5m", choices=sorted(WORKLOADS),
                    help="graph pair of the learned workload")
    ap.add_argument("--pre-sweeps", type=int, default=50)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-descent", action="store_true", help="skip the time-to-convergence descents")
    ap.add_argument("--batch-schedules", action="store_true",
                    help="batch64: also time every batch schedule set directly (sweeps 3-5 from the random start)")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    if args.impl == "reference" and args.workload in ("batch64", "triples", "quads", "greedy", "lookup",
                                                      "first_improvement"):
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the pairwise sweep "
                              "workloads; this workload's CPU baseline is the cpu_baseline of the engine line"}),
                  flush=True)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.workload in ("batch64", "triples", "quads", "greedy", "lookup", "first_improvement") or \
            (args.workload == "learned" and args.impl == "engine"):
        fn = {"batch64": run_batch, "triples": run_triples, "quads": run_quads, "learned": run_learned,
              "greedy": run_greedy, "lookup": run_lookup, "first_improvement": run_first_improvement}[args.workload]
        fn(args, world, rank, local, pg)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    p = dict(WORKLOADS[args.graph if args.workload == "learned" else args.workload])
    p["seed"] += rank  # independent replica per rank
    if args.impl == "reference":
        # the same seeded pair from the generator's host-only build, so the
        # reference arm loads none of the engine's code
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        run_reference(args, oracle.generate(**p), world, rank, pg)
    else:
        import bm
        run_engine(args, bm.generate(bm.gen_params(**p)), world, rank, local, pg)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
