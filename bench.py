#!/usr/bin/env python
"""Benchmark of the energy-game solve on B200: GTEPS of the full solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): one game of n = 2^20 vertices, owners 50/50, out-degree
floor of a continuous x^-2 power law on [1, 4097) (mean 7.9, m = 8.28M),
successors uniform without self-loops or duplicates, weights uniform in
[-1000, 1000], 64-bit credits; seeded (seed 0xE6 + 2), synthetic.

A step is one complete solve from f = 0: transpose and renumbering,
initial frontier, the persistent lifting kernels (frontier rounds, then
dense rounds over every vertex) until the least fixed point.
  value  GTEPS = out-edges scanned by lifts / device time of the solve, with
         the game resident in HBM; device time from CUDA events on the
         solver's stream; L2 flushed (256 MB write) before every step
  e2e    the same metric through the one-call public API eg_solve_i64 with
         pinned host buffers: allocation, host->device copy of the CSR, solve,
         device->host copy of the credits, per step (wall clock)
  roofline   the dominant kernel (k_lift_dense, the dense rounds): its
         algorithmic bytes per launch / its mean launch time (CUDA events
         around each launch, on the solver's stream), against the measured
         HBM copy bandwidth; `traffic` is the DRAM bytes per launch scaled
         from an ncu capture of a round-capped solve (profiles/)
  cpu_baseline   the reference's own EG_cpu_solver (oracle/_ref, compiled
         unmodified; serial worklist, 1 core) on a bounded sample of the same
         game: its first P worklist pops (reference --eg P)

With N > 1 (torchrun), every rank solves its own replica on its own GPU (the
single-game solve does not shard); value = edges of all ranks / max time.

--impl reference times the reference CPU solver alone (rank 0), each step a
bounded sample of the same workload.

--workload cfg4 (batched): the first --games games of the seeded 4096-game
stream at K = 8 mean-payoff thresholds in one persistent launch, against
one plain solve per (game, threshold) on a seeded sample.  --workload cfg5
(served): the seeded request stream (n up to --n-max) through the serving
loop at each --rates arrival rate, against the same arrivals served one at
a time with measured plain service times.  Both cut their plain-path
measurement after --plain-budget-s seconds.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "EG solve GTEPS (n=2^20, Zipf(2) out-degree, int64 credits)"
METRICS = {"cfg1": "EG solve GTEPS (n=1000, 4 successors, int64 credits)", "cfg2": METRIC,
           "cfg3": "EG solve GTEPS (n=2000 clique, int64 credits)"}
UNIT = "GTEPS"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"], default="cfg2")
    ap.add_argument("--games", type=int, default=64,
                    help="cfg4: the first G games of the 4096-game stream (same seeds)")
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="cfg4: (game, threshold) pairs timed on the plain path (0: all pairs of the batch)")
    ap.add_argument("--plain-pair-timeout-s", type=float, default=120.0,
                    help="cfg4: device-side limit of one plain solve (a pair at the limit counts at its limit)")
    ap.add_argument("--batch-timeout-s", type=float, default=120.0,
                    help="cfg4: device-side limit of one batched solve (games still running stop)")
    ap.add_argument("--plain-budget-s", type=float, default=45.0,
                    help="cfg4/cfg5: wall-clock budget of the plain-path measurements")
    ap.add_argument("--requests", type=int, default=48, help="cfg5: requests per arrival rate (at most)")
    ap.add_argument("--rates", type=str, default="2,8,32,128,512", help="cfg5: arrival rates (requests/s) swept")
    ap.add_argument("--n-max", type=int, default=1 << 16, help="cfg5: largest request game")
    ap.add_argument("--n", type=int, default=0, help="override the vertex count (smaller cases)")
    ap.add_argument("--e2e-steps", type=int, default=0, help="e2e steps (default: --steps)")
    ap.add_argument("--cpu-sample-s", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--narrow", action="store_true", help="allow 32-bit device credits where exact")
    ap.add_argument("--tune", action="store_true",
                    help="autotune the layout and dense-round knobs (eg_dgame_tune) before the timed steps "
                         "(the default for single-game workloads without --variant or --max-rounds)")
    ap.add_argument("--no-tune", action="store_true", help="time the solver's default knobs")
    ap.add_argument("--case", choices=["frontier-sparse60", "units-small24", "tail-game26"], default=None,
                    help="profiling case: one small, fixed launch of a kernel for ncu (prints a labelled line, "
                         "not a benchmark)")
    ap.add_argument("--case-rounds", type=int, default=3000, help="sweeps of the tail-game26 case")
    ap.add_argument("--max-rounds", type=int, default=-1,
                    help="profiling aid: cap every solve at this many rounds (the line is then not a benchmark)")
    return ap.parse_args()


def load_workload(name: str, n: int):
    from egsolver_b200 import workloads

    fn = getattr(workloads, name)
    return fn(n) if n else fn()


def workload_config(name: str, game, world: int) -> dict:
    deg = np.diff(game.row_ptr)
    cfg = {"workload": {"cfg1": "random 4-regular game", "cfg2": "single large sparse game",
                        "cfg3": "dense clique game"}[name],
           "n": game.num_nodes, "m": game.num_edges, "max_out_degree": int(deg.max()),
           "mean_out_degree": round(float(deg.mean()), 3), "weights": f"+-{game.max_abs_weight}",
           "credits": "int64", "seed": "0xE6+cfg", "l2": "flushed (256 MB write) before every step",
           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
    if name == "cfg2" and game.num_nodes == 1 << 20:
        cfg["degree_law"] = ("floor of a continuous x^-2 law on [1, 4097), clipped to [1, 4096]: mean 7.9 and "
                             "m = 8,309,547, against the configuration's approximate 8.4M")
    return cfg


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def full_size_pin(name: str, game):
    """The committed Jacobi pin of this workload (sweeps of the full solve), if any."""
    p = ROOT / "tests" / "golden" / f"{name}_full_size.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    if d.get("n") != game.num_nodes or d.get("m") != game.num_edges or "sweeps" not in d:
        return None
    return d


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.lines: list[str] = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dense_round_bytes(game, credit_bytes: int) -> int:
    """Algorithmic bytes of one dense sweep, by the per-edge and per-vertex
    figures of the workload's definition: per scanned edge its successor id
    (4 B), weight (4 B) and the successor's credit (S); per lifted vertex its
    two row offsets (8 B) and its own credit (S).  A raised credit's write (S)
    is added from the raise count.  Layout overheads of the kernel (padding
    pairs, chunk metadata) are not counted."""
    S = credit_bytes
    return game.num_edges * (8 + S) + game.num_nodes * (8 + S)


def lift_traffic_bytes(st, credit_bytes: int) -> float:
    """Algorithmic bytes of the frontier kernel's rounds:
    per scanned edge: successor 4 + weight 4 + successor credit S;
    per lifted vertex: two row offsets 8 + own credit S;
    per raised credit: the write S + two CSC offsets 8;
    per predecessor pushed: its id 4 + its frontier word 4."""
    S = credit_bytes
    return (st.edges * (8 + S) + st.lifts * (8 + S) + st.changes * (S + 8) + st.pushes * 8)


def cpu_sample(game, seconds: float, kind_pref: str = "reference"):
    """Times the reference worklist solver on its first P pops of `game`.
    Returns (gteps, edges, secs, pops, kind)."""
    from oracle import oracle as O

    use_ref = kind_pref == "reference" and O.ref_available()
    # calibrate P with the restatement (same pop sequence as the reference)
    P = 2_000_000
    _, st = O.eg_solve(game, bits=32, max_loop_=P)
    t0 = time.perf_counter()
    _, st = O.eg_solve(game, bits=32, max_loop_=P)
    dt = time.perf_counter() - t0
    P = max(P, int(P * seconds / max(dt, 1e-3)))
    _, st = O.eg_solve(game, bits=32, max_loop_=P)  # edges of exactly these pops (untimed)
    edges = st["edges"]
    if use_ref:
        _, rst = O.ref_cpu_solve(game, "eg", threads=1, max_loop_=P)
        secs = rst["seconds"]  # the reference's own solving time (cpu_solver(), transpose included)
    else:
        t0 = time.perf_counter()
        O.eg_solve(game, bits=32, max_loop_=P)
        secs = time.perf_counter() - t0
    return edges / secs / 1e9, edges, secs, P, "reference" if use_ref else "port"


def cpu_sample_omp(game, seconds: float):
    """Times the reference's own OpenMP EG0 (Jacobi sweeps, cpu_solver.c
    EG0_cpu_solver, compiled unmodified) on all host cores for its first S
    sweeps of `game`; every sweep scans all m edges.  Its inner index is
    shared between threads (reference src/cpu_solver.c:111,146-157), so its
    credits after the S sweeps are compared with the race-free restatement's
    after the same S sweeps (Jacobi sweeps are deterministic): a mismatch
    marks the timing invalid.  Returns (gteps, S, secs, threads, valid)."""
    from oracle import oracle as O

    # the reference indexes a per-thread array sized MAX_THREADS (256 in
    # oracle/Makefile) by the thread id
    threads = min(os.cpu_count() or 1, 256)
    S = 4
    _, st = O.ref_cpu_solve(game, "eg0", threads=threads, max_loop_=S)
    S = max(S, int(S * seconds / max(st["seconds"], 1e-3)))
    f_ref, st = O.ref_cpu_solve(game, "eg0", threads=threads, max_loop_=S)
    f_fix, _ = O.eg0_solve(game, threads=threads, max_loop_=S)
    valid = bool(np.array_equal(f_ref, f_fix))
    return game.num_edges * S / st["seconds"] / 1e9, S, st["seconds"], threads, valid


def time_to_solution(name: str, game, omp_sweeps: int, omp_secs: float, threads: int, valid: bool):
    """Projected full-solve time of the reference's OpenMP EG0 on this box:
    the committed pin's sweep count x the measured time per sweep."""
    pin = full_size_pin(name, game)
    if pin is None or omp_sweeps <= 0:
        return None
    per_sweep = omp_secs / omp_sweeps
    return {"reference_eg0_projected_s": pin["sweeps"] * per_sweep, "sweeps": pin["sweeps"],
            "per_sweep_ms": 1e3 * per_sweep, "threads": threads, "eg0_output_valid": valid,
            "how": "sweeps of the full Jacobi solve (committed pin tests/golden/" + name + "_full_size.json) x "
                   "the reference EG0's measured time per sweep on this box's cores"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import oracle as O

    # the game comes from the oracle's restated generator: this arm loads no
    # part of the solver library
    game = O.workload(args.workload, args.n)
    use_ref = O.ref_available()
    # every step is a bounded sample of the workload, sized so that all
    # warm-up and timed steps take about a minute together
    seconds = max(0.5, 60.0 / max(1, args.warmup + args.steps))
    P = 1_000_000
    t0 = time.perf_counter()
    _, st = O.eg_solve(game, bits=32, max_loop_=P)
    dt = time.perf_counter() - t0
    P = max(P, int(P * seconds / max(dt, 1e-3)))
    _, st = O.eg_solve(game, bits=32, max_loop_=P)
    edges = st["edges"]

    def step():
        # the reference's own "Solving time" (cpu_solver(), transpose included)
        if use_ref:
            _, rst = O.ref_cpu_solve(game, "eg", threads=1, max_loop_=P)
            return rst["seconds"]
        t = time.perf_counter()
        O.eg_solve(game, bits=32, max_loop_=P)
        return time.perf_counter() - t

    with stdout_to_stderr():
        for _ in range(args.warmup):
            step()
        times = [step() for _ in range(args.steps)]
        tts = None
        if use_ref and full_size_pin(args.workload, game) is not None:
            _, S, osecs, th, valid = cpu_sample_omp(game, 10.0)
            tts = time_to_solution(args.workload, game, S, osecs, th, valid)
    total = sum(times)
    value = edges * args.steps / total / 1e9
    kind = "reference" if use_ref else "port"
    line = {"impl": "reference", "metric": METRICS[args.workload], "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": workload_config(args.workload, game, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "cpu_model": cpu_model(),
                             "omp_num_threads": os.environ.get("OMP_NUM_THREADS", "unset"),
                             "sample": f"first {P} worklist pops of EG_cpu_solver (reference --eg {P}) on the "
                                       f"same game, {edges} edges relaxed per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "time_to_solution": tts}
    print(json.dumps(line), flush=True)


class stdout_to_stderr:
    """Sends file descriptor 1 to stderr for the duration: the reference's C
    solvers print progress lines, and stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def reduce_over_ranks(dist, dev_ms: float, edges: float, device: str) -> tuple[float, float]:
    """Whole-job figures of N replicas: the slowest rank's device time and
    the edges of all ranks (dist None: this process alone)."""
    if dist is None:
        return float(dev_ms), float(edges)
    import torch

    t = torch.tensor([float(dev_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e = torch.tensor([float(edges)], dtype=torch.float64, device=device)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


def progress(msg: str) -> None:
    """A progress line on stderr (the JSON result line stays alone on stdout)."""
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def run_batched(args):
    """cfg4: many uneven games x K=8 mean-payoff thresholds in one solve
    (autotuned CTA size) against the plain path that launches the
    single-game solver once per (game, threshold), on the same pairs: every
    pair of the first --games games (--plain-sample 0) or a seeded sample of
    them.  Each plain solve's credits are compared with the batched ones."""
    import egsolver_b200 as eg
    from egsolver_b200 import workloads

    G = args.games
    games = workloads.cfg4_games(G)
    p, d = workloads.cfg4_thresholds(G)
    K = p.shape[1]
    t0 = time.perf_counter()
    # stream launches, not graph replay: a step is one solve of tens of
    # seconds, so there is no launch overhead to save, and on this batch the
    # replayed graph started the tail-class kernels in another order and took
    # 49 to 58 s against 34 s
    b = eg.Batch(games, thresholds=K, scale=d, use_graph=False, timeout_ms=1e3 * args.batch_timeout_s)
    b.set_thresholds(p)
    setup_s = time.perf_counter() - t0
    progress(f"batch of {G} games packed and uploaded in {setup_s:.1f} s")
    block = b.tune()
    progress(f"tuned: block {block}")
    for _ in range(args.warmup):
        _, wst = b.solve(raise_on_error=False)
        progress(f"warm-up solve {wst.solve_ms:.1f} ms, {wst.games_failed} game(s) stopped by the time limit")
    sampler = ClockSampler(0)
    times, stats = [], []
    for _ in range(args.steps):
        _, st = b.solve(raise_on_error=False)
        times.append(st.solve_ms)
        stats.append(st)
        progress(f"timed solve {st.solve_ms:.1f} ms, {st.games_failed} game(s) stopped by the time limit")
    clocks = sampler.stop()
    ms = sum(times) / len(times)
    done = G - max(s.games_failed for s in stats)  # games solved to the fixed point in every step
    value = done / (ms / 1e3)
    batched = {g: b.credits(g) for g in range(G)}
    status = {g: b.game_result(g)[1] for g in range(G)}
    last = stats[-1]
    b.free()
    # the plain path on the same (game, threshold) pairs: one single-game
    # solve each, device time; its credits must equal the batched ones
    from oracle import oracle as O

    rng = np.random.default_rng(0)
    pairs = [(g, k) for g in range(G) for k in range(K)]
    if args.plain_sample > 0 and args.plain_sample < len(pairs):
        pairs = [pairs[i] for i in sorted(rng.choice(len(pairs), size=args.plain_sample, replace=False))]
    plain_ms, capped, mismatch = 0.0, 0, 0
    t_plain = time.perf_counter()
    for i, (g, k) in enumerate(pairs):
        tg = eg.threshold_game(games[g], int(p[g, k]), d)
        with eg.ResidentGame(tg) as r:
            st_, pst = r.solve(raise_on_error=False, timeout_ms=1e3 * args.plain_pair_timeout_s)
            if st_ != 0:
                capped += 1  # counted at its time limit: the plain total is a lower bound
                plain_ms += pst.solve_ms
                continue
            plain_ms += pst.solve_ms
            if status[g] == 0 and not np.array_equal(r.credits(64), batched[g][k]):
                mismatch += 1
        if (i + 1) % 32 == 0:
            progress(f"plain {i + 1}/{len(pairs)} pairs, {plain_ms / 1e3:.1f} s device time so far")
    plain_wall = time.perf_counter() - t_plain
    if mismatch:
        raise RuntimeError(f"{mismatch} plain solves differ from the batched credits")
    plain = (len(pairs) / K) / (plain_ms / 1e3) if plain_ms > 0 else None
    # oracle spot check: every threshold of a few small games
    checked = 0
    for g in sorted(range(G), key=lambda x: games[x].num_nodes)[:4]:
        if status[g] != 0:
            continue
        for k in range(K):
            want, _ = O.eg_solve(eg.threshold_game(games[g], int(p[g, k]), d), bits=64)
            if not np.array_equal(want, batched[g][k]):
                raise RuntimeError(f"batched credits of game {g} threshold {k} differ from the oracle")
        checked += 1
    line = {"metric": f"batched games/s (cfg4 stream, first {G} of 4096 uneven games x {K} mean-payoff thresholds, "
                      "one solve)",
            "value": value, "unit": "games/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "games_solved": done, "batch_timeout_s": args.batch_timeout_s,
            "config": {"workload": "batched uneven games", "games": G, "thresholds": K, "d": d,
                       "total_nodes": last.total_nodes, "total_edges": last.total_edges, "block": block,
                       "units": last.num_units, "graph_replayed": last.graph_replayed, "setup_s": setup_s},
            "thresholds_per_s": value * K, "gteps": last.edges / (last.solve_ms * 1e6),
            "plain": {"games_per_s": plain, "pairs": len(pairs), "of_pairs": G * K, "device_s": plain_ms / 1e3,
                      "wall_s": plain_wall, "pairs_at_time_limit": capped,
                      "pair_time_limit_s": args.plain_pair_timeout_s, "credits_equal_batched": True,
                      "how": "eg_dgame solve per (game, threshold): transpose, layout and lift per pair, device time"},
            "speedup_vs_plain": value / plain if plain else None,
            "oracle_checked_games": checked, "clocks": clocks,
            "solve": {"rounds_max": last.rounds_max, "rounds_sum": last.rounds_sum, "lifts": last.lifts,
                      "edges": last.edges, "num_top": last.num_top, "grid": last.grid}}
    print(json.dumps(line), flush=True)


def run_served(args):
    """cfg5: Poisson arrivals of mean-payoff threshold queries against the
    serving loop, with the arrival rate swept up to saturation; the plain
    reference serves the same arrivals one request at a time (FIFO), each
    request's service time being its measured plain solves (one single-game
    solve per threshold, device time).  Every served result is compared with
    the plain credits."""
    import egsolver_b200 as eg
    from egsolver_b200 import workloads

    reqs = workloads.cfg5_requests(args.requests, n_max=args.n_max)
    rng = np.random.default_rng(11)
    # plain service time of every request: K single-game solves; the stream
    # is cut after the request that exhausts the plain budget, and only the
    # requests measured here are served below
    plain_service, plain_credits = [], []
    t_plain = time.perf_counter()
    for g, p, d in reqs:
        if plain_service and time.perf_counter() - t_plain > args.plain_budget_s:
            break
        t, cr = 0.0, []
        for k in range(len(p)):
            with eg.ResidentGame(eg.threshold_game(g, int(p[k]), d)) as r:
                _, st = r.solve()
                t += st.solve_ms
                cr.append(r.credits(64))
        plain_service.append(t)
        plain_credits.append(np.stack(cr))
        progress(f"plain request {len(plain_service)}: n={g.num_nodes} K={len(p)} {t:.1f} ms")
    reqs = reqs[:len(plain_service)]
    solves = sum(len(p) for _, p, _ in reqs)
    results = []
    for rate in [float(x) for x in args.rates.split(",")]:
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
        with eg.Server() as srv:
            gids = [srv.add_game(g) for g, _, _ in reqs]
            t0 = time.perf_counter()
            qids = []
            for i, (g, p, d) in enumerate(reqs):
                delay = arrivals[i] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                qids.append(srv.submit(gids[i], p, d))
            for q in qids:
                srv.wait(q, 600_000)
            for i, q in enumerate(qids):
                got, _ = srv.result(q)
                if not np.array_equal(got, plain_credits[i]):
                    raise RuntimeError(f"served request {i} differs from its plain solves")
            st = srv.stats()
            spans = srv.trace()
        overlaps = sum(1 for i in range(len(spans)) for j in range(i + 1, len(spans))
                       if spans[j]["begin_ms"] < spans[i]["end_ms"] and spans[i]["begin_ms"] < spans[j]["end_ms"])
        progress(f"rate {rate}: {st['solves_per_s']:.1f} solves/s, p50 {st['latency_p50_ms']:.1f} ms, "
                 f"p99 {st['latency_p99_ms']:.1f} ms, {len(spans)} micro-batches, {overlaps} overlapping pairs")
        # the same arrivals served one request at a time
        fin, lat = 0.0, []
        for a, s_ in zip(arrivals, plain_service):
            start = max(a, fin)
            fin = start + s_ / 1e3
            lat.append((fin - a) * 1e3)
        results.append({"rate": rate, "p50_ms": st["latency_p50_ms"], "p99_ms": st["latency_p99_ms"],
                        "solves_per_s": st["solves_per_s"], "micro_batches": st["micro_batches"],
                        "overlapping_micro_batch_pairs": overlaps,
                        "plain_p50_ms": float(np.percentile(lat, 50)), "plain_p99_ms": float(np.percentile(lat, 99)),
                        "plain_solves_per_s": solves / fin})
    best = max(results, key=lambda r: r["solves_per_s"])
    plain_best = solves / (sum(plain_service) / 1e3)  # back-to-back plain solves: its saturated rate
    line = {"metric": "served threshold solves/s with p50/p99 latency (cfg5, Poisson arrivals)",
            "value": best["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": len(results), "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": "served threshold queries", "requests": len(reqs), "n_max": args.n_max,
                       "rates": args.rates, "thresholds": solves},
            "plain_saturated_solves_per_s": plain_best, "speedup_vs_plain": best["solves_per_s"] / plain_best,
            "results_equal_plain": True, "sweep": results}
    print(json.dumps(line), flush=True)


def run_case(args):
    """Small fixed launches for kernel profiles (ncu).  Each prints one JSON
    line labelled "profiling_case"; none is a benchmark number."""
    import egsolver_b200 as eg
    from egsolver_b200 import workloads

    out = {"profiling_case": args.case}
    if args.case == "frontier-sparse60":
        # one launch of the frontier kernel: 60 sparse rounds on the cfg2 shape at n = 2^18
        r = eg.ResidentGame(workloads.cfg2(1 << 18))
        st, s = r.solve(direction=eg.DIRECTION_SPARSE, max_rounds=60, raise_on_error=False)
        out.update(rounds=s.rounds, lift_ms=s.lift_ms, edges=s.edges, lifts=s.lifts, changes=s.changes,
                   pushes=s.pushes, grid=s.grid, block=s.block)
        r.free()
    elif args.case == "units-small24":
        # phase 1 of a batch of the 24 first cfg4 games with n <= 6000, 8 thresholds, 300 sweeps
        gs = workloads.cfg4_games(64)
        p, d = workloads.cfg4_thresholds(64)
        small = [i for i in range(64) if gs[i].num_nodes <= 6000][:24]
        with eg.Batch([gs[i] for i in small], thresholds=8, scale=d, max_rounds=300) as b:
            b.set_thresholds(p[small])
            st, s = b.solve(raise_on_error=False)
            out.update(ms=s.solve_ms, edges=s.edges, units=s.num_units, smem=s.smem_bytes)
    else:
        # one (game, threshold) on the cluster tail: cfg4 game 26 (n = 32,472) at its highest threshold
        gs = workloads.cfg4_games(64)
        p, d = workloads.cfg4_thresholds(64)
        k = int(np.argmax(p[26]))
        with eg.Batch([gs[26]], thresholds=1, scale=d, max_rounds=args.case_rounds, tail_rows=1) as b:
            b.set_thresholds(p[26:27, k:k + 1])
            st, s = b.solve(raise_on_error=False)
            out.update(ms=s.solve_ms, sweeps=s.rounds_max, us_per_sweep=1e3 * s.solve_ms / max(1, s.rounds_max),
                       tail_ms=s.tail_ms)
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.case:
        run_case(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "cfg4":
        run_batched(args)
        return
    if args.workload == "cfg5":
        run_served(args)
        return
    import torch

    import egsolver_b200 as eg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    game = load_workload(args.workload, args.n)
    credit_bits = 64
    cfg = workload_config(args.workload, game, world)
    if args.variant:
        cfg["variant"] = {1: "thread per vertex", 2: "warp per vertex (32-lane shuffle reductions)",
                          3: "CTA per vertex", 4: "one-CTA shared-memory kernel"}[args.variant]

    res = eg.ResidentGame(game, device=local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}")
    # int64 credits on the device, as the workload specifies (--narrow lets
    # the solver compute in 32 bits where that is exact)
    kw = dict(credit_bits=credit_bits, device=local, variant=args.variant, max_rounds=args.max_rounds,
              narrow=args.narrow)
    capped = args.max_rounds >= 0
    tuned = None
    # the autotuner is part of the solver: it runs once per game, outside
    # the timed region, and the line reports the knobs it chose
    if args.tune or (not args.no_tune and not args.variant and not capped):
        knobs, rep = res.tune(rounds=300, **kw)
        kw.update(knobs)
        tuned = {"knobs": knobs, **rep}
        progress(f"tuned: {knobs} ({rep['candidates']} capped solves, {rep['default_rate']:.0f} -> "
                 f"{rep['best_rate']:.0f} edges/ms)")
    for _ in range(args.warmup):
        flush.fill_(1)
        torch.cuda.synchronize()
        res.solve(raise_on_error=not capped, **kw)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    stats = []
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        _, st = res.solve(raise_on_error=not capped, **kw)
        stats.append(st)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    dev_ms = sum(s.solve_ms for s in stats)
    edges = sum(s.edges for s in stats)
    lift_ms = sum(s.lift_ms for s in stats)
    launches = sum(s.kernel_launches for s in stats)
    # correctness guard on the last timed solve: a fixed point of the lifting operator
    credits = res.credits(64)
    res.free()
    dev_ms_max, edges_all = reduce_over_ranks(dist, dev_ms, edges, f"cuda:{local}")
    value = edges_all / (dev_ms_max / 1e3) / 1e9

    # e2e through the one-call API with pinned host buffers
    e2e = None
    if not args.no_e2e and not capped:
        pin_rp = torch.from_numpy(game.row_ptr).pin_memory()
        pin_sc = torch.from_numpy(game.succ).pin_memory()
        pin_wt = torch.from_numpy(game.weight).pin_memory()
        pgame = eg.Game(row_ptr=pin_rp.numpy(), succ=pin_sc.numpy(), weight=pin_wt.numpy(),
                        num_nodes0=game.num_nodes0, max_abs_weight=game.max_abs_weight)
        assert pgame.row_ptr.ctypes.data == pin_rp.data_ptr()
        out = torch.empty(game.num_nodes, dtype=torch.int64).pin_memory()
        import ctypes

        cg = pgame.c_struct()
        opts = eg.make_opts(**kw)
        est = eg._ffi.EgStats()
        k = args.e2e_steps or args.steps
        e_edges, e_secs = 0, 0.0
        for i in range(k + 1):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s = eg.lib().eg_solve_i64(ctypes.byref(cg), ctypes.byref(opts), out.data_ptr(), ctypes.byref(est))
            dt = time.perf_counter() - t0
            if s != 0:
                raise RuntimeError(eg.lib().eg_last_error().decode())
            if i > 0:  # first call warms the allocator / module load
                e_edges += est.edges
                e_secs += dt
        if not np.array_equal(out.numpy(), credits):
            raise RuntimeError("e2e credits differ from the resident solve")
        h2d = game.row_ptr.nbytes + game.succ.nbytes + game.weight.nbytes
        # whole job: all ranks' edges over the slowest rank's time
        e_ms_max, e_edges_all = reduce_over_ranks(dist, 1e3 * e_secs, e_edges, f"cuda:{local}")
        e2e = {"value": e_edges_all / (e_ms_max / 1e3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(game.num_nodes * 8), "steps": k,
               "ms_per_step": e_ms_max / k}

    from oracle import oracle as O  # the checker, outside every timed region

    bad = 0 if capped else O.count_inconsistent(game, credits)
    if bad:
        raise RuntimeError(f"{bad} vertices are not at a fixed point after the solve")

    last = stats[-1]
    peak, peak_kind = measured_peak()
    S = credit_bits // 8
    traffic = None
    if last.dense_rounds > 0 and last.dense_ms > 0:
        # the dense-round kernel: mean over its launches in the timed steps
        d_rounds = sum(s.dense_rounds for s in stats)
        d_launch = sum(s.dense_launches for s in stats)
        d_bytes = d_rounds * dense_round_bytes(game, S) + sum(s.dense_changes for s in stats) * S
        d_ms = sum(s.dense_ms for s in stats)
        per_launch = d_bytes / d_launch
        achieved = d_bytes / (d_ms / 1e3) / 1e9
        kernel = "k_lift_dense (persistent dense-round kernel)"
        tf = ROOT / "profiles" / "k_lift_dense_traffic.json"
        if tf.exists():
            try:
                d = json.loads(tf.read_text())
                if d.get("workload") == cfg["workload"] and d.get("n") == game.num_nodes:
                    traffic = d["dram_bytes_per_sweep"] * d_rounds / d_launch
            except (ValueError, KeyError):
                traffic = None
        extra = {"launches": d_launch, "sweeps_per_launch": d_rounds / d_launch,
                 "ms_per_launch": d_ms / d_launch, "bytes_per_sweep": dense_round_bytes(game, S)}
    else:
        per_launch = lift_traffic_bytes(last, S)
        achieved = per_launch / (last.lift_ms / 1e3) / 1e9
        kernel = "k_lift (persistent frontier kernel)"
        extra = {}
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "kernel": kernel, "algorithmic_bytes_per_launch": per_launch, **extra}

    cpu = cpu_omp = tts = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with stdout_to_stderr():
            g, ed, secs, P, kind = cpu_sample(game, args.cpu_sample_s)
        cpu = {"value": g, "unit": UNIT, "cores": 1, "kind": kind, "cpu_model": cpu_model(),
               "omp_num_threads": os.environ.get("OMP_NUM_THREADS", "unset"),
               "sample": f"first {P} worklist pops of EG_cpu_solver (reference --eg {P}) on the same game: "
                         f"{ed} edges in {secs:.2f} s"}
        if kind == "reference":
            with stdout_to_stderr():
                og, S, osecs, th, valid = cpu_sample_omp(game, args.cpu_sample_s / 2)
            cpu_omp = {"value": og if valid else None, "unit": UNIT, "cores": th, "kind": "reference",
                       "valid": valid, "measured_gteps": og,
                       "sample": f"first {S} sweeps of the reference's OpenMP EG0_cpu_solver (--eg0, {th} threads): "
                                 f"{S} x m edges in {osecs:.2f} s; its credits after these sweeps "
                                 f"{'equal' if valid else 'DIFFER from'} the race-free restatement's"}
            tts = time_to_solution(args.workload, game, S, osecs, th, valid)
            if tts is not None:
                tts["gpu_solve_s"] = dev_ms_max / args.steps / 1e3
                if e2e is not None:
                    tts["gpu_e2e_s"] = e2e["ms_per_step"] / 1e3
                    tts["speedup_e2e_vs_reference_eg0"] = tts["reference_eg0_projected_s"] / tts["gpu_e2e_s"]

    if rank == 0:
        if capped:
            cfg["profiling_cap_rounds"] = args.max_rounds
        line = {"metric": METRICS[args.workload], "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": f"int{last.credit_bits}", "data": "synthetic",
                "config": cfg,
                "roofline": roofline, "cpu_baseline": cpu, "cpu_baseline_omp": cpu_omp, "e2e": e2e,
                "time_to_solution": tts, "tuned": tuned,
                "gpu_launches": int(launches),
                "clocks": clocks,
                "solve": {"rounds": last.rounds, "lifts": last.lifts, "edges": last.edges, "changes": last.changes,
                          "pushes": last.pushes, "num_top": last.num_top, "mg": last.mg,
                          "solve_ms": last.solve_ms, "lift_ms": last.lift_ms, "grid": last.grid,
                          "block": last.block, "dense_rounds": last.dense_rounds,
                          "dense_launches": last.dense_launches, "wall_s_timed": t_wall}}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
