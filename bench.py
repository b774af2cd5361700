"""Benchmark: optimal solves/s of uniformly random cubes on the d4t table, batched, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl reference]

One step = one batched solve (libccs persistent launch) of B uniformly random cubes (seeded)
against the d4t table resident in HBM.  The table is built on the GPU first (untimed, its build
time is reported).  ``value`` = cubes / device time of the search launches (CUDA events on the
library's stream), max over ranks; ``e2e`` = the same through the public API
(``GpuSolver.solve`` with host CubieState lists: packing, host->device copy, search,
device->host copy of the results, host verification of every solution).  ``plain`` = one cube
per call (the drop-in path), with p50 / p99 per-cube latency.  Under torchrun each rank is an
independent replica on its own GPU with its own cubes (weak scaling, no collective on the data
path; NCCL only for the barrier and the max-over-ranks timing).

``--impl reference``: the reference's method on the host's CPU cores -- the CPU oracle's IDA*
(oracle/ccs_oracle.c, a restatement of the reference's search) over the same cubes and table,
rank 0 only, bounded to a short sample.
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
sys.path.insert(0, str(ROOT / "cuda-cube-solver_b200"))

METRIC = "optimal solves/s (uniform random cubes, d4t) batched vs plain; p50/p99 latency"
SECTOR = 32  # bytes of one table probe (one 32-byte DRAM sector)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clock / throttle samples taken while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int, local: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n_total: int, world: int, rank: int) -> slice:
    """Replicas: rank r takes cubes [r * n, (r + 1) * n) of the seeded stream."""

    return slice(rank * n_total, (rank + 1) * n_total)


def cpu_arm(args, states, frames_words, table: np.ndarray, probes_per_cube: float | None) -> dict:
    """The reference's method on host cores: the CPU oracle's IDA* over the cubes, all threads,
    bounded by ``args.cpu_budget`` seconds.  Throughput counts finished cubes plus the unfinished
    ones' work in cube units (their probes / mean probes of a cube)."""

    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle

    o = Oracle()
    o.set_kind(args.kind)
    threads = os.cpu_count() or 1
    n = min(len(frames_words), max(threads * 2, 8))
    t0 = time.perf_counter()
    lengths, _, _, probes = o.solve_many(table, args.format, frames_words[:n], threads=threads,
                                        budget_s=args.cpu_budget)
    dt = time.perf_counter() - t0
    done = lengths >= 0
    per_cube = probes_per_cube or (float(probes[done].mean()) if done.any() else None)
    units = float(done.sum()) + (float(probes[~done].sum()) / per_cube if per_cube else 0.0)
    return {"value": units / dt, "unit": "cubes/s", "cores": threads, "kind": "port",
            "sample": f"first {n} cubes of the workload, CPU oracle IDA* (oracle/ccs_oracle.c) on {threads} threads for "
                      f"{dt:.1f} s: {int(done.sum())} solved, unfinished work counted at "
                      f"{per_cube / 1e6 if per_cube else 0:.1f} M probes per cube",
            "probes_per_s": float(probes.sum()) / dt, "probes_per_cube": per_cube}


def reference_cpu_gather(probes_per_cube: float | None) -> dict | None:
    """The reference's own CPU probe benchmark (its bench/cpu_gather.c, compiled from its checkout
    into oracle/_ref/): random byte lookups in a 7.3 GiB buffer on all host threads and on one,
    each bounded to a few seconds; with the search's probes per cube it bounds what a CPU search
    could reach."""

    exe = ROOT / "oracle" / "_ref" / "cpu_gather"
    if not exe.exists():
        return None
    out = {"source": "reference bench/cpu_gather.c", "gib": 7.3}
    for threads, iters in ((os.cpu_count() or 1, 400000), (1, 1000000)):
        try:
            line = subprocess.run([str(exe), "7.3", str(threads), str(iters)], capture_output=True, text=True,
                                  timeout=120).stdout.strip()
            rate = float(line.split()[-3]) * 1e9
        except (subprocess.SubprocessError, ValueError, IndexError):
            return None
        out[f"lookups_per_s_{'all' if threads > 1 else 1}"] = rate
        out["threads"] = out.get("threads", threads)
    if probes_per_cube:
        out["cubes_per_s_bound"] = out["lookups_per_s_all"] / probes_per_cube
    return out


def served_stream(args, solver, opts) -> dict:
    """Config 5: Poisson arrivals (seed 3) into the continuous-batching server on the resident
    table: 90% uniform cubes, 9% uniform cubes whose optimal length is >= 18, 1% superflips."""

    from cuda_cube_solver import serving, workloads

    n = args.serve
    rng = np.random.default_rng(3)
    pool = workloads.uniform_cubes(n + 200, seed=30)
    hard_pool = workloads.uniform_cubes(4 * n // 10 + 16, seed=31)
    lengths = [len(s.moves) for s in solver.solve(hard_pool)]  # set-up: find the long ones
    hard = [c for c, L in zip(hard_pool, lengths) if L >= 18]
    kinds_ = rng.choice(3, size=n, p=[0.90, 0.09, 0.01])
    cubes, hi, ui = [], 0, 0
    for k in kinds_:
        if k == 2:
            cubes.append(workloads.superflip())
        elif k == 1 and hi < len(hard):
            cubes.append(hard[hi])
            hi += 1
        else:
            cubes.append(pool[ui])
            ui += 1
    arrivals = serving.poisson_arrivals(n, args.serve_rate, seed=3)
    srv = serving.Server(solver.handle, 1024, opts, flip_rule=solver.flip_rule if solver.second_kind else None)
    try:
        stats = serving.replay(srv, cubes, arrivals)
    finally:
        srv.close()
    results = stats.pop("results")
    from cuda_cube_solver.solver import verify_solutions
    from cuda_cube_solver.device import state_words

    assert verify_solutions(state_words(cubes), [r.moves for r in results])
    # the same cubes in one batched solve (untimed): every served length must equal it
    batched = [len(sol.moves) for sol in solver.solve(cubes)]
    lat = np.array([r.latency_s for r in results])
    per_kind = {}
    for code, name in ((0, "uniform"), (1, "length_ge_18"), (2, "superflip")):
        sel = lat[kinds_ == code]
        if len(sel):
            per_kind[name] = {"p50_s": float(np.percentile(sel, 50)), "p95_s": float(np.percentile(sel, 95)),
                              "max_s": float(sel.max())}
    stats.update({"lengths_equal_to_batched": [r.length for r in results] == batched, "latency_by_kind": per_kind,
                  "slots": 1024, "search_state_bytes": 1024 * (416 + 5 * 8),
                  "mix": {"uniform": int((kinds_ == 0).sum()), "length_ge_18": int((kinds_ == 1).sum()),
                          "superflip": int((kinds_ == 2).sum())},
                  "rate_per_s": args.serve_rate, "table": config_table(args),
                  "second_table": solver.second_kind, "flip_rule": solver.flip_rule if solver.second_kind else None})
    return stats


def batched_mix(args, solver, opts) -> dict:
    """Config 4: one batch of ``--batch`` cubes in which 5% are hard positions -- uniform cubes of
    seed 20 whose optimal length is >= 19 (found by set-up solves) and the superflip -- solved on
    d4t and, with the second table attached, on d4.  Device time of each batch; the two tables
    must give the same optimal lengths."""

    from cuda_cube_solver import workloads
    from cuda_cube_solver.device import state_words

    n = args.batch
    n_hard = max(2, n * 5 // 100)
    cubes = workloads.uniform_cubes(n, seed=args.seed + 500)
    cand = workloads.uniform_cubes(n_hard * 40, seed=20)
    lengths = [len(sol.moves) for sol in solver.solve(cand)]  # set-up: find the long ones
    hard = [c for c, L in zip(cand, lengths) if L >= 19][: n_hard - 1] + [workloads.superflip()]
    where = np.random.default_rng(4).choice(n, size=len(hard), replace=False)
    for i, c in zip(where, hard):
        cubes[int(i)] = c
    words = state_words(cubes)
    out = {"cubes": n, "hard": len(hard), "length_ge_19": len(hard) - 1, "superflip": 1}
    runs = [("d4t", 0)] + ([(solver.second_kind, 1)] if solver.second_kind else [])
    lens = {}
    for name, tid in runs:
        res = solver.handle.solve(words, opts, np.full(n, tid, np.uint8))
        ms, probes, _ = solver.handle.last_solve_stats()
        lens[name] = [r.length for r in res]
        out[name] = {"cubes_per_s": n / (ms / 1000.0), "probes_per_s": probes / (ms / 1000.0), "ms": ms}
    if len(lens) == 2:
        out["lengths_equal"] = lens["d4t"] == lens[solver.second_kind]
    return out


def build_report(args, solver, peaks) -> dict:
    """The table build of the set-up (GPU BFS + encoding): entries per second and the
    algorithmic DRAM write bandwidth (one depth byte per entry, then the encoded table)."""

    from cuda_cube_solver import native

    nec, entries = native.kind_info(args.kind)
    table_bytes = solver.handle.table_bytes()
    secs = solver.build_seconds
    written = entries + table_bytes
    return {"kind": args.kind, "format": args.format, "gpu_seconds": secs, "entries": entries,
            "entries_per_s": entries / secs, "table_bytes": table_bytes,
            "write_gb_s": written / secs / 1e9, "write_frac_of_hbm": written / secs / 1e9 / float(peaks["hbm_gbs"]),
            "depth_counts": solver.build_counts}


def config_table(args) -> str:
    return args.kind if args.format == "block" else f"{args.kind}-b3"


def reference_gpu_arm(args, states, config) -> dict:
    """The reference's own kernels.cu on this GPU (baseline/ref_gpu.py): its table build and its
    per-bound host loop, the same cubes in chunks of ``--ref-batch`` (its CLI default is 100)."""

    sys.path.insert(0, str(ROOT / "baseline"))
    import ref_gpu

    if not ref_gpu.available():
        return {"impl": "reference-gpu", "unavailable": "baseline/_ref cubins not built (needs the reference checkout)"}
    drv = ref_gpu.Driver(int(os.environ.get("LOCAL_RANK", "0")))
    tables = ref_gpu.RefTables(drv, args.kind)
    ptr, _, counts, build_s = tables.build(args.format)
    solver = ref_gpu.RefSolver(drv, tables, ptr, args.format)
    n = args.batch * args.steps
    work = states[args.batch * args.warmup: args.batch * args.warmup + n]
    solver.solve(states[: args.ref_batch])  # warm-up
    t0 = time.perf_counter()
    nodes = 0
    lengths = []
    for i in range(0, n, args.ref_batch):
        for moves, nd, _ in solver.solve(work[i:i + args.ref_batch]):
            nodes += nd
            lengths.append(len(moves))
    dt = time.perf_counter() - t0
    return {"metric": METRIC, "value": n / dt, "unit": "cubes/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 integer", "data": "synthetic", "config": config,
            "impl": "reference-gpu", "nodes_per_cube": nodes / n, "table_build_s": build_s,
            "lengths_histogram": {str(k): lengths.count(k) for k in sorted(set(lengths))},
            "note": f"reference kernels.cu (unmodified, nvcc sm_100) driven with its host loop, {args.ref_batch} cubes "
                    "per solve call, wall clock including its per-bound host round trips"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=1024, help="cubes per step and rank")
    ap.add_argument("--kind", default="d4t")
    ap.add_argument("--format", default="block", choices=["block", "b3"])
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference", "reference-gpu"])
    ap.add_argument("--ref-batch", type=int, default=100, help="reference-gpu: cubes per solve call (its CLI default)")
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds of CPU work for the CPU baseline: a steady-state window with every thread busy "
                         "(a longer run ends on its single hardest cube with the other threads idle)")
    ap.add_argument("--plain", type=int, default=200, help="cubes solved one per call for the plain numbers")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--variant", type=int, default=0, help="search kernel variant (libccs ccs_solve_opts.variant)")
    ap.add_argument("--serve", type=int, default=400, help="requests in the served-stream measurement (0: skip)")
    ap.add_argument("--tune", action="store_true", help="autotune the kernel settings on a separate sample first")
    ap.add_argument("--serve-rate", type=float, default=100.0, help="Poisson arrival rate of the served stream (/s)")
    ap.add_argument("--second", default=None,
                    help="second resident table for the served stream (default: d4 beside d4t; 'none' for none)")
    ap.add_argument("--no-ceiling", action="store_true", help="skip the random-sector gather ceiling measurement")
    ap.add_argument("--mix", type=int, default=1, help="1: also time one batch with 5%% hard positions on d4t and d4")
    args = ap.parse_args()
    if args.second is None:
        args.second = "d4" if args.kind == "d4t" and args.format == "block" else ""
    elif args.second == "none":
        args.second = ""

    world, rank, local = dist_setup()
    from cuda_cube_solver import native, workloads
    from cuda_cube_solver.device import state_words
    from cuda_cube_solver.solver import GpuSolver, frames

    n_steps_cubes = args.batch * (args.warmup + args.steps)
    all_states = workloads.uniform_cubes(n_steps_cubes * world, seed=args.seed)
    my_states = all_states[shard(n_steps_cubes, world, rank)]
    config = {"workload": f"uniform random cubes (seed {args.seed}), {args.kind} {args.format} table resident in HBM, "
                          f"{args.batch} cubes per step per GPU",
              "table": args.kind if args.format == "block" else f"{args.kind}-b3", "batch": args.batch,
              "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (7.8 GB table, random probes)"}

    if args.impl == "reference-gpu":
        if rank != 0:
            return
        print(json.dumps(reference_gpu_arm(args, my_states, config)))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        h = native.Handle(local)
        h.build_table(args.kind, args.format, None, keep_resident=True)
        table = h.table_copy()
        h.close()
        fr = np.stack([state_words(frames(s)).reshape(30) for s in my_states[: 4 * (os.cpu_count() or 1)]])
        cpu = cpu_arm(args, my_states, fr, table, None)
        out = {"metric": METRIC, "value": cpu["value"], "unit": "cubes/s", "n_gpus": 1, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": 1000.0 * args.batch / cpu["value"] if cpu["value"] else None,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 integer",
               "data": "synthetic", "config": config, "impl": "reference",
               "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
               "e2e": {"value": cpu["value"], "unit": "cubes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
               "reference_cpu_gather": reference_cpu_gather(cpu.get("probes_per_cube"))}
        print(json.dumps(out))
        return

    # ---- setup (untimed): build the table on this GPU, keep it resident ----
    t = time.perf_counter()
    solver = GpuSolver.build_resident(args.kind, args.format, device=local)
    build_s = time.perf_counter() - t
    h = solver.handle
    solver.variant = args.variant
    solver.use_autotune = False
    tuned = None
    if args.tune:  # set-up: its own cubes (seed + 1000), not the timed ones
        tuned = solver.autotune(workloads.uniform_cubes(args.batch, seed=args.seed + 1000), save=False)
    opts = solver._opts(n=args.batch)
    batches = [state_words(my_states[i * args.batch:(i + 1) * args.batch]) for i in range(args.warmup + args.steps)]

    for i in range(args.warmup):
        h.solve(batches[i], opts)

    # ---- timed: K batched steps, device time of the search launches ----
    barrier(world)
    kernel_ms, probes, launches, wall = [], [], [], []
    with ClockSampler(local) as clocks:
        t_all = time.perf_counter()
        for i in range(args.warmup, args.warmup + args.steps):
            t0 = time.perf_counter()
            res = h.solve(batches[i], opts)
            wall.append(time.perf_counter() - t0)
            ms, pr, ln = h.last_solve_stats()
            kernel_ms.append(ms)
            probes.append(pr)
            launches.append(ln)
            assert all(r.status == 0 for r in res)
        t_all = time.perf_counter() - t_all
    barrier(world)
    dev_s = max_over_ranks(sum(kernel_ms) / 1000.0, world, local)
    value = world * args.batch * args.steps / dev_s

    # ---- e2e through the public API: host cubes in, verified Solutions out ----
    barrier(world)
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        sols = solver.solve(my_states[i * args.batch:(i + 1) * args.batch])
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, local)
    e2e = world * args.batch * args.steps / e2e_s

    if rank != 0:
        barrier(world)
        return

    # ---- plain: one cube per call (the drop-in path), per-cube latency: uniform cubes of seed 1 ----
    plain_lat, plain_probes, plain_dev = [], 0, 0.0
    for s in workloads.uniform_cubes(args.plain, seed=1):
        t0 = time.perf_counter()
        solver.solve([s])
        plain_lat.append(time.perf_counter() - t0)
        plain_probes += solver.last_probes
        plain_dev += solver.last_kernel_ms / 1000.0
    plain = None
    if plain_lat:
        plain = {"cubes": len(plain_lat), "workload": "uniform random cubes (seed 1), one per call",
                 "cubes_per_s": len(plain_lat) / sum(plain_lat),
                 "p50_s": float(np.percentile(plain_lat, 50)), "p99_s": float(np.percentile(plain_lat, 99)),
                 "worst_s": max(plain_lat), "probes_per_s": plain_probes / plain_dev if plain_dev else None,
                 "batched_over_plain": value / (len(plain_lat) / sum(plain_lat))}

    if args.second:  # set-up: the second resident table (d4 beside d4t)
        solver.attach_second(args.second)
    mix = batched_mix(args, solver, opts) if args.mix else None
    served = None
    if args.serve:
        served = served_stream(args, solver, opts)

    peaks = measured_peaks()
    total_probes = sum(probes)
    achieved = total_probes * SECTOR / (sum(kernel_ms) / 1000.0) / 1e9
    peak = float(peaks["hbm_gbs"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "probes_per_s": total_probes / (sum(kernel_ms) / 1000.0),
                "probes_per_cube": total_probes / (args.batch * args.steps),
                "peak_source": "measured" if not peaks.get("fallback") else "fallback",
                "note": "algorithmic bytes = 32-byte sector per table probe, counted on the device"}
    if not args.no_ceiling:  # the random 32-byte sector gather ceiling of this GPU (untimed)
        ceiling, _ = native.gather_bench(local, 8 << 30, 64)
        roofline["random_sector_ceiling"] = {"sectors_per_s": ceiling, "gb_s": ceiling * SECTOR / 1e9,
                                             "frac": roofline["probes_per_s"] / ceiling}
    traffic_file = ROOT / "profiles" / "search_traffic.json"
    if traffic_file.exists():
        tr = json.loads(traffic_file.read_text())
        roofline["traffic"] = tr["dram_bytes_per_probe"] * total_probes / max(1, sum(launches))

    cpu = None
    if not args.no_cpu:
        table = h.table_copy()
        fr = np.stack([state_words(frames(s)).reshape(30) for s in my_states[: 4 * (os.cpu_count() or 1)]])
        cpu = cpu_arm(args, my_states, fr, table, roofline["probes_per_cube"])
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    out = {"metric": METRIC, "value": value, "unit": "cubes/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 integer", "data": "synthetic",
           "config": config,
           "e2e": {"value": e2e, "unit": "cubes/s", "h2d_bytes_per_step": 20 * args.batch,
                   "d2h_bytes_per_step": native.ctypes.sizeof(native.Result) * args.batch},
           "gpu_launches": int(sum(launches)),
           "kernel_settings": {"variant": opts.variant, "base_plen": opts.base_plen, "spread": opts.spread,
                               "move_min": opts.move_min, "move_age": opts.move_age, "probe_min": opts.probe_min,
                               "autotuned": tuned is not None},
           "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
           "plain": plain, "batched_mix": mix, "served": served, "table_build_s": build_s, "table_build_gpu_s": solver.build_seconds,
           "table_build": build_report(args, solver, peaks),
           "wall_s_per_step": statistics.mean(wall)}
    print(json.dumps(out))
    barrier(world)


if __name__ == "__main__":
    main()
