"""Benchmark: optimal solves/s of the batched configuration on B200 (d4t table), beside plain
one-at-a-time solving, the served stream and the reference's own builds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference|reference-gpu]

One step = one batched solve through the public API (``GpuSolver.solve``: host cubes in,
verified ``Solution`` objects out) of the batched workload: 4,096 uniform random cubes (seed 2)
in which 5% (205) are replaced by hard positions -- 204 uniform cubes of the seed-20 stream whose
optimal length is >= 19 and the superflip (``workloads.batched_mix``) -- on the d4t block table
resident in HBM (7.8 GB, far larger than L2: every probe is a random 32-byte sector).

* ``value``: cubes / device time of the search launches (CUDA events on the library's stream),
  max over ranks.  ``e2e``: cubes / host wall time of the same ``GpuSolver.solve`` calls, which
  include packing the states, the host->device copies, the search, the device->host copy of the
  results and the host check of every solution.
* The kernel settings come from the autotuner, run untimed on a separate sample first.
* After the timed steps (untimed unless stated): the same batch on d4 (lengths must equal d4t's)
  and with the flip-count rule; 1,024 uniform cubes alone; ``plain`` = 1,000 uniform cubes of
  seed 1 solved one per call (p50 / p99 / worst); the reference's own kernels.cu with its
  per-bound host loop on the same plain cubes (``reference_gpu``; lengths compared); the served
  stream at 10 / 50 / 100 / 200 requests/s within a device-memory budget; the random-sector
  gather ceiling; the CPU baseline.

Under torchrun each rank is an independent replica on its own GPU with its own cubes (weak
scaling; NCCL only for the barrier and the max-over-ranks timing).

``--impl reference``: the reference's method on the host's CPU cores -- the CPU oracle's IDA*
(oracle/ccs_oracle.c, a restatement of the reference's search) over the same cubes, on a table
built by the reference's own BFS kernels (baseline/ref_gpu.py), all host threads, cubes finished
in a fixed window; rank 0 only.  This arm never loads libccs.
``--impl reference-gpu``: the reference's kernels.cu with its host loop on the plain cubes.
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
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900))
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


def rank_seed(seed: int, rank: int) -> int:
    """Replicas: rank 0 solves the configuration's own cubes, rank r > 0 those of seed + 97 r."""

    return seed + 97 * rank


def config_table(args) -> str:
    return args.kind if args.format == "block" else f"{args.kind}-b3"


def workload_config(args, world: int) -> dict:
    n_hard = int(round(args.hard_frac * args.batch))
    if n_hard == 0:
        return {"workload": f"{args.batch} uniform random cubes (seed {args.seed}), {config_table(args)} table "
                            "resident in HBM, one batch per step per GPU", "table": config_table(args),
                "batch": args.batch, "hard": 0, "parallelism": f"replicas{world}"}
    return {"workload": f"batched: {args.batch} uniform random cubes (seed {args.seed}) with {n_hard} (5%) replaced by "
                        f"hard positions ({n_hard - 1} seed-20 uniform cubes of optimal length >= 19 and the superflip), "
                        f"{config_table(args)} table resident in HBM, one batch per step per GPU",
            "table": config_table(args), "batch": args.batch, "hard": n_hard, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (7.8 GB table, random probes)"}


# ---------------------------------------------------------------------------------------------
# CPU side: the oracle's IDA* (the reference's method restated) and the reference's cpu_gather


def cpu_window(kind: str, fmt: str, table: np.ndarray, cubes, seconds: float, threads: int | None = None) -> dict:
    """The oracle's IDA* on host threads over ``cubes`` (in order, each thread taking the next
    cube) for a fixed window; throughput counts the cubes finished in the window only (the work on
    cubes still open when it closes is dropped, which understates the CPU a little)."""

    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle

    from cuda_cube_solver.device import state_words
    from cuda_cube_solver.prefixes import frames

    o = Oracle()
    o.set_kind(kind)
    threads = threads or os.cpu_count() or 1
    fr = np.stack([state_words(frames(s)).reshape(30) for s in cubes])
    t0 = time.perf_counter()
    lengths, _, _, probes = o.solve_many(table, fmt, fr, threads=threads, budget_s=seconds)
    dt = time.perf_counter() - t0
    done = lengths >= 0
    return {"value": float(done.sum()) / dt, "unit": "cubes/s", "cores": threads, "kind": "port",
            "sample": f"the workload's cubes in order, CPU oracle IDA* (oracle/ccs_oracle.c) on {threads} threads for "
                      f"{dt:.1f} s: {int(done.sum())} cubes finished and counted, the cubes still open when the window "
                      f"closed not counted",
            "finished": int(done.sum()), "window_s": dt, "probes_per_s": float(probes.sum()) / dt}


def coordinate_model_baseline(kind: str, seconds: float = 3.0) -> dict:
    """The host Python coordinate model (frames + table index, one cube at a time) on one core and
    on every core (a spawn pool, one process per core, each for ``seconds``)."""

    import multiprocessing as mp

    from cuda_cube_solver import workloads

    n1, t1 = workloads.coordinate_model_rate(kind, seconds)
    cores = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.starmap(workloads.coordinate_model_rate, [(kind, seconds, i) for i in range(cores)])
    return {"source": "cuda_cube_solver.prefixes.frames + coords.table_index (the reference's Python "
                      "coordinate model restated), one cube at a time", "kind": kind,
            "indexes_per_s_1": n1 / t1, "indexes_per_s_all": sum(n for n, _ in res) / max(t for _, t in res),
            "cores": cores, "seconds_per_process": seconds}


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




# ---------------------------------------------------------------------------------------------
# the reference's own GPU build (baseline/ref_gpu.py: its kernels.cu, unmodified, its host loop)


def reference_table(kind: str, fmt: str, device: int) -> tuple[np.ndarray, float]:
    """The solving table built by the reference's own BFS kernels on this GPU, copied to the host."""

    sys.path.insert(0, str(ROOT / "baseline"))
    import ref_gpu

    drv = ref_gpu.Driver(device)
    tables = ref_gpu.RefTables(drv, kind)
    ptr, nbytes, _, secs = tables.build(fmt)
    host = np.empty(nbytes, np.uint8)
    drv.d2h(host, ptr)
    drv.free(ptr)
    return host, secs


def reference_gpu_run(kind: str, fmt: str, states, batch: int, device: int, one_per_call: int = 0) -> dict:
    """The reference's kernels.cu on this GPU with its per-bound host loop, ``batch`` cubes per
    solve call (its CLI default is 100); wall clock, like the reference's own benchmark.  With
    ``one_per_call``, the first that many cubes are also solved one per call (the plain drop-in's
    shape), on the same table."""

    sys.path.insert(0, str(ROOT / "baseline"))
    import ref_gpu

    if not ref_gpu.available():
        return {"unavailable": "baseline/_ref cubins not built (needs the reference checkout at build time)"}
    drv = ref_gpu.Driver(device)
    tables = ref_gpu.RefTables(drv, kind)
    ptr, _, _, build_s = tables.build(fmt)
    solver = ref_gpu.RefSolver(drv, tables, ptr, fmt)
    solver.solve(states[:batch])  # warm-up
    t0 = time.perf_counter()
    nodes, lengths = 0, []
    for i in range(0, len(states), batch):
        for moves, nd, _ in solver.solve(states[i:i + batch]):
            nodes += nd
            lengths.append(len(moves))
    dt = time.perf_counter() - t0
    one = None
    if one_per_call:
        lat, one_len = [], []
        for s in states[:one_per_call]:
            t1 = time.perf_counter()
            (moves, _, _), = solver.solve([s])
            lat.append(time.perf_counter() - t1)
            one_len.append(len(moves))
        one = {"cubes": len(lat), "cubes_per_s": len(lat) / sum(lat), "p50_s": float(np.percentile(lat, 50)),
               "worst_s": max(lat), "lengths": one_len}
    drv.free(ptr)
    return {"cubes": len(states), "cubes_per_s": len(states) / dt, "seconds": dt, "batch": batch,
            "nodes_per_cube": nodes / len(states), "table_build_s": build_s, "lengths": lengths,
            "one_per_call": one,
            "note": f"reference kernels.cu (unmodified, nvcc sm_100) driven with its host loop, {batch} cubes per "
                    "solve call (and one per call for the first cubes), wall clock including its per-bound host "
                    "round trips"}


def presets_run(device: int, n_batch: int, n_plain: int) -> dict:
    """Every preset end to end: GPU build written to a file, the file loaded back (warm page cache:
    the double-buffered pinned copy), then n_batch uniform cubes (seed 2) in one batched solve
    (device time) and n_plain of them one per call; lengths compared across the presets."""

    import shutil
    import tempfile

    from cuda_cube_solver import kinds, native, workloads
    from cuda_cube_solver.device import state_words

    cubes = workloads.uniform_cubes(n_batch, seed=2)
    words = state_words(cubes)
    rows, ref_len = [], None
    tmp = Path(tempfile.mkdtemp(prefix="ccs_presets_"))
    try:
        for p in kinds.PRESETS:
            path = tmp / p.file
            h = native.Handle(device)
            try:
                t0 = time.perf_counter()
                counts, gpu_s = h.build_table(p.kind, p.format, path, keep_resident=False)
                build_wall = time.perf_counter() - t0
                t0 = time.perf_counter()
                h.load_table(p.kind, p.format, path)
                load_s = time.perf_counter() - t0
                res = h.solve(words, native.solve_opts(timeout_s=900))
                ms, probes, _ = h.last_solve_stats()
                lengths = [r.length for r in res]
                lat = []
                for i in range(n_plain):
                    t1 = time.perf_counter()
                    h.solve(words[i:i + 1], native.solve_opts(timeout_s=120))
                    lat.append(time.perf_counter() - t1)
            finally:
                h.close()
                path.unlink(missing_ok=True)
            ref_len = ref_len or lengths
            rows.append({"preset": p.name, "table_gb": p.table_bytes / 1e9, "build_gpu_s": gpu_s,
                         "build_and_write_s": build_wall, "load_s": load_s, "load_gb_s": p.table_bytes / 1e9 / load_s,
                         "batched_cubes_per_s": n_batch / (ms / 1e3), "probes_per_s": probes / (ms / 1e3),
                         "probes_per_cube": probes / n_batch,
                         "plain_cubes_per_s": len(lat) / sum(lat) if lat else None,
                         "plain_p50_s": float(np.percentile(lat, 50)) if lat else None,
                         "lengths_equal_to_first": lengths == ref_len})
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return {"batch": n_batch, "plain": n_plain, "cubes": "uniform random cubes (seed 2)", "presets": rows}


# ---------------------------------------------------------------------------------------------
# arms


def reference_arm(args, world: int, rank: int, local: int) -> None:
    """The reference's method on this host's CPU cores (rank 0 only).  Loads no libccs: the cubes
    and frames come from the host model, the table from the reference's own kernels."""

    if rank != 0:
        return
    from cuda_cube_solver import workloads

    cubes, _ = workloads.batched_mix(args.batch, args.seed, args.hard_frac)
    table, _ = reference_table(args.kind, args.format, local)
    if args.warmup:  # a short warm-up window (page cache, thread start)
        cpu_window(args.kind, args.format, table, cubes[:64], min(2.0, args.cpu_step_s))
    cpu = cpu_window(args.kind, args.format, table, cubes[:1024], args.cpu_step_s * args.steps)
    assert "cuda_cube_solver.native" not in sys.modules, "the reference arm must not load libccs"
    out = {"metric": METRIC, "value": cpu["value"], "unit": "cubes/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000.0 * cpu["window_s"] / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 integer", "data": "synthetic",
           "config": workload_config(args, 1), "impl": "reference",
           "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
           "e2e": {"value": cpu["value"], "unit": "cubes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "finished": cpu["finished"], "window_s": cpu["window_s"],
           "note": "each step is a time slice of one window over the workload's cubes; table from the reference's "
                   "own BFS kernels (baseline/ref_gpu.py) on this GPU",
           "reference_cpu_gather": reference_cpu_gather(None)}
    print(json.dumps(out))


def bfs_roofline(passes: list[dict], entries: int, peak_gbs: float, ceiling: float | None) -> dict:
    """The table build's passes against their rooflines: algorithmic bytes of a pass = one
    sequential scan of the depth bytes (one per entry) + one 32-byte sector per random read and
    per claim; the random sectors also against the random-sector ceiling."""

    rows = []
    for p in passes:
        random = p["random_reads"] + p["claims"]
        algo = entries + SECTOR * random
        rows.append({"depth": p["depth"], "dir": "fwd" if p["forward"] else "bwd", "found": p["found"],
                     "random_sectors": random, "seconds": p["seconds"], "algorithmic_gb": algo / 1e9,
                     "achieved_gb_s": algo / p["seconds"] / 1e9, "random_sectors_per_s": random / p["seconds"]})
    total_s = sum(r["seconds"] for r in rows)
    top = max(rows, key=lambda r: r["seconds"]) if rows else None
    out = {"passes": rows, "bfs_seconds": total_s,
           "dominant_pass": top and {k: top[k] for k in ("depth", "dir", "seconds")},
           "dominant_share": top["seconds"] / total_s if top else None}
    if top:
        out["achieved_gb_s"] = top["achieved_gb_s"]
        out["frac_of_hbm_peak"] = top["achieved_gb_s"] / peak_gbs
        if ceiling:
            # Neighbours of nearby entries share classes, so most of a pass's random accesses hit
            # L2: a rate above the DRAM random-sector ceiling says so, it is not a fraction of it.
            out["random_rate_over_dram_random_ceiling"] = top["random_sectors_per_s"] / ceiling
            out["note"] = ("random accesses costed as 32-byte sectors; a rate above the search's DRAM "
                           "random-sector ceiling means most of them hit L2 (profiles/bfs_s4_dram.md: "
                           "DRAM bytes per pass)")
    return out


def served_stream(args, solver, opts, rates) -> dict:
    """The served stream: Poisson arrivals (seed 3) into the continuous-batching server on the
    resident d4t and d4 tables (flip-count rule), 90% uniform cubes, 9% uniform cubes whose
    optimal length is >= 18, 1% superflips; admission within a stated device-memory budget."""

    from cuda_cube_solver import native, serving, workloads
    from cuda_cube_solver.device import state_words
    from cuda_cube_solver.solver import verify_solutions

    n_max = int(max(rates) * args.serve_s)
    pool = workloads.uniform_cubes(n_max + 64, seed=30)
    hard_pool = workloads.uniform_cubes(n_max // 5 + 64, seed=31)
    hard = [c for c, sol in zip(hard_pool, solver.solve(hard_pool)) if len(sol.moves) >= 18]  # set-up
    out = {"rates": {}, "budget_bytes": args.serve_budget, "table": config_table(args),
           "second_table": solver.second_kind, "flip_rule": solver.flip_rule if solver.second_kind else None,
           "mix": "90% uniform, 9% uniform of optimal length >= 18, 1% superflip (seed 3)"}
    for rate in rates:
        n = int(rate * args.serve_s)
        rng = np.random.default_rng(3)
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
        arrivals = serving.poisson_arrivals(n, rate, seed=3)
        srv = serving.Server(solver.handle, opts=native.solve_opts(variant=args.serve_variant, steal=opts.steal,
                                                                   steal_depth=opts.steal_depth),
                             flip_rule=solver.flip_rule if solver.second_kind else None,
                             budget_bytes=args.serve_budget)
        try:
            stats = serving.replay(srv, cubes, arrivals)
            stats["memory"] = srv.memory()
        finally:
            srv.close()
        results = stats.pop("results")
        assert verify_solutions(state_words(cubes), [r.moves for r in results])
        batched = [len(sol.moves) for sol in solver.solve(cubes)]  # untimed: the same cubes batched
        lat = np.array([r.latency_s for r in results])
        per_kind = {}
        for code, name in ((0, "uniform"), (1, "length_ge_18"), (2, "superflip")):
            sel = lat[kinds_ == code]
            if len(sel):
                per_kind[name] = {"n": int(len(sel)), "p50_s": float(np.percentile(sel, 50)),
                                  "p95_s": float(np.percentile(sel, 95)), "max_s": float(sel.max())}
        stats.update({"lengths_equal_to_batched": [r.length for r in results] == batched,
                      "latency_by_kind": per_kind})
        out["rates"][str(rate)] = stats
    return out


def main_arm(args, world: int, rank: int, local: int) -> None:
    from cuda_cube_solver import native, workloads
    from cuda_cube_solver.device import state_words
    from cuda_cube_solver.solver import GpuSolver

    peaks = measured_peaks()
    config = workload_config(args, world)
    if world > 1:
        # the untimed legs (plain, the reference's kernels, the served stream, the d4 pair, the
        # gather ceiling, the CPU baselines) are one-GPU measurements run by rank 0 while every
        # other rank waits: at N > 1 the line carries the batched step alone
        args.plain, args.ref_gpu, args.serve_s, args.second, args.no_ceiling, args.no_cpu = 0, 0, 0.0, "", True, True

    # ---- set-up (untimed): the table built on this GPU and kept resident; the workload ----
    t = time.perf_counter()
    solver = GpuSolver.build_resident(args.kind, args.format, device=local)
    build_wall_s = time.perf_counter() - t
    h = solver.handle
    build_passes = h.last_build_passes()
    solver.use_autotune = False
    solver.variant = args.variant
    cubes, known = workloads.batched_mix(args.batch, rank_seed(args.seed, rank), args.hard_frac)
    tuned = None
    if args.tune:  # its own cubes: uniform ones of seed + 1000 and hard ones past those of the batch
        info = workloads.hard20()
        n_hard = max(0, int(round(args.hard_frac * args.batch)) - 1)
        extra = workloads.uniform_cubes(info["indices"][-1] + 1, seed=20)
        sample = workloads.uniform_cubes(args.tune_cubes, seed=args.seed + 1000) + \
            [extra[i] for i in info["indices"][n_hard:n_hard + args.tune_hard]]
        tuned = solver.autotune(sample, save=False, budget_s=args.tune_budget, target_n=args.batch)
    opts = solver._opts(n=args.batch)

    for _ in range(args.warmup):
        solver.solve(cubes)

    # ---- timed: K batched steps through GpuSolver.solve ----
    barrier(world)
    kernel_ms, probes, launches, wall, donated = [], [], [], [], []
    lengths = None
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            sols = solver.solve(cubes)
            wall.append(time.perf_counter() - t0)
            ms, pr, ln = h.last_solve_stats()
            kernel_ms.append(ms)
            probes.append(pr)
            launches.append(ln)
            donated.append(h.last_solve_donations())
            step_lengths = [len(s.moves) for s in sols]
            assert lengths is None or step_lengths == lengths, "optimal lengths changed between steps"
            lengths = step_lengths
    barrier(world)
    h2d, d2h = h.last_solve_io_bytes()
    dev_s = max_over_ranks(sum(kernel_ms) / 1000.0, world, local)
    wall_s = max_over_ranks(sum(wall), world, local)
    value = world * args.batch * args.steps / dev_s
    e2e = world * args.batch * args.steps / wall_s
    hard_ok = all(lengths[i] == L for i, L in known.items())

    if rank != 0:
        barrier(world)
        return

    total_probes = sum(probes)
    achieved = total_probes * SECTOR / (sum(kernel_ms) / 1000.0) / 1e9
    peak = float(peaks["hbm_gbs"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "probes_per_s": total_probes / (sum(kernel_ms) / 1000.0),
                "probes_per_cube": total_probes / (args.batch * args.steps),
                "peak_source": "measured" if not peaks.get("fallback") else "fallback",
                "note": "algorithmic bytes = one 32-byte sector per table probe, probes counted on the device; "
                        "achieved over the search launches' CUDA-event time"}
    traffic_file = ROOT / "profiles" / "search_traffic.json"
    if traffic_file.exists():
        tr = json.loads(traffic_file.read_text())
        roofline["traffic"] = tr["dram_bytes_per_probe"] * total_probes / max(1, sum(launches))
        roofline["traffic_source"] = tr.get("source")

    # ---- after the timed region (untimed) ----
    words = state_words(cubes)
    uniform = uniform_full = None
    if world == 1:
        h.solve(state_words(workloads.uniform_cubes(1024, seed=args.seed)), opts)
        ms, pr, _ = h.last_solve_stats()
        uniform = {"cubes": 1024, "workload": f"uniform random cubes (seed {args.seed}) alone",
                   "cubes_per_s": 1024 / (ms / 1e3), "probes_per_s": pr / (ms / 1e3)}
        # the batch size of the timed steps, all of it uniform (the hard positions left out)
        h.solve(state_words(workloads.uniform_cubes(args.batch, seed=args.seed)), opts)
        ms, pr, _ = h.last_solve_stats()
        uniform_full = {"cubes": args.batch, "workload": f"uniform random cubes (seed {args.seed}) alone",
                        "cubes_per_s": args.batch / (ms / 1e3), "probes_per_s": pr / (ms / 1e3)}

    plain = None
    plain_len = None
    plain_states = workloads.uniform_cubes(args.plain, seed=1)
    if args.plain:  # one cube per call through the public API
        lat, pl_probes, pl_dev, plain_len = [], 0, 0.0, []
        for s in plain_states:
            t0 = time.perf_counter()
            sol = solver.solve([s])[0]
            lat.append(time.perf_counter() - t0)
            pl_probes += solver.last_probes
            pl_dev += solver.last_kernel_ms / 1000.0
            plain_len.append(len(sol.moves))
        rate = len(lat) / sum(lat)
        plain = {"cubes": len(lat), "workload": "uniform random cubes (seed 1), one per GpuSolver.solve call",
                 "cubes_per_s": rate, "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                 "worst_s": max(lat), "probes_per_s": pl_probes / pl_dev if pl_dev else None,
                 "batched_over_plain": value / rate, "e2e_batched_over_plain": e2e / rate,
                 "uniform_batched_over_plain": uniform_full["cubes_per_s"] / rate,
                 "uniform_1024_over_plain": uniform["cubes_per_s"] / rate}

    ref_gpu = None
    if args.ref_gpu and args.plain:
        ref_gpu = reference_gpu_run(args.kind, args.format, plain_states, args.ref_batch, local, args.ref_one)
        if "lengths" in ref_gpu:
            ref_gpu["lengths_equal_to_plain"] = ref_gpu.pop("lengths") == plain_len
            ref_gpu["ours_over_reference"] = {"batched": value / ref_gpu["cubes_per_s"],
                                              "e2e": e2e / ref_gpu["cubes_per_s"],
                                              "plain": plain["cubes_per_s"] / ref_gpu["cubes_per_s"]}
            one = ref_gpu.get("one_per_call")
            if one:
                one["lengths_equal_to_plain"] = one.pop("lengths") == plain_len[: one["cubes"]]
                ref_gpu["ours_over_reference"]["plain_over_one_per_call"] = plain["cubes_per_s"] / one["cubes_per_s"]

    # the same batch on d4 (second resident table) and with the flip-count rule
    mix = {config_table(args): {"cubes_per_s": value, "probes_per_s": roofline["probes_per_s"],
                                "hard_lengths_equal_to_known": hard_ok}}
    if args.second:
        solver.attach_second(args.second)
        res = h.solve(words, opts, np.ones(len(words), np.uint8))
        ms, pr, _ = h.last_solve_stats()
        mix[args.second] = {"cubes_per_s": args.batch / (ms / 1e3), "probes_per_s": pr / (ms / 1e3),
                            "lengths_equal": [r.length for r in res] == lengths}
        solver.solve(cubes)
        ms, pr, _ = h.last_solve_stats()
        mix["flip_rule"] = {"rule": f">= {solver.flip_rule} flipped edges -> {args.second}",
                            "cubes_per_s": args.batch / (ms / 1e3), "probes_per_s": pr / (ms / 1e3)}

    served = None
    if args.serve_s > 0:
        served = served_stream(args, solver, opts, [float(r) for r in args.serve_rates.split(",")])
        if plain:
            for st in served["rates"].values():
                st["sustained_over_plain"] = st["sustained_per_s"] / plain["cubes_per_s"]

    ceiling = None
    if not args.no_ceiling:  # the random 32-byte sector gather ceiling of this GPU
        ceiling, _ = native.gather_bench(local, 8 << 30, 64)
        roofline["random_sector_ceiling"] = {"sectors_per_s": ceiling, "gb_s": ceiling * SECTOR / 1e9,
                                             "frac": roofline["probes_per_s"] / ceiling}

    cpu = None
    if not args.no_cpu and world == 1:  # the host-core baselines: rank 0 at one GPU only
        c = cpu_window(args.kind, args.format, h.table_copy(), cubes[:1024], args.cpu_budget)
        cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cpu["reference_cpu_gather"] = reference_cpu_gather(roofline["probes_per_cube"])
        cpu["python_coordinate_model"] = coordinate_model_baseline(args.kind)

    _, entries = native.kind_info(args.kind)
    out = {"metric": METRIC, "value": value, "unit": "cubes/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 integer", "data": "synthetic",
           "config": config,
           "e2e": {"value": e2e, "unit": "cubes/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "api": "GpuSolver.solve (host CubieState list in, verified Solution list out)"},
           "gpu_launches": int(sum(launches)),
           "kernel_settings": {"variant": opts.variant, "base_plen": opts.base_plen, "spread": opts.spread,
                               "move_min": opts.move_min, "move_age": opts.move_age, "probe_min": opts.probe_min,
                               "steal": opts.steal, "steal_depth": opts.steal_depth, "autotuned": tuned is not None,
                               "tuning": {k: tuned[k] for k in ("cubes_per_s", "default_cubes_per_s", "trials",
                                                                 "complete", "seconds", "sample")} if tuned else None},
           "donated_subtrees_per_step": statistics.mean(donated),
           "lengths": {"histogram": {str(k): lengths.count(k) for k in sorted(set(lengths))},
                       "hard_equal_to_known": hard_ok, "equal_across_steps": True},
           "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
           "batched_mix": mix, "uniform_1024": uniform, f"uniform_{args.batch}": uniform_full, "plain": plain, "reference_gpu": ref_gpu, "served": served,
           "table_build": {"kind": args.kind, "format": args.format, "gpu_seconds": solver.build_seconds,
                           "wall_s": build_wall_s, "entries": entries, "entries_per_s": entries / solver.build_seconds,
                           "table_bytes": h.table_bytes(), "depth_counts": solver.build_counts,
                           "roofline": bfs_roofline(build_passes, entries, peak, ceiling)},
           "wall_s_per_step": statistics.mean(wall)}
    print(json.dumps(out))
    barrier(world)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=4096, help="cubes per step and rank")
    ap.add_argument("--hard-frac", type=float, default=0.05, help="share of the batch replaced by hard positions")
    ap.add_argument("--kind", default="d4t")
    ap.add_argument("--format", default="block", choices=["block", "b3"])
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference", "reference-gpu"])
    ap.add_argument("--presets", action="store_true",
                    help="instead of the bench: every preset built, loaded and solved (one JSON line)")
    ap.add_argument("--preset-cubes", type=int, default=512)
    ap.add_argument("--preset-plain", type=int, default=20)
    ap.add_argument("--variant", type=int, default=0, help="search kernel variant (ccs_solve_opts.variant)")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="skip the autotuner (library defaults)")
    ap.add_argument("--tune-budget", type=float, default=60.0, help="seconds of autotuning at most")
    ap.add_argument("--tune-cubes", type=int, default=512)
    ap.add_argument("--tune-hard", type=int, default=8)
    ap.add_argument("--plain", type=int, default=1000, help="cubes solved one per call (0: skip)")
    ap.add_argument("--ref-gpu", type=int, default=1, help="1: time the reference's kernels.cu on the plain cubes")
    ap.add_argument("--ref-batch", type=int, default=100, help="reference kernels: cubes per solve call (its default)")
    ap.add_argument("--ref-one", type=int, default=100,
                    help="reference kernels: also solve this many plain cubes one per call (0: skip)")
    ap.add_argument("--second", default="d4", help="second resident table for the d4 leg and serving ('' for none)")
    ap.add_argument("--serve-s", type=float, default=8.0, help="seconds of arrivals per served rate (0: skip)")
    ap.add_argument("--serve-rates", default="10,50,100,200")
    ap.add_argument("--serve-variant", type=int, default=0, help="server kernel variant (0: automatic)")
    ap.add_argument("--serve-budget", type=int, default=16 << 30,
                    help="device-memory budget of the served stream in bytes (tables, search state, stacks)")
    ap.add_argument("--no-ceiling", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of the CPU baseline window")
    ap.add_argument("--cpu-step-s", type=float, default=6.0, help="reference arm: seconds of CPU work per step")
    args = ap.parse_args()
    if args.format != "block" or args.kind != "d4t":
        args.second = ""  # (d4 beside d4t is the configuration's pair)

    world, rank, local = dist_setup()
    if args.presets:
        if rank == 0:
            print(json.dumps({"mode": "presets", **presets_run(local, args.preset_cubes, args.preset_plain)}))
        return
    if args.impl == "reference":
        reference_arm(args, world, rank, local)
        return
    if args.impl == "reference-gpu":
        if rank != 0:
            return
        from cuda_cube_solver import workloads

        states = workloads.uniform_cubes(args.plain or 1000, seed=1)
        r = reference_gpu_run(args.kind, args.format, states, args.ref_batch, local)
        r.pop("lengths", None)
        print(json.dumps({"metric": METRIC, "value": r.get("cubes_per_s"), "unit": "cubes/s", "n_gpus": 1,
                          "impl": "reference-gpu", "config": {"workload": f"{len(states)} uniform random cubes "
                                                                          "(seed 1), the plain drop-in set"}, **r}))
        return
    main_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
