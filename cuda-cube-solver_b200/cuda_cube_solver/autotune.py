"""Autotuner for the batched search: picks the launch settings of libccs's search kernel for a
GPU, table and batch size by measuring them.

Knobs (``native.SolveOpts``):

* ``variant``: search kernel and launch shape -- 3 = 256 threads x 3 blocks per SM (the batched
  default), 1 = 256 x 2, 2 = 256 x 2 with sibling lookahead (two probe chains per lane), 8 =
  lookahead 256 x 3, 10 = 224 x 3, 11 = 128 x 5, 6 = 128 x 4 (4 warps per block), 7 = 512 x 1
  (16 warps per block), 9 = 256 x 4 (32 warps per SM);
* ``base_plen``: cut depth of the work items (prefix length of a cube's iterations), 3-6;
* ``move`` = (``move_min``, ``move_age``): how many lanes wait, and for how many iterations,
  before the frame-update pass (push / pop) runs -- the depth of the lanes' update pipeline, 1-16;
* ``steal_depth``: the least slack (moves to the bound beyond a node's largest frame bound) of a
  node whose children a lane donates to idle lanes;
* ``spread``: over how many queued cubes the lanes spread;
* ``probe_min``: a warp keeps probing while at least this many lanes have a probe.

Coordinate descent from the library defaults: each knob in turn takes the value with the best
device time on the sample (the same cubes every time), within a time budget; a value replaces the
incumbent only when it is at least ``MIN_GAIN`` faster, so run-to-run noise on the sample does not
move the settings away from the measured defaults.  Results are cached
in a JSON file keyed by GPU name, table and batch-size bucket, and ``GpuSolver`` picks them up.
"""

from __future__ import annotations

import json
import os
import time
from pathlib import Path

from cuda_cube_solver import native
from cuda_cube_solver.device import state_words

CACHE = Path(os.environ.get("CCS_TUNE_CACHE", Path.home() / ".cache" / "cuda_cube_solver" / "autotune.json"))

SPACE = {
    "variant": [3, 1, 2, 8, 10, 11, 6, 7, 9],
    "base_plen": [3, 4, 5, 6],
    "move": [(1, 1), (4, 2), (8, 4), (16, 8)],
    "steal_depth": [1, 2, 3, 4],
    "spread": [512, 1024, 4096],
    "probe_min": [12, 16, 20, 24],
}
DEFAULT = {"variant": 3, "base_plen": 4, "move": (8, 4), "steal_depth": 2, "spread": 4096, "probe_min": 16}
MIN_GAIN = 0.02  # a setting must cut the sample's device time by 2% to replace the incumbent


def opts_of(cfg: dict, timeout_s: float = 600.0) -> native.SolveOpts:
    return native.solve_opts(base_plen=cfg["base_plen"], variant=cfg["variant"], spread=cfg["spread"],
                             move_min=cfg["move"][0], move_age=cfg["move"][1], timeout_s=timeout_s,
                             probe_min=cfg.get("probe_min", 0), steal_depth=cfg.get("steal_depth", 0))


def batch_bucket(n: int) -> str:
    return "1" if n <= 1 else ("small" if n < 64 else ("medium" if n < 1024 else "large"))


def _key(gpu: str, table: str, n: int) -> str:
    return f"{gpu}|{table}|{batch_bucket(n)}"


def measure(handle: native.Handle, words, cfg: dict) -> float:
    """Device seconds of one batched solve of ``words`` with ``cfg``."""

    handle.solve(words, opts_of(cfg))
    return handle.last_solve_stats()[0] / 1000.0


def tune(handle: native.Handle, states, table: str, rounds: int = 2, log=None, budget_s: float = 0.0) -> dict:
    """Best settings for ``states`` (a representative sample) on the handle's table; with
    ``budget_s`` > 0 the descent stops once that much time has passed (the best so far stands)."""

    words = state_words(states)
    t_start = time.perf_counter()
    best = dict(DEFAULT)
    measure(handle, words, best)  # warm-up
    best_t = measure(handle, words, best)
    trials = [(dict(best), best_t)]
    out_of_time = False
    for _ in range(rounds):
        for knob, values in SPACE.items():
            for v in values:
                if v == best[knob]:
                    continue
                if budget_s > 0 and time.perf_counter() - t_start > budget_s:
                    out_of_time = True
                    break
                cfg = dict(best, **{knob: v})
                t = measure(handle, words, cfg)
                trials.append((cfg, t))
                if log:
                    log(f"{knob}={v}: {len(states) / t:8.1f} cubes/s")
                if t < best_t * (1.0 - MIN_GAIN):
                    best, best_t = cfg, t
    return {"config": best, "cubes_per_s": len(states) / best_t, "trials": len(trials),
            "default_cubes_per_s": len(states) / trials[0][1], "complete": not out_of_time,
            "seconds": time.perf_counter() - t_start, "sample": f"{len(states)} cubes",
            "when": time.strftime("%Y-%m-%dT%H:%M:%S")}


def gpu_name(device: int = 0) -> str:
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def save(result: dict, table: str, n: int, device: int = 0) -> None:
    CACHE.parent.mkdir(parents=True, exist_ok=True)
    data = json.loads(CACHE.read_text()) if CACHE.exists() else {}
    data[_key(gpu_name(device), table, n)] = result
    CACHE.write_text(json.dumps(data, indent=1) + "\n")


def lookup(table: str, n: int, device: int = 0) -> dict | None:
    if not CACHE.exists():
        return None
    cfg = json.loads(CACHE.read_text()).get(_key(gpu_name(device), table, n))
    if cfg:
        cfg = dict(cfg["config"])
        cfg["move"] = tuple(cfg["move"])
    return cfg
