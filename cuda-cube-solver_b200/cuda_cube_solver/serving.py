"""Serving: a request stream through libccs's continuous-batching server.

``Server`` wraps ``ccs_server_*``: requests are admitted into free device slots while other cubes
are searching, and finished cubes come back as soon as they are solved.  ``replay`` drives it with
a timed arrival schedule (e.g. Poisson) and reports per-request latency (submit to result, host
clock) and sustained throughput.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from cuda_cube_solver import native
from cuda_cube_solver.cubie import CubieState
from cuda_cube_solver.device import state_words
from cuda_cube_solver.solver import flipped_edges


@dataclass
class Served:
    request: int
    length: int
    moves: list[int]
    latency_s: float
    device_s: float
    nodes: int


class Server:
    """Continuous batching on one handle (its table must be loaded).  ``flip_rule``: with a second
    table attached, requests with at least this many flipped edges are searched with it.
    ``budget_bytes``: admit cubes by device memory within this budget (tables and the other fixed
    buffers included) instead of by a slot count."""

    def __init__(self, handle: native.Handle, slots: int = 1024, opts: native.SolveOpts | None = None,
                 flip_rule: int | None = None, budget_bytes: int | None = None):
        self.h = handle
        self.flip_rule = flip_rule
        if budget_bytes:
            self.slots = self.h.server_start_budget(budget_bytes, opts or native.solve_opts())
        else:
            self.h.server_start(slots, opts or native.solve_opts())
            self.slots = slots
        self.submitted: dict[int, float] = {}

    def memory(self) -> dict:
        """Budget, fixed footprint, bytes per cube in flight and the peak number in flight."""

        return dict(self.h.server_memory(), slots=self.slots)

    def submit(self, state: CubieState) -> int:
        words = state_words([state])
        table = 0 if self.flip_rule is None else int(flipped_edges(words)[0] >= self.flip_rule)
        rid = self.h.server_submit(words[0], table)
        self.submitted[rid] = time.perf_counter()
        return rid

    def poll(self) -> list[Served]:
        now = time.perf_counter()
        out = []
        for rid, r in self.h.server_poll(256):
            if r.status != 0:
                raise RuntimeError(f"request {rid} failed with status {r.status}")
            out.append(Served(rid, r.length, list(r.moves[: r.length]), now - self.submitted.pop(rid), r.seconds,
                              int(r.nodes)))
        return out

    def close(self) -> None:
        self.h.server_stop()


def poisson_arrivals(n: int, rate: float, seed: int = 3) -> np.ndarray:
    """Arrival times (s) of a Poisson process of ``rate`` per second."""

    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def replay(server: Server, cubes: list[CubieState], arrivals: np.ndarray, timeout_s: float = 600.0) -> dict:
    """Submit ``cubes[i]`` at ``arrivals[i]`` seconds from now; wait for all; latency statistics."""

    t0 = time.perf_counter()
    done: dict[int, Served] = {}
    ids = []
    i = 0
    while len(done) < len(cubes):
        now = time.perf_counter() - t0
        while i < len(cubes) and arrivals[i] <= now:
            ids.append(server.submit(cubes[i]))
            i += 1
        for s in server.poll():
            done[s.request] = s
        if now > timeout_s:
            raise TimeoutError(f"{len(cubes) - len(done)} requests unfinished after {timeout_s} s")
        time.sleep(0.0005)
    elapsed = time.perf_counter() - t0
    lat = np.array([done[r].latency_s for r in ids])
    return {"requests": len(cubes), "offered_per_s": len(cubes) / float(arrivals[-1]) if len(arrivals) else 0.0,
            "sustained_per_s": len(cubes) / elapsed, "p50_s": float(np.percentile(lat, 50)),
            "p95_s": float(np.percentile(lat, 95)), "p99_s": float(np.percentile(lat, 99)), "max_s": float(lat.max()),
            "results": [done[r] for r in ids]}
