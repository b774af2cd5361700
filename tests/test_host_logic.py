"""Host logic without a GPU: the autotuner's coordinate descent and its cache, and the served
stream's replay loop and latency statistics, driven by fakes of the library handle and server."""

from __future__ import annotations

import json

import numpy as np

from cuda_cube_solver import autotune, serving, workloads


class FakeHandle:
    """Device time of a solve as a function of the settings, smallest at BEST."""

    BEST = {"variant": 2, "base_plen": 5, "move": (4, 2), "steal_depth": 2, "spread": 1024, "probe_min": 12}

    def __init__(self):
        self.calls = []
        self._ms = 0.0

    def solve(self, words, opts):
        self.calls.append(opts)
        cfg = {"variant": opts.variant, "base_plen": opts.base_plen, "move": (opts.move_min, opts.move_age),
               "steal_depth": opts.steal_depth, "spread": opts.spread, "probe_min": opts.probe_min}
        self._ms = 100.0 + sum(0.0 if cfg[k] == v else 7.0 + abs(hash((k, cfg[k]))) % 5 for k, v in self.BEST.items())
        return []

    def last_solve_stats(self):
        return self._ms, 0, 1


def test_autotune_finds_the_best_settings():
    h = FakeHandle()
    sample = workloads.uniform_cubes(8, seed=9)
    result = autotune.tune(h, sample, "d4t", rounds=2)
    assert result["config"] == FakeHandle.BEST
    assert result["cubes_per_s"] == len(sample) / 0.1
    assert result["trials"] == len(h.calls) - 1  # the first call is the warm-up
    assert result["cubes_per_s"] >= result["default_cubes_per_s"]
    assert result["complete"]


def test_autotune_ignores_gains_within_noise():
    """A setting 1% faster than the incumbent does not replace it (the descent needs MIN_GAIN)."""

    class Flat(FakeHandle):
        def solve(self, words, opts):
            self.calls.append(opts)
            self._ms = 100.0 if opts.base_plen != 5 else 99.0
            return []

    result = autotune.tune(Flat(), workloads.uniform_cubes(4, seed=9), "d4t", rounds=1)
    assert result["config"] == autotune.DEFAULT


def test_autotune_stops_at_its_budget():
    h = FakeHandle()
    result = autotune.tune(h, workloads.uniform_cubes(4, seed=9), "d4t", rounds=2, budget_s=1e-9)
    assert not result["complete"] and result["trials"] == 1 and len(h.calls) == 2
    # the space covers cut depth 3-6, 4-16 warps per block (variants 6, 1, 7) and update depth 1-16
    assert autotune.SPACE["base_plen"] == [3, 4, 5, 6]
    assert {6, 1, 7} <= set(autotune.SPACE["variant"])
    assert [m for m, _ in autotune.SPACE["move"]] == [1, 4, 8, 16]


def test_autotune_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "CACHE", tmp_path / "tune" / "cache.json")
    result = {"config": dict(FakeHandle.BEST, move=list(FakeHandle.BEST["move"])), "cubes_per_s": 1.0}
    autotune.save(result, "d4t", 1000)
    assert autotune.lookup("d4t", 500) == FakeHandle.BEST  # same batch-size bucket (64..1023)
    assert autotune.lookup("d4t", 10) is None  # another bucket
    assert autotune.lookup("d4", 1000) is None  # another table
    data = json.loads((tmp_path / "tune" / "cache.json").read_text())
    assert len(data) == 1 and next(iter(data)).endswith("|d4t|medium")
    assert [autotune.batch_bucket(n) for n in (1, 10, 100, 5000)] == ["1", "small", "medium", "large"]


class FakeServer:
    """Finishes request i after a fixed device latency of (i % 3 + 1) ms of host time."""

    def __init__(self):
        self.t = 0.0
        self.submitted = {}
        self.next_id = 7

    def submit(self, state):
        rid = self.next_id
        self.next_id += 1
        self.submitted[rid] = serving.time.perf_counter()
        return rid

    def poll(self):
        now = serving.time.perf_counter()
        out = []
        for rid, t0 in list(self.submitted.items()):
            if now - t0 >= ((rid - 7) % 3 + 1) * 1e-3:
                del self.submitted[rid]
                out.append(serving.Served(rid, 18, [0] * 18, now - t0, 0.0, 1))
        return out


def test_replay_reports_every_request_in_submission_order():
    cubes = workloads.uniform_cubes(30, seed=3)
    arrivals = serving.poisson_arrivals(len(cubes), 2000.0, seed=3)
    stats = serving.replay(FakeServer(), cubes, arrivals, timeout_s=30.0)
    assert stats["requests"] == 30
    assert [r.request for r in stats["results"]] == list(range(7, 37))
    lat = np.array([r.latency_s for r in stats["results"]])
    assert stats["p50_s"] == float(np.percentile(lat, 50)) and stats["max_s"] == float(lat.max())
    assert 0.0 < stats["p50_s"] <= stats["p95_s"] <= stats["p99_s"] <= stats["max_s"]
    assert lat.min() >= 1e-3


class FakeServerHandle:
    """Records what serving.Server submits to the library."""

    def __init__(self):
        self.started = None
        self.submits = []

    def server_start(self, slots, opts):
        self.started = slots

    def server_submit(self, words, table_id=0):
        self.submits.append((np.asarray(words).copy(), table_id))
        return len(self.submits)

    def server_stop(self):
        self.started = None


def test_server_picks_the_second_table_by_the_flip_rule():
    h = FakeServerHandle()
    srv = serving.Server(h, 16, None, flip_rule=12)
    srv.submit(workloads.superflip())
    for c in workloads.uniform_cubes(20, seed=11):
        srv.submit(c)
    srv.close()
    assert h.submits[0][1] == 1  # all twelve edges flipped: the d4 table
    assert all(t == 0 for _, t in h.submits[1:])  # uniform cubes with fewer flips stay on d4t
    plain = FakeServerHandle()
    srv = serving.Server(plain, 16, None)  # no second table: always table 0
    srv.submit(workloads.superflip())
    srv.close()
    assert plain.submits[0][1] == 0 and h.started is None


def test_gpusolver_refuses_unbuilt_reference_keywords():
    """The reference's GpuSolver keywords are accepted; those of its experimental search modes
    raise ValueError before any device work (as the reference does for invalid combinations)."""

    import pytest

    from cuda_cube_solver.solver import GpuSolver

    for kw, match in (({"mode": "multi"}, "mode='step'"), ({"inverse": False}, "mode='step'"),
                      ({"step_extra": 1}, "step_extra"), ({"step_defines": ("-DX",)}, "step_defines"),
                      ({"extra_kind": "s4"}, "extra_kind")):
        with pytest.raises(ValueError, match=match):
            GpuSolver(**kw)


class _TableHandle:
    """Stand-in for native.Handle that records the table calls (no device)."""

    def __init__(self):
        self.calls = []

    def build_table_files(self, kind, block_path=None, b3_path=None, mod3_path=None, log=None):
        self.calls.append(("build", kind, block_path, b3_path, mod3_path))
        for p in (block_path, b3_path, mod3_path):
            if p is not None:
                p.write_bytes(b"")
        return [1, 2, 18], 0.5

    def encode_b3_file(self, kind, mod3_path, block_path, b3_path):
        self.calls.append(("b3", kind, mod3_path, block_path, b3_path))
        b3_path.write_bytes(b"\0" * 32)

    def save_table(self, path, table=0):
        self.calls.append(("save", path, table))

    def table_histogram(self, table=0, n_bins=32):
        self.calls.append(("hist", table, n_bins))
        return [0] * n_bins


def test_table_entry_points_use_the_reference_file_names(tmp_path, monkeypatch):
    """table.build writes prune-ud-<kind>.bin (mod 3) and -blk.bin from one BFS plus the .json meta
    (table.py:140-167); build_b3_table reads those two and writes -b3.bin (table.py:52-63);
    save_device and histogram pass the table id through."""

    from cuda_cube_solver import native, table

    monkeypatch.setattr(native, "kind_info", lambda kind: (1, 9930 * 10))
    h = _TableHandle()
    mod3 = table.build(tmp_path, "d4t", log=None, handle=h)
    assert mod3 == tmp_path / "prune-ud-d4t.bin"
    assert h.calls[0] == ("build", "d4t", tmp_path / "prune-ud-d4t-blk.bin", None, mod3)
    meta = json.loads(mod3.with_suffix(".json").read_text())
    assert meta["depth_counts"] == [1, 2, 18] and meta["entries"] == 99300 and meta["classes"] == 9930
    assert meta["encoding"] == "2-bit distance mod 3, 16 entries per little-endian uint32"
    b3 = table.build_b3_table(tmp_path, "d4t", handle=h, log=lambda *_: None)
    assert b3 == tmp_path / "prune-ud-d4t-b3.bin"
    assert h.calls[1] == ("b3", "d4t", mod3, tmp_path / "prune-ud-d4t-blk.bin", b3)
    table.save_device(h, tmp_path / "x.bin", table=1)
    assert h.calls[2] == ("save", tmp_path / "x.bin", 1)
    assert table.histogram(h, table=1, n_bins=24) == [0] * 24
    assert h.calls[3] == ("hist", 1, 24)
