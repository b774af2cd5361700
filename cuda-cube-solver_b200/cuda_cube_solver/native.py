"""ctypes binding of libccs, the C-ABI library built for sm_100a (``include/ccs.h``).

This is the only way the package reaches the GPU: there is no CPU or CuPy fallback.  If the
library is missing, importing this module raises ``ImportError`` naming the build command.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("CCS_LIB", Path(__file__).with_name("_lib") / "libccs.so"))

CCS_OK = 0
CCS_E_CUDA = -1
CCS_E_NOMEM = -2
CCS_E_ARG = -3
CCS_E_FILE = -4
CCS_E_CHECK = -5
CCS_E_UNREACHABLE = -6
CCS_E_STATE = -7
CCS_E_TIMEOUT = -8
FORMATS = {"block": 0, "b3": 1}


class CcsError(RuntimeError):
    """A libccs call failed; ``code`` is the CCS_E_* value."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class SolveOpts(ctypes.Structure):
    _fields_ = [
        ("base_plen", ctypes.c_int),
        ("deeper_at0", ctypes.c_double),
        ("deeper_at1", ctypes.c_double),
        ("blocks_per_sm", ctypes.c_int),
        ("threads", ctypes.c_int),
        ("timeout_s", ctypes.c_double),
        ("spread", ctypes.c_int),
        ("variant", ctypes.c_int),
        ("shallow_at0", ctypes.c_double),
        ("shallow_at1", ctypes.c_double),
        ("move_min", ctypes.c_int),
        ("move_age", ctypes.c_int),
        ("probe_min", ctypes.c_int),
        ("steal", ctypes.c_int),
        ("steal_depth", ctypes.c_int),
        ("steal_period", ctypes.c_int),
        ("steal_target", ctypes.c_int),
        ("few_divisor", ctypes.c_int),
        ("steal_min_nodes", ctypes.c_double),
        ("rotate", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("length", ctypes.c_int32),
        ("moves", ctypes.c_uint8 * 24),
        ("nodes", ctypes.c_uint64),
        ("probes", ctypes.c_uint64),
        ("seconds", ctypes.c_double),
        ("iter_nodes", ctypes.c_uint64 * 24),
    ]


class BfsPass(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_int32), ("forward", ctypes.c_int32), ("found", ctypes.c_uint64),
                ("random_reads", ctypes.c_uint64), ("claims", ctypes.c_uint64), ("seconds", ctypes.c_double)]


LOG_FN = ctypes.CFUNCTYPE(None, ctypes.c_char_p)

# name -> (argtypes); every function returns int (status) except where noted.
_P = ctypes.POINTER
_SIGS = {
    "ccs_version": [],
    "ccs_mem_info": [ctypes.c_int, _P(ctypes.c_uint64), _P(ctypes.c_uint64)],
    "ccs_device_sms": [ctypes.c_int, _P(ctypes.c_int)],
    "ccs_open": [ctypes.c_int, _P(ctypes.c_void_p)],
    "ccs_close": [ctypes.c_void_p],
    "ccs_kind_info": [ctypes.c_char_p, _P(ctypes.c_int), _P(ctypes.c_uint64)],
    "ccs_register_group_kind": [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "ccs_kind_tables": [ctypes.c_char_p] + [ctypes.c_void_p] * 5,
    "ccs_set_kind": [ctypes.c_void_p, ctypes.c_char_p],
    "ccs_last_solve_donations": [ctypes.c_void_p, _P(ctypes.c_uint64)],
    "ccs_last_build_passes": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_int)],
    "ccs_server_start_budget": [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, _P(ctypes.c_int)],
    "ccs_server_memory": [ctypes.c_void_p] + [_P(ctypes.c_uint64)] * 4,
    "ccs_last_solve_io_bytes": [ctypes.c_void_p, _P(ctypes.c_uint64), _P(ctypes.c_uint64)],
    "ccs_load_table": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p],
    "ccs_build_table": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                        ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_double), LOG_FN],
    "ccs_build_table_files": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                              ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_double), LOG_FN],
    "ccs_encode_b3_file": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p],
    "ccs_save_table": [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p],
    "ccs_table_histogram": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int],
    "ccs_table_bytes": [ctypes.c_void_p, _P(ctypes.c_uint64)],
    "ccs_table_copy": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64],
    "ccs_index": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "ccs_unrank": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    "ccs_lower_bound": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    "ccs_root_bounds": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    "ccs_solve": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _P(SolveOpts), ctypes.c_void_p],
    "ccs_solve_noalloc": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _P(SolveOpts), ctypes.c_void_p],
    "ccs_solve_tables": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _P(SolveOpts), ctypes.c_void_p],
    "ccs_attach_table": [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p],
    "ccs_server_submit_table": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_uint64)],
    "ccs_last_solve_stats": [ctypes.c_void_p, _P(ctypes.c_double), _P(ctypes.c_uint64), _P(ctypes.c_int)],
    "ccs_gather_bench": [ctypes.c_int, ctypes.c_uint64, ctypes.c_int, _P(ctypes.c_double), _P(ctypes.c_double)],
    "ccs_probe_bench": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _P(ctypes.c_double), _P(ctypes.c_double)],
    "ccs_server_start": [ctypes.c_void_p, ctypes.c_int, _P(SolveOpts)],
    "ccs_server_submit": [ctypes.c_void_p, ctypes.c_void_p, _P(ctypes.c_uint64)],
    "ccs_server_poll": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, _P(ctypes.c_int)],
    "ccs_server_stop": [ctypes.c_void_p],
}
EXPORTED = tuple(_SIGS) + ("ccs_last_error",)
NOALLOC_MAX_CUBES = 256  # CCS_NOALLOC_MAX_CUBES of ccs.h


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                          f"or `make -C cuda-cube-solver_b200/csrc`")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.ccs_last_error.argtypes = []
    lib.ccs_last_error.restype = ctypes.c_char_p
    return lib


lib = _load()


def check(rc: int) -> None:
    if rc != CCS_OK:
        raise CcsError(rc, lib.ccs_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def mem_info(device: int = 0) -> tuple[int, int]:
    free, total = ctypes.c_uint64(), ctypes.c_uint64()
    check(lib.ccs_mem_info(device, ctypes.byref(free), ctypes.byref(total)))
    return free.value, total.value


def kind_info(kind: str) -> tuple[int, int]:
    nec, n = ctypes.c_int(), ctypes.c_uint64()
    check(lib.ccs_kind_info(kind.encode(), ctypes.byref(nec), ctypes.byref(n)))
    return nec.value, n.value


def register_group_kind(name: str, gens) -> None:
    perms = np.ascontiguousarray([g[0] for g in gens], dtype=np.int32).reshape(-1)
    flips = np.ascontiguousarray([g[1] for g in gens], dtype=np.int32).reshape(-1)
    check(lib.ccs_register_group_kind(name.encode(), len(gens), _ptr(perms), _ptr(flips)))


def kind_tables(kind: str) -> dict[str, np.ndarray]:
    out = {"classidx": np.zeros(153090, np.uint32), "class_rep": np.zeros(9930, np.uint32),
           "class_stab": np.zeros(9930, np.uint16), "gen_class": np.zeros(384, np.uint16),
           "gen_rep": np.zeros((2, 384), np.uint16)}
    check(lib.ccs_kind_tables(kind.encode(), *(_ptr(out[k]) for k in
                                               ("classidx", "class_rep", "class_stab", "gen_class", "gen_rep"))))
    return out


def gather_bench(device: int = 0, nbytes: int = 8 << 30, rounds: int = 64) -> tuple[float, float]:
    """(random 32-byte sectors per second, ms) over an ``nbytes`` device buffer."""

    rate, ms = ctypes.c_double(), ctypes.c_double()
    check(lib.ccs_gather_bench(device, nbytes, rounds, ctypes.byref(rate), ctypes.byref(ms)))
    return rate.value, ms.value


def solve_opts(base_plen: int = 4, deeper_at: tuple[float, float] = (5e7, 3e9), blocks_per_sm: int = 0,
               threads: int = 0, timeout_s: float = 0.0, spread: int = 0, variant: int = 0,
               shallow_at: tuple[float, float] = (0.0, 0.0), move_min: int = 0, move_age: int = 0,
               probe_min: int = 0, steal: int = 0, steal_depth: int = 0, steal_period: int = 0,
               steal_target: int = 0, few_divisor: int = 0, steal_min_nodes: float = 0.0,
               rotate: int = 0) -> SolveOpts:
    return SolveOpts(base_plen, float(deeper_at[0]), float(deeper_at[1]), blocks_per_sm, threads, timeout_s, spread,
                     variant, float(shallow_at[0]), float(shallow_at[1]), move_min, move_age, probe_min, steal,
                     steal_depth, steal_period, steal_target, few_divisor, float(steal_min_nodes), int(rotate))


class Handle:
    """An open libccs handle on one device (not thread-safe; the server calls are)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        check(lib.ccs_open(device, ctypes.byref(self._h)))
        self.device = device

    def close(self) -> None:
        if self._h:
            lib.ccs_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_kind(self, kind: str) -> None:
        check(lib.ccs_set_kind(self._h, kind.encode()))

    def load_table(self, kind: str, fmt: str, path) -> None:
        check(lib.ccs_load_table(self._h, kind.encode(), FORMATS[fmt], str(path).encode()))

    def build_table(self, kind: str, fmt: str, out_path=None, keep_resident: int = 0, log=None):
        """keep_resident: 0 drop, 1 keep as the table, 2 keep as the second (attached) table."""
        counts = np.zeros(64, np.uint64)
        n = ctypes.c_int()
        secs = ctypes.c_double()
        cb = LOG_FN(lambda m: log(m.decode())) if log else LOG_FN()
        check(lib.ccs_build_table(self._h, kind.encode(), FORMATS[fmt],
                                  None if out_path is None else str(out_path).encode(), int(keep_resident),
                                  _ptr(counts), 64, ctypes.byref(n), ctypes.byref(secs), cb))
        return [int(c) for c in counts[:n.value]], secs.value

    def build_table_files(self, kind: str, block_path=None, b3_path=None, mod3_path=None, log=None):
        """One BFS writing each given file (block, base-3, the reference's mod-3); returns
        (per-depth counts, seconds).  The resident tables are left as they are."""
        counts = np.zeros(64, np.uint64)
        n = ctypes.c_int()
        secs = ctypes.c_double()
        cb = LOG_FN(lambda m: log(m.decode())) if log else LOG_FN()
        enc = (lambda p: None if p is None else str(p).encode())
        check(lib.ccs_build_table_files(self._h, kind.encode(), enc(block_path), enc(b3_path), enc(mod3_path),
                                        _ptr(counts), 64, ctypes.byref(n), ctypes.byref(secs), cb))
        return [int(c) for c in counts[:n.value]], secs.value

    def encode_b3_file(self, kind: str, mod3_path, block_path, b3_path) -> None:
        check(lib.ccs_encode_b3_file(self._h, kind.encode(), str(mod3_path).encode(), str(block_path).encode(),
                                     str(b3_path).encode()))

    def save_table(self, path, table: int = 0) -> None:
        check(lib.ccs_save_table(self._h, int(table), str(path).encode()))

    def table_histogram(self, table: int = 0, n_bins: int = 32) -> list[int]:
        bins = np.zeros(n_bins, np.uint64)
        check(lib.ccs_table_histogram(self._h, int(table), _ptr(bins), int(n_bins)))
        return [int(b) for b in bins]

    def last_build_passes(self) -> list[dict]:
        """The last build's BFS passes: depth, direction, entries found, random reads, claims, seconds."""

        buf = (BfsPass * 64)()
        n = ctypes.c_int()
        check(lib.ccs_last_build_passes(self._h, ctypes.cast(buf, ctypes.c_void_p), 64, ctypes.byref(n)))
        return [{"depth": p.depth, "forward": bool(p.forward), "found": p.found, "random_reads": p.random_reads,
                 "claims": p.claims, "seconds": p.seconds} for p in buf[: n.value]]

    def table_bytes(self) -> int:
        n = ctypes.c_uint64()
        check(lib.ccs_table_bytes(self._h, ctypes.byref(n)))
        return n.value

    def table_copy(self) -> np.ndarray:
        out = np.empty(self.table_bytes(), np.uint8)
        check(lib.ccs_table_copy(self._h, _ptr(out), out.nbytes))
        return out

    def index(self, states: np.ndarray, move: int = -1) -> tuple[np.ndarray, np.ndarray]:
        states = np.ascontiguousarray(states, dtype=np.uint32).reshape(-1, 5)
        idx = np.zeros(len(states), np.uint64)
        out = np.zeros_like(states)
        check(lib.ccs_index(self._h, _ptr(states), len(states), move, _ptr(idx), _ptr(out)))
        return idx, out

    def unrank(self, idx: np.ndarray) -> np.ndarray:
        idx = np.ascontiguousarray(idx, dtype=np.uint64).reshape(-1)
        out = np.zeros((len(idx), 5), np.uint32)
        check(lib.ccs_unrank(self._h, _ptr(idx), len(idx), _ptr(out)))
        return out

    def lower_bound(self, states: np.ndarray) -> np.ndarray:
        states = np.ascontiguousarray(states, dtype=np.uint32).reshape(-1, 5)
        out = np.zeros(len(states), np.uint32)
        check(lib.ccs_lower_bound(self._h, _ptr(states), len(states), _ptr(out)))
        return out

    def root_bounds(self, states: np.ndarray) -> np.ndarray:
        states = np.ascontiguousarray(states, dtype=np.uint32).reshape(-1, 5)
        out = np.zeros((len(states), 6), np.uint32)
        check(lib.ccs_root_bounds(self._h, _ptr(states), len(states), _ptr(out)))
        return out

    def solve(self, states: np.ndarray, opts: SolveOpts | None = None, table_ids=None):
        """Solve packed states; ``table_ids`` (0 / 1 per cube) picks the first or the attached table."""

        states = np.ascontiguousarray(states, dtype=np.uint32).reshape(-1, 5)
        results = (Result * len(states))()
        ids = None if table_ids is None else np.ascontiguousarray(table_ids, dtype=np.uint8).reshape(-1)
        check(lib.ccs_solve_tables(self._h, _ptr(states), None if ids is None else _ptr(ids), len(states),
                                   ctypes.byref(opts or solve_opts()), ctypes.cast(results, ctypes.c_void_p)))
        return list(results)

    def solve_noalloc(self, states: np.ndarray, opts: SolveOpts | None = None):
        """``ccs_solve_noalloc``: the same search on the library's fixed buffers, for callers that
        cannot allocate device memory at solve time (at most ``NOALLOC_MAX_CUBES`` cubes)."""

        states = np.ascontiguousarray(states, dtype=np.uint32).reshape(-1, 5)
        results = (Result * len(states))()
        check(lib.ccs_solve_noalloc(self._h, _ptr(states), len(states), ctypes.byref(opts or solve_opts()),
                                    ctypes.cast(results, ctypes.c_void_p)))
        return list(results)

    def attach_table(self, kind: str, fmt: str, path) -> None:
        check(lib.ccs_attach_table(self._h, kind.encode(), FORMATS[fmt], str(path).encode()))

    def probe_bench(self, n_states: int = 1 << 20, rounds: int = 256) -> tuple[float, float]:
        rate, ms = ctypes.c_double(), ctypes.c_double()
        check(lib.ccs_probe_bench(self._h, n_states, rounds, ctypes.byref(rate), ctypes.byref(ms)))
        return rate.value, ms.value

    def last_solve_stats(self) -> tuple[float, int, int]:
        ms, probes, launches = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_int()
        check(lib.ccs_last_solve_stats(self._h, ctypes.byref(ms), ctypes.byref(probes), ctypes.byref(launches)))
        return ms.value, probes.value, launches.value

    def last_solve_io_bytes(self) -> tuple[int, int]:
        """(host -> device, device -> host) bytes the last solve copied."""

        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib.ccs_last_solve_io_bytes(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def last_solve_donations(self) -> int:
        """Subtrees the last solve's lanes donated to idle lanes (work stealing)."""

        n = ctypes.c_uint64()
        check(lib.ccs_last_solve_donations(self._h, ctypes.byref(n)))
        return n.value

    # server
    def server_start(self, slots: int, opts: SolveOpts | None = None) -> None:
        check(lib.ccs_server_start(self._h, slots, ctypes.byref(opts or solve_opts())))

    def server_start_budget(self, budget_bytes: int, opts: SolveOpts | None = None) -> int:
        """Start the server with admission by device memory; returns the cubes the budget admits."""

        slots = ctypes.c_int()
        check(lib.ccs_server_start_budget(self._h, int(budget_bytes), ctypes.byref(opts or solve_opts()),
                                          ctypes.byref(slots)))
        return slots.value

    def server_memory(self) -> dict:
        v = [ctypes.c_uint64() for _ in range(4)]
        check(lib.ccs_server_memory(self._h, *[ctypes.byref(x) for x in v]))
        return dict(zip(("budget_bytes", "fixed_bytes", "bytes_per_cube", "peak_in_flight"), [x.value for x in v]))

    def server_submit(self, state: np.ndarray, table_id: int = 0) -> int:
        state = np.ascontiguousarray(state, dtype=np.uint32).reshape(5)
        rid = ctypes.c_uint64()
        check(lib.ccs_server_submit_table(self._h, _ptr(state), table_id, ctypes.byref(rid)))
        return rid.value

    def server_poll(self, max_out: int = 256):
        ids = np.zeros(max_out, np.uint64)
        results = (Result * max_out)()
        n = ctypes.c_int()
        check(lib.ccs_server_poll(self._h, max_out, _ptr(ids), ctypes.cast(results, ctypes.c_void_p), ctypes.byref(n)))
        return [(int(ids[i]), results[i]) for i in range(n.value)]

    def server_stop(self) -> None:
        check(lib.ccs_server_stop(self._h))
