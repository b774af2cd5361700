"""The reference's own GPU build, run unmodified on this GPU: its kernels.cu compiled by
baseline/Makefile into baseline/_ref/*.cubin and driven through the CUDA driver API with the
reference's host-loop semantics (CuPy is not in this image; this runner stands in for CuPy's
RawModule and array plumbing only).

* ``RefTables.build(kind, fmt)`` follows table.generate / build_preset (table.py:82-129,
  170-200, 59-79): mod-3 table of 0xFF, block table of zeros with 0xFF minima, seed_solved, one
  expand_forward / expand_backward launch of (1152, 256) per depth with the reference's switch
  rule, build_b3 in chunks of 2^23 blocks for the base-3 format.
* ``RefSolver.solve(states)`` follows GpuSolver.solve in step mode (solver.py:226-320): root
  bounds by probe_block, per-bound search_step launches of (8 x SMs, 256) per prefix-length group,
  the job array copied to the host and back every bound.

Used as the reference-GPU baseline (``bench.py --impl reference-gpu``) and, by the tests, as a
byte-identity checker of libccs's tables.  Needs the constant blobs of baseline/ref_blobs (made
by baseline/make_ref_blobs.py from the reference's Python).
"""

from __future__ import annotations

import ctypes
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CUBINS = HERE / "_ref"
BLOBS = HERE / "ref_blobs"
sys.path.insert(0, str(HERE.parent / "cuda-cube-solver_b200"))

KIND_CUBIN = {"304": "k304", "s4": "g8", "d4f": "g12", "a4t": "g16", "a4": "g16", "d4t": "g24", "d4": "g24"}
JOB_DTYPE = np.dtype([("frame", np.uint32, (30,)), ("h", np.uint32, (6,)), ("bound", np.uint32),
                      ("found", np.uint32), ("solution_length", np.uint32), ("solution", np.uint8, (24,)),
                      ("nodes", np.uint64)], align=True)


def available() -> bool:
    return (CUBINS / "g24_step.cubin").exists() and (BLOBS / "d4t.bin").exists()


class Driver:
    """Minimal CUDA driver API through ctypes (primary context of one device)."""

    def __init__(self, device: int = 0):
        self.cu = ctypes.CDLL("libcuda.so.1")
        self._check(self.cu.cuInit(0), "cuInit")
        dev = ctypes.c_int()
        self._check(self.cu.cuDeviceGet(ctypes.byref(dev), device), "cuDeviceGet")
        self.ctx = ctypes.c_void_p()
        self._check(self.cu.cuDevicePrimaryCtxRetain(ctypes.byref(self.ctx), dev), "cuDevicePrimaryCtxRetain")
        self._check(self.cu.cuCtxSetCurrent(self.ctx), "cuCtxSetCurrent")
        sms = ctypes.c_int()
        self._check(self.cu.cuDeviceGetAttribute(ctypes.byref(sms), 16, dev), "SM count")  # MULTIPROCESSOR_COUNT
        self.sms = sms.value
        self.modules = {}

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed with CUDA driver error {rc}")

    def function(self, cubin: str, name: str):
        if cubin not in self.modules:
            mod = ctypes.c_void_p()
            data = (CUBINS / f"{cubin}.cubin").read_bytes()
            buf = ctypes.create_string_buffer(data, len(data))
            self._check(self.cu.cuModuleLoadData(ctypes.byref(mod), buf), f"load {cubin}")
            self.modules[cubin] = mod
        fn = ctypes.c_void_p()
        self._check(self.cu.cuModuleGetFunction(ctypes.byref(fn), self.modules[cubin], name.encode()), name)
        return fn

    def alloc(self, nbytes: int) -> int:
        p = ctypes.c_uint64()
        self._check(self.cu.cuMemAlloc_v2(ctypes.byref(p), ctypes.c_size_t(max(nbytes, 16))), f"alloc {nbytes}")
        return p.value

    def free(self, p: int) -> None:
        self.cu.cuMemFree_v2(ctypes.c_uint64(p))

    def h2d(self, dst: int, src: np.ndarray) -> None:
        src = np.ascontiguousarray(src)
        self._check(self.cu.cuMemcpyHtoD_v2(ctypes.c_uint64(dst), src.ctypes.data_as(ctypes.c_void_p),
                                            ctypes.c_size_t(src.nbytes)), "HtoD")

    def d2h(self, dst: np.ndarray, src: int) -> None:
        self._check(self.cu.cuMemcpyDtoH_v2(dst.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint64(src),
                                            ctypes.c_size_t(dst.nbytes)), "DtoH")

    def memset32(self, p: int, value: int, count: int) -> None:
        self._check(self.cu.cuMemsetD32_v2(ctypes.c_uint64(p), ctypes.c_uint(value), ctypes.c_size_t(count)), "memset")

    def memset2d32(self, p: int, pitch: int, value: int, width: int, height: int) -> None:
        self._check(self.cu.cuMemsetD2D32_v2(ctypes.c_uint64(p), ctypes.c_size_t(pitch), ctypes.c_uint(value),
                                             ctypes.c_size_t(width), ctypes.c_size_t(height)), "memset2d")

    def launch(self, fn, grid: int, block: int, *args) -> None:
        holders = [a if isinstance(a, ctypes._SimpleCData) else ctypes.c_uint64(a) for a in args]
        params = (ctypes.c_void_p * len(holders))(*[ctypes.addressof(h) for h in holders])
        self._check(self.cu.cuLaunchKernel(fn, ctypes.c_uint(grid), 1, 1, ctypes.c_uint(block), 1, 1, 0, None, params,
                                           None), "launch")

    def sync(self) -> None:
        self._check(self.cu.cuCtxSynchronize(), "synchronize")


def _u32(x):
    return ctypes.c_uint32(x)


def _i32(x):
    return ctypes.c_int32(x)


def _u64(x):
    return ctypes.c_uint64(x)


class RefTables:
    """The reference's constant tables (DeviceTables, device.py:125-141) for one kind."""

    def __init__(self, drv: Driver, kind: str):
        from cuda_cube_solver import coords, kinds

        self.drv = drv
        self.kind = kind
        blob = np.frombuffer((BLOBS / f"{kind}.bin").read_bytes(), np.uint8)
        self.tables = drv.alloc(blob.nbytes)
        drv.h2d(self.tables, blob)
        cc = coords.corner_classes()
        self.classidx = drv.alloc(cc.classidx.nbytes)
        drv.h2d(self.classidx, cc.classidx.astype(np.uint32))
        self.class_rep = drv.alloc(cc.rep.nbytes)
        drv.h2d(self.class_rep, cc.rep.astype(np.uint32))
        self.class_stab = drv.alloc(cc.stab.nbytes)
        drv.h2d(self.class_stab, cc.stab.astype(np.uint16))
        self.n_entries = 9930 * kinds.get(kind).n_edge
        self.cubin = KIND_CUBIN[kind]

    def build(self, fmt: str = "block", log=None) -> tuple[int, int, list[int], float]:
        """Returns (device pointer of the solving table, its bytes, depth counts, seconds)."""

        drv, n = self.drv, self.n_entries
        t0 = time.perf_counter()
        n_words = (n + 15) // 16
        n_blk_words = -(-n // 124) * 8
        table = drv.alloc(n_words * 4)
        drv.memset32(table, 0xFFFFFFFF, n_words)
        blk = drv.alloc(n_blk_words * 4)
        drv.memset32(blk, 0, n_blk_words)
        drv.memset2d32(blk, 32, 0xFF, 1, n_blk_words // 8)
        c32 = drv.alloc(4)
        drv.memset32(c32, 0, 1)
        drv.launch(drv.function(self.cubin, "seed_solved"), 1, 32, self.tables, table, blk, self.classidx,
                   self.class_stab, c32)
        drv.sync()
        v = np.zeros(1, np.uint32)
        drv.d2h(v, c32)
        counts = [int(v[0])]
        remaining = n - counts[0]
        fwd = drv.function(self.cubin, "expand_forward")
        bwd = drv.function(self.cubin, "expand_backward")
        counter = drv.alloc(8)
        depth = 0
        while remaining:
            drv.memset32(counter, 0, 2)
            if counts[-1] < remaining // 4:
                drv.launch(fwd, 36 * 32, 256, self.tables, table, blk, self.classidx, self.class_rep, self.class_stab,
                           _u64(n_words), _u64(n), _u32(depth), counter)
            else:
                drv.launch(bwd, 36 * 32, 256, self.tables, table, blk, self.classidx, self.class_rep,
                           _u64(n_words), _u64(n), _u32(depth), counter)
            drv.sync()
            c = np.zeros(1, np.uint64)
            drv.d2h(c, counter)
            if log:
                log(f"reference depth {depth + 1}: {int(c[0])}")
            if int(c[0]) == 0:
                raise RuntimeError(f"{remaining} entries unreachable")
            counts.append(int(c[0]))
            remaining -= int(c[0])
            depth += 1
        out, out_bytes = blk, n_blk_words * 4
        if fmt == "b3":
            n_b3 = -(-n // 155)
            b3 = drv.alloc(n_b3 * 32)
            kern = drv.function("base", "build_b3")
            chunk = (1 << 26) // 8
            for b0 in range(0, n_b3, chunk):
                nb = min(chunk, n_b3 - b0)
                drv.launch(kern, (nb + 127) // 128, 128, table, blk, _u64(b0), _u64(nb), _u64(n), b3 + b0 * 32)
            drv.sync()
            drv.free(blk)
            out, out_bytes = b3, n_b3 * 32
        drv.free(table)
        drv.free(counter)
        drv.free(c32)
        return out, out_bytes, counts, time.perf_counter() - t0


def canonical_prefixes(length: int) -> np.ndarray:
    from cuda_cube_solver.prefixes import canonical_prefixes as cp

    return np.ascontiguousarray(cp(length))


class RefSolver:
    """GpuSolver.solve of the reference in step mode (solver.py:254-320)."""

    def __init__(self, drv: Driver, tables: RefTables, table_ptr: int, fmt: str = "block", prefix_len: int = 4,
                 deeper_prefix_at=(5e7, 3e9)):
        self.drv, self.t, self.blk, self.fmt = drv, tables, table_ptr, fmt
        sc = np.frombuffer((BLOBS / "search_const.bin").read_bytes(), np.uint8)
        self.sconst = drv.alloc(sc.nbytes)
        drv.h2d(self.sconst, sc)
        step = f"{tables.cubin}_step" + ("_b3" if fmt == "b3" else "")
        probe = tables.cubin + ("_b3" if fmt == "b3" else "")
        self.k_search = drv.function(step, "search_step")
        self.k_block = drv.function(probe, "probe_block")
        self.prefix_len = prefix_len
        self.deeper = deeper_prefix_at
        self.prefixes = {}
        self.grid = 8 * drv.sms

    def _prefix(self, plen: int):
        if plen not in self.prefixes:
            p = canonical_prefixes(plen)
            d = self.drv.alloc(max(p.nbytes, 1))
            if p.nbytes:
                self.drv.h2d(d, p)
            self.prefixes[plen] = (d, len(p))
        return self.prefixes[plen]

    def root_h(self, states) -> tuple[np.ndarray, np.ndarray]:
        from cuda_cube_solver.device import state_words
        from cuda_cube_solver.prefixes import frames

        words = state_words([f for s in states for f in frames(s)])
        n = len(words)
        dw, dout = self.drv.alloc(words.nbytes), self.drv.alloc(4 * n)
        self.drv.h2d(dw, words)
        self.drv.launch(self.k_block, (n + 127) // 128, 128, self.t.tables, self.blk, self.t.classidx, dw, _i32(n), dout)
        out = np.zeros(n, np.uint32)
        self.drv.sync()
        self.drv.d2h(out, dout)
        self.drv.free(dw)
        self.drv.free(dout)
        return out.reshape(len(states), 6), words.reshape(len(states), 30)

    def solve(self, states):
        """Returns (lengths, solutions, nodes, seconds per cube)."""

        from cuda_cube_solver.cubie import CubieState

        drv = self.drv
        t0 = time.perf_counter()
        h, words = self.root_h(states)
        jobs = np.zeros(len(states), dtype=JOB_DTYPE)
        jobs["frame"] = words
        jobs["h"] = h
        jobs["bound"] = h.max(axis=1)
        results = [None] * len(states)
        for i, s in enumerate(states):
            if s == CubieState():
                results[i] = ([], 0, 0.0)
        d_jobs = drv.alloc(jobs.nbytes)
        drv.h2d(d_jobs, jobs)
        counter = drv.alloc(8)
        d_active = drv.alloc(4 * len(states))
        history = [[] for _ in states]
        prev = np.zeros(len(states), np.uint64)
        while True:
            active = [i for i, r in enumerate(results) if r is None]
            if not active:
                break
            host = np.zeros_like(jobs)
            drv.d2h(host, d_jobs)
            groups = {}
            for i in active:
                last = history[i][-1][1] if history[i] else 0
                plen = self.prefix_len + sum(last >= t for t in self.deeper)
                groups.setdefault(min(int(host["bound"][i]), plen), []).append(i)
            for plen, ids in groups.items():
                drv.memset32(counter, 0, 2)
                pre, n_pre = self._prefix(plen)
                ids_arr = np.array(ids, np.int32)
                drv.h2d(d_active, ids_arr)
                drv.launch(self.k_search, self.grid, 256, self.t.tables, self.sconst, self.blk, self.blk, self.blk,
                           self.blk, self.t.classidx, d_jobs, d_active, _i32(len(ids)), pre, _i32(n_pre), _i32(plen),
                           counter, _u64(0))
            drv.sync()
            drv.d2h(host, d_jobs)
            now = time.perf_counter() - t0
            for i in active:
                history[i].append((int(host["bound"][i]), int(host["nodes"][i] - prev[i])))
                prev[i] = host["nodes"][i]
                if host["found"][i]:
                    n = int(host["solution_length"][i])
                    results[i] = (list(host["solution"][i][:n]), int(host["nodes"][i]), now)
                else:
                    host["bound"][i] += 1
            drv.h2d(d_jobs, host)
        for p in (d_jobs, counter, d_active):
            drv.free(p)
        return results
