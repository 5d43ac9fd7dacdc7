"""Host graphs (numpy), device graphs (torch CUDA tensors) and the context wrapper.

``Context`` wraps one ``apspie_ctx`` (device + stream + scratch arena). Its methods are
thin forwards to the C ABI: every result comes from the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib as L


# ----------------------------------------------------------------------------------
# host side
# ----------------------------------------------------------------------------------
@dataclass
class HostGraph:
    """CSR in host memory (int32 offsets/indices; values float32, int32 or None)."""

    m: int
    n: int
    row_ptr: np.ndarray
    col_ind: np.ndarray
    val: Optional[np.ndarray] = None
    symmetric: bool = False  # pattern known to be symmetric (undirected graph)

    @property
    def nnz(self) -> int:
        return int(self.col_ind.shape[0])

    @property
    def val_type(self) -> int:
        if self.val is None:
            return L.VAL_NONE
        return L.VAL_F32 if self.val.dtype == np.float32 else L.VAL_I32

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_ptr)

    def to_host_struct(self) -> L.HostCSR:
        s = L.HostCSR()
        s.m, s.n, s.nnz, s.val_type = self.m, self.n, self.nnz, self.val_type
        self._keep = (np.ascontiguousarray(self.row_ptr, dtype=np.int32),
                      np.ascontiguousarray(self.col_ind, dtype=np.int32))
        s.row_ptr = self._keep[0].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        s.col_ind = self._keep[1].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        s.val = None
        return s

    def write_csr_file(self, path: str) -> None:
        """Binary CSR file read by the oracle's reference driver."""
        vt = self.val_type
        with open(path, "wb") as f:
            np.array([self.m, self.n, self.nnz, vt], dtype=np.int32).tofile(f)
            self.row_ptr.astype(np.int32).tofile(f)
            self.col_ind.astype(np.int32).tofile(f)
            if self.val is not None:
                self.val.tofile(f)


def _from_struct(s: L.HostCSR, symmetric: bool = False) -> HostGraph:
    m, nnz = s.m, s.nnz
    rp = np.ctypeslib.as_array(s.row_ptr, shape=(m + 1,)).copy()
    ci = np.ctypeslib.as_array(s.col_ind, shape=(max(nnz, 1),))[:nnz].copy()
    val = None
    if s.val_type == L.VAL_F32 and s.val:
        val = np.ctypeslib.as_array(ctypes.cast(s.val, ctypes.POINTER(ctypes.c_float)),
                                    shape=(max(nnz, 1),))[:nnz].copy()
    elif s.val_type == L.VAL_I32 and s.val:
        val = np.ctypeslib.as_array(ctypes.cast(s.val, ctypes.POINTER(ctypes.c_int32)),
                                    shape=(max(nnz, 1),))[:nnz].copy()
    n = s.n
    L.lib().apspie_host_csr_free(ctypes.byref(s))
    return HostGraph(m, n, rp, ci, val, symmetric)


def load_mtx(path: str, undirected: bool, threads: Optional[int] = None) -> HostGraph:
    """Matrix Market file -> CSR with the reference loader's semantics; threads (0 = all)
    selects the parallel parser, None the single-threaded one."""
    s = L.HostCSR()
    if threads is None:
        st = L.lib().apspie_load_mtx(str(path).encode(), int(undirected), ctypes.byref(s))
    else:
        st = L.lib().apspie_load_mtx_threads(str(path).encode(), int(undirected), int(threads), ctypes.byref(s))
    L.check(st, None, f"load_mtx({path})")
    return _from_struct(s, symmetric=bool(undirected))


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 1, weight_seed: int = 3,
             a: float = 0.57, b: float = 0.19, c: float = 0.19, weights: bool = True) -> HostGraph:
    s = L.HostCSR()
    L.check(L.lib().apspie_gen_rmat(scale, edge_factor, seed, weight_seed, a, b, c, int(weights),
                                    ctypes.byref(s)), None, "gen_rmat")
    return _from_struct(s, symmetric=True)


def gen_rmat_coo(scale: int, edge_factor: int = 16, seed: int = 1, weight_seed: int = 3,
                 a: float = 0.57, b: float = 0.19, c: float = 0.19):
    """The R-MAT edge list in generation order (self-loops and repeats included):
    (src, dst, weight) int32 arrays."""
    ne = (1 << scale) * edge_factor
    src = np.empty(ne, dtype=np.int32)
    dst = np.empty(ne, dtype=np.int32)
    w = np.empty(ne, dtype=np.int32)
    L.check(L.lib().apspie_gen_rmat_coo(scale, edge_factor, seed, weight_seed, a, b, c, src.ctypes.data,
                                        dst.ctypes.data, w.ctypes.data), None, "gen_rmat_coo")
    return src, dst, w


def gen_er(n: int, k: int = 8, seed: int = 5, val_type: int = L.VAL_F32) -> HostGraph:
    s = L.HostCSR()
    L.check(L.lib().apspie_gen_er(n, k, seed, val_type, ctypes.byref(s)), None, "gen_er")
    return _from_struct(s)


def mt19937_u32(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    L.check(L.lib().apspie_mt19937_u32(seed, count, out.ctypes.data), None, "mt19937")
    return out


def max_degree_vertex(g: HostGraph) -> int:
    return int(L.lib().apspie_max_degree_vertex(ctypes.byref(g.to_host_struct())))


def lcc_sample(g: HostGraph, count: int, seed: int = 6) -> np.ndarray:
    out = np.empty(count, dtype=np.int32)
    L.check(L.lib().apspie_lcc_sample(ctypes.byref(g.to_host_struct()), count, seed,
                                      out.ctypes.data), None, "lcc_sample")
    return out


def strict_lower(g: HostGraph) -> HostGraph:
    s = L.HostCSR()
    L.check(L.lib().apspie_csr_strict_lower(ctypes.byref(g.to_host_struct()), ctypes.byref(s)),
            None, "strict_lower")
    return _from_struct(s)


# ----------------------------------------------------------------------------------
# device side
# ----------------------------------------------------------------------------------
class DeviceGraph:
    """CSR resident in HBM as torch CUDA tensors."""

    def __init__(self, g: HostGraph, device="cuda"):
        import torch

        self.m, self.n, self.nnz = g.m, g.n, g.nnz
        self.row_ptr = torch.from_numpy(np.ascontiguousarray(g.row_ptr, dtype=np.int32)).to(device)
        self.col_ind = torch.from_numpy(np.ascontiguousarray(g.col_ind, dtype=np.int32)).to(device)
        self.val = None if g.val is None else torch.from_numpy(np.ascontiguousarray(g.val)).to(device)
        self.val_type = g.val_type
        self.symmetric = bool(g.symmetric)

    @classmethod
    def from_tensors(cls, m: int, n: int, row_ptr, col_ind, val=None, val_type: int = L.VAL_NONE,
                     symmetric: bool = False):
        """Wraps existing device tensors (no copy)."""
        self = cls.__new__(cls)
        self.m, self.n, self.nnz = m, n, int(col_ind.shape[0])
        self.row_ptr, self.col_ind, self.val = row_ptr, col_ind, val
        self.val_type = val_type if val is not None else L.VAL_NONE
        self.symmetric = symmetric
        return self

    def view(self, with_values: bool = True) -> L.CSR:
        s = L.CSR()
        s.m, s.n, s.nnz = self.m, self.n, self.nnz
        s.row_ptr = self.row_ptr.data_ptr()
        s.col_ind = self.col_ind.data_ptr() if self.nnz else None
        if with_values and self.val is not None:
            s.val_type = self.val_type
            s.val = self.val.data_ptr()
        else:
            s.val_type = L.VAL_NONE
            s.val = None
        s.flags = L.CSR_SYMMETRIC if self.symmetric else 0
        s.reserved = 0
        return s


class Context:
    """One apspie_ctx: a device, a CUDA stream (torch's current stream by default) and
    the scratch arena reused by every call."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        torch.cuda.set_device(device)
        self.device = device
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        h = ctypes.c_void_p()
        L.check(L.lib().apspie_ctx_create(device, ctypes.c_void_p(self.stream.cuda_stream),
                                          ctypes.byref(h)), None, "ctx_create")
        self.handle = h

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.lib().apspie_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- plumbing
    def _check(self, st: int, what: str) -> None:
        L.check(st, self.handle, what)

    def synchronize(self) -> None:
        self._check(L.lib().apspie_ctx_synchronize(self.handle), "synchronize")

    def set_validate(self, on: bool) -> None:
        self._check(L.lib().apspie_ctx_set_validate(self.handle, int(on)), "set_validate")

    def set_bfs_tuning(self, alpha: float, beta: float) -> None:
        self._check(L.lib().apspie_ctx_set_bfs_tuning(self.handle, alpha, beta), "set_bfs_tuning")

    def set_sssp_delta(self, delta: int) -> None:
        self._check(L.lib().apspie_ctx_set_sssp_delta(self.handle, delta), "set_sssp_delta")

    def set_sssp_band(self, edges: int) -> None:
        """Edges expanded per SSSP iteration (lowest-distance band); 0 = auto, < 0 = off."""
        self._check(L.lib().apspie_ctx_set_sssp_band(self.handle, edges), "set_sssp_band")

    def set_sssp_batch_groups(self, groups: int) -> None:
        """Batched SSSP: <= 0 = the multi-query kernel (default), > 0 = that many query groups."""
        self._check(L.lib().apspie_ctx_set_sssp_batch_groups(self.handle, groups), "set_sssp_batch_groups")

    # ---- autotuner
    def get_params(self) -> dict:
        p = L.TuneParams()
        self._check(L.lib().apspie_ctx_get_params(self.handle, ctypes.byref(p)), "get_params")
        return p.as_dict()

    def set_params(self, **knobs) -> None:
        """Sets some of the context's own knobs (names as in apspie_tune_params)."""
        p = L.TuneParams()
        self._check(L.lib().apspie_ctx_get_params(self.handle, ctypes.byref(p)), "get_params")
        for k, v in knobs.items():
            setattr(p, k, v)
        self._check(L.lib().apspie_ctx_set_params(self.handle, ctypes.byref(p)), "set_params")

    def set_autotune(self, use: bool) -> None:
        self._check(L.lib().apspie_ctx_set_autotune(self.handle, 1 if use else 0), "set_autotune")

    def autotune(self, kind: int, A: DeviceGraph, B: DeviceGraph = None, sources=None, reps: int = 3):
        """Times the candidates of `kind` on this input; returns (chosen knobs, median ms)."""
        best = L.TuneParams()
        ms = ctypes.c_double()
        src = None
        n = 0
        if sources is not None:
            arr = (ctypes.c_int32 * len(sources))(*[int(x) for x in sources])
            src, n = arr, len(sources)
        self._check(L.lib().apspie_autotune(self.handle, kind, ctypes.byref(A.view(True)),
                                            ctypes.byref(B.view(True)) if B is not None else None,
                                            src, n, reps, ctypes.byref(best), ctypes.byref(ms)), "autotune")
        return best.as_dict(), ms.value

    def tune_entries(self) -> int:
        return int(L.lib().apspie_tune_entries(self.handle))

    def tune_lookup(self, kind: int, A: DeviceGraph):
        p = L.TuneParams()
        found = ctypes.c_int32()
        self._check(L.lib().apspie_tune_lookup(self.handle, kind, ctypes.byref(A.view(False)), ctypes.byref(p),
                                               ctypes.byref(found)), "tune_lookup")
        return p.as_dict(), bool(found.value)

    def tune_save(self, path: str) -> None:
        self._check(L.lib().apspie_tune_save(self.handle, str(path).encode()), "tune_save")

    def tune_load(self, path: str) -> None:
        self._check(L.lib().apspie_tune_load(self.handle, str(path).encode()), "tune_load")

    def set_batch_push_frac(self, frac: float) -> None:
        self._check(L.lib().apspie_ctx_set_batch_push_frac(self.handle, frac), "set_batch_push_frac")

    def set_max_grid(self, blocks: int) -> None:
        self._check(L.lib().apspie_ctx_set_max_grid(self.handle, blocks), "set_max_grid")

    def set_wait_limit(self, ns: int) -> None:
        self._check(L.lib().apspie_ctx_set_wait_limit(self.handle, int(ns)), "set_wait_limit")

    def grid_barrier_check(self, rounds: int, absent_block: int = -1) -> int:
        """Runs the grid-barrier health check; returns the grid size (raises on a timeout)."""
        g = ctypes.c_int32(0)
        self._check(L.lib().apspie_grid_barrier_check(self.handle, rounds, absent_block, ctypes.byref(g)),
                    "grid_barrier_check")
        return g.value

    def reserve(self, m: int, nnz: int) -> None:
        self._check(L.lib().apspie_ctx_reserve(self.handle, m, nnz), "reserve")

    def timeline(self):
        """[(site, ns since kernel start)] of the last call made with stats=True."""
        sites = np.zeros(128, dtype=np.int32)
        ns = np.zeros(128, dtype=np.int64)
        n = ctypes.c_int32()
        self._check(L.lib().apspie_ctx_timeline(self.handle, sites.ctypes.data, ns.ctypes.data, 128,
                                                ctypes.byref(n)), "timeline")
        return list(zip(sites[:n.value].tolist(), ns[:n.value].tolist()))

    def scratch_bytes(self) -> int:
        return int(L.lib().apspie_ctx_scratch_bytes(self.handle))

    def validate(self, g: DeviceGraph) -> None:
        self._check(L.lib().apspie_csr_validate(self.handle, ctypes.byref(g.view(False))), "validate")

    # ---- algorithms (raw: caller-provided outputs, optional stats)
    def bfs_into(self, g: DeviceGraph, source: int, out, depth_cap: int = 0, stats: bool = False):
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_bfs(self.handle, ctypes.byref(g.view(False)), source, depth_cap,
                                       out.data_ptr(), ctypes.byref(st) if st else None), "bfs")
        return st.as_dict() if st else None

    def sssp_into(self, g: DeviceGraph, source: int, out, stats: bool = False):
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_sssp(self.handle, ctypes.byref(g.view(True)), source,
                                        out.data_ptr(), ctypes.byref(st) if st else None), "sssp")
        return st.as_dict() if st else None

    def sssp_f32_into(self, g: DeviceGraph, source: int, out, unreached: float = -1.0, stats: bool = False):
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_sssp_f32(self.handle, ctypes.byref(g.view(True)), source, out.data_ptr(),
                                            unreached, ctypes.byref(st) if st else None), "sssp_f32")
        return st.as_dict() if st else None

    def mis_int32_into(self, g: DeviceGraph, prio, out, stats: bool = False):
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_mis_int32(self.handle, ctypes.byref(g.view(False)), prio.data_ptr(),
                                             out.data_ptr(), ctypes.byref(st) if st else None), "mis_int32")
        return st.as_dict() if st else None

    def mis_into(self, g: DeviceGraph, prio, out, stats: bool = False):
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_mis(self.handle, ctypes.byref(g.view(False)), prio.data_ptr(),
                                       out.data_ptr(), ctypes.byref(st) if st else None), "mis")
        return st.as_dict() if st else None

    def spmspv_bool_into(self, g: DeviceGraph, x, y) -> None:
        self._check(L.lib().apspie_spmspv_bool(self.handle, ctypes.byref(g.view(False)),
                                               x.data_ptr(), y.data_ptr()), "spmspv_bool")

    def spmspv(self, g: DeviceGraph, x_ind, x_val):
        """y = x^T A for a sparse x (x_ind int32, x_val of A's value type, CUDA tensors);
        returns (y_ind, y_val) CUDA tensors of y's entries, indices ascending."""
        import torch

        nx = int(x_ind.shape[0])
        cap = max(1, min(g.n, g.nnz))
        y_ind = torch.empty(cap, dtype=torch.int32, device=x_ind.device)
        y_val = torch.empty(cap, dtype=x_val.dtype, device=x_ind.device)
        ny = ctypes.c_int32(0)
        self._check(L.lib().apspie_spmspv(self.handle, ctypes.byref(g.view(True)), x_ind.data_ptr(),
                                          x_val.data_ptr(), nx, y_ind.data_ptr(), y_val.data_ptr(),
                                          ctypes.byref(ny)), "spmspv")
        return y_ind[: ny.value], y_val[: ny.value]

    def row_checksums(self, rows, slots, coef, out) -> None:
        """out[slots[k]] += sum_i rows[k][i] * coef[i] (int32 products, int64 sum) for CUDA
        tensors rows[k] (int32 or uint8, equal length), coef (int32), out (int64, zeroed)."""
        n = len(rows)
        if n == 0:
            return
        ptrs = (ctypes.c_void_p * n)(*[r.data_ptr() for r in rows])
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        eb = 1 if rows[0].element_size() == 1 else 4
        self._check(L.lib().apspie_row_checksums(self.handle, ptrs, sl.ctypes.data, n, int(rows[0].shape[0]), eb,
                                                 coef.data_ptr(), out.data_ptr()), "row_checksums")

    # ---- batched traversal
    def bfs_batch_into(self, g: DeviceGraph, sources, out, depth_cap: int = 0, stats: bool = False):
        """sources: int32 CUDA tensor [nq]; out: int32 CUDA tensor [nq, m] (query-major)."""
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_bfs_batch(self.handle, ctypes.byref(g.view(False)), sources.data_ptr(),
                                             int(sources.shape[0]), depth_cap, out.data_ptr(),
                                             ctypes.byref(st) if st else None), "bfs_batch")
        return st.as_dict() if st else None

    def bfs_batch(self, g: DeviceGraph, sources, depth_cap: int = 0):
        import torch

        out = torch.empty((int(sources.shape[0]), g.m), dtype=torch.int32, device=f"cuda:{self.device}")
        self.bfs_batch_into(g, sources, out, depth_cap)
        return out

    def sssp_batch_into(self, g: DeviceGraph, sources, out, stats: bool = False):
        """sources: int32 CUDA tensor [nq]; out: int32 CUDA tensor [nq, m] (query-major)."""
        st = L.RunStats() if stats else None
        self._check(L.lib().apspie_sssp_batch(self.handle, ctypes.byref(g.view(True)), sources.data_ptr(),
                                              int(sources.shape[0]), out.data_ptr(),
                                              ctypes.byref(st) if st else None), "sssp_batch")
        return st.as_dict() if st else None

    def sssp_batch(self, g: DeviceGraph, sources):
        import torch

        out = torch.empty((int(sources.shape[0]), g.m), dtype=torch.int32, device=f"cuda:{self.device}")
        self.sssp_batch_into(g, sources, out)
        return out

    # ---- SpGEMM / TC
    def spgemm(self, A: DeviceGraph, B: DeviceGraph):
        """C = A*B -> (row_ptr, col_ind, val) numpy arrays (copied back, library memory freed)."""
        C = L.CSROwned()
        self._check(L.lib().apspie_spgemm(self.handle, ctypes.byref(A.view(True)), ctypes.byref(B.view(True)),
                                          ctypes.byref(C)), "spgemm")
        try:
            return _owned_to_numpy(C)
        finally:
            L.lib().apspie_csr_free(ctypes.byref(C))

    def spgemm_two_step(self, A: DeviceGraph, B: DeviceGraph):
        """Caller-owned C through apspie_spgemm_symbolic + apspie_spgemm_numeric (torch tensors)."""
        import torch

        dev = A.row_ptr.device
        rp = torch.empty(A.m + 1, dtype=torch.int32, device=dev)
        nnz = ctypes.c_int64()
        self._check(L.lib().apspie_spgemm_symbolic(self.handle, ctypes.byref(A.view(True)),
                                                   ctypes.byref(B.view(True)), rp.data_ptr(), ctypes.byref(nnz)),
                    "spgemm_symbolic")
        ci = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
        vdt = torch.float32 if A.val_type == L.VAL_F32 else torch.int32
        cv = torch.empty(max(nnz.value, 1), dtype=vdt, device=dev)
        self._check(L.lib().apspie_spgemm_numeric(self.handle, ctypes.byref(A.view(True)), ctypes.byref(B.view(True)),
                                                  rp.data_ptr(), ci.data_ptr(), cv.data_ptr()), "spgemm_numeric")
        return rp, ci[:nnz.value], cv[:nnz.value]

    def tc(self, Lg: DeviceGraph) -> int:
        out = ctypes.c_int64()
        self._check(L.lib().apspie_tc(self.handle, ctypes.byref(Lg.view(False)), ctypes.byref(out)), "tc")
        return int(out.value)

    def build_csr(self, m: int, src, dst, val=None, flags: int = 0) -> "OwnedDeviceCSR":
        """Device COO (int32 CUDA tensors; val int32 or float32 or None) -> CSR, see
        apspie_csr_build (flags: BUILD_SYMMETRIZE | BUILD_DROP_SELF_LOOPS | BUILD_DEDUP)."""
        import torch

        vt = L.VAL_NONE if val is None else (L.VAL_F32 if val.dtype == torch.float32 else L.VAL_I32)
        C = L.CSROwned()
        self._check(L.lib().apspie_csr_build(self.handle, m, int(src.shape[0]), src.data_ptr(), dst.data_ptr(),
                                             val.data_ptr() if val is not None else None, vt, flags,
                                             ctypes.byref(C)), "csr_build")
        out = OwnedDeviceCSR(C)
        out.symmetric = bool(flags & L.BUILD_SYMMETRIZE)
        return out

    def spmv_into(self, A, x, y, alpha: float = 1.0, beta: float = 0.0) -> None:
        """y = alpha * A x + beta * y (float32 CUDA tensors)."""
        self._check(L.lib().apspie_spmv(self.handle, ctypes.byref(A.view(True)), x.data_ptr(), y.data_ptr(),
                                        alpha, beta), "spmv")

    def pagerank(self, A, damping: float = 0.85, tol: float = 1e-6, max_iter: int = 100):
        """(rank float32 CUDA tensor, iterations)."""
        import torch

        r = torch.empty(A.m, dtype=torch.float32, device=f"cuda:{self.device}")
        it = ctypes.c_int32()
        self._check(L.lib().apspie_pagerank(self.handle, ctypes.byref(A.view(False)), damping, tol, max_iter,
                                            r.data_ptr(), ctypes.byref(it)), "pagerank")
        return r, it.value

    def transpose(self, A) -> "OwnedDeviceCSR":
        C = L.CSROwned()
        self._check(L.lib().apspie_csr_transpose(self.handle, ctypes.byref(A.view(True)), ctypes.byref(C)),
                    "csr_transpose")
        return OwnedDeviceCSR(C)

    def strict_lower(self, A: DeviceGraph) -> "OwnedDeviceCSR":
        C = L.CSROwned()
        self._check(L.lib().apspie_csr_strict_lower_device(self.handle, ctypes.byref(A.view(False)),
                                                          ctypes.byref(C)), "strict_lower")
        return OwnedDeviceCSR(C)

    # ---- convenience (allocate outputs)
    def bfs(self, g: DeviceGraph, source: int, depth_cap: int = 0):
        import torch

        out = torch.empty(g.m, dtype=torch.int32, device=f"cuda:{self.device}")
        self.bfs_into(g, source, out, depth_cap)
        return out

    def sssp(self, g: DeviceGraph, source: int):
        import torch

        out = torch.empty(g.m, dtype=torch.int32, device=f"cuda:{self.device}")
        self.sssp_into(g, source, out)
        return out

    def mis(self, g: DeviceGraph, prio):
        import torch

        out = torch.empty(g.m, dtype=torch.uint8, device=f"cuda:{self.device}")
        self.mis_into(g, prio, out)
        return out


def _owned_to_numpy(C: L.CSROwned):
    import torch

    m, nnz = C.m, C.nnz
    rp = np.empty(m + 1, dtype=np.int32)
    ci = np.empty(nnz, dtype=np.int32)
    val = None
    ctypes_memcpy_d2h(rp, C.row_ptr)
    if nnz:
        ctypes_memcpy_d2h(ci, C.col_ind)
    if C.val_type == L.VAL_F32:
        val = np.empty(nnz, dtype=np.float32)
    elif C.val_type == L.VAL_I32:
        val = np.empty(nnz, dtype=np.int32)
    if val is not None and nnz:
        ctypes_memcpy_d2h(val, C.val)
    torch.cuda.synchronize()
    return rp, ci, val


class _DeviceArray:
    """Raw device pointer exposed through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3}


def ctypes_memcpy_d2h(dst: np.ndarray, src_ptr: int) -> None:
    """Copies a device array (raw pointer) into a numpy array of the same dtype/length."""
    import torch

    if dst.size == 0:
        return
    t = torch.as_tensor(_DeviceArray(src_ptr, dst.size, dst.dtype.str), device="cuda")
    dst[...] = t.cpu().numpy()


class OwnedDeviceCSR:
    """A library-allocated device CSR (apspie_csr_owned), viewable as a DeviceGraph."""

    def __init__(self, C: L.CSROwned):
        self.C = C
        self.m, self.n, self.nnz, self.val_type = C.m, C.n, C.nnz, C.val_type
        self.symmetric = False

    def view(self, with_values: bool = True) -> L.CSR:
        s = L.CSR()
        s.m, s.n, s.nnz = self.m, self.n, self.nnz
        s.row_ptr, s.col_ind = self.C.row_ptr, self.C.col_ind
        s.val_type, s.val = (self.val_type, self.C.val) if with_values and self.C.val else (L.VAL_NONE, None)
        s.flags, s.reserved = 0, 0
        return s

    def to_numpy(self):
        return _owned_to_numpy(self.C)

    def free(self):
        if self.C is not None:
            L.lib().apspie_csr_free(ctypes.byref(self.C))
            self.C = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """apspie_server: HBM-resident graphs, budgeted admission, continuous batching."""

    def __init__(self, device: int = 0, budget_bytes: int = 40 << 30, slots: int = 2, max_batch: int = 512):
        h = ctypes.c_void_p()
        L.check(L.lib().apspie_server_create(device, budget_bytes, slots, max_batch, ctypes.byref(h)), None,
                "server_create")
        self.handle = h
        self.graphs = []

    def add_graph(self, g: HostGraph, mis_seed: int = 4) -> int:
        s = g.to_host_struct()
        if g.val is not None and g.val.dtype == np.int32:
            self._w = getattr(self, "_w", [])
            w = np.ascontiguousarray(g.val, dtype=np.int32)
            self._w.append(w)
            s.val_type = L.VAL_I32
            s.val = w.ctypes.data
        gid = ctypes.c_int32()
        L.check(L.lib().apspie_server_add_graph(self.handle, ctypes.byref(s), int(g.symmetric), mis_seed,
                                                ctypes.byref(gid)), None, "server_add_graph")
        self.graphs.append(g)
        return gid.value

    def set_bfs_min_batch(self, n: int) -> None:
        L.check(L.lib().apspie_server_set_bfs_min_batch(self.handle, n), None, "server_set_bfs_min_batch")

    def set_sssp_fold(self, n: int) -> None:
        L.check(L.lib().apspie_server_set_sssp_fold(self.handle, n), None, "server_set_sssp_fold")

    def set_sssp_min_batch(self, n: int) -> None:
        L.check(L.lib().apspie_server_set_sssp_min_batch(self.handle, n), None, "server_set_sssp_min_batch")

    def set_side_room(self, on: bool) -> None:
        """Persistent grids alone on the device leave room for small kernels (default on)."""
        L.check(L.lib().apspie_server_set_side_room(self.handle, int(bool(on))), None, "server_set_side_room")

    def start(self) -> None:
        L.check(L.lib().apspie_server_start(self.handle), None, "server_start")

    def submit(self, graph_id: int, kind: int, source: int, out) -> int:
        t = ctypes.c_uint64()
        L.check(L.lib().apspie_server_submit(self.handle, graph_id, kind, source, out.data_ptr(), ctypes.byref(t)),
                None, "server_submit")
        return t.value

    def submit_many(self, graph_ids, kinds, sources, outs) -> np.ndarray:
        """Queues len(outs) requests at once (one lock, one worker wake-up); returns their
        tickets. Nothing is queued if any request is invalid."""
        n = len(outs)
        g = np.ascontiguousarray(graph_ids, dtype=np.int32)
        k = np.ascontiguousarray(kinds, dtype=np.int32)
        src = np.ascontiguousarray(sources, dtype=np.int32)
        ptrs = np.array([o.data_ptr() for o in outs], dtype=np.uint64)
        if not (len(g) == len(k) == len(src) == n):
            raise ValueError("submit_many: graph_ids, kinds, sources and outs differ in length")
        t = np.zeros(n, dtype=np.uint64)
        L.check(L.lib().apspie_server_submit_many(self.handle, n, g.ctypes.data, k.ctypes.data, src.ctypes.data,
                                                  ptrs.ctypes.data, t.ctypes.data), None, "server_submit_many")
        return t

    def wait(self, ticket: int, timeout_ms: int = 600000) -> float:
        lat = ctypes.c_double()
        L.check(L.lib().apspie_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(lat)), None, "server_wait")
        return lat.value

    def take_completed(self, cap: int = 1024, timeout_ms: int = 600000):
        """[(ticket, status, latency_ms)] of requests completed since the last call (>= 1)."""
        if getattr(self, "_take_cap", 0) < cap:  # result buffers, reused across calls
            self._take_cap = cap
            self._take_buf = (np.zeros(cap, dtype=np.uint64), np.zeros(cap, dtype=np.int32),
                              np.zeros(cap, dtype=np.float64))
        t, stv, lat = self._take_buf
        n = ctypes.c_int32()
        L.check(L.lib().apspie_server_take_completed(self.handle, timeout_ms, cap, t.ctypes.data, stv.ctypes.data,
                                                     lat.ctypes.data, ctypes.byref(n)), None, "server_take_completed")
        k = n.value
        return list(zip(t[:k].tolist(), stv[:k].tolist(), lat[:k].tolist()))

    def done(self, ticket: int) -> bool:
        d = ctypes.c_int32()
        L.check(L.lib().apspie_server_poll(self.handle, ticket, ctypes.byref(d)), None, "server_poll")
        return bool(d.value)

    def stats(self) -> dict:
        st = L.ServerStats()
        L.check(L.lib().apspie_server_get_stats(self.handle, ctypes.byref(st)), None, "server_stats")
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.lib().apspie_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
