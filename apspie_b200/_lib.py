"""ctypes binding of the in-tree C-ABI library ``apspie_b200/lib/libapspie.so``.

The library is the product; this module only describes its structs and signatures
(``include/apspie.h``, ``include/apspie_host.h``) and turns status codes into exceptions.
There is no fallback: if the shared library is missing, importing the entry points
raises ``ApspieLibraryMissing``.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_void_p

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libapspie.so")

STATUS = {
    0: "APSPIE_OK",
    1: "APSPIE_ERR_INVALID_ARG",
    2: "APSPIE_ERR_OOM",
    3: "APSPIE_ERR_HASH_OVERFLOW",
    4: "APSPIE_ERR_TIMEOUT",
    5: "APSPIE_ERR_CUDA",
    6: "APSPIE_ERR_UNSUPPORTED",
    7: "APSPIE_ERR_NOT_CONVERGED",
}
VAL_NONE, VAL_F32, VAL_I32 = 0, 1, 2


class ApspieLibraryMissing(RuntimeError):
    pass


class ApspieError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))


CSR_SYMMETRIC = 1


class CSR(ctypes.Structure):
    _fields_ = [
        ("m", c_int32), ("n", c_int32), ("nnz", c_int32), ("val_type", c_int32),
        ("row_ptr", c_void_p), ("col_ind", c_void_p), ("val", c_void_p),
        ("flags", c_uint32), ("reserved", c_uint32),
    ]


class CSROwned(ctypes.Structure):
    _fields_ = [
        ("m", c_int32), ("n", c_int32), ("nnz", c_int32), ("val_type", c_int32),
        ("row_ptr", c_void_p), ("col_ind", c_void_p), ("val", c_void_p),
    ]


class HostCSR(ctypes.Structure):
    _fields_ = [
        ("m", c_int32), ("n", c_int32), ("nnz", c_int32), ("val_type", c_int32),
        ("row_ptr", POINTER(c_int32)), ("col_ind", POINTER(c_int32)), ("val", c_void_p),
    ]


class RunStats(ctypes.Structure):
    _fields_ = [
        ("iterations", c_int32), ("push_iterations", c_int32), ("pull_iterations", c_int32),
        ("reserved", c_int32), ("edges_expanded", c_int64), ("edges_component", c_int64),
        ("vertices_reached", c_int64),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class TuneParams(ctypes.Structure):
    _fields_ = [
        ("bfs_alpha", c_float), ("bfs_beta", c_float), ("batch_push_frac", c_float), ("sssp_delta", c_int32),
        ("sssp_band", c_int64), ("spgemm_reg_max", c_int32), ("spgemm_block_max", c_int32),
        ("tc_task_work", c_int32), ("tc_orient", c_int32), ("reserved", c_int32 * 4),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class ServerStats(ctypes.Structure):
    _fields_ = [(n, c_int64) for n in ("submitted", "completed", "failed", "launches", "batched_queries",
                                        "max_batch_seen", "deferred", "peak_bytes", "resident_bytes",
                                        "joined_running", "trivial", "engine_launches", "engine_levels")]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


QUERY_BFS, QUERY_SSSP, QUERY_MIS = 0, 1, 2
TUNE_BFS, TUNE_SSSP, TUNE_BFS_BATCH, TUNE_SPGEMM, TUNE_TC = 0, 1, 2, 3, 4
BUILD_SYMMETRIZE, BUILD_DROP_SELF_LOOPS, BUILD_DEDUP = 1, 2, 4

# name -> (restype, argtypes)
SIGNATURES = {
    # context
    "apspie_ctx_create": (c_int, [c_int, c_void_p, POINTER(c_void_p)]),
    "apspie_ctx_destroy": (None, [c_void_p]),
    "apspie_ctx_last_error": (c_char_p, [c_void_p]),
    "apspie_ctx_synchronize": (c_int, [c_void_p]),
    "apspie_ctx_reserve": (c_int, [c_void_p, c_int32, c_int64]),
    "apspie_ctx_set_validate": (c_int, [c_void_p, c_int]),
    "apspie_ctx_set_bfs_tuning": (c_int, [c_void_p, c_float, c_float]),
    "apspie_ctx_set_sssp_delta": (c_int, [c_void_p, c_int32]),
    "apspie_ctx_set_sssp_band": (c_int, [c_void_p, c_int64]),
    "apspie_ctx_set_sssp_batch_groups": (c_int, [c_void_p, c_int32]),
    "apspie_ctx_get_params": (c_int, [c_void_p, POINTER(TuneParams)]),
    "apspie_ctx_set_params": (c_int, [c_void_p, POINTER(TuneParams)]),
    "apspie_ctx_set_autotune": (c_int, [c_void_p, c_int32]),
    "apspie_autotune": (c_int, [c_void_p, c_int32, c_void_p, c_void_p, POINTER(c_int32), c_int32, c_int32,
                                POINTER(TuneParams), POINTER(c_double)]),
    "apspie_tune_entries": (c_int32, [c_void_p]),
    "apspie_tune_lookup": (c_int, [c_void_p, c_int32, c_void_p, POINTER(TuneParams), POINTER(c_int32)]),
    "apspie_tune_save": (c_int, [c_void_p, c_char_p]),
    "apspie_tune_load": (c_int, [c_void_p, c_char_p]),
    "apspie_ctx_set_max_grid": (c_int, [c_void_p, c_int32]),
    "apspie_ctx_set_wait_limit": (c_int, [c_void_p, c_int64]),
    "apspie_grid_barrier_check": (c_int, [c_void_p, c_int32, c_int32, POINTER(c_int32)]),
    "apspie_ctx_set_batch_push_frac": (c_int, [c_void_p, c_float]),
    "apspie_ctx_scratch_bytes": (c_int64, [c_void_p]),
    "apspie_ctx_timeline": (c_int, [c_void_p, c_void_p, c_void_p, c_int32, POINTER(c_int32)]),
    "apspie_csr_validate": (c_int, [c_void_p, POINTER(CSR)]),
    # traversal
    "apspie_bfs": (c_int, [c_void_p, POINTER(CSR), c_int32, c_int32, c_void_p, POINTER(RunStats)]),
    "apspie_sssp": (c_int, [c_void_p, POINTER(CSR), c_int32, c_void_p, POINTER(RunStats)]),
    "apspie_mis": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_void_p, POINTER(RunStats)]),
    "apspie_sssp_f32": (c_int, [c_void_p, POINTER(CSR), c_int32, c_void_p, c_float, POINTER(RunStats)]),
    "apspie_mis_int32": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_void_p, POINTER(RunStats)]),
    "apspie_spmspv_bool": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_void_p]),
    "apspie_row_checksums": (c_int, [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p]),
    "apspie_spmspv": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                              POINTER(c_int32)]),
    "apspie_bfs_batch": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_int32, c_int32, c_void_p,
                                 POINTER(RunStats)]),
    "apspie_sssp_batch": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_int32, c_void_p, POINTER(RunStats)]),
    "apspie_bfs_noalloc": (c_int, [POINTER(CSR), c_int32, c_int32, c_void_p, c_void_p, POINTER(RunStats)]),
    # SpGEMM / TC
    "apspie_spgemm": (c_int, [c_void_p, POINTER(CSR), POINTER(CSR), POINTER(CSROwned)]),
    "apspie_spgemm_symbolic": (c_int, [c_void_p, POINTER(CSR), POINTER(CSR), c_void_p, POINTER(c_int64)]),
    "apspie_spgemm_numeric": (c_int, [c_void_p, POINTER(CSR), POINTER(CSR), c_void_p, c_void_p, c_void_p]),
    "apspie_csr_free": (None, [POINTER(CSROwned)]),
    "apspie_tc": (c_int, [c_void_p, POINTER(CSR), POINTER(c_int64)]),
    "apspie_csr_strict_lower_device": (c_int, [c_void_p, POINTER(CSR), POINTER(CSROwned)]),
    "apspie_csr_build": (c_int, [c_void_p, c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_int32, c_int32,
                                 POINTER(CSROwned)]),
    "apspie_csr_transpose": (c_int, [c_void_p, POINTER(CSR), POINTER(CSROwned)]),
    "apspie_spmv": (c_int, [c_void_p, POINTER(CSR), c_void_p, c_void_p, c_float, c_float]),
    "apspie_pagerank": (c_int, [c_void_p, POINTER(CSR), c_float, c_double, c_int32, c_void_p, POINTER(c_int32)]),
    # server
    "apspie_server_create": (c_int, [c_int, c_int64, c_int32, c_int32, POINTER(c_void_p)]),
    "apspie_server_add_graph": (c_int, [c_void_p, POINTER(HostCSR), c_int32, c_uint32, POINTER(c_int32)]),
    "apspie_server_set_sssp_fold": (c_int, [c_void_p, c_int32]),
    "apspie_server_set_bfs_min_batch": (c_int, [c_void_p, c_int32]),
    "apspie_server_set_sssp_min_batch": (c_int, [c_void_p, c_int32]),
    "apspie_server_set_side_room": (c_int, [c_void_p, c_int32]),
    "apspie_server_start": (c_int, [c_void_p]),
    "apspie_server_submit": (c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, POINTER(ctypes.c_uint64)]),
    "apspie_server_submit_many": (c_int, [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "apspie_server_wait": (c_int, [c_void_p, ctypes.c_uint64, c_int32, POINTER(c_double)]),
    "apspie_server_take_completed": (c_int, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p,
                                             POINTER(c_int32)]),
    "apspie_server_poll": (c_int, [c_void_p, ctypes.c_uint64, POINTER(c_int32)]),
    "apspie_server_get_stats": (c_int, [c_void_p, POINTER(ServerStats)]),
    "apspie_server_destroy": (None, [c_void_p]),
    # host graph construction
    "apspie_host_csr_free": (None, [POINTER(HostCSR)]),
    "apspie_load_mtx": (c_int, [c_char_p, c_int, POINTER(HostCSR)]),
    "apspie_load_mtx_threads": (c_int, [c_char_p, c_int, c_int, POINTER(HostCSR)]),
    "apspie_gen_rmat": (c_int, [c_int, c_int, c_uint32, c_uint32, c_double, c_double, c_double,
                                c_int, POINTER(HostCSR)]),
    "apspie_gen_er": (c_int, [c_int, c_int, c_uint32, c_int, POINTER(HostCSR)]),
    "apspie_gen_rmat_coo": (c_int, [c_int, c_int, c_uint32, c_uint32, c_double, c_double, c_double, c_void_p,
                                    c_void_p, c_void_p]),
    "apspie_mt19937_u32": (c_int, [c_uint32, c_int64, c_void_p]),
    "apspie_max_degree_vertex": (c_int32, [POINTER(HostCSR)]),
    "apspie_lcc_sample": (c_int, [POINTER(HostCSR), c_int32, c_uint32, c_void_p]),
    "apspie_csr_strict_lower": (c_int, [POINTER(HostCSR), POINTER(HostCSR)]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads (once) and returns the shared library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ApspieLibraryMissing(
                f"{LIB_PATH} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `make -C apspie_b200/csrc`")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, ctx=None, what: str = "") -> None:
    if status != 0:
        msg = what
        if ctx is not None:
            raw = lib().apspie_ctx_last_error(ctx)
            if raw:
                msg = f"{what}: {raw.decode(errors='replace')}"
        raise ApspieError(status, msg)
