"""apspie_b200: B200-native (sm_100a) SpMSpV / hash-SpGEMM graph hot path.

The product is the C-ABI shared library built from ``apspie_b200/csrc`` (declared in
``include/apspie.h``); this package loads it with ctypes for tests and benchmarks.
"""
from ._lib import (BUILD_DEDUP, BUILD_DROP_SELF_LOOPS, BUILD_SYMMETRIZE, LIB_PATH, TUNE_BFS, TUNE_BFS_BATCH,
                   TUNE_SPGEMM, TUNE_SSSP, TUNE_TC, VAL_F32, VAL_I32, VAL_NONE, ApspieError, ApspieLibraryMissing,
                   lib)
from .graph import (
    Context,
    DeviceGraph,
    HostGraph,
    Server,
    gen_er,
    gen_rmat,
    gen_rmat_coo,
    lcc_sample,
    load_mtx,
    max_degree_vertex,
    mt19937_u32,
    strict_lower,
)

__all__ = [
    "ApspieError", "ApspieLibraryMissing", "LIB_PATH", "VAL_F32", "VAL_I32", "VAL_NONE", "lib",
    "BUILD_SYMMETRIZE", "BUILD_DROP_SELF_LOOPS", "BUILD_DEDUP", "TUNE_BFS", "TUNE_SSSP", "TUNE_BFS_BATCH", "TUNE_SPGEMM", "TUNE_TC",
    "Context", "DeviceGraph", "HostGraph", "Server", "gen_er", "gen_rmat", "gen_rmat_coo", "lcc_sample", "load_mtx",
    "max_degree_vertex", "mt19937_u32", "strict_lower",
]
