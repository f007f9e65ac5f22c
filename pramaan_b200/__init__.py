"""pramaan_b200 — B200-native (sm_100a) restarted-PDHG LP solver, a drop-in for
PRAMAAN's GPU PDHG path (src/gpu/).

The compute path is libpramaan_b200.so (hand-written CUDA for sm_100a behind
an extern "C" ABI, include/pramaan_b200.h); this package is its host-side
mirror of the reference interface.
"""
from .pdhg import (  # noqa: F401
    ModelIR,
    ObjSense,
    PdhgOptions,
    PdhgSolver,
    Session,
    SolveResult,
    SolveStatus,
    kInfinity,
    launch_pdhg_iteration,
    launch_spmv,
    launch_spmv_t,
    release_cached_memory,
    solve_batch,
)
from ._lib import LIB_PATH, PramaanError, lib  # noqa: F401
from .certificate import Certificate, certify, certify_batch  # noqa: F401
from .ladder import LadderOptions, PrecisionLadder, PrecisionLadderResult  # noqa: F401

__version__ = "0.1.0"
