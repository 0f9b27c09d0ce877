"""B200-native backend for GRG sparse matmul (``X·G`` up, ``X·Gᵀ`` down).

The package root is CPU-safe (numpy/scipy only): requirements, the ``.grg_spmv`` artifact
format, the compiler and the synthetic generator.  The GPU runtime lives in
``grg_spmv_b200.backends.b200`` and is imported explicitly, as the reference package keeps its
GPU runtimes out of its root (``pygrgl_spmv/__init__.py``).
"""

from grg_spmv_b200.artifact import (
    GRG_SPMV_FORMAT_MAGIC,
    GRG_SPMV_FORMAT_VERSION,
    CompiledOperatorState,
    iter_artifact_blocks,
    load_grg_spmv,
    save_grg_spmv,
    scan_grg_spmv,
)
from grg_spmv_b200.compile import DagGRG, build_init_biases, compile_dag
from grg_spmv_b200.grg import BoundGRG, RuntimeRequirements
from grg_spmv_b200.types import Direction, InitMode

__all__ = [
    "BoundGRG",
    "CompiledOperatorState",
    "DagGRG",
    "Direction",
    "GRG_SPMV_FORMAT_MAGIC",
    "GRG_SPMV_FORMAT_VERSION",
    "InitMode",
    "RuntimeRequirements",
    "build_init_biases",
    "compile_dag",
    "iter_artifact_blocks",
    "load_grg_spmv",
    "save_grg_spmv",
    "scan_grg_spmv",
]
