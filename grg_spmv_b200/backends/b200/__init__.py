"""B200 (sm_100a) backend: ``plan_b200_layout`` -> ``B200Layout`` -> ``B200Runtime``.

Drop-in counterpart of ``pygrgl_spmv.backends.triton`` (``plan_triton_layout``,
``TritonRuntime``) and ``pygrgl_spmv.backends.cusparse``.
"""

from grg_spmv_b200.backends.b200._native import build_library, load_library
from grg_spmv_b200.backends.b200.batch import B200BatchedMatmul, BatchItem
from grg_spmv_b200.backends.b200.plan import B200Layout, B200Plan, B200PlanPair, BudgetItem, plan_b200_layout
from grg_spmv_b200.backends.b200.runtime import B200PreparedMatmul, B200Runtime

__all__ = [
    "B200BatchedMatmul",
    "B200Layout",
    "B200Plan",
    "B200PlanPair",
    "B200PreparedMatmul",
    "B200Runtime",
    "BatchItem",
    "BudgetItem",
    "build_library",
    "load_library",
    "plan_b200_layout",
]
