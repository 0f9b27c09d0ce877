"""The vectorised compiler against artifacts that the reference's own compiler wrote.

``tests/golden/synth_haploid.grg_spmv`` and ``synth_diploid.grg_spmv`` were produced by the
reference's ``compile_grg`` (``pygrgl_spmv/grg/compile.py:385-460``), ``_build_init_biases``
(``pygrgl_spmv/grg/__init__.py:208-253``) and ``save_grg_spmv``
(``pygrgl_spmv/grg/artifact.py:109-204``) from DAGs of ``grg_spmv_b200.synth.generate_dag``
(``tests/golden/make_golden.py``).  Here the same DAGs are regenerated from their seeds,
compiled with ``compile_dag``, saved with this package's writer and read back: every array
must equal the reference's, values and dtypes.
"""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import pytest

from grg_spmv_b200.artifact import load_grg_spmv, save_grg_spmv
from grg_spmv_b200.compile import build_init_biases, compile_dag
from grg_spmv_b200.synth import SynthSpec, generate_dag

GOLDEN = Path(__file__).resolve().parent / "golden"


def _synth_cases():
    spec = importlib.util.spec_from_file_location("_make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)  # top level imports numpy only; the reference is loaded by main()
    return mod.SYNTH_CASES


# synth_repeat carries repeated mutation rows that only the reference-side duck GRG adds
CASES = [name for name in _synth_cases() if name != "synth_repeat"]


def _arrays(state):
    out = {}
    for field in ("level_offsets", "node_perm", "inv_node_perm", "sample_to_individual", "coalescence_counts",
                  "init_vector_up_bias", "init_vector_down_bias", "init_xtx_up_bias", "init_xtx_down_bias"):
        value = getattr(state, field, None)
        if value is not None:
            out[field] = np.asarray(value)
    for name in ("sel_mut", "sel_miss"):
        mat = getattr(state, name)
        out[f"{name}.indices"], out[f"{name}.indptr"] = mat.indices, mat.indptr
    for dst, row in enumerate(state.A_blocks):
        for src, block in enumerate(row):
            if block is None:
                continue
            out[f"A[{dst}][{src}].indices"], out[f"A[{dst}][{src}].indptr"] = block.indices, block.indptr
            out[f"A[{dst}][{src}].shape"] = np.asarray(block.shape)
    return out


@pytest.mark.parametrize("name", CASES)
def test_compile_dag_reproduces_reference_compiled_artifact(name, tmp_path):
    kwargs = _synth_cases()[name]
    ours = compile_dag(generate_dag(SynthSpec(**kwargs)))
    build_init_biases(ours, np.float64)
    save_grg_spmv(ours, tmp_path / f"{name}.grg_spmv")
    mine = _arrays(load_grg_spmv(tmp_path / f"{name}.grg_spmv", np.float64))
    ref = _arrays(load_grg_spmv(GOLDEN / f"{name}.grg_spmv", np.float64))
    assert mine.keys() == ref.keys()
    for key in ref:
        assert mine[key].dtype == ref[key].dtype, key
        np.testing.assert_array_equal(mine[key], ref[key], err_msg=key)
    for scalar in ("num_samples", "num_mutations", "num_nodes", "ploidy", "num_individuals", "num_edges"):
        assert getattr(ours, scalar) == getattr(load_grg_spmv(GOLDEN / f"{name}.grg_spmv", np.float64), scalar), scalar
