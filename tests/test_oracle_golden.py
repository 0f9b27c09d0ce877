"""The oracle and the kernel model against golden outputs produced by the reference itself."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import artifact_path, golden_index, golden_inputs
from grg_oracle import OracleGRG
from _kernel_model import model_matmul

CASES = golden_index()


def test_golden_index_covers_every_mode():
    cases = {c["case"] for c in CASES}
    for needed in ("up-k1-normal", "down-k8-pm1", "up-vector", "down-matrix", "up-emit", "down-emit-xtx",
                   "down-miss", "up-miss-pm1", "down-byind", "up-byind-emit"):
        assert needed in cases
    assert {c["dtype"] for c in CASES} == {"float64", "float32"}
    assert len({c["artifact"] for c in CASES}) == 6


@pytest.mark.parametrize("artifact", sorted({c["artifact"] for c in CASES}))
def test_oracle_reproduces_reference_bit_for_bit(artifact, golden_data):
    oracles = {}
    for case in (c for c in CASES if c["artifact"] == artifact):
        oracle = oracles.setdefault(case["dtype"], OracleGRG(artifact_path(artifact), dtype=np.dtype(case["dtype"])))
        x, init, miss = golden_inputs(case, golden_data)
        out = oracle.matmul(x, case["direction"], emit_all_nodes=case["emit_all_nodes"],
                            by_individual=case["by_individual"], init=init, miss=miss)
        expected = golden_data[case["key"] + "|out"]
        assert out.dtype == expected.dtype
        np.testing.assert_array_equal(out, expected, err_msg=case["key"])
        if case["miss"] and case["direction"] == "up":
            np.testing.assert_array_equal(miss, golden_data[case["key"] + "|miss_out"])


@pytest.mark.parametrize("artifact", sorted({c["artifact"] for c in CASES}))
def test_kernel_model_walks_lists_in_reference_order(artifact, golden_data):
    """The gather lists the CUDA kernels walk, summed left to right per segment, give the
    reference's outputs bit for bit (so the list order is the reference's summation order)."""
    for case in (c for c in CASES if c["artifact"] == artifact and c["dtype"] == "float64"):
        x, init, miss = golden_inputs(case, golden_data)
        out = model_matmul(artifact_path(artifact), x, case["direction"], np.float64, init=init, miss=miss,
                           by_individual=case["by_individual"], emit_all_nodes=case["emit_all_nodes"])
        np.testing.assert_array_equal(out, golden_data[case["key"] + "|out"], err_msg=case["key"])


def test_band_expectations_from_reference_suite():
    """Analytic band sums of the reference suite (``_streaming_cases.py:493-526``), restated."""

    def window(x, shift, bw):
        n = x.shape[0]
        start = (np.arange(n) + shift) % n
        dup = np.concatenate((x, x), axis=0)
        pre = np.concatenate((np.zeros((1, x.shape[1])), np.cumsum(dup, axis=0)), axis=0)
        return pre[start + bw] - pre[start]

    def band_t(x, shift, bw):
        return window(x, -shift - bw + 1, bw)

    oracle = OracleGRG(artifact_path("band3"))
    rng = np.random.default_rng(5)
    x = rng.choice(np.asarray([-1.0, 1.0]), size=(64, 3))
    bw, shifts = 8, (0, 8, 16)
    up = window(x, shifts[1], bw) + window(window(x, shifts[0], bw), shifts[2], bw)
    down = band_t(band_t(x, shifts[2], bw), shifts[0], bw) + band_t(x, shifts[1], bw)
    np.testing.assert_array_equal(oracle.matmul(x.T, "up").T, up)
    np.testing.assert_array_equal(oracle.matmul(x.T, "down").T, down)
