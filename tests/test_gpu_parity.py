"""B200 runtime vs the reference: golden vectors (bit-exact) and the oracle on larger graphs."""

from __future__ import annotations

from contextlib import ExitStack

import numpy as np
import pytest

from conftest import ATOL_F32, ATOL_F64, RTOL_F32, RTOL_F64, artifact_path, golden_index, golden_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from grg_spmv_b200 import RuntimeRequirements  # noqa: E402


def _req(k=8, **kw):
    base = dict(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=True,
                need_init_vector=True, need_init_matrix=True, need_init_xtx=True)
    base.update(kw)
    return RuntimeRequirements(**base)


def _layout(paths, *, dtype=np.float64, req=None, exact=False, heavy=None, budget=0, ring=0, allow_residency=True, stream=0,
            pair=None, variant=0, heavy_variant=None, precision="plain"):
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, plan_b200_layout

    if pair is None:
        kw = {"narrow_variant": variant, "heavy_variant": heavy_variant}
        if heavy is not None:
            kw["heavy_threshold"] = heavy
        pair = B200PlanPair(plan_up=B200Plan(exact_order=exact, **kw), plan_down=B200Plan(exact_order=exact, **kw))
    return plan_b200_layout(artifacts=list(paths), dtype=dtype, requirements=req or _req(), vram_budget_bytes=budget,
                            ring_buffer_size=ring, allow_residency=allow_residency, device=0, stream=stream, pair=pair,
                            precision=precision)


def _run_case(grg, case, data):
    x, init, miss = golden_inputs(case, data)
    out = grg.matmul(x, case["direction"], emit_all_nodes=case["emit_all_nodes"], by_individual=case["by_individual"],
                     init=init, miss=miss)
    return out, miss


def _cases_by_artifact():
    groups: dict[tuple[str, str], list[dict]] = {}
    for case in golden_index():
        groups.setdefault((case["artifact"], case["dtype"]), []).append(case)
    return groups


GROUPS = _cases_by_artifact()


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16])
@pytest.mark.parametrize("heavy", [128, 2], ids=["narrow", "heavy-rows"])
@pytest.mark.parametrize("group", sorted(GROUPS), ids=[f"{a}-{d}" for a, d in sorted(GROUPS)])
def test_golden_bit_exact_in_exact_order(group, heavy, variant, golden_data):
    """exact_order=True reproduces ReferenceRuntime bit for bit, for every golden case and
    every narrow-row kernel variant."""
    from grg_spmv_b200.backends.b200 import B200Runtime

    name, dtype = group
    layout = _layout([artifact_path(name)], dtype=np.dtype(dtype), exact=True, heavy=heavy, variant=variant)
    with B200Runtime(layout, check_bounds=True) as runtime:
        (grg,) = runtime.grgs
        for case in GROUPS[group]:
            out, miss = _run_case(grg, case, golden_data)
            expected = golden_data[case["key"] + "|out"]
            assert out.dtype == expected.dtype
            np.testing.assert_array_equal(out, expected, err_msg=case["key"])
            if case["miss"] and case["direction"] == "up":
                np.testing.assert_array_equal(miss, golden_data[case["key"] + "|miss_out"], err_msg=case["key"])
        assert runtime.device_error() == 0


@pytest.mark.parametrize("heavy_variant", [0, 1, 2, 3])
@pytest.mark.parametrize("group", sorted(GROUPS), ids=[f"{a}-{d}" for a, d in sorted(GROUPS)])
def test_golden_fast_mode_heavy_rows(group, heavy_variant, golden_data):
    """Default mode with split heavy rows (one CTA or one warp per row, the warps also fused
    into the narrow launch; fixed-order reductions): exact for integer-valued inputs,
    tolerance otherwise."""
    from grg_spmv_b200.backends.b200 import B200Runtime

    name, dtype = group
    layout = _layout([artifact_path(name)], dtype=np.dtype(dtype), exact=False, heavy=2, heavy_variant=heavy_variant,
                     variant=6 if heavy_variant == 2 else 0)
    rtol, atol = (RTOL_F64, ATOL_F64) if dtype == "float64" else (RTOL_F32, ATOL_F32)
    with B200Runtime(layout, check_bounds=True) as runtime:
        (grg,) = runtime.grgs
        for case in GROUPS[group]:
            out, _ = _run_case(grg, case, golden_data)
            expected = golden_data[case["key"] + "|out"]
            integer = any(tag in case["case"] for tag in ("pm1", "ones", "zeros"))
            if integer and case["init"] is None:
                np.testing.assert_array_equal(out, expected, err_msg=case["key"])
            else:
                np.testing.assert_allclose(out, expected, rtol=rtol, atol=atol * max(1.0, np.abs(expected).max()), err_msg=case["key"])
        assert runtime.device_error() == 0


MIXED_RTOL = 1e-10  # mixed precision: max |got - ref| / max |ref| per result


@pytest.mark.parametrize("heavy", [128, 2], ids=["narrow", "heavy-rows"])
@pytest.mark.parametrize("group", [g for g in sorted(GROUPS) if g[1] == "float64"], ids=lambda g: g[0])
def test_golden_mixed_precision(group, heavy, golden_data):
    """Mixed precision (6-byte node state, FP64 sums) against the reference's FP64 golden
    outputs: integer-valued inputs without a real-valued init are exact, everything else is
    within MIXED_RTOL of the largest output magnitude."""
    from grg_spmv_b200.backends.b200 import B200Runtime

    name, dtype = group
    layout = _layout([artifact_path(name)], dtype=np.float64, exact=False, heavy=heavy, variant=6, precision="mixed")
    with B200Runtime(layout, check_bounds=True) as runtime:
        (grg,) = runtime.grgs
        for case in GROUPS[group]:
            out, miss = _run_case(grg, case, golden_data)
            expected = golden_data[case["key"] + "|out"]
            assert out.dtype == np.float64
            integer = any(tag in case["case"] for tag in ("pm1", "ones", "zeros"))
            if integer and case["init"] is None:
                np.testing.assert_array_equal(out, expected, err_msg=case["key"])
            else:
                scale = max(float(np.abs(expected).max()), 1e-300)
                assert float(np.abs(out - expected).max()) <= MIXED_RTOL * scale, case["key"]
            if case["miss"] and case["direction"] == "up" and integer:
                np.testing.assert_array_equal(miss, golden_data[case["key"] + "|miss_out"], err_msg=case["key"])
        assert runtime.device_error() == 0


@pytest.mark.parametrize("variant", [13, 14, 15, 16])
@pytest.mark.parametrize("group", sorted(GROUPS), ids=[f"{a}-{d}" for a, d in sorted(GROUPS)])
def test_golden_entry_walks_with_heavy_rows(group, variant, golden_data):
    """The entry-parallel walks with many heavy rows (threshold 4) in the same launch, and the
    short one-slot rows: exact for integer-valued inputs, within tolerance otherwise."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, B200Runtime

    name, dtype = group
    plan = B200Plan(narrow_variant=variant, heavy_variant=2, heavy_threshold=4, narrow_split=0)
    layout = _layout([artifact_path(name)], dtype=np.dtype(dtype), pair=B200PlanPair(plan_up=plan, plan_down=plan))
    rtol, atol = (RTOL_F64, ATOL_F64) if dtype == "float64" else (RTOL_F32, ATOL_F32)
    with B200Runtime(layout, check_bounds=False) as runtime:
        (grg,) = runtime.grgs
        for case in GROUPS[group]:
            out, miss = _run_case(grg, case, golden_data)
            expected = golden_data[case["key"] + "|out"]
            integer = any(tag in case["case"] for tag in ("pm1", "ones", "zeros"))
            if integer and case["init"] is None:
                np.testing.assert_array_equal(out, expected, err_msg=case["key"])
            else:
                np.testing.assert_allclose(out, expected, rtol=rtol, atol=atol * max(1.0, np.abs(expected).max()), err_msg=case["key"])
        assert runtime.device_error() == 0


@pytest.mark.parametrize("variant", [11, 12, 13, 14, 15, 16])
@pytest.mark.parametrize("group", sorted(GROUPS), ids=[f"{a}-{d}" for a, d in sorted(GROUPS)])
def test_golden_lean_walks(group, variant, golden_data):
    """The lean walks on every golden case (no bounds-check word, rows not split, no heavy
    rows): variant 11 keeps the per-segment partial sums and reproduces the reference bit for
    bit; variants 12 and 13 sum each row in one or two partial sums, exact for integer-valued
    inputs and within tolerance otherwise."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, B200Runtime

    name, dtype = group
    plan = B200Plan(narrow_variant=variant, heavy_variant=2, heavy_threshold=128, narrow_split=0)
    layout = _layout([artifact_path(name)], dtype=np.dtype(dtype), pair=B200PlanPair(plan_up=plan, plan_down=plan))
    rtol, atol = (RTOL_F64, ATOL_F64) if dtype == "float64" else (RTOL_F32, ATOL_F32)
    with B200Runtime(layout, check_bounds=False) as runtime:
        (grg,) = runtime.grgs
        for case in GROUPS[group]:
            out, miss = _run_case(grg, case, golden_data)
            expected = golden_data[case["key"] + "|out"]
            integer = any(tag in case["case"] for tag in ("pm1", "ones", "zeros"))
            if variant == 11 or (integer and case["init"] is None):
                np.testing.assert_array_equal(out, expected, err_msg=case["key"])
            else:
                np.testing.assert_allclose(out, expected, rtol=rtol, atol=atol * max(1.0, np.abs(expected).max()), err_msg=case["key"])
            if case["miss"] and case["direction"] == "up" and variant == 11:
                np.testing.assert_array_equal(miss, golden_data[case["key"] + "|miss_out"], err_msg=case["key"])
