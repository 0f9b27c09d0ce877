"""Captured-graph adaptor (the reference's CapturedBoundGRG) on the B200 backend: results equal
``BoundGRG.matmul`` and, for integer-valued inputs, the oracle bit for bit; k padding and
truncation, int32 coercion, miss accumulation, native tensors and the reference's validation
errors."""

from __future__ import annotations

import contextlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from grg_spmv_b200 import RuntimeRequirements  # noqa: E402


@pytest.fixture(scope="module")
def artifact(tmp_path_factory):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    path = tmp_path_factory.mktemp("adaptor") / "g.grg_spmv"
    write_synthetic_artifact(SynthSpec(num_samples=1500, num_levels=10, num_nodes=20_000, num_mutations=4_000, children=(2, 12),
                                       miss_fraction=0.02, ploidy=2, with_coalescence=True, random_ids=True, seed=77), path)
    return path


def _req(k=6):
    return RuntimeRequirements(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=True,
                               need_init_vector=True, need_init_matrix=True, need_init_xtx=True)


@pytest.mark.parametrize("native", [False, True])
def test_captured_grg_matches_matmul(artifact, native):
    from grg_spmv_b200.adaptor import CaptureSpec, capture_grg
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    req = _req()
    layout = plan_b200_layout(artifacts=[str(artifact)], dtype=np.float64, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0)
    specs = (CaptureSpec("up", 6), CaptureSpec("down", 6), CaptureSpec("up", 6, by_individual=True),
             CaptureSpec("down", 6, use_miss=True), CaptureSpec("up", 6, use_miss=True),
             CaptureSpec("up", 6, init_mode="vector"), CaptureSpec("down", 6, init_mode="matrix"),
             CaptureSpec("up", 6, init_mode="xtx"))
    rng = np.random.default_rng(4)
    dev = torch.device("cuda", 0)
    conv = (lambda a: torch.from_numpy(a).to(dev)) if native else (lambda a: a)
    back = (lambda t: t.cpu().numpy()) if native else (lambda a: a)
    with B200Runtime(layout, check_bounds=True) as runtime, contextlib.ExitStack() as stack:
        (grg,) = runtime.grgs
        cap = capture_grg(grg, None, req, stack, capture_ops=specs, native=native)
        S, M, N, I = grg.num_samples, grg.num_mutations, grg.num_nodes, grg.num_individuals
        for k in (6, 3):  # full k and a smaller k (zero-padded, truncated back)
            x = rng.standard_normal((k, S))
            np.testing.assert_allclose(back(cap.matmul(conv(x), "up")), grg.matmul(x, "up"), rtol=0, atol=0)
            xd = rng.standard_normal((k, M))
            np.testing.assert_array_equal(back(cap.matmul(conv(xd), "down")), grg.matmul(xd, "down"))
            xi = rng.standard_normal((k, I))
            np.testing.assert_array_equal(back(cap.matmul(conv(xi), "up", by_individual=True)),
                                          grg.matmul(xi, "up", by_individual=True))
            miss = rng.standard_normal((k, M))
            np.testing.assert_array_equal(back(cap.matmul(conv(xd), "down", miss=conv(miss.copy()))),
                                          grg.matmul(xd, "down", miss=miss.copy()))
            acc_a, acc_b = np.ones((k, M)), np.ones((k, M))
            acc_a_in = conv(acc_a)
            got = cap.matmul(conv(x), "up", miss=acc_a_in)
            want = grg.matmul(x, "up", miss=acc_b)
            np.testing.assert_array_equal(back(got), want)
            np.testing.assert_array_equal(back(acc_a_in), acc_b)  # accumulated in place
            iv = rng.standard_normal(k)
            np.testing.assert_array_equal(back(cap.matmul(conv(x), "up", init=conv(iv))), grg.matmul(x, "up", init=iv))
            im = rng.standard_normal((k, N))
            np.testing.assert_array_equal(back(cap.matmul(conv(xd), "down", init=conv(im))), grg.matmul(xd, "down", init=im))
            np.testing.assert_array_equal(back(cap.matmul(conv(x), "up", init="xtx")), grg.matmul(x, "up", init="xtx"))
        xint = rng.integers(-3, 4, size=(6, S)).astype(np.int32)
        got = cap.matmul(conv(xint), "up")
        assert (got.dtype == torch.int32) if native else (got.dtype == np.int32)
        np.testing.assert_array_equal(back(got), grg.matmul(xint.astype(np.float64), "up").astype(np.int32))
        assert runtime.device_error() == 0


def test_captured_grg_validation_errors(artifact):
    from grg_spmv_b200.adaptor import CaptureSpec, capture_grg
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    req = _req()
    layout = plan_b200_layout(artifacts=[str(artifact)], dtype=np.float64, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0)
    with B200Runtime(layout) as runtime, contextlib.ExitStack() as stack:
        (grg,) = runtime.grgs
        cap = capture_grg(grg, None, req, stack, capture_ops=(CaptureSpec("up", 4), CaptureSpec("up", 4, init_mode="vector")))
        S = grg.num_samples
        with pytest.raises(TypeError, match="dtype mismatch"):
            cap.matmul(np.ones((2, S), dtype=np.float32), "up")
        with pytest.raises(ValueError, match="shape mismatch"):
            cap.matmul(np.ones((5, S)), "up")
        with pytest.raises(ValueError, match="shape mismatch"):
            cap.matmul(np.ones((2, S + 1)), "up")
        with pytest.raises(TypeError, match="copy mode"):
            cap.matmul(torch.ones((2, S), dtype=torch.float64, device="cuda"), "up")
        with pytest.raises(ValueError, match="emit_all_nodes"):
            cap.matmul(np.ones((2, S)), "up", emit_all_nodes=True)
        with pytest.raises(ValueError, match="Duplicate"):
            capture_grg(grg, None, req, stack, capture_ops=(CaptureSpec("up", 4), CaptureSpec("up", 4)))


def test_captured_grg_matches_oracle_exactly_on_integer_inputs(artifact):
    """The captured adaptor against the oracle (the reference's ReferenceRuntime arithmetic),
    not against this backend's own eager path: integer-valued inputs are exact in FP64 in any
    summation order, so every mode must agree bit for bit."""
    from grg_oracle import OracleGRG

    from grg_spmv_b200.adaptor import CaptureSpec, capture_grg
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    req = _req()
    layout = plan_b200_layout(artifacts=[str(artifact)], dtype=np.float64, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0)
    specs = (CaptureSpec("up", 6), CaptureSpec("down", 6), CaptureSpec("up", 6, by_individual=True),
             CaptureSpec("down", 6, by_individual=True), CaptureSpec("down", 6, use_miss=True),
             CaptureSpec("up", 6, use_miss=True), CaptureSpec("up", 6, init_mode="vector"),
             CaptureSpec("down", 6, init_mode="matrix"), CaptureSpec("up", 6, init_mode="xtx"),
             CaptureSpec("down", 6, init_mode="xtx"))
    oracle = OracleGRG(str(artifact))
    rng = np.random.default_rng(8)
    ints = lambda shape, lo=-2, hi=3: rng.integers(lo, hi, size=shape).astype(np.float64)  # noqa: E731
    with B200Runtime(layout, check_bounds=True) as runtime, contextlib.ExitStack() as stack:
        (grg,) = runtime.grgs
        cap = capture_grg(grg, None, req, stack, capture_ops=specs, native=False)
        S, M, N, I = grg.num_samples, grg.num_mutations, grg.num_nodes, grg.num_individuals
        for k in (6, 2):
            x, xd, xi = ints((k, S)), ints((k, M)), ints((k, I))
            np.testing.assert_array_equal(cap.matmul(x, "up"), oracle.matmul(x, "up"))
            np.testing.assert_array_equal(cap.matmul(xd, "down"), oracle.matmul(xd, "down"))
            np.testing.assert_array_equal(cap.matmul(xi, "up", by_individual=True), oracle.matmul(xi, "up", by_individual=True))
            np.testing.assert_array_equal(cap.matmul(xd, "down", by_individual=True),
                                          oracle.matmul(xd, "down", by_individual=True))
            miss = ints((k, M), 0, 3)
            np.testing.assert_array_equal(cap.matmul(xd, "down", miss=miss.copy()), oracle.matmul(xd, "down", miss=miss.copy()))
            acc_cap = ints((k, M))
            acc_ref = acc_cap.copy()
            np.testing.assert_array_equal(cap.matmul(x, "up", miss=acc_cap), oracle.matmul(x, "up", miss=acc_ref))
            np.testing.assert_array_equal(acc_cap, acc_ref)  # the up miss output accumulates in place
            iv = ints(k)
            np.testing.assert_array_equal(cap.matmul(x, "up", init=iv), oracle.matmul(x, "up", init=iv))
            im = ints((k, N))
            np.testing.assert_array_equal(cap.matmul(xd, "down", init=im), oracle.matmul(xd, "down", init=im))
            np.testing.assert_array_equal(cap.matmul(x, "up", init="xtx"), oracle.matmul(x, "up", init="xtx"))
            np.testing.assert_array_equal(cap.matmul(xd, "down", init="xtx"), oracle.matmul(xd, "down", init="xtx"))
        assert runtime.device_error() == 0
