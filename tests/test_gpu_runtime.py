"""B200 runtime contracts (the reference suite's Triton/cuSPARSE runtime tests, restated)."""

from __future__ import annotations

from contextlib import ExitStack
import warnings

import numpy as np
import pytest

from conftest import artifact_path

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from grg_spmv_b200 import RuntimeRequirements  # noqa: E402
from grg_oracle import OracleGRG  # noqa: E402


def _req(k=2, **kw):
    base = dict(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=True, need_init_vector=True,
                need_init_matrix=True, need_init_xtx=True)
    base.update(kw)
    return RuntimeRequirements(**base)


def _layout(paths, **kw):
    from grg_spmv_b200.backends.b200 import plan_b200_layout

    kw.setdefault("dtype", np.float64)
    kw.setdefault("requirements", _req())
    kw.setdefault("vram_budget_bytes", 0)
    kw.setdefault("ring_buffer_size", 0)
    kw.setdefault("device", 0)
    kw.setdefault("stream", 0)
    return plan_b200_layout(artifacts=[str(p) for p in paths], **kw)


def _runtime(layout, **kw):
    from grg_spmv_b200.backends.b200 import B200Runtime

    return B200Runtime(layout, check_bounds=True, **kw)


def _pm1(rng, shape):
    return rng.choice(np.asarray([-1.0, 1.0]), size=shape)


@pytest.fixture(scope="module")
def synth_artifact(tmp_path_factory):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    path = tmp_path_factory.mktemp("synth") / "mid.grg_spmv"
    write_synthetic_artifact(SynthSpec(num_samples=3000, num_levels=14, num_nodes=60_000, num_mutations=15_000, children=(2, 16),
                                       miss_fraction=0.02, ploidy=2, with_coalescence=True, random_ids=True, seed=21), path)
    return path


def test_runtime_requires_enter_and_exposes_stream():
    stream = torch.cuda.Stream(device=0)
    layout = _layout([artifact_path("band3")], stream=stream)
    runtime = _runtime(layout)
    with pytest.raises(RuntimeError, match="entered"):
        _ = runtime.grgs
    with runtime:
        assert runtime.stream_ptr == int(stream.cuda_stream) == int(runtime.stream.cuda_stream)
        assert len(runtime.grgs) == 1 and runtime.grgs[0].device == 0
    assert runtime._state is None and not runtime._entered


def test_enter_failure_releases_owned_state(monkeypatch):
    from grg_spmv_b200.backends.b200 import B200Runtime

    layout = _layout([artifact_path("band3")])
    runtime = _runtime(layout)

    def boom(self, art):
        raise RuntimeError("boom")

    monkeypatch.setattr(B200Runtime, "_build_artifact", boom)
    with pytest.raises(RuntimeError, match="boom"):
        runtime.__enter__()
    assert runtime._state is None and runtime._io0 is None and runtime._artifacts == () and not runtime._entered


def test_concurrent_calls_fail_fast():
    with _runtime(_layout([artifact_path("band3")])) as runtime:
        (grg,) = runtime.grgs
        with grg.prepare_matmul_cuda(direction="up", k=1) as op:
            with runtime._call_scope():
                with pytest.raises(RuntimeError, match="concurrent"):
                    op()


def test_up_output_aliases_down_input():
    with _runtime(_layout([artifact_path("band3")])) as runtime:
        (grg,) = runtime.grgs
        up = grg.prepare_matmul_cuda(direction="up", k=2)
        down = grg.prepare_matmul_cuda(direction="down", k=2)
        assert up.output.data_ptr() == down.input.data_ptr()
        assert up.input.shape == (2, grg.num_samples) and up.output.shape == (2, grg.num_mutations)


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 16, 33])
@pytest.mark.parametrize("variant", [0, 4, 5, 6, 7, 8, 9, 10])
def test_synthetic_graph_against_oracle(synth_artifact, k, variant):
    """Integer-valued inputs are exact; real-valued inputs agree to 1e-12 (default heavy-row
    reduction) — every mode of the hot path on a 60k-node graph with random node ids.  Heavy
    rows go to the CTA-per-row kernel with narrow variants 0/4, to the warp-per-row kernel with
    5 and to the fused narrow+heavy launch with 6, so every k runs all three."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    heavy_variant = {5: 1, 6: 2, 7: 2, 8: 2, 9: 2, 10: 2}.get(variant, 0)
    pair = B200PlanPair(plan_up=B200Plan(narrow_variant=variant, heavy_threshold=24, heavy_variant=heavy_variant),
                        plan_down=B200Plan(narrow_variant=variant, heavy_threshold=24, heavy_variant=heavy_variant))
    rng = np.random.default_rng(100 + k)
    with _runtime(_layout([synth_artifact], requirements=_req(k=max(k, 2)), pair=pair)) as runtime:
        (grg,) = runtime.grgs
        S, M, N, I = grg.num_samples, grg.num_mutations, grg.num_nodes, grg.num_individuals
        for direction, cols in (("up", S), ("down", M)):
            x = _pm1(rng, (k, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))
            x = rng.standard_normal((k, cols))
            np.testing.assert_allclose(grg.matmul(x, direction), oracle.matmul(x, direction), rtol=1e-12, atol=1e-9)
            init = rng.standard_normal(k)
            np.testing.assert_allclose(grg.matmul(x, direction, init=init), oracle.matmul(x, direction, init=init),
                                       rtol=1e-12, atol=1e-9)
            np.testing.assert_allclose(grg.matmul(x, direction, init="xtx"), oracle.matmul(x, direction, init="xtx"),
                                       rtol=1e-12, atol=1e-9)
            mat = rng.standard_normal((k, N))
            np.testing.assert_allclose(grg.matmul(x, direction, init=mat, emit_all_nodes=True),
                                       oracle.matmul(x, direction, init=mat, emit_all_nodes=True), rtol=1e-12, atol=1e-9)
        xi = _pm1(rng, (k, I))
        miss_b, miss_o = np.zeros((k, M)), np.zeros((k, M))
        np.testing.assert_array_equal(grg.matmul(xi, "up", by_individual=True, miss=miss_b),
                                      oracle.matmul(xi, "up", by_individual=True, miss=miss_o))
        np.testing.assert_array_equal(miss_b, miss_o)
        xd, miss = _pm1(rng, (k, M)), _pm1(rng, (k, M))
        np.testing.assert_array_equal(grg.matmul(xd, "down", by_individual=True, miss=miss.copy()),
                                      oracle.matmul(xd, "down", by_individual=True, miss=miss.copy()))
        assert runtime.device_error() == 0


def test_float32_runtime(synth_artifact):
    oracle = OracleGRG(synth_artifact, dtype=np.float32)
    rng = np.random.default_rng(7)
    with _runtime(_layout([synth_artifact], dtype=np.float32, requirements=_req(k=4))) as runtime:
        (grg,) = runtime.grgs
        for direction, cols in (("up", grg.num_samples), ("down", grg.num_mutations)):
            x = _pm1(rng, (4, cols)).astype(np.float32)
            out = grg.matmul(x, direction)
            assert out.dtype == np.float32
            np.testing.assert_array_equal(out, oracle.matmul(x, direction))
            x = rng.standard_normal((4, cols)).astype(np.float32)
            np.testing.assert_allclose(grg.matmul(x, direction), oracle.matmul(x, direction), rtol=2e-5, atol=1e-4)


def test_repeated_calls_are_deterministic(synth_artifact):
    rng = np.random.default_rng(8)
    with _runtime(_layout([synth_artifact], requirements=_req(k=4))) as runtime:
        (grg,) = runtime.grgs
        x = rng.standard_normal((4, grg.num_mutations))
        first = grg.matmul(x, "down")
        for _ in range(3):
            np.testing.assert_array_equal(grg.matmul(x, "down"), first)


@pytest.mark.parametrize("ring", [1, 2, 3])
def test_streamed_levels_are_exact(synth_artifact, ring):
    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(30 + ring)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        layout = _layout([synth_artifact], requirements=_req(k=3), ring_buffer_size=ring, allow_residency=False)
    assert layout.allocated_ring_buffer_size == ring
    assert layout.bytes_by_category["resident_sparse"] == 0
    with _runtime(layout) as runtime:
        (grg,) = runtime.grgs
        for direction, cols in (("up", grg.num_samples), ("down", grg.num_mutations)):
            x = _pm1(rng, (3, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))


def test_lean_mixed_streamed_layout(synth_artifact):
    """A layout without the all-node buffer, mixed-precision node state and levels streamed
    through a two-slot ring (the shape of the large streamed configuration): integer-valued
    results stay exact, and asking for an all-node output is refused."""
    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(44)
    req = _req(k=4, need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
    full = _layout([synth_artifact], requirements=req, precision="mixed", emit_all_nodes=False)
    sizes = sorted((lp.nbytes for lp in full.level_plans()), reverse=True)
    fixed = full.bytes_total - full.bytes_by_category["resident_sparse"]
    layout = _layout([synth_artifact], requirements=req, precision="mixed", emit_all_nodes=False,
                     vram_budget_bytes=fixed + 2 * sizes[0] + sum(sizes[1:3]), ring_buffer_size=2)
    assert not layout.emit_all_nodes and layout.bytes_by_category["ring_slots"] > 0
    with _runtime(layout) as runtime:
        (grg,) = runtime.grgs
        assert runtime._aux is None
        with pytest.raises(ValueError, match="emit_all_nodes"):
            grg.prepare_matmul_cuda(direction="up", k=2, emit_all_nodes=True)
        for _ in range(2):
            x_up = _pm1(rng, (4, grg.num_samples))
            x_down, miss = _pm1(rng, (4, grg.num_mutations)), _pm1(rng, (4, grg.num_mutations))
            np.testing.assert_array_equal(grg.matmul(x_up, "up"), oracle.matmul(x_up, "up"))
            np.testing.assert_array_equal(grg.matmul(x_down, "down", miss=miss.copy()),
                                          oracle.matmul(x_down, "down", miss=miss.copy()))
        assert runtime.device_error() == 0


def test_hybrid_budget_is_exact(synth_artifact):
    oracle = OracleGRG(synth_artifact)
    full = _layout([synth_artifact], requirements=_req(k=2))
    sizes = sorted((lp.nbytes for lp in full.level_plans()), reverse=True)
    fixed = full.bytes_total - full.bytes_by_category["resident_sparse"]
    budget = fixed + 2 * sizes[0] + sum(sizes[1:4])
    layout = _layout([synth_artifact], requirements=_req(k=2), vram_budget_bytes=budget, ring_buffer_size=2)
    resident = [lp for lp in layout.level_plans() if lp.resident]
    streamed = [lp for lp in layout.level_plans() if not lp.resident]
    assert resident and streamed and layout.bytes_total <= budget
    rng = np.random.default_rng(5)
    with _runtime(layout) as runtime:
        (grg,) = runtime.grgs
        used = sum(t.numel() * t.element_size() for t in (runtime._state, runtime._io0, runtime._io1, runtime._aux)) + sum(
            s.numel() for s in runtime._slots)
        assert used <= budget
        for direction, cols in (("up", grg.num_samples), ("down", grg.num_mutations)):
            x = _pm1(rng, (2, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))


def test_one_sided_layouts(synth_artifact):
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(9)
    for direction in ("up", "down"):
        pair = B200PlanPair(plan_up=B200Plan() if direction == "up" else None, plan_down=B200Plan() if direction == "down" else None)
        with _runtime(_layout([synth_artifact], requirements=_req(k=4), pair=pair)) as runtime:
            (grg,) = runtime.grgs
            cols = grg.num_samples if direction == "up" else grg.num_mutations
            x = _pm1(rng, (4, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))
            other = "down" if direction == "up" else "up"
            with pytest.raises(ValueError, match="not configured"):
                grg.prepare_matmul_cuda(direction=other, k=1)


@pytest.mark.parametrize("direction", ["up", "down"])
def test_k_below_max_with_matrix_and_emit_vector(synth_artifact, direction):
    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(10)
    with _runtime(_layout([synth_artifact], requirements=_req(k=4))) as runtime:
        (grg,) = runtime.grgs
        cols = grg.num_samples if direction == "up" else grg.num_mutations
        x = rng.standard_normal((2, cols))
        init = rng.standard_normal((2, grg.num_nodes))
        np.testing.assert_allclose(grg.matmul(x, direction, init=init), oracle.matmul(x, direction, init=init), rtol=1e-12, atol=1e-9)
        x1 = rng.standard_normal((1, cols))
        v = rng.standard_normal(1)
        np.testing.assert_allclose(grg.matmul(x1, direction, init=v, emit_all_nodes=True),
                                   oracle.matmul(x1, direction, init=v, emit_all_nodes=True), rtol=1e-12, atol=1e-9)


def _chain_expected(oracle, order, src, init_first, init_second):
    mid = oracle.matmul(src, order[0], init=init_first)
    return oracle.matmul(mid, order[1], init=init_second)


@pytest.mark.parametrize("streamed", [False, True], ids=["resident", "streamed"])
def test_prepared_chain_captures_in_a_cuda_graph(synth_artifact, streamed):
    """down -> up with vector init, captured by the caller in one CUDA graph and replayed."""
    oracle = OracleGRG(synth_artifact)
    capture_stream = torch.cuda.Stream(device=0)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        layout = _layout([synth_artifact], requirements=_req(k=2), stream=capture_stream, ring_buffer_size=2 if streamed else 0,
                         allow_residency=not streamed)
    rng = np.random.default_rng(98)
    order = ("down", "up")
    src_np = rng.standard_normal((2, oracle.num_mutations))
    i1, i2 = rng.standard_normal(2), rng.standard_normal(2)
    expected = _chain_expected(oracle, order, src_np, i1, i2)
    with _runtime(layout) as runtime, ExitStack() as stack:
        (grg,) = runtime.grgs
        first = stack.enter_context(grg.prepare_matmul_cuda(direction=order[0], k=2, init_mode="vector"))
        second = stack.enter_context(grg.prepare_matmul_cuda(direction=order[1], k=2, init_mode="vector"))
        assert first.output.data_ptr() == second.input.data_ptr()
        src = torch.from_numpy(src_np).to("cuda:0")
        t1, t2 = torch.from_numpy(i1).to("cuda:0"), torch.from_numpy(i2).to("cuda:0")
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=capture_stream):
            first.input.copy_(src)
            first.init_vector.copy_(t1)
            first()
            second.init_vector.copy_(t2)
            second()
        for _ in range(2):
            graph.replay()
            torch.cuda.synchronize()
            np.testing.assert_allclose(second.output.cpu().numpy(), expected, rtol=1e-12, atol=1e-6)


def test_multi_grg_single_graph_mixed_heights():
    oracle_tall, oracle_short = OracleGRG(artifact_path("overlap4")), OracleGRG(artifact_path("band3"))
    capture_stream = torch.cuda.Stream(device=0)
    layout = _layout([artifact_path("overlap4"), artifact_path("band3")], requirements=_req(k=1), stream=capture_stream)
    cases = []
    for idx, (oracle, order) in enumerate(((oracle_tall, ("up", "down")), (oracle_short, ("down", "up")))):
        cols = oracle.num_samples if order[0] == "up" else oracle.num_mutations
        src = np.arange(cols, dtype=np.float64).reshape(1, cols) + 100.0 * idx
        i1, i2 = np.asarray([0.25 + idx]), np.asarray([0.75 + idx])
        cases.append((order, src, i1, i2, _chain_expected(oracle, order, src, i1, i2)))
    with _runtime(layout) as runtime, ExitStack() as stack:
        results, ops = [], []
        for grg, (order, src, i1, i2, _) in zip(runtime.grgs, cases):
            a = stack.enter_context(grg.prepare_matmul_cuda(direction=order[0], k=1, init_mode="vector"))
            b = stack.enter_context(grg.prepare_matmul_cuda(direction=order[1], k=1, init_mode="vector"))
            ops.append((a, b, torch.from_numpy(src).to("cuda:0"), torch.from_numpy(i1).to("cuda:0"), torch.from_numpy(i2).to("cuda:0")))
            results.append(torch.empty_like(b.output))
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=capture_stream):
            for (a, b, src, i1, i2), res in zip(ops, results):
                a.input.copy_(src)
                a.init_vector.copy_(i1)
                a()
                b.init_vector.copy_(i2)
                b()
                res.copy_(b.output)
        graph.replay()
        torch.cuda.synchronize()
        for res, case in zip(results, cases):
            np.testing.assert_allclose(res.cpu().numpy(), case[4], rtol=1e-12, atol=1e-9)


def test_graphs_off_matches_graphs_on(synth_artifact):
    rng = np.random.default_rng(11)
    outs = []
    for use_graphs in (True, False):
        with _runtime(_layout([synth_artifact], requirements=_req(k=3)), use_graphs=use_graphs) as runtime:
            (grg,) = runtime.grgs
            x = np.asarray(rng.standard_normal((3, grg.num_mutations))) if not outs else outs[0][0]
            outs.append((x, grg.matmul(x, "down")))
    np.testing.assert_array_equal(outs[0][1], outs[1][1])


def test_foreign_stream_ordering(synth_artifact):
    """Work queued on the caller's stream before a call is seen by it; the result is ready for
    work queued after it on the same stream."""
    oracle = OracleGRG(synth_artifact)
    stream = torch.cuda.Stream(device=0)
    rng = np.random.default_rng(12)
    x = rng.standard_normal((2, oracle.num_samples))
    with _runtime(_layout([synth_artifact], requirements=_req(k=2), stream=stream)) as runtime:
        (grg,) = runtime.grgs
        with grg.prepare_matmul_cuda(direction="up", k=2) as op, torch.cuda.stream(stream):
            torch.cuda._sleep(2_000_000)
            op.input.copy_(torch.from_numpy(x).to("cuda:0"))
            op()
            out = op.output.clone()
        stream.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), oracle.matmul(x, "up"), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("split", [1, 2, 3, -1])
@pytest.mark.parametrize("k", [1, 3, 8])
def test_split_narrow_rows_against_oracle(synth_artifact, k, split):
    """Narrow rows split over 2^split lane groups (fixed, or chosen per level): integer inputs
    exact, real inputs within 1e-12, with init values and miss rows."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    plan = B200Plan(narrow_variant=6, heavy_threshold=24, narrow_split=split)
    rng = np.random.default_rng(500 + k)
    with _runtime(_layout([synth_artifact], requirements=_req(k=max(k, 2)), pair=B200PlanPair(plan_up=plan, plan_down=plan))) as runtime:
        (grg,) = runtime.grgs
        for direction, cols in (("up", grg.num_samples), ("down", grg.num_mutations)):
            x = _pm1(rng, (k, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))
            x = rng.standard_normal((k, cols))
            init = rng.standard_normal(k)
            np.testing.assert_allclose(grg.matmul(x, direction, init=init), oracle.matmul(x, direction, init=init),
                                       rtol=1e-12, atol=1e-9)
        xd, miss = rng.standard_normal((k, grg.num_mutations)), rng.standard_normal((k, grg.num_mutations))
        np.testing.assert_allclose(grg.matmul(xd, "down", miss=miss.copy()), oracle.matmul(xd, "down", miss=miss.copy()),
                                   rtol=1e-12, atol=1e-9)
        assert runtime.device_error() == 0


def test_autotune_picks_a_known_variant_and_stays_exact(synth_artifact):
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, B200Runtime

    oracle = OracleGRG(synth_artifact)
    pair = B200PlanPair(plan_up=B200Plan(autotune=True), plan_down=B200Plan(autotune=True))
    rng = np.random.default_rng(13)
    with _runtime(_layout([synth_artifact], requirements=_req(k=4), pair=pair)) as runtime:
        assert set(runtime._variant) == {"up", "down"} == set(runtime._heavy_variant)
        assert all(v in B200Runtime.TUNE_VARIANTS for v in runtime._variant.values())
        assert all(v in (0, 1, 2) for v in runtime._heavy_variant.values())
        (grg,) = runtime.grgs
        for direction, cols in (("up", grg.num_samples), ("down", grg.num_mutations)):
            x = _pm1(rng, (4, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))


@pytest.mark.parametrize("variant", [6, 7])
@pytest.mark.parametrize("k", [1, 3, 8, 33])
def test_dataflow_schedule_matches_levels_and_oracle(synth_artifact, k, variant):
    """The persistent dataflow traversal gives bit-identical results to the level-by-level
    launches of the same plan (same per-row arithmetic) and matches the oracle."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(700 + k)
    results = {}
    inputs = {}
    for schedule in ("levels", "dataflow"):
        plan = B200Plan(narrow_variant=variant, heavy_threshold=24, heavy_variant=2, narrow_split=0, schedule=schedule)
        with _runtime(_layout([synth_artifact], requirements=_req(k=max(k, 2)), pair=B200PlanPair(plan_up=plan, plan_down=plan))) as runtime:
            (grg,) = runtime.grgs
            if not inputs:
                inputs = {"up": rng.standard_normal((k, grg.num_samples)), "down": rng.standard_normal((k, grg.num_mutations)),
                          "miss": rng.standard_normal((k, grg.num_mutations)), "pm1": _pm1(rng, (k, grg.num_samples)),
                          "init": rng.standard_normal(k)}
            out = {
                "up": grg.matmul(inputs["up"], "up"),
                "down": grg.matmul(inputs["down"], "down", miss=inputs["miss"].copy()),
                "pm1": grg.matmul(inputs["pm1"], "up"),
                "init": grg.matmul(inputs["up"], "up", init=inputs["init"]),
                "xtx": grg.matmul(inputs["down"], "down", init="xtx"),
            }
            for _ in range(2):  # prepared op replayed (graph) keeps giving the same answer
                op = grg.prepare_matmul_cuda(direction="up", k=k)
                op.input.copy_(torch.from_numpy(inputs["up"]))
                op()
                np.testing.assert_array_equal(op.output.cpu().numpy(), out["up"])
            assert runtime.device_error() == 0
            results[schedule] = out
    for key in results["levels"]:
        np.testing.assert_array_equal(results["dataflow"][key], results["levels"][key], err_msg=key)
    np.testing.assert_array_equal(results["dataflow"]["pm1"], oracle.matmul(inputs["pm1"], "up"))
    np.testing.assert_allclose(results["dataflow"]["down"], oracle.matmul(inputs["down"], "down", miss=inputs["miss"].copy()),
                               rtol=1e-12, atol=1e-9)


def test_dataflow_wait_times_out_with_a_status_instead_of_hanging(synth_artifact):
    """A traversal whose levels omit one level leaves that level's rows holding the readiness
    sentinel; rows that read them must give up after the bounded wait, report
    GRG_B200_DEVICE_WAIT_TIMEOUT, and leave the context usable for the next call."""
    import ctypes

    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair
    from grg_spmv_b200.backends.b200 import _native as nat

    plan = B200Plan(narrow_variant=6, heavy_threshold=24, heavy_variant=2, schedule="dataflow")
    with _runtime(_layout([synth_artifact], requirements=_req(k=2), pair=B200PlanPair(plan_up=plan, plan_down=plan)),
                  use_graphs=False) as runtime:
        (grg,) = runtime.grgs
        x = _pm1(np.random.default_rng(1), (2, grg.num_samples))
        good = grg.matmul(x, "up")
        op = grg.prepare_matmul_cuda(direction="up", k=2)
        args = nat.TraverseArgs.from_buffer_copy(op._args)
        levels = runtime._artifacts[0].levels[op._spec.direction]
        assert levels.count >= 3
        kept = (nat.Level * (levels.count - 1))(*([levels.array[0]] + list(levels.array[2:])))  # level 2 onward never sees level 1
        args.levels = ctypes.cast(kept, ctypes.POINTER(nat.Level))
        args.num_levels = levels.count - 1
        op.input.copy_(torch.from_numpy(x))
        stream = ctypes.c_void_p(runtime.stream_ptr)
        nat.check(runtime._lib, runtime._lib.grg_b200_traverse(ctypes.byref(args), stream), "grg_b200_traverse")
        torch.cuda.synchronize()
        assert int(runtime._df_sync[2].item()) == nat.DEVICE_WAIT_TIMEOUT
        assert runtime.device_error() == nat.DEVICE_WAIT_TIMEOUT
        # the context is still usable and the next complete traversal is right
        np.testing.assert_array_equal(grg.matmul(x, "up"), good)
        assert int(runtime._df_sync[2].item()) == 0


@pytest.mark.parametrize("variant", [6, 7, 8, 9, 10])
@pytest.mark.parametrize("exact", [False, True])
def test_slot_layout_matches_row_pointer_layout(synth_artifact, variant, exact):
    """Narrow lists located from the slot table (no row_ptr load) give bit-identical results to
    the row_ptr layout, in both modes, with init values and miss rows."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(900 + variant)
    k = 8
    x_up = None
    results = {}
    for slots in (False, True):
        plan = B200Plan(narrow_variant=variant, heavy_threshold=24, exact_order=exact, slots=slots)
        with _runtime(_layout([synth_artifact], requirements=_req(k=k), pair=B200PlanPair(plan_up=plan, plan_down=plan))) as runtime:
            (grg,) = runtime.grgs
            if x_up is None:
                x_up = rng.standard_normal((k, grg.num_samples))
                x_dn = rng.standard_normal((k, grg.num_mutations))
                miss = rng.standard_normal((k, grg.num_mutations))
                init = rng.standard_normal(k)
            levels = runtime._artifacts[0].levels
            assert all((lv.num_slot_buckets > 0) == slots for d in levels for lv in levels[d].array if lv.num_rows > lv.num_heavy)
            results[slots] = (grg.matmul(x_up, "up", init=init), grg.matmul(x_dn, "down", miss=miss.copy()))
            assert runtime.device_error() == 0
    for a, b in zip(results[False], results[True]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(results[True][0], oracle.matmul(x_up, "up", init=init), rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(results[True][1], oracle.matmul(x_dn, "down", miss=miss.copy()), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("k", [1, 8, 33])
@pytest.mark.parametrize("variant", [9, 10])
def test_persistent_narrow_rows_match_variant_7(synth_artifact, variant, k):
    """The persistent narrow part (each warp walks row groups, prefetching the next group's
    list extent and codes) is bit-identical to variant 7, which has the same per-row arithmetic;
    small ``persist_ctas`` force every warp through many groups, including groups whose rows are
    partly past the end of the level, with init values, miss rows and the slot layout."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(1000 + 10 * variant + k)
    x_up = rng.standard_normal((k, 3000))
    init = rng.standard_normal(k)
    results = {}
    cases = [(7, 0, False), (variant, 1, False), (variant, 3, False), (variant, 0, False), (variant, 2, True)]
    for narrow_variant, ctas, slots in cases:
        plan = B200Plan(narrow_variant=narrow_variant, heavy_threshold=24, heavy_variant=2, narrow_split=0,
                        persist_ctas=ctas, slots=slots)
        with _runtime(_layout([synth_artifact], requirements=_req(k=max(k, 2)), pair=B200PlanPair(plan_up=plan, plan_down=plan))) as runtime:
            (grg,) = runtime.grgs
            assert grg.num_samples == x_up.shape[1]
            if "x_dn" not in results:
                results["x_dn"] = rng.standard_normal((k, grg.num_mutations))
                results["miss"] = rng.standard_normal((k, grg.num_mutations))
            x_dn, miss = results["x_dn"], results["miss"]
            results[(narrow_variant, ctas, slots)] = (grg.matmul(x_up, "up", init=init), grg.matmul(x_up, "up", init="xtx"),
                                                      grg.matmul(x_dn, "down", miss=miss.copy()))
            assert runtime.device_error() == 0
    base = results[(7, 0, False)]
    for case in cases[1:]:
        for got, want in zip(results[case], base):
            np.testing.assert_array_equal(got, want, err_msg=str(case))
    np.testing.assert_allclose(base[0], oracle.matmul(x_up, "up", init=init), rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(base[2], oracle.matmul(results["x_dn"], "down", miss=results["miss"].copy()), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("k", [2, 8])
def test_programmatic_dependent_launch_is_bit_identical(synth_artifact, k):
    """Level, seed and output kernels launched with and without programmatic dependent launch
    (on by default from k = 8) give bit-identical results, through the recorded CUDA graphs."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    rng = np.random.default_rng(1300 + k)
    results = {}
    x_up = x_dn = miss = None
    for pdl in (None, True, False):
        plan = B200Plan(heavy_threshold=24, pdl=pdl)
        with _runtime(_layout([synth_artifact], requirements=_req(k=k), pair=B200PlanPair(plan_up=plan, plan_down=plan))) as runtime:
            (grg,) = runtime.grgs
            if x_up is None:
                x_up = rng.standard_normal((k, grg.num_samples))
                x_dn, miss = rng.standard_normal((k, grg.num_mutations)), rng.standard_normal((k, grg.num_mutations))
            outs = []
            for _ in range(2):
                up = grg.prepare_matmul_cuda(direction="up", k=k)
                down = grg.prepare_matmul_cuda(direction="down", k=k, use_miss=True)
                up.input.copy_(torch.from_numpy(x_up))
                up()
                outs.append(up.output.cpu().numpy())
                down.input.copy_(torch.from_numpy(x_dn))
                down.miss_input.copy_(torch.from_numpy(miss))
                down()
                outs.append(down.output.cpu().numpy())
            results[pdl] = outs
            assert runtime.device_error() == 0
    for pdl in (True, False):
        for got, want in zip(results[pdl], results[None]):
            np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("k", [1, 8, 33])
@pytest.mark.parametrize("fuse", ["small", "all-heavy"])
def test_fused_level_runs_are_bit_identical(synth_artifact, k, fuse):
    """Stretches of small levels run as one cooperative launch with grid barriers give the
    same bits as one launch per level: with the default heavy threshold and the small levels
    fused, and with heavy rows in every level (threshold 2) and every level fused."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    rng = np.random.default_rng(1500 + k)
    threshold, entries = (24, 20_000) if fuse == "small" else (2, 1 << 40)
    results = {}
    inputs = None
    for fuse_entries in (0, entries):
        plan = B200Plan(heavy_threshold=threshold, narrow_split=0, fuse_entries=fuse_entries)
        with _runtime(_layout([synth_artifact], requirements=_req(k=max(k, 2)), pair=B200PlanPair(plan_up=plan, plan_down=plan))) as runtime:
            (grg,) = runtime.grgs
            if inputs is None:
                inputs = (rng.standard_normal((k, grg.num_samples)), rng.standard_normal((k, grg.num_mutations)),
                          rng.standard_normal((k, grg.num_mutations)), rng.standard_normal(k))
            x_up, x_dn, miss, init = inputs
            results[fuse_entries] = [grg.matmul(x_up, "up"), grg.matmul(x_up, "up", init=init), grg.matmul(x_up, "up", init="xtx"),
                                     grg.matmul(x_dn, "down", miss=miss.copy()), grg.matmul(x_dn, "down", init=init),
                                     grg.matmul(_pm1(np.random.default_rng(3), (k, grg.num_individuals)), "up", by_individual=True)]
            assert runtime.device_error() == 0
            if fuse_entries:
                levels = runtime._artifacts[0].levels
                fused = [lv for d in levels for lv in levels[d].array if 0 < lv.num_entries <= fuse_entries]
                assert len(fused) >= 4  # the runs are not empty
    for got, want in zip(results[entries], results[0]):
        np.testing.assert_array_equal(got, want)
    oracle = OracleGRG(synth_artifact)
    x_up, x_dn, miss, _ = inputs
    np.testing.assert_allclose(results[entries][0], oracle.matmul(x_up, "up"), rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(results[entries][3], oracle.matmul(x_dn, "down", miss=miss.copy()), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("k", [8, 16])
@pytest.mark.parametrize("variant", [13, 14])
def test_short_row_walk_sums_any_list_length(synth_artifact, variant, k):
    """The entry-parallel walks take a level's ``short_rows`` (the narrow suffix of lists of at
    most one quad) with one entry slot.  The count is only a speed hint: as built, with none,
    and with every narrow row walked that way (lists of several quads included), integer inputs
    give the oracle's results exactly and real ones agree within 1e-12."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, B200Runtime

    oracle = OracleGRG(synth_artifact)
    plan = B200Plan(narrow_variant=variant, heavy_threshold=24, heavy_variant=2, narrow_split=0)
    layout = _layout([synth_artifact], requirements=_req(k=k), pair=B200PlanPair(plan_up=plan, plan_down=plan))
    for mode in ("built", "none", "all"):
        rng = np.random.default_rng(900 + k)
        with B200Runtime(layout, check_bounds=False) as runtime:
            (grg,) = runtime.grgs
            levels = runtime._artifacts[0].levels
            arrays = [levels[d].array for d in levels]
            if mode == "built":
                assert any(lv.num_heavy > 0 for arr in arrays for lv in arr)
                assert any(lv.short_rows > 0 for arr in arrays for lv in arr)
                assert any(0 < lv.short_rows < lv.num_rows - lv.num_heavy for arr in arrays for lv in arr)
            for arr in arrays:
                for lv in arr:
                    if mode == "none":
                        lv.short_rows = 0
                    elif mode == "all":
                        lv.short_rows = lv.num_rows - lv.num_heavy
            S, M = grg.num_samples, grg.num_mutations
            for direction, cols in (("up", S), ("down", M)):
                xi, xr = _pm1(rng, (k, cols)), rng.standard_normal((k, cols))
                np.testing.assert_array_equal(grg.matmul(xi, direction), oracle.matmul(xi, direction))
                np.testing.assert_allclose(grg.matmul(xr, direction), oracle.matmul(xr, direction), rtol=1e-12, atol=1e-9)
            xd, miss = _pm1(rng, (k, M)), _pm1(rng, (k, M))
            np.testing.assert_array_equal(grg.matmul(xd, "down", miss=miss.copy()), oracle.matmul(xd, "down", miss=miss.copy()))
            assert runtime.device_error() == 0


@pytest.mark.parametrize("k", [1, 2, 3, 8, 16, 33])
def test_lean_walks_match_variant_7_and_the_oracle(synth_artifact, k):
    """Narrow variants 11 to 14 (the lean walks, used by launches without a bounds-check word
    and without row splits) on every mode of the hot path: 11 returns the same bits as 7 and 14
    the same as 13; 12 (one partial sum per row) and 13 (entry-parallel rows, in 32-byte
    chunks, or one vector per lane at k = 1 and 2, where the init allows it) are exact for
    integer-valued inputs and within 1e-12 otherwise."""
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, B200Runtime

    oracle = OracleGRG(synth_artifact)
    results = {}
    for variant in (7, 11, 12, 13, 14, 15, 16):
        plan = B200Plan(narrow_variant=variant, heavy_threshold=24, heavy_variant=2, narrow_split=0)
        layout = _layout([synth_artifact], requirements=_req(k=max(k, 2)), pair=B200PlanPair(plan_up=plan, plan_down=plan))
        rng = np.random.default_rng(300 + k)  # the same inputs for every variant
        with B200Runtime(layout, check_bounds=False) as runtime:
            (grg,) = runtime.grgs
            S, M, N, I = grg.num_samples, grg.num_mutations, grg.num_nodes, grg.num_individuals
            out = []
            for direction, cols in (("up", S), ("down", M)):
                xi, xr = _pm1(rng, (k, cols)), rng.standard_normal((k, cols))
                out.append(("int", grg.matmul(xi, direction), oracle.matmul(xi, direction)))
                out.append(("real", grg.matmul(xr, direction), oracle.matmul(xr, direction)))
                init = rng.standard_normal(k)
                out.append(("real", grg.matmul(xr, direction, init=init), oracle.matmul(xr, direction, init=init)))
                out.append(("real", grg.matmul(xr, direction, init="xtx"), oracle.matmul(xr, direction, init="xtx")))
                mat = rng.standard_normal((k, N))
                out.append(("real", grg.matmul(xr, direction, init=mat, emit_all_nodes=True),
                            oracle.matmul(xr, direction, init=mat, emit_all_nodes=True)))
            xi = _pm1(rng, (k, I))
            miss_b, miss_o = np.zeros((k, M)), np.zeros((k, M))
            out.append(("int", grg.matmul(xi, "up", by_individual=True, miss=miss_b),
                        oracle.matmul(xi, "up", by_individual=True, miss=miss_o)))
            out.append(("int", miss_b, miss_o))
            xd, miss = _pm1(rng, (k, M)), _pm1(rng, (k, M))
            out.append(("int", grg.matmul(xd, "down", by_individual=True, miss=miss.copy()),
                        oracle.matmul(xd, "down", by_individual=True, miss=miss.copy())))
            results[variant] = out
    for (kind, got7, ref), (_, got11, _), (_, got12, _), (_, got13, _), (_, got14, _), (_, got15, _), (_, got16, _) in zip(
            results[7], results[11], results[12], results[13], results[14], results[15], results[16]):
        np.testing.assert_array_equal(got11, got7)
        np.testing.assert_array_equal(got14, got13)  # the same sums, codes loaded earlier
        np.testing.assert_array_equal(got15, got14)  # the same walk in 4-warp CTAs
        np.testing.assert_array_equal(got16, got14)  # and in 2-warp CTAs
        if kind == "int":
            np.testing.assert_array_equal(got12, ref)
            np.testing.assert_array_equal(got13, ref)
            np.testing.assert_array_equal(got7, ref)
        else:
            np.testing.assert_allclose(got12, ref, rtol=1e-12, atol=1e-9)
            np.testing.assert_allclose(got13, ref, rtol=1e-12, atol=1e-9)
