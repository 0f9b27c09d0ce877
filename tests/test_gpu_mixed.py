"""Mixed precision (6-byte node state: FP32 value + 16-bit correction, FP64 sums) against the
FP64 oracle on a synthetic graph with random node ids, every mode of the hot path."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from grg_spmv_b200 import RuntimeRequirements  # noqa: E402
from grg_oracle import OracleGRG  # noqa: E402

MIXED_RTOL = 1e-10  # max |got - ref| / max |ref| per result


def _rel(got, ref):
    return float(np.abs(got - ref).max() / max(float(np.abs(ref).max()), 1e-300))


def _req(k):
    return RuntimeRequirements(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=True,
                               need_init_vector=True, need_init_matrix=True, need_init_xtx=True)


def _runtime(path, k, **kw):
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    layout = plan_b200_layout(artifacts=[str(path)], dtype=np.float64, requirements=_req(k), vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0, precision="mixed", **kw)
    return B200Runtime(layout, check_bounds=True)


def _pm1(rng, shape):
    return rng.choice(np.asarray([-1.0, 1.0]), size=shape)


@pytest.fixture(scope="module")
def synth_artifact(tmp_path_factory):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    path = tmp_path_factory.mktemp("mixed") / "mid.grg_spmv"
    write_synthetic_artifact(SynthSpec(num_samples=3000, num_levels=14, num_nodes=60_000, num_mutations=15_000, children=(2, 16),
                                       miss_fraction=0.02, ploidy=2, with_coalescence=True, random_ids=True, seed=23), path)
    return path


@pytest.mark.parametrize("k", [1, 3, 4, 8, 32, 33])
@pytest.mark.parametrize("heavy", [24, 10_000], ids=["heavy-rows", "narrow"])
def test_mixed_against_oracle(synth_artifact, k, heavy):
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair

    oracle = OracleGRG(synth_artifact)
    pair = B200PlanPair(plan_up=B200Plan(heavy_threshold=heavy), plan_down=B200Plan(heavy_threshold=heavy))
    rng = np.random.default_rng(300 + k)
    with _runtime(synth_artifact, k, pair=pair) as runtime:
        (grg,) = runtime.grgs
        S, M, N, I = grg.num_samples, grg.num_mutations, grg.num_nodes, grg.num_individuals
        for direction, cols in (("up", S), ("down", M)):
            x = _pm1(rng, (k, cols))
            np.testing.assert_array_equal(grg.matmul(x, direction), oracle.matmul(x, direction))
            x = rng.standard_normal((k, cols))
            assert _rel(grg.matmul(x, direction), oracle.matmul(x, direction)) <= MIXED_RTOL
            init = rng.standard_normal(k)
            assert _rel(grg.matmul(x, direction, init=init), oracle.matmul(x, direction, init=init)) <= MIXED_RTOL
            assert _rel(grg.matmul(x, direction, init="xtx"), oracle.matmul(x, direction, init="xtx")) <= MIXED_RTOL
            mat = rng.standard_normal((k, N))
            assert _rel(grg.matmul(x, direction, init=mat, emit_all_nodes=True),
                        oracle.matmul(x, direction, init=mat, emit_all_nodes=True)) <= MIXED_RTOL
        xi = _pm1(rng, (k, I))
        miss_b, miss_o = np.zeros((k, M)), np.zeros((k, M))
        np.testing.assert_array_equal(grg.matmul(xi, "up", by_individual=True, miss=miss_b),
                                      oracle.matmul(xi, "up", by_individual=True, miss=miss_o))
        np.testing.assert_array_equal(miss_b, miss_o)
        xd, miss = _pm1(rng, (k, M)), _pm1(rng, (k, M))
        np.testing.assert_array_equal(grg.matmul(xd, "down", by_individual=True, miss=miss.copy()),
                                      oracle.matmul(xd, "down", by_individual=True, miss=miss.copy()))
        xd, miss = rng.standard_normal((k, M)), rng.standard_normal((k, M))
        assert _rel(grg.matmul(xd, "down", miss=miss.copy()), oracle.matmul(xd, "down", miss=miss.copy())) <= MIXED_RTOL
        assert runtime.device_error() == 0


def test_mixed_large_integers_stay_exact(synth_artifact):
    """Integer inputs whose node sums reach ~2^33 are still exact (stored values carry 39 bits)."""
    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(7)
    with _runtime(synth_artifact, 4) as runtime:
        (grg,) = runtime.grgs
        x = rng.integers(-(2**21), 2**21, size=(4, grg.num_samples)).astype(np.float64)
        ref = oracle.matmul(x, "up")
        assert np.abs(ref).max() > 2**24  # beyond FP32's exact range
        np.testing.assert_array_equal(grg.matmul(x, "up"), ref)
        assert runtime.device_error() == 0


def test_mixed_prepared_ops_and_graph_replay(synth_artifact):
    """Prepared ops (captured CUDA graphs) in mixed precision: up then down in place, replayed."""
    oracle = OracleGRG(synth_artifact)
    rng = np.random.default_rng(11)
    k = 8
    with _runtime(synth_artifact, k) as runtime:
        (grg,) = runtime.grgs
        up = grg.prepare_matmul_cuda(direction="up", k=k)
        down = grg.prepare_matmul_cuda(direction="down", k=k, use_miss=True)
        x = rng.standard_normal((k, grg.num_samples))
        miss = rng.standard_normal((k, grg.num_mutations))
        ref_up = oracle.matmul(x, "up")
        ref_down = oracle.matmul(ref_up, "down", miss=miss.copy())
        stream = runtime._torch_caller_stream()
        with torch.cuda.stream(stream):
            for _ in range(3):
                up.input.copy_(torch.from_numpy(x))
                down.miss_input.copy_(torch.from_numpy(miss))
                up()
                got_up = up.output.cpu().numpy()
                down()
                got_down = down.output.cpu().numpy()
                assert _rel(got_up, ref_up) <= MIXED_RTOL
                assert _rel(got_down, ref_down) <= MIXED_RTOL
        assert runtime.device_error() == 0


def test_mixed_layout_sizes(synth_artifact):
    from grg_spmv_b200.backends.b200 import _native as nat

    with _runtime(synth_artifact, 8) as runtime:
        lay = runtime.layout
        assert lay.precision == "mixed"
        assert lay.bytes_by_category["state"] == nat.mix_bytes(lay.max_num_nodes, 8) == runtime._state.numel()
        assert runtime._mix_scratch.numel() == lay.mix_scratch_bytes == 2 * nat.mix_bytes(lay.max_num_mutations, 8)
