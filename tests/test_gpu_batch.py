"""Batched matmuls (several GRGs and uneven RHS blocks in one CUDA graph) against the FP64
oracle, plain and mixed precision, merged and tiled, autotuned."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from grg_spmv_b200 import RuntimeRequirements  # noqa: E402
from grg_oracle import OracleGRG  # noqa: E402

MIXED_RTOL = 1e-10  # max |got - ref| / max |ref| per item
PLAIN_RTOL = 1e-12


def _rel(got, ref):
    return float(np.abs(got - ref).max() / max(float(np.abs(ref).max()), 1e-300))


@pytest.fixture(scope="module")
def two_artifacts(tmp_path_factory):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    root = tmp_path_factory.mktemp("batch")
    paths = []
    for i, (nodes, muts) in enumerate(((40_000, 8_000), (25_000, 5_000))):
        path = root / f"g{i}.grg_spmv"
        write_synthetic_artifact(SynthSpec(num_samples=2000 + 500 * i, num_levels=12, num_nodes=nodes, num_mutations=muts,
                                           children=(2, 16), miss_fraction=0.02, random_ids=True, seed=40 + i), path)
        paths.append(path)
    return paths


def _runtime(paths, precision="plain"):
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    req = RuntimeRequirements(max_k_up=8, max_k_down=8, need_down_miss_input=True, need_up_miss_output=False,
                              need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
    layout = plan_b200_layout(artifacts=[str(p) for p in paths], dtype=np.float64, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0, precision=precision)
    return B200Runtime(layout, check_bounds=True)


BLOCKS = (1, 3, 16, 5)


@pytest.mark.parametrize("precision", ["plain", "mixed"])
@pytest.mark.parametrize("tile_k", [None, 8, 4])
def test_batch_matches_oracle(two_artifacts, precision, tile_k):
    oracles = [OracleGRG(p) for p in two_artifacts]
    rng = np.random.default_rng(5)
    with _runtime(two_artifacts) as runtime:
        grgs = runtime.grgs
        items = []
        for g in grgs:
            for k in BLOCKS:
                items.append((g, "up", k))
                items.append((g, "down", k, True))
        with runtime.prepare_batch(items, precision=precision, tile_k=tile_k) as batch:
            assert batch.num_tiles >= 4
            refs = []
            for i, (g, direction, k, *miss) in enumerate(items):
                oracle = oracles[grgs.index(g)]
                cols = g.num_samples if direction == "up" else g.num_mutations
                x = rng.standard_normal((k, cols)) if i % 3 else rng.choice([-1.0, 1.0], size=(k, cols))
                batch.inputs[i].copy_(torch.from_numpy(x))
                m = None
                if miss:
                    m = rng.standard_normal((k, g.num_mutations)) if i % 3 else rng.choice([-1.0, 1.0], size=(k, g.num_mutations))
                    batch.miss_inputs[i].copy_(torch.from_numpy(m))
                refs.append(oracle.matmul(x, direction, miss=None if m is None else m.copy()))
            for _ in range(2):  # replays give the same results
                batch()
                torch.cuda.synchronize()
                for i, ref in enumerate(refs):
                    got = batch.outputs[i].cpu().numpy()
                    assert got.shape == ref.shape
                    tol = MIXED_RTOL if precision == "mixed" else PLAIN_RTOL
                    assert _rel(got, ref) <= tol, (i, items[i][1:], _rel(got, ref))
                    if i % 3 == 0:  # integer-valued inputs are exact in both precisions
                        np.testing.assert_array_equal(got, ref)
        assert runtime.device_error() == 0


def test_batch_autotune_picks_a_tile_and_stays_correct(two_artifacts):
    oracle = OracleGRG(two_artifacts[0])
    rng = np.random.default_rng(9)
    with _runtime(two_artifacts, precision="mixed") as runtime:
        g = runtime.grgs[0]
        with runtime.prepare_batch([(g, "up", 24), (g, "up", 40)], autotune=True) as batch:
            assert batch.precision == "mixed"
            assert batch.tuned_ms and batch.tile_k in (None, 32, 16)
            xs = [rng.standard_normal((k, g.num_samples)) for k in (24, 40)]
            for i, x in enumerate(xs):
                batch.inputs[i].copy_(torch.from_numpy(x))
            batch()
            for i, x in enumerate(xs):
                assert _rel(batch.outputs[i].cpu().numpy(), oracle.matmul(x, "up")) <= MIXED_RTOL
            assert batch.edge_rhs() == g.num_edges * 64
        assert runtime.device_error() == 0


def test_batch_rejects_bad_items(two_artifacts):
    with _runtime(two_artifacts) as runtime:
        g = runtime.grgs[0]
        with pytest.raises(ValueError):
            runtime.prepare_batch([])
        with pytest.raises(ValueError):
            runtime.prepare_batch([(g, "up", 4, True)])
        with pytest.raises(ValueError):
            runtime.prepare_batch([(g, "up", 4)], precision="mixed", tile_k=6)
