"""Standardised genotype Gram operator (the reference's PreparedXTX) and randomized PCA on the
B200 backend, against a CPU model built on the oracle."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from _xtx_model import standardized_xtx_reference  # noqa: E402
from grg_oracle import OracleGRG  # noqa: E402
from grg_spmv_b200 import RuntimeRequirements  # noqa: E402

PLAIN_RTOL = 1e-11   # max |got - ref| / max |ref|
MIXED_RTOL = 1e-10


@pytest.fixture(scope="module")
def diploid_artifact(tmp_path_factory):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    path = tmp_path_factory.mktemp("xtx") / "dip.grg_spmv"
    write_synthetic_artifact(SynthSpec(num_samples=1200, num_levels=10, num_nodes=12_000, num_mutations=700, children=(2, 12),
                                       miss_fraction=0.02, ploidy=2, random_ids=True, seed=31), path)
    return path


def _runtime(path, q, precision):
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    req = RuntimeRequirements(max_k_up=q, max_k_down=q, need_down_miss_input=True, need_up_miss_output=True,
                              need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
    layout = plan_b200_layout(artifacts=[str(path)], dtype=np.float64, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0, precision=precision)
    return B200Runtime(layout, check_bounds=True)


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_standardized_xtx_matches_cpu_model(diploid_artifact, precision):
    from grg_spmv_b200.xtx import StandardizedXTX

    oracle = OracleGRG(diploid_artifact)
    rng = np.random.default_rng(3)
    q = 6
    with _runtime(diploid_artifact, q, precision) as runtime:
        (grg,) = runtime.grgs
        assert grg.has_missing_data and grg.ploidy == 2
        op = StandardizedXTX(runtime, grg, q)
        for _ in range(2):
            v = rng.standard_normal((grg.num_mutations, q))
            got = op.apply(torch.from_numpy(v).cuda()).cpu().numpy()
            ref = standardized_xtx_reference(oracle, grg.ploidy, True, v)
            err = float(np.abs(got - ref).max() / np.abs(ref).max())
            assert err <= (PLAIN_RTOL if precision == "plain" else MIXED_RTOL), err
        assert runtime.device_error() == 0


def test_randomized_pca_finds_the_top_eigenvalues(diploid_artifact):
    from grg_spmv_b200.xtx import StandardizedXTX, randomized_eigh

    oracle = OracleGRG(diploid_artifact)
    pcs, over = 4, 8
    with _runtime(diploid_artifact, pcs + over, "plain") as runtime:
        (grg,) = runtime.grgs
        op = StandardizedXTX(runtime, grg, pcs + over)
        values, vectors = randomized_eigh(op, pcs, oversample=over, power_iters=10, seed=1)
        values = values.cpu().numpy()
        vectors = vectors.cpu().numpy()
    dense = standardized_xtx_reference(oracle, 2, True, np.eye(oracle.num_mutations))
    dense = 0.5 * (dense + dense.T)
    exact = np.sort(np.linalg.eigvalsh(dense))[::-1][:pcs]
    np.testing.assert_allclose(values, exact, rtol=1e-4)  # subspace iteration converged to 1e-4
    assert vectors.shape == (oracle.num_mutations, pcs)
    np.testing.assert_allclose(vectors.T @ vectors, np.eye(pcs), atol=1e-10)


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_kinship_cg_solve(diploid_artifact, precision):
    """(Z Zᵀ / M + delta I) x = b for 5 right-hand sides by block CG against a dense solve."""
    from grg_spmv_b200.xtx import StandardizedXXT, conj_grad_solve

    oracle = OracleGRG(diploid_artifact)
    rng = np.random.default_rng(12)
    c, delta = 5, 0.7
    with _runtime(diploid_artifact, c, precision) as runtime:
        (grg,) = runtime.grgs
        M, I = grg.num_mutations, grg.num_individuals
        op = StandardizedXXT(runtime, grg, c)
        b = rng.standard_normal((I, c))
        x, iters, rels = conj_grad_solve(lambda v: op.apply(v) / M + delta * v, torch.from_numpy(b).cuda(),
                                         rel_tol=1e-9, max_iter=200)
        x = x.cpu().numpy()
        assert float(rels.max()) <= 1e-9 and iters < 200
    z = _dense_z(oracle, grg_ploidy=2)
    k_mat = z @ z.T / M + delta * np.eye(I)
    ref = np.linalg.solve(k_mat, b)
    assert float(np.abs(x - ref).max() / np.abs(ref).max()) <= 1e-7


def _dense_z(oracle, grg_ploidy):
    """Dense standardised genotype matrix (individuals x mutations) with missing entries set to
    the allele mean, from oracle products of identity blocks."""
    M, I = oracle.num_mutations, oracle.num_individuals
    geno = oracle.matmul(np.eye(I), "up", by_individual=True)            # (I, M): X
    miss = np.zeros((I, M))
    oracle.matmul(np.eye(I), "up", by_individual=True, miss=miss)        # missing indicators per individual
    ones_miss = np.zeros((1, M))
    counts = oracle.matmul(np.ones((1, I)), "up", by_individual=True, miss=ones_miss)[0]
    denom = float(oracle.num_samples) - ones_miss[0]
    freqs = np.where(denom != 0, counts / np.where(denom != 0, denom, 1.0), 0.0)
    center = grg_ploidy * freqs
    sigma = np.sqrt(grg_ploidy * freqs * (1.0 - freqs))
    sigma = np.where(sigma == 0.0, 1.0, sigma)
    x = geno + miss * freqs[None, :]
    return (x - center[None, :]) / sigma[None, :]
