"""The vectorised compiler and the synthetic generator."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from grg_spmv_b200.compile import DagGRG, build_init_biases, compile_dag, compute_node_levels
from grg_spmv_b200.synth import CONFIG1, SynthSpec, generate_dag, generate_state
from grg_oracle import OracleGRG


def _tiny_dag(**kw):
    # samples 0..3; node 4 = {0,1}; node 5 = {2,3}; node 6 = {4,5}; node 7 = {6} ... levels 0,1,2,3
    base = dict(num_samples=4, num_nodes=8,
                child_indptr=np.asarray([0, 0, 0, 0, 0, 2, 4, 6, 7]),
                child_indices=np.asarray([0, 1, 2, 3, 4, 5, 6]),
                mut_node=np.asarray([4, 7, -1, 2]), miss_node=np.asarray([-1, -1, 5, -1]))
    base.update(kw)
    return DagGRG(**base)


def test_levels_and_stable_order():
    state = compile_dag(_tiny_dag())
    np.testing.assert_array_equal(state.level_offsets, [0, 4, 6, 7, 8])
    np.testing.assert_array_equal(state.node_perm, np.arange(8))
    assert state.num_edges == 7
    assert state.sel_mut.nnz == 3 and state.sel_miss.nnz == 1


def test_cycle_and_duplicate_edge_are_rejected():
    with pytest.raises(RuntimeError, match="Duplicate"):
        compile_dag(_tiny_dag(child_indptr=np.asarray([0, 0, 0, 0, 0, 2, 4, 6, 8]),
                              child_indices=np.asarray([0, 1, 2, 3, 4, 5, 6, 6])))
    with pytest.raises(ValueError, match="1 \\+ max child level"):
        compile_dag(_tiny_dag(node_levels=np.asarray([0, 0, 0, 0, 1, 1, 2, 2])))


def test_init_biases_are_descendant_path_counts():
    state = compile_dag(_tiny_dag())
    build_init_biases(state)
    # vector bias up: sum over the mutation node's sub-DAG of 1 per node visit.
    np.testing.assert_array_equal(state.init_vector_up_bias, [3.0, 8.0, 0.0, 1.0])


def test_generator_has_no_duplicate_sample_paths():
    spec = dataclasses.replace(CONFIG1, num_nodes=20_000, num_mutations=3000, random_ids=True)
    dag = generate_dag(spec)
    np.testing.assert_array_equal(compute_node_levels(dag.num_nodes, dag.child_indptr, dag.child_indices), dag.node_levels)
    state = compile_dag(dag)
    assert len(state.level_offsets) - 1 == spec.num_levels + 1
    assert not np.array_equal(state.node_perm, np.arange(state.num_nodes))
    build_init_biases(state)


def test_generator_allele_counts_bounded(tmp_path):
    from grg_spmv_b200.artifact import save_grg_spmv

    spec = SynthSpec(num_samples=300, num_levels=10, num_nodes=4000, num_mutations=800, children=(2, 12), seed=4)
    state = generate_state(spec)
    save_grg_spmv(state, tmp_path / "g.grg_spmv")
    counts = OracleGRG(tmp_path / "g.grg_spmv").matmul(np.ones((1, 300)), "up")
    assert counts.max() <= 300 and counts.min() >= 0
