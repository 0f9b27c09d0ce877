"""Regenerate the golden fixtures in this directory from the reference package itself.

Run from the repository root, in a container where the reference checkout exists:

    python tests/golden/make_golden.py /path/to/reference

What it does (the reference cannot travel to GPU machines, so its outputs are committed):

1. Imports the reference package with the test-only ``_standin/pygrgl.py`` on ``sys.path``
   (``pygrgl`` itself is not installable offline; the stand-in only supplies names).
2. Writes artifacts with the *reference's own* writers:
   - ``band3.grg_spmv`` / ``overlap4.grg_spmv``: ``write_three_level_band_artifact`` and
     ``write_overlap_band_artifact`` from ``pygrgl_spmv/tests/runtime/_streaming_cases.py``;
   - ``synth_*.grg_spmv``: small DAGs from ``grg_spmv_b200.synth`` compiled by the
     reference's ``compile_grg`` through a duck-typed GRG, biases by ``_build_init_biases``,
     saved by ``save_grg_spmv`` (one of them with repeated mutation rows, which gives a
     mutation several nodes);
   - ``sparse_selector.grg_spmv``: the one-sample sparse-selector case of
     ``pygrgl_spmv/tests/runtime/test_directional_layouts.py:104-132``.
3. Checks that ``grg_spmv_b200.compile.compile_dag`` reproduces the reference compile array
   for array (values and dtypes).
4. Runs ``ReferenceRuntime`` (``BoundGRG.matmul``) over seeded inputs for every mode the hot
   path supports and stores inputs and outputs in ``cases.npz``; asserts that the oracle
   (``oracle/grg_oracle.py``) reproduces every output exactly.
"""

from __future__ import annotations

import dataclasses
import json
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _setup(reference_root: Path) -> None:
    sys.path.insert(0, str(HERE / "_standin"))
    sys.path.insert(0, str(reference_root))
    sys.path.insert(0, str(REPO))


class DuckGRG:
    """The attributes and methods of ``pygrgl.ImmutableGRG`` that ``compile_grg`` uses."""

    def __init__(self, dag, pygrgl, repeat_every: int = 0):
        self.dag = dag
        self._pygrgl = pygrgl
        self.num_samples = dag.num_samples
        self.num_nodes = dag.num_nodes
        self.num_mutations = dag.num_mutations
        self.num_edges = dag.num_edges
        self.ploidy = dag.ploidy
        self.num_individuals = dag.num_individuals
        self.has_missing_data = bool(np.any(dag.miss_node >= 0))
        self.has_individual_coals = dag.coalescence_counts is not None
        self.repeat_every = repeat_every

    def get_down_edges(self, node):
        lo, hi = int(self.dag.child_indptr[node]), int(self.dag.child_indptr[node + 1])
        return [int(c) for c in self.dag.child_indices[lo:hi]]

    def get_mutation_node_miss(self):
        inv = int(self._pygrgl.INVALID_NODE)
        rows = []
        for m in range(self.num_mutations):
            node = int(self.dag.mut_node[m])
            miss = int(self.dag.miss_node[m])
            rows.append((m, inv if node < 0 else node, inv if miss < 0 else miss))
            if self.repeat_every and m % self.repeat_every == 0:
                # A repeated mutation row: same id, another node, no missingness node.
                rows.append((m, (node * 7 + 3) % self.num_nodes, inv))
        return rows

    def get_num_individual_coals(self, node):
        if self.dag.coalescence_counts is None:
            return int(self._pygrgl.COAL_COUNT_NOT_SET)
        return int(self.dag.coalescence_counts[node])

    def get_mutation_by_id(self, m):
        return self._pygrgl.Mutation(float(m) * 10.0 + 0.5, "T", "C", float(m % 7))


def _compare_states(ref_state, ours) -> None:
    for field in ("level_offsets", "node_perm", "inv_node_perm", "sample_to_individual"):
        a, b = np.asarray(getattr(ref_state, field)), np.asarray(getattr(ours, field))
        assert a.dtype == b.dtype and np.array_equal(a, b), field
    for name in ("sel_mut", "sel_miss"):
        a, b = getattr(ref_state, name), getattr(ours, name)
        for part in ("indices", "indptr"):
            x, y = getattr(a, part), getattr(b, part)
            assert x.dtype == y.dtype and np.array_equal(x, y), (name, part)
    for dst, row in enumerate(ref_state.A_blocks):
        for src, block in enumerate(row):
            mine = ours.A_blocks[dst][src]
            assert block.shape == mine.shape, (dst, src)
            for part in ("indices", "indptr"):
                x, y = getattr(block, part), getattr(mine, part)
                assert x.dtype == y.dtype and np.array_equal(x, y), (dst, src, part)
    if ref_state.coalescence_counts is None:
        assert ours.coalescence_counts is None
    else:
        assert np.array_equal(ref_state.coalescence_counts, ours.coalescence_counts)


SYNTH_CASES = {
    "synth_haploid": dict(num_samples=96, num_levels=6, num_nodes=700, num_mutations=160, children=(2, 8), random_ids=True, seed=11,
                          neighbor_scale=0.5, prefer_largest=0.0),
    "synth_diploid": dict(num_samples=120, num_levels=7, num_nodes=900, num_mutations=200, children=(2, 6), ploidy=2,
                          miss_fraction=0.05, with_coalescence=True, random_ids=True, seed=12, neighbor_scale=0.5,
                          prefer_largest=0.0),
    "synth_repeat": dict(num_samples=64, num_levels=5, num_nodes=400, num_mutations=90, children=(2, 5), miss_fraction=0.1,
                         random_ids=True, seed=13, neighbor_scale=0.5, prefer_largest=0.0),
}


def _write_artifacts(out: Path):
    import scipy.sparse as sp
    import pygrgl
    from pygrgl_spmv.grg import _build_init_biases
    from pygrgl_spmv.grg.artifact import save_grg_spmv
    from pygrgl_spmv.grg.compile import compile_grg
    from pygrgl_spmv.grg.sparse import binary_csr_from_parts
    from pygrgl_spmv.tests.runtime._streaming_cases import (
        _synthetic_state,
        write_overlap_band_artifact,
        write_three_level_band_artifact,
    )

    from grg_spmv_b200.compile import compile_dag
    from grg_spmv_b200.synth import SynthSpec, generate_dag

    paths = {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        p = write_three_level_band_artifact(tmp, "band3", n=64, bandwidth=8, shifts=(0, 8, 16))
        shutil.copy(p, out / "band3.grg_spmv")
        paths["band3"] = out / "band3.grg_spmv"
        p = write_overlap_band_artifact(tmp, "overlap4", n=16, bandwidth=4)
        shutil.copy(p, out / "overlap4.grg_spmv")
        paths["overlap4"] = out / "overlap4.grg_spmv"

    for name, kwargs in SYNTH_CASES.items():
        dag = generate_dag(SynthSpec(**kwargs))
        repeat = 9 if name == "synth_repeat" else 0
        ref_state = compile_grg(DuckGRG(dag, pygrgl, repeat_every=repeat))
        if not repeat:
            _compare_states(ref_state, compile_dag(dataclasses.replace(dag, node_levels=None)))
            _compare_states(ref_state, compile_dag(dag))
        _build_init_biases(ref_state, np.dtype(np.float64))
        save_grg_spmv(ref_state, out / f"{name}.grg_spmv")
        paths[name] = out / f"{name}.grg_spmv"

    # One sample, one internal node, five mutations of which only the first is placed.
    sel_mut = binary_csr_from_parts(indices=np.asarray([1], np.int32), indptr=np.asarray([0, 1, 1, 1, 1, 1], np.int32),
                                    shape=(5, 2), shared_data=True)
    sel_miss = binary_csr_from_parts(indices=np.empty(0, np.int32), indptr=np.zeros(6, np.int32), shape=(5, 2), shared_data=True)
    state = _synthetic_state(blocks=[[], [sp.csr_matrix((1, 1), dtype=np.bool_)]], level_offsets=np.asarray([0, 1, 2], np.int32),
                             num_samples=1, num_mutations=5, num_nodes=2, sel_mut=sel_mut, sel_miss=sel_miss)
    save_grg_spmv(state, out / "sparse_selector.grg_spmv")
    paths["sparse_selector"] = out / "sparse_selector.grg_spmv"
    return paths


def _cases_for(name: str, grg, rng):
    """(case id, kwargs) pairs; inputs are drawn here and stored alongside the outputs."""
    cases = []
    S, M, N, I = grg.num_samples, grg.num_mutations, grg.num_nodes, grg.num_individuals
    kinds = ("pm1", "normal", "ones", "zeros")

    def draw(kind, shape):
        if kind == "pm1":
            return rng.choice(np.asarray([-1.0, 1.0]), size=shape)
        if kind == "normal":
            return rng.standard_normal(shape)
        if kind == "ones":
            return np.ones(shape)
        return np.zeros(shape)

    for direction, cols in (("up", S), ("down", M)):
        for k in (1, 2, 3, 8):
            for kind in kinds:
                cases.append((f"{direction}-k{k}-{kind}", dict(x=draw(kind, (k, cols)), direction=direction)))
        k = 3
        cases.append((f"{direction}-vector", dict(x=draw("normal", (k, cols)), direction=direction, init=rng.standard_normal(k))))
        cases.append((f"{direction}-matrix", dict(x=draw("normal", (k, cols)), direction=direction, init=rng.standard_normal((k, N)))))
        cases.append((f"{direction}-emit", dict(x=draw("normal", (k, cols)), direction=direction, emit_all_nodes=True)))
        cases.append((f"{direction}-emit-vector", dict(x=draw("normal", (k, cols)), direction=direction, emit_all_nodes=True,
                                                       init=rng.standard_normal(k))))
        cases.append((f"{direction}-emit-matrix", dict(x=draw("normal", (k, cols)), direction=direction, emit_all_nodes=True,
                                                       init=rng.standard_normal((k, N)))))
        if grg.coalescence_counts is not None:
            cases.append((f"{direction}-xtx", dict(x=draw("normal", (k, cols)), direction=direction, init="xtx")))
            cases.append((f"{direction}-emit-xtx", dict(x=draw("normal", (k, cols)), direction=direction, init="xtx",
                                                        emit_all_nodes=True)))
        cases.append((f"{direction}-miss", dict(x=draw("normal", (k, cols)), direction=direction,
                                                 miss=draw("normal", (k, M)) if direction == "down" else np.zeros((k, M)))))
        cases.append((f"{direction}-miss-pm1", dict(x=draw("pm1", (k, cols)), direction=direction,
                                                     miss=draw("pm1", (k, M)) if direction == "down" else draw("pm1", (k, M)))))
    if I != S:
        k = 2
        cases.append(("up-byind", dict(x=draw("normal", (k, I)), direction="up", by_individual=True)))
        cases.append(("down-byind", dict(x=draw("normal", (k, M)), direction="down", by_individual=True)))
        cases.append(("down-byind-vector", dict(x=draw("normal", (k, M)), direction="down", by_individual=True,
                                                init=rng.standard_normal(k))))
        cases.append(("up-byind-miss", dict(x=draw("normal", (k, I)), direction="up", by_individual=True, miss=np.zeros((k, M)))))
        cases.append(("down-byind-miss", dict(x=draw("normal", (k, M)), direction="down", by_individual=True,
                                              miss=draw("normal", (k, M)))))
        cases.append(("up-byind-emit", dict(x=draw("normal", (k, I)), direction="up", by_individual=True, emit_all_nodes=True)))
    return cases


def _run_reference(paths):
    from pygrgl_spmv.backends.reference import ReferencePlan, ReferencePlanPair, ReferenceRuntime, plan_reference_layout
    from pygrgl_spmv.grg import RuntimeRequirements

    sys.path.insert(0, str(REPO / "oracle"))
    from grg_oracle import OracleGRG

    req = RuntimeRequirements(max_k_up=8, max_k_down=8, need_down_miss_input=True, need_up_miss_output=True,
                              need_init_vector=True, need_init_matrix=True, need_init_xtx=True)
    pair = ReferencePlanPair(plan_up=ReferencePlan(store="N", fmt="CSR"), plan_down=ReferencePlan(store="T", fmt="CSC"))
    store: dict[str, np.ndarray] = {}
    index: list[dict] = []
    for art_idx, (name, path) in enumerate(sorted(paths.items())):
        for dtype in (np.float64, np.float32):
            layout = plan_reference_layout(artifacts=[path], pair=pair, dtype=dtype, requirements=req)
            oracle = OracleGRG(path, dtype=dtype)
            rng = np.random.default_rng(1000 + art_idx)
            with ReferenceRuntime(layout) as runtime:
                (grg,) = runtime.grgs
                for case_id, kw in _cases_for(name, grg, rng):
                    if dtype == np.float32 and not case_id.startswith(("up-k", "down-k", "up-emit", "down-emit", "down-miss")):
                        continue
                    kw = dict(kw)
                    x = np.asarray(kw.pop("x"), dtype=dtype)
                    init = kw.pop("init", None)
                    if isinstance(init, np.ndarray):
                        init = init.astype(dtype)
                    miss = kw.pop("miss", None)
                    miss_ref = None if miss is None else np.asarray(miss, dtype=dtype).copy()
                    miss_orc = None if miss is None else np.asarray(miss, dtype=dtype).copy()
                    out = grg.matmul(x, kw["direction"], emit_all_nodes=kw.get("emit_all_nodes", False),
                                     by_individual=kw.get("by_individual", False), init=init, miss=miss_ref)
                    mine = oracle.matmul(x, kw["direction"], emit_all_nodes=kw.get("emit_all_nodes", False),
                                         by_individual=kw.get("by_individual", False), init=init, miss=miss_orc)
                    assert mine.dtype == out.dtype and np.array_equal(mine, out), (name, case_id, dtype)
                    if miss is not None:
                        assert np.array_equal(miss_ref, miss_orc), (name, case_id, "miss")
                    key = f"{name}|{np.dtype(dtype).name}|{case_id}"
                    store[f"{key}|x"] = x
                    store[f"{key}|out"] = np.ascontiguousarray(out)
                    if isinstance(init, np.ndarray):
                        store[f"{key}|init"] = init
                    if miss is not None:
                        store[f"{key}|miss_in"] = np.asarray(miss, dtype=dtype)
                        store[f"{key}|miss_out"] = miss_ref
                    index.append(dict(key=key, artifact=name, dtype=np.dtype(dtype).name, case=case_id,
                                      direction=kw["direction"], emit_all_nodes=bool(kw.get("emit_all_nodes", False)),
                                      by_individual=bool(kw.get("by_individual", False)),
                                      init=("xtx" if isinstance(init, str) else None if init is None else ("vector" if init.ndim == 1 else "matrix")),
                                      miss=miss is not None))
    return store, index


def main(argv) -> None:
    if len(argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    reference_root = Path(argv[1])
    _setup(reference_root)
    paths = _write_artifacts(HERE)
    store, index = _run_reference(paths)
    np.savez_compressed(HERE / "cases.npz", **store)
    (HERE / "cases_index.json").write_text(json.dumps(index, indent=0))
    print(f"wrote {len(index)} golden cases for {len(paths)} artifacts")


if __name__ == "__main__":
    main(sys.argv)
