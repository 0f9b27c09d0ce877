"""ORACLE — test infrastructure only; never imported by the product package.

A CPU restatement of the reference's FP64/FP32 GRG matmul path, used by ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg as the checker.  It follows
the reference step for step, with the same SciPy sparse products in the same order, so its
results equal ``ReferenceRuntime``'s bit for bit (pinned by ``tests/golden``):

* ``OracleGRG.run`` = ``ReferenceRuntime._run`` (``pygrgl_spmv/backends/reference.py:365-432``):
  zero the node state, add init (xtx: 2·coalescence count, vector, matrix), then
  - up: add the input into the sample rows; for every destination level ascending, add each
    source level's block product ``A[dst][src] @ v[src]`` in ascending ``src`` order
    (``:396-407``); output ``sel_mut @ v`` and optionally ``sel_miss @ v`` (``:410-414``);
  - down: add ``sel_mut.T @ x`` and optionally ``sel_miss.T @ miss`` (``:416-419``); for every
    destination level descending, add ``A[src][dst].T @ v[src]`` for ``src`` descending
    (``:420-429``; order from ``pygrgl_spmv/backends/base.py:106-119``); output the sample rows.
* ``OracleGRG.matmul`` = ``BoundGRG.matmul`` on a CPU runtime
  (``pygrgl_spmv/grg/__init__.py:636-734``): matrix init reordered by ``node_perm``
  (``:406-408``), vector/xtx init applied as an endpoint bias unless all nodes are emitted
  (``:645-653``, ``:427-444``), up miss output accumulated into the caller's array
  (``:692-693``), down ``by_individual`` summed with ``np.add.at`` (``:730-733``), all-node
  output returned in original node order (``:449-452``).

The artifact is read straight from the ``.grg_spmv`` archive (format v8 keys).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import scipy.sparse as sp


def _csr(indices, indptr, shape) -> sp.csr_matrix:
    idx = np.asarray(indices)
    return sp.csr_matrix((np.ones(idx.size, dtype=np.bool_), idx, np.asarray(indptr)), shape=tuple(int(v) for v in shape))


def _canonical_block(indices, indptr, shape) -> sp.csr_matrix:
    """Level blocks are canonicalised before use, as ``materialize_sparse_block`` does
    (``pygrgl_spmv/backends/base.py:128-139``): duplicate entries merge and columns are
    sorted within each row (hand-built artifacts may store unsorted rows)."""
    block = _csr(indices, indptr, shape)
    block.sum_duplicates()
    block.sort_indices()
    return block


class OracleGRG:
    def __init__(self, artifact_path, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        with np.load(Path(artifact_path), allow_pickle=False) as data:
            if int(np.asarray(data["grg_spmv_format_version"]).item()) != 8:
                raise ValueError("oracle reads .grg_spmv format version 8 only")
            self.num_samples = int(np.asarray(data["num_samples"]).item())
            self.num_mutations = int(np.asarray(data["num_mutations"]).item())
            self.num_nodes = int(np.asarray(data["num_nodes"]).item())
            self.num_individuals = int(np.asarray(data["num_individuals"]).item())
            self.num_edges = int(np.asarray(data["num_edges"]).item())
            self.level_offsets = np.asarray(data["level_offsets"], dtype=np.int64)
            self.node_perm = np.asarray(data["node_perm"])
            self.inv_node_perm = np.empty_like(self.node_perm)
            self.inv_node_perm[self.node_perm] = np.arange(self.node_perm.size, dtype=self.node_perm.dtype)
            self.sample_to_individual = np.asarray(data["sample_to_individual"])
            M, N = self.num_mutations, self.num_nodes
            self.sel_mut = _csr(data["sel_mut_indices"], data["sel_mut_indptr"], (M, N))
            self.sel_miss = _csr(data["sel_miss_indices"], data["sel_miss_indptr"], (M, N))
            self.coalescence_counts = np.asarray(data["coalescence_counts"], dtype=np.int64) if bool(np.asarray(data["has_individual_coals"]).item()) else None
            self.bias = {
                ("vector", "up"): np.asarray(data["init_vector_up_bias"], dtype=self.dtype),
                ("vector", "down"): np.asarray(data["init_vector_down_bias"], dtype=self.dtype),
            }
            if bool(np.asarray(data["has_xtx_bias"]).item()):
                self.bias[("xtx", "up")] = np.asarray(data["init_xtx_up_bias"], dtype=self.dtype)
                self.bias[("xtx", "down")] = np.asarray(data["init_xtx_down_bias"], dtype=self.dtype)
            h = self.level_offsets.size - 1
            self.height = h
            self.blocks: dict[tuple[int, int], sp.csr_matrix] = {}
            levels = np.asarray(data["scan_block_levels"]).reshape(-1, 2)
            shapes = np.asarray(data["scan_block_shapes"]).reshape(-1, 2)
            for (dst, src), shape in zip(levels, shapes):
                block = _canonical_block(data[f"A_blocks_{dst}_{src}_indices"], data[f"A_blocks_{dst}_{src}_indptr"], shape)
                if block.nnz:
                    self.blocks[(int(dst), int(src))] = block
        # Per-destination-level operation lists in execution order.
        self.up_ops = [[(src, self.blocks[(dst, src)]) for src in range(dst) if (dst, src) in self.blocks] for dst in range(h)]
        self.down_ops = [[(src, self.blocks[(src, dst)]) for src in range(h - 1, dst, -1) if (src, dst) in self.blocks] for dst in range(h)]

    def _levels(self, level: int) -> slice:
        return slice(int(self.level_offsets[level]), int(self.level_offsets[level + 1]))

    def run(self, direction: str, primary: np.ndarray, *, miss=None, init_mode="none", init_payload=None,
            need_miss_output=False, emit_all_nodes=False):
        """Node-major run: ``primary`` is ``[cols, k]``; returns node-major results."""
        x = np.asarray(primary, dtype=self.dtype, order="C")
        k = x.shape[1]
        v = np.zeros((self.num_nodes, k), dtype=self.dtype)
        if init_mode == "xtx":
            v += (2.0 * self.coalescence_counts.astype(self.dtype, copy=False))[:, None]
        elif init_mode == "vector":
            v += init_payload[None, :]
        elif init_mode == "matrix":
            v += init_payload
        if direction == "up":
            v[: self.num_samples] += x
            for dst in range(1, self.height):
                for src, block in self.up_ops[dst]:
                    v[self._levels(dst)] += block @ v[self._levels(src)]
            if emit_all_nodes:
                return v.copy()
            out = np.asarray(self.sel_mut @ v, dtype=self.dtype) if self.sel_mut.nnz else np.zeros((self.num_mutations, k), self.dtype)
            out_miss = None
            if need_miss_output:
                out_miss = np.asarray(self.sel_miss @ v, dtype=self.dtype) if self.sel_miss.nnz else np.zeros((self.num_mutations, k), self.dtype)
            return out, out_miss
        if self.sel_mut.nnz:
            v += self.sel_mut.T @ x
        if miss is not None and self.sel_miss.nnz:
            v += self.sel_miss.T @ np.asarray(miss, dtype=self.dtype, order="C")
        for dst in range(self.height - 2, -1, -1):
            for src, block in self.down_ops[dst]:
                v[self._levels(dst)] += block.T @ v[self._levels(src)]
        if emit_all_nodes:
            return v.copy()
        return v[: self.num_samples].copy()

    def matmul(self, x: np.ndarray, direction: str, *, emit_all_nodes=False, by_individual=False, init=None, miss=None):
        """``(k, cols)`` in, ``(k, out_cols)`` out, like ``BoundGRG.matmul``."""
        direction = str(direction).lower()
        rows = x.shape[0]
        init_mode, payload = "none", None
        if isinstance(init, str):
            init_mode = "xtx"
        elif isinstance(init, np.ndarray) and init.ndim == 1:
            init_mode, payload = "vector", init.astype(self.dtype, copy=False)
        elif isinstance(init, np.ndarray):
            init_mode, payload = "matrix", init[:, self.node_perm].T.astype(self.dtype, order="C", copy=False)
        if emit_all_nodes:
            backend_mode, backend_payload = init_mode, payload
        elif init_mode in ("vector", "xtx"):
            backend_mode, backend_payload = "none", None
        else:
            backend_mode, backend_payload = init_mode, payload
        xi = x.astype(self.dtype, order="C", copy=False).T
        if direction == "up":
            if by_individual:
                xi = xi[self.sample_to_individual]
            if emit_all_nodes:
                v = self.run("up", xi, init_mode=backend_mode, init_payload=backend_payload, emit_all_nodes=True)
                return np.asarray(v, dtype=self.dtype)[self.inv_node_perm].T
            res, res_miss = self.run("up", xi, init_mode=backend_mode, init_payload=backend_payload, need_miss_output=miss is not None)
            self._endpoint_bias(res, "up", init_mode, payload)
            if miss is not None:
                miss += res_miss.T.astype(miss.dtype, copy=False)
            return res.T
        if emit_all_nodes:
            v = self.run("down", xi, init_mode=backend_mode, init_payload=backend_payload, emit_all_nodes=True)
            return np.asarray(v, dtype=self.dtype)[self.inv_node_perm].T
        miss_internal = None if miss is None else miss.T.astype(self.dtype, order="C", copy=False)
        res = self.run("down", xi, miss=miss_internal, init_mode=backend_mode, init_payload=backend_payload)
        self._endpoint_bias(res, "down", init_mode, payload)
        if by_individual:
            agg = np.zeros((self.num_individuals, rows), dtype=self.dtype)
            np.add.at(agg, self.sample_to_individual, res)
            res = agg
        return res.T

    def _endpoint_bias(self, res: np.ndarray, direction: str, init_mode: str, payload) -> None:
        if init_mode == "xtx":
            res += self.bias[("xtx", direction)][:, None]
        elif init_mode == "vector":
            res += self.bias[("vector", direction)][:, None] * payload[None, :]


__all__ = ["OracleGRG"]
