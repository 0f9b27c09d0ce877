"""The runtime-bound GRG operator: requirements, the prepared-call spec and ``BoundGRG``.

These mirror the reference's public surface in ``pygrgl_spmv/grg/__init__.py`` so that
code written against ``TritonRuntime``/``CusparseRuntime`` runs unchanged on the B200
runtime:

* ``RuntimeRequirements`` (``:26-40``) and its fail-fast validation (``:63-84``);
* ``CudaMatmulSpec`` (the reference's ``_CudaMatmulSpec``, ``:43-54``) built by
  ``BoundGRG._prepare_cuda_spec`` (``:454-516``), which fixes input/output widths and moves
  vector/xtx init out of the traversal into an endpoint bias unless all nodes are emitted;
* ``BoundGRG.prepare_matmul_cuda`` (``:541-562``) and the eager ``matmul`` (``:564-734``),
  which on a CUDA runtime copies host inputs into the prepared op's device views, runs it
  and copies results back.

A runtime passes its own ``BoundGRG`` class; a runtime constructed with the reference's
``pygrgl_spmv.grg.BoundGRG`` works the same way, because only the hooks below are used:
``runtime.layout.requirements``, ``runtime.layout.dtype``, ``runtime._prepare_matmul_cuda``,
``runtime._call_scope`` and ``runtime._torch_caller_stream``.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

from grg_spmv_b200.types import Direction, InitMode, parse_direction, parse_init_mode


@dataclass(frozen=True)
class RuntimeRequirements:
    max_k_up: int
    max_k_down: int
    need_down_miss_input: bool
    need_up_miss_output: bool
    need_init_vector: bool
    need_init_matrix: bool
    need_init_xtx: bool

    def __post_init__(self) -> None:
        if int(self.max_k_up) < 1:
            raise ValueError(f"max_k_up must be >= 1, got {self.max_k_up}")
        if int(self.max_k_down) < 1:
            raise ValueError(f"max_k_down must be >= 1, got {self.max_k_down}")


@dataclass(frozen=True)
class CudaMatmulSpec:
    direction: Direction
    k: int
    emit_all_nodes: bool
    by_individual: bool
    init_mode: InitMode
    backend_init_mode: InitMode
    use_miss: bool
    input_cols: int
    output_cols: int
    apply_endpoint_bias: bool


def validate_runtime_requirements(requirements, *, direction: Direction, k: int, init_mode: InitMode, uses_miss: bool) -> None:
    if direction == Direction.UP and int(k) > int(requirements.max_k_up):
        raise ValueError(f"UP runtime k={k} exceeds declared max_k_up={requirements.max_k_up}")
    if direction == Direction.DOWN and int(k) > int(requirements.max_k_down):
        raise ValueError(f"DOWN runtime k={k} exceeds declared max_k_down={requirements.max_k_down}")
    if direction == Direction.UP and uses_miss and not requirements.need_up_miss_output:
        raise ValueError("UP miss output was not declared in RuntimeRequirements")
    if direction == Direction.DOWN and uses_miss and not requirements.need_down_miss_input:
        raise ValueError("DOWN miss input was not declared in RuntimeRequirements")
    if init_mode == InitMode.VECTOR and not requirements.need_init_vector:
        raise ValueError("init vector use was not declared in RuntimeRequirements")
    if init_mode == InitMode.MATRIX and not requirements.need_init_matrix:
        raise ValueError("init matrix use was not declared in RuntimeRequirements")
    if init_mode == InitMode.XTX and not requirements.need_init_xtx:
        raise ValueError("init='xtx' use was not declared in RuntimeRequirements")


@dataclass(frozen=True)
class Mutation:
    """Mutation record (``pygrgl.Mutation`` fields) decoded from the artifact's mutation table."""

    position: float
    allele: str
    ref_allele: str
    time: float


def _decode(data: np.ndarray, offsets: np.ndarray, idx: int) -> str:
    return bytes(np.asarray(data[int(offsets[idx]):int(offsets[idx + 1])], dtype=np.uint8)).decode("utf-8")


class BoundGRG:
    """One artifact bound to an entered runtime."""

    def __init__(self, runtime, artifact_index: int, state, artifact_path: Path, device_id: int | None = None):
        self._runtime = runtime
        self._artifact_index = int(artifact_index)
        self._state = state
        self._artifact_path = Path(artifact_path)
        self._dtype = np.dtype(runtime.layout.dtype)
        self._device_id = device_id

    # -- metadata -------------------------------------------------------------------------
    device = property(lambda self: self._device_id)
    artifact_path = property(lambda self: self._artifact_path)
    num_samples = property(lambda self: int(self._state.num_samples))
    num_individuals = property(lambda self: int(self._state.num_individuals))
    num_mutations = property(lambda self: int(self._state.num_mutations))
    ploidy = property(lambda self: int(self._state.ploidy))
    num_nodes = property(lambda self: int(self._state.num_nodes))
    num_edges = property(lambda self: int(self._state.num_edges))
    has_missing_data = property(lambda self: bool(self._state.has_missing_data))
    level_offsets = property(lambda self: self._state.level_offsets)
    node_perm = property(lambda self: self._state.node_perm)
    inv_node_perm = property(lambda self: self._state.inv_node_perm)
    sel_mut = property(lambda self: self._state.sel_mut)
    sel_miss = property(lambda self: self._state.sel_miss)
    sample_to_individual = property(lambda self: self._state.sample_to_individual)
    coalescence_counts = property(lambda self: self._state.coalescence_counts)
    init_vector_up_bias = property(lambda self: self._state.init_vector_up_bias)
    init_vector_down_bias = property(lambda self: self._state.init_vector_down_bias)
    init_xtx_up_bias = property(lambda self: self._state.init_xtx_up_bias)
    init_xtx_down_bias = property(lambda self: self._state.init_xtx_down_bias)

    @property
    def shape(self) -> tuple[int, int]:
        return (self.num_samples, self.num_mutations)

    def get_mutation_by_id(self, mutation_id: int) -> Mutation:
        idx = int(mutation_id)
        if idx < 0 or idx >= self.num_mutations:
            raise IndexError(f"mutation id out of range: {mutation_id}")
        st = self._state
        return Mutation(
            float(st.mutation_positions[idx]),
            _decode(st.mutation_alleles, st.mutation_allele_offsets, idx),
            _decode(st.mutation_ref_alleles, st.mutation_ref_allele_offsets, idx),
            float(st.mutation_times[idx]),
        )

    # -- spec -----------------------------------------------------------------------------
    def _prepare_cuda_spec(self, *, direction, k: int, emit_all_nodes: bool, by_individual: bool, init_mode, use_miss: bool) -> CudaMatmulSpec:
        direction = parse_direction(direction)
        init_mode = parse_init_mode(init_mode)
        k = int(k)
        if k < 1:
            raise ValueError(f"k must be >= 1, got {k}")
        if emit_all_nodes and use_miss:
            raise RuntimeError('the "use_miss" parameter cannot be mixed with "emit_all_nodes=True"')
        if init_mode != InitMode.NONE and use_miss:
            raise ValueError('the "use_miss" parameter cannot be mixed with a non-none init_mode')
        if init_mode == InitMode.XTX and self.coalescence_counts is None:
            raise ValueError(
                "init_mode='xtx' requires per-node coalescence counts in the GRG. "
                "This artifact was loaded without coalescence counts."
            )
        validate_runtime_requirements(self._runtime.layout.requirements, direction=direction, k=k, init_mode=init_mode, uses_miss=bool(use_miss))
        if direction == Direction.UP:
            input_cols = self.num_individuals if by_individual else self.num_samples
        else:
            input_cols = self.num_mutations
        if emit_all_nodes:
            output_cols = self.num_nodes
        elif direction == Direction.UP:
            output_cols = self.num_mutations
        else:
            output_cols = self.num_individuals if by_individual else self.num_samples
        backend_init = init_mode if (emit_all_nodes or init_mode == InitMode.MATRIX) else InitMode.NONE
        return CudaMatmulSpec(
            direction=direction,
            k=k,
            emit_all_nodes=bool(emit_all_nodes),
            by_individual=bool(by_individual),
            init_mode=init_mode,
            backend_init_mode=backend_init,
            use_miss=bool(use_miss),
            input_cols=int(input_cols),
            output_cols=int(output_cols),
            apply_endpoint_bias=bool((not emit_all_nodes) and init_mode in (InitMode.VECTOR, InitMode.XTX)),
        )

    def prepare_matmul_cuda(self, *, direction, k: int, emit_all_nodes: bool = False, by_individual: bool = False,
                            init_mode="none", use_miss: bool = False):
        prepare = getattr(self._runtime, "_prepare_matmul_cuda", None)
        if prepare is None:
            raise NotImplementedError("prepare_matmul_cuda() is implemented only for CUDA backends")
        spec = self._prepare_cuda_spec(direction=direction, k=int(k), emit_all_nodes=bool(emit_all_nodes),
                                       by_individual=bool(by_individual), init_mode=init_mode, use_miss=bool(use_miss))
        return prepare(self, spec)

    # -- eager host API ---------------------------------------------------------------------
    def _parse_init(self, init, rows: int, input_dtype: np.dtype):
        if init is None:
            return InitMode.NONE, None
        if isinstance(init, str):
            if init != "xtx":
                raise ValueError(f"unexpected init value: {init}")
            if self.coalescence_counts is None:
                raise ValueError(
                    "init='xtx' requires per-node coalescence counts in the GRG. "
                    "This artifact was loaded without coalescence counts."
                )
            return InitMode.XTX, None
        if not isinstance(init, np.ndarray):
            raise TypeError(f"init must be None, 'xtx', or a numpy.ndarray, got {type(init).__name__}")
        if init.dtype != input_dtype:
            raise TypeError(f"the init matrix must match the dtype of the input matrix. Got: {init.dtype}")
        if init.ndim == 1:
            if init.shape[0] != rows:
                raise ValueError("if init has a single dimension, it must match the number of rows in the input matrix")
            return InitMode.VECTOR, init.astype(self._dtype, order="C", copy=False)
        if init.ndim == 2:
            if init.shape != (rows, self.num_nodes):
                raise ValueError(f"if init is a matrix, it must match the dimensions ({rows}, {self.num_nodes})")
            return InitMode.MATRIX, init.astype(self._dtype, order="C", copy=False)
        raise ValueError("init must be None, 'xtx', a vector, or a matrix")

    def _validate_miss(self, miss, rows: int, direction: Direction, input_dtype: np.dtype) -> np.ndarray:
        if not isinstance(miss, np.ndarray):
            raise TypeError(f'the "miss" input must be a numpy.ndarray. Got: {type(miss).__name__}')
        if miss.dtype != input_dtype:
            raise TypeError(f'the "miss" input must match the dtype of the input matrix. Got: {miss.dtype}')
        if miss.ndim != 2:
            raise ValueError(f'"miss" must be a two-dimension numpy array (matrix). ndim={miss.ndim}')
        if miss.shape[0] != rows:
            raise ValueError(f'"miss" has {miss.shape[0]} rows, but must match the input/output matrices ({rows})')
        if miss.shape[1] != self.num_mutations:
            if direction == Direction.DOWN:
                raise ValueError(f'the "miss" matrix must match the number of columns in the input matrix. Got: {miss.shape[1]}')
            raise ValueError(f'the "miss" matrix must match the number of columns in the output matrix. Got: {miss.shape[1]}')
        return miss

    def _copy_host_to_cuda(self, dst, src: np.ndarray) -> None:
        import torch

        host = torch.from_numpy(np.ascontiguousarray(np.asarray(src, dtype=self._dtype)))
        stream = getattr(self._runtime, "_torch_caller_stream", None)
        if stream is None:
            dst.copy_(host)
            return
        with torch.cuda.device(dst.device), torch.cuda.stream(stream()):
            dst.copy_(host)

    def _copy_cuda_to_host(self, src) -> np.ndarray:
        import torch

        stream = getattr(self._runtime, "_torch_caller_stream", None)
        if stream is None:
            return src.detach().cpu().numpy().astype(self._dtype, copy=False).copy()
        with torch.cuda.device(src.device), torch.cuda.stream(stream()):
            host = src.detach().cpu()
        return host.numpy().astype(self._dtype, copy=False).copy()

    def matmul(self, input, direction, emit_all_nodes: bool = False, by_individual: bool = False, init=None, miss=None):
        if not isinstance(input, np.ndarray):
            raise TypeError(f"matmul() requires input to be a numpy.ndarray, got {type(input).__name__}")
        if input.ndim != 2:
            raise ValueError("matmul() only supports two-dimensional numpy arrays as input.")
        rows, cols = input.shape
        if rows == 0 or cols == 0:
            raise ValueError("matmul() requires non-zero dimensions.")
        direction = parse_direction(direction)
        if direction == Direction.UP:
            expected = self.num_individuals if by_individual else self.num_samples
        else:
            expected = self.num_mutations
        if cols != expected:
            if direction == Direction.UP:
                raise ValueError("input matrix has wrong number of columns for UP direction (numSamples or numIndividuals depending on by_individual)")
            raise ValueError("input matrix has wrong number of columns for DOWN direction (numMutations)")
        if emit_all_nodes and miss is not None:
            raise RuntimeError('the "miss" parameter cannot be mixed with the "emit_all_nodes" parameter')
        if init is not None and miss is not None:
            raise ValueError('the "miss" parameter cannot be mixed with the "init" parameter')
        if getattr(self._runtime, "_prepare_matmul_cuda", None) is None:
            raise NotImplementedError("this BoundGRG only runs on CUDA runtimes")
        init_mode, init_payload = self._parse_init(init, rows, input.dtype)
        spec = self._prepare_cuda_spec(direction=direction, k=rows, emit_all_nodes=bool(emit_all_nodes),
                                       by_individual=bool(by_individual), init_mode=init_mode, use_miss=miss is not None)
        miss_matrix = None if miss is None else self._validate_miss(miss, rows, direction, input.dtype)
        with self._runtime._call_scope():
            with self.prepare_matmul_cuda(direction=spec.direction, k=spec.k, emit_all_nodes=spec.emit_all_nodes,
                                          by_individual=spec.by_individual, init_mode=spec.init_mode, use_miss=spec.use_miss) as op:
                self._copy_host_to_cuda(op.input, input)
                if spec.direction == Direction.DOWN and miss_matrix is not None:
                    self._copy_host_to_cuda(op.miss_input, miss_matrix)
                if init_mode == InitMode.VECTOR:
                    self._copy_host_to_cuda(op.init_vector, init_payload)
                elif init_mode == InitMode.MATRIX:
                    self._copy_host_to_cuda(op.init_matrix, init_payload)
                op._call_prelocked()
                result = self._copy_cuda_to_host(op.output)
                if spec.direction == Direction.UP and miss_matrix is not None:
                    miss_matrix += self._copy_cuda_to_host(op.miss_output).astype(miss_matrix.dtype, copy=False)
                return result


__all__ = ["BoundGRG", "CudaMatmulSpec", "Mutation", "RuntimeRequirements", "validate_runtime_requirements"]
