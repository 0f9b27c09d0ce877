"""``B200Runtime``: the runtime-owned execution arena of the B200 backend.

Mirrors ``TritonRuntime`` (``pygrgl_spmv/backends/triton/backend.py:609-1225``) as seen by
``BoundGRG`` and by user code:

* ``B200Runtime(layout)`` is a context manager; every device buffer is allocated in
  ``__enter__`` and released in ``__exit__``; a failed ``__enter__`` releases everything
  (``:690-762``); ``.grgs`` raises before entry (``:645-649``).
* ``grg.prepare_matmul_cuda(...)`` returns a prepared op whose ``input``/``output`` are
  transposed views of the shared ``io0`` buffer (so an up op's output aliases a down op's
  input, ``:564-593``), ``miss_input``/``miss_output``/``init_vector``/``init_matrix`` are
  views of ``io1``, and all-node output lives in ``aux``.
* A call runs asynchronously on the layout's caller stream, ordered after earlier work on
  that stream; it allocates nothing and never synchronises the host, so it can be captured
  in a CUDA graph.  Concurrent calls on one runtime fail fast (``:773-783``).
* Each prepared op records its traversal as a CUDA graph when it is prepared (unless the
  caller's stream is capturing) and replays it on every call: one graph launch instead of one
  kernel launch per level.

The whole prepared call is one C-ABI call, ``grg_b200_traverse`` (``include/grg_b200.h``):
seed, one fused gather pass per level, output stage.  There is no CPU or PyTorch fallback.
"""

from __future__ import annotations

import ctypes
from contextlib import contextmanager
from dataclasses import dataclass, field
import os

import numpy as np

from grg_spmv_b200.artifact import iter_artifact_blocks, load_grg_spmv_header
from grg_spmv_b200.backends.b200 import _native as nat
from grg_spmv_b200.backends.b200.plan import B200Layout, side_io_rows
from grg_spmv_b200.backends.b200.structures import build_down_levels, build_up_levels, load_blocks
from grg_spmv_b200.grg import BoundGRG, CudaMatmulSpec
from grg_spmv_b200.types import Direction, InitMode

_INIT_CODE = {InitMode.NONE: nat.INIT_NONE, InitMode.VECTOR: nat.INIT_VECTOR, InitMode.XTX: nat.INIT_XTX,
              InitMode.MATRIX: nat.INIT_MATRIX}


def _ptr(tensor) -> int | None:
    return None if tensor is None else int(tensor.data_ptr())


@dataclass
class _DeviceLevels:
    """The gather lists of one direction of one artifact, ready for ``grg_b200_traverse``."""

    array: ctypes.Array
    keepalive: list = field(default_factory=list)

    @property
    def count(self) -> int:
        return len(self.array)


@dataclass
class _DeviceArtifact:
    path: object
    state: object
    node_perm: object
    inv_node_perm: object
    sample_to_individual: object
    ind_ptr: object
    ind_samples: object
    xtx_node: object
    bias: dict
    sel_mut_ptr: object
    sel_mut_idx: object
    sel_miss_ptr: object
    sel_miss_idx: object
    levels: dict  # Direction -> _DeviceLevels
    level0_rows: int


class B200PreparedMatmul:
    def __init__(self, runtime: "B200Runtime", artifact: _DeviceArtifact, spec: CudaMatmulSpec) -> None:
        self._runtime = runtime
        self._artifact = artifact
        self._spec = spec
        st = artifact.state
        k = int(spec.k)
        self._input_internal = runtime._io0[: spec.input_cols, :k]
        self.input = self._input_internal.T
        if spec.emit_all_nodes:
            self._output_internal = runtime._aux[: st.num_nodes, :k]
        else:
            self._output_internal = runtime._io0[: spec.output_cols, :k]
        self.output = self._output_internal.T
        miss_view = None
        if spec.use_miss:
            miss_view = runtime._io1[: st.num_mutations, :k]
            if spec.direction == Direction.DOWN:
                self._miss_input_internal = miss_view
                self.miss_input = miss_view.T
            else:
                self._miss_output_internal = miss_view
                self.miss_output = miss_view.T
        init_vector = init_matrix = None
        if spec.init_mode == InitMode.VECTOR:
            init_vector = runtime._io1[0, :k]
            self._init_vector_internal = init_vector
            self.init_vector = init_vector
        if spec.init_mode == InitMode.MATRIX:
            init_matrix = runtime._io1[: st.num_nodes, :k]
            self._init_matrix_internal = init_matrix
            self.init_matrix = init_matrix.T
        self._args = runtime._traverse_args(artifact, spec, self._input_internal, self._output_internal, miss_view,
                                            init_vector, init_matrix)
        self._graph = runtime._capture(self._args)

    def __enter__(self) -> "B200PreparedMatmul":
        return self

    def __exit__(self, exc_type, exc, tb) -> None:
        return None

    def __call__(self) -> None:
        with self._runtime._call_scope():
            self._call_prelocked()

    def _call_prelocked(self) -> None:
        self._runtime._launch(self._args, self._graph)


GPU_LIST_BUILD_MIN_EDGES = 1 << 21  # graphs at least this large build their level lists on the GPU


class B200Runtime:
    """Runtime-owned B200 execution with resident or streamed level gather lists."""

    _bound_grg_cls = BoundGRG

    def __init__(self, layout: B200Layout, *, check_bounds: bool | None = None, use_graphs: bool | None = None) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("B200 runtime requires CUDA")
        self._lib = nat.load_library()
        self.layout = layout
        self.device = torch.device("cuda", int(layout.device))
        self.stream_ptr = int(layout.stream_ptr)
        self.stream = None
        self._stream_owner = layout.stream_owner
        if check_bounds is None:
            check_bounds = os.environ.get("GRG_B200_CHECK_BOUNDS", "0") not in ("", "0")
        self._check_bounds = bool(check_bounds)
        if use_graphs is None:
            use_graphs = os.environ.get("GRG_B200_GRAPHS", "1") not in ("", "0")
        self._use_graphs = bool(use_graphs)
        self._reset_owned_state()

    # -- lifecycle ----------------------------------------------------------------------------
    def _reset_owned_state(self) -> None:
        self._caller_stream = None
        self.stream = None
        self._state = None
        self._mix_scratch = None
        self._io0 = None
        self._io1 = None
        self._aux = None
        self._error_word = None
        self._df_sync = None
        self._slots = []
        self._slot_ptrs = None
        self._slot_bytes = None
        self._ring = None
        self._artifacts = ()
        self._grgs = ()
        self._variant = {}
        self._heavy_variant = {}
        self._entered = False
        self._active_call = False

    @property
    def grgs(self):
        if not self._entered:
            raise RuntimeError("B200Runtime must be entered before accessing grgs")
        return self._grgs

    def _arena_max_k(self) -> int:
        req = self.layout.requirements
        ks = []
        if self.layout.pair.plan_up is not None:
            ks.append(int(req.max_k_up))
        if self.layout.pair.plan_down is not None:
            ks.append(int(req.max_k_down))
        return max(ks)

    def _torch_dtype(self):
        import torch

        return torch.float64 if self.layout.dtype == np.float64 else torch.float32

    def __enter__(self) -> "B200Runtime":
        import torch

        try:
            lay = self.layout
            max_k = self._arena_max_k()
            tdt = self._torch_dtype()
            with torch.cuda.device(self.device):
                self._caller_stream = torch.cuda.get_stream_from_external(self.stream_ptr, device=self.device)
                self.stream = self._caller_stream
                if lay.precision == "mixed":  # float hi plane + int16 lo plane (grg_b200.h GRG_B200_MIXED)
                    self._state = torch.zeros(nat.mix_bytes(lay.max_num_nodes, nat.mix_ld(max_k)), device=self.device,
                                              dtype=torch.uint8)
                    if lay.mix_scratch_bytes:
                        self._mix_scratch = torch.zeros(lay.mix_scratch_bytes, device=self.device, dtype=torch.uint8)
                else:
                    self._state = torch.zeros(lay.max_num_nodes * max_k, device=self.device, dtype=tdt)
                self._io0 = torch.zeros((max(lay.max_num_samples, lay.max_num_mutations), max_k), device=self.device, dtype=tdt)
                io1_rows = side_io_rows(lay.pair, lay.requirements, max_num_mutations=lay.max_num_mutations,
                                        max_num_nodes=lay.max_num_nodes)
                self._io1 = None if io1_rows == 0 else torch.zeros((io1_rows, max_k), device=self.device, dtype=tdt)
                if lay.emit_all_nodes:
                    self._aux = torch.zeros((lay.max_num_nodes, max_k), device=self.device, dtype=tdt)
                self._error_word = torch.zeros(64, device=self.device, dtype=torch.int32)
                self._df_sync = torch.zeros(4, device=self.device, dtype=torch.int32)  # dataflow task counter/flags
                self._slots = [torch.empty(int(n), device=self.device, dtype=torch.uint8) for n in lay.slot_bytes]
                if self._slots:
                    self._slot_ptrs = (ctypes.c_void_p * len(self._slots))(*[s.data_ptr() for s in self._slots])
                    self._slot_bytes = (ctypes.c_int64 * len(self._slots))(*[int(s.numel()) for s in self._slots])
                    ring = ctypes.c_void_p()
                    nat.check(self._lib, self._lib.grg_b200_ring_create(int(lay.device), len(self._slots), ctypes.byref(ring)),
                              "grg_b200_ring_create")
                    self._ring = ring
                self._artifacts = tuple(self._build_artifact(art) for art in lay.artifacts)
            self._grgs = tuple(self._bound_grg_cls(self, idx, art.state, art.path, lay.device) for idx, art in enumerate(self._artifacts))
            for direction in (Direction.UP, Direction.DOWN):
                plan = lay.pair.plan_for(direction)
                if plan is not None and plan.autotune and lay.precision == "plain":
                    self._variant[direction], self._heavy_variant[direction] = self._tune_direction(direction)
            self._entered = True
            return self
        except Exception:
            self._release()
            raise

    def __exit__(self, exc_type, exc, tb) -> None:
        self._release()

    def _release(self) -> None:
        if self._caller_stream is not None:
            self._caller_stream.synchronize()
        if self._ring is not None:
            self._lib.grg_b200_ring_destroy(self._ring)
        self._reset_owned_state()

    # -- artifact upload ----------------------------------------------------------------------
    def _build_artifact(self, art) -> _DeviceArtifact:
        import torch

        lay = self.layout
        req = lay.requirements
        dev = self.device
        st = load_grg_spmv_header(art.path, lay.dtype)
        tdt = self._torch_dtype()

        def i32(values):
            arr = np.asarray(values, dtype=np.int64).astype(np.int32)
            if arr.size == 0:  # keep a valid device address for empty index arrays
                arr = np.zeros(1, dtype=np.int32)
            return torch.from_numpy(np.ascontiguousarray(arr)).to(dev)

        def flt(values):
            return torch.from_numpy(np.ascontiguousarray(np.asarray(values, dtype=lay.dtype))).to(dev)

        up_on, down_on = lay.pair.plan_up is not None, lay.pair.plan_down is not None
        s2i = np.asarray(st.sample_to_individual, dtype=np.int64)
        order = np.argsort(s2i, kind="stable")
        ind_ptr = np.zeros(st.num_individuals + 1, dtype=np.int64)
        np.cumsum(np.bincount(s2i, minlength=st.num_individuals)[: st.num_individuals], out=ind_ptr[1:])
        bias = {}
        if req.need_init_vector:
            if up_on:
                bias[("vector", Direction.UP)] = flt(st.init_vector_up_bias)
            if down_on:
                bias[("vector", Direction.DOWN)] = flt(st.init_vector_down_bias)
        if req.need_init_xtx and st.init_xtx_up_bias is not None:
            if up_on:
                bias[("xtx", Direction.UP)] = flt(st.init_xtx_up_bias)
            if down_on:
                bias[("xtx", Direction.DOWN)] = flt(st.init_xtx_down_bias)
        xtx_node = None
        if req.need_init_xtx and st.coalescence_counts is not None:
            xtx_node = flt(2.0 * np.asarray(st.coalescence_counts, dtype=lay.dtype))
        coo = load_blocks(iter_artifact_blocks(art.path))
        levels = {}
        off = np.asarray(st.level_offsets, dtype=np.int64)
        # Large graphs build their lists with PyTorch on the GPU (thousands of small launches,
        # seconds saved at millions of edges); small ones with the NumPy builder, which gives
        # identical lists and leaves the device to the traversal kernels.
        list_device = self.device if int(art.scan.num_edges) >= GPU_LIST_BUILD_MIN_EDGES else None
        if up_on:
            plan = lay.pair.plan_up
            built = {lv.level: lv for lv in build_up_levels(off, coo, plan.heavy_threshold, plan.locality(Direction.UP), plan.balance,
                                                            plan.pad_lists, plan.long_first, plan.slots, device=list_device,
                                                            heavy_buckets=plan.heavy_buckets)}
            levels[Direction.UP] = self._upload_levels(art.levels_up, built, plan.short_rows)
        if down_on:
            sel_miss = (st.sel_miss.indptr, st.sel_miss.indices, st.num_mutations) if req.need_down_miss_input else None
            plan = lay.pair.plan_down
            built = {lv.level: lv for lv in build_down_levels(
                off, coo, (st.sel_mut.indptr, st.sel_mut.indices, st.num_mutations), sel_miss, plan.heavy_threshold,
                plan.locality(Direction.DOWN), plan.balance, plan.pad_lists, plan.long_first, plan.slots, device=list_device,
                heavy_buckets=plan.heavy_buckets)}
            levels[Direction.DOWN] = self._upload_levels(art.levels_down, built, plan.short_rows)
        del coo
        return _DeviceArtifact(
            path=art.path,
            state=st,
            node_perm=i32(st.node_perm),
            inv_node_perm=i32(st.inv_node_perm),
            sample_to_individual=i32(s2i),
            ind_ptr=i32(ind_ptr),
            ind_samples=i32(order),
            xtx_node=xtx_node,
            bias=bias,
            sel_mut_ptr=i32(st.sel_mut.indptr) if up_on else None,
            sel_mut_idx=i32(st.sel_mut.indices) if up_on else None,
            sel_miss_ptr=i32(st.sel_miss.indptr) if up_on and req.need_up_miss_output else None,
            sel_miss_idx=i32(st.sel_miss.indices) if up_on and req.need_up_miss_output else None,
            levels=levels,
            level0_rows=int(off[1]) if off.size > 1 else 0,
        )

    def _upload_levels(self, plans, built, short_rows: bool = True) -> _DeviceLevels:
        import torch

        arr = (nat.Level * len(plans))()
        keep = []
        for i, lp in enumerate(plans):
            lv = built[lp.level]
            off_ptr, off_heavy, off_ids, off_entries, nbytes = lv.layout()
            if nbytes > lp.nbytes:
                raise RuntimeError(f"level {lp.level} needs {nbytes} bytes, more than the {lp.nbytes} planned")
            blob = torch.from_numpy(lv.pack())
            if lp.resident:
                blob = blob.to(self.device)
                slot = -1
            else:
                blob = blob.pin_memory()
                slot = int(lp.slot)
            keep.append(blob)
            arr[i] = nat.Level(row_begin=lv.row_begin, num_rows=lv.num_rows, num_entries=lv.num_entries,
                               num_heavy=int(lv.heavy_rows.size), heavy_threshold=lv.heavy_threshold, ring_slot=slot,
                               blob=blob.data_ptr(), blob_bytes=nbytes, off_row_ptr=off_ptr, off_heavy=off_heavy,
                               off_row_ids=off_ids, off_entries=off_entries, list_align=lv.list_align,
                               short_rows=lv.short_rows() if short_rows else 0)
            if lv.slots is not None:
                arr[i].num_slot_buckets = int(lv.slots.shape[0])
                for b, (pos, entry, width) in enumerate(lv.slots):
                    arr[i].slot_pos[b], arr[i].slot_entry[b], arr[i].slot_width[b] = int(pos), int(entry), int(width)
        return _DeviceLevels(array=arr, keepalive=keep)

    # -- autotuning ------------------------------------------------------------------------------
    TUNE_VARIANTS = (5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 0, 1, 4)

    def _tune_direction(self, direction: Direction) -> tuple[int, int]:
        """Fastest (narrow variant, heavy variant) for ``direction`` on the first artifact at
        the declared max k (the counterpart of ``TritonRuntime._tune_direction``,
        ``pygrgl_spmv/backends/triton/backend.py:1062-1079``): narrow variants first, then the
        two heavy-row kernels with the chosen narrow variant.  Each candidate runs once to warm
        up and is then timed over three traversals with CUDA events."""
        import torch

        from grg_spmv_b200.grg import CudaMatmulSpec

        art = self._artifacts[0]
        st = art.state
        k = int(self.layout.requirements.max_k_up if direction == Direction.UP else self.layout.requirements.max_k_down)
        cols_in = st.num_samples if direction == Direction.UP else st.num_mutations
        cols_out = st.num_mutations if direction == Direction.UP else st.num_samples
        spec = CudaMatmulSpec(direction=direction, k=k, emit_all_nodes=False, by_individual=False, init_mode=InitMode.NONE,
                              backend_init_mode=InitMode.NONE, use_miss=False, input_cols=cols_in, output_cols=cols_out,
                              apply_endpoint_bias=False)
        args = self._traverse_args(art, spec, self._io0[:cols_in, :k], self._io0[:cols_out, :k], None, None, None)
        plan = self.layout.pair.plan_for(direction)

        def timed() -> float:
            self._launch(args)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(3):
                self._launch(args)
            end.record()
            end.synchronize()
            return start.elapsed_time(end)

        with torch.cuda.device(self.device), torch.cuda.stream(self._caller_stream):
            narrow_ms = {}
            for variant in self.TUNE_VARIANTS:
                if variant >= 6 and not plan.pad_lists:
                    continue
                args.narrow_variant = variant
                narrow_ms[variant] = timed()
            args.narrow_variant = min(narrow_ms, key=narrow_ms.get)
            heavy_ms = {}
            for heavy in (0, 1, 2):
                args.heavy_variant = heavy
                heavy_ms[heavy] = timed()
        return int(args.narrow_variant), int(min(heavy_ms, key=heavy_ms.get))

    # -- calls ----------------------------------------------------------------------------------
    def _torch_caller_stream(self):
        return self._caller_stream

    @contextmanager
    def _call_scope(self):
        if not self._entered:
            raise RuntimeError("B200Runtime must be entered before matmul")
        if self._active_call:
            raise RuntimeError("concurrent runtime.grgs calls are not supported")
        self._active_call = True
        try:
            yield
        finally:
            self._active_call = False

    def _prepare_matmul_cuda(self, grg, spec) -> B200PreparedMatmul:
        if spec.direction == Direction.UP and self.layout.pair.plan_up is None:
            raise ValueError("UP plan is not configured")
        if spec.direction == Direction.DOWN and self.layout.pair.plan_down is None:
            raise ValueError("DOWN plan is not configured")
        if spec.emit_all_nodes and not self.layout.emit_all_nodes:
            raise ValueError("emit_all_nodes needs a layout planned with emit_all_nodes=True")
        return B200PreparedMatmul(self, self._artifacts[int(grg._artifact_index)], spec)

    def _traverse_args(self, art: _DeviceArtifact, spec, input_view, output_view, miss_view, init_vector, init_matrix, *,
                       state=None, mixed: bool | None = None, mix_scratch=None, df_sync=None):
        st = art.state
        k = int(spec.k)
        direction = Direction(spec.direction)
        plan = self.layout.pair.plan_for(direction)
        levels = art.levels[direction]
        bias_mode = nat.BIAS_NONE
        bias = None
        if spec.apply_endpoint_bias:
            kind = "xtx" if spec.init_mode == InitMode.XTX else "vector"
            bias = art.bias.get((kind, direction))
            if bias is None:
                raise RuntimeError(f"missing B200 {direction.value} {kind} endpoint bias")
            bias_mode = nat.BIAS_XTX if kind == "xtx" else nat.BIAS_VECTOR
        backend_init = InitMode(spec.backend_init_mode)
        if backend_init == InitMode.XTX and art.xtx_node is None:
            raise ValueError("init_mode=xtx requires GRG coalescence counts")
        a = nat.TraverseArgs()
        mixed = self.layout.precision == "mixed" if mixed is None else bool(mixed)
        state = self._state if state is None else state
        mix_scratch = self._mix_scratch if mix_scratch is None else mix_scratch
        a.dtype = nat.MIXED if mixed else (nat.F64 if self.layout.dtype == np.float64 else nat.F32)
        a.direction = nat.UP if direction == Direction.UP else nat.DOWN
        a.init_mode = _INIT_CODE[backend_init]
        a.bias_mode = bias_mode
        a.emit_all_nodes = int(bool(spec.emit_all_nodes))
        a.by_individual = int(bool(spec.by_individual))
        a.use_miss = int(bool(spec.use_miss))
        a.exact_order = int(bool(plan.exact_order))
        a.k = k
        a.num_nodes = st.num_nodes
        a.num_samples = st.num_samples
        a.num_mutations = st.num_mutations
        a.num_individuals = st.num_individuals
        a.state = _ptr(state)
        a.ld_state = nat.mix_ld(k) if mixed else k
        if mixed and mix_scratch is not None:
            a.mix_scratch = _ptr(mix_scratch)
            a.mix_scratch_bytes = int(mix_scratch.numel())
        a.input = _ptr(input_view)
        a.ld_input = int(input_view.stride(0))
        a.output = _ptr(output_view)
        a.ld_output = int(output_view.stride(0))
        if miss_view is not None:
            a.miss = _ptr(miss_view)
            a.ld_miss = int(miss_view.stride(0))
        a.init_vector = _ptr(init_vector)
        if init_matrix is not None:
            a.init_matrix = _ptr(init_matrix)
            a.ld_init = int(init_matrix.stride(0))
        a.node_perm = _ptr(art.node_perm)
        a.inv_node_perm = _ptr(art.inv_node_perm)
        a.xtx_node = _ptr(art.xtx_node)
        a.endpoint_bias = _ptr(bias)
        a.sample_to_individual = _ptr(art.sample_to_individual)
        a.ind_ptr = _ptr(art.ind_ptr)
        a.ind_samples = _ptr(art.ind_samples)
        a.sel_mut_ptr = _ptr(art.sel_mut_ptr)
        a.sel_mut_idx = _ptr(art.sel_mut_idx)
        a.sel_miss_ptr = _ptr(art.sel_miss_ptr)
        a.sel_miss_idx = _ptr(art.sel_miss_idx)
        a.level0_rows = art.level0_rows if direction == Direction.UP else 0
        a.num_levels = levels.count
        a.levels = ctypes.cast(levels.array, ctypes.POINTER(nat.Level))
        if self._ring is not None:
            a.ring = self._ring
            a.slot_buffers = ctypes.cast(self._slot_ptrs, ctypes.POINTER(ctypes.c_void_p))
            a.slot_bytes = ctypes.cast(self._slot_bytes, ctypes.POINTER(ctypes.c_int64))
            a.num_slots = len(self._slots)
        a.error_word = _ptr(self._error_word) if self._check_bounds else None
        a.narrow_variant = int(self._variant.get(direction, plan.resolve_narrow_variant(k)))
        heavy = self._heavy_variant.get(direction, plan.heavy_variant)
        if heavy is None:  # as measured on B200: warps fused into the narrow launch (k = 1, 8, 32)
            heavy = 2 if a.narrow_variant >= 6 else (1 if k <= 16 else 0)
        a.heavy_variant = int(heavy)
        a.narrow_split = int(plan.narrow_split)
        a.persist_ctas = int(plan.persist_ctas)
        a.fuse_entries = int(plan.fuse_entries)
        a.launch_flags = nat.LAUNCH_PDL if plan.resolve_pdl(k) else 0
        a.schedule = nat.SCHEDULE_DATAFLOW if plan.schedule == "dataflow" else nat.SCHEDULE_LEVELS
        a.dataflow_sync = _ptr(self._df_sync if df_sync is None else df_sync)
        return a

    def _capturing(self) -> bool:
        import torch

        with torch.cuda.device(self.device), torch.cuda.stream(self._caller_stream):
            return bool(torch.cuda.is_current_stream_capturing())

    def _capture(self, args: nat.TraverseArgs):
        """Record one traversal as a CUDA graph (replayed by every later call: one launch
        instead of one per level).  Skipped when graphs are off or the caller's stream is
        itself being captured, in which case calls launch the kernels into that capture."""
        import torch

        if not self._use_graphs or self._capturing():
            return None
        with torch.cuda.device(self.device):
            graph = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream(device=self.device)
            with torch.cuda.stream(side):
                graph.capture_begin(capture_error_mode="thread_local")
                try:
                    status = self._lib.grg_b200_traverse(ctypes.byref(args), ctypes.c_void_p(side.cuda_stream))
                finally:
                    graph.capture_end()
        nat.check(self._lib, status, "grg_b200_traverse (graph capture)")
        return graph

    def _launch(self, args: nat.TraverseArgs, graph=None) -> None:
        import torch

        with torch.cuda.device(self.device):
            if graph is not None and not self._capturing():
                with torch.cuda.stream(self._caller_stream):
                    graph.replay()
                return
            status = self._lib.grg_b200_traverse(ctypes.byref(args), ctypes.c_void_p(self.stream_ptr))
        nat.check(self._lib, status, "grg_b200_traverse")

    def prepare_batch(self, items, *, precision: str | None = None, tile_k: int | None = None, autotune: bool = False):
        """Several (grg, direction, k) matmuls run together as one CUDA graph; see
        ``grg_spmv_b200.backends.b200.batch.B200BatchedMatmul``."""
        from .batch import B200BatchedMatmul

        if not self._entered:
            raise RuntimeError("B200Runtime must be entered before preparing a batch")
        return B200BatchedMatmul(self, items, precision=precision, tile_k=tile_k, autotune=autotune)

    def device_error(self) -> int:
        """Synchronise the caller stream and return the first device error code (0 = none): a
        failed bounds check, or a dataflow wait that timed out."""
        self._caller_stream.synchronize()
        return int(self._error_word[0].item()) or int(self._df_sync[2].item())


__all__ = ["B200PreparedMatmul", "B200Runtime"]
