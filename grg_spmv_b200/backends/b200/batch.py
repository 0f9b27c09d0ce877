"""Batched GRG matmuls: many right-hand-side blocks over several GRGs in one CUDA graph.

The reference runs one prepared call per (GRG, direction, RHS block) and each call walks its
levels alone (``TritonRuntime._execute_prepared``, ``pygrgl_spmv/backends/triton/backend.py:
1221-1225``; callers loop over GRGs and blocks, e.g. ``scripts/bolt_lmm_inf/core.py:1173-1178``
and ``scripts/pca_bench/__main__.py:656-669``).  A level of a GRG traversal is a short,
latency-bound gather, so one such walk leaves most of a B200 idle.  A batch instead

* merges every block of the same (GRG, direction) into one traversal over the concatenated
  columns, so each gather list is read once for all of them;
* cuts that traversal into column tiles (``tile_k`` columns each, chosen by the autotuner
  or given), each with its own node state, and
* records all tiles of all GRGs as one CUDA graph with one stream per tile, so independent
  traversals overlap on the GPU; one replay runs the whole batch.

With ``precision="mixed"`` the tiles keep their node state in the 6-byte mixed form of
``grg_b200.h`` (FP32 value + 16-bit correction, FP64 sums); inputs and outputs stay FP64.

Every buffer of the batch is allocated when it is prepared and freed by ``close()``; calls
allocate nothing.  Levels must be resident (a streamed level would share the runtime's one
copy ring between concurrent traversals).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from grg_spmv_b200.grg import CudaMatmulSpec
from grg_spmv_b200.types import Direction, InitMode

from . import _native as nat


@dataclass(frozen=True)
class BatchItem:
    """One matmul of a batch: ``k`` right-hand sides of ``grg`` in ``direction``; ``use_miss``
    (down only) adds the miss rows of ``miss_input``."""

    grg: object
    direction: str
    k: int
    use_miss: bool = False


@dataclass
class _Tile:
    args: nat.TraverseArgs
    state: object
    scratch: object
    stream: object
    sync: object


@dataclass
class _Group:
    artifact_index: int
    direction: Direction
    use_miss: bool
    k_total: int
    io_in: object
    io_out: object
    miss_in: object
    tiles: list


class B200BatchedMatmul:
    """Prepared batch (context manager).  ``inputs[i]`` / ``outputs[i]`` / ``miss_inputs[i]``
    are the ``(k_i, cols)`` views of item i (like a prepared op's ``input``/``output``);
    ``batch()`` runs every item, asynchronously on the runtime's caller stream."""

    TILE_CANDIDATES = (None, 256, 128, 64, 32, 16)

    def __init__(self, runtime, items, *, precision: str | None = None, tile_k: int | None = None, autotune: bool = False):
        import torch

        self._runtime = runtime
        self._items = [it if isinstance(it, BatchItem) else BatchItem(*it) for it in items]
        if not self._items:
            raise ValueError("a batch needs at least one item")
        lay = runtime.layout
        self.precision = lay.precision if precision is None else precision
        if self.precision not in ("plain", "mixed"):
            raise ValueError(f"precision must be 'plain' or 'mixed', got {self.precision!r}")
        if self.precision == "mixed":
            if lay.dtype != np.float64:
                raise ValueError("a mixed-precision batch keeps FP64 inputs and outputs; the layout dtype must be float64")
            for plan in (lay.pair.plan_up, lay.pair.plan_down):
                if plan is not None and (plan.exact_order or not plan.pad_lists):
                    raise ValueError("a mixed-precision batch needs plans with pad_lists=True and exact_order=False")
        if tile_k is not None and (int(tile_k) < 1 or (self.precision == "mixed" and int(tile_k) % 4)):
            raise ValueError(f"tile_k must be >= 1 (and a multiple of 4 for mixed precision), got {tile_k}")
        self._tdt = torch.float64 if lay.dtype == np.float64 else torch.float32
        self._groups: list[_Group] = []
        self.inputs, self.outputs, self.miss_inputs = [], [], []
        self._build_groups()
        self.tile_k = tile_k
        self.tuned_ms = {}
        self._graph = None
        if autotune:
            self.tile_k = self._autotune()
        self._build_tiles(self.tile_k)

    # -- construction ----------------------------------------------------------------------------
    def _build_groups(self) -> None:
        import torch

        rt = self._runtime
        keyed: dict[tuple, list[int]] = {}
        for i, it in enumerate(self._items):
            direction = Direction(it.direction)
            if int(it.k) < 1:
                raise ValueError(f"batch item {i}: k must be >= 1")
            if it.use_miss and direction != Direction.DOWN:
                raise ValueError(f"batch item {i}: miss rows are supported for down only")
            if rt.layout.pair.plan_for(direction) is None:
                raise ValueError(f"{direction.value.upper()} plan is not configured")
            idx = int(it.grg._artifact_index)
            if any(lv.ring_slot >= 0 for lv in rt._artifacts[idx].levels[direction].array):
                raise ValueError("a batch needs every level of its GRGs resident (vram_budget_bytes too small)")
            keyed.setdefault((idx, direction, bool(it.use_miss)), []).append(i)
        self.inputs = [None] * len(self._items)
        self.outputs = [None] * len(self._items)
        self.miss_inputs = [None] * len(self._items)
        dev = rt.device
        for (idx, direction, use_miss), members in keyed.items():
            st = rt._artifacts[idx].state
            k_total = sum(int(self._items[i].k) for i in members)
            cols_in = st.num_samples if direction == Direction.UP else st.num_mutations
            cols_out = st.num_mutations if direction == Direction.UP else st.num_samples
            io_in = torch.zeros((cols_in, k_total), device=dev, dtype=self._tdt)
            io_out = torch.zeros((cols_out, k_total), device=dev, dtype=self._tdt)
            miss_in = torch.zeros((st.num_mutations, k_total), device=dev, dtype=self._tdt) if use_miss else None
            off = 0
            for i in members:
                k = int(self._items[i].k)
                self.inputs[i] = io_in[:, off:off + k].T
                self.outputs[i] = io_out[:, off:off + k].T
                if use_miss:
                    self.miss_inputs[i] = miss_in[:, off:off + k].T
                off += k
            self._groups.append(_Group(artifact_index=idx, direction=direction, use_miss=use_miss, k_total=k_total,
                                       io_in=io_in, io_out=io_out, miss_in=miss_in, tiles=[]))

    def _tile_widths(self, k_total: int, tile_k: int | None) -> list[int]:
        if tile_k is None or int(tile_k) >= k_total:
            return [k_total]
        w = int(tile_k)
        return [w] * (k_total // w) + ([k_total % w] if k_total % w else [])

    def _build_tiles(self, tile_k: int | None) -> None:
        import torch

        rt = self._runtime
        mixed = self.precision == "mixed"
        self._release_tiles()
        streams = []
        for g in self._groups:
            art = rt._artifacts[g.artifact_index]
            st = art.state
            c0 = 0
            for w in self._tile_widths(g.k_total, tile_k):
                if mixed:
                    state = torch.zeros(nat.mix_bytes(st.num_nodes, nat.mix_ld(w)), device=rt.device, dtype=torch.uint8)
                    scratch = None
                    if g.direction == Direction.DOWN:
                        nbytes = nat.mix_bytes(st.num_mutations, nat.mix_ld(w)) * (2 if g.use_miss else 1)
                        scratch = torch.zeros(nbytes, device=rt.device, dtype=torch.uint8)
                else:
                    state = torch.zeros(st.num_nodes * w, device=rt.device, dtype=self._tdt)
                    scratch = None
                spec = CudaMatmulSpec(direction=g.direction, k=w, emit_all_nodes=False, by_individual=False,
                                      init_mode=InitMode.NONE, backend_init_mode=InitMode.NONE, use_miss=g.use_miss,
                                      input_cols=g.io_in.shape[0], output_cols=g.io_out.shape[0], apply_endpoint_bias=False)
                miss_view = g.miss_in[:, c0:c0 + w] if g.use_miss else None
                sync = torch.zeros(4, device=rt.device, dtype=torch.int32)  # own dataflow counter per tile
                args = rt._traverse_args(art, spec, g.io_in[:, c0:c0 + w], g.io_out[:, c0:c0 + w], miss_view, None, None,
                                         state=state, mixed=mixed, mix_scratch=scratch, df_sync=sync)
                args.ring = None  # resident levels only (checked when the groups were built)
                stream = torch.cuda.Stream(device=rt.device)
                streams.append(stream)
                g.tiles.append(_Tile(args=args, state=state, scratch=scratch, stream=stream, sync=sync))
                c0 += w
        self._graph = self._capture() if rt._use_graphs else None

    def _release_tiles(self) -> None:
        self._graph = None
        for g in self._groups:
            g.tiles = []

    # -- execution -------------------------------------------------------------------------------
    def _enqueue(self, origin) -> None:
        """Fork every tile off ``origin`` (its own stream), run it, join back into ``origin``."""
        import torch

        rt = self._runtime
        fork = torch.cuda.Event()
        fork.record(origin)
        joins = []
        for g in self._groups:
            for t in g.tiles:
                t.stream.wait_event(fork)
                status = rt._lib.grg_b200_traverse(ctypes.byref(t.args), ctypes.c_void_p(t.stream.cuda_stream))
                nat.check(rt._lib, status, "grg_b200_traverse (batch)")
                done = torch.cuda.Event()
                done.record(t.stream)
                joins.append(done)
        for done in joins:
            origin.wait_event(done)

    def _capture(self):
        import torch

        rt = self._runtime
        if rt._capturing():
            return None
        with torch.cuda.device(rt.device):
            graph = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream(device=rt.device)
            side.wait_stream(torch.cuda.current_stream(rt.device))
            with torch.cuda.stream(side):
                graph.capture_begin(capture_error_mode="thread_local")
                try:
                    self._enqueue(side)
                finally:
                    graph.capture_end()
        return graph

    def __call__(self) -> None:
        import torch

        rt = self._runtime
        with rt._call_scope(), torch.cuda.device(rt.device):
            if self._graph is not None and not rt._capturing():
                with torch.cuda.stream(rt._caller_stream):
                    self._graph.replay()
            else:
                self._enqueue(rt._caller_stream)

    def _autotune(self) -> int | None:
        """Column tile width with the shortest batch (three timed replays each, after one warm-up)."""
        import torch

        rt = self._runtime
        k_max = max(g.k_total for g in self._groups)
        best, best_ms = None, None
        for cand in self.TILE_CANDIDATES:
            if cand is not None and cand >= k_max:
                continue
            self._build_tiles(cand)
            with torch.cuda.device(rt.device), torch.cuda.stream(rt._caller_stream):
                self()
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record()
                for _ in range(3):
                    self()
                end.record()
                end.synchronize()
            ms = start.elapsed_time(end) / 3
            self.tuned_ms[cand if cand is not None else "merged"] = ms
            if best_ms is None or ms < best_ms:
                best, best_ms = cand, ms
        return best

    @property
    def num_tiles(self) -> int:
        return sum(len(g.tiles) for g in self._groups)

    def edge_rhs(self) -> int:
        """Edge x right-hand-side products of one call (the batch's unit of work)."""
        rt = self._runtime
        return sum(int(rt._artifacts[g.artifact_index].state.num_edges) * g.k_total for g in self._groups)

    def close(self) -> None:
        self._release_tiles()
        self._groups = []
        self.inputs, self.outputs, self.miss_inputs = [], [], []

    def __enter__(self) -> "B200BatchedMatmul":
        return self

    def __exit__(self, exc_type, exc, tb) -> None:
        self.close()


__all__ = ["B200BatchedMatmul", "BatchItem"]
