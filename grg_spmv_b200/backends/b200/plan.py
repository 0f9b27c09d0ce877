"""Layout planner of the B200 backend: ``plan_b200_layout`` -> ``B200Layout``.

The call signature and the budget semantics follow ``plan_triton_layout``
(``pygrgl_spmv/backends/triton/backend.py:343-561``) so it is a drop-in:

* ``dtype`` float32/float64; ``ring_buffer_size >= 0``; ``vram_budget_bytes >= 0`` with 0
  meaning "whatever full residency needs" (``:355-366``, ``:442-445``);
* ``stream`` is an int handle or a ``__cuda_stream__`` object and must live on ``device``
  (``:365-371``);
* full residency when it fits; otherwise every sparse unit is streamed through the ring and
  units are promoted to resident greedily, largest first (``_promotion_key`` ``:276-278``),
  while the total stays within the budget (``:471-495``); ``allow_residency=False`` streams
  everything (``:446-460``); ``ValueError`` when even that does not fit; a
  ``RuntimeWarning`` when the allocated ring differs from the requested one (``:281-295``);
* the layout reports ``budget_items``, ``bytes_by_category``, ``bytes_total`` and
  ``required_budget_for_full_residency``.

The unit of residency/streaming is one destination level of one direction (the gather list
the kernels walk for that level, ``structures.py``), not one (dst, src) block: up and down
have separate atomic-free gather lists.  Byte counts are computed from the artifact scan
alone (metadata only, like the reference); heavy-row lists are budgeted at their upper bound.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path
from typing import Mapping
import warnings

import numpy as np

from grg_spmv_b200.artifact import ArtifactScan, scan_grg_spmv
from grg_spmv_b200.backends.b200 import _native as nat
from grg_spmv_b200.backends.b200.structures import blob_layout, down_entry_bound, up_entry_bound
from grg_spmv_b200.types import Direction

DEFAULT_HEAVY_THRESHOLD = 32
PDL_MIN_K = 8  # automatic programmatic dependent launch from this many right-hand sides


@dataclass(frozen=True)
class BudgetItem:
    kind: str
    name: str
    nbytes: int
    artifact_index: int | None = None
    dst_level: int | None = None
    src_level: int | None = None
    slot: int | None = None
    direction: str | None = None


@dataclass(frozen=True)
class B200Plan:
    """Per-direction options.

    ``exact_order``: heavy rows are also summed in list order, which makes every result
    bit-identical to the reference's ReferenceRuntime (default: heavy rows are split over a
    CTA and tree-reduced, deterministic and exact for integer-valued data).
    ``heavy_threshold``: rows with more entries than this go to the heavy-row kernel.
    ``row_order``: "natural" (node order) or "locality" (rows that share source rows are
    processed together); None picks the direction's default (up natural, down locality).
    ``narrow_variant``: shape of the narrow-row kernel (``GRG_B200_NARROW_VARIANTS``); None
    picks per call, as measured on B200: in the default mode the lean entry-parallel walk in
    4-warp CTAs, 15 (run as 12 where its shape does not apply: k not a power of two, or above 64 in FP64 and
    128 in FP32); in exact
    order 7 for k <= 16 and 6 above; with ``pad_lists=False``, 5.  Runtimes with bounds
    checking run 7 in place of 11-14.
    ``balance``: group narrow rows by length (power-of-two buckets) so a warp's rows finish
    together.
    ``autotune``: time the narrow-kernel variants, then the heavy-row kernels, when the runtime
    is entered and use the fastest for this direction (instead of ``narrow_variant`` and
    ``heavy_variant``).
    ``pad_lists``: pad every gather list to a multiple of 4 entries (needed by variant 6).
    ``heavy_variant``: heavy rows one CTA each (0), one warp each (1), or one warp each inside
    the narrow-row launch (2, with ``narrow_variant`` 6 or 7); None picks 2 with the padded
    variants and otherwise 1 for k <= 16, 0 above.  Exact order always uses CTAs.
    ``long_first``: with ``balance``, the longest length bucket is processed first.
    ``pdl``: launch the level, seed and output kernels with programmatic dependent launch
    (each overlaps the end of the previous one; ignored when levels are streamed).  None turns
    it on for k >= 8: measured on B200, +3% to +4.5% at k = 8, +1% at k = 32, -15% at k = 1.
    ``slots``: with ``balance`` and ``pad_lists``, pad each narrow row to its bucket's width
    (1, 2, 4, 8 quads of 4 entries) so kernels locate its list from its position instead of
    loading ``row_ptr`` (one dependent load fewer per row, up to twice the list bytes).
    ``narrow_split``: split each narrow row over 2^narrow_split lane groups (0..3; -1 chooses
    per level; default mode with ``narrow_variant`` 6 or 7 only).
    ``schedule``: "levels" (one launch per level) or "dataflow" (one persistent launch per
    traversal, rows wait only for their own sources; default mode, resident levels, padded
    lists, plain precision; other calls fall back to "levels").  Its readiness sentinel is one
    specific quiet NaN: an input holding exactly that NaN makes the wait time out (status
    ``GRG_B200_DEVICE_WAIT_TIMEOUT``, undefined result).
    ``persist_ctas``: with ``narrow_variant`` 9 or 10, the CTAs of a level launch's persistent
    narrow part (each walks row groups); 0 sizes it to what the GPU holds at once.
    ``heavy_buckets``: with ``balance``, also group the heavy rows (the suffix) into
    power-of-two length buckets.  Off by default: heavy rows then stay in row order (locality
    order for down), so rows that share source rows run together.  On config 2 at k = 8 this
    is what lets down level 0 read each parent row from DRAM about once.
    ``short_rows``: let narrow variants 13 and 14 walk each level's narrow suffix of lists of at
    most one quad (4 entries) with one entry slot, so a CTA covers twice the rows there.  On
    by default; most rows of the upper down levels are that short.
    ``fuse_entries``: > 0 runs each stretch of consecutive resident levels with at most this many
    gather entries (default mode, plain precision, padded variants) as one cooperative launch
    with a grid barrier between levels instead of one launch per level; results are
    bit-identical.  0 launches every level on its own.
    """

    exact_order: bool = False
    heavy_threshold: int = DEFAULT_HEAVY_THRESHOLD
    row_order: str | None = None
    narrow_variant: int | None = None
    balance: bool = True
    autotune: bool = False
    pad_lists: bool = True
    heavy_variant: int | None = None
    long_first: bool = True
    slots: bool = False
    pdl: bool | None = None
    narrow_split: int = -1
    schedule: str = "levels"
    persist_ctas: int = 0
    fuse_entries: int = 0
    heavy_buckets: bool = False
    short_rows: bool = True

    def __post_init__(self) -> None:
        if int(self.heavy_threshold) < 1:
            raise ValueError(f"heavy_threshold must be >= 1, got {self.heavy_threshold}")
        if self.row_order not in (None, "natural", "locality"):
            raise ValueError(f"row_order must be 'natural' or 'locality', got {self.row_order!r}")
        if self.narrow_variant is not None and not 0 <= int(self.narrow_variant) < nat.NARROW_VARIANTS:
            raise ValueError(f"narrow_variant must be in [0, {nat.NARROW_VARIANTS}), got {self.narrow_variant}")
        if self.narrow_variant is not None and int(self.narrow_variant) >= 6 and not self.pad_lists:
            raise ValueError(f"narrow_variants 6-{nat.NARROW_VARIANTS - 1} read padded gather lists; they need pad_lists=True")
        if self.heavy_variant is not None and int(self.heavy_variant) not in (0, 1, 2, 3):
            raise ValueError(f"heavy_variant must be 0, 1, 2 or 3, got {self.heavy_variant}")
        if not -1 <= int(self.narrow_split) <= 3:
            raise ValueError(f"narrow_split must be in [-1, 3], got {self.narrow_split}")
        if self.schedule not in ("levels", "dataflow"):
            raise ValueError(f"schedule must be 'levels' or 'dataflow', got {self.schedule!r}")
        if int(self.persist_ctas) < 0:
            raise ValueError(f"persist_ctas must be >= 0, got {self.persist_ctas}")
        if int(self.fuse_entries) < 0:
            raise ValueError(f"fuse_entries must be >= 0, got {self.fuse_entries}")

    def resolve_narrow_variant(self, k: int) -> int:
        """The narrow-row kernel variant used for a call with ``k`` right-hand sides."""
        if self.narrow_variant is not None:
            return int(self.narrow_variant)
        if not self.pad_lists:
            return 5
        if self.exact_order:
            return 7 if int(k) <= 16 else 6
        # the lean walks, measured on B200 (config 2): one partial sum per row (12) +17% over 7
        # at k = 8 and +14% over 6 at k = 32; entry-parallel rows (13, else as 12) a further +2%
        # at k = 8 and +3% at k = 16 and 32, but -2% at k = 4; their codes loaded before the
        # previous level ends (14) +2.5% at k = 8 and +1% at k = 16 over 13; with one-slot short
        # rows, 14 over 13 +0.6% at k = 32 and over 12 +1.1% at k = 4; below a 32-byte chunk,
        # one vector per lane, +9.5% over 7 at k = 1 and +8.4% over 12 at k = 2; the same walk
        # in 4-warp CTAs (15) a further +1.9% at k = 8, +2.7% at k = 32, +0.9% at k = 1
        return 15

    def resolve_pdl(self, k: int) -> bool:
        """Whether calls with ``k`` right-hand sides use programmatic dependent launch."""
        if self.pdl is not None:
            return bool(self.pdl)
        return int(k) >= PDL_MIN_K

    def locality(self, direction: Direction) -> bool:
        if self.row_order is None:
            return direction == Direction.DOWN
        return self.row_order == "locality"

    @classmethod
    def from_dict(cls, value: Mapping[str, object]) -> "B200Plan":
        allowed = {"exact_order", "heavy_threshold", "row_order", "narrow_variant", "balance", "autotune", "pad_lists",
                   "heavy_variant", "long_first", "narrow_split", "schedule", "slots", "pdl", "persist_ctas", "fuse_entries",
                   "heavy_buckets", "short_rows"}
        extra = sorted(set(value) - allowed)
        if extra:
            raise ValueError(f"unknown B200Plan field(s): {extra}")
        return cls(exact_order=bool(value.get("exact_order", False)),
                   heavy_threshold=int(value.get("heavy_threshold", DEFAULT_HEAVY_THRESHOLD)),
                   row_order=value.get("row_order"), narrow_variant=value.get("narrow_variant"),
                   balance=bool(value.get("balance", True)), autotune=bool(value.get("autotune", False)),
                   pad_lists=bool(value.get("pad_lists", True)), heavy_variant=value.get("heavy_variant"),
                   long_first=bool(value.get("long_first", True)), narrow_split=int(value.get("narrow_split", -1)),
                   schedule=str(value.get("schedule", "levels")), slots=bool(value.get("slots", False)),
                   pdl=None if value.get("pdl") is None else bool(value.get("pdl")),
                   persist_ctas=int(value.get("persist_ctas", 0)), fuse_entries=int(value.get("fuse_entries", 0)),
                   heavy_buckets=bool(value.get("heavy_buckets", False)), short_rows=bool(value.get("short_rows", True)))


@dataclass(frozen=True)
class B200PlanPair:
    plan_up: B200Plan | None = field(default_factory=B200Plan)
    plan_down: B200Plan | None = field(default_factory=B200Plan)

    def __post_init__(self) -> None:
        if self.plan_up is None and self.plan_down is None:
            raise ValueError("at least one of plan_up/plan_down must be provided")

    @classmethod
    def from_dicts(cls, plan_up: Mapping[str, object] | None, plan_down: Mapping[str, object] | None) -> "B200PlanPair":
        return cls(plan_up=None if plan_up is None else B200Plan.from_dict(plan_up),
                   plan_down=None if plan_down is None else B200Plan.from_dict(plan_down))

    def plan_for(self, direction: Direction) -> B200Plan | None:
        return self.plan_up if direction == Direction.UP else self.plan_down


@dataclass
class LevelPlan:
    artifact_index: int
    direction: Direction
    level: int
    order: int  # execution position within its traversal
    num_rows: int
    max_entries: int
    max_heavy: int
    nbytes: int
    resident: bool = True
    slot: int | None = None


@dataclass(frozen=True)
class ArtifactLayout:
    path: Path
    scan: ArtifactScan
    levels_up: tuple[LevelPlan, ...]
    levels_down: tuple[LevelPlan, ...]


@dataclass
class B200Layout:
    artifacts: tuple[ArtifactLayout, ...]
    pair: B200PlanPair
    dtype: np.dtype
    precision: str
    emit_all_nodes: bool
    mix_scratch_bytes: int
    requirements: object
    device: int
    stream_ptr: int
    stream_owner: object | None
    allow_residency: bool
    requested_ring_buffer_size: int
    allocated_ring_buffer_size: int
    vram_budget_bytes: int
    max_num_samples: int
    max_num_mutations: int
    max_num_nodes: int
    max_num_individuals: int
    max_levels: int
    slot_bytes: tuple[int, ...]
    budget_items: tuple[BudgetItem, ...]
    required_budget_for_full_residency: int
    bytes_by_category: dict[str, int]
    bytes_total: int

    def level_plans(self):
        for art in self.artifacts:
            yield from art.levels_up
            yield from art.levels_down


# -- validation helpers ---------------------------------------------------------------------

def parse_cuda_device(device) -> int:
    """Non-bool int ordinal of a visible CUDA device (``pygrgl_spmv/backends/_cuda_stream.py:108-118``)."""
    if isinstance(device, bool) or not isinstance(device, (int, np.integer)):
        raise TypeError(f"CUDA device must be a non-bool int ordinal, got {type(device).__name__}")
    device = int(device)
    if device < 0:
        raise ValueError(f"CUDA device ordinal must be non-negative, got {device}")
    import torch

    count = torch.cuda.device_count()
    if device >= count:
        raise ValueError(f"CUDA device ordinal {device} is out of range for {count} visible CUDA devices")
    return device


def parse_cuda_stream(stream) -> tuple[int, object | None]:
    """``(cudaStream_t, owner)`` from an int or a ``__cuda_stream__`` object (``_cuda_stream.py:140-174``)."""
    if isinstance(stream, bool):
        raise TypeError("CUDA stream must be a non-bool int handle or an object implementing __cuda_stream__()")
    if isinstance(stream, (int, np.integer)):
        if int(stream) < 0:
            raise ValueError(f"CUDA stream handle must be non-negative, got {int(stream)}")
        return int(stream), None
    method = getattr(stream, "__cuda_stream__", None)
    if method is None:
        cuda_stream = getattr(stream, "cuda_stream", None)  # torch.cuda.Stream
        if isinstance(cuda_stream, int):
            return int(cuda_stream), stream
        raise TypeError("CUDA stream must be a non-bool int handle or an object implementing __cuda_stream__()")
    token = method()
    if isinstance(token, bool):
        raise TypeError("__cuda_stream__() must return an int handle or a (version, handle) pair")
    if isinstance(token, (tuple, list)):
        if len(token) != 2:
            raise TypeError("__cuda_stream__() tuple/list return must be exactly (version, handle)")
        if int(token[0]) != 0:
            raise ValueError(f"Unsupported CUDA stream protocol version {int(token[0])}; expected 0")
        ptr = int(token[1])
    elif isinstance(token, (int, np.integer)):
        ptr = int(token)
    else:
        raise TypeError("__cuda_stream__() must return an int handle or a (version, handle) pair")
    if ptr < 0:
        raise ValueError(f"CUDA stream handle must be non-negative, got {ptr}")
    return ptr, stream


def _stream_device(ptr: int) -> int:
    import ctypes

    import torch

    torch.cuda.init()
    cudart = ctypes.CDLL("libcudart.so.12")
    dev = ctypes.c_int()
    status = cudart.cudaStreamGetDevice(ctypes.c_void_p(ptr), ctypes.byref(dev))
    if status != 0:
        raise RuntimeError(f"cudaStreamGetDevice failed with status {status}")
    return int(dev.value)


def _resolve_artifacts(artifacts) -> tuple[Path, ...]:
    paths = tuple(Path(p) for p in artifacts)
    if not paths:
        raise ValueError("artifacts must be non-empty")
    for p in paths:
        if p.suffix != ".grg_spmv":
            raise ValueError(f"planner expects .grg_spmv artifacts, got {p}")
        if not p.exists():
            raise FileNotFoundError(p)
    return paths


# -- byte accounting ------------------------------------------------------------------------

def _enabled_max_k(pair: B200PlanPair, requirements) -> int:
    ks = []
    if pair.plan_up is not None:
        ks.append(int(requirements.max_k_up))
    if pair.plan_down is not None:
        ks.append(int(requirements.max_k_down))
    return max(ks)


def side_io_rows(pair: B200PlanPair, requirements, *, max_num_mutations: int, max_num_nodes: int) -> int:
    """Rows of the side buffer ``io1`` (miss in/out, init vector or init matrix)."""
    need_miss = (pair.plan_down is not None and requirements.need_down_miss_input) or (
        pair.plan_up is not None and requirements.need_up_miss_output)
    return max(int(max_num_mutations) if need_miss else 0, 1 if requirements.need_init_vector else 0,
               int(max_num_nodes) if requirements.need_init_matrix else 0)


def _level_plans(artifact_index: int, scan: ArtifactScan, direction: Direction, plan: B200Plan, with_miss: bool) -> tuple[LevelPlan, ...]:
    h = scan.num_levels
    order = range(1, h) if direction == Direction.UP else range(h - 1, -1, -1)
    out = []
    for pos, level in enumerate(order):
        rows = int(scan.level_sizes[level])
        if rows == 0:
            continue
        slots = plan.slots and plan.pad_lists and plan.balance
        entries = (up_entry_bound(scan, level, plan.pad_lists, slots) if direction == Direction.UP
                   else down_entry_bound(scan, level, with_miss, plan.pad_lists, slots))
        heavy = min(rows, entries // (int(plan.heavy_threshold) + 1))
        nbytes = blob_layout(rows, heavy, entries, True)[4]  # row map: locality order or heavy suffix
        out.append(LevelPlan(artifact_index, direction, level, pos, rows, entries, heavy, nbytes))
    return tuple(out)


def _assign_slots(levels: list[LevelPlan], ring: int) -> tuple[tuple[int, ...], int]:
    for lp in levels:
        lp.slot = None
    streamed = sorted((lp for lp in levels if not lp.resident),
                      key=lambda lp: (lp.artifact_index, 0 if lp.direction == Direction.UP else 1, lp.order))
    if not streamed:
        return (), 0
    count = min(int(ring), len(streamed))
    if count < 1:
        raise ValueError("ring_buffer_size must be >= 1 when any B200 level is streamed")
    sizes = [0] * count
    for i, lp in enumerate(streamed):
        lp.slot = i % count
        sizes[lp.slot] = max(sizes[lp.slot], lp.nbytes)
    return tuple(sizes), int(sum(sizes))


def _promotion_key(lp: LevelPlan):
    return (-lp.nbytes, -lp.artifact_index, -lp.level, 0 if lp.direction == Direction.UP else 1)


def _warn_ring_mismatch(requested: int, allocated: int) -> None:
    if allocated == requested:
        return
    if allocated == 0 and requested > 0:
        warnings.warn(f"requested ring_buffer_size={requested}, but all sparse levels fit resident so no ring slots were allocated",
                      RuntimeWarning, stacklevel=3)
        return
    warnings.warn(f"requested ring_buffer_size={requested}, but only {allocated} ring slot(s) were allocated",
                  RuntimeWarning, stacklevel=3)


def plan_b200_layout(
    *,
    artifacts,
    dtype,
    requirements,
    vram_budget_bytes: int,
    ring_buffer_size: int,
    allow_residency: bool = True,
    device,
    stream,
    pair: B200PlanPair | None = None,
    precision: str = "plain",
    emit_all_nodes: bool = True,
) -> B200Layout:
    """Plan device memory for ``artifacts`` (the counterpart of ``plan_triton_layout``,
    ``pygrgl_spmv/backends/triton/backend.py:343-371``).

    ``precision="plain"`` computes and stores in ``dtype``.  ``precision="mixed"`` (``dtype``
    must be float64: inputs and outputs stay FP64) keeps the node state in 6 bytes per value,
    an FP32 value plus a 16-bit correction (relative rounding <= 2^-39 per node, integers below
    2^39 exact), with FP64 accumulation; it needs padded lists and the default (not
    exact-order) heavy-row mode.

    ``emit_all_nodes=False`` leaves out the all-node output buffer (``max_nodes x max_k``
    values, as large as an FP64 node state): the runtime then refuses
    ``prepare_matmul_cuda(..., emit_all_nodes=True)``, and the budget goes to level lists."""
    dtype = np.dtype(dtype)
    if dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError(f"B200 runtime supports only float32/float64, got {dtype}")
    pair = B200PlanPair() if pair is None else pair
    _check_precision(precision, dtype, pair)
    requested_ring = int(ring_buffer_size)
    requested_budget = int(vram_budget_bytes)
    if requested_ring < 0:
        raise ValueError("ring_buffer_size must be >= 0")
    if requested_budget < 0:
        raise ValueError("vram_budget_bytes must be >= 0")
    paths = _resolve_artifacts(artifacts)
    device_id = parse_cuda_device(device)
    stream_ptr, stream_owner = parse_cuda_stream(stream)
    if stream_ptr != 0:
        owner_device = getattr(stream_owner, "device", None)
        stream_device = int(owner_device.index) if owner_device is not None and owner_device.index is not None else _stream_device(stream_ptr)
        if stream_device != device_id:
            raise ValueError(f"CUDA stream device {stream_device} does not match requested CUDA device {device_id}")
    return plan_layout_from_scans(
        scans=tuple(scan_grg_spmv(p) for p in paths), paths=paths, dtype=dtype, requirements=requirements,
        requested_budget=requested_budget, requested_ring=requested_ring, allow_residency=bool(allow_residency),
        device_id=device_id, stream_ptr=stream_ptr, stream_owner=stream_owner, pair=pair, precision=precision,
        emit_all_nodes=emit_all_nodes)


PRECISIONS = ("plain", "mixed")


def _check_precision(precision: str, dtype, pair: B200PlanPair) -> None:
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {precision!r}")
    if precision != "mixed":
        return
    if np.dtype(dtype) != np.dtype(np.float64):
        raise ValueError("precision='mixed' keeps FP64 inputs and outputs; pass dtype=np.float64")
    for plan in (pair.plan_up, pair.plan_down):
        if plan is not None and (plan.exact_order or not plan.pad_lists):
            raise ValueError("precision='mixed' needs pad_lists=True and exact_order=False")


def mixed_state_bytes(num_nodes: int, max_k: int) -> int:
    """Node state of mixed precision: float hi plane + int16 lo plane, ld = k rounded up to 4."""
    ld = (int(max_k) + 3) // 4 * 4
    return _plane(num_nodes * ld * 4) + _plane(num_nodes * ld * 2)


def _plane(nbytes: int) -> int:
    return (int(nbytes) + 15) // 16 * 16


def plan_layout_from_scans(*, scans, paths, dtype, requirements, requested_budget: int, requested_ring: int,
                           allow_residency: bool, device_id: int, stream_ptr: int, stream_owner, pair: B200PlanPair,
                           precision: str = "plain", emit_all_nodes: bool = True) -> B200Layout:
    """The device-independent part of the planner (exercised by the CPU tests)."""
    _check_precision(precision, dtype, pair)
    itemsize = int(np.dtype(dtype).itemsize)
    max_S = max(s.num_samples for s in scans)
    max_M = max(s.num_mutations for s in scans)
    max_N = max(s.num_nodes for s in scans)
    max_I = max(s.num_individuals for s in scans)
    max_levels = max(s.num_levels for s in scans)
    max_k = _enabled_max_k(pair, requirements)
    up_on, down_on = pair.plan_up is not None, pair.plan_down is not None
    down_miss = down_on and bool(requirements.need_down_miss_input)
    up_miss = up_on and bool(requirements.need_up_miss_output)

    selectors = metadata = xtx = 0
    artifacts = []
    all_levels: list[LevelPlan] = []
    for idx, (path, scan) in enumerate(zip(paths, scans, strict=True)):
        if up_on:  # the up output gathers through sel_mut (and sel_miss for the miss output)
            selectors += 4 * (scan.num_mutations + 1 + scan.selector_mut_nnz)
            if up_miss:
                selectors += 4 * (scan.num_mutations + 1 + scan.selector_miss_nnz)
        # node_perm + inv_node_perm (matrix init / all-node output), sample->individual maps
        metadata += 4 * (2 * scan.num_nodes + 2 * scan.num_samples + scan.num_individuals + 1)
        if requirements.need_init_vector:
            metadata += itemsize * ((scan.num_mutations if up_on else 0) + (scan.num_samples if down_on else 0))
        if requirements.need_init_xtx and scan.has_xtx_bias:
            metadata += itemsize * ((scan.num_mutations if up_on else 0) + (scan.num_samples if down_on else 0))
        if requirements.need_init_xtx and scan.has_individual_coals:
            xtx += itemsize * scan.num_nodes
        lu = _level_plans(idx, scan, Direction.UP, pair.plan_up, False) if up_on else ()
        ld = _level_plans(idx, scan, Direction.DOWN, pair.plan_down, down_miss) if down_on else ()
        all_levels.extend(lu)
        all_levels.extend(ld)
        artifacts.append(ArtifactLayout(path=Path(path), scan=scan, levels_up=lu, levels_down=ld))

    state_bytes = max_N * max_k * itemsize
    mix_scratch = 0
    if precision == "mixed":
        state_bytes = mixed_state_bytes(max_N, max_k)
        if down_on:  # encoded down input (and miss) rows
            mix_scratch = mixed_state_bytes(max_M, max_k) * (2 if down_miss else 1)
    io0_rows = max(max_S, max_M)
    io1_rows = side_io_rows(pair, requirements, max_num_mutations=max_M, max_num_nodes=max_N)
    aux_rows = max_N if emit_all_nodes else 0  # all-node output
    dense_arena = (io0_rows + io1_rows + aux_rows) * max_k * itemsize
    scratch = 256 + mix_scratch  # device error word (+ mixed-precision encoded down inputs)
    fixed = selectors + metadata + xtx + state_bytes + dense_arena + scratch
    resident_full = sum(lp.nbytes for lp in all_levels)
    required_full = fixed + resident_full
    budget = required_full if requested_budget == 0 else requested_budget

    if not allow_residency:
        if all_levels and requested_ring < 1:
            raise ValueError("ring_buffer_size must be >= 1 when any B200 level is streamed")
        for lp in all_levels:
            lp.resident = False
        slot_bytes, ring_bytes = _assign_slots(all_levels, requested_ring) if all_levels else ((), 0)
        resident_bytes = 0
        total = fixed + ring_bytes
        if total > budget:
            raise ValueError(f"B200 layout requires at least {total} owned device bytes, exceeds vram_budget_bytes={budget}")
        _warn_ring_mismatch(requested_ring, len(slot_bytes))
    elif required_full <= budget:
        for lp in all_levels:
            lp.resident = True
            lp.slot = None
        slot_bytes, ring_bytes, resident_bytes, total = (), 0, resident_full, required_full
        _warn_ring_mismatch(requested_ring, 0)
    else:
        if requested_ring < 1:
            raise ValueError("ring_buffer_size must be >= 1 when any B200 level is streamed")
        for lp in all_levels:
            lp.resident = False
        slot_bytes, ring_bytes = _assign_slots(all_levels, requested_ring)
        if fixed + ring_bytes > budget:
            raise ValueError(f"B200 layout requires at least {fixed + ring_bytes} owned device bytes, exceeds vram_budget_bytes={budget}")
        for lp in sorted(all_levels, key=_promotion_key):
            lp.resident = True
            resident_bytes = sum(x.nbytes for x in all_levels if x.resident)
            slot_bytes, ring_bytes = _assign_slots(all_levels, requested_ring)
            if fixed + resident_bytes + ring_bytes > budget:
                lp.resident = False
        resident_bytes = sum(x.nbytes for x in all_levels if x.resident)
        slot_bytes, ring_bytes = _assign_slots(all_levels, requested_ring)
        total = fixed + resident_bytes + ring_bytes
        _warn_ring_mismatch(requested_ring, len(slot_bytes))
    if total > budget:
        raise ValueError(f"B200 layout requires {total} owned device bytes, exceeds vram_budget_bytes={budget}")

    bytes_by_category = {
        "resident_sparse": int(resident_bytes),
        "ring_slots": int(ring_bytes),
        "selectors": int(selectors),
        "metadata": int(metadata),
        "xtx_bias": int(xtx),
        "dense_arena": int(dense_arena),
        "state": int(state_bytes),
        "scratch": int(scratch),
    }
    items = [BudgetItem(kind="fixed", name=name, nbytes=int(bytes_by_category[name]))
             for name in ("selectors", "metadata", "xtx_bias", "dense_arena", "state", "scratch")]
    for lp in all_levels:
        if lp.resident:
            items.append(BudgetItem(kind="resident_sparse", name="resident_sparse", nbytes=int(lp.nbytes),
                                    artifact_index=lp.artifact_index, dst_level=lp.level, direction=lp.direction.value))
    for slot, nbytes in enumerate(slot_bytes):
        items.append(BudgetItem(kind="ring_slot", name="ring_slots", nbytes=int(nbytes), slot=slot))
    return B200Layout(
        artifacts=tuple(artifacts),
        pair=pair,
        dtype=np.dtype(dtype),
        precision=precision,
        emit_all_nodes=bool(emit_all_nodes),
        mix_scratch_bytes=int(mix_scratch),
        requirements=requirements,
        device=device_id,
        stream_ptr=stream_ptr,
        stream_owner=stream_owner,
        allow_residency=allow_residency,
        requested_ring_buffer_size=requested_ring,
        allocated_ring_buffer_size=len(slot_bytes),
        vram_budget_bytes=int(budget),
        max_num_samples=max_S,
        max_num_mutations=max_M,
        max_num_nodes=max_N,
        max_num_individuals=max_I,
        max_levels=max_levels,
        slot_bytes=tuple(int(b) for b in slot_bytes),
        budget_items=tuple(i for i in items if i.nbytes > 0),
        required_budget_for_full_residency=int(required_full),
        bytes_by_category=bytes_by_category,
        bytes_total=int(sum(i.nbytes for i in items)),
    )


__all__ = ["B200Layout", "B200Plan", "B200PlanPair", "BudgetItem", "LevelPlan", "plan_b200_layout", "plan_layout_from_scans"]
