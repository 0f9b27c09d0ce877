"""The ``.grg_spmv`` artifact: format version 8, an uncompressed ``numpy.savez`` archive.

This module reads and writes the same file format as the reference package
(``pygrgl_spmv/grg/artifact.py``): the magic/version keys (``:19-22``), the key set written
by ``save_grg_spmv`` (``:124-184``), the metadata-only scan (``:245-343``), the block
iterator (``:346-369``) and the host header loader (``:372-439``).  Artifacts written by
either package load in the other; ``tests/golden`` holds reference-written files that the
tests read back with this module.

Block ``A_blocks[dst][src]`` is a 0/1 CSR matrix whose rows are the nodes of level
``dst`` and whose columns are the nodes of level ``src < dst`` (level-local ids, sorted
unique columns per row).  An edge ``parent -> child`` lives in the block of
``(level(parent), level(child))``.
"""

from __future__ import annotations

from dataclasses import dataclass
import functools
import logging
import os
from pathlib import Path
import tempfile

import numpy as np
import scipy.sparse as sp

GRG_SPMV_FORMAT_MAGIC = "grg_spmv"
GRG_SPMV_FORMAT_VERSION = 8
_MAGIC_KEY = "grg_spmv_magic"
_VERSION_KEY = "grg_spmv_format_version"
_LOGGER = logging.getLogger(__name__)
_STRUCT_DTYPES = (np.dtype(np.int32), np.dtype(np.int64))


def smallest_struct_dtype(max_value: int) -> np.dtype:
    """int32 when every structural value fits, else int64 (reference ``grg/sparse.py:13-19``)."""
    if int(max_value) < 0:
        raise ValueError(f"Structural integer values must be non-negative, got {max_value}")
    return np.dtype(np.int32) if int(max_value) <= np.iinfo(np.int32).max else np.dtype(np.int64)


def compact_struct_array(values) -> np.ndarray:
    arr = np.asarray(values)
    if arr.dtype.kind not in "iu":
        raise TypeError(f"structural arrays must be integer, got {arr.dtype}")
    arr = arr.reshape(-1) if arr.ndim == 0 else arr
    if arr.size == 0:
        return arr.astype(np.int32, copy=False)
    if int(arr.min()) < 0:
        raise ValueError("structural arrays must be non-negative")
    return arr.astype(smallest_struct_dtype(int(arr.max())), copy=False)


def binary_csr(indices, indptr, shape) -> sp.csr_matrix:
    """A 0/1 CSR matrix with bool data built from saved index arrays (no copies of the index arrays)."""
    idx = np.asarray(indices)
    ptr = np.asarray(indptr)
    if idx.ndim != 1 or ptr.ndim != 1:
        raise ValueError("CSR indices and indptr must be one-dimensional")
    if idx.dtype not in _STRUCT_DTYPES or ptr.dtype not in _STRUCT_DTYPES:
        raise TypeError(f"CSR index arrays must be int32/int64, got {idx.dtype}/{ptr.dtype}")
    data = np.ones(idx.size, dtype=np.bool_)
    return sp.csr_matrix((data, idx, ptr), shape=tuple(int(v) for v in shape))


@dataclass
class CompiledOperatorState:
    """In-memory form of one artifact (field names follow ``pygrgl_spmv/grg/compile.py:18-46``)."""

    A_blocks: list | None
    level_offsets: np.ndarray
    node_perm: np.ndarray
    inv_node_perm: np.ndarray
    sel_mut: sp.csr_matrix
    sel_miss: sp.csr_matrix
    num_samples: int
    num_mutations: int
    num_nodes: int
    ploidy: int
    num_individuals: int
    num_edges: int
    has_missing_data: bool
    sample_to_individual: np.ndarray
    mutation_positions: np.ndarray
    mutation_times: np.ndarray
    mutation_alleles: np.ndarray
    mutation_allele_offsets: np.ndarray
    mutation_ref_alleles: np.ndarray
    mutation_ref_allele_offsets: np.ndarray
    coalescence_counts: np.ndarray | None
    init_vector_up_bias: np.ndarray | None = None
    init_vector_down_bias: np.ndarray | None = None
    init_xtx_up_bias: np.ndarray | None = None
    init_xtx_down_bias: np.ndarray | None = None


@dataclass(frozen=True)
class ArtifactBlockScan:
    dst_level: int
    src_level: int
    shape: tuple[int, int]
    nnz: int
    indices_dtype: np.dtype
    indptr_dtype: np.dtype


@dataclass(frozen=True)
class ArtifactBlock:
    dst_level: int
    src_level: int
    shape: tuple[int, int]
    indices: np.ndarray
    indptr: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.indices.size)


@dataclass(frozen=True)
class ArtifactScan:
    path: Path
    num_samples: int
    num_mutations: int
    num_nodes: int
    num_individuals: int
    num_edges: int
    ploidy: int
    has_missing_data: bool
    has_xtx_bias: bool
    level_offsets: np.ndarray
    level_sizes: tuple[int, ...]
    num_levels: int
    selector_mut_nnz: int
    selector_miss_nnz: int
    has_individual_coals: bool
    selector_nnz_by_level: np.ndarray
    node_perm_dtype: np.dtype
    sample_to_individual_dtype: np.dtype
    blocks: tuple[ArtifactBlockScan, ...]

    @property
    def max_block_nnz(self) -> int:
        return max((block.nnz for block in self.blocks), default=0)


def _nnz_per_level(indices: np.ndarray, level_offsets: np.ndarray) -> np.ndarray:
    offsets = np.asarray(level_offsets, dtype=np.int64)
    num_levels = max(int(offsets.size) - 1, 0)
    idx = np.asarray(indices, dtype=np.int64)
    if idx.size == 0:
        return np.zeros(num_levels, dtype=np.int64)
    levels = np.searchsorted(offsets, idx, side="right") - 1
    if levels.min() < 0 or levels.max() >= num_levels:
        raise ValueError("selector indices are outside level_offsets")
    return np.bincount(levels, minlength=num_levels).astype(np.int64)


def save_grg_spmv(state: CompiledOperatorState, artifact_path) -> None:
    """Write ``state`` atomically: a temporary file in the target directory, fsync, rename."""
    if state.A_blocks is None:
        raise RuntimeError("compiled operator blocks are required for .grg_spmv save")
    if state.init_vector_up_bias is None or state.init_vector_down_bias is None:
        raise RuntimeError("init vector bias cache must be populated before .grg_spmv save")
    offsets = np.asarray(state.level_offsets)
    sel_mut_idx = np.asarray(state.sel_mut.indices)
    sel_miss_idx = np.asarray(state.sel_miss.indices)
    by_level = np.column_stack((_nnz_per_level(sel_mut_idx, offsets), _nnz_per_level(sel_miss_idx, offsets))).astype(np.int64)
    node_perm = np.asarray(state.node_perm)
    s2i = np.asarray(state.sample_to_individual)
    arrays: dict[str, np.ndarray] = {
        _MAGIC_KEY: np.asarray(GRG_SPMV_FORMAT_MAGIC),
        _VERSION_KEY: np.asarray(GRG_SPMV_FORMAT_VERSION, dtype=np.int32),
        "num_samples": np.asarray(state.num_samples, dtype=np.int64),
        "num_mutations": np.asarray(state.num_mutations, dtype=np.int64),
        "num_nodes": np.asarray(state.num_nodes, dtype=np.int64),
        "ploidy": np.asarray(state.ploidy, dtype=np.int64),
        "num_individuals": np.asarray(state.num_individuals, dtype=np.int64),
        "num_edges": np.asarray(state.num_edges, dtype=np.int64),
        "has_missing_data": np.asarray(state.has_missing_data, dtype=bool),
        "level_offsets": offsets,
        "node_perm": node_perm,
        "sample_to_individual": s2i,
        "mutation_positions": np.asarray(state.mutation_positions, dtype=np.float64),
        "mutation_times": np.asarray(state.mutation_times, dtype=np.float64),
        "mutation_alleles": np.asarray(state.mutation_alleles),
        "mutation_allele_offsets": np.asarray(state.mutation_allele_offsets),
        "mutation_ref_alleles": np.asarray(state.mutation_ref_alleles),
        "mutation_ref_allele_offsets": np.asarray(state.mutation_ref_allele_offsets),
        "has_individual_coals": np.asarray(state.coalescence_counts is not None, dtype=bool),
        "init_vector_up_bias": np.asarray(state.init_vector_up_bias),
        "init_vector_down_bias": np.asarray(state.init_vector_down_bias),
        "has_xtx_bias": np.asarray(state.init_xtx_up_bias is not None and state.init_xtx_down_bias is not None, dtype=bool),
        "sel_mut_indices": sel_mut_idx,
        "sel_mut_indptr": np.asarray(state.sel_mut.indptr),
        "sel_miss_indices": sel_miss_idx,
        "sel_miss_indptr": np.asarray(state.sel_miss.indptr),
    }
    if state.coalescence_counts is not None:
        arrays["coalescence_counts"] = np.asarray(state.coalescence_counts, dtype=np.int64)
    if state.init_xtx_up_bias is not None:
        arrays["init_xtx_up_bias"] = np.asarray(state.init_xtx_up_bias)
    if state.init_xtx_down_bias is not None:
        arrays["init_xtx_down_bias"] = np.asarray(state.init_xtx_down_bias)
    levels, shapes, nnzs, itemsizes = [], [], [], []
    for dst, row in enumerate(state.A_blocks):
        for src, block in enumerate(row):
            indices = np.asarray(block.indices)
            indptr = np.asarray(block.indptr)
            arrays[f"A_blocks_{dst}_{src}_indices"] = indices
            arrays[f"A_blocks_{dst}_{src}_indptr"] = indptr
            levels.append((dst, src))
            shapes.append((int(block.shape[0]), int(block.shape[1])))
            nnzs.append(int(indices.size))
            itemsizes.append((indices.dtype.itemsize, indptr.dtype.itemsize))
    arrays["scan_block_levels"] = np.asarray(levels, dtype=np.int32).reshape(-1, 2)
    arrays["scan_block_shapes"] = np.asarray(shapes, dtype=np.int64).reshape(-1, 2)
    arrays["scan_block_nnzs"] = np.asarray(nnzs, dtype=np.int64)
    arrays["scan_block_struct_itemsize"] = np.asarray(itemsizes, dtype=np.uint8).reshape(-1, 2)
    arrays["scan_selector_nnzs"] = np.asarray((int(state.sel_mut.nnz), int(state.sel_miss.nnz)), dtype=np.int64)
    arrays["scan_selector_nnz_by_level"] = by_level
    arrays["scan_metadata_struct_itemsize"] = np.asarray((node_perm.dtype.itemsize, s2i.dtype.itemsize), dtype=np.uint8)

    path = Path(artifact_path)
    path.parent.mkdir(parents=True, exist_ok=True)
    fd, tmp_name = tempfile.mkstemp(prefix=f".{path.name}.", suffix=".tmp", dir=path.parent)
    tmp = Path(tmp_name)
    try:
        with os.fdopen(fd, "wb") as handle:
            np.savez(handle, **arrays)
            handle.flush()
            os.fsync(handle.fileno())
        tmp.replace(path)
    except Exception:
        tmp.unlink(missing_ok=True)
        raise
    _scan_cached.cache_clear()


def _open(path) -> np.lib.npyio.NpzFile:
    return np.load(path, allow_pickle=False)


def _check_header(data, path) -> None:
    if _MAGIC_KEY not in data.files:
        raise ValueError(f"unsupported .grg_spmv artifact in {path}: missing {_MAGIC_KEY}")
    magic = str(np.asarray(data[_MAGIC_KEY]).item())
    if magic != GRG_SPMV_FORMAT_MAGIC:
        raise ValueError(f"unsupported .grg_spmv artifact in {path}: got magic {magic!r}")
    if _VERSION_KEY not in data.files:
        raise ValueError(f"unsupported .grg_spmv artifact in {path}: missing {_VERSION_KEY}")
    version = int(np.asarray(data[_VERSION_KEY]).item())
    if version != GRG_SPMV_FORMAT_VERSION:
        raise ValueError(
            f"unsupported .grg_spmv artifact in {path}: got version {version}, expected {GRG_SPMV_FORMAT_VERSION}"
        )


def _struct(data, key: str) -> np.ndarray:
    arr = np.asarray(data[key])
    if arr.dtype not in _STRUCT_DTYPES:
        raise ValueError(f"unsupported structural dtype for {key}: {arr.dtype}")
    if arr.size and int(arr.min()) < 0:
        raise ValueError(f"structural array {key} must be non-negative")
    return arr


def _dtype_of_itemsize(itemsize: int) -> np.dtype:
    if int(itemsize) == 4:
        return np.dtype(np.int32)
    if int(itemsize) == 8:
        return np.dtype(np.int64)
    raise ValueError(f"unsupported structural itemsize: {itemsize}")


def _scalar(data, key):
    return np.asarray(data[key]).item()


@functools.cache
def _scan_cached(path: Path) -> ArtifactScan:
    with _open(path) as data:
        _check_header(data, path)
        offsets = _struct(data, "level_offsets")
        offsets.setflags(write=False)
        sizes = tuple(int(offsets[i + 1]) - int(offsets[i]) for i in range(len(offsets) - 1))
        blk_levels = np.asarray(data["scan_block_levels"])
        blk_shapes = np.asarray(data["scan_block_shapes"])
        blk_nnzs = np.asarray(data["scan_block_nnzs"])
        blk_items = np.asarray(data["scan_block_struct_itemsize"])
        sel_nnzs = np.asarray(data["scan_selector_nnzs"])
        sel_by_level = np.asarray(data["scan_selector_nnz_by_level"], dtype=np.int64)
        meta_items = np.asarray(data["scan_metadata_struct_itemsize"])
        for name, arr in (("scan_block_levels", blk_levels), ("scan_block_shapes", blk_shapes), ("scan_block_struct_itemsize", blk_items)):
            if arr.ndim != 2 or arr.shape[1] != 2:
                raise ValueError(f"{name} must have shape (num_blocks, 2), got {arr.shape}")
        if blk_nnzs.ndim != 1:
            raise ValueError(f"scan_block_nnzs must be one-dimensional, got {blk_nnzs.shape}")
        nblk = blk_levels.shape[0]
        if blk_shapes.shape[0] != nblk or blk_nnzs.shape[0] != nblk or blk_items.shape[0] != nblk:
            raise ValueError("scan block metadata arrays must have matching lengths")
        if sel_nnzs.shape != (2,):
            raise ValueError(f"scan_selector_nnzs must have shape (2,), got {sel_nnzs.shape}")
        if sel_by_level.shape != (len(sizes), 2):
            raise ValueError(f"scan_selector_nnz_by_level must have shape ({len(sizes)}, 2), got {sel_by_level.shape}")
        if meta_items.shape != (2,):
            raise ValueError(f"scan_metadata_struct_itemsize must have shape (2,), got {meta_items.shape}")
        for arr in (blk_levels, blk_shapes, blk_nnzs, sel_nnzs, sel_by_level):
            if arr.size and np.any(arr < 0):
                raise ValueError("scan metadata arrays must be non-negative")
        if np.any(sel_by_level.sum(axis=0) != sel_nnzs):
            raise ValueError("scan selector metadata arrays must have matching nnz totals")
        sel_by_level.setflags(write=False)
        blocks = tuple(
            ArtifactBlockScan(int(lv[0]), int(lv[1]), (int(sh[0]), int(sh[1])), int(nz),
                              _dtype_of_itemsize(int(it[0])), _dtype_of_itemsize(int(it[1])))
            for lv, sh, nz, it in zip(blk_levels, blk_shapes, blk_nnzs, blk_items, strict=True)
        )
        return ArtifactScan(
            path=path,
            num_samples=int(_scalar(data, "num_samples")),
            num_mutations=int(_scalar(data, "num_mutations")),
            num_nodes=int(_scalar(data, "num_nodes")),
            num_individuals=int(_scalar(data, "num_individuals")),
            num_edges=int(_scalar(data, "num_edges")),
            ploidy=int(_scalar(data, "ploidy")),
            has_missing_data=bool(_scalar(data, "has_missing_data")),
            has_xtx_bias=bool(_scalar(data, "has_xtx_bias")),
            level_offsets=np.asarray(offsets),
            level_sizes=sizes,
            num_levels=len(sizes),
            selector_mut_nnz=int(sel_nnzs[0]),
            selector_miss_nnz=int(sel_nnzs[1]),
            has_individual_coals=bool(_scalar(data, "has_individual_coals")),
            selector_nnz_by_level=sel_by_level,
            node_perm_dtype=_dtype_of_itemsize(int(meta_items[0])),
            sample_to_individual_dtype=_dtype_of_itemsize(int(meta_items[1])),
            blocks=blocks,
        )


def scan_grg_spmv(path) -> ArtifactScan:
    """Metadata of an artifact without loading block or selector arrays (cached per path)."""
    return _scan_cached(Path(path).resolve())


def iter_artifact_blocks(path):
    """Yield every stored ``A_blocks`` entry in file order."""
    path = Path(path)
    with _open(path) as data:
        _check_header(data, path)
        levels = np.asarray(data["scan_block_levels"])
        shapes = np.asarray(data["scan_block_shapes"])
        if levels.ndim != 2 or levels.shape[1] != 2 or shapes.ndim != 2 or shapes.shape[1] != 2:
            raise ValueError("scan block metadata must have shape (num_blocks, 2)")
        if levels.shape[0] != shapes.shape[0]:
            raise ValueError("scan block metadata arrays must have matching lengths")
        for (dst, src), shape in zip(levels, shapes, strict=True):
            dst, src = int(dst), int(src)
            yield ArtifactBlock(
                dst_level=dst,
                src_level=src,
                shape=(int(shape[0]), int(shape[1])),
                indices=_struct(data, f"A_blocks_{dst}_{src}_indices"),
                indptr=_struct(data, f"A_blocks_{dst}_{src}_indptr"),
            )


def invert_permutation(perm: np.ndarray) -> np.ndarray:
    perm = compact_struct_array(perm)
    inv = np.empty(perm.size, dtype=perm.dtype)
    inv[perm] = np.arange(perm.size, dtype=perm.dtype)
    return inv


def load_grg_spmv_header(path, dtype) -> CompiledOperatorState:
    """Everything but the level blocks, with float arrays cast to ``dtype``."""
    path = Path(path)
    with _open(path) as data:
        _check_header(data, path)
        num_mutations = int(_scalar(data, "num_mutations"))
        num_nodes = int(_scalar(data, "num_nodes"))
        node_perm = _struct(data, "node_perm")
        coal = np.asarray(data["coalescence_counts"], dtype=np.int64) if bool(_scalar(data, "has_individual_coals")) else None
        has_xtx = bool(_scalar(data, "has_xtx_bias"))
        return CompiledOperatorState(
            A_blocks=None,
            level_offsets=_struct(data, "level_offsets"),
            node_perm=node_perm,
            inv_node_perm=invert_permutation(node_perm),
            sel_mut=binary_csr(_struct(data, "sel_mut_indices"), _struct(data, "sel_mut_indptr"), (num_mutations, num_nodes)),
            sel_miss=binary_csr(_struct(data, "sel_miss_indices"), _struct(data, "sel_miss_indptr"), (num_mutations, num_nodes)),
            num_samples=int(_scalar(data, "num_samples")),
            num_mutations=num_mutations,
            num_nodes=num_nodes,
            ploidy=int(_scalar(data, "ploidy")),
            num_individuals=int(_scalar(data, "num_individuals")),
            num_edges=int(_scalar(data, "num_edges")),
            has_missing_data=bool(_scalar(data, "has_missing_data")),
            sample_to_individual=_struct(data, "sample_to_individual"),
            mutation_positions=np.asarray(data["mutation_positions"], dtype=np.float64),
            mutation_times=np.asarray(data["mutation_times"], dtype=np.float64),
            mutation_alleles=np.asarray(data["mutation_alleles"]),
            mutation_allele_offsets=np.asarray(data["mutation_allele_offsets"]),
            mutation_ref_alleles=np.asarray(data["mutation_ref_alleles"]),
            mutation_ref_allele_offsets=np.asarray(data["mutation_ref_allele_offsets"]),
            coalescence_counts=coal,
            init_vector_up_bias=np.asarray(data["init_vector_up_bias"], dtype=dtype),
            init_vector_down_bias=np.asarray(data["init_vector_down_bias"], dtype=dtype),
            init_xtx_up_bias=np.asarray(data["init_xtx_up_bias"], dtype=dtype) if has_xtx else None,
            init_xtx_down_bias=np.asarray(data["init_xtx_down_bias"], dtype=dtype) if has_xtx else None,
        )


def load_grg_spmv(path, dtype) -> CompiledOperatorState:
    """Header plus the full ``A_blocks`` grid; absent blocks become empty CSR matrices."""
    state = load_grg_spmv_header(path, dtype)
    offsets = np.asarray(state.level_offsets, dtype=np.int64)
    sizes = np.diff(offsets)
    num_levels = sizes.size
    grid: list[list] = [[None] * dst for dst in range(num_levels)]
    for block in iter_artifact_blocks(path):
        grid[block.dst_level][block.src_level] = binary_csr(block.indices, block.indptr, block.shape)
    for dst in range(num_levels):
        for src in range(dst):
            if grid[dst][src] is None:
                grid[dst][src] = binary_csr(np.empty(0, np.int32), np.zeros(int(sizes[dst]) + 1, np.int32), (int(sizes[dst]), int(sizes[src])))
    state.A_blocks = grid
    return state


__all__ = [
    "ArtifactBlock",
    "ArtifactBlockScan",
    "ArtifactScan",
    "CompiledOperatorState",
    "GRG_SPMV_FORMAT_MAGIC",
    "GRG_SPMV_FORMAT_VERSION",
    "binary_csr",
    "compact_struct_array",
    "invert_permutation",
    "iter_artifact_blocks",
    "load_grg_spmv",
    "load_grg_spmv_header",
    "save_grg_spmv",
    "scan_grg_spmv",
    "smallest_struct_dtype",
]
