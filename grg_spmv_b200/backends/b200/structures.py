"""Host-side construction of the per-level gather lists that the B200 kernels walk.

For every destination level the traversal needs, for each row, the list of rows it adds up.
The lists are built from the artifact's ``A_blocks`` and selectors and ordered so that a
left-to-right sum with a fresh partial sum per segment reproduces ``ReferenceRuntime``:

* up, level ``L >= 1``: the row's children, one segment per child level in ascending level
  order, ascending node id inside a segment (``dst += A[L][src] @ v[src]`` for ``src``
  ascending, ``pygrgl_spmv/backends/reference.py:399-407``; CSR rows summed left to right).
* down, every level from the top down: first the row's mutations (``sel_mut^T x``, ascending
  mutation id, duplicates kept, ``reference.py:416-417``), then its missingness mutations
  (``sel_miss^T miss``, ``:418-419``), then its parents, one segment per parent level in
  descending level order, ascending id inside a segment (``A[src][D].T @ v[src]`` for ``src``
  descending, ``:420-429`` with ``pygrgl_spmv/backends/base.py:115-117``; a CSC product adds
  columns in ascending order).

Blocks are canonicalised first (duplicates merged, columns sorted), as the reference does in
``materialize_sparse_block`` (``pygrgl_spmv/backends/base.py:128-139``).  Each level is packed
into one byte blob ``[int32 row_ptr | int32 heavy_rows | int32 row_ids | uint32 entries]`` with 16-byte
aligned sections, the unit of residency and of streaming through the ring.

Rows may be stored in a locality order instead of node order (``row_ids`` maps processing
position to row): the kernels' results do not depend on the order in which rows are
processed, only on each row's own list.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from grg_spmv_b200.backends.b200 import _native as nat

ALIGN = 16


def _stable_argsort(keys: np.ndarray) -> np.ndarray:
    """Stable argsort of integer keys: PyTorch's multithreaded CPU sort when available (about
    7x NumPy's single-threaded one on tens of millions of keys), else NumPy; same result."""
    keys = np.asarray(keys)
    if keys.size < (1 << 16):
        return np.argsort(keys, kind="stable")
    try:
        import torch
    except ImportError:  # pragma: no cover - torch is a dependency of the runtime
        return np.argsort(keys, kind="stable")
    return torch.sort(torch.from_numpy(np.ascontiguousarray(keys.astype(np.int64, copy=False))), stable=True)[1].numpy()


def _align(n: int) -> int:
    return (int(n) + ALIGN - 1) // ALIGN * ALIGN


def blob_layout(num_rows: int, num_heavy: int, num_entries: int, with_row_ids: bool) -> tuple[int, int, int, int, int]:
    """(off_row_ptr, off_heavy, off_row_ids or -1, off_entries, blob_bytes) of a level blob."""
    off_heavy = _align(4 * (int(num_rows) + 1))
    off_ids = off_heavy + _align(4 * int(num_heavy))
    off_entries = off_ids + (_align(4 * int(num_rows)) if with_row_ids else 0)
    return 0, off_heavy, (off_ids if with_row_ids else -1), off_entries, off_entries + _align(4 * max(int(num_entries), 1))


@dataclass
class LevelGather:
    """One level's gather lists in processing order (position p computes row ``row_ids[p]``)."""

    level: int
    row_begin: int
    num_rows: int
    row_ptr: np.ndarray  # int32 [num_rows + 1], by processing position
    entries: np.ndarray  # uint32
    heavy_rows: np.ndarray  # int32 processing positions
    heavy_threshold: int
    row_ids: np.ndarray | None = None  # int32 level-local row of each position (None: identity)
    list_align: int = 1  # 4: lists padded to multiples of 4 entries with null codes
    # slot layout: int64 [buckets, 3] = (first position, first entry, width in 4-entry quads);
    # every narrow row of a bucket holds exactly `width` quads, so its list starts at
    # first entry + (position - first position) * 4 * width
    slots: np.ndarray | None = None

    @property
    def num_entries(self) -> int:
        return int(self.entries.size)

    def short_rows(self) -> int:
        """The longest suffix of the narrow positions whose lists hold at most one quad (4
        entries): the rows the entry-parallel walks take with one entry slot.  Under the
        default long-first bucketing these are all narrow rows of at most 3 entries (and the
        empty ones).  0 for unpadded lists."""
        narrow = self.num_rows - int(self.heavy_rows.size)
        if self.list_align != 4 or narrow <= 0:
            return 0
        longer = np.flatnonzero(np.diff(self.row_ptr[:narrow + 1].astype(np.int64)) > 4)
        return narrow - (int(longer[-1]) + 1 if longer.size else 0)

    def layout(self) -> tuple[int, int, int, int, int]:
        return blob_layout(self.num_rows, self.heavy_rows.size, self.entries.size, self.row_ids is not None)

    def pack(self) -> np.ndarray:
        off_ptr, off_heavy, off_ids, off_entries, nbytes = self.layout()
        blob = np.zeros(nbytes, dtype=np.uint8)
        blob[off_ptr:off_ptr + 4 * self.row_ptr.size] = self.row_ptr.view(np.uint8)
        blob[off_heavy:off_heavy + 4 * self.heavy_rows.size] = self.heavy_rows.view(np.uint8)
        if self.row_ids is not None:
            blob[off_ids:off_ids + 4 * self.row_ids.size] = self.row_ids.view(np.uint8)
        blob[off_entries:off_entries + 4 * self.entries.size] = self.entries.view(np.uint8)
        return blob

    def row_lists(self):
        """(level-local row, entries) per processing position (test helper)."""
        for p in range(self.num_rows):
            row = p if self.row_ids is None else int(self.row_ids[p])
            yield row, self.entries[int(self.row_ptr[p]):int(self.row_ptr[p + 1])]


def canonical_coo(indices: np.ndarray, indptr: np.ndarray, shape) -> tuple[np.ndarray, np.ndarray]:
    """(rows, cols) of a 0/1 CSR block, sorted by (row, col) with duplicates merged."""
    nrows, ncols = int(shape[0]), int(shape[1])
    ptr = np.asarray(indptr, dtype=np.int64)
    cols = np.asarray(indices, dtype=np.int64)
    rows = np.repeat(np.arange(nrows, dtype=np.int64), np.diff(ptr))
    key = rows * max(ncols, 1) + cols
    if key.size > 1 and not np.all(key[1:] > key[:-1]):
        key = np.unique(key)
        rows, cols = key // max(ncols, 1), key % max(ncols, 1)
    return rows, cols


def _bit_length(counts: np.ndarray) -> np.ndarray:
    """ceil(log2(c + 1)) of non-negative integers, exactly: the number of powers of two <= c."""
    return np.searchsorted(_POW2, np.asarray(counts, dtype=np.int64), side="right").astype(np.int64)


_POW2 = np.asarray([1 << i for i in range(62)], dtype=np.int64)


def _quad_class(counts: np.ndarray) -> np.ndarray:
    """Slot width in 4-entry quads of rows with ``counts`` entries: 0, 1, 2, 4, 8, ..."""
    quads = (np.asarray(counts, dtype=np.int64) + 3) // 4
    width = np.ones_like(quads)
    while np.any(width < quads):
        width = np.where(width < quads, width * 2, width)
    return np.where(quads == 0, 0, width)


def _finish(level: int, row_begin: int, num_rows: int, rows: np.ndarray, ids: np.ndarray, src: np.ndarray,
            group: np.ndarray, heavy_threshold: int, locality: bool = False, balance: bool = True,
            pad: bool = False, long_first: bool = True, slots: bool = False, heavy_buckets: bool = False) -> LevelGather:
    """Stable-sort the concatenated pieces by row, flag segment starts, build row_ptr.

    With ``locality`` the rows are stored in the order of the id of their last state entry
    (the lowest-level parent for down), so rows that share source rows are processed close
    together and the shared rows are fetched from L2; each row still writes its own slot.
    """
    order = _stable_argsort(rows)
    rows, ids, src, group = rows[order], ids[order], src[order], group[order]
    if ids.size and int(ids.max()) > nat.MAX_ID:
        raise ValueError(f"level {level} names ids above {nat.MAX_ID}, beyond the B200 backend's limit")
    counts = np.bincount(rows, minlength=num_rows) if rows.size else np.zeros(num_rows, dtype=np.int64)
    row_ptr = np.zeros(num_rows + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    if row_ptr[-1] > np.iinfo(np.int32).max:
        raise ValueError(f"level {level} has {int(row_ptr[-1])} entries, above the 2^31-1 per-level limit")
    start = np.ones(ids.size, dtype=bool)
    if ids.size > 1:
        start[1:] = (rows[1:] != rows[:-1]) | (group[1:] != group[:-1])
    entries = (ids.astype(np.uint32) | (src.astype(np.uint32) << np.uint32(nat.SRC_SHIFT))
               | np.where(start, np.uint32(nat.SEG_START), np.uint32(0))).astype(np.uint32)
    # Processing order: narrow rows first, grouped into power-of-two length buckets so the rows
    # of a warp need similar trip counts (in locality order inside a bucket when asked), the
    # longest bucket first (``long_first``: CTAs start in index order, so the longest chains of
    # dependent loads start earliest and short rows fill in behind them); heavy rows last.
    perm = np.arange(num_rows, dtype=np.int64)
    if locality and num_rows > 1:
        key = np.full(num_rows, np.iinfo(np.int64).max, dtype=np.int64)
        state_pos = np.flatnonzero(src == nat.SRC_STATE)
        # Last state entry of each row: entries are sorted by row, so it is where the row changes.
        if state_pos.size:
            rs = rows[state_pos]
            last = np.flatnonzero(np.append(rs[1:] != rs[:-1], True))
            key[rs[last]] = ids[state_pos[last]]
        perm = _stable_argsort(key)
    use_slots = slots and pad and balance
    heavy_mask = counts[perm] > heavy_threshold
    narrow_perm, heavy_perm = perm[~heavy_mask], perm[heavy_mask]
    if balance and narrow_perm.size > 1:
        if use_slots:  # buckets of equal padded width (power-of-two quads)
            bucket = _quad_class(counts[narrow_perm])
        else:
            bucket = _bit_length(counts[narrow_perm])
        narrow_perm = narrow_perm[_stable_argsort(-bucket if long_first else bucket)]
    if balance and heavy_buckets and heavy_perm.size > 1:
        bucket = _bit_length(counts[heavy_perm])
        heavy_perm = heavy_perm[_stable_argsort(-bucket if long_first else bucket)]
    perm = np.concatenate((narrow_perm, heavy_perm))
    num_heavy = int(heavy_perm.size)
    row_ids = None
    if not np.array_equal(perm, np.arange(num_rows)):
        lengths = counts[perm]
        new_ptr = np.zeros(num_rows + 1, dtype=np.int64)
        np.cumsum(lengths, out=new_ptr[1:])
        gather = np.repeat(row_ptr[:-1][perm] - new_ptr[:-1], lengths) + np.arange(int(new_ptr[-1]), dtype=np.int64)
        entries = entries[gather]
        row_ptr, row_ids = new_ptr, perm.astype(np.int32)
    counts = np.diff(row_ptr)
    slot_table = None
    if pad:
        # Every list starts at a multiple of 4 entries and holds a multiple of 4 (null padding);
        # with slots a narrow row is padded to its bucket's width.
        padded = (counts + 3) // 4 * 4
        if use_slots:
            narrow = num_rows - num_heavy
            width = _quad_class(counts[:narrow])
            padded = padded.copy()
            padded[:narrow] = 4 * width
            starts = np.concatenate(([0], np.flatnonzero(width[1:] != width[:-1]) + 1)) if narrow else np.empty(0, np.int64)
            first_entry = np.concatenate(([0], np.cumsum(padded[:narrow])))
            slot_table = np.stack([starts, first_entry[starts], width[starts]], axis=1).astype(np.int64) if narrow else \
                np.zeros((0, 3), dtype=np.int64)
        new_ptr = np.zeros(num_rows + 1, dtype=np.int64)
        np.cumsum(padded, out=new_ptr[1:])
        out = np.full(int(new_ptr[-1]), np.uint32(nat.SRC_NULL << nat.SRC_SHIFT), dtype=np.uint32)
        owner = np.repeat(np.arange(num_rows, dtype=np.int64), counts)
        out[new_ptr[:-1][owner] + (np.arange(entries.size, dtype=np.int64) - row_ptr[:-1][owner])] = entries
        entries, row_ptr = out, new_ptr
        if row_ptr[-1] > np.iinfo(np.int32).max:
            raise ValueError(f"level {level} has {int(row_ptr[-1])} padded entries, above the 2^31-1 per-level limit")
    heavy = np.arange(num_rows - num_heavy, num_rows, dtype=np.int32)
    if slot_table is not None and slot_table.shape[0] > nat.MAX_SLOT_BUCKETS:
        slot_table = None  # more width classes than the kernels take: row_ptr is still exact
    return LevelGather(level, int(row_begin), int(num_rows), row_ptr.astype(np.int32), entries, heavy,
                       int(heavy_threshold), row_ids, 4 if pad else 1, slot_table)


def _finish_torch(level: int, row_begin: int, num_rows: int, rows: np.ndarray, ids: np.ndarray, src: np.ndarray,
                  group: np.ndarray, heavy_threshold: int, locality: bool = False, balance: bool = True,
                  pad: bool = False, long_first: bool = True, slots: bool = False, heavy_buckets: bool = False,
                  device="cuda") -> LevelGather:
    """``_finish`` with PyTorch on ``device`` (the GPU when the runtime builds its levels):
    the same steps as the NumPy version, in integer arithmetic only, so the lists, row
    pointers, processing order and slot tables are identical to it."""
    import torch

    dev = torch.device(device)
    i64 = torch.int64
    rows_t = torch.as_tensor(np.asarray(rows, dtype=np.int64)).to(dev)
    ids_t = torch.as_tensor(np.asarray(ids, dtype=np.int64)).to(dev)
    src_t = torch.as_tensor(np.asarray(src, dtype=np.int64)).to(dev)
    grp_t = torch.as_tensor(np.asarray(group, dtype=np.int64)).to(dev)
    n = int(num_rows)
    if rows_t.numel():
        order = torch.sort(rows_t, stable=True).indices
        rows_t, ids_t, src_t, grp_t = rows_t[order], ids_t[order], src_t[order], grp_t[order]
        if int(ids_t.max()) > nat.MAX_ID:
            raise ValueError(f"level {level} names ids above {nat.MAX_ID}, beyond the B200 backend's limit")
    counts = torch.bincount(rows_t, minlength=n) if rows_t.numel() else torch.zeros(n, dtype=i64, device=dev)
    row_ptr = torch.zeros(n + 1, dtype=i64, device=dev)
    row_ptr[1:] = torch.cumsum(counts, 0)
    if int(row_ptr[-1]) > np.iinfo(np.int32).max:
        raise ValueError(f"level {level} has {int(row_ptr[-1])} entries, above the 2^31-1 per-level limit")
    start = torch.ones(ids_t.numel(), dtype=torch.bool, device=dev)
    if ids_t.numel() > 1:
        start[1:] = (rows_t[1:] != rows_t[:-1]) | (grp_t[1:] != grp_t[:-1])
    entries = ids_t | (src_t << nat.SRC_SHIFT) | torch.where(start, nat.SEG_START, 0)
    perm = torch.arange(n, dtype=i64, device=dev)
    if locality and n > 1:
        key = torch.full((n,), np.iinfo(np.int64).max, dtype=i64, device=dev)
        state_pos = torch.nonzero(src_t == nat.SRC_STATE).flatten()
        if state_pos.numel():
            rs = rows_t[state_pos]
            change = torch.ones(rs.numel(), dtype=torch.bool, device=dev)
            change[:-1] = rs[1:] != rs[:-1]
            last = torch.nonzero(change).flatten()
            key[rs[last]] = ids_t[state_pos[last]]
        perm = torch.sort(key, stable=True).indices
    use_slots = slots and pad and balance
    pow2 = torch.as_tensor(_POW2, device=dev)

    def quad_class(c):
        quads = (c + 3) // 4
        width = torch.ones_like(quads)
        while bool((width < quads).any()):
            width = torch.where(width < quads, width * 2, width)
        return torch.where(quads == 0, torch.zeros_like(width), width)

    heavy_mask = counts[perm] > int(heavy_threshold)
    narrow_perm, heavy_perm = perm[~heavy_mask], perm[heavy_mask]
    if balance and narrow_perm.numel() > 1:
        c = counts[narrow_perm]
        bucket = quad_class(c) if use_slots else torch.searchsorted(pow2, c, right=True)
        narrow_perm = narrow_perm[torch.sort(-bucket if long_first else bucket, stable=True).indices]
    if balance and heavy_buckets and heavy_perm.numel() > 1:
        bucket = torch.searchsorted(pow2, counts[heavy_perm], right=True)
        heavy_perm = heavy_perm[torch.sort(-bucket if long_first else bucket, stable=True).indices]
    perm = torch.cat((narrow_perm, heavy_perm))
    num_heavy = int(heavy_perm.numel())
    row_ids = None
    if not torch.equal(perm, torch.arange(n, dtype=i64, device=dev)):
        lengths = counts[perm]
        new_ptr = torch.zeros(n + 1, dtype=i64, device=dev)
        new_ptr[1:] = torch.cumsum(lengths, 0)
        total = int(new_ptr[-1])
        gather = torch.repeat_interleave(row_ptr[:-1][perm] - new_ptr[:-1], lengths, output_size=total) + \
            torch.arange(total, dtype=i64, device=dev)
        entries = entries[gather]
        row_ptr, row_ids = new_ptr, perm
    counts = row_ptr[1:] - row_ptr[:-1]
    slot_table = None
    if pad:
        padded = (counts + 3) // 4 * 4
        if use_slots:
            narrow = n - num_heavy
            width = quad_class(counts[:narrow])
            padded = padded.clone()
            padded[:narrow] = 4 * width
            if narrow:
                change = torch.ones(narrow, dtype=torch.bool, device=dev)
                change[1:] = width[1:] != width[:-1]
                starts = torch.nonzero(change).flatten()
                first_entry = torch.zeros(narrow + 1, dtype=i64, device=dev)
                first_entry[1:] = torch.cumsum(padded[:narrow], 0)
                slot_table = torch.stack([starts, first_entry[starts], width[starts]], dim=1).cpu().numpy().astype(np.int64)
            else:
                slot_table = np.zeros((0, 3), dtype=np.int64)
        new_ptr = torch.zeros(n + 1, dtype=i64, device=dev)
        new_ptr[1:] = torch.cumsum(padded, 0)
        out = torch.full((int(new_ptr[-1]),), nat.SRC_NULL << nat.SRC_SHIFT, dtype=i64, device=dev)
        owner = torch.repeat_interleave(torch.arange(n, dtype=i64, device=dev), counts, output_size=entries.numel())
        out[new_ptr[:-1][owner] + (torch.arange(entries.numel(), dtype=i64, device=dev) - row_ptr[:-1][owner])] = entries
        entries, row_ptr = out, new_ptr
        if int(row_ptr[-1]) > np.iinfo(np.int32).max:
            raise ValueError(f"level {level} has {int(row_ptr[-1])} padded entries, above the 2^31-1 per-level limit")
    if slot_table is not None and slot_table.shape[0] > nat.MAX_SLOT_BUCKETS:
        slot_table = None
    heavy = np.arange(n - num_heavy, n, dtype=np.int32)
    return LevelGather(level, int(row_begin), n, row_ptr.to(torch.int32).cpu().numpy(),
                       entries.cpu().numpy().astype(np.uint32), heavy, int(heavy_threshold),
                       None if row_ids is None else row_ids.to(torch.int32).cpu().numpy(), 4 if pad else 1, slot_table)


def load_blocks(blocks) -> dict[tuple[int, int], tuple[np.ndarray, np.ndarray]]:
    """Canonical COO of every non-empty block, keyed by (dst level, src level)."""
    out = {}
    for block in blocks:
        if block.nnz == 0:
            continue
        out[(block.dst_level, block.src_level)] = canonical_coo(block.indices, block.indptr, block.shape)
    return out


def build_up_levels(level_offsets: np.ndarray, coo: dict, heavy_threshold: int, locality: bool = False,
                    balance: bool = True, pad: bool = False, long_first: bool = True, slots: bool = False,
                    device=None, heavy_buckets: bool = False) -> list[LevelGather]:
    """Gather lists for up levels 1..h-1 (level 0 is seeded from the input); built with
    PyTorch on ``device`` when given (identical results), else with NumPy."""
    finish = _finish if device is None else (lambda *a: _finish_torch(*a, device=device))
    off = np.asarray(level_offsets, dtype=np.int64)
    h = off.size - 1
    levels = []
    for dst in range(1, h):
        n = int(off[dst + 1] - off[dst])
        rows, ids, src = [], [], []
        for s in range(dst):
            if (dst, s) not in coo:
                continue
            r, c = coo[(dst, s)]
            rows.append(r)
            ids.append(c + off[s])
            src.append(np.full(r.size, s, dtype=np.int16))
        cat = (lambda parts, dt: np.concatenate(parts) if parts else np.empty(0, dtype=dt))
        r, i, g = cat(rows, np.int64), cat(ids, np.int64), cat(src, np.int16)
        levels.append(finish(dst, int(off[dst]), n, r, i, np.zeros(i.size, np.uint8), g, heavy_threshold, locality, balance, pad, long_first, slots, heavy_buckets))
    return levels


def _selector_by_node(ptr: np.ndarray, idx: np.ndarray, num_rows: int) -> tuple[np.ndarray, np.ndarray]:
    """(node, mutation) pairs of a selector sorted by node, ascending mutation inside a node."""
    ptr = np.asarray(ptr, dtype=np.int64)
    muts = np.repeat(np.arange(num_rows, dtype=np.int64), np.diff(ptr))
    nodes = np.asarray(idx, dtype=np.int64)
    order = _stable_argsort(nodes)
    return nodes[order], muts[order]


def build_down_levels(level_offsets: np.ndarray, coo: dict, sel_mut, sel_miss, heavy_threshold: int,
                      locality: bool = True, balance: bool = True, pad: bool = False,
                      long_first: bool = True, slots: bool = False, device=None,
                      heavy_buckets: bool = False) -> list[LevelGather]:
    """Gather lists for down levels h-1..0 in execution order (PyTorch on ``device`` when
    given, identical results).

    ``sel_mut``/``sel_miss`` are (indptr, indices, num_mutations) triples; ``sel_miss`` may be
    None when no miss input is needed.
    """
    finish = _finish if device is None else (lambda *a: _finish_torch(*a, device=device))
    off = np.asarray(level_offsets, dtype=np.int64)
    h = off.size - 1
    mut_nodes, mut_ids = _selector_by_node(sel_mut[0], sel_mut[1], sel_mut[2])
    miss_nodes, miss_ids = (None, None) if sel_miss is None else _selector_by_node(sel_miss[0], sel_miss[1], sel_miss[2])
    levels = []
    for dst in range(h - 1, -1, -1):
        lo, hi = int(off[dst]), int(off[dst + 1])
        rows, ids, src, grp = [], [], [], []
        for nodes, mids, code, g in ((mut_nodes, mut_ids, nat.SRC_INPUT, 0), (miss_nodes, miss_ids, nat.SRC_MISS, 1)):
            if nodes is None:
                continue
            a, b = np.searchsorted(nodes, [lo, hi])
            rows.append(nodes[a:b] - lo)
            ids.append(mids[a:b])
            src.append(np.full(b - a, code, dtype=np.uint8))
            grp.append(np.full(b - a, g, dtype=np.int16))
        for s in range(h - 1, dst, -1):
            if (s, dst) not in coo:
                continue
            p, c = coo[(s, dst)]  # rows: parents (level s), cols: children (level dst)
            # canonical COO is sorted by parent, so the stable sort by row in _finish already
            # leaves each child's parents of this block in ascending order
            rows.append(c)
            ids.append(p + off[s])
            src.append(np.zeros(p.size, dtype=np.uint8))
            grp.append(np.full(p.size, 2 + (h - 1 - s), dtype=np.int16))
        cat = (lambda parts, dt: np.concatenate(parts) if parts else np.empty(0, dtype=dt))
        levels.append(finish(dst, lo, hi - lo, cat(rows, np.int64), cat(ids, np.int64), cat(src, np.uint8),
                              cat(grp, np.int16), heavy_threshold, locality, balance, pad, long_first, slots,
                              heavy_buckets))
    return levels


def _padded_bound(total: int, rows: int, pad: bool, slots: bool) -> int:
    """Entries after padding: multiples of 4 add < 4 per row; slot widths at most double a
    padded narrow list (+4 per row covers the rounding)."""
    if not pad:
        return int(total)
    if slots:
        return int(2 * total + 4 * rows)
    return int(total + 3 * rows)


def up_entry_bound(scan, level: int, pad: bool = False, slots: bool = False) -> int:
    total = sum(b.nnz for b in scan.blocks if b.dst_level == level)
    return _padded_bound(total, int(scan.level_sizes[level]), pad, slots)


def down_entry_bound(scan, level: int, with_miss: bool, pad: bool = False, slots: bool = False) -> int:
    total = sum(b.nnz for b in scan.blocks if b.src_level == level)
    total += int(scan.selector_nnz_by_level[level, 0])
    if with_miss:
        total += int(scan.selector_nnz_by_level[level, 1])
    return _padded_bound(total, int(scan.level_sizes[level]), pad, slots)


__all__ = [
    "LevelGather",
    "blob_layout",
    "build_down_levels",
    "build_up_levels",
    "canonical_coo",
    "down_entry_bound",
    "load_blocks",
    "up_entry_bound",
]
