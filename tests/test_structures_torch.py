"""The PyTorch level builder (used on the GPU by the runtime) produces exactly the NumPy
builder's lists: same processing order, row pointers, entries, row maps and slot tables."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import artifact_path

torch = pytest.importorskip("torch")

NAMES = ["band3", "overlap4", "synth_haploid", "synth_diploid", "synth_repeat", "sparse_selector"]


def _same(a, b):
    assert (a.level, a.row_begin, a.num_rows, a.heavy_threshold, a.list_align) == (b.level, b.row_begin, b.num_rows,
                                                                                   b.heavy_threshold, b.list_align)
    np.testing.assert_array_equal(a.row_ptr, b.row_ptr)
    np.testing.assert_array_equal(a.entries, b.entries)
    np.testing.assert_array_equal(a.heavy_rows, b.heavy_rows)
    assert (a.row_ids is None) == (b.row_ids is None)
    if a.row_ids is not None:
        np.testing.assert_array_equal(a.row_ids, b.row_ids)
    assert (a.slots is None) == (b.slots is None)
    if a.slots is not None:
        np.testing.assert_array_equal(a.slots, b.slots)
    assert a.row_ptr.dtype == b.row_ptr.dtype and a.entries.dtype == b.entries.dtype


@pytest.mark.parametrize("opts", [dict(heavy=2, pad=True, slots=False, long_first=True),
                                  dict(heavy=2, pad=True, slots=False, long_first=True, heavy_buckets=True),
                                  dict(heavy=128, pad=True, slots=True, long_first=True),
                                  dict(heavy=3, pad=False, slots=False, long_first=False),
                                  dict(heavy=3, pad=False, slots=False, long_first=False, heavy_buckets=True),
                                  dict(heavy=6, pad=True, slots=True, long_first=False)],
                         ids=["pad", "pad-heavy-buckets", "slots", "plain", "plain-heavy-buckets", "slots-short"])
@pytest.mark.parametrize("name", NAMES)
def test_torch_builder_matches_numpy(name, opts):
    from grg_spmv_b200.artifact import iter_artifact_blocks, load_grg_spmv_header
    from grg_spmv_b200.backends.b200.structures import build_down_levels, build_up_levels, load_blocks

    st = load_grg_spmv_header(artifact_path(name), np.float64)
    coo = load_blocks(iter_artifact_blocks(artifact_path(name)))
    kw = dict(pad=opts["pad"], long_first=opts["long_first"], slots=opts["slots"], heavy_buckets=opts.get("heavy_buckets", False))
    for locality in (False, True):
        a = build_up_levels(st.level_offsets, coo, opts["heavy"], locality, True, **kw)
        b = build_up_levels(st.level_offsets, coo, opts["heavy"], locality, True, device="cpu", **kw)
        assert len(a) == len(b)
        for x, y in zip(a, b):
            _same(x, y)
        sel = (st.sel_mut.indptr, st.sel_mut.indices, st.num_mutations)
        miss = (st.sel_miss.indptr, st.sel_miss.indices, st.num_mutations)
        a = build_down_levels(st.level_offsets, coo, sel, miss, opts["heavy"], locality, True, **kw)
        b = build_down_levels(st.level_offsets, coo, sel, miss, opts["heavy"], locality, True, device="cpu", **kw)
        assert len(a) == len(b)
        for x, y in zip(a, b):
            _same(x, y)


def test_torch_builder_matches_numpy_on_a_larger_synthetic_graph(tmp_path):
    from grg_spmv_b200.artifact import iter_artifact_blocks, load_grg_spmv_header
    from grg_spmv_b200.backends.b200.structures import build_down_levels, build_up_levels, load_blocks
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    path = tmp_path / "g.grg_spmv"
    write_synthetic_artifact(SynthSpec(num_samples=3000, num_levels=14, num_nodes=60_000, num_mutations=15_000, children=(2, 16),
                                       miss_fraction=0.02, random_ids=True, seed=3), path)
    st = load_grg_spmv_header(path, np.float64)
    coo = load_blocks(iter_artifact_blocks(path))
    for x, y in zip(build_up_levels(st.level_offsets, coo, 32, False, True, True),
                    build_up_levels(st.level_offsets, coo, 32, False, True, True, device="cpu")):
        _same(x, y)
    sel = (st.sel_mut.indptr, st.sel_mut.indices, st.num_mutations)
    miss = (st.sel_miss.indptr, st.sel_miss.indices, st.num_mutations)
    for x, y in zip(build_down_levels(st.level_offsets, coo, sel, miss, 32, True, True, True),
                    build_down_levels(st.level_offsets, coo, sel, miss, 32, True, True, True, device="cpu")):
        _same(x, y)


@pytest.mark.gpu
def test_gpu_builder_matches_numpy():
    """The runtime builds its levels on the GPU; those lists equal the NumPy builder's."""
    from grg_spmv_b200.artifact import iter_artifact_blocks, load_grg_spmv_header
    from grg_spmv_b200.backends.b200.structures import build_down_levels, build_up_levels, load_blocks

    for name in NAMES:
        st = load_grg_spmv_header(artifact_path(name), np.float64)
        coo = load_blocks(iter_artifact_blocks(artifact_path(name)))
        for x, y in zip(build_up_levels(st.level_offsets, coo, 2, False, True, True),
                        build_up_levels(st.level_offsets, coo, 2, False, True, True, device="cuda")):
            _same(x, y)
        sel = (st.sel_mut.indptr, st.sel_mut.indices, st.num_mutations)
        miss = (st.sel_miss.indptr, st.sel_miss.indices, st.num_mutations)
        for x, y in zip(build_down_levels(st.level_offsets, coo, sel, miss, 2, True, True, True, slots=True),
                        build_down_levels(st.level_offsets, coo, sel, miss, 2, True, True, True, slots=True, device="cuda")):
            _same(x, y)


def test_heavy_rows_keep_row_order_unless_bucketed():
    """Heavy rows (the suffix) stay in row order by default and are grouped by length only with
    ``heavy_buckets``; narrow rows are grouped by length either way."""
    from grg_spmv_b200.backends.b200.structures import _finish

    # row r has lengths[r] entries; threshold 4: rows 1, 3, 4 are heavy
    lengths = np.asarray([2, 9, 1, 5, 20, 3])
    rows = np.repeat(np.arange(lengths.size), lengths)
    ids = np.arange(rows.size)
    z = np.zeros(rows.size, dtype=np.int64)
    plain = _finish(0, 0, lengths.size, rows, ids, z, z, 4)
    assert list(plain.row_ids[-3:]) == [1, 3, 4]
    assert list(plain.row_ids[:3]) == [0, 5, 2]  # narrow: 2 and 3 entries (bucket 2) in row order, then 1 entry
    grouped = _finish(0, 0, lengths.size, rows, ids, z, z, 4, heavy_buckets=True)
    assert list(grouped.row_ids[-3:]) == [4, 1, 3]  # 20 entries (bucket 5), then 9 and 5 (bucket 4) in row order


def test_short_rows_is_the_suffix_of_one_quad_lists():
    """``short_rows``: the narrow positions at the end of the narrow range whose padded lists
    hold at most one quad; with long-first bucketing, at least every narrow row of at most 3
    entries."""
    from grg_spmv_b200.backends.b200.structures import _finish

    # threshold 8: row 5 (12 entries) is heavy; narrow lengths 4, 7 (bucket 3), 2, 3 (bucket 2),
    # 1 (bucket 1), 0
    lengths = np.asarray([2, 7, 0, 4, 1, 12, 3])
    rows = np.repeat(np.arange(lengths.size), lengths)
    ids = np.arange(rows.size)
    z = np.zeros(rows.size, dtype=np.int64)
    lv = _finish(0, 0, lengths.size, rows, ids, z, z, 8, pad=True)
    assert list(lv.row_ids) == [1, 3, 0, 6, 4, 2, 5]
    assert lv.short_rows() == 5  # rows 3 (4 entries: one quad, after its bucket's 7), 0, 6, 4, 2
    assert _finish(0, 0, lengths.size, rows, ids, z, z, 8, pad=False).short_rows() == 0  # unpadded
    # short-first order: the last bucket holds rows 1 (7 entries) and 3 (4), in row order
    assert _finish(0, 0, lengths.size, rows, ids, z, z, 8, pad=True, long_first=False).short_rows() == 1
    # every narrow row short; at threshold 0 only the empty row stays narrow
    one = np.asarray([1, 2, 3, 0])
    r1 = np.repeat(np.arange(one.size), one)
    z1 = np.zeros(r1.size, dtype=np.int64)
    assert _finish(0, 0, one.size, r1, np.arange(r1.size), z1, z1, 8, pad=True).short_rows() == 4
    assert _finish(0, 0, one.size, r1, np.arange(r1.size), z1, z1, 0, pad=True).short_rows() == 1
