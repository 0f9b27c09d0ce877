"""The planner's budget semantics (metadata only, no GPU)."""

from __future__ import annotations

import warnings

import numpy as np
import pytest

from conftest import artifact_path
from grg_spmv_b200 import RuntimeRequirements, scan_grg_spmv
from grg_spmv_b200.backends.b200.plan import B200Plan, B200PlanPair, plan_layout_from_scans
from grg_spmv_b200.types import Direction


def _req(k=2, **kw):
    base = dict(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=True, need_init_vector=True,
                need_init_matrix=True, need_init_xtx=True)
    base.update(kw)
    return RuntimeRequirements(**base)


def _plan(names=("band3",), *, budget=0, ring=0, allow=True, pair=None, req=None, dtype=np.float64, precision="plain",
          emit_all_nodes=True):
    paths = tuple(artifact_path(n) for n in names)
    return plan_layout_from_scans(scans=tuple(scan_grg_spmv(p) for p in paths), paths=paths, dtype=dtype,
                                  requirements=req or _req(), requested_budget=budget, requested_ring=ring,
                                  allow_residency=allow, device_id=0, stream_ptr=0, stream_owner=None,
                                  pair=pair or B200PlanPair(), precision=precision, emit_all_nodes=emit_all_nodes)


def _keys(layout, resident: bool):
    return sorted((lp.direction.value, lp.level) for lp in layout.level_plans() if lp.resident == resident)


def test_budget_zero_means_full_residency():
    layout = _plan()
    assert _keys(layout, False) == []
    assert layout.allocated_ring_buffer_size == 0
    assert layout.vram_budget_bytes == layout.required_budget_for_full_residency == layout.bytes_total
    assert sum(i.nbytes for i in layout.budget_items) == layout.bytes_total
    # band3: up levels 1, 2; down levels 2, 1, 0
    assert _keys(layout, True) == [("down", 0), ("down", 1), ("down", 2), ("up", 1), ("up", 2)]


def test_lean_layout_drops_the_all_node_buffer():
    full = _plan(names=("synth_haploid",), req=_req(k=3))
    lean = _plan(names=("synth_haploid",), req=_req(k=3), emit_all_nodes=False)
    scan = scan_grg_spmv(artifact_path("synth_haploid"))
    assert full.emit_all_nodes and not lean.emit_all_nodes
    assert full.bytes_total - lean.bytes_total == scan.num_nodes * 3 * 8
    assert full.bytes_by_category["dense_arena"] - lean.bytes_by_category["dense_arena"] == scan.num_nodes * 3 * 8
    # the bytes saved go to level lists: a budget that streams levels in the full layout keeps them all resident
    assert _keys(_plan(names=("synth_haploid",), req=_req(k=3), emit_all_nodes=False, budget=lean.bytes_total, ring=1),
                 False) == []


def test_ring_request_with_full_residency_warns():
    with pytest.warns(RuntimeWarning, match="requested ring_buffer_size=2"):
        layout = _plan(ring=2)
    assert layout.allocated_ring_buffer_size == 0


def test_tight_budget_streams_and_promotes_largest_first():
    full = _plan()
    fixed = full.bytes_total - full.bytes_by_category["resident_sparse"]
    sizes = sorted((lp.nbytes for lp in full.level_plans()), reverse=True)
    # Room for the fixed part, one slot of the largest level and the largest level resident.
    budget = fixed + sizes[0] + sizes[0]
    layout = _plan(budget=budget, ring=1)
    assert layout.allocated_ring_buffer_size == 1
    assert layout.bytes_total <= budget < layout.required_budget_for_full_residency
    resident = [lp for lp in layout.level_plans() if lp.resident]
    assert resident and max(lp.nbytes for lp in resident) == sizes[0]
    assert all(lp.slot == 0 for lp in layout.level_plans() if not lp.resident)
    with pytest.raises(ValueError):
        _plan(budget=fixed + sizes[0] - 1, ring=1)


def test_streaming_requires_a_ring():
    full = _plan()
    with pytest.raises(ValueError, match="ring_buffer_size must be >= 1"):
        _plan(budget=full.bytes_total - 1, ring=0)
    with pytest.raises(ValueError, match="ring_buffer_size must be >= 1"):
        _plan(allow=False, ring=0)


def test_allow_residency_false_streams_everything_round_robin():
    layout = _plan(allow=False, ring=2)
    assert _keys(layout, True) == []
    assert layout.allocated_ring_buffer_size == 2
    assert layout.bytes_by_category["resident_sparse"] == 0
    up = [lp.slot for lp in layout.artifacts[0].levels_up]
    assert up == [0, 1]
    with pytest.warns(RuntimeWarning, match="only 5 ring slot"):
        _plan(allow=False, ring=9)


def test_one_sided_layout_drops_the_other_direction():
    both = _plan()
    up_only = _plan(pair=B200PlanPair(plan_up=B200Plan(), plan_down=None))
    assert up_only.bytes_total < both.bytes_total
    assert all(lp.direction == Direction.UP for lp in up_only.level_plans())
    hostile = _plan(pair=B200PlanPair(plan_up=B200Plan(), plan_down=None), req=_req(k=2, max_k_down=1024))
    assert hostile.bytes_total == up_only.bytes_total


def test_plan_options_validate():
    with pytest.raises(ValueError):
        B200Plan(heavy_threshold=0)
    with pytest.raises(ValueError):
        B200Plan(row_order="random")
    with pytest.raises(ValueError):
        B200Plan.from_dict({"exact_order": True, "bogus": 1})
    with pytest.raises(ValueError):
        B200PlanPair(plan_up=None, plan_down=None)
    with pytest.raises(ValueError):
        B200Plan(heavy_variant=4)
    assert B200Plan.from_dict({"heavy_variant": 1}).heavy_variant == 1
    assert B200Plan().locality(Direction.DOWN) and not B200Plan().locality(Direction.UP)


def test_float32_halves_dense_bytes():
    f64 = _plan()
    f32 = _plan(dtype=np.float32)
    assert f32.bytes_by_category["state"] * 2 == f64.bytes_by_category["state"]
    assert f32.bytes_by_category["resident_sparse"] == f64.bytes_by_category["resident_sparse"]


def test_mixed_precision_state_and_scratch_bytes():
    from grg_spmv_b200.backends.b200 import _native as nat

    req = _req()
    f64 = _plan(req=req)
    mixed = _plan(req=req, precision="mixed")
    k = max(req.max_k_up, req.max_k_down)
    assert mixed.precision == "mixed" and f64.precision == "plain"
    assert mixed.bytes_by_category["state"] == nat.mix_bytes(mixed.max_num_nodes, nat.mix_ld(k))
    assert mixed.mix_scratch_bytes == nat.mix_bytes(mixed.max_num_mutations, nat.mix_ld(k)) * (2 if req.need_down_miss_input else 1)
    assert mixed.bytes_by_category["scratch"] == 256 + mixed.mix_scratch_bytes
    assert mixed.bytes_by_category["resident_sparse"] == f64.bytes_by_category["resident_sparse"]


def test_mixed_precision_rejects_incompatible_options():
    with pytest.raises(ValueError, match="precision"):
        _plan(precision="half")
    with pytest.raises(ValueError, match="float64"):
        _plan(dtype=np.float32, precision="mixed")
    with pytest.raises(ValueError, match="exact_order"):
        _plan(precision="mixed", pair=B200PlanPair(plan_up=B200Plan(exact_order=True)))
    with pytest.raises(ValueError, match="pad_lists"):
        _plan(precision="mixed", pair=B200PlanPair(plan_down=B200Plan(pad_lists=False, narrow_variant=5)))


@pytest.mark.parametrize("heavy", [1, 2, 128])
@pytest.mark.parametrize("name", ["band3", "overlap4", "synth_haploid", "synth_diploid", "synth_repeat", "sparse_selector"])
@pytest.mark.parametrize("slots", [False, True])
def test_planned_bytes_bound_the_built_level_blobs(name, heavy, slots):
    """Every level blob the runtime builds fits the bytes the planner budgeted for it."""
    from grg_spmv_b200.artifact import iter_artifact_blocks, load_grg_spmv_header
    from grg_spmv_b200.backends.b200.structures import build_down_levels, build_up_levels, load_blocks

    pair = B200PlanPair(plan_up=B200Plan(heavy_threshold=heavy, slots=slots), plan_down=B200Plan(heavy_threshold=heavy, slots=slots))
    layout = _plan((name,), pair=pair)
    st = load_grg_spmv_header(artifact_path(name), np.float64)
    coo = load_blocks(iter_artifact_blocks(artifact_path(name)))
    up = {lv.level: lv for lv in build_up_levels(st.level_offsets, coo, heavy, False, True, True, slots=slots)}
    down = {lv.level: lv for lv in build_down_levels(st.level_offsets, coo, (st.sel_mut.indptr, st.sel_mut.indices, st.num_mutations),
                                                     (st.sel_miss.indptr, st.sel_miss.indices, st.num_mutations), heavy, True, True, True,
                                                     slots=slots)}
    for lp in layout.artifacts[0].levels_up:
        assert up[lp.level].layout()[4] <= lp.nbytes
    for lp in layout.artifacts[0].levels_down:
        assert down[lp.level].layout()[4] <= lp.nbytes
    for lv in list(up.values()) + list(down.values()):
        if not slots:
            assert lv.slots is None
            continue
        # the slot table locates every narrow list exactly where row_ptr does
        narrow = lv.num_rows - lv.heavy_rows.size
        assert lv.slots is not None and lv.slots.shape[0] <= 8
        bounds = list(lv.slots[:, 0]) + [narrow]
        for b, (pos0, entry0, width) in enumerate(lv.slots):
            pos = np.arange(pos0, bounds[b + 1])
            np.testing.assert_array_equal(lv.row_ptr[pos], entry0 + (pos - pos0) * 4 * width)
            np.testing.assert_array_equal(lv.row_ptr[pos + 1] - lv.row_ptr[pos], 4 * width)
            assert b == 0 or width < lv.slots[b - 1, 2]  # longest bucket first


def test_programmatic_dependent_launch_defaults_on_from_k8():
    assert not B200Plan().resolve_pdl(1) and not B200Plan().resolve_pdl(7)
    assert B200Plan().resolve_pdl(8) and B200Plan().resolve_pdl(64)
    assert B200Plan(pdl=False).resolve_pdl(64) is False and B200Plan(pdl=True).resolve_pdl(1) is True
    assert B200Plan.from_dict({}).pdl is None and B200Plan.from_dict({"pdl": True}).pdl is True


def test_kernel_shape_options_validate_and_round_trip():
    with pytest.raises(ValueError, match="persist_ctas"):
        B200Plan(persist_ctas=-1)
    with pytest.raises(ValueError, match="fuse_entries"):
        B200Plan(fuse_entries=-5)
    with pytest.raises(ValueError, match="narrow_variant"):
        B200Plan(narrow_variant=17)
    with pytest.raises(ValueError, match="padded"):
        B200Plan(narrow_variant=9, pad_lists=False)
    plan = B200Plan.from_dict({"narrow_variant": 10, "persist_ctas": 3, "fuse_entries": 600_000, "pdl": False})
    assert (plan.narrow_variant, plan.persist_ctas, plan.fuse_entries, plan.pdl) == (10, 3, 600_000, False)
    with pytest.raises(ValueError, match="unknown B200Plan field"):
        B200Plan.from_dict({"fuse": 1})
    assert (B200Plan().heavy_buckets, B200Plan().short_rows) == (False, True)
    plan = B200Plan.from_dict({"heavy_buckets": True, "short_rows": False})
    assert (plan.heavy_buckets, plan.short_rows) == (True, False)
