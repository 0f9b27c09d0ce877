"""The .grg_spmv v8 format: reading reference-written files, writing, validation."""

from __future__ import annotations

from pathlib import Path
import zipfile

import numpy as np
import pytest

from conftest import artifact_path
from grg_spmv_b200 import artifact as art
from grg_spmv_b200.artifact import (GRG_SPMV_FORMAT_MAGIC, GRG_SPMV_FORMAT_VERSION, iter_artifact_blocks, load_grg_spmv,
                                    save_grg_spmv, scan_grg_spmv)

NAMES = ("band3", "overlap4", "synth_haploid", "synth_diploid", "synth_repeat", "sparse_selector")


@pytest.mark.parametrize("name", NAMES)
def test_scan_matches_loaded_reference_artifact(name):
    path = artifact_path(name)
    scan = scan_grg_spmv(path)
    state = load_grg_spmv(path, np.float64)
    assert scan.num_nodes == state.num_nodes and scan.num_samples == state.num_samples
    assert scan.num_mutations == state.num_mutations and scan.num_edges == state.num_edges
    np.testing.assert_array_equal(scan.level_offsets, state.level_offsets)
    assert scan.selector_mut_nnz == state.sel_mut.nnz and scan.selector_miss_nnz == state.sel_miss.nnz
    assert scan.has_individual_coals == (state.coalescence_counts is not None)
    blocks = {(b.dst_level, b.src_level): b for b in iter_artifact_blocks(path)}
    assert len(blocks) == len(scan.blocks)
    for b in scan.blocks:
        loaded = state.A_blocks[b.dst_level][b.src_level]
        assert loaded.shape == b.shape and loaded.nnz == b.nnz
        assert blocks[(b.dst_level, b.src_level)].indices.dtype == b.indices_dtype


@pytest.mark.parametrize("name", NAMES)
def test_round_trip_is_array_identical(name, tmp_path):
    src = artifact_path(name)
    state = load_grg_spmv(src, np.float64)
    out = tmp_path / f"{name}.grg_spmv"
    save_grg_spmv(state, out)
    with np.load(src) as a, np.load(out) as b:
        assert set(a.files) == set(b.files)
        for key in a.files:
            assert a[key].dtype == b[key].dtype, key
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    with zipfile.ZipFile(out) as zf:
        assert {i.compress_type for i in zf.infolist()} == {zipfile.ZIP_STORED}


@pytest.mark.parametrize("version", [5, 6, 7, 9])
def test_other_versions_are_rejected(tmp_path, version):
    path = tmp_path / "old.grg_spmv"
    with path.open("wb") as handle:
        np.savez(handle, grg_spmv_magic=np.asarray(GRG_SPMV_FORMAT_MAGIC), grg_spmv_format_version=np.asarray(version, np.int32))
    with pytest.raises(ValueError, match=f"got version {version}, expected {GRG_SPMV_FORMAT_VERSION}"):
        scan_grg_spmv(path)


def test_bad_magic_is_rejected(tmp_path):
    path = tmp_path / "bad.grg_spmv"
    with path.open("wb") as handle:
        np.savez(handle, grg_spmv_magic=np.asarray("other"), grg_spmv_format_version=np.asarray(8, np.int32))
    with pytest.raises(ValueError, match="got magic"):
        scan_grg_spmv(path)


def test_save_is_atomic_on_failure(tmp_path, monkeypatch):
    state = load_grg_spmv(artifact_path("band3"), np.float64)
    target = tmp_path / "band3.grg_spmv"
    target.write_bytes(artifact_path("band3").read_bytes())
    before = target.read_bytes()

    def broken(handle, *a, **k):
        handle.write(b"partial")
        raise RuntimeError("save failed")

    monkeypatch.setattr(np, "savez", broken)
    with pytest.raises(RuntimeError, match="save failed"):
        save_grg_spmv(state, target)
    assert target.read_bytes() == before
    assert not list(tmp_path.glob(".band3.grg_spmv.*.tmp"))


def test_scan_reads_metadata_only(monkeypatch, tmp_path):
    path = tmp_path / "scan.grg_spmv"
    path.write_bytes(artifact_path("band3").read_bytes())
    real = art._struct

    def guarded(data, key):
        if key != "level_offsets":
            raise AssertionError(f"scan loaded structural array {key}")
        return real(data, key)

    art._scan_cached.cache_clear()
    monkeypatch.setattr(art, "_struct", guarded)
    scan = scan_grg_spmv(path)
    assert scan.num_levels == 3
    assert [(b.dst_level, b.src_level, b.nnz) for b in scan.blocks] == [(1, 0, 512), (2, 0, 512), (2, 1, 512)]
