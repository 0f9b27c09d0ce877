"""BoundGRG / RuntimeRequirements / spec semantics, with a fake runtime (no GPU)."""

from __future__ import annotations

from contextlib import contextmanager
import json
import subprocess
import sys
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import REPO, artifact_path
from grg_spmv_b200 import BoundGRG, RuntimeRequirements
from grg_spmv_b200.artifact import load_grg_spmv_header
from grg_spmv_b200.types import Direction, InitMode, parse_direction


class _FakeRuntime:
    def __init__(self, requirements, cuda=True):
        self.layout = SimpleNamespace(requirements=requirements, dtype=np.float64)
        self.specs = []
        self.active = False
        if cuda:
            self._prepare_matmul_cuda = lambda grg, spec: self.specs.append(spec) or spec

    @contextmanager
    def _call_scope(self):
        if self.active:
            raise RuntimeError("concurrent runtime.grgs calls are not supported")
        self.active = True
        try:
            yield
        finally:
            self.active = False


def _req(**kw):
    base = dict(max_k_up=4, max_k_down=4, need_down_miss_input=True, need_up_miss_output=True, need_init_vector=True,
                need_init_matrix=True, need_init_xtx=True)
    base.update(kw)
    return RuntimeRequirements(**base)


def _grg(name="synth_diploid", **req):
    rt = _FakeRuntime(_req(**req))
    state = load_grg_spmv_header(artifact_path(name), np.float64)
    return BoundGRG(rt, 0, state, artifact_path(name), 0), rt


def test_requirements_validate_k():
    with pytest.raises(ValueError, match="max_k_up"):
        RuntimeRequirements(0, 1, False, False, False, False, False)
    with pytest.raises(ValueError, match="max_k_down"):
        RuntimeRequirements(1, 0, False, False, False, False, False)


def test_spec_widths_and_backend_init():
    grg, rt = _grg()
    spec = grg.prepare_matmul_cuda(direction="up", k=2, by_individual=True)
    assert (spec.input_cols, spec.output_cols) == (grg.num_individuals, grg.num_mutations)
    spec = grg.prepare_matmul_cuda(direction="down", k=2, by_individual=True, init_mode="vector")
    assert (spec.input_cols, spec.output_cols) == (grg.num_mutations, grg.num_individuals)
    assert spec.backend_init_mode == InitMode.NONE and spec.apply_endpoint_bias
    spec = grg.prepare_matmul_cuda(direction="down", k=2, init_mode="xtx", emit_all_nodes=True)
    assert spec.backend_init_mode == InitMode.XTX and not spec.apply_endpoint_bias and spec.output_cols == grg.num_nodes
    spec = grg.prepare_matmul_cuda(direction="up", k=2, init_mode="matrix")
    assert spec.backend_init_mode == InitMode.MATRIX and not spec.apply_endpoint_bias


def test_requirements_fail_fast_like_the_reference():
    grg, _ = _grg(max_k_up=1, max_k_down=1, need_down_miss_input=False, need_up_miss_output=False, need_init_vector=False,
                  need_init_matrix=False, need_init_xtx=False)
    with pytest.raises(ValueError, match="max_k_up"):
        grg.prepare_matmul_cuda(direction="up", k=2)
    with pytest.raises(ValueError, match="UP miss output"):
        grg.prepare_matmul_cuda(direction="up", k=1, use_miss=True)
    with pytest.raises(ValueError, match="DOWN miss input"):
        grg.prepare_matmul_cuda(direction="down", k=1, use_miss=True)
    with pytest.raises(ValueError, match="init vector"):
        grg.prepare_matmul_cuda(direction="up", k=1, init_mode="vector")
    with pytest.raises(ValueError, match="init matrix"):
        grg.prepare_matmul_cuda(direction="up", k=1, init_mode="matrix")
    with pytest.raises(ValueError, match="xtx"):
        grg.prepare_matmul_cuda(direction="up", k=1, init_mode="xtx")


def test_mode_conflicts():
    grg, _ = _grg()
    with pytest.raises(RuntimeError, match="cannot be mixed"):
        grg.prepare_matmul_cuda(direction="up", k=1, emit_all_nodes=True, use_miss=True)
    with pytest.raises(ValueError, match="cannot be mixed"):
        grg.prepare_matmul_cuda(direction="down", k=1, init_mode="vector", use_miss=True)
    nocoal, _ = _grg("band3")
    with pytest.raises(ValueError, match="coalescence"):
        nocoal.prepare_matmul_cuda(direction="up", k=1, init_mode="xtx")
    with pytest.raises(ValueError, match="k must be >= 1"):
        grg.prepare_matmul_cuda(direction="up", k=0)


def test_matmul_input_validation_messages():
    grg, _ = _grg()
    x = np.ones((1, grg.num_samples))
    with pytest.raises(TypeError, match="numpy.ndarray"):
        grg.matmul(x.tolist(), "up")
    with pytest.raises(ValueError, match="two-dimensional"):
        grg.matmul(np.ones(grg.num_samples), "up")
    with pytest.raises(ValueError, match="non-zero"):
        grg.matmul(np.ones((0, grg.num_samples)), "up")
    with pytest.raises(ValueError, match="UP direction"):
        grg.matmul(np.ones((1, 3)), "up")
    with pytest.raises(ValueError, match="DOWN direction"):
        grg.matmul(np.ones((1, 3)), "down")
    with pytest.raises(RuntimeError, match="cannot be mixed"):
        grg.matmul(x, "up", emit_all_nodes=True, miss=np.zeros((1, grg.num_mutations)))
    with pytest.raises(ValueError, match="cannot be mixed"):
        grg.matmul(x, "up", init=np.ones(1), miss=np.zeros((1, grg.num_mutations)))
    with pytest.raises(TypeError, match="dtype"):
        grg.matmul(x, "up", init=np.ones(1, dtype=np.float32))
    with pytest.raises(ValueError, match="dimensions"):
        grg.matmul(x, "up", init=np.ones((1, 3)))


def test_cpu_runtime_rejects_prepare():
    rt = _FakeRuntime(_req(), cuda=False)
    grg = BoundGRG(rt, 0, load_grg_spmv_header(artifact_path("band3"), np.float64), artifact_path("band3"))
    with pytest.raises(NotImplementedError):
        grg.prepare_matmul_cuda(direction="up", k=1)


def test_metadata_and_mutation_records():
    grg, _ = _grg()
    assert grg.shape == (grg.num_samples, grg.num_mutations)
    np.testing.assert_array_equal(grg.sample_to_individual, np.arange(grg.num_samples) // grg.ploidy)
    m = grg.get_mutation_by_id(3)
    assert (m.position, m.allele, m.ref_allele, m.time) == (30.5, "T", "C", 3.0)
    with pytest.raises(IndexError):
        grg.get_mutation_by_id(grg.num_mutations)


def test_direction_parsing_accepts_enum_members_by_name():
    class TraversalDirection:
        UP = SimpleNamespace(name="UP")
        DOWN = SimpleNamespace(name="DOWN")

    assert parse_direction(TraversalDirection.UP) == Direction.UP
    assert parse_direction("DOWN") == Direction.DOWN
    with pytest.raises(ValueError):
        parse_direction("sideways")


def test_root_import_is_cpu_safe():
    script = (
        "import importlib.abc, json, sys\n"
        "class B(importlib.abc.MetaPathFinder):\n"
        "    def find_spec(self, name, path=None, target=None):\n"
        "        if name.split('.')[0] in ('torch', 'triton', 'cupy'):\n"
        "            raise ModuleNotFoundError(name)\n"
        "sys.meta_path.insert(0, B())\n"
        f"sys.path.insert(0, {str(REPO)!r})\n"
        "import grg_spmv_b200, grg_spmv_b200.backends\n"
        "print(json.dumps({'runtime': hasattr(grg_spmv_b200, 'B200Runtime')}))\n"
    )
    out = subprocess.run([sys.executable, "-c", script], check=True, capture_output=True, text=True).stdout
    assert json.loads(out) == {"runtime": False}


def test_capture_spec_validation_mirrors_the_reference():
    from grg_spmv_b200 import RuntimeRequirements
    from grg_spmv_b200.adaptor import CaptureSpec, validate_capture_spec

    req = RuntimeRequirements(max_k_up=4, max_k_down=4, need_down_miss_input=False, need_up_miss_output=False,
                              need_init_vector=False, need_init_matrix=True, need_init_xtx=False)
    validate_capture_spec(CaptureSpec("up", 4), req)
    validate_capture_spec(CaptureSpec("down", 4, init_mode="matrix"), req)
    for spec, msg in ((CaptureSpec("up", 4, init_mode="bogus"), "invalid"),
                      (CaptureSpec("up", 4, init_mode="matrix", use_miss=True), "mutually exclusive"),
                      (CaptureSpec("up", 4, use_miss=True), "need_up_miss_output"),
                      (CaptureSpec("down", 4, use_miss=True), "need_down_miss_input"),
                      (CaptureSpec("up", 4, init_mode="vector"), "need_init_vector"),
                      (CaptureSpec("up", 4, init_mode="xtx"), "need_init_xtx")):
        with pytest.raises(ValueError, match=msg):
            validate_capture_spec(spec, req)
