"""Captured-graph adaptor: a ``BoundGRG`` whose matmuls replay pre-recorded CUDA graphs.

Restates the reference's ``CapturedBoundGRG`` / ``_capture_grg`` (``pygrgl_spmv/adaptor.py:
29-420`` and ``:826-965``) for the B200 backend.
* Every ``CaptureSpec`` (direction, k, by_individual, init_mode, use_miss) is prepared once.
* Its staging copy plus the traversal are recorded as one CUDA graph.
* ``matmul`` stages the caller's arrays into the captured buffers and replays the graph.

Caller contract, as in the reference:
* ``k`` may be smaller than the captured ``k``: the inputs are zero-padded and the output is
  truncated back;
* int32 inputs to an FP64 capture are cast, and the result is returned as int32;
* an UP miss output is accumulated into the caller's array (``+=``).

Modes:
* Copy mode takes and returns NumPy arrays.
* Native mode takes and returns CUDA tensors on the capture device. The reference's native
  mode takes CuPy arrays; this package is built on PyTorch, so native arrays are
  ``torch.Tensor``s here.
"""

from __future__ import annotations

import contextlib
from dataclasses import dataclass, field

import numpy as np

_VALID_INIT_MODES = {"none", "vector", "matrix", "xtx"}


@dataclass(frozen=True)
class CaptureSpec:
    """One ``prepare_matmul_cuda`` call to capture as a CUDA graph."""

    direction: str
    k: int
    by_individual: bool = False
    init_mode: str = "none"   # "none" | "vector" | "matrix" | "xtx"
    use_miss: bool = False


@dataclass(frozen=True)
class RunConfigs:
    """``RuntimeRequirements`` plus the graphs to capture (empty: one up and one down at the
    declared maximum k)."""

    req: object
    capture_ops: tuple = field(default_factory=tuple)


def validate_capture_spec(spec: CaptureSpec, req) -> None:
    """The reference's ``_validate_capture_spec`` (``adaptor.py:826-847``)."""
    if spec.init_mode not in _VALID_INIT_MODES:
        raise ValueError(f"CaptureSpec.init_mode {spec.init_mode!r} invalid; expected one of {sorted(_VALID_INIT_MODES)}")
    if spec.init_mode != "none" and spec.use_miss:
        raise ValueError(f"CaptureSpec direction={spec.direction!r}: init_mode and use_miss are mutually exclusive")
    if spec.use_miss:
        if spec.direction == "up" and not req.need_up_miss_output:
            raise ValueError("CaptureSpec use_miss=True for 'up' but need_up_miss_output is False")
        if spec.direction == "down" and not req.need_down_miss_input:
            raise ValueError("CaptureSpec use_miss=True for 'down' but need_down_miss_input is False")
    if spec.init_mode == "vector" and not req.need_init_vector:
        raise ValueError("CaptureSpec init_mode='vector' but need_init_vector is False")
    if spec.init_mode == "matrix" and not req.need_init_matrix:
        raise ValueError("CaptureSpec init_mode='matrix' but need_init_matrix is False")
    if spec.init_mode == "xtx" and not req.need_init_xtx:
        raise ValueError("CaptureSpec init_mode='xtx' but need_init_xtx is False")


def _np_dtype(d) -> np.dtype:
    if isinstance(d, np.dtype):
        return d
    if getattr(type(d), "__module__", "").startswith("torch"):
        import torch

        table = {torch.float32: np.float32, torch.float64: np.float64, torch.int32: np.int32}
        if d not in table:
            raise TypeError(f"unsupported torch dtype {d!r}")
        return np.dtype(table[d])
    return np.dtype(d)


class CapturedBoundGRG:
    """``BoundGRG`` backed by pre-captured CUDA graphs; other attributes come from the wrapped
    GRG.  ``matmul`` runs on the capture stream and returns when the result is ready."""

    def __init__(self, grg, prepared_ops, graphs, src_tensors, init_tensors, miss_tensors, capture_stream, *,
                 native: bool = False, device_lock=None) -> None:
        self._grg = grg
        self._prepared_ops = prepared_ops
        self._graphs = graphs
        self._src_tensors = src_tensors
        self._init_tensors = init_tensors
        self._miss_tensors = miss_tensors
        self._capture_stream = capture_stream
        self._native = bool(native)
        self._device_lock = device_lock if device_lock is not None else contextlib.nullcontext()

    @property
    def native(self) -> bool:
        return self._native

    def __getattr__(self, name):
        if name == "_grg":
            raise AttributeError(name)
        return getattr(self._grg, name)

    def _key(self, direction, by_individual, init_mode="none", use_miss=False):
        key = (direction, bool(by_individual), init_mode, bool(use_miss))
        return key if key in self._src_tensors else (direction, bool(by_individual), "none", False)

    def _validate(self, arr, *, name, role, expected_shape, expected_dtype, device):
        if arr is None:
            raise ValueError(f"matmul(): {name} ({role}) is required but got None")
        exp = _np_dtype(expected_dtype)
        if device is not None:
            import torch

            if not isinstance(arr, torch.Tensor) or arr.device != device:
                raise TypeError(f"matmul(): {name} ({role}) expected torch.Tensor on {device} (native mode), "
                                f"got {type(arr).__name__}" + (f" on {arr.device}" if isinstance(arr, torch.Tensor) else ""))
            actual = _np_dtype(arr.dtype)
        else:
            if not isinstance(arr, np.ndarray):
                raise TypeError(f"matmul(): {name} ({role}) expected numpy.ndarray (copy mode), got {type(arr).__name__}")
            actual = arr.dtype
        if actual != exp and not (exp == np.dtype(np.float64) and actual == np.dtype(np.int32)):
            raise TypeError(f"matmul(): {name} ({role}) dtype mismatch: expected {exp}, got {actual}")
        shape, want = tuple(arr.shape), tuple(expected_shape)
        if len(shape) != len(want) or shape[0] > want[0] or shape[1:] != want[1:]:
            raise ValueError(f"matmul(): {name} ({role}) shape mismatch: expected k <= {want[0]} with trailing dims "
                             f"{want[1:]}, got {shape}")

    def _as_torch(self, arr, target_dtype):
        import torch

        t = arr if isinstance(arr, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(arr))
        return t.to(target_dtype) if t.dtype != target_dtype else t

    def matmul(self, input, direction, emit_all_nodes=False, by_individual=False, init=None, miss=None):
        """Replay the captured graph for this call's key (``BoundGRG.matmul`` arguments)."""
        import torch

        if emit_all_nodes:
            raise ValueError("emit_all_nodes=True is not supported by CapturedBoundGRG.matmul()")
        with self._device_lock:
            if init is None:
                init_mode, payload = "none", None
            elif isinstance(init, str):
                if init != "xtx":
                    raise ValueError(f"unexpected init value: {init!r}")
                init_mode, payload = "xtx", None
            elif getattr(init, "ndim", 2) == 1:
                init_mode, payload = "vector", init
            else:
                init_mode, payload = "matrix", init
            use_miss = miss is not None
            key = self._key(direction, by_individual, init_mode, use_miss)
            if key not in self._src_tensors:
                raise ValueError(f"no captured graph for direction={direction!r} by_individual={by_individual}")
            src = self._src_tensors[key]
            device = src.device if self._native else None
            int32_in = src.dtype == torch.float64 and _np_dtype(input.dtype) == np.dtype(np.int32)
            self._validate(input, name="input", role="input", expected_shape=tuple(src.shape), expected_dtype=src.dtype,
                           device=device)
            k_prime, k_full = int(input.shape[0]), int(src.shape[0])

            def expect(shape):
                return (k_prime,) + tuple(shape[1:])

            if key in self._init_tensors:
                if payload is None:
                    raise ValueError(f"matmul() requires init data for captured graph key={key!r}")
                self._validate(payload, name="init", role="init", expected_shape=expect(self._init_tensors[key].shape),
                               expected_dtype=src.dtype, device=device)
            op = self._prepared_ops[key]
            if key in self._miss_tensors:
                self._validate(miss, name="miss", role="miss-in", expected_shape=expect(self._miss_tensors[key].shape),
                               expected_dtype=src.dtype, device=device)
            elif use_miss:
                self._validate(miss, name="miss", role="miss-out", expected_shape=expect(op.miss_output.shape),
                               expected_dtype=src.dtype, device=device)
            cap = self._capture_stream
            if self._native:
                cap.wait_stream(torch.cuda.current_stream(src.device))  # inputs produced on the caller's stream

            def stage(dst, value):
                value = self._as_torch(value, dst.dtype)
                if k_prime < k_full:
                    dst[:k_prime].copy_(value)
                    dst[k_prime:].zero_()
                else:
                    dst.copy_(value)

            with torch.cuda.stream(cap):
                stage(src, input)
                if key in self._init_tensors:
                    stage(self._init_tensors[key], payload)
                if key in self._miss_tensors:
                    stage(self._miss_tensors[key], miss)
                if use_miss and direction == "up":
                    op.miss_output.zero_()
                self._graphs[key].replay()
                out = op.output[:k_prime, :].clone()
                miss_out = op.miss_output[:k_prime, :].clone() if use_miss and direction == "up" else None
                if not self._native:
                    out = out.cpu()
                    miss_out = miss_out.cpu() if miss_out is not None else None
            cap.synchronize()
            if self._native:
                result = out.to(torch.int32) if int32_in else out
                if miss_out is not None:
                    miss += miss_out.to(miss.dtype)
                return result
            result = out.numpy()
            if int32_in:
                result = result.astype(np.int32)
            if miss_out is not None:
                miss += miss_out.numpy().astype(miss.dtype, copy=False)
            return result


def capture_grg(grg, capture_stream, req, stack: contextlib.ExitStack, *, capture_ops=(), native: bool = False,
                device_lock=None) -> CapturedBoundGRG:
    """Prepare and capture every spec of ``capture_ops`` (default: up and down at the
    declared maximum k) for ``grg``; the prepared ops live in ``stack``.  One staging buffer
    (and one init / miss buffer) sized for the largest spec is shared by all captures of the
    GRG, which never run concurrently (the reference's ``_capture_grg``).

    The graphs are recorded on ``capture_stream`` (a fresh stream when None or the default
    stream, which cannot capture) and replayed, with the staging copies, on the runtime's
    stream (the layout's ``stream``)."""
    import ctypes

    import torch

    from grg_spmv_b200.backends.b200 import _native as nat

    runtime = grg._runtime
    run_stream = runtime._torch_caller_stream()
    if capture_stream is None or int(capture_stream.cuda_stream) == 0:
        capture_stream = torch.cuda.Stream(device=run_stream.device)

    specs = tuple(capture_ops) or (CaptureSpec("up", int(req.max_k_up)), CaptureSpec("down", int(req.max_k_down)))
    prepared = {}
    in_n, init_n, miss_n = [], [], []
    for spec in specs:
        validate_capture_spec(spec, req)
        key = (spec.direction, bool(spec.by_individual), spec.init_mode, bool(spec.use_miss))
        if key in prepared:
            raise ValueError(f"Duplicate CaptureSpec key {key!r} in capture_ops")
        op = stack.enter_context(grg.prepare_matmul_cuda(direction=spec.direction, k=spec.k, by_individual=spec.by_individual,
                                                         init_mode=spec.init_mode, use_miss=spec.use_miss))
        prepared[key] = op
        in_n.append(op.input.numel())
        init_n.append(op.init_vector.numel() if spec.init_mode == "vector" else
                      op.init_matrix.numel() if spec.init_mode == "matrix" else 0)
        miss_n.append(op.miss_input.numel() if spec.use_miss and spec.direction == "down" else
                      op.miss_output.numel() if spec.use_miss else 0)
    first = next(iter(prepared.values()))
    dtype, device = first.input.dtype, first.input.device
    shared_src = torch.zeros(max(in_n), dtype=dtype, device=device)
    shared_init = torch.zeros(max(init_n), dtype=dtype, device=device) if max(init_n) else None
    shared_miss = torch.zeros(max(miss_n), dtype=dtype, device=device) if max(miss_n) else None
    graphs, srcs, inits, misses = {}, {}, {}, {}
    for spec in specs:
        key = (spec.direction, bool(spec.by_individual), spec.init_mode, bool(spec.use_miss))
        op = prepared[key]
        k, cols = op.input.shape
        src = torch.as_strided(shared_src, size=(k, cols), stride=(1, k))
        graph = torch.cuda.CUDAGraph()
        capture_stream.wait_stream(run_stream)
        with torch.cuda.graph(graph, stream=capture_stream, capture_error_mode="thread_local"):
            op.input.copy_(src)
            if spec.init_mode == "vector":
                inits[key] = shared_init[:k]
                op.init_vector.copy_(inits[key])
            elif spec.init_mode == "matrix":
                inits[key] = torch.as_strided(shared_init, size=(k, op.init_matrix.shape[1]), stride=(1, k))
                op.init_matrix.copy_(inits[key])
            elif spec.use_miss and spec.direction == "down":
                misses[key] = torch.as_strided(shared_miss, size=(k, op.miss_input.shape[1]), stride=(1, k))
                op.miss_input.copy_(misses[key])
            # the traversal itself, launched into this capture (the prepared op's own launch
            # path targets the runtime's stream)
            status = runtime._lib.grg_b200_traverse(ctypes.byref(op._args), ctypes.c_void_p(capture_stream.cuda_stream))
        nat.check(runtime._lib, status, "grg_b200_traverse (adaptor capture)")
        srcs[key] = src
        graphs[key] = graph
    return CapturedBoundGRG(grg, prepared, graphs, srcs, inits, misses, run_stream, native=native,
                            device_lock=device_lock)


__all__ = ["CaptureSpec", "CapturedBoundGRG", "RunConfigs", "capture_grg", "validate_capture_spec"]
