"""The allocation-free traversal entry point, called through the C ABI.

``grg_b200_traverse_static`` exists for callers that cannot allocate device memory (C/FFI
hosts without a device allocator, plugins inside another framework's memory manager, code
that must not allocate during stream capture): it keeps the traversal's node state in a fixed
array inside the library instead of a caller buffer.  It runs the same kernels as
``grg_b200_traverse``, so it must give the same bits on the same inputs, call after call (the
array is reused and keeps the previous call's contents), and must refuse what it cannot serve
(a node state larger than the array, the mixed dtype, streamed levels) before launching
anything.  This file is collected last so that a failure here does not stop the rest of the
suite.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def small_artifact(tmp_path_factory):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    path = tmp_path_factory.mktemp("noalloc") / "small.grg_spmv"
    write_synthetic_artifact(SynthSpec(num_samples=800, num_levels=10, num_nodes=20_000, num_mutations=5_000, children=(2, 12),
                                       miss_fraction=0.02, random_ids=True, seed=5), path)
    return path


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_static_state_entry_point_matches_traverse(small_artifact, dtype):
    from grg_spmv_b200 import RuntimeRequirements
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout
    from grg_spmv_b200.backends.b200 import _native as nat

    k = 4
    req = RuntimeRequirements(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=False,
                              need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
    layout = plan_b200_layout(artifacts=[small_artifact], dtype=dtype, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=0, stream=0)
    lib = nat.load_library()
    rng = np.random.default_rng(17)
    with B200Runtime(layout, use_graphs=False, check_bounds=True) as runtime:
        (grg,) = runtime.grgs
        stream = ctypes.c_void_p(runtime.stream_ptr)
        for direction in ("up", "down"):
            op = grg.prepare_matmul_cuda(direction=direction, k=k, use_miss=direction == "down")
            cols = grg.num_samples if direction == "up" else grg.num_mutations
            x = torch.from_numpy(rng.standard_normal((k, cols)).astype(dtype)).to("cuda:0")
            if direction == "down":
                op.miss_input.copy_(torch.from_numpy(rng.standard_normal((k, grg.num_mutations)).astype(dtype)).to("cuda:0"))
            # input and output share one buffer, so the input is restored before every call
            op.input.copy_(x)
            nat.check(lib, lib.grg_b200_traverse(ctypes.byref(op._args), stream), "grg_b200_traverse")
            torch.cuda.synchronize()
            expected = op.output.cpu().numpy().copy()
            for _ in range(2):  # two calls in a row on the shared static array
                op.input.copy_(x)
                nat.check(lib, lib.grg_b200_traverse_static(ctypes.byref(op._args), stream), "grg_b200_traverse_static")
                torch.cuda.synchronize()
                # the same kernels on the same inputs: the same bits
                np.testing.assert_array_equal(op.output.cpu().numpy(), expected)
                assert runtime.device_error() == 0, "device bounds check failed"

        # Refusals, all before anything is launched:
        # a node state larger than the fixed array,
        big = nat.TraverseArgs.from_buffer_copy(op._args)
        big.k = (16 << 20) // (np.dtype(dtype).itemsize * grg.num_nodes) + 1
        assert lib.grg_b200_traverse_static(ctypes.byref(big), stream) == nat.ERR_UNSUPPORTED
        assert "holds at most" in nat.last_error(lib)
        # the mixed node state,
        mixed = nat.TraverseArgs.from_buffer_copy(op._args)
        mixed.dtype = nat.MIXED
        assert lib.grg_b200_traverse_static(ctypes.byref(mixed), stream) == nat.ERR_UNSUPPORTED
        assert "FP64 and FP32" in nat.last_error(lib)
        # and a level streamed through the ring.
        streamed = nat.TraverseArgs.from_buffer_copy(op._args)
        levels = (nat.Level * streamed.num_levels)(*[streamed.levels[i] for i in range(streamed.num_levels)])
        levels[0].ring_slot = 0
        streamed.levels = ctypes.cast(levels, ctypes.POINTER(nat.Level))
        assert lib.grg_b200_traverse_static(ctypes.byref(streamed), stream) == nat.ERR_UNSUPPORTED
        assert "resident" in nat.last_error(lib)
        torch.cuda.synchronize()
        assert runtime.device_error() == 0
