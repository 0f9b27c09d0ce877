"""World-size-2 gloo tests of the region-sharded multi-GPU host path: the host logic on CPU, and
the same exchange over B200Runtime ranks on one GPU (gpu-marked; the ranks never wait on each
other's kernels, only on the host all-reduce)."""

from __future__ import annotations

import os
from pathlib import Path
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from grg_spmv_b200.distributed import assign_regions, reduce_job_time, sum_region_down


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_regions_is_balanced_and_complete():
    edges = [100, 90, 80, 30, 20, 10, 5]
    owned = assign_regions(edges, 3)
    assert sorted(r for rs in owned for r in rs) == list(range(len(edges)))
    loads = [sum(edges[r] for r in rs) for rs in owned]
    assert max(loads) - min(loads) <= max(edges)
    assert assign_regions(edges, 1) == [list(range(len(edges)))]
    with pytest.raises(ValueError):
        assign_regions(edges, 0)


def _worker(rank, world, port, paths, xs, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    from grg_oracle import OracleGRG

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = assign_regions([OracleGRG(p).num_edges for p in paths], world)[rank]
        k, samples = xs[0].shape[0], OracleGRG(paths[0]).num_samples
        partial = torch.zeros((samples, k), dtype=torch.float64)
        for region in mine:
            partial += torch.from_numpy(OracleGRG(paths[region]).matmul(xs[region], "down").T.copy())
        sum_region_down(partial)
        max_ms, work = reduce_job_time(10.0 * (rank + 1), 5.0)
        np.save(Path(out_dir) / f"r{rank}.npy", partial.numpy())
        np.save(Path(out_dir) / f"t{rank}.npy", np.asarray([max_ms, work]))
    finally:
        dist.destroy_process_group()


def test_region_sharded_down_sums_over_ranks(tmp_path):
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    from grg_oracle import OracleGRG

    paths = []
    for seed in range(3):  # three "regions" over the same 200 samples
        p = tmp_path / f"region{seed}.grg_spmv"
        write_synthetic_artifact(SynthSpec(num_samples=200, num_levels=6, num_nodes=1500 + 300 * seed, num_mutations=150 + 40 * seed,
                                           children=(2, 6), seed=seed), p)
        paths.append(str(p))
    rng = np.random.default_rng(0)
    xs = [rng.standard_normal((3, OracleGRG(p).num_mutations)) for p in paths]
    mp.spawn(_worker, args=(2, _free_port(), paths, xs, str(tmp_path)), nprocs=2, join=True)
    expected = sum(OracleGRG(p).matmul(x, "down").T for p, x in zip(paths, xs))
    for rank in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"r{rank}.npy"), expected, rtol=1e-12, atol=1e-12)
        np.testing.assert_array_equal(np.load(tmp_path / f"t{rank}.npy"), [20.0, 10.0])


def _gpu_worker(rank, world, port, paths, xs, out_dir):
    """One rank: a B200Runtime over the regions it owns, their ``down`` outputs summed on the
    device, then the one exchange (an all-reduce SUM over gloo on a host copy)."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    from grg_spmv_b200 import RuntimeRequirements, scan_grg_spmv
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        mine = assign_regions([scan_grg_spmv(p).num_edges for p in paths], world)[rank]
        k = xs[0].shape[0]
        samples = scan_grg_spmv(paths[0]).num_samples
        partial = torch.zeros((samples, k), dtype=torch.float64)
        if mine:
            req = RuntimeRequirements(max_k_up=k, max_k_down=k, need_down_miss_input=False, need_up_miss_output=False,
                                      need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
            layout = plan_b200_layout(artifacts=[paths[r] for r in mine], dtype=np.float64, requirements=req,
                                      vram_budget_bytes=0, ring_buffer_size=0, device=0, stream=0)
            with B200Runtime(layout, check_bounds=True) as runtime:
                acc = torch.zeros((k, samples), dtype=torch.float64, device="cuda:0")
                for grg, region in zip(runtime.grgs, mine):
                    acc += torch.from_numpy(grg.matmul(xs[region], "down")).to("cuda:0")
                torch.cuda.synchronize()
                assert runtime.device_error() == 0
            partial += acc.T.cpu()
        sum_region_down(partial)
        np.save(Path(out_dir) / f"g{rank}.npy", partial.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_region_sharded_down_on_b200_runtimes_sums_to_oracle(tmp_path):
    """Two ranks, each a B200Runtime over its own regions, one all-reduce: the summed ``down``
    equals the oracle's sum over all regions, exactly for integer-valued inputs."""
    from grg_spmv_b200.synth import SynthSpec, write_synthetic_artifact

    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    from grg_oracle import OracleGRG

    paths = []
    for seed in range(3):
        p = tmp_path / f"region{seed}.grg_spmv"
        write_synthetic_artifact(SynthSpec(num_samples=400, num_levels=8, num_nodes=4000 + 900 * seed, num_mutations=300 + 80 * seed,
                                           children=(2, 8), seed=20 + seed), p)
        paths.append(str(p))
    rng = np.random.default_rng(5)
    xs = [rng.integers(-2, 3, size=(4, OracleGRG(p).num_mutations)).astype(np.float64) for p in paths]
    mp.spawn(_gpu_worker, args=(2, _free_port(), paths, xs, str(tmp_path)), nprocs=2, join=True)
    expected = sum(OracleGRG(p).matmul(x, "down").T for p, x in zip(paths, xs))
    for rank in range(2):
        np.testing.assert_array_equal(np.load(tmp_path / f"g{rank}.npy"), expected)
