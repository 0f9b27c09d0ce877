"""World-size-2 gloo tests of the region-sharded multi-GPU host path (CPU only)."""

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
