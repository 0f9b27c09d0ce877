"""GRG up+down throughput benchmark of the B200 backend (one JSON line on rank 0).

Workload: the synthetic GRG with the shape of the "plain FP64 drop-in on B200" configuration
(100k haploid samples, 40 internal levels, ~5M nodes, ~60M edges, 1M mutations, 1% missing
entries via per-mutation missingness nodes), fully resident, FP64, k right-hand sides.  One
step = one ``up`` traversal (X·G) of a resident sample-major input followed by one ``down``
traversal (X·Gᵀ, with the miss input) that consumes the up output in place (the prepared
ops' shared ``io0`` buffer).  Metric: edge·RHS/s = steps · 2·E·k / device time.

* ``value``: device time of K steps (CUDA events on the caller stream, inputs resident);
  the working set (~0.8 GB of gather lists and node rows) exceeds the 126 MB L2, so no L2
  flush is needed between steps.
* ``e2e``: the same steps through the public prepared-op API with the inputs copied from
  pinned host memory and both outputs copied back every step; ``--e2e-inflight`` steps (8)
  run at once, each on its own runtime and stream, so one step's copies overlap another's
  kernels (the host link moves 70 MB each way per step at about 95 GB/s in both directions
  together, 1.5 ms, against 1.4 ms of kernels).
* ``roofline``: the level gather kernels timed live in one instrumented up+down pass: events
  around each direction's level launches, issued back to back as in the recorded graph (a
  second pass with events around every launch prints the per-level breakdown to stderr).  Algorithmic bytes per level: 4 per gather entry and row
  pointer, plus each destination row written once and read once later (2·k·8); plus, for
  down, the mutation and miss input rows read once.  ``traffic`` is the DRAM traffic (read +
  write) of one up-level-1 launch measured by ncu on the same configuration;
  ``traffic_launches`` lists it with down levels 3, 1 and 0, beside this run's own timing
  and algorithmic bytes of those launches.
* ``cpu_baseline``: the oracle (SciPy restatement of the reference's ReferenceRuntime) on one
  step of the same graph, RHS columns split over one process per host core (up to k), rank 0,
  N=1 only.
* ``tiers``: RHS-block batching and mixed precision against the plain FP64 drop-in on the same
  graph and on eight generated graphs, the standardised Gram operator, and the precision
  configuration (diploid config-2 graph, k = 32, init_xtx, plain and mixed node state against
  the oracle) (N=1 only; ``--no-tiers`` skips it).
* ``--impl reference``: the reference's CPU path (the oracle port; the pure-Python reference
  cannot be installed offline) timed on the same workload, on the same host cores.

Multi-GPU (``torchrun``): every rank runs its own graph (a different seed, as a genomic region
would be), no data-path collective; ``value`` sums the ranks' work over the max of their times.
"""

from __future__ import annotations

import argparse
import ctypes
import dataclasses
import json
import os
from pathlib import Path
import subprocess
import sys
import shutil
import tempfile
import time

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "GRG up+down edge·RHS/s (k RHS, FP64)"
UNIT = "edge·RHS/s"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--k", type=int, default=8)
    p.add_argument("--workload", choices=["config2", "medium", "small"], default="config2")
    p.add_argument("--exact-order", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-k1", action="store_true", help="skip the second measurement of the same step at k = 1")
    p.add_argument("--e2e-inflight", type=int, default=8, help="end-to-end steps in flight (one runtime and stream each)")
    p.add_argument("--no-tiers", action="store_true",
                   help="skip the batched / mixed-precision comparison on uneven RHS blocks (runs at N=1 only)")
    p.add_argument("--tier-blocks", default="1,3,16,64,256", help="RHS block widths of the tier comparison")
    p.add_argument("--tier-steps", type=int, default=3)
    p.add_argument("--tier-grgs", type=int, default=8, help="graphs of the multi-graph tier (0: skip it)")
    p.add_argument("--tier-scale", type=float, default=1.0, help="size of the multi-graph tier's graphs vs 5M-40M edges")
    p.add_argument("--tier-artifacts", default=None, help="directory for (reused) multi-graph tier artifacts")
    p.add_argument("--no-clocks", action="store_true", help="skip clock sampling and its untimed busy loops")
    p.add_argument("--artifact", default=None, help=".grg_spmv to use (generated there first if missing)")
    p.add_argument("--heavy-threshold", type=int, default=None)
    p.add_argument("--variant", type=int, default=None, help="narrow-row kernel variant")
    p.add_argument("--no-graphs", action="store_true", help="launch kernels per level instead of replaying a CUDA graph")
    p.add_argument("--no-balance", action="store_true", help="do not group narrow rows by length")
    p.add_argument("--autotune", action="store_true", help="pick the narrow and heavy kernels per direction at runtime entry")
    p.add_argument("--heavy-variant", type=int, default=None,
                   help="heavy-row kernel: 0 CTA per row, 1 warp per row, 2 warp per row fused into the narrow launch")
    p.add_argument("--short-first", action="store_true", help="process length buckets shortest first")
    p.add_argument("--heavy-buckets", action="store_true", help="also group heavy rows by length (default: row order)")
    p.add_argument("--no-short-rows", action="store_true",
                   help="walk the one-quad narrow rows with two entry slots like the rest (default: one slot)")
    p.add_argument("--slots", choices=["none", "up", "down", "both"], default="none",
                   help="directions whose narrow rows are padded to their bucket width (list offset from position)")
    p.add_argument("--pdl", choices=["auto", "on", "off"], default="auto",
                   help="programmatic dependent launch of the level kernels (auto: on for k >= 8)")
    p.add_argument("--budget-frac", type=float, default=1.0,
                   help="VRAM budget as a fraction of full residency; below 1 the largest levels stream from pinned memory")
    p.add_argument("--ring", type=int, default=4, help="ring slots when levels stream")
    p.add_argument("--narrow-split", type=int, default=None, help="narrow rows split over 2^n lane groups (-1: per level)")
    p.add_argument("--fuse-entries", type=int, default=None,
                   help="run stretches of levels with at most this many entries as one cooperative launch (0: off)")
    p.add_argument("--schedule", choices=["levels", "dataflow"], default=None,
                   help="one launch per level, or one persistent dataflow launch per traversal")
    p.add_argument("--precision", choices=["plain", "mixed"], default="plain",
                   help="node state in FP64 (plain) or FP32 + 16-bit correction with FP64 sums (mixed)")
    p.add_argument("--row-order-up", choices=["natural", "locality"], default=None)
    p.add_argument("--row-order-down", choices=["natural", "locality"], default=None)
    p.add_argument("--apps", action="store_true",
                   help="time the application harnesses instead (randomized PCA on this graph; block CG on a "
                        "streamed graph of the large configuration's shape) and print their JSON line")
    p.add_argument("--apps-scale", type=float, default=0.1,
                   help="size of the CG graph vs the large configuration (1M samples, 60M nodes, 600M edges, "
                        "20M mutations); its VRAM budget scales with it (16 GB at 1.0)")
    p.add_argument("--apps-artifact", default=None, help=".grg_spmv for the CG graph (generated there first if missing)")
    p.add_argument("--apps-only", choices=["all", "pca", "cg", "precision"], default="all",
                   help="which application harnesses to run")
    p.add_argument("--precision-artifact", default=None,
                   help=".grg_spmv for the precision harness (diploid config-2 graph; generated there first if missing)")
    return p.parse_args()


def workload_spec(name: str, seed: int):
    from grg_spmv_b200.synth import CONFIG2, SynthSpec

    if name == "config2":
        return dataclasses.replace(CONFIG2, seed=seed)
    if name == "medium":  # profiling case: the same generator at 30% scale, working set still above L2
        return SynthSpec(num_samples=30_000, num_levels=40, num_nodes=1_500_000, num_mutations=300_000, children=(2, 22),
                         miss_fraction=0.01, seed=seed)
    return SynthSpec(num_samples=20_000, num_levels=20, num_nodes=600_000, num_mutations=100_000, children=(2, 28),
                     miss_fraction=0.01, seed=seed)


def make_artifact(args, rank: int) -> tuple[Path, float]:
    from grg_spmv_b200.synth import write_synthetic_artifact

    if args.artifact and Path(args.artifact).exists():
        return Path(args.artifact), 0.0
    out = Path(args.artifact) if args.artifact else Path(tempfile.mkdtemp(prefix="grg_bench_")) / f"{args.workload}_r{rank}.grg_spmv"
    t0 = time.perf_counter()
    write_synthetic_artifact(workload_spec(args.workload, seed=rank), out)
    return out, time.perf_counter() - t0


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])

    def __enter__(self):
        if self.device_index < 0:
            return self
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def wait_for_samples(self, count: int = 2, timeout_s: float = 3.0) -> None:
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < timeout_s:
            if self.path.exists() and len(self.path.read_text().splitlines()) >= count:
                return
            time.sleep(0.05)

    def summary(self) -> dict:
        rows = []
        for line in self.path.read_text().splitlines() if self.path.exists() else []:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][2]) if rows else None,
                "reasons": reasons, "samples": len(rows)}


def workload_description(name: str, scan, streamed: bool) -> str:
    """The workload string both arms report: the configuration's name and the graph's sizes."""
    return (f"{name}: S={scan.num_samples}, levels={scan.num_levels}, N={scan.num_nodes}, E={scan.num_edges}, "
            f"M={scan.num_mutations}, 1% missing, {'levels partly streamed' if streamed else 'fully resident'}, up+down per step")


def host_info(workers: int) -> dict:
    """What every CPU number is recorded with: the host's logical CPUs and physical cores, its
    CPU model, and the processes x threads the measurement actually used."""
    try:
        import psutil

        physical = psutil.cpu_count(logical=False)
    except ImportError:  # pragma: no cover - psutil is in the image
        physical = None
    model = None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.lower().startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"host_logical_cpus": os.cpu_count(), "host_physical_cores": physical, "cpu_model": model,
            "processes": int(workers), "threads_per_process": 1}


def measured_peak_hbm() -> tuple[float, str]:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


# DRAM bytes (read + write) and ncu duration of single level launches on the config-2 graph at
# k = 8, FP64, default plan, measured with ncu -c 1 and L2 left warm (profiles/
# level_traffic_config2_k8.md gives the commands).  Keys: (direction, level).
CONFIG2_K8_TRAFFIC = {
    ("up", 1): {"kernel": "level_entry_pre_kernel", "dram_bytes": 12052480 + 45312, "ncu_us": 24.58},
    ("down", 3): {"kernel": "level_entry_pre_kernel", "dram_bytes": 126545664 + 20910848, "ncu_us": 33.73},
    ("down", 1): {"kernel": "level_entry_pre_kernel", "dram_bytes": 525780224 + 21631744, "ncu_us": 110.72},
    ("down", 0): {"kernel": "level_lean_warp_kernel", "dram_bytes": 458001152 + 17115392, "ncu_us": 208.93},
}
CONFIG2_K8_VARIANT = 15  # the narrow variant those launches ran
TRAFFIC_SOURCE = "profiles/level_traffic_config2_k8.md (ncu -c 1 per launch on the config-2 graph, k = 8)"


def traversal_level_launches(levels, fused_heavy: bool, fuse_entries: int) -> int:
    """Kernel launches of a traversal's levels: one per level (two when heavy rows run apart),
    with each stretch of two or more resident levels of at most ``fuse_entries`` entries as one."""
    launches, run = 0, 0
    for lv in levels:
        if lv.num_rows == 0:
            continue
        if fuse_entries > 0 and lv.ring_slot < 0 and lv.num_entries <= fuse_entries and run < 48:
            run += 1
            continue
        launches += (1 if run >= 2 else run) + 1 + (1 if 0 < lv.num_heavy < lv.num_rows and not fused_heavy else 0)
        run = 0
    return launches + (1 if run >= 2 else run)


def level_units(scan, direction: str, level: int, use_miss: bool) -> tuple[int, int]:
    """(rows, gather entries) of one level from the artifact scan (real edges, no padding)."""
    from grg_spmv_b200.backends.b200.structures import down_entry_bound, up_entry_bound

    rows = int(scan.level_sizes[level])
    entries = up_entry_bound(scan, level) if direction == "up" else down_entry_bound(scan, level, use_miss)
    return rows, entries


def level_bytes(units, k: int, itemsize: int, direction: str, num_mutations: int, use_miss: bool) -> int:
    """Algorithmic bytes of one traversal's level kernels: each gather entry (4 B) and row
    pointer (4 B) read once, each destination row written once and read once by later levels
    or the output stage (2·k·b), plus (down) the mutation inputs read once."""
    total = 0
    for rows, entries in units:
        total += 4 * int(entries) + 4 * (int(rows) + 1) + 2 * int(rows) * k * itemsize
    if direction == "down":
        total += num_mutations * k * itemsize * (2 if use_miss else 1)
    return total


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local_rank))
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)

    from grg_spmv_b200 import RuntimeRequirements, scan_grg_spmv
    from grg_spmv_b200.backends.b200 import B200Plan, B200PlanPair, B200Runtime, plan_b200_layout
    from grg_spmv_b200.backends.b200 import _native as nat
    from grg_spmv_b200.types import Direction

    path, gen_s = make_artifact(args, rank)
    scan = scan_grg_spmv(path)
    k = int(args.k)
    req = RuntimeRequirements(max_k_up=k, max_k_down=k, need_down_miss_input=True, need_up_miss_output=False,
                              need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
    extra = {} if args.heavy_threshold is None else {"heavy_threshold": args.heavy_threshold}
    if args.variant is not None:
        extra["narrow_variant"] = args.variant
    if args.no_balance:
        extra["balance"] = False
    if args.autotune:
        extra["autotune"] = True
    if args.heavy_variant is not None:
        extra["heavy_variant"] = args.heavy_variant
    if args.short_first:
        extra["long_first"] = False
    if args.heavy_buckets:
        extra["heavy_buckets"] = True
    if args.no_short_rows:
        extra["short_rows"] = False
    if args.pdl != "auto":
        extra["pdl"] = args.pdl == "on"
    if args.narrow_split is not None:
        extra["narrow_split"] = args.narrow_split
    if args.fuse_entries is not None:
        extra["fuse_entries"] = args.fuse_entries
    if args.schedule is not None:
        extra["schedule"] = args.schedule
    pair = B200PlanPair(plan_up=B200Plan(exact_order=args.exact_order, row_order=args.row_order_up,
                                         slots=args.slots in ("up", "both"), **extra),
                        plan_down=B200Plan(exact_order=args.exact_order, row_order=args.row_order_down,
                                           slots=args.slots in ("down", "both"), **extra))
    stream = torch.cuda.Stream(device=device)
    layout = plan_b200_layout(artifacts=[path], dtype=np.float64, requirements=req, vram_budget_bytes=0, ring_buffer_size=0,
                              device=local_rank, stream=stream, pair=pair, precision=args.precision)
    budget, ring = 0, 0
    if args.budget_frac < 1.0:  # keep about this fraction of the level lists resident, stream the rest
        list_bytes = layout.bytes_by_category["resident_sparse"]
        budget, ring = int(layout.required_budget_for_full_residency - (1.0 - args.budget_frac) * list_bytes), args.ring
        for _ in range(40):  # the ring slots come out of the same budget: grow it until the plan fits
            try:
                layout = plan_b200_layout(artifacts=[path], dtype=np.float64, requirements=req, vram_budget_bytes=budget,
                                          ring_buffer_size=ring, device=local_rank, stream=stream, pair=pair,
                                          precision=args.precision)
                break
            except ValueError:
                budget = int(budget + 0.02 * list_bytes)
    streamed_bytes = sum(lp.nbytes for lp in layout.level_plans() if not lp.resident)
    t0 = time.perf_counter()
    runtime = B200Runtime(layout, use_graphs=not args.no_graphs).__enter__()
    enter_s = time.perf_counter() - t0
    (grg,) = runtime.grgs
    S, M, E = grg.num_samples, grg.num_mutations, grg.num_edges
    rng = np.random.default_rng(100 + rank)
    x_up_np = rng.standard_normal((k, S))
    miss_np = rng.choice(np.asarray([0.0, 1.0]), size=(k, M), p=[0.99, 0.01])
    with torch.cuda.device(device), torch.cuda.stream(stream):
        up = grg.prepare_matmul_cuda(direction="up", k=k)
        down = grg.prepare_matmul_cuda(direction="down", k=k, use_miss=True)
        x_up = torch.from_numpy(x_up_np).to(device)
        down.miss_input.copy_(torch.from_numpy(miss_np).to(device))
    assert up.output.data_ptr() == down.input.data_ptr()

    def step():
        up.input.copy_(x_up)
        up()
        down()

    def synced_barrier():
        torch.cuda.synchronize(device)
        if world > 1:
            dist.barrier()

    with torch.cuda.device(device), torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 0)):
            step()
        synced_barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def busy(seconds: float) -> None:  # untimed load so the clock samples see the GPU busy
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < seconds:
                for _ in range(4):
                    step()
                torch.cuda.synchronize(device)

        with ClockSampler(local_rank if not args.no_clocks else -1) as clocks:
            if not args.no_clocks:
                clocks.wait_for_samples(1)
                busy(0.6)
            synced_barrier()
            start.record(stream)
            for _ in range(args.steps):
                step()
            end.record(stream)
            synced_barrier()
            if not args.no_clocks:
                busy(0.6)
        elapsed_ms = start.elapsed_time(end)
    max_ms = elapsed_ms
    total_work = args.steps * 2.0 * E * k
    if world > 1:
        t = torch.tensor([elapsed_ms, total_work], device=device, dtype=torch.float64)
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        max_ms, total_work = float(mx[0]), float(t[1])
    value = total_work / (max_ms / 1e3)

    # The same step at k = 1 (the configuration's other RHS width) on the same runtime.
    k1 = None
    if k != 1 and not args.no_k1:
        with torch.cuda.device(device), torch.cuda.stream(stream):
            up1 = grg.prepare_matmul_cuda(direction="up", k=1)
            down1 = grg.prepare_matmul_cuda(direction="down", k=1, use_miss=True)
            assert up1.output.data_ptr() == down1.input.data_ptr()
            x1 = x_up[:1].clone()
            down1.miss_input.copy_(torch.from_numpy(miss_np[:1]).to(device))

            def step1():
                up1.input.copy_(x1)
                up1()
                down1()

            for _ in range(max(args.warmup, 0)):
                step1()
            synced_barrier()
            a1, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a1.record(stream)
            for _ in range(args.steps):
                step1()
            b1.record(stream)
            synced_barrier()
            ms1 = a1.elapsed_time(b1)
        if world > 1:
            t = torch.tensor([ms1], device=device, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms1 = float(t[0])
        k1 = {"value": args.steps * 2.0 * E * world / (ms1 / 1e3), "unit": UNIT, "ms_per_step": ms1 / args.steps, "k": 1,
              "launch": "same runtime, prepared ops at k = 1, CUDA-graph replay"}
        del up1, down1

    # Live per-kernel timing of the level gathers (one instrumented up+down pass).
    vb = 8 if args.precision == "plain" else 6  # bytes per stored node value
    lib = runtime._lib
    level_ms = {"up": 0.0, "down": 0.0}
    level_launches = 0
    lv_bytes = 0
    all_evs = []
    with torch.cuda.device(device), torch.cuda.stream(stream):
        up.input.copy_(x_up)
        # Hold the stream for ~50 ms so the host enqueues every launch and event before the
        # GPU reaches them: event deltas then time kernels, not host launch latency.
        torch.cuda._sleep(100_000_000)
        whole_traversals = pair.plan_down.schedule == "dataflow" or streamed_bytes or pair.plan_down.fuse_entries > 0
        for name, op in (("up", up), ("down", down)):
            args_c = op._args
            if whole_traversals:  # streamed levels live in pinned host memory until the traversal copies
                # them into its ring; fused level runs are formed by the traversal
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                nat.check(lib, lib.grg_b200_traverse(ctypes.byref(args_c), ctypes.c_void_p(stream.cuda_stream)), "traverse")
                b.record(stream)
                if pair.plan_down.schedule == "dataflow":
                    level_launches += 3 if name == "up" else 2  # sentinel fill (+ seed) + dataflow kernel + output
                else:
                    fused = op._args.heavy_variant == 2 and op._args.narrow_variant >= 6 and not op._args.exact_order
                    lv_arr = runtime._artifacts[0].levels[op._spec.direction].array
                    level_launches += traversal_level_launches(lv_arr, fused, int(op._args.fuse_entries)) + (2 if name == "up" else 1)
                lv_order = range(1, scan.num_levels) if name == "up" else range(scan.num_levels - 1, -1, -1)
                units = [level_units(scan, name, L, True) for L in lv_order if scan.level_sizes[L] > 0]
                all_evs.append((name, [(a, b)], [], units))
                continue
            if name == "up":
                nat.check(lib, lib.grg_b200_seed_up(ctypes.byref(args_c), ctypes.c_void_p(stream.cuda_stream)), "seed_up")
            levels = runtime._artifacts[0].levels[op._spec.direction]
            # One pair of events around the direction's level launches, issued back to back as in
            # the recorded graph (events between launches would add their own gaps and break the
            # programmatic-dependent-launch overlap); per-level events follow in a second pass.
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for i in range(levels.count):
                nat.check(lib, lib.grg_b200_run_level(ctypes.byref(args_c), ctypes.byref(levels.array[i]),
                                                      ctypes.c_void_p(stream.cuda_stream)), "run_level")
                fused = op._args.heavy_variant == 2 and op._args.narrow_variant >= 6 and not op._args.exact_order
                lv = levels.array[i]
                level_launches += 1 + (1 if 0 < lv.num_heavy < lv.num_rows and not fused else 0)
            b.record(stream)
            evs = [(a, b)]
            if name == "up":
                nat.check(lib, lib.grg_b200_output_up(ctypes.byref(args_c), ctypes.c_void_p(stream.cuda_stream)), "output_up")
            else:
                nat.check(lib, lib.grg_b200_output_down(ctypes.byref(args_c), ctypes.c_void_p(stream.cuda_stream)), "output_down")
            lv_order = range(1, scan.num_levels) if name == "up" else range(scan.num_levels - 1, -1, -1)
            units = [level_units(scan, name, L, True) for L in lv_order if scan.level_sizes[L] > 0]
            all_evs.append((name, evs, list(levels.array), units))
        per_level = []  # diagnostic pass: events around every level launch (values are not used)
        for name, op in (("up", up), ("down", down)):
            if pair.plan_down.schedule == "dataflow" or streamed_bytes:
                break  # (fused level runs: the per-level breakdown shows the unfused launches)
            levels = runtime._artifacts[0].levels[op._spec.direction]
            for i in range(levels.count):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                nat.check(lib, lib.grg_b200_run_level(ctypes.byref(op._args), ctypes.byref(levels.array[i]),
                                                      ctypes.c_void_p(stream.cuda_stream)), "run_level")
                b.record(stream)
                per_level.append((name, a, b, levels.array[i]))
        torch.cuda.synchronize(device)
        for name, evs, lvs, units in all_evs:
            level_ms[name] = sum(a.elapsed_time(b) for a, b in evs)
            print(f"[traversal] {name} entries={sum(u[1] for u in units)} ms={level_ms[name]:.4f}", file=sys.stderr)
            lv_bytes += level_bytes(units, k, vb, name, M, use_miss=True)
        per_level_ms = 0.0
        launch_ms = {}  # (direction, level) -> ms of that level's launch, events around it alone
        for name, _, _, units in all_evs:
            lv_order = range(1, scan.num_levels) if name == "up" else range(scan.num_levels - 1, -1, -1)
            lv_ids = [L for L in lv_order if scan.level_sizes[L] > 0]
            for (_, a, b, lv), unit, L in zip([x for x in per_level if x[0] == name], units, lv_ids):
                ms = a.elapsed_time(b)
                per_level_ms += ms
                launch_ms[(name, L)] = (ms, level_bytes([unit], k, vb, "up", M, False))
                nbytes = level_bytes([unit], k, vb, "up", M, False)
                print(f"[level] {name} rows={unit[0]} entries={unit[1]} heavy={lv.num_heavy} "
                      f"ms={ms:.4f} GB/s={nbytes / ms / 1e6:.1f}", file=sys.stderr)
    whole = whole_traversals  # seed/output already counted
    launches_per_step = level_launches + (0 if whole else 3)  # + seed_up + outputs
    level_total_ms = level_ms["up"] + level_ms["down"]
    peak, peak_kind = measured_peak_hbm()
    achieved = lv_bytes / (level_total_ms / 1e3) / 1e9

    # End-to-end through the public API with pinned host buffers: every step copies its input
    # and miss rows in and both outputs out.  ``--e2e-inflight`` steps are in flight, each on its
    # own runtime and stream, so one step's copies overlap the others' kernels.
    e2e = None
    if not args.no_e2e:
        lanes = [(stream, runtime, up, down)]
        extra_runtimes = []
        for _ in range(max(args.e2e_inflight, 1) - 1):
            s2 = torch.cuda.Stream(device=device)
            lay2 = plan_b200_layout(artifacts=[path], dtype=np.float64, requirements=req, vram_budget_bytes=budget,
                                    ring_buffer_size=ring, device=local_rank, stream=s2, pair=pair, precision=args.precision)
            rt2 = B200Runtime(lay2, use_graphs=not args.no_graphs).__enter__()
            extra_runtimes.append(rt2)
            (g2,) = rt2.grgs
            with torch.cuda.device(device), torch.cuda.stream(s2):
                lanes.append((s2, rt2, g2.prepare_matmul_cuda(direction="up", k=k),
                              g2.prepare_matmul_cuda(direction="down", k=k, use_miss=True)))
        x_host = torch.from_numpy(x_up_np).pin_memory()
        miss_host = torch.from_numpy(miss_np).pin_memory()
        outs = [(torch.empty((k, M), dtype=torch.float64).pin_memory(), torch.empty((k, S), dtype=torch.float64).pin_memory())
                for _ in lanes]

        def e2e_step(i: int) -> None:
            st, _, op_up, op_down = lanes[i % len(lanes)]
            out_up_host, out_down_host = outs[i % len(lanes)]
            with torch.cuda.stream(st):
                op_up.input.copy_(x_host, non_blocking=True)
                op_up()
                out_up_host.copy_(op_up.output, non_blocking=True)
                op_down.miss_input.copy_(miss_host, non_blocking=True)
                op_down()
                out_down_host.copy_(op_down.output, non_blocking=True)

        with torch.cuda.device(device):
            for i in range(max(args.warmup, 1) * len(lanes)):
                e2e_step(i)
            synced_barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for st, *_ in lanes[1:]:
                st.wait_stream(stream)
            for i in range(args.steps):
                e2e_step(i)
            for st, *_ in lanes[1:]:
                stream.wait_stream(st)
            b.record(stream)
            synced_barrier()
            e2e_ms = a.elapsed_time(b)
        # every lane computed the same step: their host outputs must agree bit for bit
        lanes_agree = all(np.array_equal(o[0].numpy(), outs[0][0].numpy()) and np.array_equal(o[1].numpy(), outs[0][1].numpy())
                          for o in outs[1:])
        for rt2 in extra_runtimes:
            rt2.__exit__(None, None, None)
        del extra_runtimes, lanes
        if world > 1:
            t = torch.tensor([e2e_ms], device=device, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t[0])
        e2e = {"value": total_work / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms / args.steps,
               "h2d_bytes_per_step": int((S + M) * k * 8), "d2h_bytes_per_step": int((M + S) * k * 8),
               "steps_in_flight": max(args.e2e_inflight, 1), "lanes_agree": bool(lanes_agree)}

    # CPU baseline (oracle) and a parity spot check of the same step, rank 0 at N=1.
    cpu = None
    max_rel = None
    integer_check = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        workers = min(k, os.cpu_count() or 1)
        pool = ParallelOracle(path, workers)
        try:
            pool.step(x_up_np, miss_np)  # warm-up: workers load the graph
            t0 = time.perf_counter()
            ref_up, ref_down = pool.step(x_up_np, miss_np)
            cpu_s = time.perf_counter() - t0
        finally:
            pool.close()
        cpu = {"value": 2.0 * E * k / cpu_s, "unit": UNIT, "cores": workers, "kind": "port",
               "sample": f"1 up+down step (k={k}) of the same graph; SciPy ReferenceRuntime restatement, "
                         f"{workers} processes x 1 thread (RHS columns split, at most one process per column)",
               "seconds": cpu_s, **host_info(workers)}
        with torch.cuda.device(device), torch.cuda.stream(stream):
            up.input.copy_(x_up)
            up()
            got_up = up.output.cpu().numpy()
            down()
            got_down = down.output.cpu().numpy()
        rel = lambda got, ref: float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))
        max_rel = max(rel(got_up, ref_up), rel(got_down, ref_down))
        # Integer-valued inputs at full size: +-1 samples up, then down from the up output
        # (allele-count-like sums) with 0/1/2 miss rows; exact in FP64, so the error must be 0.
        xi = rng.choice(np.asarray([-1.0, 1.0]), size=(k, S))
        mi = rng.integers(0, 3, size=(k, M)).astype(np.float64)
        pool = ParallelOracle(path, workers)
        try:
            ref_up_i, ref_down_i = pool.step(xi, mi)
        finally:
            pool.close()
        with torch.cuda.device(device), torch.cuda.stream(stream):
            up.input.copy_(torch.from_numpy(xi).to(device))
            down.miss_input.copy_(torch.from_numpy(mi).to(device))
            up()
            got_up_i = up.output.cpu().numpy()
            down()
            got_down_i = down.output.cpu().numpy()
            down.miss_input.copy_(torch.from_numpy(miss_np).to(device))
        integer_check = {"inputs": "up: +-1 samples; down: the up output with 0/1/2 miss rows", "k": k,
                         "max_abs_err_vs_oracle": float(max(np.max(np.abs(got_up_i - ref_up_i)),
                                                            np.max(np.abs(got_down_i - ref_down_i)))),
                         "max_abs_value": float(max(np.max(np.abs(ref_up_i)), np.max(np.abs(ref_down_i))))}

    tuned = {d.value: [v, runtime._heavy_variant.get(d)] for d, v in runtime._variant.items()}
    heavy_used = {"up": int(up._args.heavy_variant), "down": int(down._args.heavy_variant)}
    narrow_used = {"up": int(up._args.narrow_variant), "down": int(down._args.narrow_variant)}
    runtime.__exit__(None, None, None)
    del up, down, runtime
    torch.cuda.empty_cache()
    tiers = None
    if world == 1 and not args.no_tiers:
        config_blocks = [int(b) for b in args.tier_blocks.split(",") if b]
        tiers = {"single_graph": measure_tiers(args, [path], device, stream, [config_blocks])[0]}
        torch.cuda.empty_cache()
        tiers["pca_operator"] = measure_xtx_operator(path, device)
        torch.cuda.empty_cache()

        def timed(st, fn):  # events on the stream, host clock beside them
            torch.cuda.synchronize(device)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            a.record(st)
            res = fn()
            b.record(st)
            torch.cuda.synchronize(device)
            return res, a.elapsed_time(b), (time.perf_counter() - t0) * 1e3

        # the precision configuration (diploid config-2 graph, k = 32, init_xtx; plain and mixed)
        tiers["precision"] = run_precision(args, timed, device)
        torch.cuda.empty_cache()
        if args.tier_grgs > 0:
            t0 = time.perf_counter()
            multi = make_multi_artifacts(args)
            gen_multi = time.perf_counter() - t0
            # the configuration's blocks, then many narrow blocks (where merging blocks and
            # overlapping graphs pay most)
            tiers["multi_graph"], tiers["multi_graph_small_blocks"] = measure_tiers(
                args, multi, device, stream, [config_blocks, [1, 1, 2, 3, 3, 4]])
            tiers["multi_graph"]["generate_s"] = gen_multi
    # Per-launch view of the captured launches: this run's own event timing of each launch (events
    # around it alone) and its algorithmic bytes, beside the DRAM bytes ncu measured for the same
    # launch of the same configuration.
    traffic, traffic_launches = None, None
    captured = (args.workload == "config2" and k == 8 and args.precision == "plain" and pair.plan_down.schedule == "levels"
                and not args.heavy_buckets and not args.no_short_rows and launch_ms
                and narrow_used == {"up": CONFIG2_K8_VARIANT, "down": CONFIG2_K8_VARIANT})
    if captured:
        traffic_launches = []
        for (direction, level), cap in CONFIG2_K8_TRAFFIC.items():
            ms, alg = launch_ms.get((direction, level), (None, None))
            traffic_launches.append({"launch": f"{direction} level {level}", "kernel": cap["kernel"], "dram_bytes": cap["dram_bytes"],
                                     "algorithmic_bytes": alg, "traffic_over_algorithmic": cap["dram_bytes"] / alg if alg else None,
                                     "ms_this_run": ms, "achieved_gbs_this_run": alg / ms / 1e6 if ms else None,
                                     "ncu_us": cap["ncu_us"]})
        traffic = CONFIG2_K8_TRAFFIC[("up", 1)]["dram_bytes"]
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "plain" else "f64 sums, f32+i16 node state",
            "data": "synthetic (seeded generator with the configuration's shapes; no public GRG dataset offline)",
            "config": {"workload": workload_description(args.workload, scan, streamed=bool(streamed_bytes)),
                       "k": k, "precision": args.precision, "num_samples": S, "num_nodes": grg.num_nodes, "num_edges": E, "num_mutations": M,
                       "num_levels": scan.num_levels, "exact_order": bool(args.exact_order),
                       "heavy_threshold": pair.plan_down.heavy_threshold, "narrow_variant": narrow_used,
                       "cuda_graphs": not args.no_graphs, "balance": pair.plan_down.balance, "pad_lists": pair.plan_down.pad_lists,
                       "long_first": pair.plan_down.long_first, "heavy_buckets": pair.plan_down.heavy_buckets, "short_rows": pair.plan_down.short_rows, "slots": {"up": pair.plan_up.slots, "down": pair.plan_down.slots}, "pdl": pair.plan_down.resolve_pdl(k), "narrow_split": pair.plan_down.narrow_split, "fuse_entries": pair.plan_down.fuse_entries,
                       "schedule": pair.plan_down.schedule,
                       "heavy_variant": heavy_used, "autotuned_variants": tuned,
                       "row_order": {"up": "locality" if pair.plan_up.locality(Direction.UP) else "natural",
                                     "down": "locality" if pair.plan_down.locality(Direction.DOWN) else "natural"},
                       "l2": "working set > 126 MB L2 (no flush)", "parallelism": f"replicas x{world} (one graph per GPU)",
                       "vram_budget_frac": args.budget_frac, "streamed_bytes_per_step": int(streamed_bytes),
                       "ring_slots": layout.allocated_ring_buffer_size},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_unit": "DRAM bytes of one launch: up level 1 (level_entry_pre_kernel)",
                         "traffic_source": TRAFFIC_SOURCE if traffic is not None else None,
                         "traffic_launches": traffic_launches, "kernel": ("dataflow traversal (sentinel fill + persistent gather kernel + seed/output), per direction"
                                    if pair.plan_down.schedule == "dataflow" else
                                    "level gathers (one fused narrow+heavy launch per level)"),
                         "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback",
                         "level_ms_per_step": level_total_ms, "level_bytes_per_step": lv_bytes,
                         "launches_in_level_timing": level_launches,
                         "level_ms_per_step_with_events_around_each_launch": per_level_ms or None},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks.summary(),
            "max_rel_err_vs_oracle": max_rel,
            "integer_inputs_vs_oracle": integer_check,
            "k1": k1,
            "tiers": tiers,
            "setup_s": {"generate": gen_s, "runtime_enter": enter_s},
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def measure_xtx_operator(path, device, q: int = 64, applies: int = 5) -> dict:
    """The standardised Gram operator Zᵀ Z (randomized PCA's operator) at block width ``q`` on
    ``path``: device time per application (one down and one up traversal by individual plus
    the three fused FP64 passes around them), CUDA events on the runtime's stream."""
    import torch

    from grg_spmv_b200 import RuntimeRequirements, scan_grg_spmv
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout
    from grg_spmv_b200.xtx import StandardizedXTX

    scan = scan_grg_spmv(path)
    req = RuntimeRequirements(max_k_up=q, max_k_down=q, need_down_miss_input=scan.has_missing_data,
                              need_up_miss_output=scan.has_missing_data, need_init_vector=False, need_init_matrix=False,
                              need_init_xtx=False)
    stream = torch.cuda.Stream(device=device)
    layout = plan_b200_layout(artifacts=[path], dtype=np.float64, requirements=req, vram_budget_bytes=0, ring_buffer_size=0,
                              device=device.index or 0, stream=stream, emit_all_nodes=False)
    with B200Runtime(layout) as rt, torch.cuda.stream(stream):
        (grg,) = rt.grgs
        op = StandardizedXTX(rt, grg, q)
        v = torch.randn((grg.num_mutations, q), dtype=torch.float64, device=device, generator=torch.Generator(device=device).manual_seed(5))
        for _ in range(2):
            op.apply(v)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(applies):
            v = op.apply(v)
            v = v / torch.linalg.vector_norm(v, dim=0, keepdim=True)
        b.record(stream)
        torch.cuda.synchronize(device)
        ms = a.elapsed_time(b) / applies
    del op, rt
    torch.cuda.empty_cache()
    return {"q": q, "applications": applies, "ms_per_application": ms,
            "edge_rhs_per_s": 2.0 * scan.num_edges * q / (ms / 1e3),
            "note": "each application: fused encode pass, down traversal, fused centring pass, up traversal, fused "
                    "finish pass (plus the harness's column normalisation between applications)"}


def multi_grg_specs(count: int, scale: float):
    """``count`` GRGs of the batching configuration's shape (5M-40M edges and 20k-400k
    mutations, evenly spread) from the same generator, each scaled by ``scale``."""
    from grg_spmv_b200.synth import SynthSpec

    specs = []
    for i in range(count):
        f = i / max(count - 1, 1)
        edges = (5e6 + f * 35e6) * scale
        nodes = int(edges / 11.8)  # the generator's edges per node at 40 levels
        specs.append(SynthSpec(num_samples=max(2000, nodes // 50), num_levels=40, num_nodes=nodes,
                               num_mutations=int((20_000 + f * 380_000) * scale), children=(2, 22),
                               miss_fraction=0.01, seed=1000 + i))
    return specs


def make_multi_artifacts(args) -> list[Path]:
    from grg_spmv_b200.synth import write_synthetic_artifact

    root = Path(args.tier_artifacts) if args.tier_artifacts else Path(tempfile.mkdtemp(prefix="grg_tiers_"))
    root.mkdir(parents=True, exist_ok=True)
    jobs, paths = [], []
    for i, spec in enumerate(multi_grg_specs(args.tier_grgs, args.tier_scale)):
        path = root / f"multi_{args.tier_scale:g}_{i}.grg_spmv"
        if not path.exists():
            jobs.append((spec, str(path)))
        paths.append(path)
    # The graphs are independent: a few spawned processes generate them (about 3 GB of host
    # memory each at 40M edges).
    workers = min(len(jobs), 4, max(1, (os.cpu_count() or 1) // 2))
    if workers > 1:
        import multiprocessing

        with multiprocessing.get_context("spawn").Pool(workers) as pool:
            pool.starmap(write_synthetic_artifact, jobs)
    else:
        for spec, path in jobs:
            write_synthetic_artifact(spec, Path(path))
    return paths


def measure_tiers(args, paths, device, stream, block_sets) -> list[dict]:
    """Uneven RHS blocks on every graph of ``paths``, three ways, same work (sum of blocks, up
    and down, every graph): the plain FP64 drop-in (one prepared op per block, direction and
    graph, one after another), a plain FP64 batch (one CUDA graph: blocks of a graph merged and
    tiled, graphs on concurrent streams, autotuned) and a mixed-precision batch.  Device time
    with CUDA events; errors of each batch against the FP64 drop-in's outputs and, for the
    blocks of width <= 3 on the first graph, against the CPU oracle.  One result per block set
    of ``block_sets``, all on one runtime."""
    import torch

    from grg_spmv_b200 import RuntimeRequirements
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout

    kmax = max(max(b) for b in block_sets)
    req = RuntimeRequirements(max_k_up=kmax, max_k_down=kmax, need_down_miss_input=True, need_up_miss_output=False,
                              need_init_vector=False, need_init_matrix=False, need_init_xtx=False)
    layout = plan_b200_layout(artifacts=[str(p) for p in paths], dtype=np.float64, requirements=req, vram_budget_bytes=0,
                              ring_buffer_size=0, device=device.index or 0, stream=stream)
    rng = np.random.default_rng(7)
    rel = lambda got, ref: float(np.max(np.abs(got - ref)) / max(float(np.max(np.abs(ref))), 1e-300))
    oracle = None
    results = []
    with B200Runtime(layout) as rt, torch.cuda.device(device), torch.cuda.stream(stream):
        def timed(step) -> float:
            for _ in range(max(args.warmup, 3)):
                step()
            torch.cuda.synchronize(device)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.tier_steps):
                step()
            b.record(stream)
            torch.cuda.synchronize(device)
            return a.elapsed_time(b) / args.tier_steps

        for blocks in block_sets:
            out = {"blocks": list(blocks), "steps": args.tier_steps, "warmup": max(args.warmup, 3)}
            items = []
            for g in rt.grgs:
                items += [(g, "up", kb) for kb in blocks] + [(g, "down", kb, True) for kb in blocks]
            xs, misses = [], []
            for it in items:
                g = it[0]
                cols = g.num_samples if it[1] == "up" else g.num_mutations
                xs.append(torch.from_numpy(rng.standard_normal((it[2], cols))).to(device))
                misses.append(torch.from_numpy(rng.standard_normal((it[2], g.num_mutations))).to(device) if it[1] == "down" else None)
            work = 2.0 * sum(g.num_edges for g in rt.grgs) * sum(blocks)
            out["graphs"] = [{"num_edges": g.num_edges, "num_nodes": g.num_nodes, "num_mutations": g.num_mutations}
                             for g in rt.grgs]
            # 1) plain FP64 drop-in: one prepared op per block and direction.
            ops = [it[0].prepare_matmul_cuda(direction=it[1], k=it[2], use_miss=it[1] == "down") for it in items]
            plain_out = [None] * len(items)

            def dropin_step(keep=False):
                for i, op in enumerate(ops):
                    op.input.copy_(xs[i])
                    if misses[i] is not None:
                        op.miss_input.copy_(misses[i])
                    op()
                    if keep:
                        plain_out[i] = op.output.cpu().numpy()

            ms = timed(dropin_step)
            dropin_step(keep=True)
            out["plain_f64_dropin"] = {"value": work / (ms / 1e3), "ms_per_step": ms, "launch": "one prepared op per block"}
            del ops
            small = [i for i, it in enumerate(items) if it[2] <= 3 and it[0] is rt.grgs[0]]
            refs = {}
            if small and not args.no_cpu_baseline:
                if oracle is None:
                    sys.path.insert(0, str(REPO / "oracle"))
                    from grg_oracle import OracleGRG

                    oracle = OracleGRG(paths[0])
                for i in small:
                    m_np = misses[i].cpu().numpy() if misses[i] is not None else None
                    refs[i] = oracle.matmul(xs[i].cpu().numpy(), items[i][1], miss=m_np)
                out["plain_f64_dropin"]["max_rel_err_vs_oracle_blocks_le3"] = max(rel(plain_out[i], refs[i]) for i in refs)
            # 2) and 3) batches.
            for name, precision in (("plain_f64_batched", "plain"), ("mixed_batched", "mixed")):
                with rt.prepare_batch(items, precision=precision, autotune=True) as batch:
                    def batch_step():
                        for i in range(len(items)):
                            batch.inputs[i].copy_(xs[i])
                            if misses[i] is not None:
                                batch.miss_inputs[i].copy_(misses[i])
                        batch()

                    ms_b = timed(batch_step)
                    batch_step()
                    torch.cuda.synchronize(device)
                    errs = [rel(batch.outputs[i].cpu().numpy(), plain_out[i]) for i in range(len(items))]
                    out[name] = {"value": work / (ms_b / 1e3), "ms_per_step": ms_b, "tile_k": batch.tile_k,
                                 "tiles": batch.num_tiles, "tuned_ms": {str(k): v for k, v in batch.tuned_ms.items()},
                                 "max_rel_err_vs_plain_f64": max(errs), "speedup_vs_dropin": ms / ms_b}
                    if refs:
                        out[name]["max_rel_err_vs_oracle_blocks_le3"] = max(rel(batch.outputs[i].cpu().numpy(), refs[i])
                                                                            for i in refs)
                torch.cuda.empty_cache()
            out["workload"] = (f"{len(paths)} graph(s); RHS blocks {list(blocks)} in both directions on each (down with "
                               f"miss rows), inputs copied into the op/batch buffers every step")
            results.append(out)
            del xs, misses, plain_out
            torch.cuda.empty_cache()
    return results


_WORKER_ORACLE = None


def _oracle_worker_init(path: str) -> None:
    global _WORKER_ORACLE
    sys.path.insert(0, str(REPO / "oracle"))
    from grg_oracle import OracleGRG

    _WORKER_ORACLE = OracleGRG(path)


def _oracle_worker_step(task):
    x, miss = task
    mid = _WORKER_ORACLE.matmul(x, "up")
    return mid, _WORKER_ORACLE.matmul(mid, "down", miss=miss.copy())


class ParallelOracle:
    """The oracle (the reference's single-threaded ReferenceRuntime arithmetic) on all host
    cores: right-hand-side columns are independent, so each of ``workers`` spawned processes
    runs the reference algorithm on a slice of the columns."""

    def __init__(self, path, workers: int) -> None:
        import multiprocessing

        self.workers = max(1, int(workers))
        self.pool = multiprocessing.get_context("spawn").Pool(self.workers, initializer=_oracle_worker_init,
                                                              initargs=(str(path),))

    def step(self, x: np.ndarray, miss: np.ndarray):
        parts = [p for p in np.array_split(np.arange(x.shape[0]), min(self.workers, x.shape[0])) if p.size]
        res = self.pool.map(_oracle_worker_step, [(x[p], miss[p]) for p in parts])
        return np.concatenate([r[0] for r in res]), np.concatenate([r[1] for r in res])

    def close(self) -> None:
        self.pool.close()
        self.pool.join()


def run_reference(args) -> None:
    """The reference's CPU path (oracle port of ReferenceRuntime) on the same workload, on all
    host cores (one process per right-hand-side column, up to the core count)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from grg_spmv_b200.artifact import scan_grg_spmv

    path, _ = make_artifact(args, 0)
    with np.load(path) as data:
        S, M, E = (int(np.asarray(data[key]).item()) for key in ("num_samples", "num_mutations", "num_edges"))
    k = int(args.k)
    workers = min(k, os.cpu_count() or 1)
    rng = np.random.default_rng(100)
    x = rng.standard_normal((k, S))
    miss = rng.choice(np.asarray([0.0, 1.0]), size=(k, M), p=[0.99, 0.01])
    oracle = ParallelOracle(path, workers)
    try:
        for _ in range(max(args.warmup, 1)):  # the first step also waits for the workers to load the graph
            oracle.step(x, miss)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            oracle.step(x, miss)
        secs = time.perf_counter() - t0
    finally:
        oracle.close()
    value = args.steps * 2.0 * E * k / secs
    sample = (f"full up+down steps (k={k}) of the same graph; SciPy restatement of ReferenceRuntime, "
              f"{workers} processes x 1 thread, RHS columns split across them")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_description(args.workload, scan_grg_spmv(path), streamed=False), "k": k,
                   "precision": "plain", "num_samples": S, "num_edges": E, "num_mutations": M},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample, **host_info(workers)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def large_spec(scale: float):
    """The streamed large configuration (1M haploid samples, 60 internal levels, 60M nodes,
    ~600M edges, 20M mutations) from the same generator, every count times ``scale``."""
    from grg_spmv_b200.synth import SynthSpec

    return SynthSpec(num_samples=int(1_000_000 * scale), num_levels=60, num_nodes=int(60_000_000 * scale),
                     num_mutations=int(20_000_000 * scale), children=(2, 22), seed=0)


def run_apps(args) -> None:
    """Application harnesses on one GPU, one JSON line, both on a graph of the large
    configuration's shape scaled by ``--apps-scale``.

    * ``pca``: randomized PCA (``randomized_eigh``: 10 power iterations of Zᵀ(Z V) with a block
      of 64 vectors, FP64 QR and Rayleigh-Ritz), with the node state in plain FP64 and in the
      mixed format; eigenvalue agreement between the two.
    * ``cg``: block CG on (Z Zᵀ / M + 0.5 I) x = b, 16 right-hand sides, 50 iterations, FP64
      dot products and residuals: fully resident in plain FP64 (the reference solution), then
      under a VRAM budget of 16 GB x scale with 4 ring slots, so the largest level lists stream
      from pinned host memory every traversal, in plain FP64 and with the mixed node state.
    Each timed region is bracketed by device synchronisation (CUDA events on the runtime's
    stream plus the host clock: CG reads its residuals on the host every iteration, as the
    reference's solver does)."""
    import torch

    from grg_spmv_b200 import RuntimeRequirements, scan_grg_spmv
    from grg_spmv_b200.synth import write_synthetic_artifact

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)

    def requirements(q):
        miss = bool(scan.has_missing_data)
        return RuntimeRequirements(max_k_up=q, max_k_down=q, need_down_miss_input=miss, need_up_miss_output=miss,
                                   need_init_vector=False, need_init_matrix=False, need_init_xtx=False)

    def timed(stream, fn):
        torch.cuda.synchronize(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        res = fn()
        b.record(stream)
        torch.cuda.synchronize(device)
        return res, a.elapsed_time(b), (time.perf_counter() - t0) * 1e3

    out = {"metric": "GRG application harnesses (randomized PCA, block CG)", "n_gpus": 1, "data": "synthetic",
           "dtype": "f64 (plain) / f64 sums with f32+i16 node state (mixed)"}

    # The large configuration's graph (no missingness: the configuration states none, and the
    # generator draws each mutation's missingness node independently of its carriers, so an
    # allele frequency over non-missing samples could exceed 1 and its 1/sqrt(p(1-p)) scale be NaN).
    if args.apps_only == "precision":
        out["precision"] = run_precision(args, timed, device)
        print(json.dumps(out))
        return
    scale = float(args.apps_scale)
    path = Path(args.apps_artifact) if args.apps_artifact else Path(tempfile.mkdtemp(prefix="grg_apps_")) / f"large_{scale:g}.grg_spmv"
    gen_s = 0.0
    if not path.exists():
        t0 = time.perf_counter()
        write_synthetic_artifact(large_spec(scale), path)
        gen_s = time.perf_counter() - t0
    scan = scan_grg_spmv(path)

    if args.apps_only == "all":
        out["precision"] = run_precision(args, timed, device)
    if args.apps_only in ("all", "pca"):
        out["pca"] = run_pca(args, path, scan, gen_s, requirements, timed, device)
    if args.apps_only in ("all", "cg"):
        out["cg"] = run_cg(args, path, scan, gen_s, scale, requirements, timed, device)
    print(json.dumps(out))


def run_precision(args, timed, device) -> dict:
    """The precision configuration: the config-2 graph in its diploid variant with coalescence
    counts, k = 32, up and down with init_xtx (the 2·coalescence-count node initialisation and
    its endpoint bias, in FP64), N(0,1) and integer allele-count (0, 1, 2) inputs.  The node
    state in plain FP64 and in the mixed format (FP32 + 16-bit correction, FP64 sums); device
    time per up+down pair and the max relative error of each against the CPU oracle (FP64, the
    reference's arithmetic) on the first 4 of the 32 columns, and of mixed against plain FP64 on
    all 32."""
    import torch

    from grg_spmv_b200 import RuntimeRequirements
    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout
    from grg_spmv_b200.synth import CONFIG2, write_synthetic_artifact

    tmpdir = None if args.precision_artifact else Path(tempfile.mkdtemp(prefix="grg_prec_"))
    path = Path(args.precision_artifact) if args.precision_artifact else tmpdir / "config2_diploid.grg_spmv"
    gen_s = 0.0
    if not path.exists():
        t0 = time.perf_counter()
        write_synthetic_artifact(dataclasses.replace(CONFIG2, ploidy=2, with_coalescence=True, seed=0), path)
        gen_s = time.perf_counter() - t0
    k, check_cols = 32, 4
    req = RuntimeRequirements(max_k_up=k, max_k_down=k, need_down_miss_input=False, need_up_miss_output=False,
                              need_init_vector=False, need_init_matrix=False, need_init_xtx=True)
    rng = np.random.default_rng(21)
    out = {"graph": {"path_kind": "config-2 generator, ploidy 2, coalescence counts", "generate_s": gen_s}, "k": k,
           "init": "xtx", "oracle_columns": check_cols}
    results = {}
    for precision in ("plain", "mixed"):
        stream = torch.cuda.Stream(device=device)
        layout = plan_b200_layout(artifacts=[path], dtype=np.float64, requirements=req, vram_budget_bytes=0, ring_buffer_size=0,
                                  device=0, stream=stream, precision=precision, emit_all_nodes=False)
        with B200Runtime(layout) as rt, torch.cuda.stream(stream):
            (grg,) = rt.grgs
            out["graph"].update(num_edges=grg.num_edges, num_nodes=grg.num_nodes, num_mutations=grg.num_mutations,
                                num_samples=grg.num_samples, ploidy=grg.ploidy)
            if "inputs" not in results:
                results["inputs"] = {
                    "normal": (rng.standard_normal((k, grg.num_samples)), rng.standard_normal((k, grg.num_mutations))),
                    "allele_counts": (rng.integers(0, 3, (k, grg.num_samples)).astype(np.float64),
                                      rng.integers(0, 3, (k, grg.num_mutations)).astype(np.float64)),
                }
            up = grg.prepare_matmul_cuda(direction="up", k=k, init_mode="xtx")
            down = grg.prepare_matmul_cuda(direction="down", k=k, init_mode="xtx")
            x_up = torch.from_numpy(results["inputs"]["normal"][0]).to(device)
            x_dn = torch.from_numpy(results["inputs"]["normal"][1]).to(device)

            def pair():
                up.input.copy_(x_up)
                up()
                down.input.copy_(x_dn)
                down()

            for _ in range(3):
                pair()
            _, ms, _ = timed(stream, lambda: [pair() for _ in range(5)])
            out[precision] = {"ms_per_up_down": ms / 5, "edge_rhs_per_s": 2.0 * grg.num_edges * k / (ms / 5 / 1e3)}
            for name, (xu, xd) in results["inputs"].items():
                results[(precision, name)] = (grg.matmul(xu, "up", init="xtx"), grg.matmul(xd, "down", init="xtx"))
        del up, down, rt
        torch.cuda.empty_cache()
    sys.path.insert(0, str(REPO / "oracle"))
    from grg_oracle import OracleGRG

    oracle = OracleGRG(path)
    rel = lambda got, ref: float(np.max(np.abs(got - ref)) / max(float(np.max(np.abs(ref))), 1e-300))
    for name, (xu, xd) in results["inputs"].items():
        ref_up = oracle.matmul(xu[:check_cols], "up", init="xtx")
        ref_dn = oracle.matmul(xd[:check_cols], "down", init="xtx")
        for precision in ("plain", "mixed"):
            got_up, got_dn = results[(precision, name)]
            out[precision][f"max_rel_err_vs_oracle_{name}"] = max(rel(got_up[:check_cols], ref_up), rel(got_dn[:check_cols], ref_dn))
        m_up, m_dn = results[("mixed", name)]
        p_up, p_dn = results[("plain", name)]
        out["mixed"][f"max_rel_err_vs_plain_f64_{name}"] = max(rel(m_up, p_up), rel(m_dn, p_dn))
    if tmpdir is not None:  # the generated graph is this call's own
        shutil.rmtree(tmpdir, ignore_errors=True)
    return out


def run_pca(args, path, scan, gen_s, requirements, timed, device) -> dict:
    """Randomized PCA timing (see ``run_apps``)."""
    import torch

    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout
    from grg_spmv_b200.xtx import StandardizedXTX, randomized_eigh

    pcs, over, power = 16, 48, 10
    q = pcs + over
    pca = {"graph": {"num_edges": scan.num_edges, "num_nodes": scan.num_nodes, "num_mutations": scan.num_mutations,
                     "num_samples": scan.num_samples, "generate_s": gen_s},
           "block": q, "pcs": pcs, "power_iters": power}
    eig = {}
    for precision in ("plain", "mixed"):
        stream = torch.cuda.Stream(device=device)
        layout = plan_b200_layout(artifacts=[path], dtype=np.float64, requirements=requirements(q), vram_budget_bytes=0,
                                  ring_buffer_size=0, device=0, stream=stream, precision=precision, emit_all_nodes=False)
        with B200Runtime(layout) as rt, torch.cuda.stream(stream):
            (grg,) = rt.grgs
            op = StandardizedXTX(rt, grg, q)
            randomized_eigh(op, pcs, oversample=over, power_iters=1, seed=3)  # warm-up (graph capture, tuning)
            (values, _), ms, wall_ms = timed(stream, lambda: randomized_eigh(op, pcs, oversample=over, power_iters=power, seed=3))
            applies = power + 2
            work = applies * 2.0 * grg.num_edges * q
            eig[precision] = values.cpu().numpy()
            v = torch.randn((grg.num_mutations, q), dtype=torch.float64, device=device)
            _, apply_ms, _ = timed(stream, lambda: [op.apply(v) for _ in range(3)])
            pca[precision] = {"ms": ms, "wall_ms": wall_ms, "operator_applies": applies, "ms_per_operator_apply": apply_ms / 3,
                              "edge_rhs_per_s": work / (ms / 1e3), "top_eigenvalues": [float(v) for v in eig[precision][:4]]}
        del op, rt
        torch.cuda.empty_cache()
    pca["max_rel_eigenvalue_diff_mixed_vs_plain"] = float(np.max(np.abs(eig["mixed"] - eig["plain"]) / np.abs(eig["plain"])))
    return pca


def run_cg(args, cg_path, scan, gen_s, scale, requirements, timed, device) -> dict:
    """Block CG with the largest level lists streamed (see ``run_apps``)."""
    import torch

    from grg_spmv_b200.backends.b200 import B200Runtime, plan_b200_layout
    from grg_spmv_b200.xtx import StandardizedXXT, conj_grad_solve

    # delta = 0.5 is LMM-like (h2 about 2/3); this graph's kinship has top eigenvalues near 8e3,
    # so that system is far from converged after 50 iterations and CG amplifies rounding
    # differences between precisions.  delta = 200 converges within the 50 iterations and is
    # the one whose solutions are compared across precisions.
    c, iters, delta, delta_conv = 16, 50, 0.5, 200.0
    budget = int(16e9 * scale)
    cg = {"graph": {"num_edges": scan.num_edges, "num_nodes": scan.num_nodes, "num_mutations": scan.num_mutations,
                    "num_samples": scan.num_samples, "num_levels": scan.num_levels, "scale_vs_configuration": scale,
                    "generate_s": gen_s},
          "rhs": c, "iterations": iters, "delta": delta, "delta_converging": delta_conv}
    rng = np.random.default_rng(11)
    b_np = rng.standard_normal((scan.num_samples, c))  # haploid: individuals = samples
    sols, applied, conv = {}, {}, {}

    def plan(precision, vram, ring, stream=0):
        return plan_b200_layout(artifacts=[cg_path], dtype=np.float64, requirements=requirements(c), vram_budget_bytes=vram,
                                ring_buffer_size=ring, device=0, stream=stream, precision=precision, emit_all_nodes=False)

    def fixed_bytes(precision):  # everything but the level lists
        full = plan(precision, 0, 0)
        return full.bytes_total - full.bytes_by_category["resident_sparse"]

    # The configuration's budget applies to the plain FP64 layout; the mixed layout gets the same
    # room for level lists (its node state is smaller but it adds encoded down-input rows).
    mixed_budget = budget + fixed_bytes("mixed") - fixed_bytes("plain")
    variants = (("plain_f64_resident", "plain", 0, 0), ("plain_f64_streamed", "plain", budget, 4),
                ("mixed_streamed", "mixed", mixed_budget, 4))
    for name, precision, vram, ring in variants:
        stream = torch.cuda.Stream(device=device)
        layout = plan(precision, vram, ring, stream)
        streamed = sum(lp.nbytes for lp in layout.level_plans() if not lp.resident)
        lists = sum(lp.nbytes for lp in layout.level_plans())
        t0 = time.perf_counter()
        with B200Runtime(layout) as rt, torch.cuda.stream(stream):
            enter_s = time.perf_counter() - t0
            (grg,) = rt.grgs
            op = StandardizedXXT(rt, grg, c)
            M = grg.num_mutations
            b = torch.from_numpy(b_np).to(device)
            matvec = lambda v: op.apply(v) / M + delta * v
            conj_grad_solve(matvec, b, rel_tol=0.0, max_iter=2)  # warm-up
            (x, it, rels), ms, wall_ms = timed(stream, lambda: conj_grad_solve(matvec, b, rel_tol=0.0, max_iter=iters))
            sols[name] = x.cpu().numpy()
            applied[name] = op.apply(b).cpu().numpy()  # one Z Zᵀ b
            x_c, _, rels_c = conj_grad_solve(lambda v: op.apply(v) / M + delta_conv * v, b, rel_tol=0.0, max_iter=iters)
            conv[name] = x_c.cpu().numpy()
            work = it * 2.0 * grg.num_edges * c
            cg[name] = {"ms": ms, "wall_ms": wall_ms, "ms_per_iteration": ms / it, "iterations": it,
                        "edge_rhs_per_s": work / (ms / 1e3), "max_rel_residual": float(rels.max()),
                        "vram_budget_bytes": vram, "ring_slots": layout.allocated_ring_buffer_size,
                        "bytes_total": int(layout.bytes_total), "level_list_bytes": int(lists),
                        "streamed_list_bytes_per_iteration": int(streamed),
                        "streamed_gb_per_s": streamed * it / (ms / 1e3) / 1e9, "runtime_enter_s": enter_s,
                        "max_rel_residual_delta_converging": float(rels_c.max())}
        del op, rt
        torch.cuda.empty_cache()
    rel = lambda got, ref: float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    for name in ("plain_f64_streamed", "mixed_streamed"):
        cg[name]["operator_max_rel_diff_vs_plain_resident"] = rel(applied[name], applied["plain_f64_resident"])
        cg[name]["solution_max_rel_diff_vs_plain_resident"] = rel(sols[name], sols["plain_f64_resident"])
        cg[name]["solution_max_rel_diff_vs_plain_resident_delta_converging"] = rel(conv[name], conv["plain_f64_resident"])
    return cg


def main() -> None:
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.apps:
        run_apps(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
