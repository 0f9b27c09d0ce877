"""Seeded synthetic GRGs with the shapes of the benchmark configurations.

There is no public GRG dataset available offline, so benchmarks and tests use generated
graphs.  Construction (level by level, vectorised):

* Samples sit at random positions ``0..S-1`` of a line.  Every node covers an interval
  ``[a, b)`` of positions; its sample set is the samples in that interval.
* A level-``L`` node starts from an *anchor* child drawn from level ``L-1`` and grows by
  appending ``c-1`` further children, each an existing node whose interval abuts the
  current union on the left or right and whose length is at most a random fraction of the
  anchor's.  Children therefore have pairwise disjoint sample sets, so an all-ones ``up``
  traversal returns descendant-sample counts ``<= S`` (no duplicate sample paths), and
  nodes are shared by many parents (a DAG, not a forest).
* ``c`` is uniform in ``children``; a node's stable level is exactly ``L`` because the
  anchor is at ``L-1`` and every other child is lower.
* Mutations attach to nodes whose descendant count follows a ``1/x`` site-frequency
  spectrum; with ``miss_fraction > 0`` every mutation also gets a missingness node covering
  about that fraction of the samples.
* Original node ids are topological (children before parents) but not level-sorted, so the
  compiled stable height order is a non-trivial permutation; within a level, nodes are
  ordered by interval start (positional locality, as in sequentially built GRGs).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from grg_spmv_b200.artifact import CompiledOperatorState, save_grg_spmv
from grg_spmv_b200.compile import DagGRG, build_init_biases, compile_dag


@dataclass(frozen=True)
class SynthSpec:
    num_samples: int
    num_levels: int  # internal levels (the compiled GRG has num_levels + 1 levels)
    num_nodes: int  # target total node count, samples included
    num_mutations: int
    children: tuple[int, int] = (2, 8)
    neighbor_scale: float = 0.08  # abutting children are at most ~this fraction of the anchor
    prefer_largest: float = 0.7  # probability of taking the longest fitting neighbor
    level_decay: float = 1.0
    miss_fraction: float = 0.0
    ploidy: int = 1
    with_coalescence: bool = False
    random_ids: bool = False  # random topological original ids (non-identity stable order)
    seed: int = 0


# Shapes of the benchmark configurations: CONFIG1 the reference's CPU-runnable case (S = 2k,
# 16 levels), CONFIG2 the plain-FP64 drop-in case (S = 100k, 40 levels, 5M nodes; the
# generator gives E = 58.8M for it).
CONFIG1 = SynthSpec(num_samples=2_000, num_levels=16, num_nodes=80_000, num_mutations=20_000, children=(2, 8), seed=0)
CONFIG2 = SynthSpec(num_samples=100_000, num_levels=40, num_nodes=5_000_000, num_mutations=1_000_000,
                    children=(2, 22), miss_fraction=0.01, seed=0)


def _level_sizes(spec: SynthSpec) -> np.ndarray:
    internal = max(int(spec.num_nodes) - int(spec.num_samples), spec.num_levels)
    weights = np.exp(-spec.level_decay * np.arange(spec.num_levels) / max(spec.num_levels - 1, 1))
    sizes = np.maximum(np.floor(weights / weights.sum() * internal).astype(np.int64), 1)
    sizes[0] += internal - int(sizes.sum())
    return sizes


class _IntervalIndex:
    """Nodes sorted by (boundary position, length) for 'abutting node no longer than cap' queries.

    Keys are kept sorted; each level's new nodes are merged in with one insert.
    """

    def __init__(self, span: int):
        self.span = np.int64(span + 1)
        self.key = np.empty(0, dtype=np.int64)
        self.ids = np.empty(0, dtype=np.int64)

    def add(self, bound: np.ndarray, length: np.ndarray, first_id: int) -> None:
        key = bound.astype(np.int64) * self.span + length.astype(np.int64)
        order = np.argsort(key, kind="stable")
        key = key[order]
        at = np.searchsorted(self.key, key, side="right")
        self.key = np.insert(self.key, at, key)
        self.ids = np.insert(self.ids, at, first_id + order)

    def _search(self, needles: np.ndarray, side: str) -> np.ndarray:
        # Sorted needles let searchsorted reuse the previous bound (far fewer cache misses).
        order = np.argsort(needles)
        out = np.empty(needles.size, dtype=np.int64)
        out[order] = np.searchsorted(self.key, needles[order], side=side)
        return out

    def pick(self, rng, bound: np.ndarray, cap: np.ndarray, largest: float) -> np.ndarray:
        """An abutting node no longer than ``cap``: with probability ``largest`` the longest
        such node (which tends to come from a recent level), otherwise a uniform one."""
        base = bound.astype(np.int64) * self.span
        lo = self._search(base + 1, "left")
        hi = self._search(base + cap.astype(np.int64), "right")
        hi = np.maximum(hi, lo + 1)  # the single-sample node (length 1) always qualifies
        uniform = lo + (rng.random(lo.size) * (hi - lo)).astype(np.int64)
        if largest <= 0.0:  # uniform picks only (no second draw, so seeds give the same DAGs as before the option)
            return self.ids[uniform]
        return self.ids[np.where(rng.random(lo.size) < largest, hi - 1, uniform)]


def generate_dag(spec: SynthSpec) -> DagGRG:
    rng = np.random.default_rng(spec.seed)
    S = int(spec.num_samples)
    sample_pos = rng.permutation(S).astype(np.int64)  # position of sample s
    start = [sample_pos]
    end = [sample_pos + 1]
    level = [np.zeros(S, dtype=np.int64)]
    child_lists: list[np.ndarray] = []  # per level: (n_L, cmax) padded with -1, in creation ids
    sizes = _level_sizes(spec)
    cmin, cmax = int(spec.children[0]), int(spec.children[1])
    level_first = [0, S]
    by_start = _IntervalIndex(S)
    by_end = _IntervalIndex(S)
    all_start = sample_pos.copy()
    all_end = sample_pos + 1
    by_start.add(all_start, np.ones(S, np.int64), 0)
    by_end.add(all_end, np.ones(S, np.int64), 0)
    for L in range(1, spec.num_levels + 1):
        prev_lo, prev_hi = level_first[L - 1], level_first[L]
        n = int(sizes[L - 1])
        anchor = rng.integers(prev_lo, prev_hi, size=n)
        a = all_start[anchor].copy()
        b = all_end[anchor].copy()
        target = rng.integers(cmin, cmax + 1, size=n)
        kids = np.full((n, cmax), -1, dtype=np.int64)
        kids[:, 0] = anchor
        anchor_len = (b - a).astype(np.float64)
        for step in range(1, cmax):
            active = (step < target) & ((a > 0) | (b < S))
            if not np.any(active):
                break
            idx = np.flatnonzero(active)
            go_right = rng.random(idx.size) < 0.5
            go_right = np.where(b[idx] >= S, False, np.where(a[idx] <= 0, True, go_right))
            cap = np.maximum(1, (anchor_len[idx] * spec.neighbor_scale * rng.random(idx.size) ** 2).astype(np.int64))
            right = idx[go_right]
            left = idx[~go_right]
            if right.size:
                pick = by_start.pick(rng, b[right], cap[go_right], spec.prefer_largest)
                kids[right, step] = pick
                b[right] = all_end[pick]
            if left.size:
                pick = by_end.pick(rng, a[left], cap[~go_right], spec.prefer_largest)
                kids[left, step] = pick
                a[left] = all_start[pick]
        # Order the level's nodes by interval start for positional locality.
        order = np.argsort(a, kind="stable")
        a, b = a[order], b[order]
        start.append(a)
        end.append(b)
        level.append(np.full(n, L, dtype=np.int64))
        child_lists.append(kids[order])
        by_start.add(a, b - a, level_first[-1])
        by_end.add(b, b - a, level_first[-1])
        all_start = np.concatenate((all_start, a))
        all_end = np.concatenate((all_end, b))
        level_first.append(level_first[-1] + n)

    N = level_first[-1]
    all_start = np.concatenate(start)
    all_end = np.concatenate(end)
    all_level = np.concatenate(level)
    # Original ids: samples first, then internal nodes ordered by a key that is always larger
    # than every child's key (so ids are topological).  By default the key is level + start/S,
    # giving level-sorted ids with positional order inside a level; with ``random_ids`` it is
    # max(child keys) + U(0,1), which interleaves levels and shuffles nodes within a level.
    if spec.random_ids:
        node_key = np.zeros(N, dtype=np.float64)
        for L, kids in enumerate(child_lists, start=1):
            lo, hi = level_first[L], level_first[L + 1]
            child_keys = np.where(kids >= 0, node_key[np.maximum(kids, 0)], -1.0)
            node_key[lo:hi] = child_keys.max(axis=1) + rng.random(hi - lo)
        key = node_key[S:]
    else:
        key = all_level[S:] + all_start[S:] / (S + 1.0)
    internal_order = np.argsort(key, kind="stable")
    new_id = np.empty(N, dtype=np.int64)
    new_id[:S] = np.arange(S)
    new_id[S + internal_order] = S + np.arange(N - S)

    kids_all = np.concatenate(child_lists, axis=0)  # rows in creation order of internal nodes
    counts = (kids_all >= 0).sum(axis=1)
    rows_by_new = np.empty(N - S, dtype=np.int64)
    rows_by_new[new_id[S:] - S] = np.arange(N - S)
    kids_new = kids_all[rows_by_new]
    counts_new = counts[rows_by_new]
    child_indptr = np.zeros(N + 1, dtype=np.int64)
    child_indptr[S + 1:] = np.cumsum(counts_new)
    flat = kids_new[kids_new >= 0]
    child_indices = new_id[flat]
    levels_new = np.empty(N, dtype=np.int64)
    levels_new[new_id] = all_level
    lengths_new = np.empty(N, dtype=np.int64)
    lengths_new[new_id] = all_end - all_start

    # Mutations: descendant counts ~ 1/x (log-uniform on [1, S]).
    M = int(spec.num_mutations)
    length_order = np.lexsort((rng.random(N), lengths_new))
    sorted_len = lengths_new[length_order]

    def nodes_with_length(target_len: np.ndarray) -> np.ndarray:
        jitter = rng.random(target_len.size)
        lo = np.searchsorted(sorted_len, np.floor(target_len), side="left")
        hi = np.searchsorted(sorted_len, np.ceil(target_len * 1.25) + 1, side="right")
        hi = np.maximum(hi, lo + 1)
        pos = np.minimum(lo + (jitter * (hi - lo)).astype(np.int64), N - 1)
        return length_order[pos]

    mut_node = nodes_with_length(np.exp(rng.random(M) * np.log(S)))
    miss_node = np.full(M, -1, dtype=np.int64)
    if spec.miss_fraction > 0:
        miss_node = nodes_with_length(np.full(M, max(1.0, spec.miss_fraction * S)))
    positions = np.sort(rng.random(M) * 1e8).astype(np.float64)
    coal = None
    if spec.with_coalescence:
        # Synthetic per-node individual-coalescence counts: small non-negative integers on
        # internal nodes (0 on samples), used only as the xtx initialisation payload.
        coal = np.zeros(N, dtype=np.int64)
        coal[S:] = rng.poisson(0.5, size=N - S)
    return DagGRG(
        num_samples=S,
        num_nodes=N,
        child_indptr=child_indptr,
        child_indices=child_indices,
        mut_node=mut_node,
        miss_node=miss_node,
        ploidy=int(spec.ploidy),
        coalescence_counts=coal,
        mutation_positions=positions,
        node_levels=levels_new,
    )


def generate_state(spec: SynthSpec, dtype=np.float64) -> CompiledOperatorState:
    state = compile_dag(generate_dag(spec))
    build_init_biases(state, dtype)
    return state


def write_synthetic_artifact(spec: SynthSpec, path, dtype=np.float64):
    state = generate_state(spec, dtype)
    save_grg_spmv(state, path)
    return path


__all__ = ["CONFIG1", "CONFIG2", "SynthSpec", "generate_dag", "generate_state", "write_synthetic_artifact"]
