"""CPU model of the B200 kernels' arithmetic (test utility, small graphs only).

It walks the same gather lists the CUDA kernels walk (``structures.py``) and sums each row
left to right with a fresh partial sum per flagged segment, in the artifact's dtype, so the
structure ordering can be checked against the reference's golden outputs without a GPU.
"""

from __future__ import annotations

import numpy as np

from grg_spmv_b200.artifact import iter_artifact_blocks, load_grg_spmv_header
from grg_spmv_b200.backends.b200 import _native as nat
from grg_spmv_b200.backends.b200.structures import build_down_levels, build_up_levels, load_blocks


def _row_sum(codes, state, x, miss, acc):
    seg = np.zeros_like(acc)
    for code in codes:
        code = int(code)
        if code & nat.SEG_START:
            acc = acc + seg
            seg = np.zeros_like(acc)
        src = (code >> nat.SRC_SHIFT) & 3
        i = code & nat.ID_MASK
        if src == nat.SRC_STATE:
            seg = seg + state[i]
        elif src == nat.SRC_INPUT:
            seg = seg + x[i]
        elif src == nat.SRC_MISS and miss is not None:
            seg = seg + miss[i]
    return acc + seg


def model_matmul(path, x, direction, dtype=np.float64, *, init=None, miss=None, by_individual=False, emit_all_nodes=False):
    st = load_grg_spmv_header(path, dtype)
    coo = load_blocks(iter_artifact_blocks(path))
    off = np.asarray(st.level_offsets, dtype=np.int64)
    k = x.shape[0]
    dt = np.dtype(dtype)
    xi = np.ascontiguousarray(x.T.astype(dt))
    init_mode = "none" if init is None else ("xtx" if isinstance(init, str) else ("vector" if init.ndim == 1 else "matrix"))
    backend = init_mode if (emit_all_nodes or init_mode == "matrix") else "none"

    def init_row(r):
        if backend == "vector":
            return init.astype(dt).copy()
        if backend == "xtx":
            return np.full(k, 2.0 * st.coalescence_counts[r], dtype=dt)
        if backend == "matrix":
            return init[:, int(st.node_perm[r])].astype(dt).copy()
        return np.zeros(k, dtype=dt)

    state = np.zeros((st.num_nodes, k), dtype=dt)
    if direction == "up":
        s2i = np.asarray(st.sample_to_individual)
        for r in range(int(off[1])):
            v = init_row(r)
            if r < st.num_samples:
                v = v + xi[s2i[r] if by_individual else r]
            state[r] = v
        for lv in build_up_levels(off, coo, 1 << 30, locality=True, pad=True):
            for r, codes in lv.row_lists():
                state[lv.row_begin + r] = _row_sum(codes, state, xi, None, init_row(lv.row_begin + r))
    else:
        sel_mut = (st.sel_mut.indptr, st.sel_mut.indices, st.num_mutations)
        sel_miss = (st.sel_miss.indptr, st.sel_miss.indices, st.num_mutations)
        mi = None if miss is None else np.ascontiguousarray(miss.T.astype(dt))
        for lv in build_down_levels(off, coo, sel_mut, sel_miss, 1 << 30, locality=True, pad=True):
            for r, codes in lv.row_lists():
                state[lv.row_begin + r] = _row_sum(codes, state, xi, mi, init_row(lv.row_begin + r))
    if emit_all_nodes:
        return state[np.asarray(st.inv_node_perm)].T
    if direction == "up":
        out = np.zeros((st.num_mutations, k), dtype=dt)
        ptr, idx = st.sel_mut.indptr, st.sel_mut.indices
        for m in range(st.num_mutations):
            s = np.zeros(k, dtype=dt)
            for e in range(ptr[m], ptr[m + 1]):
                s = s + state[idx[e]]
            out[m] = s
        if miss is not None:
            ptr, idx = st.sel_miss.indptr, st.sel_miss.indices
            for m in range(st.num_mutations):
                s = np.zeros(k, dtype=dt)
                for e in range(ptr[m], ptr[m + 1]):
                    s = s + state[idx[e]]
                miss[:, m] += s.astype(miss.dtype)
    else:
        out = state[: st.num_samples].copy()
    if init_mode == "xtx" and not emit_all_nodes:
        bias = st.init_xtx_up_bias if direction == "up" else st.init_xtx_down_bias
        out = out + bias[:, None]
    elif init_mode == "vector" and not emit_all_nodes:
        bias = st.init_vector_up_bias if direction == "up" else st.init_vector_down_bias
        out = out + bias[:, None] * init.astype(dt)[None, :]
    if direction == "down" and by_individual:
        agg = np.zeros((st.num_individuals, k), dtype=dt)
        for s_ in range(st.num_samples):
            agg[int(st.sample_to_individual[s_])] = agg[int(st.sample_to_individual[s_])] + out[s_]
        out = agg
    return out.T
