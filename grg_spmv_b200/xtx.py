"""Standardised genotype Gram operators on the B200 backend, randomized PCA and CG over them.

``StandardizedXTX`` applies ``Zᵀ Z`` to a block of vectors, where ``Z`` is the genotype matrix
of a GRG (individuals x mutations) centred by ``ploidy * p`` and scaled by
``1 / sqrt(ploidy * p * (1 - p))`` per mutation, ``p`` being the allele frequency among the
non-missing samples.  It restates ``PreparedXTX`` of the reference
(``scripts/pca_bench/__main__.py:183-360``): frequencies from one ``up`` pass of ones
(``:201-236``), then per call one ``down`` and one ``up`` prepared op by individual, with the
centring folded in as rank-one corrections (``_body``, ``:326-347``):

    d   = (V / sigma)ᵀ                   miss rows: d * p      c_down = d · centre
    u   = down(d) - c_down               c_up = row sums of u
    out = (up(u) (+ p * up_miss)) / sigma - c_up * centre / sigma

Everything outside the two traversals is FP64 work on the runtime's stream, fused into one
library pass per step (``grg_b200_rowop``: the per-row scaling, the miss rows, the centring and
the deterministic column sums that replace the reference's CuPy elementwise chain, its cuBLAS
``d @ centre`` and its ``row_weighted_sum`` kernel, ``:32-61``).  One application is three such
passes around the two traversals; the traversals are the B200 kernels, in plain FP64 or in
the mixed precision of the runtime's layout.  ``randomized_eigh`` is the reference's
randomized Rayleigh-Ritz solver (``_run_randomized_rr``, ``:656-669``) with FP64 QR and eigh.

``StandardizedXXT`` is the individual-space counterpart ``Z Zᵀ`` (the kinship product of the
reference's BOLT-LMM ops, ``scripts/bolt_lmm_inf/core.py:1241-1301``, one GRG), and
``conj_grad_solve`` restates ``bolt_conj_grad_solve`` (``core.py:1304-1353``) with all
right-hand sides in one block: one operator call per iteration instead of one per column,
FP64 dot products and residuals.
"""

from __future__ import annotations

import ctypes

from grg_spmv_b200.backends.b200 import _native as nat


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


class _RowStep:
    """One ``grg_b200_rowop`` pass with fixed buffers (the source may change per call)."""

    def __init__(self, lib, stream_ptr: int, *, rows: int, k: int, src=None, dst, miss_in=None, miss_scale=None,
                 pre_scale=None, col_sub=None, sub_scale=None, post_scale=None, miss_out=None, miss_out_scale=None,
                 sums=None, sum_weight=None, partials=None) -> None:
        self._lib = lib
        self._stream = ctypes.c_void_p(stream_ptr)
        self.args = nat.RowopArgs(rows=int(rows), k=int(k), ld=int(k), src=_ptr(src), dst=_ptr(dst), miss_in=_ptr(miss_in),
                                  miss_scale=_ptr(miss_scale), pre_scale=_ptr(pre_scale), col_sub=_ptr(col_sub),
                                  sub_scale=_ptr(sub_scale), post_scale=_ptr(post_scale), miss_out=_ptr(miss_out),
                                  miss_out_scale=_ptr(miss_out_scale), col_sums=int(sums is not None),
                                  sum_weight=_ptr(sum_weight), partials=_ptr(partials), sums=_ptr(sums))

    def __call__(self, src=None) -> None:
        if src is not None:
            self.args.src = int(src.data_ptr())
        nat.check(self._lib, self._lib.grg_b200_rowop(ctypes.byref(self.args), self._stream), "grg_b200_rowop")


class StandardizedXTX:
    """``Zᵀ Z`` for blocks of ``q`` vectors (``apply(V)`` with ``V`` of shape ``(M, q)``)."""

    def __init__(self, runtime, grg, q: int) -> None:
        import torch

        self._runtime = runtime
        self.grg = grg
        self.q = int(q)
        self.has_missing = bool(grg.has_missing_data)
        self.shape = (int(grg.num_mutations), int(grg.num_mutations))
        dev = torch.device(runtime.device)
        self._stream = runtime._torch_caller_stream()
        with torch.cuda.device(dev), torch.cuda.stream(self._stream):
            ones_op = grg.prepare_matmul_cuda(direction="up", k=1, by_individual=True, use_miss=self.has_missing)
            ones_op.input.fill_(1.0)
            if self.has_missing:
                ones_op.miss_output.fill_(0.0)
            ones_op()
            counts = ones_op.output[0].clone()
            miss_counts = ones_op.miss_output[0].clone() if self.has_missing else torch.zeros_like(counts)
            denom = float(grg.num_samples) - miss_counts
            valid = denom != 0.0
            self.freqs = torch.where(valid, counts / torch.where(valid, denom, torch.ones_like(denom)), torch.zeros_like(denom))
            ploidy = float(grg.ploidy)
            self.center = ploidy * self.freqs
            sigma = torch.sqrt(ploidy * self.freqs * (1.0 - self.freqs))
            self.sigma = torch.where(sigma == 0.0, torch.ones_like(sigma), sigma)
            self.inv_sigma = 1.0 / self.sigma
            self.center_over_sigma = self.center * self.inv_sigma
            self._down = grg.prepare_matmul_cuda(direction="down", k=self.q, by_individual=True, use_miss=self.has_missing)
            self._up = grg.prepare_matmul_cuda(direction="up", k=self.q, by_individual=True, use_miss=self.has_missing)
            self._out = torch.empty((self.shape[0], self.q), device=dev, dtype=torch.float64)
            M, I = int(grg.num_mutations), int(grg.num_individuals)
            self._partials = torch.empty((nat.rowop_blocks(max(M, I)), self.q), device=dev, dtype=torch.float64)
            self.c_down = torch.empty(self.q, device=dev, dtype=torch.float64)
            self.c_up = torch.empty(self.q, device=dev, dtype=torch.float64)
        lib, sp = runtime._lib, int(self._stream.cuda_stream)
        down, up, miss = self._down, self._up, self.has_missing
        # d = v / sigma (and its miss rows d * p), c_down = d . centre
        self._encode = _RowStep(lib, sp, rows=M, k=self.q, dst=down.input, pre_scale=self.inv_sigma,
                                miss_out=down.miss_input if miss else None, miss_out_scale=self.freqs if miss else None,
                                sums=self.c_down, sum_weight=self.center, partials=self._partials)
        # u = down(d) - c_down in place (it is up's input), c_up = column sums of u
        self._center = _RowStep(lib, sp, rows=I, k=self.q, src=down.output, dst=up.input, col_sub=self.c_down,
                                sums=self.c_up, partials=self._partials)
        # out = (up(u) + p * up_miss) / sigma - c_up * centre / sigma
        self._finish = _RowStep(lib, sp, rows=M, k=self.q, src=up.output, dst=self._out,
                                miss_in=up.miss_output if miss else None, miss_scale=self.freqs if miss else None,
                                pre_scale=self.inv_sigma, col_sub=self.c_up, sub_scale=self.center_over_sigma)

    def apply(self, v):
        """``Zᵀ Z v`` for ``v`` of shape ``(M, q)`` (a CUDA FP64 tensor); returns a new ``(M, q)`` tensor."""
        import torch

        if tuple(v.shape) != (self.shape[0], self.q):
            raise ValueError(f"operand has shape {tuple(v.shape)}, expected ({self.shape[0]}, {self.q})")
        if v.dtype != torch.float64 or v.device != self._out.device:
            raise ValueError("operand must be a float64 tensor on the runtime's device")
        with torch.cuda.stream(self._stream):
            v = v.contiguous()
            self._encode(v)
            self._down()
            self._center()
            self._up()
            self._finish()
            return self._out.clone()


class StandardizedXXT:
    """``Z Zᵀ`` for blocks of ``q`` vectors over individuals (``apply(W)``, ``W`` of shape
    ``(I, q)``): ``Zᵀ`` by one ``up`` pass, ``Z`` by one ``down`` pass, with the same centring,
    scaling and missing-data terms as ``StandardizedXTX``."""

    def __init__(self, runtime, grg, q: int) -> None:
        import torch

        self._xtx = StandardizedXTX(runtime, grg, q)
        self.q = int(q)
        self.shape = (int(grg.num_individuals), int(grg.num_individuals))
        self._out = torch.empty(self.shape[0], self.q, device=self._xtx._out.device, dtype=torch.float64)
        x = self._xtx
        lib, sp = runtime._lib, int(x._stream.cuda_stream)
        down, up, miss = x._down, x._up, x.has_missing
        M, I = int(grg.num_mutations), int(grg.num_individuals)
        # up's input = w, c_up = column sums of w
        self._load = _RowStep(lib, sp, rows=I, k=self.q, dst=up.input, sums=x.c_up, partials=x._partials)
        # t = (up(w) + p * up_miss) / sigma - c_up * centre / sigma; down's input d = t / sigma,
        # its miss rows d * p, c_down = d . centre
        self._mid = _RowStep(lib, sp, rows=M, k=self.q, src=up.output, dst=down.input,
                             miss_in=up.miss_output if miss else None, miss_scale=x.freqs if miss else None,
                             pre_scale=x.inv_sigma, col_sub=x.c_up, sub_scale=x.center_over_sigma, post_scale=x.inv_sigma,
                             miss_out=down.miss_input if miss else None, miss_out_scale=x.freqs if miss else None,
                             sums=x.c_down, sum_weight=x.center, partials=x._partials)
        # out = down(d) - c_down
        self._finish = _RowStep(lib, sp, rows=I, k=self.q, src=down.output, dst=self._out, col_sub=x.c_down)

    def apply(self, w):
        import torch

        x = self._xtx
        if tuple(w.shape) != (self.shape[0], self.q):
            raise ValueError(f"operand has shape {tuple(w.shape)}, expected ({self.shape[0]}, {self.q})")
        if w.dtype != torch.float64 or w.device != self._out.device:
            raise ValueError("operand must be a float64 tensor on the runtime's device")
        with torch.cuda.stream(x._stream):
            w = w.contiguous()
            self._load(w)
            x._up()
            self._mid()
            x._down()
            self._finish()
            return self._out.clone()


def conj_grad_solve(matvec, rhs, *, rel_tol: float, max_iter: int, project=None):
    """Solve ``A x = b`` for every column of ``rhs`` (``(n, c)``, FP64 CUDA tensor) by conjugate
    gradients with one block ``matvec`` per iteration; the control flow of the reference's
    ``bolt_conj_grad_solve`` (full-batch CG, no active-column mask, no denominator guard,
    stop when every column's relative residual is within ``rel_tol`` or after ``max_iter``).
    Returns ``(x, iterations, relative residuals)``."""
    import torch

    proj = project if project is not None else (lambda v: v)
    b = proj(rhs.clone())
    x = torch.zeros_like(b)
    r = b.clone()
    p = r.clone()
    r2_orig = (r * r).sum(dim=0)
    r2_old = r2_orig.clone()
    rels = torch.sqrt(r2_old / r2_orig)
    for it in range(1, int(max_iter) + 1):
        hp = matvec(p)
        alpha = r2_old / (p * hp).sum(dim=0)
        x += p * alpha[None, :]
        r -= hp * alpha[None, :]
        r = proj(r)
        r2_new = (r * r).sum(dim=0)
        rels = torch.sqrt(r2_new / r2_orig)
        if not bool((rels > float(rel_tol)).any()):
            return proj(x), it, rels
        p = p * (r2_new / r2_old)[None, :] + r
        r2_old = r2_new
    return proj(x), int(max_iter), rels


def randomized_eigh(op: StandardizedXTX, pcs: int, *, oversample: int = 0, power_iters: int = 10, seed: int = 0):
    """Top ``pcs`` eigenpairs of ``op`` by randomized subspace iteration with a Rayleigh-Ritz
    step (FP64 QR and eigh on the GPU).  ``op.q`` must equal ``pcs + oversample``."""
    import torch

    width = int(pcs) + int(oversample)
    if width != op.q:
        raise ValueError(f"operator block width {op.q} != pcs + oversample = {width}")
    gen = torch.Generator(device="cuda").manual_seed(int(seed))
    omega = torch.randn((op.shape[0], width), dtype=torch.float64, device="cuda", generator=gen)
    y = op.apply(omega)
    for _ in range(int(power_iters)):
        q, _ = torch.linalg.qr(y, mode="reduced")
        y = op.apply(q)
    q, _ = torch.linalg.qr(y, mode="reduced")
    aq = op.apply(q)
    small = q.T @ aq
    small = 0.5 * (small + small.T)
    values, vectors = torch.linalg.eigh(small)
    order = torch.flip(torch.argsort(values), dims=(0,))[: int(pcs)]
    return values[order], q @ vectors[:, order]


__all__ = ["StandardizedXTX", "StandardizedXXT", "conj_grad_solve", "randomized_eigh"]
