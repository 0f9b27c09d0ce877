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

Everything outside the two traversals is FP64 elementwise work on the runtime's stream (the
reference does it with CuPy); the traversals are the B200 kernels, in plain FP64 or in the
mixed precision of the runtime's layout.  ``randomized_eigh`` is the reference's
randomized Rayleigh-Ritz solver (``_run_randomized_rr``, ``:656-669``) with FP64 QR and eigh.

``StandardizedXXT`` is the individual-space counterpart ``Z Zᵀ`` (the kinship product of the
reference's BOLT-LMM ops, ``scripts/bolt_lmm_inf/core.py:1241-1301``, one GRG), and
``conj_grad_solve`` restates ``bolt_conj_grad_solve`` (``core.py:1304-1353``) with all
right-hand sides in one block: one operator call per iteration instead of one per column,
FP64 dot products and residuals.
"""

from __future__ import annotations


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

    def apply(self, v):
        """``Zᵀ Z v`` for ``v`` of shape ``(M, q)`` (a CUDA FP64 tensor); returns a new ``(M, q)`` tensor."""
        import torch

        if tuple(v.shape) != (self.shape[0], self.q):
            raise ValueError(f"operand has shape {tuple(v.shape)}, expected ({self.shape[0]}, {self.q})")
        down, up = self._down, self._up
        with torch.cuda.stream(self._stream):
            torch.mul(v.T, self.inv_sigma[None, :], out=down.input)
            if self.has_missing:
                torch.mul(down.input, self.freqs[None, :], out=down.miss_input)
            c_down = down.input @ self.center
            down()
            u = down.output - c_down[:, None]
            c_up = u.sum(dim=1)
            up.input.copy_(u)
            if self.has_missing:
                up.miss_output.fill_(0.0)
            up()
            res = up.output
            if self.has_missing:
                res = res + up.miss_output * self.freqs[None, :]
            res = res * self.inv_sigma[None, :] - c_up[:, None] * self.center_over_sigma[None, :]
            self._out.copy_(res.T)
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

    def apply(self, w):
        import torch

        x = self._xtx
        if tuple(w.shape) != (self.shape[0], self.q):
            raise ValueError(f"operand has shape {tuple(w.shape)}, expected ({self.shape[0]}, {self.q})")
        down, up = x._down, x._up
        with torch.cuda.stream(x._stream):
            up.input.copy_(w.T)  # Zᵀ w
            c_up = up.input.sum(dim=1)
            if x.has_missing:
                up.miss_output.fill_(0.0)
            up()
            t = up.output.clone()
            if x.has_missing:
                t += up.miss_output * x.freqs[None, :]
            t = t * x.inv_sigma[None, :] - c_up[:, None] * x.center_over_sigma[None, :]
            torch.mul(t, x.inv_sigma[None, :], out=down.input)  # Z t
            if x.has_missing:
                torch.mul(down.input, x.freqs[None, :], out=down.miss_input)
            c_down = down.input @ x.center
            down()
            self._out.copy_((down.output - c_down[:, None]).T)
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
