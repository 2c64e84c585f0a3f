"""Sharded calls over several GPUs, one process per GPU (torch.distributed).

The reference runs on one device (core/src/ocl/ocl_toolkit.cpp:118-141, one
queue per handle); these calls split the same BLAS work over the ranks of a
process group so that every GPU computes on data in its own HBM:

  * GEMM  C = alpha op(A) op(B) + beta C: each rank holds a block of columns
    of B and C (``column_blocks``); A is replicated into every rank's memory
    by one broadcast, then each rank runs the library's GEMM on its block.
    No reduction is needed.
  * TRSM (left side) op(A) X = alpha B: the right-hand sides are independent,
    so B is split by columns the same way; A is broadcast.
  * batched TRSM: the instances are split into contiguous ranges of about
    equal cost (sum of m^2 n, ``instance_ranges``); each rank runs its own
    plan.  No collective.
  * level 1: each rank holds a contiguous segment of the vectors.  dot / asum
    combine the per-rank results with one all-gather, summed in rank order in
    FP64 (every rank gets the same value); nrm2 combines sum-of-squares the
    same way; iamax all-gathers (|x| of the local winner, global index) and
    takes the largest value, ties to the smallest index, so the result is the
    0-based first index of the whole vector.

Data moves only through the process group's collectives (NCCL between GPUs);
no kernel reads another GPU's memory.  The local arithmetic goes through a
``local`` object with the library's calls (``LibraryLocal``, the default);
tests may pass another implementation of the same methods.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def column_blocks(n: int, parts: int, align: int = 64) -> list[tuple[int, int]]:
    """(first column, count) for each of `parts` ranks: every column in
    exactly one block, block starts multiples of `align` (except when n is
    small), counts differing by at most `align`."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    units = (n + align - 1) // align
    out = []
    start = 0
    for r in range(parts):
        u = units // parts + (1 if r < units % parts else 0)
        cnt = min(u * align, n - start)
        out.append((start, max(cnt, 0)))
        start += max(cnt, 0)
    return out


def instance_ranges(costs, parts: int) -> list[tuple[int, int]]:
    """Contiguous (first instance, count) ranges of about equal total cost:
    range r ends at the first instance boundary where the running cost
    reaches r+1 parts of the total."""
    costs = np.asarray(costs, dtype=np.float64)
    acc = np.concatenate([[0.0], np.cumsum(costs)])   # acc[i]: cost of instances [0, i)
    total = acc[-1]
    bounds = [0]
    for r in range(1, parts):
        b = int(np.searchsorted(acc, total * r / parts, side="left"))
        bounds.append(max(bounds[-1], min(b, len(costs))))
    bounds.append(len(costs))
    return [(bounds[r], bounds[r + 1] - bounds[r]) for r in range(parts)]


def combine_sum(parts: list[float]) -> float:
    """Per-rank partial results summed in rank order in FP64."""
    s = 0.0
    for v in parts:
        s += float(v)
    return s


def combine_iamax(cands: list[tuple[float, int]]) -> int:
    """(|x| of the local winner, its global 0-based index) per rank -> the
    first index of the largest |x|.  A rank with an empty segment sends
    (-1, -1); NaN never wins (the library's iamax never returns one unless
    x[0] is NaN, which the rank holding index 0 reports as +inf)."""
    best_v, best_i = -1.0, -1
    for v, i in cands:
        if i < 0:
            continue
        if v > best_v or (v == best_v and (best_i < 0 or i < best_i)):
            best_v, best_i = v, i
    return best_i


class LibraryLocal:
    """The local arithmetic of one rank: the library's C-ABI calls on this
    rank's device buffers (torch CUDA tensors)."""

    def __init__(self, handle):
        from . import iclblas as B
        self.B = B
        self.h = handle

    def sdot(self, n, x, y) -> float:
        import torch
        r = torch.zeros(1, device=x.device)
        self.B.check(self.B.iclblasSdot(self.h, n, x, 1, y, 1, r), "iclblasSdot")
        return float(r.item())

    def sasum(self, n, x) -> float:
        import torch
        r = torch.zeros(1, device=x.device)
        self.B.check(self.B.iclblasSasum(self.h, n, x, 1, r), "iclblasSasum")
        return float(r.item())

    def snrm2(self, n, x) -> float:
        import torch
        r = torch.zeros(1, device=x.device)
        self.B.check(self.B.iclblasSnrm2(self.h, n, x, 1, r), "iclblasSnrm2")
        return float(r.item())

    def isamax(self, n, x) -> tuple[int, float]:
        import torch
        ri = torch.zeros(1, dtype=torch.int32, device=x.device)
        self.B.check(self.B.iclblasIsamax(self.h, n, x, 1, ri), "iclblasIsamax")
        i = int(ri.item())
        return i, float(x[i].abs().item())

    def sgemm(self, ta, tb, m, n, k, alpha, A, lda, Bm, ldb, beta, Cm, ldc):
        self.B.check(self.B.iclblasSgemm(self.h, ta, tb, m, n, k, alpha, A, lda, Bm, ldb, beta, Cm, ldc),
                     "iclblasSgemm")

    def strsm(self, uplo, trans, diag, m, n, alpha, A, lda, Bm, ldb):
        self.B.check(self.B.iclblasStrsm(self.h, 0, uplo, trans, diag, m, n, alpha, A, lda, Bm, ldb),
                     "iclblasStrsm")


@dataclass
class Sharded:
    """Sharded calls of one rank.  `group`: a torch.distributed process group
    (None: the default group); `local`: the rank's arithmetic."""

    local: object
    group: object = None

    def _dist(self):
        import torch.distributed as dist
        return dist

    def rank_world(self):
        dist = self._dist()
        return dist.get_rank(self.group), dist.get_world_size(self.group)

    def _gather_objects(self, obj):
        dist = self._dist()
        out = [None] * dist.get_world_size(self.group)
        dist.all_gather_object(out, obj, group=self.group)
        return out

    # ---- level 1 on contiguous segments (this rank: n_local elements)
    def sdot(self, n_local, x, y) -> float:
        v = self.local.sdot(n_local, x, y) if n_local > 0 else 0.0
        return combine_sum(self._gather_objects(v))

    def sasum(self, n_local, x) -> float:
        v = self.local.sasum(n_local, x) if n_local > 0 else 0.0
        return combine_sum(self._gather_objects(v))

    def snrm2(self, n_local, x) -> float:
        v = self.local.snrm2(n_local, x) if n_local > 0 else 0.0
        return float(np.sqrt(combine_sum(self._gather_objects(float(v) * float(v)))))

    def isamax(self, n_local, x, offset) -> int:
        """0-based global index of the first largest |x|; `offset`: the
        global index of this rank's first element."""
        cand = (-1.0, -1)
        start = 0
        while start < n_local:
            i, v = self.local.isamax(n_local - start, x[start:])
            i += start
            if v == v:
                cand = (v, offset + i)
                break
            # a NaN comes back only as the segment's first element: it pins
            # the whole vector's answer to 0 only when it is the first element
            # of the whole vector; elsewhere it is skipped, as the library
            # skips every NaN past the first element
            if offset + i == 0:
                cand = (float("inf"), 0)
                break
            start = i + 1
        return combine_iamax(self._gather_objects(cand))

    # ---- replicated A, column blocks of B / C
    def broadcast_(self, tensor, src: int = 0):
        """A (any rank's tensor of the same shape) replicated from rank `src`
        into every rank's own buffer, in place."""
        self._dist().broadcast(tensor, src=src, group=self.group)
        return tensor

    def sgemm(self, ta, tb, m, n_local, k, alpha, A, lda, B_local, ldb, beta, C_local, ldc):
        """This rank's columns of C = alpha op(A) op(B) + beta C: B_local and
        C_local hold the rank's column block (n_local columns) of op(B) and
        C; A is the replicated operand."""
        if n_local > 0:
            self.local.sgemm(ta, tb, m, n_local, k, alpha, A, lda, B_local, ldb, beta, C_local, ldc)

    def strsm(self, uplo, trans, diag, m, n_local, alpha, A, lda, B_local, ldb):
        """Left-side solve of this rank's right-hand-side columns."""
        if n_local > 0:
            self.local.strsm(uplo, trans, diag, m, n_local, alpha, A, lda, B_local, ldb)
