"""Shot-parallel FWI over several processes, one per GPU.

Shots are independent until the gradient.  Each rank runs the forward, misfit
and adjoint of its own shots.  The misfit and the lambda / mu gradients of an
inversion with several sources are sums over the shots, so one all-reduce each
per evaluation finishes them.  The sums go through torch.distributed: NCCL for
device tensors, gloo for host arrays.  The reference inverts one source on a
mesh decomposed over MPI ranks, and its reductions run over mesh partitions
(e.g. the L-BFGS inner products, S4/LBFGS_Coupled.F90:87-111).  One GPU holds
the whole mesh here, so ranks split the shots instead.

The model update (TV, gradient mass, L-BFGS, Armijo) runs replicated on every
rank from identical inputs, so all ranks hold the same model without a
broadcast.
"""
from __future__ import annotations

import numpy as np


def shard(n_items: int, world: int, rank: int) -> range:
    """Contiguous, balanced block of item indices for this rank (the first
    n_items % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


class ShotParallelBackend:
    """Wraps the backend of one rank, whose forward() and gradient() cover only
    that rank's shots, so that forward() returns the misfit summed over all ranks
    and gradient() leaves the summed gradient in g_l, g_m.  Every other backend
    method (vector algebra, TV, L-BFGS) passes through unchanged."""

    def __init__(self, backend, group=None):
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            raise RuntimeError("torch.distributed is not initialized")
        self._torch = torch
        self._dist = dist
        self.backend = backend
        self.group = group

    def __getattr__(self, name):
        return getattr(self.backend, name)

    def _allreduce(self, x):
        t = self._torch.from_numpy(x) if isinstance(x, np.ndarray) else x
        stream = getattr(self.backend, "stream", None)
        if stream is not None and not isinstance(x, np.ndarray):
            # device vectors: order the collective after the library's kernels on the
            # backend's stream, and later work on that stream after the collective
            with self._torch.cuda.stream(stream):
                self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)
        else:
            self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)

    def forward(self, lam, mu):
        j = np.array([self.backend.forward(lam, mu)], dtype=np.float64)
        t = self._torch.from_numpy(j)
        if self._dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)
        return float(t.cpu()[0])

    def gradient(self, g_l, g_m):
        self.backend.gradient(g_l, g_m)
        self._allreduce(g_l)
        self._allreduce(g_m)
