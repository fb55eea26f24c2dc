"""Many small instances (charge sectors, coupling sweeps) solved in one
persistent device launch (``edg_lanczos_small_batched``), optionally replayed
from a CUDA graph.

This replaces a host loop of ``diagonalize_Hamiltonian`` calls over
instances, each an ``eigsh`` in the reference
(edlgt/modeling/qmb_hamiltonian.py:260-332).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = ["SmallBatch"]


class SmallBatch:
    """Concatenated real DeviceMatrix instances ready for the batched solver."""

    def __init__(self, mats, k=1, max_iter=None, tol=1e-12, check_every=8, seed=1234, want_vectors=False):
        if not mats:
            raise ValueError("need at least one instance")
        if any(m.is_complex for m in mats):
            raise NotImplementedError("the batched solver takes real (gauge-transformed) instances")
        dev = mats[0].rowptr.device
        dims = np.array([m.n for m in mats], dtype=np.int64)
        self.dims = dims
        max_dim = int(dims.max())
        if max_iter is None:
            max_iter = max_dim
        self.k, self.max_iter = k, int(max_iter)
        row_off = np.concatenate([[0], np.cumsum(dims)[:-1]]).astype(np.int64)
        rp_len = dims + 1
        rowptr_off = np.concatenate([[0], np.cumsum(rp_len)[:-1]]).astype(np.int64)
        nnz = np.array([m.nnz for m in mats], dtype=np.int64)
        nnz_off = np.concatenate([[0], np.cumsum(nnz)[:-1]]).astype(np.int64)
        # concatenated CSR: rowptr blocks shifted to global entry indices
        self.rowptr = torch.cat([m.rowptr + int(o) for m, o in zip(mats, nnz_off)]).contiguous()
        self.cols = torch.cat([m.cols[: m.nnz] for m in mats]).contiguous()
        self.vals = torch.cat([m.vals[: m.nnz] for m in mats]).contiguous()
        self.diag = torch.cat([m.diag[: m.n] for m in mats]).contiguous()
        per = np.array([lib.edg_small_batch_work_elems(int(d), self.max_iter, k) for d in dims], dtype=np.int64)
        work_off = np.concatenate([[0], np.cumsum(per)[:-1]]).astype(np.int64)
        self.work = torch.empty(int(per.sum()), dtype=torch.float64, device=dev)
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.d_dims, self.d_row_off, self.d_rp_off, self.d_work_off = up(dims), up(row_off), up(rowptr_off), up(work_off)
        self.evals = torch.empty((len(mats), k), dtype=torch.float64, device=dev)
        self.evecs = torch.empty(int(dims.sum()), dtype=torch.float64, device=dev) if want_vectors else None
        self.iters = torch.empty(len(mats), dtype=torch.int32, device=dev)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        b = _lib.SmallBatch()
        b.n_inst = len(mats)
        b.max_dim = max_dim
        b.dims, b.row_off, b.rowptr_off = ptr(self.d_dims), ptr(self.d_row_off), ptr(self.d_rp_off)
        b.rowptr, b.cols, b.vals, b.diag = ptr(self.rowptr), ptr(self.cols), ptr(self.vals), ptr(self.diag)
        b.work, b.work_off = ptr(self.work), ptr(self.d_work_off)
        b.k, b.max_iter, b.check_every, b.tol, b.seed = k, self.max_iter, check_every, tol, seed
        b.evals = ptr(self.evals)
        b.evecs = ptr(self.evecs) if want_vectors else None
        b.iters = ptr(self.iters)
        self.b = b
        self.graph = None

    def launch(self):
        check(lib.edg_lanczos_small_batched(ctypes.byref(self.b), ptr(self.queue), stream_handle()),
              "edg_lanczos_small_batched")

    def capture(self):
        """Record the launch (queue reset + kernel) in a CUDA graph."""
        self.launch()  # warm-up outside capture (sets kernel attributes)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        self.graph = g
        return g

    def solve(self, use_graph=True):
        if use_graph and self.graph is not None:
            self.graph.replay()
        else:
            self.launch()
        return self.evals
