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


class _TiledPlan:
    """Plan and device tables of one launch of edg_lanczos_tiled_batch."""

    def __init__(self, dims, dtype, max_iter, k, tile_rows, check_every, dev):
        n = len(dims)
        d = np.ascontiguousarray(dims, dtype=np.int64)
        n_items = ctypes.c_int32(0)
        wbytes = ctypes.c_int64(0)
        check(lib.edg_tiled_batch_plan(n, d.ctypes.data, dtype, max_iter, k, tile_rows, check_every, None, None, None,
                                       ctypes.byref(n_items), ctypes.byref(wbytes)), "edg_tiled_batch_plan")
        inst = np.zeros((n, 8), dtype=np.int64)
        items = np.zeros(n_items.value, dtype=np.int32)
        check_at = np.zeros(max_iter, dtype=np.uint8)
        check(lib.edg_tiled_batch_plan(n, d.ctypes.data, dtype, max_iter, k, tile_rows, check_every, inst.ctypes.data,
                                       items.ctypes.data, check_at.ctypes.data, ctypes.byref(n_items),
                                       ctypes.byref(wbytes)), "edg_tiled_batch_plan")
        self.n_items = n_items.value
        self.inst = torch.from_numpy(inst).to(dev)
        self.items = torch.from_numpy(items).to(dev)
        self.check_at = torch.from_numpy(check_at).to(dev)
        self.workspace = torch.empty(int(wbytes.value), dtype=torch.uint8, device=dev)
        self.dtype, self.max_iter, self.k, self.tile_rows = dtype, max_iter, k, tile_rows


class TiledBatch:
    """Instances of any dimension solved together over an (instance,
    row-tile) work queue (``edg_lanczos_tiled_batch``): one cooperative launch
    per precision phase, no host synchronisation inside a solve, so a whole
    solve is replayed from a CUDA graph.

    ``precision="mixed"``: f32 Krylov basis and matvec (f64 dots, recurrence
    and eigen-solve) to ``tol32``, then an f64 Lanczos of ``refine_iter`` steps
    restarted from each instance's f32 Ritz vector (``k`` must be 1);
    ``"fp64"``: f64 throughout to ``tol``.  ``tile_rows`` / ``lanes`` (threads
    per matrix row) default to the autotuner's choice for this batch, kept in
    ``ctx`` (an :class:`edgpu.Context`).

    Replaces a host loop of ``diagonalize_Hamiltonian`` calls over instances,
    each an ``eigsh`` in the reference (edlgt/modeling/qmb_hamiltonian.py:
    260-332).
    """

    TILE_CHOICES = (256, 512, 1024, 2048, 4096)
    LANE_CHOICES = (2, 4, 8, 16)

    def __init__(self, mats, k=1, precision="mixed", tol=1e-12, tol32=1e-5, max_iter=300, refine_iter=5,
                 check_every=8, seed=1234, tile_rows=None, lanes=None, want_vectors=False, ctx=None):
        if not mats:
            raise ValueError("need at least one instance")
        if any(m.is_complex for m in mats):
            raise NotImplementedError("the batched solver takes real (gauge-transformed) instances")
        if precision not in ("mixed", "fp64"):
            raise ValueError("precision must be 'mixed' or 'fp64'")
        if precision == "mixed" and k != 1:
            raise ValueError("mixed precision refines the ground state only (k=1)")
        dev = mats[0].rowptr.device
        self.dev, self.k, self.precision = dev, k, precision
        self.tol, self.tol32, self.max_iter, self.refine_iter = tol, tol32, int(max_iter), int(refine_iter)
        self.check_every, self.seed, self.want_vectors = check_every, seed, want_vectors
        dims = np.array([m.n for m in mats], dtype=np.int64)
        self.dims = dims
        nnz = np.array([m.nnz for m in mats], dtype=np.int64)
        nnz_off = np.concatenate([[0], np.cumsum(nnz)[:-1]]).astype(np.int64)
        self.rowptr = torch.cat([m.rowptr + int(o) for m, o in zip(mats, nnz_off)]).contiguous()
        self.cols = torch.cat([m.cols[: m.nnz] for m in mats] + [torch.zeros(1, dtype=torch.int32, device=dev)])
        self.vals64 = torch.cat([m.vals[: m.nnz] for m in mats] + [torch.zeros(1, dtype=torch.float64, device=dev)])
        self.diag64 = torch.cat([m.diag[: m.n] for m in mats]).contiguous()
        self.vals32 = self.vals64.to(torch.float32) if precision == "mixed" else None
        self.diag32 = self.diag64.to(torch.float32) if precision == "mixed" else None
        n_inst, total = len(mats), int(dims.sum())
        self.evals = torch.empty((n_inst, k), dtype=torch.float64, device=dev)
        self.resid = torch.empty((n_inst, k), dtype=torch.float64, device=dev)
        self.iters = torch.empty(n_inst, dtype=torch.int32, device=dev)
        self.evals32 = torch.empty((n_inst, 1), dtype=torch.float64, device=dev)
        self.resid32 = torch.empty((n_inst, 1), dtype=torch.float64, device=dev)
        self.iters32 = torch.empty(n_inst, dtype=torch.int32, device=dev)
        self.status = torch.zeros(2, dtype=torch.int32, device=dev)
        self.v0 = torch.empty(total, dtype=torch.float64, device=dev) if precision == "mixed" else None
        self.evecs = torch.empty(total, dtype=torch.float64, device=dev) if want_vectors else None
        self.ctx = ctx
        if tile_rows is None or lanes is None:
            tile_rows, lanes = self._tuned(tile_rows, lanes)
        self._configure(tile_rows, lanes)
        self.graph = None

    # ------------------------------------------------------------------ setup
    def _configure(self, tile_rows, lanes):
        self.tile_rows, self.lanes = int(tile_rows), int(lanes)
        if self.precision == "mixed":
            self.plan32 = _TiledPlan(self.dims, 1, self.max_iter, 1, self.tile_rows, self.check_every, self.dev)
            self.plan64 = _TiledPlan(self.dims, 0, self.refine_iter, 1, self.tile_rows, self.refine_iter, self.dev)
        else:
            self.plan32 = None
            self.plan64 = _TiledPlan(self.dims, 0, self.max_iter, self.k, self.tile_rows, self.check_every, self.dev)
        self.graph = None

    def _struct(self, plan, v0, evals, resid, iters, evecs, status, tol):
        b = _lib.TiledBatch()
        b.dtype = plan.dtype
        b.n_inst = len(self.dims)
        b.n_items = plan.n_items
        b.tile_rows = plan.tile_rows
        b.lanes = self.lanes
        b.k = plan.k
        b.max_iter = plan.max_iter
        b.tol = tol
        b.seed = self.seed
        b.inst, b.item_inst, b.check_at = ptr(plan.inst), ptr(plan.items), ptr(plan.check_at)
        b.rowptr, b.cols = ptr(self.rowptr), ptr(self.cols)
        b.vals = ptr(self.vals32 if plan.dtype == 1 else self.vals64)
        b.diag = ptr(self.diag32 if plan.dtype == 1 else self.diag64)
        b.v0 = ptr(v0)
        b.workspace = ptr(plan.workspace)
        b.evals, b.resid, b.iters = ptr(evals), ptr(resid), ptr(iters)
        b.evecs = ptr(evecs)
        b.status = ptr(status)
        return b

    def launch(self):
        """Enqueue one solve on the current stream (no host synchronisation)."""
        st = stream_handle()
        if self.precision == "mixed":
            b32 = self._struct(self.plan32, None, self.evals32, self.resid32, self.iters32, self.v0, self.status[0:1],
                               self.tol32)
            check(lib.edg_lanczos_tiled_batch(ctypes.byref(b32), st), "edg_lanczos_tiled_batch")
            b64 = self._struct(self.plan64, self.v0, self.evals, self.resid, self.iters, self.evecs, self.status[1:2],
                               self.tol)
        else:
            b64 = self._struct(self.plan64, None, self.evals, self.resid, self.iters, self.evecs, self.status[1:2],
                               self.tol)
        check(lib.edg_lanczos_tiled_batch(ctypes.byref(b64), st), "edg_lanczos_tiled_batch")

    def capture(self):
        """Record one solve (both launches) in a CUDA graph."""
        self.launch()  # first launch outside capture
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

    def check_status(self):
        """Raise when a launch's grid-wide wait ran out (synchronises)."""
        s = self.status.cpu().numpy()
        for v in s:
            if int(v) != 0:
                raise _lib.EdgError(int(v), "edg_lanczos_tiled_batch: a grid-wide wait ran out")

    # ------------------------------------------------------------ autotuning
    def _shape_key(self):
        h = 1469598103934665603
        for x in (len(self.dims), *self.dims.tolist(), int(self.rowptr.numel()), self.max_iter,
                  1 if self.precision == "mixed" else 0):
            h = ((h ^ (int(x) & 0xFFFFFFFFFFFFFFFF)) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        return h

    def _tuned(self, tile_rows, lanes):
        from .context import default_context

        ctx = self.ctx if self.ctx is not None else default_context(self.dev)
        key = self._shape_key()
        got = ctx.get(key, 2)
        if got is not None:
            return (tile_rows or got[0], lanes or got[1])
        best, best_t = None, float("inf")
        tiles = (tile_rows,) if tile_rows else self.TILE_CHOICES
        lanes_c = (lanes,) if lanes else self.LANE_CHOICES
        max_dim = int(self.dims.max())
        for tr in tiles:
            if tr > 4 * max(max_dim, 256) and tr != tiles[0]:
                continue  # tiles far larger than every instance behave alike
            for ln in lanes_c:
                self._configure(tr, ln)
                self.launch()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                self.launch()
                b.record()
                torch.cuda.synchronize()
                self.check_status()
                t = a.elapsed_time(b)
                if t < best_t:
                    best, best_t = (tr, ln), t
        ctx.put(key, best)
        self.tuned_ms = best_t
        return best
