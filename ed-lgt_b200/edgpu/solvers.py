"""Ground-state solvers on the device.

* :func:`lanczos` -- the drop-in for ``scipy.sparse.linalg.eigsh(H, k,
  which="SA")`` (called at edlgt/modeling/qmb_hamiltonian.py:313): Lanczos with
  full reorthogonalisation, f64 vectors, f64 recurrence and device tridiagonal
  eigen-solve.
* :func:`lanczos_mixed` -- f32 Krylov vectors and matvec (f64 accumulation,
  f64 inner products / recurrence / reorthogonalisation / tridiagonal solve),
  then a short f64 Lanczos restarted from the f32 Ritz vector refines the
  pair ("residual-correction" refinement).  Works on up to four problems that
  share the off-diagonal matrix and differ in the diagonal (coupling sweeps),
  in one batched matvec.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = ["LanczosResult", "PackedLayout", "SellLayout", "lanczos", "lanczos_mixed", "packed_layout", "sell_layout",
           "stack_diagonals", "tune_matvec32", "tune_spmv_group"]

SPMV_GROUPS = (2, 4, 8, 16, 32)


def _spmv_key(n, nnz, dtype, nvec):
    h = 1469598103934665603
    for x in (0x5350, n, nnz, dtype, nvec):  # 0x5350: the matvec tuner's tag
        h = ((h ^ (int(x) & 0xFFFFFFFFFFFFFFFF)) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def tune_spmv_group(mat, nvec=1, dtype=0, reps=5, vals=None, diag=None, ctx=None):
    """Autotuner: threads per matvec row that is fastest on this matrix.

    Times ``edg_spmv_group`` for every group size with CUDA events (after one
    warm-up launch each) on the real matrix and the requested precision and
    batch width.  The choice is kept in the tuning context ``ctx`` (an
    :class:`edgpu.Context`; the device's default context when None) under the
    matrix shape (n, nnz), precision and batch width, so later matrices of the
    same shape reuse it (a performance choice only: every group size gives the
    same result).
    """
    from .context import default_context

    ctx = ctx if ctx is not None else default_context(mat.rowptr.device)
    key = _spmv_key(mat.n, mat.nnz, dtype, nvec)
    got = ctx.get(key, 1)
    if got is not None:
        return got[0]
    dev = mat.rowptr.device
    tdt = {0: torch.float64, 1: torch.float32}[dtype]
    if vals is None:
        vals = mat.vals.to(tdt)
    if diag is None:
        diag = torch.zeros((mat.n, nvec), dtype=tdt, device=dev)
    x = torch.ones((mat.n, nvec), dtype=tdt, device=dev)
    y = torch.empty_like(x)
    best, best_t = 0, float("inf")
    for g in SPMV_GROUPS:
        def launch():
            check(lib.edg_spmv_group(dtype, mat.n, mat.nnz, ptr(mat.rowptr), ptr(mat.cols) if mat.nnz else None,
                                     ptr(vals) if mat.nnz else None, ptr(diag), nvec, ptr(x), ptr(y), g,
                                     stream_handle()), "edg_spmv_group")
        launch()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            launch()
        b.record()
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / reps
        if t < best_t:
            best, best_t = g, t
    ctx.put(key, (best,))
    return best


class SellLayout:
    """SELL-32-sigma copy of a matrix's off-diagonal part with f32 values
    (``edg_sell_order`` / ``edg_scan_i64`` / ``edg_sell_fill``), a layout of
    the f32 Krylov path's matvec: rows sorted by length inside windows of
    ``window`` rows (32 keeps the basis order), slices of 32 rows, each
    slice's entries column-major as 8-byte (column, value) pairs."""

    def __init__(self, mat, vals=None, window=32):
        dev = mat.rowptr.device
        n = mat.n
        st = stream_handle()
        ns = int(lib.edg_sell_slices(n))
        self.n, self.n_slices, self.window = n, ns, int(window)
        self.perm = torch.empty(max(ns * 32, 1), dtype=torch.int32, device=dev)
        self.width = torch.empty(max(ns, 1), dtype=torch.int32, device=dev)
        counts = torch.empty(max(ns, 1), dtype=torch.int64, device=dev)
        self.off = torch.empty(ns + 1, dtype=torch.int64, device=dev)
        check(lib.edg_sell_order(ptr(mat.rowptr), n, self.window, ptr(self.perm), ptr(self.width), ptr(counts), st),
              "edg_sell_order")
        scratch = torch.empty(max(1, lib.edg_scan_scratch_elems(ns)), dtype=torch.int64, device=dev)
        check(lib.edg_scan_i64(ptr(counts), ptr(self.off), ns, ptr(scratch), st), "edg_scan_i64")
        self.pairs = int(self.off[ns].item()) if ns else 0
        self.entries = torch.empty(max(self.pairs, 1) * 2, dtype=torch.int32, device=dev)
        v = mat.vals if vals is None else vals
        dt = 1 if v.dtype == torch.float32 else 0
        if mat.nnz:
            check(lib.edg_sell_fill(dt, ptr(mat.rowptr), ptr(mat.cols), ptr(v), n, ptr(self.perm), ptr(self.width),
                                    ptr(self.off), ptr(self.entries), st), "edg_sell_fill")
        else:
            self.entries.fill_(-1)
        self.nnz = mat.nnz

    @property
    def padding(self):
        """Fraction of stored pairs that are slice padding."""
        return 1.0 - self.nnz / max(self.pairs, 1)


def sell_layout(mat, vals32=None, window=32):
    """The matrix's SELL layout for a sort window (built once, kept on the
    matrix)."""
    cache = getattr(mat, "_sell32", None)
    if cache is None:
        cache = mat._sell32 = {}
    if window not in cache:
        cache[window] = SellLayout(mat, vals32, window)
    return cache[window]


SELL_WINDOWS = (32, 256, 4096)

PACK_MAX_VALUES = _lib.PACK_MAX_VALUES
_PACK_LOG2_SLOTS = 14  # hash set of the distinct values (4x the table limit)


class PackedLayout:
    """Dictionary-packed tiled copy of a matrix's off-diagonal part
    (``edg_pack_collect`` / ``edg_pack_tile_counts`` / ``edg_pack_encode``):
    one 32-bit word per entry, ``column | (value index << colbits)``, the
    distinct values in an ascending table -- ``table64`` (the f64 values) and
    ``table32`` (the same values rounded to f32, so that entry i's f32 value
    is ``vals.to(float32)[i]``) -- and the rows in tiles of 16, each tile as
    wide as its longest row and stored k-major (``tile_off`` [n_tiles+1];
    padding words all ones).  The lattice models' Hamiltonians have a handful
    of distinct off-diagonal values, so the entry stream is 4 bytes an entry
    plus the tiles' padding.  ``PackedLayout.build`` returns None for a
    matrix with too many distinct values or too many words."""

    TILE_ROWS = 16

    def __init__(self, n, nnz, tile_off, words, total, table64, colbits):
        self.n, self.nnz, self.total = n, nnz, int(total)
        self.tile_off, self.words = tile_off, words
        self.table64 = table64
        self.table32 = table64.to(torch.float32)
        self.count = int(table64.numel())
        self.colbits = int(colbits)

    def table(self, dtype):
        return self.table32 if dtype == 1 else self.table64

    @classmethod
    def build(cls, mat):
        if mat.is_complex or mat.n == 0 or mat.nnz == 0:
            return None
        dev = mat.rowptr.device
        st = stream_handle()
        colbits = max(1, int(mat.n).bit_length())  # n < 2^colbits: the all-ones column marks padding
        if colbits > 31:
            return None
        vals = mat.vals.to(torch.float64).contiguous()
        slots = torch.full((1 << _PACK_LOG2_SLOTS,), -1, dtype=torch.int64, device=dev)
        flags = torch.zeros(2, dtype=torch.int32, device=dev)
        check(lib.edg_pack_collect(0, ptr(vals), mat.nnz, ptr(slots), _PACK_LOG2_SLOTS, ptr(flags), st),
              "edg_pack_collect")
        host = slots.cpu().numpy()
        if int(flags[0].item()):
            return None
        bits = np.unique(host[host != -1])
        # ascending values; -0.0 before +0.0 (they compare equal, the bits differ)
        uniq = bits.view(np.float64)[np.lexsort((bits, bits.view(np.float64)))]
        count = int(uniq.size)
        if count > PACK_MAX_VALUES or (count - 1) >> (32 - colbits):
            return None
        n_tiles = int(lib.edg_pack_tiles(mat.n))
        counts = torch.empty(n_tiles, dtype=torch.int64, device=dev)
        offsets = torch.empty(n_tiles + 1, dtype=torch.int64, device=dev)
        check(lib.edg_pack_tile_counts(mat.n, ptr(mat.rowptr), ptr(counts), st), "edg_pack_tile_counts")
        scratch = torch.empty(max(1, lib.edg_scan_scratch_elems(n_tiles)), dtype=torch.int64, device=dev)
        check(lib.edg_scan_i64(ptr(counts), ptr(offsets), n_tiles, ptr(scratch), st), "edg_scan_i64")
        total = int(offsets[n_tiles].item())
        if total >= 2**31 - 8:
            return None
        table64 = torch.from_numpy(np.ascontiguousarray(uniq)).to(dev)
        tile_off = torch.empty(n_tiles + 1, dtype=torch.int32, device=dev)
        words = torch.empty(total + 4, dtype=torch.int32, device=dev)
        check(lib.edg_pack_encode(0, mat.n, total, ptr(mat.rowptr), ptr(mat.cols), ptr(vals), ptr(table64), count,
                                  colbits, ptr(offsets), ptr(tile_off), ptr(words), ptr(flags[1:]), st),
              "edg_pack_encode")
        if int(flags[1].item()):
            raise _lib.EdgError(-1, "edg_pack_encode: a value is missing from the table")
        return cls(mat.n, mat.nnz, tile_off, words, total, table64, colbits)

    @property
    def stream_bytes(self):
        """Bytes of the entry stream (padding included) and the tile offsets."""
        return 4 * self.total + 4 * self.tile_off.numel()

    @property
    def padding(self):
        """Fraction of the stream's words that are tile padding."""
        return 1.0 - self.nnz / max(self.total, 1)

    def launch(self, dtype, nvec, diag, x, x_stride, y, y_plane=0, err=None):
        """y (f64, planar [nvec][y_plane]) = (A + diag) x (``edg_spmv_packed``)."""
        check(lib.edg_spmv_packed(dtype, self.n, nvec, ptr(self.tile_off), ptr(self.words), ptr(self.table(dtype)),
                                  self.count, self.colbits, ptr(diag), ptr(x), x_stride, ptr(y), y_plane or self.n,
                                  ptr(err) if err is not None else None, stream_handle()), "edg_spmv_packed")


def packed_layout(mat):
    """The matrix's dictionary-packed layout (built once, kept on the matrix),
    or None when the matrix does not pack."""
    if not hasattr(mat, "_packed"):
        mat._packed = PackedLayout.build(mat)
    return mat._packed


def tune_matvec32(mat, nvec, vals32=None, reps=5, ctx=None):
    """Autotuner of the f32 Krylov path's matvec: times, in that path's
    configuration (f32 values and x with padded rows, f64 planar output),
    the CSR kernel for every threads-per-row choice, the SELL kernel for
    every sort window and the dictionary-packed kernel when the matrix packs
    (CUDA events after a warm-up launch), and keeps the fastest in the
    tuning context under the matrix shape.  Returns ("csr", threads per
    row), ("sell", window) or ("packed", 2)."""
    from .context import default_context

    ctx = ctx if ctx is not None else default_context(mat.rowptr.device)
    key = _spmv_key(mat.n, mat.nnz, 0x5E11, nvec)
    got = ctx.get(key, 2)
    names = {0: "csr", 1: "sell", 2: "packed"}
    if got is not None and (got[0] != 2 or packed_layout(mat) is not None):
        return (names[got[0]], got[1])
    dev = mat.rowptr.device
    # the packed layout's f32 table holds the f64 values rounded to f32
    vals32_is_rounded = vals32 is None or bool(torch.equal(vals32, mat.vals.to(torch.float32)))
    vals32 = mat.vals.to(torch.float32) if vals32 is None else vals32
    xs = 4 if nvec == 3 else nvec
    diag = torch.zeros((mat.n, nvec), dtype=torch.float32, device=dev)
    x = torch.ones((mat.n, xs), dtype=torch.float32, device=dev)
    y = torch.empty((nvec, mat.n), dtype=torch.float64, device=dev)

    def t_of(launch):
        launch()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            launch()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    best, best_t = None, float("inf")
    for g in SPMV_GROUPS:
        t = t_of(lambda: check(lib.edg_spmv_f32_planar(mat.n, mat.nnz, ptr(mat.rowptr),
                                                       ptr(mat.cols) if mat.nnz else None,
                                                       ptr(vals32) if mat.nnz else None, ptr(diag), nvec, ptr(x), xs,
                                                       ptr(y), mat.n, g, stream_handle()), "edg_spmv_f32_planar"))
        if t < best_t:
            best, best_t = ("csr", g), t
    for wdw in SELL_WINDOWS:
        lay = sell_layout(mat, vals32, wdw)
        t = t_of(lambda: check(lib.edg_spmv_sell(mat.n, nvec, ptr(lay.perm), ptr(lay.width), ptr(lay.off),
                                                 ptr(lay.entries), ptr(diag), ptr(x), xs, ptr(y), mat.n,
                                                 stream_handle()), "edg_spmv_sell"))
        if t < best_t:
            best, best_t = ("sell", wdw), t
    pk = packed_layout(mat) if vals32_is_rounded else None
    if pk is not None:
        t = t_of(lambda: pk.launch(1, nvec, diag, x, xs, y, mat.n))
        if t < best_t:
            best, best_t = ("packed", 2), t
    # layouts that lost are not kept on the matrix
    keep = best[1] if best[0] == "sell" else None
    mat._sell32 = {w: l for w, l in getattr(mat, "_sell32", {}).items() if w == keep}
    ctx.put(key, ({"csr": 0, "sell": 1, "packed": 2}[best[0]], best[1]))
    return best


class LanczosResult:
    def __init__(self, evals, evecs, iters, resid):
        self.evals = evals      # (nvec, k) float64 numpy
        self.evecs = evecs      # device tensor (k, n, nvec) or None
        self.iters = iters      # (nvec,) int
        self.resid = resid      # (nvec, k)


def _problem(dtype, n, nnz, rowptr, cols, vals, diag, nvec, k, max_iter, tol, check_every, seed, v0, stats=None,
             group=0, sell=None, window=0, packed=None):
    p = _lib.LanczosProblem()
    p.dtype = dtype
    p.n_rows = n
    p.nnz = nnz
    p.rowptr = ptr(rowptr)
    p.cols = ptr(cols) if nnz else None
    p.vals = ptr(vals) if nnz else None
    p.diag = ptr(diag)
    p.nvec = nvec
    p.k = k
    p.max_iter = max_iter
    p.tol = tol
    p.check_every = check_every
    p.seed = seed
    p.v0 = ptr(v0) if v0 is not None else None
    p.stats = stats.ctypes.data if stats is not None else None
    p.spmv_group = group
    if sell is not None:
        p.sell_perm, p.sell_width, p.sell_off = ptr(sell.perm), ptr(sell.width), ptr(sell.off)
        p.sell_entries = ptr(sell.entries)
    p.reorth_window = int(window)
    if packed is not None:
        p.pk_tile_off, p.pk_words = ptr(packed.tile_off), ptr(packed.words)
        p.pk_table, p.pk_count, p.pk_colbits = ptr(packed.table(dtype)), packed.count, packed.colbits
    return p


_PROGRESS = {}


def _progress_words(device):
    """Pinned host words the device-driven solver reports its progress in
    (one buffer per device; calls on a device are stream-ordered)."""
    idx = torch.device(device).index or 0
    if idx not in _PROGRESS:
        _PROGRESS[idx] = torch.zeros(4, dtype=torch.int32, pin_memory=True)
    return _PROGRESS[idx]


def run_lanczos(dtype, n, nnz, rowptr, cols, vals, diag, nvec=1, k=1, max_iter=300, tol=1e-12, check_every=5,
                seed=1234, v0=None, want_vectors=True, allow_unconverged=False, workspace=None, stats=None,
                group=0, poll_host=True, sell=None, window=0, packed=None):
    """Low-level call of ``edg_lanczos``; ``diag`` is ``[n][nvec]`` in the dtype.

    ``stats``: optional float64 numpy array of 6 entries filled with the
    phase timings of the run (see edg_lanczos_problem.stats); the steps are
    then launched one by one with events around each phase.  Without it the
    steps run as replays of a CUDA graph; ``poll_host=False`` makes the host
    synchronise once per replay instead of polling pinned progress words.
    ``sell``: a :class:`SellLayout` of the matrix (f32 path only) for the
    matvec.  ``window``: 0 for full reorthogonalisation, W > 0 to
    orthogonalise each step against the last W Krylov vectors only.
    ``packed``: a :class:`PackedLayout` of the matrix for the matvec (its
    table in the call's dtype; either dtype).
    """
    max_iter = int(min(max_iter, n))
    p = _problem(dtype, n, nnz, rowptr, cols, vals, diag, nvec, k, max_iter, tol, check_every, seed, v0, stats,
                 group, sell if dtype == 1 else None, window, packed)
    progress = _progress_words(rowptr.device) if poll_host else None
    p.host_progress = progress.data_ptr() if poll_host else None
    wb = lib.edg_lanczos_workspace_bytes(ctypes.byref(p))
    if wb < 0:
        raise _lib.EdgError(-1, _lib.last_error())
    dev = rowptr.device
    ws = workspace if (workspace is not None and workspace.numel() >= wb) else torch.empty(wb, dtype=torch.uint8, device=dev)
    tdt = torch.float64 if dtype == 0 else torch.float32
    evecs = torch.empty((k, n, nvec), dtype=tdt, device=dev) if want_vectors else None
    evals = np.zeros(nvec * k)
    iters = np.zeros(nvec, dtype=np.int32)
    resid = np.zeros(nvec * k)
    st = lib.edg_lanczos(ctypes.byref(p), ptr(ws), wb, evals.ctypes.data, ptr(evecs) if want_vectors else None,
                         iters.ctypes.data, resid.ctypes.data, stream_handle())
    if st == -5 and allow_unconverged:
        pass
    else:
        check(st, "edg_lanczos")
    return LanczosResult(evals.reshape(nvec, k), evecs, iters, resid.reshape(nvec, k))


def lanczos(mat, k=1, tol=1e-12, max_iter=400, check_every=5, seed=1234, v0=None, stats=None, tune=True, group=0):
    """f64 Lanczos on a real DeviceMatrix; returns (evals[k], evecs (n, k) device)."""
    if mat.is_complex:
        raise NotImplementedError("complex Hermitian Lanczos: assemble the real form of the model")
    g = group or (tune_spmv_group(mat, 1, 0, vals=mat.vals) if tune else 0)
    r = run_lanczos(0, mat.n, mat.nnz, mat.rowptr, mat.cols, mat.vals, mat.diag, nvec=1, k=k, max_iter=max_iter,
                    tol=tol, check_every=check_every, seed=seed, v0=v0, stats=stats, group=g)
    return r.evals[0], r.evecs[:, :, 0].T.contiguous(), r


def stack_diagonals(diags, dtype):
    """[n] diagonals of several problems -> interleaved [n][nvec] tensor."""
    return torch.stack([d.to(dtype) for d in diags], dim=1).contiguous()


def lanczos_mixed(mat, diags=None, k=1, tol32=1e-4, tol=1e-12, max_iter=400, refine_iter=5, check_every=5,
                  seed=1234, stats32=None, stats64=None, vals32=None, diag32=None, diag64=None, tune=True,
                  group32=0, group64=0, sell=None, window32=4, packed=None):
    """Mixed-precision (f32 Krylov, f64 recurrence) Lanczos + f64 refinement.

    ``diags``: list of f64 device diagonals (one per problem, <= 4) sharing the
    off-diagonal part of ``mat``; default ``[mat.diag]``.  Returns the refined
    f64 eigenvalues (nvec, k), the f64 Ritz vectors and diagnostics.

    The f32 phase only has to bring the ground state to a tol32 relative
    residual: it reorthogonalises each step against the last ``window32``
    Krylov vectors (local reorthogonalisation; 0 = full).  Without full
    reorthogonalisation the lowest Ritz pair converges at the same rate and
    its Ritz vector is accurate once its residual bound is small (Paige,
    J. Inst. Maths Applics 18 (1976) 341); what is lost is the suppression of
    later copies of converged pairs, which a ground-state solve stopped at
    convergence never meets.  The f64 refinement reorthogonalises fully.
    """
    if k != 1 and window32:
        window32 = 0  # several Ritz pairs: keep the basis orthogonal
    if mat.is_complex:
        raise NotImplementedError("mixed Lanczos needs the real form")
    diags = [mat.diag] if diags is None else list(diags)
    nvec = len(diags)
    if vals32 is None:
        vals32 = mat.vals.to(torch.float32)
    if diag32 is None:
        diag32 = stack_diagonals(diags, torch.float32)
    if diag64 is None:
        diag64 = stack_diagonals(diags, torch.float64)
    if sell is None and packed is None and tune and not group32:
        fmt, param = tune_matvec32(mat, nvec, vals32)
        if fmt == "sell":
            sell = sell_layout(mat, vals32, param)
        elif fmt == "packed":
            sell, packed = False, packed_layout(mat)
        else:
            sell, group32 = False, param
    lay = sell_layout(mat, vals32) if sell is True else (sell or None)
    pk = packed_layout(mat) if packed is True else (packed or None)
    g32 = group32 or (tune_spmv_group(mat, nvec, 1, vals=vals32) if tune and pk is None else 0)
    g64 = group64 or (tune_spmv_group(mat, nvec, 0, vals=mat.vals) if tune and pk is None else 0)
    r32 = run_lanczos(1, mat.n, mat.nnz, mat.rowptr, mat.cols, vals32, diag32, nvec=nvec, k=k, max_iter=max_iter,
                      tol=tol32, check_every=check_every, seed=seed, stats=stats32, group=g32, sell=lay,
                      window=window32, packed=pk)
    # f64 refinement: short Lanczos restarted from the f32 Ritz vector (ground state)
    v0 = torch.empty((mat.n, nvec), dtype=torch.float64, device=diag64.device)
    check(lib.edg_convert(1, ptr(r32.evecs), 0, ptr(v0), mat.n * nvec, stream_handle()), "edg_convert")
    r64 = run_lanczos(0, mat.n, mat.nnz, mat.rowptr, mat.cols, mat.vals, diag64, nvec=nvec, k=1,
                      max_iter=refine_iter, tol=tol, check_every=refine_iter, seed=seed, v0=v0,
                      allow_unconverged=True, stats=stats64, group=g64, packed=pk)
    return r64, r32
