"""Krylov time evolution on the device.

:func:`krylov_evolve` advances a state along a uniform time grid with
``edg_krylov_step`` (exp(-i H dt) by an m-dimensional Lanczos/Krylov basis,
f64 recurrence and small exponential), the drop-in for the
``expm_multiply(-iH, psi0, start, stop, num)`` call of
edlgt/modeling/qmb_hamiltonian.py:377-420.  Precision ``"c128"`` keeps the
basis in complex128 with the f64 matrix; ``"c64"`` keeps it in complex64 with
an f32 copy of the matrix.  Local observables can be measured on the device
at every time point instead of keeping the states.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = ["KrylovEvolver", "krylov_evolve"]


class KrylovEvolver:
    """Holds the device copies and the workspace of one Hamiltonian.

    ``matvec``: "auto" uses the dictionary-packed tiled layout of a real
    matrix when it packs (a complex vector is two real right-hand sides of
    it; f32 lane sums for complex64, f64 for complex128), else CSR;
    "csr" forces CSR."""

    def __init__(self, mat, m=30, precision="c128", reorth_passes=1, spmv_group=None, matvec="auto"):
        if precision not in ("c128", "c64"):
            raise ValueError("precision must be 'c128' or 'c64'")
        self.mat = mat
        self.m = int(min(m, mat.n))
        self.precision = precision
        dev = mat.rowptr.device
        if mat.is_complex:
            vals = mat.vals.view(torch.complex128)
            diag = mat.diag.view(torch.complex128)
            mdt = 2
        else:
            vals, diag, mdt = mat.vals, mat.diag, 0
        if precision == "c64":
            vals = vals.to(torch.complex64 if mat.is_complex else torch.float32)
            diag = diag.to(torch.complex64 if mat.is_complex else torch.float32)
            mdt += 1
        self.vals, self.diag = vals, diag
        p = _lib.KrylovProblem()
        p.vec_dtype = 2 if precision == "c128" else 3
        p.mat_dtype = mdt
        p.n_rows = mat.n
        p.nnz = mat.nnz
        p.rowptr = ptr(mat.rowptr)
        p.cols = ptr(mat.cols) if mat.nnz else None
        p.vals = ptr(vals) if mat.nnz else None
        p.diag = ptr(diag)
        p.m = self.m
        p.reorth_passes = reorth_passes
        self.packed = None
        if matvec == "auto" and not mat.is_complex:
            from .solvers import packed_layout

            self.packed = packed_layout(mat)
        if spmv_group is None:
            # a complex vector is two real right-hand sides for a real matrix:
            # tune the CSR kernel on that shape (real forms only)
            from .solvers import tune_spmv_group

            spmv_group = 0 if (mat.is_complex or self.packed is not None) else tune_spmv_group(
                mat, 2, 0 if precision == "c128" else 1, vals=mat.vals if precision == "c128" else vals)
        p.spmv_group = int(spmv_group)
        if self.packed is not None:
            pk = self.packed
            p.pk_tile_off, p.pk_words = ptr(pk.tile_off), ptr(pk.words)
            p.pk_table = ptr(pk.table(0 if precision == "c128" else 1))
            p.pk_count, p.pk_colbits = pk.count, pk.colbits
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        p.status = ptr(self.status)
        self.p = p
        wb = lib.edg_krylov_workspace_bytes(ctypes.byref(p))
        if wb < 0:
            raise _lib.EdgError(-1, _lib.last_error())
        self.ws = torch.empty(wb, dtype=torch.uint8, device=dev)
        self.wb = wb
        self.vdtype = torch.complex128 if precision == "c128" else torch.complex64

    def check_status(self):
        """Raise if a stage wait of the packed matvec ran out (one host read)."""
        st = int(self.status.item())
        if st != 0:
            raise _lib.EdgError(st, "edg_krylov_step: a stage wait of the packed matvec ran out")

    def step(self, psi: torch.Tensor, dt: float, want_error=False):
        err = np.zeros(1) if want_error else None
        check(lib.edg_krylov_step(ctypes.byref(self.p), ptr(psi), float(dt), ptr(self.ws), self.wb,
                                  err.ctypes.data if want_error else None, stream_handle()), "edg_krylov_step")
        return float(err[0]) if want_error else None


def krylov_evolve(mat, psi0, time_line, m=30, precision="c128", keep_states=True, observables=None,
                  reorth_passes=1, matvec="auto"):
    """psi(t_k) on a uniform grid (list of device vectors) or, when
    ``observables`` maps names to ``(sector, site_op)`` pairs, the per-site
    expectation values ``{name: (n_t, n_sites) array}``."""
    t = np.asarray(time_line, dtype=float)
    ev = KrylovEvolver(mat, m=m, precision=precision, reorth_passes=reorth_passes, matvec=matvec)
    psi = psi0.to(ev.vdtype).clone().contiguous()
    states = []
    results = {}
    if observables:
        from .models.quantum_model import site_expval_device

        for name in observables:
            results[name] = torch.zeros((len(t), observables[name][1].shape[0]), dtype=torch.float64,
                                        device=psi.device)
    for k in range(len(t)):
        if k > 0:
            ev.step(psi, t[k] - t[k - 1])
        if keep_states:
            states.append(psi.clone())
        if observables:
            for name, (sector, op) in observables.items():
                site_expval_device(sector, op, psi, out=results[name][k])
    ev.check_status()
    if observables:
        return {name: r.cpu().numpy() for name, r in results.items()}
    return states
