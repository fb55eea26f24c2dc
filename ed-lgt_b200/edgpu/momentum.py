"""Momentum (translation) sectors on the device.

Mirrors ``QuantumModel.set_momentum_sector`` (edlgt/models/quantum_model.py:
213-276) with ``get_momentum_basis`` and its zero-k / finite-k projectors
(edlgt/symmetries/translational_sym.py:508-949, 1307-1358).  The projector B
(sector rows x momentum states) is built by ``edg_momentum_translations``,
``edg_momentum_references``, ``edg_momentum_columns`` and
``edg_momentum_rowmap``; the reference then assembles B^dagger O B term by
term (``nbody_data_momentum*``, :1394-1969), here H_k = B^dagger H B is
applied without being formed: ``edg_momentum_expand``, the sector matvec,
``edg_momentum_reduce``.  Spectra come from a dense Hermitian solve of H_k
(columns applied to unit vectors) up to ``DENSE_MAX`` momentum states and from
a fully reorthogonalised Lanczos above that.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = ["MomentumBasis", "translation_sources", "krylov_evolve", "DENSE_MAX"]

DENSE_MAX = 4096


def translation_sources(lvals, unit_cell):
    """source[s, dest] = site whose local state lands on ``dest`` under the
    block shift s; shifts and sites both enumerated row-major (first axis
    slowest), as _prepare_translation_source_sites
    (translational_sym.py:508-560)."""
    lvals = np.asarray(lvals, dtype=np.int64)
    ucs = np.asarray(unit_cell, dtype=np.int64)
    if lvals.shape != ucs.shape or np.any(ucs < 1) or np.any(lvals % ucs):
        raise ValueError("unit cell sizes must divide the lattice lengths, one per axis")
    R = lvals // ucs
    n_sites = int(np.prod(lvals))
    coords = np.stack(np.unravel_index(np.arange(n_sites), tuple(lvals)), axis=1)
    n_shifts = int(np.prod(R))
    src = np.empty((n_shifts, n_sites), dtype=np.int32)
    for s in range(n_shifts):
        t = np.array(np.unravel_index(s, tuple(R)))
        dest = np.ravel_multi_index(tuple(((coords + t * ucs) % lvals).T), tuple(lvals))
        src[s, dest] = np.arange(n_sites)
    return src, R.astype(np.int32)


def _phase_table(k_vals, R):
    """exp(-2 pi i k_d t / R_d) by repeated products, [dim][max R]
    (_prepare_phase_table, translational_sym.py:344-365)."""
    D, max_r = len(R), int(np.max(R))
    tab = np.zeros((D, max_r), dtype=np.complex128)
    for d in range(D):
        tab[d, 0] = 1.0
        if R[d] <= 1:
            continue
        step = np.exp(-1j * 2.0 * np.pi * (int(k_vals[d]) % int(R[d])) / float(R[d]))
        for t in range(1, int(R[d])):
            tab[d, t] = tab[d, t - 1] * step
    return tab


class MomentumBasis:
    """The projector B of one momentum sector, on the device."""

    def __init__(self, sector, lvals, unit_cell, k_vals, local_map=None, label_sign=None):
        """``local_map`` / ``label_sign``: the translation-charge variant (1D,
        unit cell 1): the local map applied with every unit shift and the
        per-state signs whose product twists the odd shifts."""
        sector.require_narrow("momentum basis")
        dev = sector.device
        self.sector = sector
        self.device = dev
        n = len(sector)
        src, R = translation_sources(lvals, unit_cell)
        tc = local_map is not None
        if tc and (len(R) != 1 or src.shape[0] != src.shape[1]):
            raise ValueError("the translation-charge basis is defined on a 1D ring with a one-site unit cell")
        k_vals = np.asarray(k_vals, dtype=np.int64).reshape(-1)
        if len(k_vals) != len(R):
            raise ValueError(f"expected {len(R)} momentum labels, got {len(k_vals)}")
        if len(R) > 3:
            raise ValueError("momentum sectors support 1 to 3 lattice dimensions")
        n_shifts = src.shape[0]
        self.n_rows = n
        self.zero_k = not np.any(k_vals != 0)
        g = _lib.MomentumGroup()
        g.lattice_dim = len(R)
        g.n_shifts = n_shifts
        stride = 1
        for d in range(len(R) - 1, -1, -1):
            g.shifts_per_dir[d] = int(R[d])
            g.shift_strides[d] = stride
            g.k_vals[d] = int(k_vals[d])
            stride *= int(R[d])
        self.group = g
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        src_d = up(src)
        strides = up(sector.strides.astype(np.int64))
        loc = up(sector.loc_dims.astype(np.int32))
        flag = torch.zeros(1, dtype=torch.int32, device=dev)
        trans = torch.empty((max(n, 1), n_shifts), dtype=torch.int32, device=dev)
        if tc:
            cmap = up(np.asarray(local_map, dtype=np.int32))
            lsign = up(np.asarray(label_sign, dtype=np.float64))
            row_sign = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
            map_args = (ptr(cmap), int(cmap.shape[0]), ptr(lsign), ptr(row_sign))
        else:
            row_sign = None
            map_args = (None, 0, None, None)
        check(lib.edg_momentum_translations(sector.lookup_table(), ptr(strides), ptr(loc), int(sector.n_sites),
                                            ptr(src_d), n_shifts, *map_args, ptr(trans), ptr(flag), stream_handle()),
              "edg_momentum_translations")
        rs = ptr(row_sign) if tc else None
        ns = lib.edg_momentum_scratch_elems(n)
        scratch = torch.empty(max(ns, 1), dtype=torch.int64, device=dev)
        pvec = torch.empty((max(n, 1), len(R)), dtype=torch.int32, device=dev)
        refs = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
        n_cols = ctypes.c_int64(0)
        check(lib.edg_momentum_references(ptr(trans), n, ctypes.byref(g), ptr(pvec), ptr(refs), ctypes.byref(n_cols),
                                          ptr(scratch), ns, stream_handle()), "edg_momentum_references")
        m = int(n_cols.value)
        self.n_cols = m
        tab = up(_phase_table(k_vals, R))
        col_ptr = torch.empty(m + 1, dtype=torch.int64, device=dev)
        nnz = ctypes.c_int64(0)
        cs = lib.edg_scan_scratch_elems(m)
        cscratch = torch.empty(max(cs, 1), dtype=torch.int64, device=dev)
        zk = 1 if self.zero_k else 0
        check(lib.edg_momentum_columns(ptr(trans), ptr(refs), m, ptr(pvec), ctypes.byref(g), ptr(tab), tab.shape[1],
                                       zk, rs, ptr(col_ptr), ctypes.byref(nnz), None, None, ptr(cscratch), cs,
                                       stream_handle()), "edg_momentum_columns")
        self.nnz = int(nnz.value)
        row_idx = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        data = torch.empty(max(self.nnz, 1), dtype=torch.complex128, device=dev)
        check(lib.edg_momentum_columns(ptr(trans), ptr(refs), m, ptr(pvec), ctypes.byref(g), ptr(tab), tab.shape[1],
                                       zk, rs, ptr(col_ptr), ctypes.byref(nnz), ptr(row_idx), ptr(data),
                                       ptr(cscratch), cs, stream_handle()), "edg_momentum_columns")
        row_col = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
        row_val = torch.empty(max(n, 1), dtype=torch.complex128, device=dev)
        check(lib.edg_momentum_rowmap(ptr(col_ptr), ptr(row_idx), ptr(data), m, n, ptr(row_col), ptr(row_val),
                                      ptr(flag), stream_handle()), "edg_momentum_rowmap")
        self.col_ptr, self.row_idx, self.data = col_ptr, row_idx, data
        self.row_col, self.row_val = row_col, row_val
        self.refs = refs[:m]
        self._bound = None

    # ------------------------------------------------------------ host view
    def host_arrays(self) -> dict:
        """The reference's momentum_basis dict (CSC and CSR of B, host)."""
        cp = self.col_ptr.cpu().numpy()
        ri = self.row_idx[: self.nnz].cpu().numpy().astype(np.int32)
        dv = self.data[: self.nnz].cpu().numpy()
        if self.zero_k:
            dv = dv.real.copy()
        rc = self.row_col[: self.n_rows].cpu().numpy()
        rv = self.row_val[: self.n_rows].cpu().numpy()
        has = rc >= 0
        r_ptr = np.zeros(self.n_rows + 1, dtype=np.int32)
        r_ptr[1:] = np.cumsum(has)
        r_val = rv[has].real.copy() if self.zero_k else rv[has]
        return {"pair_mode": False, "n_rows": self.n_rows, "n_cols": self.n_cols, "L_col_ptr": cp.astype(np.int32),
                "L_row_idx": ri, "L_data": dv, "R_row_ptr": r_ptr, "R_col_idx": rc[has].astype(np.int32),
                "R_data": r_val}

    # ------------------------------------------------------------ operator
    def bind(self, ham):
        """Attach the sector Hamiltonian (``QMB_hamiltonian`` with a built
        matrix); a real-form matrix gets its gauge phases folded into B."""
        mat = ham.mat
        ph = ham._row_phase()
        if ph is None:
            rv, dv = self.row_val, self.data
        else:
            rv = torch.conj(ph) * self.row_val[: self.n_rows]
            rows = self.row_idx[: self.nnz].to(torch.int64)
            dv = torch.conj(ph[rows]) * self.data[: self.nnz] if self.nnz else self.data
        # a complex vector on a real matrix runs as two interleaved real
        # right-hand sides, whose diagonals the batched matvec reads per side
        diag = mat.diag if mat.is_complex else mat.diag.repeat_interleave(2).contiguous()
        self._bound = (mat, rv.contiguous(), dv.contiguous(), diag)

    def matvec(self, x: torch.Tensor) -> torch.Tensor:
        """y = B^dagger H B x for a complex128 momentum-space vector."""
        mat, rv, dv, diag = self._bound
        x = x.to(torch.complex128).contiguous()
        v = torch.empty(self.n_rows, dtype=torch.complex128, device=self.device)
        check(lib.edg_momentum_expand(self.n_rows, ptr(self.row_col), ptr(rv), ptr(x), ptr(v), stream_handle()),
              "edg_momentum_expand")
        w = torch.empty_like(v)
        if mat.is_complex:
            code, nvec = 2, 1
        else:
            code, nvec = 0, 2  # a complex vector is two interleaved real ones
        check(lib.edg_spmv(code, mat.n, mat.nnz, ptr(mat.rowptr), ptr(mat.cols) if mat.nnz else None,
                           ptr(mat.vals) if mat.nnz else None, ptr(diag), nvec, ptr(v), ptr(w), stream_handle()),
              "edg_spmv")
        y = torch.empty(self.n_cols, dtype=torch.complex128, device=self.device)
        check(lib.edg_momentum_reduce(self.n_cols, ptr(self.col_ptr), ptr(self.row_idx), ptr(dv), ptr(w), ptr(y),
                                      stream_handle()), "edg_momentum_reduce")
        return y

    def dense(self) -> torch.Tensor:
        """H_k as a dense (n_cols, n_cols) complex128 matrix (column by column)."""
        m = self.n_cols
        out = torch.empty((m, m), dtype=torch.complex128, device=self.device)
        e = torch.zeros(m, dtype=torch.complex128, device=self.device)
        for c in range(m):
            e.zero_()
            e[c] = 1.0
            out[:, c] = self.matvec(e)
        return out

    def lowest(self, k, tol=1e-12, max_iter=None, seed=0):
        """(energies, vectors [n_cols, k]) of H_k, ascending."""
        m = self.n_cols
        if m == 0:
            raise ValueError("the momentum sector is empty")
        if k > m:
            raise ValueError(f"n_eigs must be <= {m}")
        if m <= DENSE_MAX:
            h = self.dense()
            h = 0.5 * (h + h.conj().T)
            w, v = torch.linalg.eigh(h)
            self.last_matvecs = m
            return w[:k].cpu().numpy(), v[:, :k]
        w, v, its = _lanczos(self.matvec, m, k, tol, max_iter or min(m, 400), self.device, seed)
        self.last_matvecs = its
        return w, v


def krylov_evolve(apply, psi0, time_line, m_krylov=40, tol=1e-12):
    """psi(t) = exp(-i H t) psi0 at every (absolute) time of ``time_line``, the
    role of expm_multiply in QMB_hamiltonian.time_evolution
    (edlgt/modeling/qmb_hamiltonian.py:370-384): each interval is covered by
    Lanczos-exponential steps whose size halves until the a-posteriori error
    estimate beta_m |[exp(-i T dt)]_{m-1,0}| is at most ``tol``."""
    from scipy.linalg import expm

    time_line = np.asarray(time_line, dtype=np.float64)
    if len(time_line) == 0 or time_line[0] < 0 or np.any(np.diff(time_line) < 0):
        raise ValueError("time_line must be ascending and start at t >= 0")
    psi = psi0.to(torch.complex128).clone()
    n = psi.shape[0]
    m_k = max(1, min(m_krylov, n))
    out = []
    t_prev = 0.0  # expm_multiply returns exp(-i H t) psi0 at the absolute times
    dt_try = None
    for t in time_line:
        remaining = float(t) - t_prev
        while remaining > 0:
            nrm = float(torch.linalg.vector_norm(psi))
            if nrm == 0.0:
                break
            V = torch.empty((m_k + 1, n), dtype=torch.complex128, device=psi.device)
            V[0] = psi / nrm
            a, b = [], []
            j_used = m_k
            for j in range(m_k):
                w = apply(V[j])
                a.append(float(torch.vdot(V[j], w).real))
                for _ in range(2):
                    w = w - V[: j + 1].T @ (V[: j + 1].conj() @ w)
                bj = float(torch.linalg.vector_norm(w))
                b.append(bj)
                if bj <= 1e-14 * max(1.0, abs(a[-1])):
                    j_used = j + 1
                    break
                V[j + 1] = w / bj
            T = np.diag(a[:j_used]) + np.diag(b[: j_used - 1], 1) + np.diag(b[: j_used - 1], -1)
            dt = remaining if dt_try is None else min(remaining, dt_try)
            while True:
                E = expm(-1j * dt * T)
                err = (b[j_used - 1] if j_used == m_k else 0.0) * abs(E[j_used - 1, 0]) * nrm
                if err <= tol or dt < 1e-12:
                    break
                dt *= 0.5
            coef = torch.from_numpy(np.ascontiguousarray(E[:, 0] * nrm)).to(psi.device)
            psi = V[:j_used].T @ coef
            remaining -= dt
            dt_try = 2 * dt
        t_prev = float(t)
        out.append(psi.clone())
    return out


def _lanczos(apply, m, k, tol, max_iter, device, seed):
    """Lanczos with two classical Gram-Schmidt passes against the whole basis
    on complex128 vectors; converged when every wanted Ritz pair has
    |beta_j s_jk| <= tol max(1, |theta_k|)."""
    from scipy.linalg import eigh_tridiagonal

    gen = torch.Generator(device=device).manual_seed(seed)
    q = torch.randn(m, dtype=torch.complex128, device=device, generator=gen)
    Q = torch.empty((max_iter + 1, m), dtype=torch.complex128, device=device)
    Q[0] = q / torch.linalg.vector_norm(q)
    alpha, beta = [], []
    theta = s = None
    for j in range(max_iter):
        w = apply(Q[j])
        a = float(torch.vdot(Q[j], w).real)
        alpha.append(a)
        for _ in range(2):
            w = w - Q[: j + 1].T @ (Q[: j + 1].conj() @ w)
        b = float(torch.linalg.vector_norm(w))
        done = b <= 1e-14 * max(1.0, abs(a)) or j + 1 == max_iter
        if j + 1 >= k and (done or (j + 1) % 5 == 0):
            theta, s = eigh_tridiagonal(np.array(alpha), np.array(beta), select="i", select_range=(0, k - 1))
            res = np.abs(b * s[-1, :])
            if done or np.all(res <= tol * np.maximum(1.0, np.abs(theta))):
                break
        beta.append(b)
        Q[j + 1] = w / b
    n_used = len(alpha)
    vecs = Q[:n_used].T @ torch.from_numpy(s.astype(np.complex128)).to(device)
    return theta, vecs, n_used
