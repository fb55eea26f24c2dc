"""Device assembly of the sector Hamiltonian from term blocks.

Host side: the term blocks are flattened into local transition tables (the
nonzero entries, ``|op| > 1e-10``, of every site operator used, as
``_prepare_local_transition_data`` does, edlgt/symmetries/
sym_qmb_operations.py:32-92) plus one record per term instance.  The device
builds the canonical matrix (duplicates summed, columns ascending) in three
kernels: per-row entry bounds, generation + per-row merge, compaction.

Real form.  The gauge models' hoppings carry factors ``-i t``; a diagonal
unitary ``D = prod_s phi_s(c_s)`` with ``phi_s(c) = i**(w_s(c))`` (``w`` a
per-site integer weight, typically x-coordinate times matter number) maps
``H`` to ``D^dagger H D``, applied here factor by factor to the site
operators.  When every transformed site table has a single common phase and
every instance's total phase is real, the matrix is assembled real; otherwise
the faithful complex matrix is assembled.  Eigenvalues are unchanged and
eigenvectors map back by ``psi = D psi'``.
"""

from __future__ import annotations

import hashlib

import numpy as np
import torch

from .. import _lib
from .._lib import check, lib, ptr, stream_handle
from .terms import TermBlock

__all__ = ["DeviceMatrix", "assemble_blocks", "OP_TOL"]

OP_TOL = 1e-10


class DeviceMatrix:
    """Canonical sector matrix: off-diagonal CSR + dense diagonal, on the device.

    ``vals``/``diag`` are float64 tensors (interleaved re/im when ``is_complex``).
    ``diag_present`` marks rows whose (r, r) entry exists in the reference's
    triplet set (a local term with ``|op_cc| >= 1e-10`` or a diagonal hit).
    ``phase_weights`` (n_sites, dmax) integer exponents of ``i`` of the real
    form's gauge transform, or None.
    """

    def __init__(self, n, rowptr, cols, vals, diag, diag_present, is_complex, phase_weights=None):
        self.n = int(n)
        self.rowptr = rowptr
        self.cols = cols
        self.vals = vals
        self.diag = diag
        self.diag_present = diag_present
        self.is_complex = bool(is_complex)
        self.phase_weights = phase_weights
        self.nnz = int(cols.shape[0]) if cols is not None else 0

    @property
    def shape(self):
        return (self.n, self.n)

    def dtype_code(self):
        return 2 if self.is_complex else 0

    def to_scipy(self, include_diag=True):
        """Host canonical CSR (pattern of the reference after summing duplicates)."""
        from scipy.sparse import csr_matrix

        rp = self.rowptr.cpu().numpy()
        cols = self.cols.cpu().numpy()[: self.nnz].astype(np.int64)
        v = self.vals.cpu().numpy()
        d = self.diag.cpu().numpy()
        if self.is_complex:
            v = v.view(np.complex128)[: self.nnz]
            d = d.view(np.complex128)
        else:
            v = v[: self.nnz]
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        if include_diag:
            pres = self.diag_present.cpu().numpy().astype(bool)
            r = np.nonzero(pres)[0]
            rows = np.concatenate([rows, r])
            cols = np.concatenate([cols, r])
            v = np.concatenate([v, d[r]])
            order = np.lexsort((cols, rows))
            rows, cols, v = rows[order], cols[order], v[order]
        indptr = np.zeros(self.n + 1, dtype=np.int64)
        np.add.at(indptr, rows + 1, 1)
        indptr = np.cumsum(indptr)
        return csr_matrix((v, cols, indptr), shape=self.shape)

    def matvec(self, x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """y = H x on the device (x: float64 or complex128 tensor of length n)."""
        if self.is_complex:
            x = x.to(torch.complex128)
            code = 2
        else:
            if x.is_complex():
                raise TypeError("real matrix: use a real vector (or apply to real and imaginary parts)")
            x = x.to(torch.float64)
            code = 0
        y = torch.empty_like(x) if out is None else out
        check(lib.edg_spmv(code, self.n, self.nnz, ptr(self.rowptr), ptr(self.cols) if self.nnz else None,
                           ptr(self.vals) if self.nnz else None, ptr(self.diag), 1, ptr(x), ptr(y), stream_handle()),
              "edg_spmv")
        return y


def _uniform_phase(mat, tol=1e-12):
    """Common phase e^{i theta} of all entries above OP_TOL, or None."""
    nz = mat[np.abs(mat) > OP_TOL]
    if nz.size == 0:
        return 1.0 + 0.0j
    ph = nz[np.argmax(np.abs(nz))]
    ph = ph / abs(ph)
    rot = nz / ph
    if np.all(np.abs(rot.imag) <= tol * np.maximum(1.0, np.abs(rot))):
        return ph
    return None


def _phase_vec(weights_row):
    return np.power(1j, np.asarray(weights_row, dtype=np.int64) % 4)


def _offdiag_signature(blocks, phase_weights, force_complex, dmax):
    """Content hash of everything the off-diagonal part of the matrix depends
    on: the off-diagonal blocks' operators, instances, strengths and h.c.
    flags, the real form's phase weights and the form request."""
    h = hashlib.sha256(repr((bool(force_complex), int(dmax))).encode())
    if phase_weights is not None:
        h.update(np.ascontiguousarray(np.asarray(phase_weights, dtype=np.int64)).tobytes())
    for b in blocks:
        if b.diagonal:
            continue
        h.update(repr((b.strength, b.add_dagger, len(b.ops))).encode())
        h.update(np.ascontiguousarray(b.sites).tobytes())
        for o in b.ops:
            o = np.ascontiguousarray(o)
            h.update(repr((str(o.dtype), o.shape)).encode())
            h.update(o.tobytes())
    return h.hexdigest()


def _offdiag_tables(blocks, phase_weights, force_complex, dmax):
    """Local transition tables and instance records of the off-diagonal
    blocks, and whether they admit the real form (every gauge-transformed
    table has one common phase and every instance's total phase is real)."""
    raw_tables = []  # list of (d x d) complex matrices
    table_site = []
    table_index = {}
    terms = []  # (sites tuple, tables tuple, coef)
    for bi, b in enumerate(blocks):
        if b.diagonal:
            continue
        for dag in ([False, True] if b.add_dagger else [False]):
            for inst in b.sites:
                tabs = []
                for j, s in enumerate(inst):
                    key = (bi, j, int(s), dag)
                    if key not in table_index:
                        m = np.asarray(b.ops[j][int(s)], dtype=np.complex128)
                        if dag:
                            m = m.conj().T
                        table_index[key] = len(raw_tables)
                        raw_tables.append(m)
                        table_site.append(int(s))
                    tabs.append(table_index[key])
                if len(set(int(s) for s in inst)) != len(inst):
                    raise ValueError("a term instance acts twice on the same site")
                coef = np.conj(b.strength) if dag else b.strength
                terms.append((tuple(int(s) for s in inst), tuple(tabs), complex(coef)))
    real_ok, tables_real, coefs_real = False, None, None
    if not force_complex and raw_tables:
        # every table at once: gauge-transform, then its common phase (the
        # phase of its largest entry above OP_TOL, the first in row-major
        # order), as _uniform_phase does table by table
        M = np.stack(raw_tables)
        if phase_weights is not None:
            phi = _phase_vec(np.asarray(phase_weights)[np.asarray(table_site)])  # (nt, d)
            M = np.conj(phi)[:, :, None] * M * phi[:, None, :]
        mag = np.abs(M)
        keep = mag > OP_TOL
        flat = np.where(keep, mag, -1.0).reshape(len(raw_tables), -1)
        big = np.take_along_axis(M.reshape(len(raw_tables), -1), flat.argmax(axis=1)[:, None], axis=1)[:, 0]
        ph = np.where(keep.reshape(len(raw_tables), -1).any(axis=1), big / np.where(big == 0, 1.0, np.abs(big)),
                      1.0 + 0.0j)
        rot = M / ph[:, None, None]
        bad = keep & (np.abs(rot.imag) > 1e-12 * np.maximum(1.0, np.abs(rot)))
        ok = not bad.any()
        if ok:
            tabs_t = list(rot.real)
            phases = list(ph)
        if ok:
            cr = []
            for sites, tabs, coef in terms:
                z = coef
                for t in tabs:
                    z *= phases[t]
                if abs(z.imag) > 1e-12 * max(1.0, abs(z)):
                    ok = False
                    break
                cr.append(z.real)
        if ok:
            real_ok, tables_real, coefs_real = True, tabs_t, cr
    return raw_tables, terms, real_ok, tables_real, coefs_real


def _table_arrays(raw_tables, terms, dmax, is_complex, tables_real, coefs_real):
    """Device table arrays: per table and bra the kets whose |amplitude| >
    OP_TOL in ascending order (t_count, t_ket, t_amp, zero beyond the
    count), and the instance records (term_nops, term_site, term_table,
    term_coef).  Vectorised over all tables at once."""
    nt = max(len(raw_tables), 1)
    t_count = np.zeros((nt, dmax), dtype=np.int32)
    t_ket = np.zeros((nt, dmax, dmax), dtype=np.uint8)
    t_amp = np.zeros((nt, dmax, dmax, 2 if is_complex else 1), dtype=np.float64)
    if raw_tables:
        mags = np.abs(np.stack([np.asarray(m, dtype=np.complex128) for m in raw_tables]))[:, :dmax, :dmax]
        vals = np.stack(raw_tables if is_complex else [np.asarray(m) for m in tables_real])[:, :dmax, :dmax]
        keep = mags > OP_TOL
        k = mags.shape[-1]
        order = np.argsort(~keep, axis=-1, kind="stable")  # kept kets first, ascending
        cnt = keep.sum(axis=-1)
        valid = np.arange(k)[None, None, :] < cnt[..., None]
        t_count[:, : mags.shape[1]] = cnt
        t_ket[:, : mags.shape[1], :k] = np.where(valid, order, 0)
        picked = np.take_along_axis(vals, order, axis=-1)
        if is_complex:
            t_amp[:, : mags.shape[1], :k, 0] = np.where(valid, picked.real, 0.0)
            t_amp[:, : mags.shape[1], :k, 1] = np.where(valid, picked.imag, 0.0)
        else:
            t_amp[:, : mags.shape[1], :k, 0] = np.where(valid, np.real(picked), 0.0)
    n_terms = len(terms)
    term_nops = np.zeros(max(n_terms, 1), dtype=np.int32)
    term_site = np.zeros((max(n_terms, 1), _lib.MAX_OPS), dtype=np.int32)
    term_table = np.zeros((max(n_terms, 1), _lib.MAX_OPS), dtype=np.int32)
    term_coef = np.zeros((max(n_terms, 1), 2 if is_complex else 1), dtype=np.float64)
    for k_, (sites, tabs, coef) in enumerate(terms):
        if len(sites) > _lib.MAX_OPS:
            raise ValueError(f"at most {_lib.MAX_OPS} operator factors per term instance")
        term_nops[k_] = len(sites)
        term_site[k_, : len(sites)] = sites
        term_table[k_, : len(tabs)] = tabs
    if n_terms:
        if is_complex:
            c = np.array([t[2] for t in terms], dtype=np.complex128)
            term_coef[:n_terms, 0], term_coef[:n_terms, 1] = c.real, c.imag
        else:
            term_coef[:n_terms, 0] = coefs_real
    return [t_count, t_ket, t_amp, term_nops, term_site, term_table, term_coef]


def assemble_blocks(sector, blocks, phase_weights=None, force_complex=False, extra_diag=None):
    """Assemble the canonical matrix of ``sum(blocks)`` in ``sector``.

    ``extra_diag``: optional constant added to every diagonal element (identity
    terms).  Returns a :class:`DeviceMatrix`.

    The off-diagonal part (CSR plus the diagonal contributions of instances
    that map a state to itself) depends only on the off-diagonal blocks, the
    phase weights and the form; the sector keeps the last one built, and a
    build whose off-diagonal blocks hash to the same content (a coupling
    sweep that changes diagonal terms only) reuses it and computes only the
    diagonal.
    """
    import ctypes

    loc_dims = sector.loc_dims
    dmax = None
    for b in blocks:
        dmax = b.ops[0].shape[-1] if dmax is None else dmax
    if dmax is None:
        dmax = int(loc_dims.max())
    dev = sector.device
    st = stream_handle()
    n = len(sector)

    # diagonal terms: (site, diag vector, coef)
    dterms = []
    for b in blocks:
        if not b.diagonal:
            continue
        for inst in b.sites:
            s = int(inst[0])
            dterms.append((s, np.diagonal(np.asarray(b.ops[0][s], dtype=np.complex128)).copy(), complex(b.strength)))
    dterms_real = all(not np.any(np.abs(dvec.imag) > 1e-12) and abs(coef.imag) <= 1e-12 for _, dvec, coef in dterms)

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    # ---- off-diagonal part: reused or built ----
    sig = _offdiag_signature(blocks, phase_weights, force_complex, dmax)
    off = getattr(sector, "_offdiag_cache", None)
    reused = off is not None and off["sig"] == sig and off["use_real"] == (off["real_ok"] and dterms_real)
    keep = []
    if not reused:
        raw_tables, terms, real_ok, tables_real, coefs_real = _offdiag_tables(blocks, phase_weights, force_complex,
                                                                              dmax)
        use_real = real_ok and dterms_real
        arrays = _table_arrays(raw_tables, terms, dmax, not use_real, tables_real, coefs_real)
        keep = [up(a) for a in arrays]
        off = _assemble_offdiag(sector, dev, st, n, 1 if use_real else 2, dmax, not use_real, len(terms), keep)
        off.update(sig=sig, real_ok=real_ok, use_real=use_real)
        sector._offdiag_cache = off
    is_complex = not off["use_real"]
    w = 2 if is_complex else 1

    # ---- diagonal terms: one pass without off-diagonal instances ----
    diag = off["diag"].clone()
    present = off["present"].clone()
    n_d = len(dterms)
    if n_d > 0 and n > 0:
        dterm_site = np.zeros(n_d, dtype=np.int32)
        dterm_diag = np.zeros((n_d, dmax, w), dtype=np.float64)
        dterm_coef = np.zeros((n_d, w), dtype=np.float64)
        for k, (s, dvec, coef) in enumerate(dterms):
            dterm_site[k] = s
            dterm_diag[k, : len(dvec), 0] = dvec.real
            dterm_coef[k, 0] = coef.real
            if is_complex:
                dterm_diag[k, : len(dvec), 1] = dvec.imag
                dterm_coef[k, 1] = coef.imag
        dk = [up(dterm_site), up(dterm_diag), up(dterm_coef)]
        keep += dk
        a = _assembly_struct(sector, dmax, is_complex)
        a.n_terms = 0
        a.n_dterms = n_d
        a.dterm_site, a.dterm_diag, a.dterm_coef = ptr(dk[0]), ptr(dk[1]), ptr(dk[2])
        zeros = torch.zeros(n + 1, dtype=torch.int64, device=dev)
        one_i = torch.empty(1, dtype=torch.int32, device=dev)
        one_d = torch.empty(w, dtype=torch.float64, device=dev)
        row_nnz = torch.empty(n, dtype=torch.int64, device=dev)
        d_diag = torch.empty(n * w, dtype=torch.float64, device=dev)
        d_present = torch.empty(n, dtype=torch.uint8, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        check(lib.edg_assemble_fill(ctypes.byref(a), ptr(zeros), ptr(one_i), ptr(one_d), ptr(row_nnz), ptr(d_diag),
                                    ptr(d_present), ptr(err), st), "edg_assemble_fill")
        diag += d_diag
        present |= d_present
    if extra_diag is not None and extra_diag != 0:
        if is_complex:
            diag.view(-1, 2)[:, 0] += float(np.real(extra_diag))
            diag.view(-1, 2)[:, 1] += float(np.imag(extra_diag))
        else:
            diag += float(np.real(extra_diag))
        present.fill_(1)
    mat = DeviceMatrix(n, off["rowptr"], off["cols"], off["vals"], diag, present, is_complex,
                       phase_weights if (not is_complex and phase_weights is not None) else None)
    mat._keep = keep  # device tables uploaded by this build
    mat.raw_entries = off["raw_entries"]  # generated entries before the per-row merge
    mat.offdiag_reused = reused  # off-diagonal part shared with an earlier build
    return mat


def _assembly_struct(sector, dmax, is_complex):
    a = _lib.Assembly()
    a.n_sites = sector.n_sites
    a.dmax = dmax
    for s in range(sector.n_sites):
        a.loc_dims[s] = int(sector.loc_dims[s])
        a.strides[s] = int(sector.strides[s])
    a.sector = sector.lookup_table()
    a.complex_values = 1 if is_complex else 0
    return a


def _assemble_offdiag(sector, dev, st, n, w, dmax, is_complex, n_terms, tabs):
    """Off-diagonal instances only: count, scan, fill (with per-row merge)
    and compaction; returns the CSR, the diagonal contributions of
    instances whose ket is the bra, and their presence flags."""
    import ctypes

    a = _assembly_struct(sector, dmax, is_complex)
    a.t_count, a.t_ket, a.t_amp = ptr(tabs[0]), ptr(tabs[1]), ptr(tabs[2])
    a.n_terms = n_terms
    a.term_nops, a.term_site, a.term_table, a.term_coef = ptr(tabs[3]), ptr(tabs[4]), ptr(tabs[5]), ptr(tabs[6])
    a.n_dterms = 0
    bound = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    check(lib.edg_assemble_count(ctypes.byref(a), ptr(bound), st), "edg_assemble_count")
    offsets = torch.empty(n + 1, dtype=torch.int64, device=dev)
    scratch = torch.empty(lib.edg_scan_scratch_elems(n), dtype=torch.int64, device=dev)
    check(lib.edg_scan_i64(ptr(bound), ptr(offsets), n, ptr(scratch), st), "edg_scan_i64")
    total = int(offsets[n].item())
    tmp_cols = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
    tmp_vals = torch.empty(max(total, 1) * w, dtype=torch.float64, device=dev)
    row_nnz = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    diag = torch.empty(max(n, 1) * w, dtype=torch.float64, device=dev)
    present = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    check(lib.edg_assemble_fill(ctypes.byref(a), ptr(offsets), ptr(tmp_cols), ptr(tmp_vals), ptr(row_nnz),
                                ptr(diag), ptr(present), ptr(err), st), "edg_assemble_fill")
    rowptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
    check(lib.edg_scan_i64(ptr(row_nnz), ptr(rowptr), n, ptr(scratch), st), "edg_scan_i64")
    nnz = int(rowptr[n].item())
    e = int(err.item())
    if e != 0:
        raise _lib.EdgError(e, "an operator maps a sector configuration outside the sector")
    cols = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    vals = torch.empty(max(nnz, 1) * w, dtype=torch.float64, device=dev)
    check(lib.edg_assemble_compact(n, 1 if is_complex else 0, ptr(offsets), ptr(tmp_cols), ptr(tmp_vals),
                                   ptr(rowptr), ptr(cols), ptr(vals), st), "edg_assemble_compact")
    del tmp_cols, tmp_vals
    return {"rowptr": rowptr, "cols": cols[:nnz], "vals": vals[: nnz * w], "diag": diag[: n * w],
            "present": present[:n], "raw_entries": total, "keep": tabs}
