"""Python side of the multithreaded C port (edlgt_port.c) -- TEST AND CPU-BASELINE
INFRASTRUCTURE ONLY.

``assemble_port`` builds the reference's triplets term instance by term
instance (two-pass count/fill, h.c. by transposition, diagonal terms with the
1e-10 cut) and sums them into the canonical CSR as SciPy does;
``lowest_eigs_port`` runs scipy's ARPACK eigsh on a LinearOperator whose
matvec is the row-parallel complex128 CSR product -- the reference's
``"linear"`` Hamiltonian format (edlgt/modeling/qmb_hamiltonian.py:186-193,
705-730).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.linalg import LinearOperator, eigsh

from .build_port import OUT, build_port

OP_TOL = 1e-10

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_port() if not OUT.exists() else OUT
        h = C.CDLL(str(path))
        P, I64, I32 = C.c_void_p, C.c_int64, C.c_int
        h.port_nbody_count.restype = I64
        h.port_nbody_count.argtypes = [P, I64, P, P, I32, P, P, I32, P]
        h.port_nbody_fill.restype = None
        h.port_nbody_fill.argtypes = [P, I64, P, P, I32, P, P, P, P, I32, P, P, P, P]
        h.port_local_diag.restype = I64
        h.port_local_diag.argtypes = [P, I64, P, P, I32, P, P, P]
        h.port_csr_spmv.restype = None
        h.port_csr_spmv.argtypes = [I64, P, P, P, P, P]
        h.port_csr_spmv_real.restype = None
        h.port_csr_spmv_real.argtypes = [I64, P, P, P, P, P]
        _lib = h
    return _lib


def threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def _p(a):
    return a.ctypes.data


def _strides(loc_dims):
    s = np.ones(len(loc_dims), dtype=np.uint64)
    for k in range(len(loc_dims) - 2, -1, -1):
        s[k] = s[k + 1] * np.uint64(loc_dims[k + 1])
    return s


def assemble_port(blocks, keys, loc_dims):
    """Canonical complex CSR of the sum of term blocks (C port of the builders)."""
    h = lib()
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    n = len(keys)
    ld = np.ascontiguousarray(loc_dims, dtype=np.int32)
    st = _strides(ld)
    R, Cc, V = [], [], []
    for b in blocks:
        dmax = b.ops[0].shape[-1]
        rr, cc, vv = [], [], []
        for inst in np.asarray(b.sites, dtype=np.int64).reshape(-1, len(b.ops)):
            if b.diagonal:
                diag = np.ascontiguousarray(np.diagonal(np.asarray(b.ops[0][inst[0]], dtype=np.complex128)))
                rows = np.empty(n, dtype=np.int32)
                vals = np.empty(n, dtype=np.complex128)
                m = h.port_local_diag(_p(keys), n, _p(st), _p(ld), int(inst[0]), _p(diag), _p(rows), _p(vals))
                rr.append(rows[:m])
                cc.append(rows[:m])
                vv.append(vals[:m])
                continue
            nops = len(inst)
            counts = np.zeros((nops, dmax), dtype=np.int32)
            kets = np.zeros((nops, dmax, dmax), dtype=np.int32)
            amps = np.zeros((nops, dmax, dmax), dtype=np.complex128)
            for j, s in enumerate(inst):
                op = np.asarray(b.ops[j][int(s)], dtype=np.complex128)
                for bra in range(dmax):
                    nz = np.nonzero(np.abs(op[bra]) > OP_TOL)[0]
                    counts[j, bra] = len(nz)
                    kets[j, bra, : len(nz)] = nz
                    amps[j, bra, : len(nz)] = op[bra, nz]
            sites = np.ascontiguousarray(inst, dtype=np.int32)
            row_nnz = np.empty(n, dtype=np.int64)
            total = h.port_nbody_count(_p(keys), n, _p(st), _p(ld), nops, _p(sites), _p(counts), dmax, _p(row_nnz))
            offsets = np.zeros(n, dtype=np.int64)
            np.cumsum(row_nnz[:-1], out=offsets[1:])
            rows = np.empty(total, dtype=np.int32)
            cols = np.empty(total, dtype=np.int32)
            vals = np.empty(total, dtype=np.complex128)
            h.port_nbody_fill(_p(keys), n, _p(st), _p(ld), nops, _p(sites), _p(counts), _p(kets), _p(amps), dmax,
                              _p(offsets), _p(rows), _p(cols), _p(vals))
            rr.append(rows)
            cc.append(cols)
            vv.append(vals)
        if not rr:
            continue
        r = np.concatenate(rr)
        c = np.concatenate(cc)
        v = np.concatenate(vv) * complex(b.strength)
        R.append(r)
        Cc.append(c)
        V.append(v)
        if b.add_dagger:
            R.append(c)
            Cc.append(r)
            V.append(np.conj(v))
    r = np.concatenate(R)
    c = np.concatenate(Cc)
    if np.any(c < 0):
        raise ValueError("a ket is outside the sector")
    m = coo_matrix((np.concatenate(V), (r, c)), shape=(n, n)).tocsr()
    m.sum_duplicates()
    return m


def lowest_eigs_port(H, k=1):
    """eigsh(k, "SA") with the multithreaded complex128 CSR matvec."""
    h = lib()
    n = H.shape[0]
    indptr = np.ascontiguousarray(H.indptr, dtype=np.int64)
    indices = np.ascontiguousarray(H.indices, dtype=np.int32)
    data = np.ascontiguousarray(H.data, dtype=np.complex128)

    def mv(x):
        x = np.ascontiguousarray(np.ravel(x), dtype=np.complex128)
        y = np.empty(n, dtype=np.complex128)
        h.port_csr_spmv(n, _p(indptr), _p(indices), _p(data), _p(x), _p(y))
        return y

    op = LinearOperator((n, n), matvec=mv, dtype=np.complex128)
    w, v = eigsh(op, k=k, which="SA")
    o = np.argsort(w)
    return w[o], v[:, o]
