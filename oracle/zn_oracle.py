"""CPU oracle for the Z_n lattice gauge theory with staggered fermions
(periodic Lx x Ly), TEST INFRASTRUCTURE ONLY: imported by tests/ and by the
golden-fixture scripts, never by the library.

The reference has no Z_n model with matter for odd n
(edlgt/operators/Zn_operators.py:153-157 raises), so this oracle restates the
model's conventions on its own, in plain numpy, with none of the device
engine's tricks (no cotree ranking, no orbit table, no bit rotations):

* basis: every (occupations, link fields) satisfying the Gauss law
  E_(s,x) + E_(s,y) - E_(s-x,x) - E_(s-y,y) = n_s - [x_s odd] (mod n) with
  sum_s n_s = #odd-x sites, enumerated level by level over the links with the
  Gauss check of a site applied once its four links are set (the prefix
  expansion of edlgt/symmetries/symmetry_sector.py:785-967), sorted by the
  packed key (link l's field at bits [b l, b (l+1)), occupation of site s at
  bit 2 b N + s, b = 1 for n = 2 else 2);
* terms are applied to every basis state and the image located by a sorted
  key search, as edlgt/symmetries/sym_qmb_operations.py:297-396 does per row:
  hopping -t eta_l (c^dag_s U_l c_s' + h.c.) with Jordan-Wigner sign over the
  occupied sites strictly between s and s' (linear order s = x + Lx y),
  eta_x = 1, eta_y = (-1)^x; mass m (-1)^x n_s; (g^2/2) E^2 on the symmetric
  representative; -1/(2 g^2) (U_p + U_p^dag);
* zero momentum (edlgt/symmetries/translational_sym.py:567-819 builds the
  same projector from a translation table): translations (a even, b) act as
  explicit site permutations, the fermionic sign is the parity of the
  inversions the permutation makes among occupied sites; the representative
  of an orbit is its smallest key; the projector column of representative r
  is sum_g sign_g T_g |r> / sqrt(|G| |Stab r|); orbits with a -1 stabiliser
  sign are dropped.
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix, csr_matrix
from scipy.sparse.linalg import eigsh

__all__ = ["ZnOracle"]


class ZnOracle:
    def __init__(self, lx, ly, n, momentum=True):
        self.lx, self.ly, self.n = lx, ly, n
        self.N = N = lx * ly
        self.L = 2 * N
        self.b = 1 if n == 2 else 2
        self.momentum = momentum
        self.xs = np.array([s % lx for s in range(N)])
        self.ys = np.array([s // lx for s in range(N)])
        self.offset = (self.xs % 2).astype(np.int64)  # static charge offset [x odd]
        self.n_f = int(self.offset.sum())
        self.tail = np.repeat(np.arange(N), 2)
        self.head = np.array([self._site(self.xs[s] + (1 - mu), self.ys[s] + mu) for s in range(N) for mu in (0, 1)])
        self._enumerate()

    def _site(self, x, y):
        return int(x % self.lx + self.lx * (y % self.ly))

    # ------------------------------------------------------------ basis
    def _enumerate(self):
        N, L, n = self.N, self.L, self.n
        # links touching each site with their sign in the divergence
        touch = [[] for _ in range(N)]
        for l in range(L):
            touch[self.tail[l]].append((l, 1))
            touch[self.head[l]].append((l, -1))
        close_at = {}
        for v in range(N):
            close_at.setdefault(max(l for l, _ in touch[v]), []).append(v)
        occs, Es = [], []
        from itertools import combinations

        for occ_sites in combinations(range(N), self.n_f):
            occ = np.zeros(N, dtype=np.int64)
            occ[list(occ_sites)] = 1
            q = occ - self.offset
            E = np.zeros((1, 0), dtype=np.int64)
            for l in range(L):
                E = np.concatenate([np.repeat(E, n, axis=0), np.tile(np.arange(n), len(E))[:, None]], axis=1)
                for v in close_at.get(l, []):
                    div = sum(sg * E[:, ll] for ll, sg in touch[v])
                    E = E[(div - q[v]) % n == 0]
            occs.append(np.repeat(occ[None, :], len(E), axis=0))
            Es.append(E)
        occ = np.concatenate(occs)
        E = np.concatenate(Es)
        keys = self.pack(occ, E)
        order = np.argsort(keys)
        self.occ, self.E, self.keys = occ[order], E[order], keys[order]
        self.dim = len(self.keys)

    def pack(self, occ, E):
        k = np.zeros(len(occ), dtype=np.uint64)
        for l in range(self.L):
            k |= E[:, l].astype(np.uint64) << np.uint64(self.b * l)
        for s in range(self.N):
            k |= occ[:, s].astype(np.uint64) << np.uint64(self.b * self.L + s)
        return k

    def index(self, keys):
        i = np.searchsorted(self.keys, keys)
        i = np.minimum(i, self.dim - 1)
        if not np.all(self.keys[i] == keys):
            raise AssertionError("image outside the Gauss-law sector")
        return i

    # ------------------------------------------------------------ terms
    def components(self):
        """Sparse matrices (hop, mass, esq, plaq) with H = t hop + m mass +
        (g^2/2) esq - 1/(2 g^2) plaq."""
        if hasattr(self, "_comp"):
            return self._comp
        S, N, n = self.dim, self.N, self.n
        rows, cols, vals = [], [], []
        occ, E = self.occ, self.E
        cols_all = np.arange(S)
        for l in range(self.L):
            s, sp = int(self.tail[l]), int(self.head[l])
            mu = l % 2
            eta = 1 if mu == 0 else (1 if self.xs[s] % 2 == 0 else -1)
            lo, hi = min(s, sp), max(s, sp)
            between = occ[:, lo + 1:hi].sum(axis=1) if hi > lo + 1 else np.zeros(S, dtype=np.int64)
            jw = 1 - 2 * (between % 2)
            for fwd in (True, False):
                # forward: c^dag_s U_l c_s' ; backward: c^dag_s' U_l^dag c_s
                sel = (occ[:, s] == 0) & (occ[:, sp] == 1) if fwd else (occ[:, s] == 1) & (occ[:, sp] == 0)
                o2 = occ[sel].copy()
                e2 = E[sel].copy()
                o2[:, s] ^= 1
                o2[:, sp] ^= 1
                e2[:, l] = (e2[:, l] + (1 if fwd else -1)) % n
                rows.append(self.index(self.pack(o2, e2)))
                cols.append(cols_all[sel])
                vals.append(-eta * jw[sel].astype(float))
        hop = self._mat(rows, cols, vals)
        rows, cols, vals = [], [], []
        for s in range(N):
            x, y = self.xs[s], self.ys[s]
            sx, sy = self._site(x + 1, y), self._site(x, y + 1)
            links = (2 * s, 2 * sx + 1, 2 * sy, 2 * s + 1)
            for dirn in (1, -1):
                e2 = E.copy()
                for k, l in enumerate(links):
                    e2[:, l] = (e2[:, l] + (dirn if k < 2 else -dirn)) % n
                rows.append(self.index(self.pack(occ, e2)))
                cols.append(cols_all)
                vals.append(np.ones(S))
        plaq = self._mat(rows, cols, vals)
        sym = np.where(np.arange(n) > n // 2, np.arange(n) - n, np.arange(n))
        esq = (sym[E] ** 2).sum(axis=1).astype(float)
        eta_s = np.where(self.xs % 2 == 0, 1.0, -1.0)
        mass = (occ * eta_s[None, :]).sum(axis=1)
        self._comp = {
            "hop": hop,
            "mass": csr_matrix((mass, (cols_all, cols_all)), shape=(S, S)),
            "esq": csr_matrix((esq, (cols_all, cols_all)), shape=(S, S)),
            "plaq": plaq,
        }
        return self._comp

    def _mat(self, rows, cols, vals):
        S = self.dim
        m = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(S, S))
        return m.tocsr()

    def hamiltonian(self, t, m, g, momentum=None):
        c = self.components()
        H = t * c["hop"] + m * c["mass"] + (g * g / 2) * c["esq"] - (1.0 / (2 * g * g)) * c["plaq"]
        use_k = self.momentum if momentum is None else momentum
        if use_k:
            B = self.momentum_basis()[0]
            H = (B.T @ H @ B).tocsr()
        return H

    # ------------------------------------------------------------ momentum
    def group(self):
        return [(a, b) for b in range(self.ly) for a in range(0, self.lx, 2)] if self.momentum else [(0, 0)]

    def translate(self, a, b, occ, E):
        """Images of all states under (x, y) -> (x + a, y + b) and their signs."""
        N = self.N
        p = np.array([self._site(self.xs[s] + a, self.ys[s] + b) for s in range(N)])
        o2 = np.zeros_like(occ)
        o2[:, p] = occ
        e2 = np.zeros_like(E)
        for s in range(N):
            for mu in (0, 1):
                e2[:, 2 * p[s] + mu] = E[:, 2 * s + mu]
        inv = np.zeros(len(occ), dtype=np.int64)
        for s in range(N):
            for sp in range(s + 1, N):
                if p[s] > p[sp]:
                    inv += occ[:, s] * occ[:, sp]
        return o2, e2, 1 - 2 * (inv % 2)

    def momentum_basis(self):
        """(B, rep_keys, stab): B is dim x n_reps with orthonormal columns."""
        if hasattr(self, "_mb"):
            return self._mb
        G = self.group()
        S = self.dim
        img = np.zeros((len(G), S), dtype=np.int64)
        sgn = np.zeros((len(G), S), dtype=np.int64)
        for k, (a, b) in enumerate(G):
            o2, e2, sg = self.translate(a, b, self.occ, self.E)
            img[k] = self.index(self.pack(o2, e2))
            sgn[k] = sg
        # orbits: smallest key = smallest index (keys are sorted)
        rep = img.min(axis=0)
        is_rep = rep == np.arange(S)
        stab = (img == np.arange(S)[None, :]).sum(axis=0)
        bad = ((img == np.arange(S)[None, :]) & (sgn < 0)).any(axis=0)
        reps = np.nonzero(is_rep & ~bad)[0]
        col_of = np.full(S, -1)
        col_of[reps] = np.arange(len(reps))
        rows, cols, vals = [], [], []
        for k in range(len(G)):
            rows.append(img[k, reps])
            cols.append(col_of[reps])
            vals.append(sgn[k, reps] / np.sqrt(len(G) * stab[reps]))
        B = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(S, len(reps))).tocsr()
        self._mb = (B, self.keys[reps], stab[reps])
        return self._mb

    # ------------------------------------------------------------ spectra
    def lowest(self, t, m, g, k=1, momentum=None):
        H = self.hamiltonian(t, m, g, momentum)
        if H.shape[0] <= 2000:
            return np.linalg.eigvalsh(H.toarray())[:k]
        return np.sort(eigsh(H, k=k, which="SA", tol=0, return_eigenvectors=False))
