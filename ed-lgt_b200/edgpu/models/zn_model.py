"""Z_n lattice gauge theory with staggered fermions on a periodic Lx x Ly
lattice, in the Gauss-law, zero-charge and (optionally) zero-momentum
sector, solved matrix-free on the device.

ed-lgt has Z_n dressed-site operators only for even n with matter
(edlgt/operators/Zn_operators.py:130-201: the fermionic rishons need a Z_2
grading, and :153-157 raises for odd n) and no Z_n model class, so this model
fixes its own conventions:

* degrees of freedom: a fermion occupation n_s in {0, 1} per site and a link
  field E_l in Z_n = {0..n-1} per link l = 2 s + mu (mu = 0: x, 1: y), the
  link from s to s + mu (periodic);
* staggering eta_s = (-1)^x (along x only: Ly may be odd, and a checkerboard
  is not consistent with periodic Ly odd); static charge q_s = n_s - [x odd];
* Gauss law  E_(s,x) + E_(s,y) - E_(s-x,x) - E_(s-y,y) = q_s  (mod n);
  total charge zero, i.e. sum_s n_s = number of odd-x sites;
* H = -t sum_l eta_l (c^dag_s U_l c_(s+mu) + h.c.) + m sum_s eta_s n_s
      + (g^2/2) sum_l E_l^2 - 1/(2 g^2) sum_p (U_p + U_p^dag),
  U_l: E_l -> E_l + 1 (mod n), E^2 taken on the symmetric representative
  E in (-n/2, n/2], Kogut-Susskind phases eta_x = 1, eta_y(s) = (-1)^x_s,
  U_p = U_(s,x) U_(s+x,y) U^dag_(s+y,x) U^dag_(s,y);
* fermions are ordered by the linear site index s = x + Lx y (Jordan-Wigner),
  |n> = (c^dag_0)^n_0 (c^dag_1)^n_1 ... |0>;
* the translations that keep eta, (x, y) -> (x + a, y + b) with a even, act
  as T c^dag_s T^-1 = c^dag_T(s); the zero-momentum states are
  |R> = sum_g T_g |r> / sqrt(|G| |Stab r|), r the representative of the orbit
  (smallest packed key), and orbits whose stabiliser contains a T_g with
  T_g |r> = -|r> have no zero-momentum state.

Packed configuration (64-bit key): link l's field at bits
[link_bits * l, link_bits * (l + 1)), i.e. site s owns 2 * link_bits bits
starting at 2 * link_bits * s (x link first); occupations at bit
field_bits + s.  A row of sites is one lane of Lx * 2 * link_bits bits, so a
translation is a rotation of the lane array plus a rotation inside every lane.

Dense Gauss index.  A spanning tree of the torus graph leaves
n_cot = links - sites + 1 cotree links; given the occupations, the cotree
fields are free and the tree fields follow from the Gauss law.  So
    gidx = colex_rank(occupied sites) * n^n_cot + sum_c E_(cot c) n^c
enumerates the Gauss-law sector densely; the device decodes it by peeling the
tree from the leaves and encodes it with two small lookup tables.
"""

from __future__ import annotations

from math import comb

import numpy as np

__all__ = ["ZnLattice", "ZnModel"]

_MAX_SITES = 14
_MAX_GROUP = 32


class ZnLattice:
    """Geometry, sector ranking and packed-key layout of a Z_n lattice."""

    def __init__(self, lvals=(4, 3), n=3, momentum=True):
        lx, ly = int(lvals[0]), int(lvals[1])
        if lx < 2 or ly < 2 or lx % 2:
            raise ValueError("need Lx even >= 2 and Ly >= 2 (periodic, x-staggered)")
        if n not in (2, 3, 4):
            raise ValueError("n must be 2, 3 or 4")
        N = lx * ly
        if N > _MAX_SITES:
            raise ValueError(f"at most {_MAX_SITES} sites")
        self.lx, self.ly, self.n = lx, ly, n
        self.n_sites = N
        self.n_links = 2 * N
        self.link_bits = 1 if n == 2 else 2
        self.field_bits = self.link_bits * self.n_links
        if self.field_bits + N > 64:
            raise ValueError("packed key does not fit 64 bits")
        self.momentum = bool(momentum)
        self.link_from = np.repeat(np.arange(N), 2)
        self.link_to = np.array([self.site(self.xy(s)[0] + (1 - mu), self.xy(s)[1] + mu)
                                 for s in range(N) for mu in (0, 1)])
        self.eta = np.array([1 if self.xy(s)[0] % 2 == 0 else -1 for s in range(N)])
        self.odd_mask = sum(1 << s for s in range(N) if self.eta[s] < 0)
        self.n_fermions = bin(self.odd_mask).count("1")
        self._build_tree()
        self.n_cot = len(self.cotree)
        self.pow_cot = n**self.n_cot
        self.n_matter = comb(N, self.n_fermions)
        self.n_gauss = self.n_matter * self.pow_cot
        if momentum:
            self.group = [(a, b) for b in range(ly) for a in range(0, lx, 2)]
        else:
            self.group = [(0, 0)]
        if len(self.group) > _MAX_GROUP:
            raise ValueError("translation group too large")
        self.plaquettes = []
        for s in range(N):
            x, y = self.xy(s)
            sx, sy = self.site(x + 1, y), self.site(x, y + 1)
            # raised, raised, lowered, lowered
            self.plaquettes.append((2 * s + 0, 2 * sx + 1, 2 * sy + 0, 2 * s + 1))
        self.plaquettes = np.array(self.plaquettes, dtype=np.int64)

    # ------------------------------------------------------------ geometry
    def xy(self, s):
        return s % self.lx, s // self.lx

    def site(self, x, y):
        return (x % self.lx) + self.lx * (y % self.ly)

    def link_eta(self, l):
        """Kogut-Susskind phase of link l: 1 along x, (-1)^x along y."""
        s, mu = divmod(int(l), 2)
        return 1 if mu == 0 else (1 if self.xy(s)[0] % 2 == 0 else -1)

    def _build_tree(self):
        N = self.n_sites
        adj = [[] for _ in range(N)]
        for l in range(self.n_links):
            a, b = int(self.link_from[l]), int(self.link_to[l])
            adj[a].append(l)
            adj[b].append(l)
        self.incident = adj
        parent_link = [-1] * N
        order = [0]
        seen = [False] * N
        seen[0] = True
        for u in order:
            for l in adj[u]:
                v = int(self.link_to[l]) if int(self.link_from[l]) == u else int(self.link_from[l])
                if not seen[v]:
                    seen[v] = True
                    parent_link[v] = l
                    order.append(v)
        tree = set(parent_link[v] for v in range(1, N))
        self.cotree = [l for l in range(self.n_links) if l not in tree]
        # Peeling order: children before parents (reverse BFS); at child v
        # every incident link except its parent link is known by then.
        self.peel = []
        for v in reversed(order[1:]):
            pl = parent_link[v]
            others = [l for l in adj[v] if l != pl]
            self.peel.append((v, pl, self._sign_at(pl, v), [(l, self._sign_at(l, v)) for l in others]))

    def _sign_at(self, l, v):
        """Coefficient of E_l in the divergence at site v (+1 tail, -1 head)."""
        return 1 if int(self.link_from[l]) == v else -1

    # ------------------------------------------------------------ packing
    def pack(self, occ, E):
        key = 0
        for l in range(self.n_links):
            key |= int(E[l]) << (self.link_bits * l)
        for s in range(self.n_sites):
            key |= int(occ[s]) << (self.field_bits + s)
        return key

    def unpack(self, key):
        key = int(key)
        m = (1 << self.link_bits) - 1
        E = np.array([(key >> (self.link_bits * l)) & m for l in range(self.n_links)], dtype=np.int64)
        occ = np.array([(key >> (self.field_bits + s)) & 1 for s in range(self.n_sites)], dtype=np.int64)
        return occ, E

    def unpack_many(self, keys):
        keys = np.asarray(keys, dtype=np.uint64)
        m = np.uint64((1 << self.link_bits) - 1)
        E = np.stack([(keys >> np.uint64(self.link_bits * l)) & m for l in range(self.n_links)], axis=1)
        occ = np.stack([(keys >> np.uint64(self.field_bits + s)) & np.uint64(1) for s in range(self.n_sites)], axis=1)
        return occ.astype(np.int64), E.astype(np.int64)

    # ------------------------------------------------------------ ranking
    def matter_rank(self, occ_bits):
        r, i = 0, 0
        for p in range(self.n_sites):
            if (occ_bits >> p) & 1:
                i += 1
                r += comb(p, i)
        return r

    def gauss_index(self, key):
        occ = int(key) >> self.field_bits
        m = (1 << self.link_bits) - 1
        g = 0
        for c, l in enumerate(self.cotree):
            g += ((int(key) >> (self.link_bits * l)) & m) * self.n**c
        return self.matter_rank(occ) * self.pow_cot + g

    # ------------------------------------------------------ device tables
    def lookup_tables(self):
        """(chunk_lut uint64 [n_chunks, 256], occ_rank uint32 [2^N],
        rank_occ uint32 [n_matter])."""
        N, b = self.n_sites, self.link_bits
        n_chunks = (self.field_bits + 7) // 8
        chunk = np.zeros((n_chunks, 256), dtype=np.uint64)
        m = (1 << b) - 1
        for c, l in enumerate(self.cotree):
            off = b * l
            k, sh = divmod(off, 8)
            v = np.arange(256, dtype=np.uint64)
            chunk[k] += ((v >> np.uint64(sh)) & np.uint64(m)) * np.uint64(self.n**c)
        occ_rank = np.full(1 << N, 0xFFFFFFFF, dtype=np.uint32)
        rank_occ = np.zeros(self.n_matter, dtype=np.uint32)
        for bits in range(1 << N):
            if bin(bits).count("1") == self.n_fermions:
                r = self.matter_rank(bits)
                occ_rank[bits] = r
                rank_occ[r] = bits
        return chunk, occ_rank, rank_occ

    def translation_masks(self, a, by):
        """Shifts and masks of the translation (x, y) -> (x + a, y + by)."""
        N, lx, ly, b = self.n_sites, self.lx, self.ly, self.link_bits
        R = 2 * b * lx
        F = self.field_bits

        def lane_masks(width, lanes, s):
            hi = lo = 0
            for k in range(lanes):
                for bit in range(width):
                    if bit >= s:
                        hi |= 1 << (k * width + bit)
                    else:
                        lo |= 1 << (k * width + bit)
            return hi, lo

        hif, lof = lane_masks(R, ly, 2 * b * a)
        him, lom = lane_masks(lx, ly, a)
        rows_low = sum(1 << s for s in range(N) if self.xy(s)[1] < ly - by)
        head = sum(1 << x for x in range(lx - a))  # row-0 sites that move right
        return dict(sf=by * R, sx=2 * b * a, hif=hif, lof=lof, sm=by * lx, smx=a, him=him, lom=lom,
                    ylow=rows_low, yhigh=((1 << N) - 1) & ~rows_low, xhead=head,
                    xtail=((1 << lx) - 1) & ~head, F=F)

    def divisors(self):
        G = len(self.group)
        return [d for d in range(1, G + 1) if G % d == 0]


class ZnModel:
    """Host driver of the matrix-free Z_n engine (basis, orbit table, matvec
    and batched Lanczos), in the shape of ed-lgt's model API:
    ``ZnModel(lvals, n)`` then ``build_Hamiltonian(g, m)`` and
    ``diagonalize_Hamiltonian(n_eigs)`` (edlgt/models/quantum_model.py:606-611
    for the call shape)."""

    def __init__(self, lvals=(4, 3), n=3, momentum=True, t=1.0, device="cuda"):
        from ..zn import ZnEngine

        self.lattice = ZnLattice(lvals, n, momentum)
        self.t = float(t)
        self.engine = ZnEngine(self.lattice, device=device)
        self.engine.build_basis()
        self.sector_dim = self.engine.n_rows
        self.couplings = None

    def build_Hamiltonian(self, g, m):
        """One instance per (g, m) pair; g is the coupling g (E^2 weight
        g^2/2, plaquette weight 1/(2 g^2))."""
        g = np.atleast_1d(np.asarray(g, dtype=float))
        m = np.broadcast_to(np.atleast_1d(np.asarray(m, dtype=float)), g.shape)
        self.couplings = np.stack([np.full_like(g, self.t), m, g**2 / 2, -1.0 / (2 * g**2)], axis=1)
        return self.couplings

    def diagonalize_Hamiltonian(self, n_eigs=1, precision="mixed", **kw):
        from ..zn import zn_lowest

        if self.couplings is None:
            raise RuntimeError("call build_Hamiltonian first")
        self.res = zn_lowest(self.engine, self.couplings, k=n_eigs, precision=precision, **kw)
        self.energies = self.res.evals
        self.Nenergies = self.res.evals / self.lattice.n_sites
        return self.res
