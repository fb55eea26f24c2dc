"""Golden fixture for the Z_n model with matter, made by ed-lgt's own
model-agnostic kernels.

ed-lgt has no Z_n model with matter for odd n, but its sector builder
(symmetry_sector_configs, edlgt/symmetries/symmetry_sector.py:68-145) and its
n-body term builder (nbody_term, edlgt/symmetries/sym_qmb_operations.py:167-294)
work on any dressed-site operator tables.  This script builds those tables
for the Z_n conventions of the engine (periodic Lx x Ly, staggering (-1)^x,
Kogut-Susskind phases, Jordan-Wigner order by linear site index) as dressed
sites (occupation, E_mx, E_my, E_px, E_py) with the Gauss law applied per
site and the two ends of a link tied by link constraints, and records what
the reference computes from them in the full Gauss-law sector: the sector
dimension, tr H, ||H||_F^2 and the lowest eigenvalues (eigsh, tol=0).
These are basis independent, so the tests compare them with the oracle's
own construction (oracle/zn_oracle.py).

    python tests/golden/make_zn_golden.py      # writes zn_cases.npz here
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402,F401

import logging  # noqa: E402

logging.disable(logging.INFO)

from scipy.sparse import coo_matrix  # noqa: E402
from scipy.sparse.linalg import eigsh  # noqa: E402

from edlgt.symmetries.sym_qmb_operations import nbody_term  # noqa: E402
from edlgt.symmetries.symmetry_sector import symmetry_sector_configs  # noqa: E402

CASES = [(2, 2, 3), (2, 3, 3), (2, 2, 2), (2, 3, 2), (2, 2, 4)]
COUPLINGS = [(1.0, 0.5, 1.0), (1.0, 0.0, 0.7), (0.8, 1.2, 1.6)]
K = 3
MX, MY, PX, PY = 1, 2, 3, 4  # positions in the local state tuple (occ first)


def local_states(n, odd):
    out = []
    for occ in (0, 1):
        for emx in range(n):
            for emy in range(n):
                for epx in range(n):
                    for epy in range(n):
                        if (epx + epy - emx - emy - (occ - odd)) % n == 0:
                            out.append((occ, emx, emy, epx, epy))
    return out


class Lattice:
    def __init__(self, lx, ly, n):
        self.lx, self.ly, self.n = lx, ly, n
        self.N = lx * ly
        self.odd = [(s % lx) % 2 for s in range(self.N)]
        self.states = [local_states(n, self.odd[s]) for s in range(self.N)]
        self.index = [{st: i for i, st in enumerate(sts)} for sts in self.states]
        self.d = len(self.states[0])

    def site(self, x, y):
        return x % self.lx + self.lx * (y % self.ly)

    def op(self, fn):
        """(n_sites, d, d) table of a local map state -> (state', amp) or None."""
        A = np.zeros((self.N, self.d, self.d), dtype=np.complex128)
        for s in range(self.N):
            for j, st in enumerate(self.states[s]):
                r = fn(list(st))
                if r is not None:
                    st2, amp = r
                    A[s, self.index[s][tuple(st2)], j] += amp
        return A


def shift(pos, delta, n):
    def f(st):
        st[pos] = (st[pos] + delta) % n
        return st, 1.0

    return f


def compose(*fns):
    """Local operator product, rightmost applied first."""
    def f(st):
        amp = 1.0
        for g in reversed(fns):
            r = g(st)
            if r is None:
                return None
            st, a = r
            amp *= a
        return st, amp

    return f


def cdag(st):
    if st[0] == 1:
        return None
    st[0] = 1
    return st, 1.0


def c(st):
    if st[0] == 0:
        return None
    st[0] = 0
    return st, 1.0


def parity(st):
    return st, -1.0 if st[0] else 1.0


def build_case(lx, ly, n):
    lat = Lattice(lx, ly, n)
    N, d = lat.N, lat.d
    sym = np.where(np.arange(n) > n // 2, np.arange(n) - n, np.arange(n))
    esq = (sym**2).astype(float)
    occ_op = lat.op(lambda st: (st, float(st[0])))
    glob = np.real(np.stack([np.diagonal(occ_op[s]) for s in range(N)]))[None]
    link_diags = np.zeros((2, 2, N, d))
    pairs = [[], []]
    for s in range(N):
        x, y = s % lx, s // lx
        for mu, (dx, dy) in enumerate(((1, 0), (0, 1))):
            pairs[mu].append((s, lat.site(x + dx, y + dy)))
    for s in range(N):
        for j, st in enumerate(lat.states[s]):
            link_diags[0, 0, s, j] = st[PX]
            link_diags[0, 1, s, j] = -st[MX]
            link_diags[1, 0, s, j] = st[PY]
            link_diags[1, 1, s, j] = -st[MY]
    pair_list = [np.array(p, dtype=np.int32) for p in pairs]
    n_f = sum(lat.odd)
    configs = symmetry_sector_configs(np.full(N, d, dtype=np.int32), glob, np.array([float(n_f)]), "U",
                                      link_diags, np.zeros(2), pair_list)
    # term blocks: (list of (site, local op), kind) with kind in hop / plaq / diag parts
    blocks = {"hop": [], "plaq": [], "esq": [], "mass": []}
    for s in range(N):
        x, y = s % lx, s // lx
        for mu, (dx, dy) in enumerate(((1, 0), (0, 1))):
            sp = lat.site(x + dx, y + dy)
            eta = 1.0 if mu == 0 else (1.0 if x % 2 == 0 else -1.0)
            lo, hi = min(s, sp), max(s, sp)
            between = [(k, lat.op(parity)) for k in range(lo + 1, hi)]
            pe, me = (PX, MX) if mu == 0 else (PY, MY)
            fwd = [(s, lat.op(compose(cdag, shift(pe, 1, n)))), (sp, lat.op(compose(c, shift(me, 1, n))))]
            bwd = [(s, lat.op(compose(c, shift(pe, -1, n)))), (sp, lat.op(compose(cdag, shift(me, -1, n))))]
            blocks["hop"].append((fwd + between, -eta))
            blocks["hop"].append((bwd + between, -eta))
        sx, sy, sxy = lat.site(x + 1, y), lat.site(x, y + 1), lat.site(x + 1, y + 1)
        for dirn in (1, -1):
            blocks["plaq"].append(([
                (s, lat.op(compose(shift(PX, dirn, n), shift(PY, -dirn, n)))),
                (sx, lat.op(compose(shift(MX, dirn, n), shift(PY, dirn, n)))),
                (sxy, lat.op(compose(shift(MY, dirn, n), shift(MX, -dirn, n)))),
                (sy, lat.op(compose(shift(PX, -dirn, n), shift(MY, -dirn, n)))),
            ], 1.0))
        blocks["esq"].append(([(s, lat.op(lambda st: (st, esq[st[PX]] + esq[st[PY]])))], 1.0))
        blocks["mass"].append(([(s, lat.op(lambda st: (st, float(st[0]))))], 1.0 if x % 2 == 0 else -1.0))
    D = len(configs)
    mats = {}
    for name, terms in blocks.items():
        rows, cols, vals = [], [], []
        for ops, coef in terms:
            sites = np.array([s for s, _ in ops], dtype=np.int32)
            op_list = np.stack([A for _, A in ops])
            r, cc, v = nbody_term(op_list, sites, configs)
            rows.append(np.asarray(r))
            cols.append(np.asarray(cc))
            vals.append(coef * np.real(np.asarray(v)))
        mats[name] = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                                shape=(D, D)).tocsr()
    return D, mats


def main():
    out = {}
    for lx, ly, n in CASES:
        t0 = time.time()
        D, mats = build_case(lx, ly, n)
        tag = f"{lx}x{ly}_z{n}"
        out[f"{tag}_dim"] = np.array(D)
        energies, traces, fro = [], [], []
        for t, m, g in COUPLINGS:
            H = t * mats["hop"] + m * mats["mass"] + (g * g / 2) * mats["esq"] - (1 / (2 * g * g)) * mats["plaq"]
            traces.append(H.diagonal().sum())
            fro.append((abs(H).power(2)).sum())
            if D <= 3000:
                e = np.linalg.eigvalsh(H.toarray())[:K]
            else:
                e = np.sort(eigsh(H, k=K, which="SA", tol=0, return_eigenvectors=False))
            energies.append(e)
        out[f"{tag}_energies"] = np.array(energies)
        out[f"{tag}_trace"] = np.array(traces)
        out[f"{tag}_fro2"] = np.array(fro)
        print(tag, D, np.array(energies)[:, 0], f"{time.time() - t0:.1f}s", flush=True)
    out["couplings"] = np.array(COUPLINGS)
    np.savez(os.path.join(HERE, "zn_cases.npz"), **out)


if __name__ == "__main__":
    main()
