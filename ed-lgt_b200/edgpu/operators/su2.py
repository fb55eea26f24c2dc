"""SU(2) hard-core-gluon (j_max = 1/2) dressed-site operators and singlet bases.

The local space is ``[background] x matter(4) x rishons(3)^(2D)``; a rishon
carries ``j in {0, 1/2}`` (states ``|0>, |1/2,+1/2>, |1/2,-1/2>``), the
matter carries two coloured staggered fermions.  Gauge invariance at a site
means an SU(2) singlet of all its spins; singlets are built by sequential
Clebsch-Gordan coupling and grouped by their intermediate total spins, which
fixes the basis order and phases of ``edlgt/operators/SU2_singlets.py:188-447``
and ``edlgt/operators/SU2_operators.py:625-714``.  Operators follow
``edlgt/operators/SU2_operators.py:35-299`` and
``edlgt/operators/SU2_rishons.py:25-88``.

Clebsch-Gordan coefficients are computed here from the Racah formula in exact
rational arithmetic (Condon-Shortley phases); a coefficient is carried as a
sign times the square root of a rational until the final product.
"""

from __future__ import annotations

from decimal import Decimal, getcontext
from fractions import Fraction
from functools import lru_cache
from itertools import product
from math import factorial

import numpy as np
from scipy.sparse import block_diag, csr_matrix, diags, identity, kron

from .common import border_classes, fermion_ops, kron_chain

__all__ = [
    "clebsch_gordan_sq",
    "su2_singlets",
    "su2_gauge_invariant_states",
    "su2_dressed_site_operators",
    "su2_gen_dressed_site_operators",
]

getcontext().prec = 50

# Spins are carried as twice their value (integers) throughout.


def clebsch_gordan_sq(j1, m1, j2, m2, J, M):
    """``(sign, CG^2)`` of <j1 m1; j2 m2 | J M> with all arguments doubled."""
    if m1 + m2 != M or abs(m1) > j1 or abs(m2) > j2 or abs(M) > J:
        return 0, Fraction(0)
    if not (abs(j1 - j2) <= J <= j1 + j2) or (j1 + j2 + J) % 2:
        return 0, Fraction(0)
    f = lambda x: factorial(x // 2)  # noqa: E731  (x is even here)
    pref = Fraction((J + 1) * f(J + j1 - j2) * f(J - j1 + j2) * f(j1 + j2 - J), f(j1 + j2 + J + 2))
    pref *= f(J + M) * f(J - M) * f(j1 - m1) * f(j1 + m1) * f(j2 - m2) * f(j2 + m2)
    total = Fraction(0)
    k = 0
    while True:
        args = [j1 + j2 - J - 2 * k, j1 - m1 - 2 * k, j2 + m2 - 2 * k, J - j2 + m1 + 2 * k, J - j1 - m2 + 2 * k]
        if min(args[:3]) < 0:
            break
        if min(args[3:]) >= 0:
            den = factorial(k)
            for a in args:
                den *= f(a)
            total += Fraction((-1) ** k, den)
        k += 1
    if total == 0:
        return 0, Fraction(0)
    return (1 if total > 0 else -1), pref * total * total


def _m_values(j2):
    """Magnetic numbers (doubled) in descending order."""
    return list(range(j2, -j2 - 1, -2))


def _couple(j1, j2, singlet_only, m1_fixed=None):
    """Nonzero couplings of (j1, m1) with j2; ordered m1, m2, J (as the reference)."""
    m1s = [m1_fixed] if m1_fixed is not None else _m_values(j1)
    Js = [0] if singlet_only else list(range(abs(j1 - j2), j1 + j2 + 1, 2))
    out = []
    for m1, m2, J in product(m1s, _m_values(j2), Js):
        M = m1 + m2
        if abs(M) > J:
            continue
        sgn, sq = clebsch_gordan_sq(j1, m1, j2, m2, J, M)
        if sgn != 0:
            out.append((m1, m2, sgn, sq, J, M))
    return out


def su2_singlets(spins2):
    """All singlets of the doubled spins ``spins2`` (sequential coupling).

    Returns a list of singlets, each a list of ``(m_tuple, sign, cg_sq)``;
    singlets are ordered by their tuple of intermediate total spins, and the
    components of one singlet keep the coupling enumeration order.
    """
    n = len(spins2)
    if n < 2:
        raise ValueError("a singlet needs at least two spins")
    # chain entries: (ms tuple, sign, sq, Jtots tuple, current J, current M)
    chains = []
    for m1, m2, sgn, sq, J, M in _couple(spins2[0], spins2[1], singlet_only=(n == 2)):
        chains.append(((m1, m2), sgn, sq, (J,), J, M))
    for k in range(2, n):
        last = k == n - 1
        nxt = []
        for ms, sgn, sq, jt, J, M in chains:
            for _, m2, s2, q2, J2, M2 in _couple(J, spins2[k], singlet_only=last, m1_fixed=M):
                nxt.append((ms + (m2,), sgn * s2, sq * q2, jt + (J2,), J2, M2))
        chains = nxt
    if not chains:
        return []
    chains = sorted(chains, key=lambda c: c[3])  # stable: grouping by intermediate spins
    groups, cur, key = [], [], None
    for c in chains:
        if key is not None and c[3] != key:
            groups.append(cur)
            cur = []
        key = c[3]
        cur.append((c[0], c[1], c[2]))
    groups.append(cur)
    return groups


def _cg_float(sign, sq):
    return float(sign * (Decimal(sq.numerator) / Decimal(sq.denominator)).sqrt())


def su2_gauge_invariant_states(spin, pure_theory, lattice_dim, background=0):
    basis, states = _su2_states_cached(float(spin), pure_theory, lattice_dim, float(background))
    return dict(basis), dict(states)


@lru_cache(maxsize=32)
def _su2_states_cached(spin, pure_theory, lattice_dim, background=0):
    """Singlet bases of a dressed site (``spin`` = 1/2 rishon truncation).

    Returns ``(gauge_basis, gauge_states)`` keyed by ``site`` and
    ``site_<border>``; each basis is a dense column matrix over the canonical
    product space ``[bg] x matter(V, +, -, P) x rishons``.
    """
    from ..lattice import border_labels

    s2 = int(round(2 * spin))
    D = lattice_dim
    rishon_js = list(range(0, s2 + 1))  # doubled j values 0..2s
    factors = [rishon_js for _ in range(2 * D)]
    if not pure_theory:
        factors.insert(0, [0, 1, 2])  # matter sectors: vacuum (j=0), single (1/2), pair (j=0)
    if background:
        factors.insert(0, list(range(0, int(round(2 * background)) + 1)))
    nbg = 1 if background else 0
    # Canonical product basis of each factor: list of (label, doubled m).
    def irreps(jmax2):
        out = []
        for j in range(0, jmax2 + 1):
            out += [(j, m) for m in _m_values(j)]
        return out

    canon = [irreps(s2) for _ in range(2 * D)]
    if not pure_theory:
        canon.insert(0, [("V", 0), (1, 1), (1, -1), ("P", 0)])
    if background:
        canon.insert(0, irreps(int(round(2 * background))))
    canon_index = {}
    for idx, cfg in enumerate(product(*canon)):
        canon_index[cfg] = idx
    full_dim = len(canon_index)
    states = {"site": []}
    cols = {"site": []}
    for b in border_labels(D):
        states[f"site_{b}"] = []
        cols[f"site_{b}"] = []
    for cfg in product(*factors):
        cfg = list(cfg)
        if not pure_theory:
            sector = cfg[nbg]
            spins2 = list(cfg)
            spins2[nbg] = 1 if sector == 1 else 0
            matter_label = {0: "V", 1: 1, 2: "P"}[sector]
        else:
            spins2 = list(cfg)
            matter_label = None
        total = sum(spins2)
        if total % 2 or max(spins2) > total - max(spins2):
            continue
        for singlet in su2_singlets(spins2):
            vec = np.zeros(full_dim)
            for ms, sgn, sq in singlet:
                key = []
                for pos, (j2, m2) in enumerate(zip(spins2, ms)):
                    if not pure_theory and pos == nbg:
                        key.append((matter_label, m2))
                    else:
                        key.append((j2, m2))
                vec[canon_index[tuple(key)]] = _cg_float(sgn, sq)
            if abs(np.sum(vec**2) - 1.0) > 1e-10:
                raise ValueError("singlet vector is not normalised")
            label = tuple(cfg)
            states["site"].append(label)
            cols["site"].append(vec)
            rishons = spins2[nbg + (0 if pure_theory else 1):]
            for b in border_classes(rishons, 0, D):
                states[f"site_{b}"].append(label)
                cols[f"site_{b}"].append(vec)
    basis = {k: csr_matrix(np.column_stack(v)) for k, v in cols.items() if v}
    return basis, {k: np.asarray(v) for k, v in states.items() if v}


def _rishon_ops_half():
    """Rishon operators for j_max = 1/2 (3 states: j=0, (1/2,+), (1/2,-))."""
    ops = {}
    ops["P"] = diags([1.0, -1.0, -1.0], 0, format="csr")
    ops["Iz"] = identity(3, format="csr")
    cf = 1.0 / (2 ** 0.25)
    ops["Zr"] = cf * csr_matrix(([1.0, 1.0], ([0, 2], [1, 0])), shape=(3, 3))
    ops["Zg"] = cf * csr_matrix(([1.0, -1.0], ([0, 1], [2, 0])), shape=(3, 3))
    for c in "rg":
        ops[f"Z{c}_dag"] = csr_matrix(ops[f"Z{c}"].T)
        ops[f"Z{c}_P"] = csr_matrix(ops[f"Z{c}"] @ ops["P"])
        ops[f"P_Z{c}_dag"] = csr_matrix(ops["P"] @ ops[f"Z{c}_dag"])
        ops[f"Z{c}_dag_P"] = csr_matrix(ops[f"Z{c}_dag"] @ ops["P"])
    return ops


def _spin_block(j2):
    """Sz, S+ and S^2 of one irrep (doubled j), m descending."""
    j = j2 / 2
    m = np.array(_m_values(j2), dtype=float) / 2
    sp = np.sqrt(j * (j + 1) - m[1:] * (m[1:] + 1))
    return (
        diags(m, 0, format="csr"),
        diags(sp, 1, shape=(j2 + 1, j2 + 1), format="csr"),
        diags([j * (j + 1)] * (j2 + 1), 0, format="csr"),
    )


def su2_generators(jmax, matter=False):
    """Block-diagonal SU(2) generators over irreps 0..jmax (or on the matter space)."""
    zero = csr_matrix((1, 1))
    if not matter:
        blocks = [_spin_block(j2) for j2 in range(1, int(round(2 * jmax)) + 1)]
        gen = {}
        for k, name in enumerate(("Tz", "Tp", "T2")):
            gen[name] = csr_matrix(block_diag([zero] + [b[k] for b in blocks], format="csr"))
        gen["Tm"] = csr_matrix(gen["Tp"].T)
        gen["Tx"] = csr_matrix(0.5 * (gen["Tp"] + gen["Tm"]))
        gen["Ty"] = csr_matrix(-0.5j * (gen["Tp"] - gen["Tm"]))
        return gen
    sz, sp, s2 = _spin_block(1)
    gen = {}
    for name, b in (("Sz_psi", sz), ("Sp_psi", sp), ("S2_psi", s2)):
        gen[name] = csr_matrix(block_diag([zero, b, zero], format="csr"))
    return gen


def su2_dressed_site_operators(spin, pure_theory, lattice_dim, background=0) -> dict:
    """Dressed-site operators for j_max = 1/2 (full local space, scipy CSR)."""
    return dict(_su2_ops_cached(float(spin), pure_theory, lattice_dim, float(background)))


@lru_cache(maxsize=32)
def _su2_ops_cached(spin, pure_theory, lattice_dim, background=0):
    if abs(spin - 0.5) > 1e-12:
        raise ValueError("the hard-core-gluon SU(2) operators exist only for spin = 1/2")
    D = lattice_dim
    dirs = "xyz"[:D]
    base = _rishon_ops_half() | su2_generators(spin)
    if background:
        base["T2_bg"] = su2_generators(background)["T2"]
    if not pure_theory:
        base |= fermion_ops(two_species=True)
        base |= su2_generators(0.5, matter=True)
    ops = {}

    def chain(place):
        names = ["Iz"] * (2 * D)
        for k, v in place.items():
            names[k] = v
        return names

    for name in ("T2", "P", "Tx", "Ty", "Tz"):
        for d, ax in enumerate(dirs):
            ops[f"{name}_m{ax}"] = kron_chain(base, chain({d: name}))
            ops[f"{name}_p{ax}"] = kron_chain(base, chain({D + d: name}))
    if D == 1:
        u = None
        for c in "rg":
            t = kron_chain(base, [f"Z{c}_dag_P", f"Z{c}"]) / np.sqrt(2)
            u = t if u is None else u + t
        ops["U"] = csr_matrix(u)
    mx, my, px, py = 0, 1, D, D + 1
    if D == 2:
        corners = {
            "C_px,py": {px: "Z{c}_P", py: "Z{c}_dag"},
            "C_py,mx": {mx: "P_Z{c}_dag", my: "P", px: "P", py: "Z{c}"},
            "C_mx,my": {mx: "Z{c}_P", my: "Z{c}_dag"},
            "C_my,px": {my: "Z{c}_P", px: "Z{c}_dag"},
        }
    elif D == 3:
        mz, pz = 2, 5
        corners = {
            "C_px,py": {px: "Z{c}_P", py: "Z{c}_dag"},
            "C_py,mx": {mx: "P_Z{c}_dag", my: "P", mz: "P", px: "P", py: "Z{c}"},
            "C_mx,my": {mx: "Z{c}_P", my: "Z{c}_dag"},
            "C_my,px": {my: "Z{c}_P", mz: "P", px: "Z{c}_dag"},
            "C_px,pz": {px: "Z{c}_P", py: "P", pz: "Z{c}_dag"},
            "C_pz,mx": {mx: "P_Z{c}_dag", my: "P", mz: "P", px: "P", py: "P", pz: "Z{c}"},
            "C_mx,mz": {mx: "Z{c}_P", my: "P", mz: "Z{c}_dag"},
            "C_mz,px": {mz: "Z{c}_P", px: "Z{c}_dag"},
            "C_py,pz": {py: "Z{c}_P", pz: "Z{c}_dag"},
            "C_pz,my": {my: "P_Z{c}_dag", mz: "P", px: "P", py: "P", pz: "Z{c}"},
            "C_my,mz": {my: "Z{c}_P", mz: "Z{c}_dag"},
            "C_mz,py": {mz: "Z{c}_P", px: "P", py: "Z{c}_dag"},
        }
    else:
        corners = {}
    for name, place in corners.items():
        acc = None
        for c in "rg":
            t = kron_chain(base, chain({k: v.format(c=c) for k, v in place.items()}))
            acc = t if acc is None else acc + t
        ops[name] = csr_matrix(acc)
    if not pure_theory:
        for name in list(ops):
            ops[name] = csr_matrix(kron(base["ID_psi"], ops[name]))
        hop = {}
        for side in "pm":
            for d, ax in enumerate(dirs):
                slot = d if side == "m" else D + d
                acc = None
                for c in "rg":
                    names = [f"psi_{c}_dag_P"] + ["P"] * slot + [f"Z{c}"] + ["Iz"] * (2 * D - slot - 1)
                    t = kron_chain(base, names)
                    acc = t if acc is None else acc + t
                hop[f"Q{side}{ax}_dag"] = csr_matrix(acc)
        ops |= hop
        # Every operator's adjoint is stored under the name without "_dag"
        # (this also replaces the Polyakov operator U by its adjoint).
        adj = {name.replace("_dag", ""): csr_matrix(op.conj().T) for name, op in ops.items()}
        ops |= adj
        for label in ("r", "g", "tot", "single", "pair", "zero"):
            ops[f"N_{label}"] = kron_chain(base, [f"N_{label}"] + ["Iz"] * (2 * D))
        ops["N-1"] = csr_matrix(ops["N_tot"] - identity(ops["N_tot"].shape[0]))
    e2 = None
    for side in "pm":
        for ax in dirs:
            t = 0.5 * ops[f"T2_{side}{ax}"]
            e2 = t if e2 is None else e2 + t
    ops["E_square"] = csr_matrix(e2)
    if background:
        bg_len = sum(j2 + 1 for j2 in range(0, int(round(2 * background)) + 1))
        for name in list(ops):
            ops[name] = csr_matrix(kron(identity(bg_len), ops[name]))
        ids = ["Iz"] * (2 * D) if pure_theory else ["ID_psi"] + ["Iz"] * (2 * D)
        ops["bg"] = kron_chain(base, ["T2_bg"] + ids)
        if D == 1:
            for side, names in (("m", ["Z{c}_dag", "P_psi", "Z{c}", "Iz"]), ("p", ["Z{c}_dag", "P_psi", "P", "Z{c}"])):
                acc = None
                for c in "rg":
                    # the first factor acts on the (3-dim) background space
                    t = kron_chain(base, [n.format(c=c) for n in names])
                    acc = t if acc is None else acc + t
                ops[f"V{side}x_dag"] = csr_matrix(acc)
            ops["Vmx"] = csr_matrix(ops["Vmx_dag"].conj().T)
            ops["Vpx"] = csr_matrix(ops["Vpx_dag"].conj().T)
    return ops



# ---------------------------------------------------------------------------
# Generic truncation j_max (any half-integer), the reference's generalized
# rishon construction (edlgt/operators/SU2_rishons.py:105-234,
# edlgt/operators/SU2_operators.py:302-622).
# ---------------------------------------------------------------------------


def _rishon_ops_gen(s2):
    """Rishon operators of one half-link truncated at doubled spin ``s2``.

    The space is the direct sum of the irreps j = 0, 1/2, ..., s2/2 (block by
    block, m descending inside a block).  ``Zr`` and ``Zg`` lower the irrep by
    one half: the state k of irrep j + 1/2 goes to the state k (red) or
    k - 1 (green) of irrep j, with the amplitude
    sqrt((j + m + 1) / sqrt((2j + 1)(2j + 2))) (red) or
    sqrt((j - m + 1) / sqrt((2j + 1)(2j + 2))) (green), m the magnetic number of
    the target state; this is the normalisation of the reference's generic
    construction (its ``chi_function``).  Two rishon species: B = (Zr, Zg) and
    A = (Zg^dag, -Zr^dag).  ``P`` is (-1)^(2j) on each block.
    """
    starts = [j2 * (j2 + 1) // 2 for j2 in range(s2 + 2)]
    size = starts[s2 + 1]
    ops = {}
    pdiag = []
    for j2 in range(s2 + 1):
        pdiag += [(-1.0) ** j2] * (j2 + 1)
    ops["P"] = diags(pdiag, 0, shape=(size, size), format="csr")
    ops["Iz"] = identity(size, format="csr")
    for color in "rg":
        rows, cols, vals = [], [], []
        for j2 in range(s2):  # target irrep j2, source irrep j2 + 1
            j = j2 / 2
            norm = np.sqrt((2 * j + 1) * (2 * j + 2))
            for k, m2 in enumerate(_m_values(j2)):
                m = m2 / 2
                num = (j + m + 1) if color == "r" else (j - m + 1)
                rows.append(starts[j2] + k)
                cols.append(starts[j2 + 1] + k + (0 if color == "r" else 1))
                vals.append(np.sqrt(num / norm))
        z = csr_matrix((vals, (rows, cols)), shape=(size, size))
        ops[f"Z{color}"] = z
        ops[f"Z{color}_dag"] = csr_matrix(z.T)
        ops[f"ZB_{color}"] = z
        ops[f"ZB_{color}_dag"] = ops[f"Z{color}_dag"]
    ops["ZA_r"] = ops["ZB_g_dag"]
    ops["ZA_g"] = csr_matrix(-ops["ZB_r_dag"])
    ops["ZA_r_dag"] = csr_matrix(ops["ZA_r"].T)
    ops["ZA_g_dag"] = csr_matrix(ops["ZA_g"].T)
    for sp in "AB":
        for color in "rg":
            ops[f"Z{sp}_{color}_P"] = csr_matrix(ops[f"Z{sp}_{color}"] @ ops["P"])
            ops[f"P_Z{sp}_{color}_dag"] = csr_matrix(ops["P"] @ ops[f"Z{sp}_{color}_dag"])
    return ops


# Corner operators of the generic model: slot -> factor (with {a} / {b} the
# first / second rishon species of C{a}{b}, {c} the colour), slots ordered
# [m_x, m_y, (m_z,) p_x, p_y, (p_z)]; as listed in
# edlgt/operators/SU2_operators.py:381-397 (2D) and 455-503 (3D).
_GEN_CORNERS_2D = {
    "px,py": {2: "Z{a}_{c}_P", 3: "Z{b}_{c}_dag"},
    "py,mx": {0: "P_Z{b}_{c}_dag", 1: "P", 2: "P", 3: "Z{a}_{c}"},
    "mx,my": {0: "Z{a}_{c}_P", 1: "Z{b}_{c}_dag"},
    "my,px": {1: "Z{a}_{c}_P", 2: "Z{b}_{c}_dag"},
}
_GEN_CORNERS_3D = {
    "px,py": {3: "Z{a}_{c}_P", 4: "Z{b}_{c}_dag"},
    "py,mx": {0: "P_Z{b}_{c}_dag", 1: "P", 2: "P", 3: "P", 4: "Z{a}_{c}"},
    "mx,my": {0: "Z{a}_{c}_P", 1: "Z{b}_{c}_dag"},
    "my,px": {1: "Z{a}_{c}_P", 2: "P", 3: "Z{b}_{c}_dag"},
    "px,pz": {3: "Z{a}_{c}_P", 4: "P", 5: "Z{b}_{c}_dag"},
    "pz,mx": {0: "P_Z{b}_{c}_dag", 1: "P", 2: "P", 3: "P", 4: "P", 5: "Z{a}_{c}"},
    "mx,mz": {0: "Z{a}_{c}_P", 1: "P", 2: "Z{b}_{c}_dag"},
    "mz,px": {2: "Z{a}_{c}_P", 3: "Z{b}_{c}_dag"},
    "py,pz": {4: "Z{a}_{c}_P", 5: "Z{b}_{c}_dag"},
    "pz,my": {1: "P_Z{b}_{c}_dag", 2: "P", 3: "P", 4: "P", 5: "Z{a}_{c}"},
    "my,mz": {1: "Z{a}_{c}_P", 2: "Z{b}_{c}_dag"},
    "mz,py": {2: "Z{a}_{c}_P", 3: "P", 4: "Z{b}_{c}_dag"},
}


def su2_gen_dressed_site_operators(spin, pure_theory, lattice_dim, background=0) -> dict:
    """Dressed-site operators of the generic SU(2) model (full local space).

    Electric Casimirs and parities per half-link, corner operators
    C{a}{b}_{corner} of both rishon species (2D and 3D), the two hopping
    species Q1 = psi_r^dag Zg^dag - psi_g^dag Zr^dag and
    Q2 = psi_r^dag Zr + psi_g^dag Zg (parity strings over the half-links in
    front of the target one) with their adjoints, matter numbers, E_square and
    the background Casimir."""
    return dict(_su2_gen_ops_cached(float(spin), pure_theory, lattice_dim, float(background)))


@lru_cache(maxsize=32)
def _su2_gen_ops_cached(spin, pure_theory, lattice_dim, background=0):
    s2 = int(round(2 * spin))
    if abs(s2 - 2 * spin) > 1e-12 or s2 < 1:
        raise ValueError(f"spin must be a positive half-integer, got {spin}")
    D = lattice_dim
    dirs = "xyz"[:D]
    base = _rishon_ops_gen(s2) | su2_generators(spin)
    if background:
        base["T2_bg"] = su2_generators(background)["T2"]
    if not pure_theory:
        base |= fermion_ops(two_species=True)
        base |= su2_generators(0.5, matter=True)
    ops = {}

    def chain(place):
        names = ["Iz"] * (2 * D)
        for k, v in place.items():
            names[k] = v
        return names

    for name in ("T2", "P"):
        for d, ax in enumerate(dirs):
            ops[f"{name}_m{ax}"] = kron_chain(base, chain({d: name}))
            ops[f"{name}_p{ax}"] = kron_chain(base, chain({D + d: name}))
    corners = _GEN_CORNERS_2D if D == 2 else (_GEN_CORNERS_3D if D == 3 else {})
    for a in "AB":
        for b in "AB":
            for corner, place in corners.items():
                acc = None
                for c in "rg":
                    t = kron_chain(base, chain({k: v.format(a=a, b=b, c=c) for k, v in place.items()}))
                    acc = t if acc is None else acc + t
                ops[f"C{a}{b}_{corner}"] = csr_matrix(acc)
    if not pure_theory:
        for name in list(ops):
            ops[name] = csr_matrix(kron(base["ID_psi"], ops[name]))
        hop = {}
        for side in "mp":
            for d, ax in enumerate(dirs):
                slot = d if side == "m" else D + d

                def term(c, z):
                    return kron_chain(base, [f"psi_{c}_dag_P"] + ["P"] * slot + [z] + ["Iz"] * (2 * D - slot - 1))

                hop[f"Q1_{side}{ax}_dag"] = csr_matrix(term("r", "Zg_dag") - term("g", "Zr_dag"))
                hop[f"Q2_{side}{ax}_dag"] = csr_matrix(term("r", "Zr") + term("g", "Zg"))
        ops |= hop
        # every operator's adjoint under the name without "_dag"
        adj = {name.replace("_dag", ""): csr_matrix(op.conj().T) for name, op in ops.items()}
        ops |= adj
        for label in ("r", "g", "tot", "single", "pair", "zero"):
            ops[f"N_{label}"] = kron_chain(base, [f"N_{label}"] + ["Iz"] * (2 * D))
    e2 = None
    for side in "pm":
        for ax in dirs:
            t = 0.5 * ops[f"T2_{side}{ax}"]
            e2 = t if e2 is None else e2 + t
    ops["E_square"] = csr_matrix(e2)
    if background:
        bg_len = sum(j2 + 1 for j2 in range(0, int(round(2 * background)) + 1))
        for name in list(ops):
            ops[name] = csr_matrix(kron(identity(bg_len), ops[name]))
        ids = ["Iz"] * (2 * D) if pure_theory else ["ID_psi"] + ["Iz"] * (2 * D)
        ops["bg"] = kron_chain(base, ["T2_bg"] + ids)
    return ops
