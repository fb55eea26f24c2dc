"""U(1) quantum-link (QED) dressed-site operators and gauge-invariant bases.

A dressed site is the tensor product ``[background] x [matter] x rishons``
with the rishons ordered ``[m_x, m_y, m_z, p_x, p_y, p_z][:2D]`` and the first
factor slowest.  Conventions (shift operator, rishon parity strings, corner
signs, Gauss law with staggered matter charge ``n - (site odd)``) reproduce
``edlgt/operators/QED_operators.py:26-331`` (operators) and ``:410-538``
(gauge-invariant states), so projected operators agree entry by entry.
"""

from __future__ import annotations

from functools import lru_cache
from itertools import product

import numpy as np
from scipy.sparse import csr_matrix, diags, identity, kron

from .common import border_classes, fermion_ops, kron_chain, selection_basis

__all__ = ["qed_rishon_operators", "qed_dressed_site_operators", "qed_gauge_invariant_states"]


def qed_rishon_operators(spin: int, U: str = "ladder", fermionic: bool = True, background: int = 0) -> dict:
    """Single-link-end operators in the electric basis ``E = -s..s``."""
    size = int(2 * spin + 1)
    ops = {}
    ops["P"] = diags([(-1.0) ** i for i in range(size)], 0, format="csr") if fermionic else identity(size, format="csr")
    if U == "ladder":
        shift = np.ones(size - 1)
    elif U == "spin":
        m = np.arange(-spin, spin + 1, dtype=float)[::-1]
        shift = np.sqrt(spin * (spin + 1) - m[1:] * (m[1:] - 1)) / spin
    else:
        raise ValueError(f"U must be 'ladder' or 'spin', got {U!r}")
    # Parallel transporter raising E by one unit.
    ops["U"] = diags(shift, -1, shape=(size, size), format="csr")
    ops["Zp"] = csr_matrix(ops["U"] @ ops["P"])
    ops["Zm_dag"] = ops["U"]
    ops["Zp_dag"] = csr_matrix(ops["Zp"].T)
    ops["Zm"] = csr_matrix(ops["Zm_dag"].T)
    ops["Zm_P"] = csr_matrix(ops["Zm"] @ ops["P"])
    ops["Zp_P"] = csr_matrix(ops["Zp"] @ ops["P"])
    ops["P_Zm_dag"] = csr_matrix(ops["P"] @ ops["Zm_dag"])
    ops["P_Zp_dag"] = csr_matrix(ops["P"] @ ops["Zp_dag"])
    ops["Iz"] = identity(size, format="csr")
    evals = np.arange(-spin, spin + 1, dtype=float)
    ops["E"] = diags(evals, 0, format="csr")
    ops["E2"] = diags(evals**2, 0, format="csr")
    if background > 0:
        ops["bg"] = diags(np.arange(-background, background + 1, dtype=float), 0, format="csr")
    return ops


def _rishon_chain(dim: int, placements: dict) -> list[str]:
    """Names for the 2*dim rishon factors; unspecified factors are identities."""
    names = ["Iz"] * (2 * dim)
    for k, v in placements.items():
        names[k] = v
    return names


def qed_dressed_site_operators(spin, pure_theory, lattice_dim, U="ladder", fermionic=True, background=0) -> dict:
    """Dressed-site operator dictionary (scipy CSR, full local space)."""
    return dict(_qed_ops_cached(spin, pure_theory, lattice_dim, U, fermionic, background))


@lru_cache(maxsize=32)
def _qed_ops_cached(spin, pure_theory, lattice_dim, U, fermionic, background):
    if lattice_dim not in (1, 2, 3):
        raise ValueError("lattice_dim must be 1, 2 or 3")
    D = lattice_dim
    dirs = "xyz"[:D]
    base = qed_rishon_operators(spin, U, fermionic, background)
    if not pure_theory:
        base |= fermion_ops(two_species=False)
    ops = {}
    # Electric-field operators on each rishon: m_<d> at slot d, p_<d> at slot D+d.
    for name in ("E", "E2", "P"):
        for d, ax in enumerate(dirs):
            ops[f"{name}_m{ax}"] = kron_chain(base, _rishon_chain(D, {d: name}))
            ops[f"{name}_p{ax}"] = kron_chain(base, _rishon_chain(D, {D + d: name}))
    # Corner (plaquette) operators; slots: mx=0,my=1,(mz=2),px=D,py=D+1,(pz=D+2)
    mx, my, px, py = 0, 1, D, D + 1
    if D == 2:
        ops["C_px,py"] = -kron_chain(base, _rishon_chain(D, {px: "Zp_P", py: "Zp_dag"}))
        ops["C_py,mx"] = kron_chain(base, _rishon_chain(D, {mx: "P_Zm_dag", my: "P", px: "P", py: "Zp"}))
        ops["C_mx,my"] = kron_chain(base, _rishon_chain(D, {mx: "Zm_P", my: "Zm_dag"}))
        ops["C_my,px"] = kron_chain(base, _rishon_chain(D, {my: "Zm_P", px: "Zp_dag"}))
    elif D == 3:
        mz, pz = 2, 5
        ops["C_px,py"] = -kron_chain(base, _rishon_chain(D, {px: "Zp_P", py: "Zp_dag"}))
        ops["C_py,mx"] = kron_chain(base, _rishon_chain(D, {mx: "P_Zm_dag", my: "P", mz: "P", px: "P", py: "Zp"}))
        ops["C_mx,my"] = kron_chain(base, _rishon_chain(D, {mx: "Zm_P", my: "Zm_dag"}))
        ops["C_my,px"] = kron_chain(base, _rishon_chain(D, {my: "Zm_P", mz: "P", px: "Zp_dag"}))
        ops["C_px,pz"] = -kron_chain(base, _rishon_chain(D, {px: "Zp_P", py: "P", pz: "Zp_dag"}))
        ops["C_pz,mx"] = kron_chain(base, _rishon_chain(D, {mx: "P_Zm_dag", my: "P", mz: "P", px: "P", py: "P", pz: "Zp"}))
        ops["C_mx,mz"] = kron_chain(base, _rishon_chain(D, {mx: "Zm_P", my: "P", mz: "Zm_dag"}))
        ops["C_mz,px"] = kron_chain(base, _rishon_chain(D, {mz: "Zm_P", px: "Zp_dag"}))
        ops["C_py,pz"] = -kron_chain(base, _rishon_chain(D, {py: "Zp_P", pz: "Zp_dag"}))
        ops["C_pz,my"] = kron_chain(base, _rishon_chain(D, {my: "P_Zm_dag", mz: "P", px: "P", py: "P", pz: "Zp"}))
        ops["C_my,mz"] = kron_chain(base, _rishon_chain(D, {my: "Zm_P", mz: "Zm_dag"}))
        ops["C_mz,py"] = kron_chain(base, _rishon_chain(D, {mz: "Zm_P", px: "P", py: "Zp_dag"}))
        ops["EzC_px,py"] = csr_matrix(1j * (ops["E_pz"] + ops["E_mz"]) @ ops["C_px,py"])
        ops["EyC_px,pz"] = csr_matrix(-1j * (ops["E_py"] + ops["E_my"]) @ ops["C_px,pz"])
        ops["ExC_py,pz"] = csr_matrix(1j * (ops["E_px"] + ops["E_mx"]) @ ops["C_py,pz"])
    if not pure_theory:
        for name in list(ops):
            ops[name] = csr_matrix(kron(base["ID_psi"], ops[name]))
        # Hopping: matter creation times rishon annihilation on the chosen side,
        # with parity strings on the rishons in front of it (3D has no matter parity).
        mat = "psi_dag" if D == 3 else "psi_dag_P"
        for side in "mp":
            for d, ax in enumerate(dirs):
                slot = d if side == "m" else D + d
                chain = [mat] + ["P"] * slot + ["Zm" if side == "m" else "Zp"] + ["Iz"] * (2 * D - slot - 1)
                ops[f"Q_{side}{ax}_dag"] = kron_chain(base, chain)
        for name in [n for n in ops if n.endswith("_dag")]:
            ops[name[:-4]] = csr_matrix(ops[name].conj().T)
        ops["N"] = kron_chain(base, ["N"] + ["Iz"] * (2 * D))
        ops["N_zero"] = kron_chain(base, ["N_zero"] + ["Iz"] * (2 * D))
    e2 = None
    for ax in dirs:
        for side in "mp":
            term = 0.5 * ops[f"E2_{side}{ax}"]
            e2 = term if e2 is None else e2 + term
    ops["E2"] = csr_matrix(e2)
    if background > 0:
        bg_dim = 2 * background + 1
        for name in list(ops):
            ops[name] = csr_matrix(kron(identity(bg_dim), ops[name]))
        ids = ["Iz"] * (2 * D) if pure_theory else ["ID_psi"] + ["Iz"] * (2 * D)
        ops["bg"] = kron_chain(base, ["bg"] + ids)
    return ops


def qed_gauge_invariant_states(spin, pure_theory, lattice_dim, background=0, get_only_bulk=False):
    basis, states = _qed_states_cached(spin, pure_theory, lattice_dim, background, get_only_bulk)
    return dict(basis), dict(states)


@lru_cache(maxsize=32)
def _qed_states_cached(spin, pure_theory, lattice_dim, background, get_only_bulk):
    """Gauss-law-satisfying local states and their selection bases.

    Returns ``(gauge_basis, gauge_states)`` keyed by ``site``/``even``/``odd``
    and ``<core>_<border>`` labels.  States are tuples ``(bg?, n?, E...)`` in
    product order; a state passes when ``sum_d (E_p - E_m) = n - odd + q_bg``.
    """
    from ..lattice import border_labels

    D = lattice_dim
    factors = [list(range(-spin, spin + 1)) for _ in range(2 * D)]
    cores = ["site"] if pure_theory else ["even", "odd"]
    if not pure_theory:
        factors.insert(0, [0, 1])
    if background > 0:
        factors.insert(0, list(range(-background, background + 1)))
    nbg = 1 if background > 0 else 0
    full_dim = int(np.prod([len(f) for f in factors]))
    states, rows = {}, {}
    for ci, core in enumerate(cores):
        keys = [core] + [f"{core}_{b}" for b in border_labels(D)]
        for k in keys:
            states[k], rows[k] = [], []
        odd = 1 if core == "odd" else 0
        for row, cfg in enumerate(product(*factors)):
            q_bg = cfg[0] if nbg else 0
            phys = cfg[nbg:]
            charge = 0 if pure_theory else int(phys[0]) - odd
            links = phys if pure_theory else phys[1:]
            div = sum(links[D + d] - links[d] for d in range(D))
            if div != charge + q_bg:
                continue
            states[core].append(cfg)
            rows[core].append(row)
            if get_only_bulk:
                continue
            for b in border_classes(links, 0, D):
                states[f"{core}_{b}"].append(cfg)
                rows[f"{core}_{b}"].append(row)
    basis = {k: selection_basis(rows[k], full_dim) for k in states}
    return basis, {k: np.asarray(v) for k, v in states.items()}
