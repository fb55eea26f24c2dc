"""Shared helpers for the local (single dressed-site) operator factories.

Operators are small scipy.sparse matrices; they are built once per model on
the host and projected onto the gauge-invariant site bases.
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix, diags, identity, kron

__all__ = [
    "kron_chain",
    "fermion_ops",
    "border_classes",
    "selection_basis",
    "project",
]


def kron_chain(ops: dict, names: list[str]):
    """Tensor product of named single-mode operators, first factor slowest."""
    out = csr_matrix(ops[names[0]])
    for name in names[1:]:
        out = kron(out, ops[name], format="csr")
    return csr_matrix(out)


def fermion_ops(two_species: bool = False) -> dict:
    """Matter operators of one staggered fermion mode (or two colours).

    Basis of one mode: index 0 empty, index 1 occupied; ``psi`` maps 1 -> 0 and
    ``P_psi = diag(1, -1)`` is the fermion parity.  With two species the
    product basis is (second species) x (first species), matching
    ``edlgt/operators/bose_fermi_operators.py:14-64``: ``psi_up`` carries the
    parity string of the slow factor.
    """
    ops = {}
    ops["psi"] = csr_matrix(np.array([[0.0, 1.0], [0.0, 0.0]]))
    ops["psi_dag"] = csr_matrix(ops["psi"].T)
    ops["P_psi"] = diags([1.0, -1.0], 0, format="csr")
    ops["N"] = csr_matrix(ops["psi_dag"] @ ops["psi"])
    ops["ID_psi"] = identity(2, format="csr")
    ops["ID"] = identity(2, format="csr")
    ops["psi_dag_P"] = csr_matrix(ops["psi_dag"] @ ops["P_psi"])
    if not two_species:
        ops["N_zero"] = csr_matrix(ops["ID"] - ops["N"])
        return ops
    one = dict(ops)
    ops["psi_down"] = kron_chain(one, ["psi", "ID"])
    ops["psi_up"] = kron_chain(one, ["P_psi", "psi"])
    ops["N_down"] = kron_chain(one, ["N", "ID"])
    ops["N_up"] = kron_chain(one, ["ID", "N"])
    ops["N_pair"] = csr_matrix(ops["N_up"] @ ops["N_down"])
    ops["N_tot"] = csr_matrix(ops["N_up"] + ops["N_down"])
    ops["N_single"] = csr_matrix(ops["N_tot"] - 2 * ops["N_pair"])
    ops["N_zero"] = csr_matrix(identity(4) - ops["N_pair"] - ops["N_single"])
    ops["ID_psi"] = identity(4, format="csr")
    ops["P_psi"] = kron_chain(one, ["P_psi", "P_psi"])
    ops["psi_r"] = ops["psi_up"]
    ops["psi_g"] = ops["psi_down"]
    ops["N_r"] = ops["N_up"]
    ops["N_g"] = ops["N_down"]
    for s in ("up", "down", "r", "g"):
        ops[f"psi_{s}_dag"] = csr_matrix(ops[f"psi_{s}"].T)
        ops[f"psi_{s}_dag_P"] = csr_matrix(ops[f"psi_{s}_dag"] @ ops["P_psi"])
    return ops


def border_classes(rishons, trivial, lattice_dim: int) -> list[str]:
    """OBC border/corner classes a local rishon configuration belongs to.

    ``rishons`` lists the link values in the order ``[m_x, m_y, m_z, p_x, p_y,
    p_z][:2*lattice_dim]``; a border class ``mx_py`` requires the rishons on
    every named side to hold the trivial value (no flux leaves the lattice).
    The set of classes matches ``edlgt/modeling/lattice_geometry.py:327-490``.
    """
    from ..lattice import AXES, border_labels

    def pos(side):
        ax = AXES.index(side[1])
        return ax if side[0] == "m" else lattice_dim + ax

    out = []
    for label in border_labels(lattice_dim):
        if all(rishons[pos(side)] == trivial for side in label.split("_")):
            out.append(label)
    return out


def selection_basis(rows: list[int], full_dim: int) -> csr_matrix:
    """Isometry whose columns are the selected canonical basis vectors."""
    k = len(rows)
    data = np.ones(k, dtype=float)
    return csr_matrix((data, (np.asarray(rows, dtype=np.int64), np.arange(k))), shape=(full_dim, k))


def _dense(a) -> np.ndarray:
    return a.toarray() if hasattr(a, "toarray") else np.asarray(a)


def project(basis, operator) -> np.ndarray:
    """Dense ``B^dagger O B`` for a column basis ``B`` (local spaces are a few
    dozen states, so dense products beat sparse ones here)."""
    b = _dense(basis)
    return b.conj().T @ _dense(operator) @ b
