"""Hamiltonian terms, device assembly and the QMB_hamiltonian container."""

from .hamiltonian import QMB_hamiltonian, QMB_state
from .terms import LocalTerm, NBodyTerm, PlaquetteTerm, TermBlock, TwoBodyTerm

__all__ = ["QMB_hamiltonian", "QMB_state", "LocalTerm", "TwoBodyTerm", "PlaquetteTerm", "NBodyTerm", "TermBlock"]
