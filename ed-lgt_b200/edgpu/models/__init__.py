"""Lattice gauge models on the device engine (ed-lgt model API)."""

from .qed_model import QED_Model
from .quantum_model import QuantumModel
from .su2_model import SU2_Model

__all__ = ["QuantumModel", "QED_Model", "SU2_Model"]
