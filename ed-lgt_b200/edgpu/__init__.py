"""edgpu: B200-native exact diagonalisation for lattice gauge theories.

Sector enumeration, config->index lookup, sector-Hamiltonian assembly,
matvec, Lanczos ground states and Krylov time evolution run as sm_100a CUDA
kernels in libedgpu.so (C ABI in include/edgpu.h); this package is the host
side that mirrors the ed-lgt model API (QED_Model / SU2_Model ->
build_Hamiltonian -> diagonalize / time_evolution).
"""

from . import _lib  # noqa: F401  (loads libedgpu.so; fails loudly if it is missing)
from .context import Context, default_context
from .models import QED_Model, QuantumModel, SU2_Model

__all__ = ["QED_Model", "SU2_Model", "QuantumModel", "Context", "default_context"]
__version__ = "0.1.0"
