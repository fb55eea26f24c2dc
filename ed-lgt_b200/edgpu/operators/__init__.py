"""Local dressed-site operator factories (host side, small matrices)."""

from .qed import qed_dressed_site_operators, qed_gauge_invariant_states, qed_rishon_operators
from .su2 import su2_dressed_site_operators, su2_gauge_invariant_states, su2_gen_dressed_site_operators

__all__ = [
    "qed_dressed_site_operators",
    "qed_gauge_invariant_states",
    "qed_rishon_operators",
    "su2_dressed_site_operators",
    "su2_gauge_invariant_states",
    "su2_gen_dressed_site_operators",
]
