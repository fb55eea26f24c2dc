"""SU(2) Yang-Mills (+ staggered matter): the hard-core-gluon model
(j_max = 1/2) and the generic model (any j_max, or ``use_generic_model``).

Mirrors edlgt/models/SU2_model.py: constructor and sector (:31-171: total
fermion number ``sectors``, link Casimir constraints T2_p - T2_m = 0, Z2 flux
parities for pure PBC theories, optional static charges ``bg_list``),
couplings ``SU2_Hamiltonian_couplings`` (:555-624), ``build_base_Hamiltonian``
(:200-355) and ``build_gen_Hamiltonian`` (:357-472).
"""

from __future__ import annotations

import logging

import numpy as np

from ..lattice import origin_surfaces, staggered_mask
from ..modeling import LocalTerm, PlaquetteTerm, QMB_hamiltonian, TwoBodyTerm
from ..operators import su2_dressed_site_operators, su2_gauge_invariant_states, su2_gen_dressed_site_operators
from .quantum_model import QuantumModel

logger = logging.getLogger(__name__)

__all__ = ["SU2_Model"]


class SU2_Model(QuantumModel):
    def __init__(self, spin, pure_theory, bg_list=None, sectors=None, use_generic_model=False, **kwargs):
        super().__init__(**kwargs)
        self.spin = spin
        self.use_generic_model = bool(use_generic_model)
        self.generic = self.use_generic_model or spin >= 1
        self.pure_theory = pure_theory
        self.background = max(bg_list) if bg_list is not None else 0
        self.bg_list = bg_list if self.background != 0 else None
        self.gauge_basis, self.gauge_states = su2_gauge_invariant_states(spin, pure_theory, lattice_dim=self.dim,
                                                                         background=self.background)
        factory = su2_gen_dressed_site_operators if self.generic else su2_dressed_site_operators
        ops = factory(spin, pure_theory, lattice_dim=self.dim, background=self.background)
        self.project_operators(ops, bg_sector_list=self.bg_list)
        if pure_theory:
            global_ops, global_sectors = None, None
            self.zero_density = None
        else:
            global_ops, global_sectors = [self.ops["N_tot"]], sectors
            self.zero_density = sectors[0] == self.n_sites
        link_ops = [[self.ops[f"T2_p{d}"], -self.ops[f"T2_m{d}"]] for d in self.directions]
        link_sectors = [0 for _ in self.directions]
        nbody_ops = nbody_sectors = nbody_sites = None
        nbody_type = None
        if pure_theory and not any(self.has_obc) and self.dim > 1:
            surfaces = origin_surfaces(self.lvals)
            face = {"x": "y", "y": "x"} if self.dim == 2 else {"x": "yz", "y": "xz", "z": "xy"}
            nbody_sectors = list(np.ones(self.dim))
            nbody_ops, nbody_sites = [], []
            for d in self.directions:
                nbody_sites.append(np.array(surfaces[face[d]], dtype=np.int64))
                nbody_ops.append(self.ops[f"P_p{d}"])
            nbody_type = "Z"
        self.get_abelian_symmetry_sector(global_ops=global_ops, global_sectors=global_sectors, link_ops=link_ops,
                                         link_sectors=link_sectors, nbody_ops=nbody_ops, nbody_sectors=nbody_sectors,
                                         nbody_sites_list=nbody_sites, nbody_sym_type=nbody_type)
        if self.sector is not None and len(self.sector) == 0:
            raise ValueError("No configurations found for the given symmetry sectors")
        if not pure_theory:
            self.phase_weights = self._matter_phase_weights(self.ops["N_tot"])
        self.default_params()

    def _bg_values(self, states):
        # first label of a local state is twice the background spin
        return np.asarray(states, dtype=float)[:, 0] / 2.0

    def SU2_Hamiltonian_couplings(self, g, m=None, theta=0.0):
        if self.dim == 1:
            E, B = 8 * g / 3, 0
        else:
            E, B = g / 2, -1 / (2 * g)
        self.coeffs = {"g": g, "E": E, "B": B, "theta": -theta * g}
        if not self.pure_theory and m is not None:
            t = 2 * np.sqrt(2)
            self.coeffs |= {
                "tx_even": -complex(0, t),
                "tx_odd": -complex(0, t),
                "ty_even": -t,
                "ty_odd": t,
                "tz_even": -t,
                "tz_odd": t,
                "m": m,
                "m_odd": -m,
                "m_even": m,
            }

    # named benchmark configurations of the j = 1/2 dressed-site basis
    # (SU2_Model.overlap_QMB_state, edlgt/models/SU2_model.py:486-553): 1D
    # labels give (even-site state, odd-site state, left edge, right edge)
    _OVERLAP_1D = {"V": (0, 4, 0, 2), "PV": (1, 5, 1, 1), "T": (6, 12, 1, 1), "M": (2, 3, 1, 1),
                   "B": (7, 11, 1, 1)}
    _OVERLAP_2D_OBC = {"V": [0, 9, 0, 4, 4, 0, 9, 0], "PV1": [1, 12, 3, 5, 5, 2, 11, 1],
                       "PV2": [1, 11, 1, 5, 5, 3, 10, 1]}

    def overlap_QMB_state(self, name):
        """Configuration (local-state index per site) of a named benchmark state:
        V bare vacuum, PV polarized vacuum, T, M, B, and the domain walls DW /
        DW2 in 1D; V, PV1, PV2 on the 2x2 lattice with matter; V of the pure
        theory.  Unknown 1D labels give the all-zero configuration, as in the
        reference."""
        n = self.n_sites
        if len(self.lvals) == 1:
            if name == "DW":
                cfg = [0 if ii < n // 2 else 4 for ii in range(n)]
                edges = (0, 2)
            elif name == "DW2":
                cfg = [0 if (ii // 2) % 2 == 0 else 4 for ii in range(n)]
                edges = (0, 2)
            else:
                even, odd, left, right = self._OVERLAP_1D.get(name, (0, 0, 0, 0))
                cfg = [even if ii % 2 == 0 else odd for ii in range(n)]
                edges = (left, right)
            if self.has_obc[0]:
                cfg[0], cfg[-1] = edges
            return np.array(cfg)
        if self.pure_theory:
            if name != "V":
                raise ValueError(f"unknown pure-theory state {name}")
            return np.zeros(n, dtype=np.int64)
        if not self.has_obc[0]:
            return np.array([0, 9, 0, 9, 9, 0, 9, 0])
        if name not in self._OVERLAP_2D_OBC:
            raise ValueError(f"unknown 2D state {name}")
        return np.array(self._OVERLAP_2D_OBC[name])

    def get_mask(self, sites_list):
        """Boolean lattice mask selecting the given sites (SU2_model.py:701-706)."""
        mask = np.zeros(self.lvals, dtype=bool)
        for site in sites_list:
            mask[site] = True
        return mask

    def build_local_Hamiltonian(self, g, m, R0):
        """``self.Hlocal``: the 1D Hamiltonian density around site R0 (electric
        and mass terms at R0, half of the hoppings on the bonds (R0-1, R0) and
        (R0, R0+1) with their conjugates), SU2_Model.build_local_Hamiltonian
        (edlgt/models/SU2_model.py:626-699), assembled on the device."""
        if self.dim > 1:
            raise ValueError(f"Local Hamiltonian valid only for D=1, got {self.dim}")
        self.SU2_Hamiltonian_couplings(g, m)
        dp = self.def_params
        c = self.coeffs
        self.Hlocal = QMB_hamiltonian(self.lvals, len(self.sector), sector=self.sector,
                                      phase_weights=self.phase_weights)
        here, left = self.get_mask([R0]), self.get_mask([(R0 - 1) % self.n_sites])
        self.Hlocal.add_term(LocalTerm(self.ops["E_square"], "E_square", **dp).get_Hamiltonian(c["E"], here))
        self.Hlocal.add_term(LocalTerm(self.ops["N-1"], "N-1", **dp).get_Hamiltonian(((-1) ** R0) * c["m"], here))
        hop = TwoBodyTerm("x", [self.ops["Qpx_dag"], self.ops["Qmx"]], ["Qpx_dag", "Qmx"], **dp)
        hop_dag = TwoBodyTerm("x", [self.ops["Qpx"], self.ops["Qmx_dag"]], ["Qpx", "Qmx_dag"], **dp)
        half = 0.5 * c["tx_even"]
        for term, sign in ((hop, 1.0), (hop_dag, -1.0)):
            self.Hlocal.add_term(term.get_Hamiltonian(sign * half, mask=here))
            self.Hlocal.add_term(term.get_Hamiltonian(sign * half, mask=left))

    def build_Hamiltonian(self, g, m=None, theta=0.0, lambda_noise=0.0, dtype_mode="auto"):
        if self.generic:
            self.build_gen_Hamiltonian(g, m, dtype_mode)
        else:
            self.build_base_Hamiltonian(g, m, theta, lambda_noise, dtype_mode)

    # the 16 species patterns of a plaquette's four corners in the generic
    # model (edlgt/models/SU2_model.py:428-445), corners in the order
    # (p0, p1), (p1, m0), (m1, p0), (m0, m1)
    _GEN_PLAQUETTE_SET = (
        "AB AB AB AB", "AA AB BB AB", "AB AB AA BB", "AA AB BA BB", "AB BB AB AA", "AA BB BB AA", "AB BB AA BA",
        "AA BB BA BA", "BB AA AB AB", "BA AA BB AB", "BB AA AA BB", "BA AA BA BB", "BB BA AB AA", "BA BA BB AA",
        "BB BA AA BA", "BA BA BA BA",
    )

    def gen_hamiltonian_blocks(self, g, m=None):
        """Term blocks of the generic model: electric Casimir, staggered mass on
        N_tot, the two hopping species [Q1_p^dag, Q2_m] and [Q2_p^dag, Q1_m]
        with their conjugates, and the plaquettes of the 16 corner-species
        patterns (edlgt/models/SU2_model.py:357-472)."""
        self.SU2_Hamiltonian_couplings(g, m)
        c = self.coeffs
        dp = self.def_params
        blocks = [LocalTerm(self.ops["E_square"], "E_square", **dp).get_Hamiltonian(strength=c["E"])]
        if not self.pure_theory:
            for lab in ("even", "odd"):
                term = LocalTerm(self.ops["N_tot"], "N_tot", **dp)
                blocks.append(term.get_Hamiltonian(c[f"m_{lab}"], staggered_mask(self.lvals, lab)))
            for d in self.directions:
                for lab in ("even", "odd"):
                    for names in ([f"Q1_p{d}_dag", f"Q2_m{d}"], [f"Q2_p{d}_dag", f"Q1_m{d}"]):
                        term = TwoBodyTerm(d, [self.ops[o] for o in names], names, **dp)
                        blocks.append(term.get_Hamiltonian(strength=c[f"t{d}_{lab}"], add_dagger=True,
                                                           mask=staggered_mask(self.lvals, lab)))
        if self.dim > 1:
            planes = ["xy"] if self.dim == 2 else ["xy", "xz", "yz"]
            for pdir in planes:
                for pat in self._GEN_PLAQUETTE_SET:
                    s0, s1, s2, s3 = pat.split()
                    names = [f"C{s0}_p{pdir[0]},p{pdir[1]}", f"C{s1}_p{pdir[1]},m{pdir[0]}",
                             f"C{s2}_m{pdir[1]},p{pdir[0]}", f"C{s3}_m{pdir[0]},m{pdir[1]}"]
                    term = PlaquetteTerm([pdir[0], pdir[1]], [self.ops[o] for o in names], names, **dp)
                    blocks.append(term.get_Hamiltonian(strength=c["B"], add_dagger=True))
        return blocks

    def build_gen_Hamiltonian(self, g, m=None, dtype_mode="auto"):
        self.default_params()
        for b in self.gen_hamiltonian_blocks(g, m):
            self.H.add_term(b)
        self.H.build(self.ham_format, force_complex=(self._resolve_dtype_mode(dtype_mode) == "complex"))

    def hamiltonian_blocks(self, g, m=None, theta=0.0, lambda_noise=0.0):
        if self.generic:
            return self.gen_hamiltonian_blocks(g, m)
        self.SU2_Hamiltonian_couplings(g, m, theta)
        c = self.coeffs
        dp = self.def_params
        blocks = [LocalTerm(self.ops["E_square"], "E_square", **dp).get_Hamiltonian(strength=c["E"])]
        planes = []
        if self.dim > 1:
            planes.append((["x", "y"], ["C_px,py", "C_py,mx", "C_my,px", "C_mx,my"]))
        if self.dim == 3:
            planes.append((["x", "z"], ["C_px,pz", "C_pz,mx", "C_mz,px", "C_mx,mz"]))
            planes.append((["y", "z"], ["C_py,pz", "C_pz,my", "C_mz,py", "C_my,mz"]))
        for axes, names in planes:
            term = PlaquetteTerm(axes, [self.ops[o] for o in names], names, **dp)
            blocks.append(term.get_Hamiltonian(strength=c["B"], add_dagger=True))
        if not self.pure_theory:
            for lab in ("even", "odd"):
                term = LocalTerm(self.ops["N-1"], "N-1", **dp)
                blocks.append(term.get_Hamiltonian(c[f"m_{lab}"], staggered_mask(self.lvals, lab)))
            for d in self.directions:
                for lab in ("even", "odd"):
                    names = [f"Qp{d}_dag", f"Qm{d}"]
                    term = TwoBodyTerm(d, [self.ops[o] for o in names], names, **dp)
                    blocks.append(term.get_Hamiltonian(strength=c[f"t{d}_{lab}"], add_dagger=True,
                                                       mask=staggered_mask(self.lvals, lab)))
        if self.dim == 3 and abs(c["theta"]) > 10e-10:
            raise NotImplementedError("the 3D theta term is not part of the device engine yet")
        noise = [self.background > 0, lambda_noise > 0] + [not obc for obc in self.has_obc]
        if all(noise):
            names = ["Vpx_dag", "Vmx"]
            term = TwoBodyTerm("x", [self.ops[o] for o in names], names, **dp)
            blocks.append(term.get_Hamiltonian(strength=-lambda_noise, add_dagger=True))
        return blocks

    def build_base_Hamiltonian(self, g, m=None, theta=0.0, lambda_noise=0.0, dtype_mode="auto"):
        self.default_params()
        for b in self.hamiltonian_blocks(g, m, theta, lambda_noise):
            self.H.add_term(b)
        self.H.build(self.ham_format, force_complex=(self._resolve_dtype_mode(dtype_mode) == "complex"))
