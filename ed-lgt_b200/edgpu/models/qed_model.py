"""U(1) quantum-link model (QED) on the device engine.

Mirrors edlgt/models/QED_model.py: constructor and sector specification
(:23-201: N = n_sites/2 for matter, link constraints E_p - E_m = 0, surface
flux constraints for pure PBC theories), couplings ``QED_Hamiltonian_couplings``
(:719-776) and the truncated Hamiltonian (``build_truncated_Hamiltonian``
:235-394: electric energy, plaquettes, theta term, staggered mass, hopping).
"""

from __future__ import annotations

import logging

import numpy as np

from ..lattice import origin_surfaces, staggered_mask
from ..modeling import LocalTerm, PlaquetteTerm, TwoBodyTerm
from ..operators import qed_dressed_site_operators, qed_gauge_invariant_states
from .quantum_model import QuantumModel

logger = logging.getLogger(__name__)

__all__ = ["QED_Model"]


class QED_Model(QuantumModel):
    def __init__(self, spin, pure_theory, bg_list=None, plaq_basis=False, link_symmetries=True, get_only_bulk=False,
                 charge=0, **kwargs):
        super().__init__(**kwargs)
        if isinstance(spin, str):
            self._init_integrated(spin, pure_theory, bg_list)
            return
        if plaq_basis:
            raise NotImplementedError("the plaquette basis is not part of the device engine yet")
        if bg_list is not None:
            bg = np.asarray(bg_list, dtype=float)
            if bg.shape != (self.n_sites,):
                raise ValueError(f"len(bg_list) must match n_sites = {self.n_sites}: got {bg.shape}")
            self.bg_list = bg.tolist()
        else:
            self.bg_list = None
        self.spin = spin
        self.pure_theory = pure_theory
        self.plaq_basis = plaq_basis
        self.link_symmetries = link_symmetries
        self.staggered_basis = not pure_theory
        self.background = 0
        if self.bg_list is not None:
            self.background = int(max(np.abs(self.bg_list)))
            if self.background == 0:
                self.bg_list = None
        self.gauge_basis, self.gauge_states = qed_gauge_invariant_states(
            spin, pure_theory, lattice_dim=self.dim, background=self.background, get_only_bulk=get_only_bulk)
        ops = qed_dressed_site_operators(spin, pure_theory, self.dim, background=self.background)
        self.project_operators(ops, self.bg_list)
        # global symmetry
        if pure_theory:
            global_ops, global_sectors = None, None
        else:
            # total charge Q = N - n_sites/2 (nonzero Q needs static charges summing to -Q)
            global_ops, global_sectors = [self.ops["N"]], [int(self.n_sites / 2) + int(charge)]
        # link symmetries
        if link_symmetries:
            link_ops = [[self.ops[f"E_p{d}"], -self.ops[f"E_m{d}"]] for d in self.directions]
            link_sectors = [0 for _ in self.directions]
        else:
            link_ops, link_sectors = None, None
        # electric-flux n-body constraints (pure theory, PBC, D > 1)
        nbody_ops = nbody_sectors = nbody_sites = None
        nbody_type = None
        if pure_theory and not any(self.has_obc) and self.dim > 1:
            surfaces = origin_surfaces(self.lvals)
            face = {"x": "y", "y": "x"} if self.dim == 2 else {"x": "yz", "y": "xz", "z": "xy"}
            nbody_sectors = np.zeros(self.dim)
            nbody_ops, nbody_sites = [], []
            for d in self.directions:
                nbody_sites.append(np.array(surfaces[face[d]], dtype=np.int64))
                nbody_ops.append(self.ops[f"E_p{d}"])
            nbody_type = "U"
        self.get_abelian_symmetry_sector(global_ops=global_ops, global_sectors=global_sectors, link_ops=link_ops,
                                         link_sectors=link_sectors, nbody_ops=nbody_ops, nbody_sectors=nbody_sectors,
                                         nbody_sites_list=nbody_sites, nbody_sym_type=nbody_type)
        if not pure_theory:
            self.phase_weights = self._matter_phase_weights(self.ops["N"])
        self.default_params()

    def _init_integrated(self, spin, pure_theory, bg_list):
        """Gauge fields integrated out through Gauss's law (1D with matter):
        one two-state matter site per lattice site, Pauli operators with
        basis index 0 occupied (N = (Sz + 1) / 2), sector N = n_sites / 2
        (QED_Model.__init__, edlgt/models/QED_model.py:49-64, 120-125, and
        QED_gauge_integrated_operators, edlgt/operators/QED_operators.py:541-545)."""
        if spin != "integrated":
            raise ValueError(f"spin must be integer or 'integrated': got {spin}")
        if pure_theory or self.dim != 1:
            raise ValueError("QED with integrated gauge fields is only in 1D with matter")
        if bg_list is not None:
            bg = np.asarray(bg_list, dtype=float)
            if bg.shape != (self.n_sites,):
                raise ValueError(f"len(bg_list) must match n_sites = {self.n_sites}: got {bg.shape}")
            self.bg_list = bg.tolist()
        else:
            self.bg_list = None
        self.spin = spin
        self.pure_theory = False
        self.plaq_basis = False
        self.link_symmetries = False
        self.staggered_basis = False
        self.background = 0
        self.gauge_basis = self.gauge_states = None
        eye = np.eye(2)
        sz = np.diag([1.0, -1.0])
        sp = np.array([[0.0, 1.0], [0.0, 0.0]])
        ops = {"I": eye, "Sz": sz, "Sp": sp, "Sm": sp.T.copy(), "Sx": sp + sp.T, "Sy": -1j * (sp - sp.T)}
        ops["N"] = 0.5 * (sz + eye)
        ops["N_zero"] = eye - ops["N"]
        self.project_operators(ops)
        self.get_abelian_symmetry_sector(global_ops=[self.ops["N"]], global_sectors=[int(self.n_sites / 2)])
        self.phase_weights = self._matter_phase_weights(self.ops["N"])
        self.default_params()

    def _integrated_static_charges(self):
        return np.zeros(self.n_sites) if self.bg_list is None else np.asarray(self.bg_list, dtype=float)

    def integrated_blocks(self, g, m):
        """(term blocks, constant) of the integrated Hamiltonian
        (build_integrated_Hamiltonian, edlgt/models/QED_model.py:396-492):
        staggered mass, hopping t Sp_i Sm_{i+1} + h.c., and the electric energy
        sum over links of [sum_{k<=n} (q_k + (Sz_k + (-1)^k) / 2)]^2 expanded
        into Sz fields, Sz_i Sz_j couplings J_ij = E (L - 1 - j) / 2 and a
        constant."""
        from ..modeling import NBodyTerm

        self.QED_Hamiltonian_couplings(g, m)
        c, dp, n = self.coeffs, self.def_params, self.n_sites
        n_links = n - 1
        blocks = []
        for lab in ("even", "odd"):
            blocks.append(LocalTerm(self.ops["N"], "N", **dp).get_Hamiltonian(c[f"m_{lab}"],
                                                                               staggered_mask(self.lvals, lab)))
        hop = TwoBodyTerm("x", [self.ops["Sp"], self.ops["Sm"]], ["Sp", "Sm"], **dp)
        blocks.append(hop.get_Hamiltonian(strength=c["t"], add_dagger=True))
        stagger = np.array([1.0 if ii % 2 == 0 else -1.0 for ii in range(n)])
        prefix = np.cumsum(self._integrated_static_charges() + 0.5 * stagger)
        site_mask = [self._single_site_mask(ii) for ii in range(n)]
        sz = LocalTerm(self.ops["Sz"], "Sz", **dp)
        for kk in range(n_links):
            h = c["E"] * np.sum(prefix[kk:n_links])
            if abs(h) >= 1e-14:
                blocks.append(sz.get_Hamiltonian(strength=h, mask=site_mask[kk]))
        for jj in range(1, n_links):
            w = 0.5 * c["E"] * (n - 1 - jj)
            if abs(w) > 1e-14:
                for ii in range(jj):
                    term = NBodyTerm([self.ops["Sz"], self.ops["Sz"]], ["Sz", "Sz"], [(jj - ii,)], **dp)
                    blocks.append(term.get_Hamiltonian(strength=w, mask=site_mask[ii]))
        const = 0.0
        if n_links > 0:
            const = c["E"] * (np.sum(prefix[:n_links] ** 2) + 0.25 * 0.5 * n_links * (n_links + 1))
        return blocks, float(const)

    def reconstruct_integrated_E2_from_N(self, density_obs_name="N", density_corr_obs_name="N_N", state_index=None,
                                         dynamics=False, compute_density_corr=True, print_values=True):
        """<E_n^2> per link of the integrated model from the measured densities
        <N_k> and correlators <N_k N_l> (E_n = sum_{k<=n} (q_k + ((-1)^k - 1)/2
        + N_k)), QED_Model.reconstruct_integrated_E2_from_N
        (edlgt/models/QED_model.py:505-665).  A missing correlator is measured
        on the device on the chosen eigenstate or time step."""
        if self.spin != "integrated" or self.dim != 1 or self.pure_theory:
            raise ValueError("Integrated E2 reconstruction is defined only for 1D QED with matter")
        if density_obs_name not in self.res:
            raise KeyError(f"Missing '{density_obs_name}' in self.res. Measure local density first.")
        dens = np.asarray(self.res[density_obs_name], dtype=float)
        if dens.shape != (self.n_sites,):
            raise ValueError(f"Expected {density_obs_name}.shape=({self.n_sites},) got {dens.shape}.")
        n_links = self.n_sites - 1
        if n_links <= 0:
            self.res["E2"], self.res["E2_avg"] = np.zeros(0), 0.0
            return self.res["E2"]
        if density_corr_obs_name in self.res:
            corr = np.asarray(self.res[density_corr_obs_name], dtype=float)
        else:
            if not compute_density_corr:
                raise KeyError(f"Missing '{density_corr_obs_name}' in self.res. "
                               "Measure ['N','N_N'] or set compute_density_corr=True.")
            states = self.H.psi_time if dynamics else self.H.Npsi
            if state_index is None:
                if len(states) != 1:
                    raise ValueError("state_index is required when several states are available")
                state_index = 0
            term = TwoBodyTerm("x", [self.ops["N"], self.ops["N"]], ["N", "N"], **self.def_params)
            term.get_expval(states[state_index])
            corr = np.asarray(term.corr, dtype=float)
            self.res[density_corr_obs_name] = corr
        if corr.shape != (self.n_sites, self.n_sites):
            raise ValueError(f"Expected '{density_corr_obs_name}' shape ({self.n_sites}, {self.n_sites}), "
                             f"got {corr.shape}.")
        corr = np.array(corr, dtype=float, copy=True)
        np.fill_diagonal(corr, dens)  # N_k^2 = N_k
        k = np.arange(self.n_sites, dtype=float)
        prefix_charge = np.cumsum(self._integrated_static_charges() + 0.5 * ((-1.0) ** k - 1.0))
        prefix_dens = np.cumsum(dens)
        prefix_corr = np.diag(corr.cumsum(axis=0).cumsum(axis=1))
        e2 = prefix_charge[:n_links] ** 2 + 2.0 * prefix_charge[:n_links] * prefix_dens[:n_links] + \
            prefix_corr[:n_links]
        self.res["E2"] = e2
        self.res["E2_avg"] = float(np.mean(e2))
        if print_values:
            for ii in range(n_links):
                logger.info(f"E2[{ii}] = {e2[ii]:.12f}")
        return e2

    def _single_site_mask(self, site_index):
        mask = np.zeros(tuple(self.lvals), dtype=bool)
        mask[(site_index,)] = True
        return mask

    def build_integrated_Hamiltonian(self, g, m, theta=0.0, dtype_mode="auto"):
        from scipy.sparse import identity

        self.default_params()
        blocks, const = self.integrated_blocks(g, m)
        for b in blocks:
            self.H.add_term(b)
        if abs(const) > 1e-14:
            self.H.add_term(const * identity(self.H.shape[0], format="csc"))
        self.H.build(self.ham_format, force_complex=(self._resolve_dtype_mode(dtype_mode) == "complex"))

    def _bg_values(self, states):
        return np.asarray(states, dtype=float)[:, 0]

    def QED_Hamiltonian_couplings(self, g, m=None, theta=0.0, magnetic_basis=False):
        if magnetic_basis:
            self.coeffs = {"g": g, "E": -g, "B": -0.5 / g}
            return
        E, B = g / 2, -1 / (2 * g)
        coeffs = {"g": g, "E": E, "B": B, "theta": -theta * g}
        if not self.pure_theory and m is not None:
            t = 1 / 2
            coeffs |= {
                "t": -complex(0, t),
                "tx_even": -complex(0, t),
                "tx_odd": -complex(0, t),
                "ty_even": -t,
                "ty_odd": t,
                "tz_even": -complex(0, t),
                "tz_odd": complex(0, t),
                "m": m,
                "m_odd": -m,
                "m_even": m,
            }
        self.coeffs = coeffs

    def overlap_QMB_state(self, name):
        """Named benchmark configurations of 1D QED with matter and the
        truncated spin-1 basis (QED_Model.overlap_QMB_state,
        edlgt/models/QED_model.py:778-849): ``V`` (alias ``PV``) the vacuum,
        states 1 / 3 on even / odd sites (0 and 1 at the open edges), and
        ``meson_center``, states 4 / 1 on the central (even, odd) pair.  The
        integrated basis and the 3D string states are not built."""
        key = name.strip().lower().replace(" ", "_")
        key = "v" if key == "pv" else key
        if self.dim != 1 or self.pure_theory or key not in ("v", "meson_center"):
            raise NotImplementedError("named states are built for 1D QED with matter ('V', 'meson_center')")
        if not (np.isscalar(self.spin) and int(self.spin) == 1):
            raise NotImplementedError("named 1D states need the truncated spin=1 basis")
        n = self.n_sites
        cfg = np.array([1 if ii % 2 == 0 else 3 for ii in range(n)], dtype=np.int32)
        if all(self.has_obc):
            cfg[0] = 0
            if n >= 2:
                cfg[-1] = 1
        if key == "meson_center":
            even = n // 2
            even -= even % 2
            even = max(0, min(even, n - 2))
            cfg[even], cfg[even + 1] = 4, 1
        return cfg

    def build_Hamiltonian(self, g, m=None, theta=0.0, dtype_mode="auto"):
        if self.spin == "integrated":
            return self.build_integrated_Hamiltonian(g, m, theta, dtype_mode)
        return self.build_truncated_Hamiltonian(g, m, theta, dtype_mode)

    def hamiltonian_blocks(self, g, m=None, theta=0.0):
        """Term blocks of the truncated Hamiltonian (reference term order)."""
        self.QED_Hamiltonian_couplings(g, m, theta)
        c = self.coeffs
        dp = self.def_params
        blocks = [LocalTerm(self.ops["E2"], "E2", **dp).get_Hamiltonian(strength=c["E"])]
        planes = []
        if self.dim > 1:
            planes.append((["x", "y"], ["C_px,py", "C_py,mx", "C_my,px", "C_mx,my"]))
        if self.dim == 3:
            planes.append((["x", "z"], ["C_px,pz", "C_pz,mx", "C_mz,px", "C_mx,mz"]))
            planes.append((["y", "z"], ["C_py,pz", "C_pz,my", "C_mz,py", "C_my,mz"]))
        for axes, names in planes:
            term = PlaquetteTerm(axes, [self.ops[o] for o in names], names, **dp)
            blocks.append(term.get_Hamiltonian(strength=c["B"], add_dagger=True))
        if self.dim == 2 and abs(c["theta"]) > 10e-10:
            names = ["C_px,py", "C_py,mx", "C_my,px", "C_mx,my"]
            term = PlaquetteTerm(["x", "y"], [self.ops[o] for o in names], names, **dp)
            blocks.append(term.get_Hamiltonian(strength=c["theta"], add_dagger=True))
        if self.dim == 3 and abs(c["theta"]) > 10e-10:
            for axes, names in (
                (["x", "y"], ["EzC_px,py", "C_py,mx", "C_my,px", "C_mx,my"]),
                (["x", "z"], ["EyC_px,pz", "C_pz,mx", "C_mz,px", "C_mx,mz"]),
                (["y", "z"], ["ExC_py,pz", "C_pz,my", "C_mz,py", "C_my,mz"]),
            ):
                term = PlaquetteTerm(axes, [self.ops[o] for o in names], names, **dp)
                blocks.append(term.get_Hamiltonian(strength=c["theta"], add_dagger=True))
        if not self.pure_theory:
            for lab in ("even", "odd"):
                term = LocalTerm(self.ops["N"], "N", **dp)
                blocks.append(term.get_Hamiltonian(c[f"m_{lab}"], staggered_mask(self.lvals, lab)))
            for d in self.directions:
                for lab in ("even", "odd"):
                    names = [f"Q_p{d}_dag", f"Q_m{d}"]
                    term = TwoBodyTerm(d, [self.ops[o] for o in names], names, **dp)
                    blocks.append(term.get_Hamiltonian(strength=c[f"t{d}_{lab}"], add_dagger=True,
                                                       mask=staggered_mask(self.lvals, lab)))
        if not self.link_symmetries:
            blocks.append(LocalTerm(self.ops["E2"], "E2", **dp).get_Hamiltonian(strength=100))
            for d in self.directions:
                names = [f"E_p{d}", f"E_m{d}"]
                term = TwoBodyTerm(d, [self.ops[o] for o in names], names, **dp)
                blocks.append(term.get_Hamiltonian(strength=-100))
        return blocks

    def build_truncated_Hamiltonian(self, g, m=None, theta=0.0, dtype_mode="auto"):
        self.default_params()
        for b in self.hamiltonian_blocks(g, m, theta):
            self.H.add_term(b)
        self.H.build(self.ham_format, force_complex=(self._resolve_dtype_mode(dtype_mode) == "complex"))
