"""``QuantumModel``: operator projection, device sector, Hamiltonian container,
diagonalisation, dynamics and observables.

Mirrors edlgt/models/quantum_model.py (``project_operators`` :400-502,
``get_abelian_symmetry_sector`` :504-604, ``default_params`` :171-211,
``diagonalize_Hamiltonian`` :606-611, ``time_evolution_Hamiltonian``
:613-615, ``get_qmb_state_from_configs`` :826-862, ``get_observables`` /
``measure_observables`` / ``link_avg`` / ``stag_avg`` :1158-1333).  The
sector lives on the device as sorted keys; ``sector_configs`` is the
reference's uint16 table, decoded on demand.
"""

from __future__ import annotations

import ctypes
import logging
from math import prod

import numpy as np
import torch

from .. import _lib
from .._lib import check, lib, ptr, stream_handle
from ..lattice import lattice_labels, link_site_pairs, neighbor_sites, staggered_mask, zig_zag
from ..modeling import LocalTerm, NBodyTerm, PlaquetteTerm, QMB_hamiltonian, QMB_state, TwoBodyTerm
from ..modeling.assembly import assemble_blocks
from ..operators.common import project
from ..symmetries import SectorSpec, enumerate_sector, get_symmetry_sector_generators

logger = logging.getLogger(__name__)

__all__ = ["QuantumModel"]


_DIAG_CACHE = {}


def site_expval_device(sector, op, psi, out=None):
    """Device vector of <psi| op_s |psi> over sites (op diagonal only)."""
    key = (id(op), sector.device)
    if key not in _DIAG_CACHE:
        diag = np.real(np.array([np.diagonal(op[s]) for s in range(op.shape[0])])).astype(np.float64)
        _DIAG_CACHE[key] = (op, torch.from_numpy(np.ascontiguousarray(diag)).to(sector.device))
    dd = _DIAG_CACHE[key][1]
    codes = {torch.float64: 0, torch.float32: 1, torch.complex128: 2, torch.complex64: 3}
    if psi.dtype not in codes:
        psi = psi.to(torch.complex128)
    p = psi.contiguous()
    n_sites = sector.n_sites
    if out is None:
        out = torch.empty(n_sites, dtype=torch.float64, device=sector.device)
    dims = _lib.SiteDims()
    for s in range(n_sites):
        dims.d[s] = int(sector.loc_dims[s])
    if sector.wide:
        check(lib.edg_local_expval_wide(ptr(sector.keys), len(sector), sector.n_hi, ctypes.byref(dims), n_sites, ptr(p),
                                        codes[p.dtype], 1, ptr(dd), dd.shape[1], ptr(out), stream_handle()),
              "edg_local_expval_wide")
    else:
        check(lib.edg_local_expval(ptr(sector.keys), len(sector), ctypes.byref(dims), n_sites, ptr(p), codes[p.dtype],
                                   1, ptr(dd), dd.shape[1], ptr(out), stream_handle()), "edg_local_expval")
    return out


def _transition_tables(ops, dmax, tol=1e-10):
    """Per site and bra state, the kets with |<bra|op|ket>| > tol and their
    amplitudes (the threshold of _prepare_local_transition_data,
    edlgt/symmetries/sym_qmb_operations.py:32-92)."""
    n_sites = ops.shape[0]
    count = np.zeros((n_sites, dmax), dtype=np.int32)
    ket = np.zeros((n_sites, dmax, dmax), dtype=np.uint8)
    amp = np.zeros((n_sites, dmax, dmax, 2), dtype=np.float64)
    for s in range(n_sites):
        m = np.asarray(ops[s], dtype=np.complex128)
        for b in range(min(dmax, m.shape[0])):
            ks = np.nonzero(np.abs(m[b]) > tol)[0]
            count[s, b] = len(ks)
            ket[s, b, : len(ks)] = ks
            amp[s, b, : len(ks), 0] = m[b, ks].real
            amp[s, b, : len(ks), 1] = m[b, ks].imag
    return count, ket, amp


def twobody_corr_device(sector, op_a, op_b, psi, pairs=None):
    """Device matrix corr[i][j] = corr[j][i] = Re <psi| A_i B_j |psi> over site
    pairs i < j (all pairs by default), zero diagonal: TwoBodyTerm.get_expval
    with lattice_twobody_exp_val (edlgt/modeling/twobody_term.py:160-264).
    op_a, op_b: (n_sites, dmax, dmax) projected site operators; psi: device
    vector in the sector basis."""
    sector.require_narrow("two-body correlators")
    n_sites = sector.n_sites
    dmax = int(op_a.shape[-1])
    key = ("tb", id(op_a), id(op_b), sector.device, tuple(int(d) for d in sector.loc_dims))
    if key not in _DIAG_CACHE:
        ca, ka, aa = _transition_tables(op_a, dmax)
        cb, kb, ab = _transition_tables(op_b, dmax)
        dev = sector.device
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        _DIAG_CACHE[key] = (op_a, op_b, up(np.stack([ca, cb])), up(np.stack([ka, kb])), up(np.stack([aa, ab])),
                            up(sector.strides.astype(np.int64)), up(sector.loc_dims.astype(np.int32)))
    _, _, t_count, t_ket, t_amp, strides, loc_dims = _DIAG_CACHE[key]
    if pairs is None:
        pairs = [(i, j) for i in range(n_sites) for j in range(i + 1, n_sites)]
    pairs = np.asarray(pairs, dtype=np.int32).reshape(-1, 2)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(sector.device)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(sector.device)
    codes = {torch.float64: 0, torch.float32: 1, torch.complex128: 2, torch.complex64: 3}
    if psi.dtype not in codes:
        psi = psi.to(torch.complex128)
    p = psi.contiguous()
    n_pairs = len(pairs)
    ns = lib.edg_twobody_scratch_elems(n_pairs)
    scratch = torch.empty(max(ns, 1), dtype=torch.float64, device=sector.device)
    corr = torch.empty((n_sites, n_sites), dtype=torch.float64, device=sector.device)
    check(lib.edg_twobody_expval(sector.lookup_table(), ptr(strides), ptr(loc_dims), n_sites, ptr(t_count),
                                 ptr(t_ket), ptr(t_amp), dmax, ptr(pi), ptr(pj), n_pairs, ptr(p), codes[p.dtype], 1,
                                 ptr(corr), ptr(scratch), ns, stream_handle()), "edg_twobody_expval")
    return corr


class QuantumModel:
    def __init__(self, lvals, has_obc, ham_format="gpu", basis_projector=None, device=None):
        self.lvals = list(lvals)
        self.dim = len(self.lvals)
        self.directions = "xyz"[: self.dim]
        self.n_sites = prod(self.lvals)
        self.has_obc = list(has_obc)
        self.ham_format = ham_format
        self.basis_projector = basis_projector
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.sector = None
        self.gauge_basis = None
        self.gauge_states = None
        self.staggered_basis = False
        self.momentum_basis = None
        self.phase_weights = None
        self.res = {}
        self.H = None
        self._partition_cache = {}
        self._momentum = None
        self.dtype_mode = "auto"

    # ------------------------------------------------------------- sector
    @property
    def sector_configs(self):
        return None if self.sector is None else self.sector.configs

    @property
    def sector_dim(self):
        return None if self.sector is None else len(self.sector)

    # ------------------------------------------------------- projection
    def project_operators(self, ops_dict, bg_sector_list=None, bg_label_col=None):
        """Project local operators onto each site's gauge-invariant basis.

        ``self.ops[name]`` becomes a ``(n_sites, dmax, dmax)`` complex array,
        zero-padded beyond each site's local dimension.
        """
        if self.gauge_basis is not None:
            labels = lattice_labels(self.lvals, self.has_obc, self.staggered_basis)
            loc_dims = np.array([self.gauge_basis[l].shape[1] for l in labels], dtype=np.int64)
            self.lattice_labels = np.array(labels, dtype=object)
        else:
            d = next(iter(ops_dict.values())).shape[0]
            loc_dims = np.full(self.n_sites, d, dtype=np.int64)
            self.lattice_labels = None
        if self.basis_projector is not None:
            loc_dims = np.full(self.n_sites, self.basis_projector.shape[1], dtype=np.int64)
            bg_sector_list = None
        self.loc_dims = loc_dims.copy()
        cols_per_site = None
        self.gauge_states_per_site = []
        if bg_sector_list is not None and self.gauge_basis is not None:
            if len(bg_sector_list) != self.n_sites:
                raise ValueError("bg_sector_list must have length n_sites")
            cols_per_site = []
            for ii in range(self.n_sites):
                lab = self.lattice_labels[ii]
                col = self._bg_values(self.gauge_states[lab])
                cols = np.flatnonzero(np.isclose(col, float(bg_sector_list[ii]), rtol=0.0, atol=1e-12))
                if cols.size == 0:
                    raise ValueError(f"No GI states at site {ii} label={lab} with bg {bg_sector_list[ii]}")
                cols_per_site.append(cols)
                self.loc_dims[ii] = cols.size
                self.gauge_states_per_site.append(self.gauge_states[lab][cols])
        elif self.gauge_basis is not None:
            for ii in range(self.n_sites):
                self.gauge_states_per_site.append(self.gauge_states[self.lattice_labels[ii]])
        dmax = int(np.max(self.loc_dims))
        self.ops = {}
        cache = {}
        for name, op in ops_dict.items():
            arr = np.zeros((self.n_sites, dmax, dmax), dtype=np.complex128)
            for jj in range(self.n_sites):
                d = int(self.loc_dims[jj])
                if self.gauge_basis is not None:
                    lab = self.lattice_labels[jj]
                    cols = None if cols_per_site is None else tuple(cols_per_site[jj])
                    key = (name, lab, cols)
                    if key not in cache:
                        basis = self.gauge_basis[lab]
                        if cols is not None:
                            basis = basis[:, list(cols)]
                        cache[key] = project(basis, op)
                    eff = cache[key]
                else:
                    eff = op.toarray() if hasattr(op, "toarray") else np.asarray(op)
                if self.basis_projector is not None:
                    eff = project(self.basis_projector, eff)
                arr[jj, :d, :d] = eff
            self.ops[name] = arr

    def _bg_values(self, states):
        """Background charge of each local basis state (first label column)."""
        return np.asarray(states, dtype=float)[:, 0]

    # ---------------------------------------------------------- symmetries
    def get_abelian_symmetry_sector(self, global_ops=None, global_sectors=None, global_sym_type="U", link_ops=None,
                                    link_sectors=None, nbody_ops=None, nbody_sectors=None, nbody_sites_list=None,
                                    nbody_sym_type=None, string_ops=None, string_sectors=None):
        g_diags = get_symmetry_sector_generators(global_ops, "global") if global_ops is not None else None
        l_diags = get_symmetry_sector_generators(link_ops, "link") if link_ops is not None else None
        pairs = link_site_pairs(self.lvals, self.has_obc) if link_ops is not None else None
        n_diags = get_symmetry_sector_generators(nbody_ops, "nbody") if nbody_ops is not None else None
        s_diags = get_symmetry_sector_generators(string_ops, "global") if string_ops is not None else None
        if g_diags is None and l_diags is None and n_diags is None:
            logger.info("NO SYMMETRY DETECTED: no sector_configs")
            self.sector = None
            return
        nb_type = nbody_sym_type if nbody_sym_type is not None else "U"
        # plain description of the constraints (also what the CPU oracle consumes)
        self.sector_inputs = dict(loc_dims=self.loc_dims, glob_diags=g_diags, glob_sectors=global_sectors,
                                  glob_type=global_sym_type, link_diags=l_diags, link_sectors=link_sectors,
                                  pair_list=pairs, string_diags=s_diags, string_sectors=string_sectors,
                                  nbody_diags=n_diags, nbody_sectors=nbody_sectors, nbody_sites=nbody_sites_list,
                                  nbody_type=nb_type)
        self.sector_spec = SectorSpec(self.loc_dims, g_diags, global_sectors, global_sym_type, l_diags, link_sectors,
                                      pairs, s_diags, string_sectors, n_diags, nbody_sectors, nbody_sites_list, nb_type)
        if self.device.type != "cuda":
            # description only: every compute call needs the device engine
            self.sector = None
            return
        self.sector = enumerate_sector(self.sector_spec, self.device)
        logger.info(f"SEC DIM: {len(self.sector)}")

    def default_params(self):
        self.def_params = {
            "lvals": self.lvals,
            "has_obc": self.has_obc,
            "loc_dims": self.loc_dims,
            "staggered_basis": self.staggered_basis,
            "gauge_basis": self.gauge_basis,
            "sector_configs": None,
            "momentum_basis": self.momentum_basis,
            "sector": self.sector,
            "phase_weights": self.phase_weights,
        }
        if self.sector is not None:
            self.H = QMB_hamiltonian(self.lvals, len(self.sector), sector=self.sector,
                                     phase_weights=self.phase_weights)
        else:
            self.H = None

    def _matter_phase_weights(self, number_op):
        """Per-site exponents x_s * n(c) of the real form's gauge transform."""
        n = np.rint(np.real(np.array([np.diagonal(number_op[s]) for s in range(self.n_sites)]))).astype(np.int64)
        xs = np.array([zig_zag(self.lvals, s)[0] for s in range(self.n_sites)], dtype=np.int64)
        return (xs[:, None] * n) % 4

    # ---------------------------------------------------------- solve
    def set_momentum_sector(self, k_unit_cell_size, k_vals, TC_symmetry=False):
        """QuantumModel.set_momentum_sector (edlgt/models/quantum_model.py:213-276):
        the projector B of the momentum sector k_vals (labels in units of
        2 pi / R_d, R_d = L_d / unit cell d), built on the device.  The
        Hamiltonian is then diagonalised as B^dagger H B."""
        from ..momentum import MomentumBasis

        if self.sector is None:
            raise ValueError("symmetry sector_configs not defined yet")
        if self.has_obc[0]:
            raise ValueError("Momentum is not conserved with OBC.")
        k_vals = np.atleast_1d(np.asarray(k_vals, dtype=np.int32))
        if k_vals.size != self.dim:
            raise ValueError(f"expected k_vals shape {self.dim}, got {k_vals.shape}")
        tc = {}
        if TC_symmetry:
            # translation combined with the charge-conjugation map of the
            # six-state SU(2) j=1/2 dressed site and its state signs, the
            # fixed tables of momentum_basis_zero_k_TC / _finite_k_TC
            # (edlgt/symmetries/translational_sym.py:995-997, 1161-1163)
            if self.dim != 1 or np.any(np.asarray(self.loc_dims) != 6):
                raise ValueError("the TC momentum basis is defined for 1D chains of six-state dressed sites")
            tc = dict(local_map=np.array([4, 5, 2, 3, 0, 1], dtype=np.int32),
                      label_sign=np.array([1.0, 1.0, 1.0, -1.0, 1.0, 1.0]))
            k_unit_cell_size = [1]
        self._momentum = MomentumBasis(self.sector, self.lvals, k_unit_cell_size, k_vals, **tc)
        self.momentum_basis = self._momentum.host_arrays()

    @staticmethod
    def _normalize_dtype_mode(dtype_mode, allow_auto=True):
        """bool / None / "real" / "complex" / "auto" -> a mode string
        (QuantumModel._normalize_dtype_mode, quantum_model.py:1342-1371)."""
        if isinstance(dtype_mode, (bool, np.bool_)):
            return "complex" if bool(dtype_mode) else "real"
        if dtype_mode is None:
            if allow_auto:
                return "auto"
            raise ValueError("dtype_mode cannot be None in this context")
        if not isinstance(dtype_mode, str):
            raise TypeError(f"dtype_mode must be bool/str/None, got {type(dtype_mode)}")
        mode = dtype_mode.strip().lower()
        valid = {"real", "complex", "auto"} if allow_auto else {"real", "complex"}
        if mode not in valid:
            raise ValueError(f"dtype_mode must be one of {sorted(valid)}, got {dtype_mode!r}")
        return mode

    def configure_dtype_mode(self, dtype_mode="auto", auto_mode="complex"):
        """The model's value type for later builds (quantum_model.py:1373-1408).
        On the device a matrix whose phases can be gauged away is stored in
        real form whatever the mode (its spectrum and the states mapped back
        are those of the complex matrix); "complex" stores it complex."""
        mode = self._normalize_dtype_mode(dtype_mode, allow_auto=True)
        if mode == "auto":
            mode = self._normalize_dtype_mode(auto_mode, allow_auto=False)
        self.dtype_mode = mode
        return mode

    def _resolve_dtype_mode(self, dtype_mode):
        mode = self._normalize_dtype_mode(dtype_mode, allow_auto=True)
        return self.dtype_mode if mode == "auto" else mode

    def set_momentum_pair(self, k_left, k_right, k_unit_cell_size, TC_symmetry=False):
        """Two momentum sectors at once (QuantumModel.set_momentum_pair,
        edlgt/models/quantum_model.py:278-348): the CSC arrays of B_left and the
        CSR arrays of B_right, for operators projected as B_left^dagger O
        B_right."""
        self.set_momentum_sector(k_unit_cell_size, k_left, TC_symmetry)
        left = self.momentum_basis
        self.set_momentum_sector(k_unit_cell_size, k_right, TC_symmetry)
        right = self.momentum_basis
        self._momentum = None  # pair mode projects operators, it has no single sector to diagonalise
        self.momentum_basis = {
            "pair_mode": True, "n_rows_full": len(self.sector), "n_cols_L": left["n_cols"],
            "n_cols_R": int(right["R_col_idx"].max()) + 1 if len(right["R_col_idx"]) else 0,
            "L_col_ptr": left["L_col_ptr"], "L_row_idx": left["L_row_idx"], "L_data": left["L_data"],
            "R_row_ptr": right["R_row_ptr"], "R_col_idx": right["R_col_idx"], "R_data": right["R_data"],
            "k_left": np.asarray(k_left, dtype=np.int32), "k_right": np.asarray(k_right, dtype=np.int32)}

    def _momentum_matrices(self):
        from scipy.sparse import csc_matrix, csr_matrix

        mb = self.momentum_basis
        if mb is None:
            raise ValueError("Basis projector B is not set.")
        if mb.get("pair_mode"):
            n = mb["n_rows_full"]
            left = csc_matrix((mb["L_data"], mb["L_row_idx"], mb["L_col_ptr"]), shape=(n, mb["n_cols_L"]))
            right = csr_matrix((mb["R_data"], mb["R_col_idx"], mb["R_row_ptr"]), shape=(n, mb["n_cols_R"]))
            return left, right
        b = csr_matrix((mb["R_data"], mb["R_col_idx"], mb["R_row_ptr"]), shape=(mb["n_rows"], mb["n_cols"]))
        return b, b

    def check_momentum_pair(self):
        """Frobenius norms of B_L^dagger B_L - 1, B_R^dagger B_R - 1 and
        B_L^dagger B_R (quantum_model.py:350-398)."""
        from scipy.sparse import identity
        from scipy.sparse.linalg import norm

        left, right = self._momentum_matrices()
        out = (float(norm(left.conj().T @ left - identity(left.shape[1]))),
               float(norm(right.conj().T @ right - identity(right.shape[1]))),
               float(norm(left.conj().T @ right)))
        logger.info(f"norms: {out}")
        return out

    def _original_basis_scipy(self):
        """The sector Hamiltonian as a host scipy matrix in the reference basis."""
        h = self.H.to_scipy()
        ph = self.H._row_phase()
        if ph is None:
            return h
        from scipy.sparse import diags

        p = diags(ph.cpu().numpy())
        return (p @ h @ p.conj()).tocsr()

    def momentum_basis_projection(self, operator):
        """B^dagger A B (B_L^dagger A B_R in pair mode) for a dense or sparse
        sector operator, or for "H", stored in ``H.Ham``
        (quantum_model.py:680-713)."""
        from scipy.sparse import csr_matrix, isspmatrix

        left, right = self._momentum_matrices()
        a = self._original_basis_scipy() if isinstance(operator, str) and operator == "H" else operator
        if not isspmatrix(a):
            a = csr_matrix(a)
        proj = (left.conj().T @ (a.tocsr() @ right)).tocsr()
        if isinstance(operator, str) and operator == "H":
            self.H.Ham = proj
            return None
        return proj

    def _project_state_with_basis(self, state_realspace):
        """psi_k = B^dagger psi (quantum_model.py:654-678), on the device
        (``edg_momentum_reduce``) when a single momentum sector is set."""
        mom = self._momentum
        if self.momentum_basis is None:
            return np.asarray(state_realspace).astype(np.complex128, copy=False)
        if mom is None:
            left, _ = self._momentum_matrices()
            return left.conj().T @ np.asarray(state_realspace, dtype=np.complex128)
        x = torch.from_numpy(np.ascontiguousarray(state_realspace, dtype=np.complex128)).to(self.device)
        y = torch.empty(mom.n_cols, dtype=torch.complex128, device=self.device)
        check(lib.edg_momentum_reduce(mom.n_cols, ptr(mom.col_ptr), ptr(mom.row_idx), ptr(mom.data), ptr(x), ptr(y),
                                      stream_handle()), "edg_momentum_reduce")
        return y.cpu().numpy()

    def build_projector_from_sector_to_fullspace(self, indices):
        """Sparse (prod loc_dims[indices], subsys_dim) map from the subsystem's
        sector configurations to the product basis (quantum_model.py:793-824)."""
        from scipy.sparse import csc_matrix

        cfg = self._get_partition(indices)["unique_subsys_configs"]
        dims = np.asarray(self.loc_dims)[sorted(int(i) for i in indices)].astype(np.int64)
        rows = np.zeros(cfg.shape[0], dtype=np.int64)
        for k, d in enumerate(dims):
            rows = rows * d + cfg[:, k].astype(np.int64)
        return csc_matrix((np.ones(cfg.shape[0]), (rows, np.arange(cfg.shape[0]))),
                          shape=(int(np.prod(dims)), cfg.shape[0]))

    def diagonalize_Hamiltonian(self, n_eigs, format="gpu", print_results=False, precision="fp64", tol=1e-12):
        mom = getattr(self, "_momentum", None)
        if mom is not None:
            if self.H.mat is None:
                self.H.build(format)
            mom.bind(self.H)
            k = mom.n_cols if (isinstance(n_eigs, str) and n_eigs == "full") else int(n_eigs)
            evals, vecs = mom.lowest(k, tol=tol)
            self.H.n_eigs = k
            self.H.Nenergies = np.asarray(evals) / self.n_sites
            self.H.Npsi = [QMB_state(vecs[:, i].contiguous(), self.lvals, self.loc_dims) for i in range(k)]
            self.H.GSenergy = self.H.Nenergies[0]
            self.H.GSpsi = self.H.Npsi[0]
        else:
            self.H.diagonalize(n_eigs, format, self.loc_dims, print_results, tol=tol, precision=precision)
        self.n_eigs = self.H.n_eigs
        self.res["energy"] = self.H.Nenergies

    def time_evolution_Hamiltonian(self, initial_state, time_line, **kwargs):
        mom = getattr(self, "_momentum", None)
        if mom is not None:
            from ..momentum import krylov_evolve

            if self.H.mat is None:
                self.H.build()
            mom.bind(self.H)
            psi0 = initial_state if isinstance(initial_state, torch.Tensor) else torch.from_numpy(
                np.asarray(initial_state, dtype=np.complex128))
            if psi0.shape[0] != mom.n_cols:
                raise ValueError(f"the initial state must live in the momentum sector ({mom.n_cols} states)")
            states = krylov_evolve(mom.matvec, psi0.to(self.device), np.asarray(time_line, dtype=np.float64),
                                   m_krylov=kwargs.get("m_krylov", 40), tol=kwargs.get("tol", 1e-12))
            self.H.psi_time = [QMB_state(x, self.lvals, self.loc_dims) for x in states]
            return
        self.H.time_evolution(initial_state, time_line, self.loc_dims, **kwargs)

    def get_qmb_state_from_configs(self, configs):
        idx = self.sector.index_of(np.asarray(configs).reshape(len(configs), -1))
        if np.any(idx < 0):
            raise ValueError("config not compatible with the symmetry sector")
        state = np.zeros(len(self.sector), dtype=np.complex128)
        state[idx] = complex(1 / np.sqrt(len(configs)), 0)
        return state

    # ------------------------------------------------------- observables
    def local_expval(self, op, psi) -> np.ndarray:
        """<psi| op_s |psi> for every site (diagonal of op, as LocalTerm)."""
        if isinstance(psi, QMB_state):
            psi = psi.device(self.device)
        elif not isinstance(psi, torch.Tensor):
            psi = torch.from_numpy(np.asarray(psi)).to(self.device)
        return site_expval_device(self.sector, op, psi).cpu().numpy()

    # ------------------------------------------------- full-spectrum ensembles
    def measure_fidelity(self, state, index, dynamics=False, print_value=False):
        """|<ref|state>|^2 with ref = Npsi[index] or psi_time[index]
        (edlgt/models/quantum_model.py:864-898)."""
        state = np.asarray(state)
        if len(state) != self.H.shape[0]:
            raise ValueError(f"len(state) must be {self.H.shape[0]} not {len(state)}")
        ref = self.H.Npsi[index].psi if not dynamics else self.H.psi_time[index].psi
        fid = float(np.abs(state.conj().dot(ref)) ** 2)
        if print_value:
            logger.info(f"FIDELITY: {fid}")
        return fid

    def compute_expH(self, beta):
        """exp(-beta H) (dense, host; quantum_model.py:904-906), from the
        eigen-system of the sector matrix (the stored full spectrum, or one
        dense eigen-solve on the device)."""
        v, e = self._thermal_spectrum()
        w = torch.exp(-beta * torch.from_numpy(e).to(v.device))
        return ((v * w[None, :]) @ v.conj().T).cpu().numpy()

    def get_thermal_beta(self, state, threshold):
        return self.H.get_beta(state, threshold)

    def _thermal_spectrum(self):
        """(eigenvectors in the reference basis, total eigenvalues) for
        traces of exp(-beta H), whether or not all eigenpairs were asked for."""
        if self.H._full():
            return self.H._evecs, self.H._evals_total
        w, v, _ = self.H._thermal_system(vectors=True)
        return v, w

    def _full_spectrum(self):
        if not self.H._full():
            raise ValueError(f"Need all H eigvals {self.H.shape[0]}, not only {getattr(self, 'n_eigs', None)}")
        return self.H._evecs, self.H._evals_total

    def _eig_site_obs(self, name, v=None):
        """(n_eigs, n_sites) array of <E_i| op_s |E_i> for a diagonal local
        operator, for all eigenstates at once: |V|^2 (rows x states)
        contracted with the per-row site values."""
        if v is None:
            v, _ = self._full_spectrum()
        op = self.ops[name]
        diag = torch.from_numpy(np.real(np.array([np.diagonal(op[s]) for s in range(op.shape[0])]))
                                .astype(np.float64)).to(v.device)
        cfg = torch.from_numpy(self.sector_configs.astype(np.int64)).to(v.device)
        site = torch.arange(self.n_sites, device=v.device)[None, :]
        d_rows = diag[site, cfg]
        p = (v.conj() * v).real if v.is_complex() else v * v
        return (p.T @ d_rows).cpu().numpy()

    def _site_value(self, name, site_vals, special_norms, staggered_avgs):
        if special_norms.get(name) is not None:
            return float(np.dot(site_vals, special_norms[name]) / self.n_sites)
        if staggered_avgs.get(name) is not None:
            self.res[name] = site_vals
            return self.stag_avg(name, staggered_avgs[name])
        return float(np.mean(site_vals))

    def canonical_avg(self, local_obs, beta):
        """Tr(O exp(-beta H)) / (Z n_sites), O = sum_s op_s
        (edlgt/models/quantum_model.py:911-938), from the eigen-system of the
        sector matrix (the stored full spectrum, or one dense eigen-solve on
        the device)."""
        v, e = self._thermal_spectrum()
        w = np.exp(-beta * (e - e.min()))
        obs = self._eig_site_obs(local_obs, v).sum(axis=1)
        return float(np.dot(w, obs) / (np.sum(w) * self.n_sites))

    def microcanonical_avg(self, local_obs_list, state, special_norms=None, staggered_avgs=None):
        """Shell average over eigenstates with |e_i - e_q| < delta_e
        (edlgt/models/quantum_model.py:940-1045)."""
        special_norms = special_norms or {}
        staggered_avgs = staggered_avgs or {}
        v, _ = self._full_spectrum()
        Eq = self.H.energy_of(state)
        x = self.H.from_original_basis(torch.from_numpy(np.asarray(state, dtype=np.complex128)).to(v.device))
        hx = self.H._apply(x)
        E2q = float(torch.vdot(hx.to(torch.complex128), hx.to(torch.complex128)).real)
        delta_e = np.sqrt(E2q - Eq ** 2) / self.n_sites
        e_q = Eq / self.n_sites
        shell = np.nonzero(np.abs(self.H.Nenergies - e_q) < delta_e)[0]
        if len(shell) == 0:
            raise ValueError(f"ME shell empty: no eigstate |e_i-e_q|<delta_e={delta_e}.")
        idx = torch.from_numpy(shell).to(v.device)
        psi_thermal = (v[:, idx].to(torch.complex128).sum(dim=1) / np.sqrt(len(shell))).cpu().numpy()
        me = {}
        for name in local_obs_list:
            vals = self._eig_site_obs(name)[shell]
            me[f"ME_{name}"] = float(np.mean([self._site_value(name, row, special_norms, staggered_avgs)
                                              for row in vals]))
        return psi_thermal, me

    def diagonal_avg(self, local_obs_list, state, special_norms=None, staggered_avgs=None, tol_deg=1e-10):
        """Diagonal-ensemble averages with degenerate blocks
        (edlgt/models/quantum_model.py:1047-1156)."""
        special_norms = special_norms or {}
        staggered_avgs = staggered_avgs or {}
        v, _ = self._full_spectrum()
        E = np.real_if_close(np.asarray(self.H.Nenergies))
        block = np.zeros(len(E), dtype=np.int64)
        for kk in range(1, len(E)):
            block[kk] = block[kk - 1] + (0 if abs(E[kk] - E[kk - 1]) < tol_deg else 1)
        n_blocks = int(block[-1]) + 1
        st = torch.from_numpy(np.asarray(state, dtype=np.complex128)).to(v.device)
        coeffs = v.to(torch.complex128).conj().T @ st
        de = {f"DE_{name}": 0.0 for name in local_obs_list}
        if np.all(np.bincount(block, minlength=n_blocks) <= 1):
            prob = (coeffs.abs() ** 2).cpu().numpy()
            for name in local_obs_list:
                vals = self._eig_site_obs(name)
                de[f"DE_{name}"] = float(sum(prob[i] * self._site_value(name, vals[i], special_norms, staggered_avgs)
                                             for i in range(len(prob))))
            return de
        for b in range(n_blocks):
            idx = torch.from_numpy(np.nonzero(block == b)[0]).to(v.device)
            psi_b = v[:, idx].to(torch.complex128) @ coeffs[idx]
            if float(torch.vdot(psi_b, psi_b).real) < 1e-14:
                continue
            for name in local_obs_list:
                site_vals = self.local_expval(self.ops[name], psi_b)
                de[f"DE_{name}"] += self._site_value(name, site_vals, special_norms, staggered_avgs)
        return de

    def _get_partition(self, keep_indices):
        """QuantumModel._get_partition (edlgt/models/quantum_model.py:715-791):
        subsystem/environment maps and unique configurations, built on the
        device (``edg_part_map``) and cached per sorted site tuple."""
        from ..entanglement import get_partition

        key = tuple(sorted(int(i) for i in keep_indices))
        if key not in self._partition_cache:
            if self.sector is None:
                raise ValueError("_get_partition needs a symmetry sector")
            self._partition_cache[key] = get_partition(self.sector, self.n_sites, key)
        return self._partition_cache[key]

    def twobody_expval(self, op_a, op_b, psi) -> np.ndarray:
        """Correlator matrix Re <psi| A_i B_j |psi>, i != j (TwoBodyTerm.get_expval)."""
        if isinstance(psi, QMB_state):
            psi = psi.device(self.device)
        elif not isinstance(psi, torch.Tensor):
            psi = torch.from_numpy(np.asarray(psi)).to(self.device)
        return twobody_corr_device(self.sector, op_a, op_b, psi).cpu().numpy()

    def get_observables(self, local_obs=(), twobody_obs=(), plaquette_obs=(), nbody_obs=(), nbody_dist=(),
                        twobody_axes=None):
        self.local_obs = list(local_obs)
        self.twobody_obs = [list(x) for x in twobody_obs]
        self.twobody_axes = twobody_axes
        self.plaquette_obs = [list(x) for x in plaquette_obs]
        self.nbody_obs = [list(x) for x in nbody_obs]
        self.nbody_dist = [[tuple(d) for d in dl] for dl in nbody_dist]
        if len(self.nbody_dist) != len(self.nbody_obs):
            raise ValueError("nbody_dist needs one list of distances per n-body observable")
        self.obs_list = {}
        self._plaq_mats = {}
        for names in self.plaquette_obs:
            axes = [names[-1][3], names[-1][6]]
            term = PlaquetteTerm(axes, [self.ops[o] for o in names], names, **self.def_params)
            self.obs_list["_".join(names)] = term

    def _state(self, index, dynamics):
        return self.H.Npsi[index] if not dynamics else self.H.psi_time[index]

    def measure_observables(self, index, dynamics=False):
        st = self._state(index, dynamics)
        for obs in self.local_obs:
            self.res[obs] = self.local_expval(self.ops[obs], st)
        for names in self.twobody_obs:
            self.res["_".join(names)] = self.twobody_expval(self.ops[names[0]], self.ops[names[1]], st)
        for names in self.plaquette_obs:
            key = "_".join(names)
            self.res[key] = self.plaquette_avg(names, st)
        for names, dist in zip(self.nbody_obs, self.nbody_dist):
            self.res["_".join(names)] = self.nbody_expval(names, dist, st)

    def nbody_expval(self, names, distances, st, component="real"):
        """NBodyTerm.get_expval (edlgt/modeling/nbody_term.py:164-257): for every
        starting site whose pattern stays on the lattice, <psi| prod_j op_j |psi>
        (real or imaginary part), each instance assembled once on the device."""
        cache = self.__dict__.setdefault("_nb_mats", {})
        key = (tuple(names), tuple(tuple(d) for d in distances))
        if key not in cache:
            term = NBodyTerm([self.ops[o] for o in names], list(names), [list(d) for d in distances],
                             **self.def_params)
            mats = []
            for inst in term.get_Hamiltonian(1.0).sites:
                blk = term.get_Hamiltonian(1.0)
                blk.sites = np.array([inst])
                mats.append(assemble_blocks(self.sector, [blk], phase_weights=self.phase_weights, force_complex=True))
            cache[key] = mats
        psi = st.device(self.device) if isinstance(st, QMB_state) else st
        if not isinstance(psi, torch.Tensor):
            psi = torch.from_numpy(np.asarray(psi)).to(self.device)
        psi_c = psi.to(torch.complex128)
        vals = []
        for m in cache[key]:
            z = torch.vdot(psi_c, m.matvec(psi_c)).item()
            vals.append(z.real if component == "real" else z.imag)
        return np.array(vals)

    def plaquette_avg(self, names, st, component="real"):
        """Average over plaquettes of <Re P> (PlaquetteTerm.get_expval)."""
        key = "_".join(names)
        psi = st.device(self.device) if isinstance(st, QMB_state) else st  # reference basis
        if key not in self._plaq_mats:
            term = self.obs_list[key]
            mats = []
            from ..lattice import plaquette_sites

            for ii in range(self.n_sites):
                sl = plaquette_sites(zig_zag(self.lvals, ii), self.lvals, term.axes, self.has_obc)
                if sl is None:
                    continue
                blk = term.get_Hamiltonian(1.0, add_dagger=False)
                blk.sites = np.array([sl])
                mats.append(assemble_blocks(self.sector, [blk], phase_weights=self.phase_weights, force_complex=True))
            self._plaq_mats[key] = mats
        vals = []
        psi_c = psi.to(torch.complex128)
        for m in self._plaq_mats[key]:
            y = m.matvec(psi_c)
            z = torch.vdot(psi_c, y).item()
            vals.append(z.real if component == "real" else z.imag)
        return float(np.mean(vals))

    def link_avg(self, obs_name):
        avg, cnt = 0.0, 0
        for ii in range(self.n_sites):
            coords = zig_zag(self.lvals, ii)
            for d in self.directions:
                if neighbor_sites(coords, self.lvals, d, self.has_obc) is not None:
                    avg += self.res[f"{obs_name}_p{d}"][ii]
                    cnt += 1
        return avg / cnt

    def stag_avg(self, obs_name, staggered_avg=None):
        values = np.asarray(self.res[obs_name])
        if staggered_avg is None:
            return float(np.mean(values))
        mask2d = staggered_mask(self.lvals, staggered_avg)
        mask1d = np.array([mask2d[zig_zag(self.lvals, s)] for s in range(self.n_sites)])
        return float(np.mean(values[mask1d]))
