"""``QMB_hamiltonian`` backed by the device engine.

Same surface as edlgt/modeling/qmb_hamiltonian.py:24-426: ``add_term``,
``build(format)``, ``diagonalize(n_eigs, format, loc_dims)``,
``time_evolution(initial_state, time_line, loc_dims)`` and the attributes
``shape``, ``Ham_type``, ``Nenergies`` (energy densities, ascending),
``Npsi`` (list of :class:`QMB_state`), ``GSenergy``, ``GSpsi``, ``psi_time``.
Terms are :class:`TermBlock` objects (or scipy/dense matrices that are
diagonal, e.g. identity shifts); the matrix lives on the device.
"""

from __future__ import annotations

import logging

import numpy as np
import torch

from .assembly import assemble_blocks
from .terms import TermBlock

logger = logging.getLogger(__name__)

__all__ = ["QMB_hamiltonian", "QMB_state"]


class QMB_state:
    """A state vector in the sector basis (host copy made on first access)."""

    def __init__(self, psi, lvals=None, loc_dims=None):
        self._psi_dev = psi if isinstance(psi, torch.Tensor) else None
        self._psi = None if isinstance(psi, torch.Tensor) else np.asarray(psi)
        self.lvals = lvals
        self.loc_dims = loc_dims

    @property
    def psi(self) -> np.ndarray:
        if self._psi is None:
            self._psi = self._psi_dev.detach().cpu().numpy()
        return self._psi

    def device(self, dev=None) -> torch.Tensor:
        if self._psi_dev is None:
            self._psi_dev = torch.from_numpy(np.ascontiguousarray(self._psi)).to(dev or "cuda")
        return self._psi_dev

    def get_norm(self):
        return float(np.sqrt(np.real(np.vdot(self.psi, self.psi))))

    def normalize(self, threshold=1e-14):
        """Divide by the norm when it differs from 1 by more than threshold;
        returns the norm (QMB_state.normalize, qmb_state.py:79-95)."""
        nrm = self.get_norm()
        if abs(nrm - 1) > threshold:
            if self._psi_dev is not None:
                self._psi_dev = self._psi_dev / nrm
                self._psi = None
            else:
                self._psi = self._psi / nrm
        return nrm

    def truncate(self, threshold=1e-14):
        """The amplitudes with |psi_r| > threshold, zero elsewhere (a copy;
        QMB_state.truncate, qmb_state.py:97-110)."""
        psi = self.psi
        return np.where(np.abs(psi) > threshold, psi, 0)

    def expectation_value(self, operator, component="real"):
        """<psi| O |psi> for O given as (rows, cols, values) triplets or as a
        dense / scipy sparse matrix, real or imaginary part
        (QMB_state.expectation_value, edlgt/modeling/qmb_state.py:112-157)."""
        from scipy.sparse import csr_matrix, isspmatrix

        psi = self.psi
        if isinstance(operator, tuple) and len(operator) == 3:
            rows, cols, vals = (np.asarray(x) for x in operator)
            ev = np.sum(np.conj(psi[rows]) * vals * psi[cols])
        elif isinstance(operator, np.ndarray) or isspmatrix(operator):
            if operator.shape[0] != psi.shape[0]:
                raise ValueError(f"quantum state dim {psi.shape[0]} is NOT the operator dim {operator.shape[0]}")
            op = csr_matrix(operator) if isinstance(operator, np.ndarray) else operator
            ev = np.vdot(psi, op.dot(psi))
        else:
            raise TypeError("Operator must be provided as a tuple (row_list, col_list, value_list), "
                            "a dense matrix (np.ndarray), or a sparse matrix (scipy sparse matrix).")
        if component == "real":
            return float(np.real(ev))
        if component == "imag":
            return float(np.imag(ev))
        raise ValueError(f"Unknown component='{component}'")

    def get_state_configurations(self, threshold=1e-2, sector_configs=None, return_configs=False):
        """Configurations with |psi|^2 above ``threshold`` (relaxed tenfold until
        one qualifies), largest first (qmb_state.py:293-354)."""
        psi = self.psi
        prob = np.abs(psi) ** 2
        thr = float(threshold)
        idx = np.nonzero(prob > thr)[0]
        while idx.size == 0:
            thr /= 10
            idx = np.nonzero(prob > thr)[0]
        vals = psi[idx]
        order = np.argsort(-np.abs(vals))
        idx, vals = idx[order], vals[order]
        if sector_configs is not None:
            cfgs = np.asarray(sector_configs)[idx, :]
        else:
            if self.loc_dims is None:
                raise ValueError("sector_configs or loc_dims are needed to decode the configurations")
            dims = np.asarray(self.loc_dims, dtype=np.int64)
            cfgs = np.empty((len(idx), len(dims)), dtype=np.uint8)
            rem = idx.astype(np.int64)
            for s in range(len(dims) - 1, -1, -1):
                cfgs[:, s] = rem % dims[s]
                rem //= dims[s]
        for config, amp in zip(cfgs, vals):
            coords = " ".join(f"{c:>3d}" for c in config)
            logger.info(f"[{coords}] |psi|^2={abs(amp) ** 2:6f} ({amp:6f})")
        if return_configs:
            return cfgs, vals

    def participation_renyi_entropy(self, alpha=2):
        """PE_alpha = log(sum_r |psi_r|^(2 alpha) + 1e-16) / (1 - alpha)
        (qmb_state.py:356-391)."""
        if alpha <= 0 or alpha == 1:
            raise ValueError(f"alpha must be > 0 and != 1. Got alpha={alpha}.")
        prob = np.abs(self.psi) ** 2
        return float(1.0 / (1.0 - float(alpha)) * np.log(np.sum(prob ** alpha) + 1e-16))

    def _psi_for(self, keep_indices, partitions_dict):
        from ..entanglement import _record

        return self.device(_record(keep_indices, partitions_dict)["subsys_map_dev"].device)

    def reduced_density_matrix(self, keep_indices, partitions_dict) -> np.ndarray:
        """QMB_state.reduced_density_matrix (edlgt/modeling/qmb_state.py:211-243)
        for a partition made by ``QuantumModel._get_partition``."""
        from ..entanglement import reduced_density_matrix

        return reduced_density_matrix(self._psi_for(keep_indices, partitions_dict), keep_indices, partitions_dict)

    def entanglement_entropy(self, keep_indices, partitions_dict) -> float:
        """QMB_state.entanglement_entropy (edlgt/modeling/qmb_state.py:245-291),
        in bits, from the exact spectrum of the reduced density matrix."""
        from ..entanglement import entanglement_entropy

        return entanglement_entropy(self._psi_for(keep_indices, partitions_dict), keep_indices, partitions_dict)


class QMB_hamiltonian:
    def __init__(self, lvals, size, sector=None, phase_weights=None):
        self.lvals = list(lvals)
        self.shape = (int(size), int(size))
        self.sector = sector
        self.phase_weights = phase_weights
        self.blocks: list[TermBlock] = []
        self.extra_diag = 0.0
        self.mat = None
        self.Ham_type = None

    # ------------------------------------------------------------------ terms
    def add_term(self, term):
        if isinstance(term, TermBlock):
            self.blocks.append(term)
            self.mat = None
            return
        from scipy.sparse import issparse

        m = term
        if issparse(m) or isinstance(m, np.ndarray):
            mm = m.tocoo() if issparse(m) else None
            if mm is not None:
                off = mm.row != mm.col
                if np.any(np.abs(mm.data[off]) > 0):
                    raise TypeError("only diagonal matrix terms are accepted besides term blocks")
                d = np.zeros(self.shape[0], dtype=complex)
                np.add.at(d, mm.row[~off], mm.data[~off])
            else:
                if np.any(m - np.diag(np.diagonal(m))):
                    raise TypeError("only diagonal matrix terms are accepted besides term blocks")
                d = np.diagonal(m)
            if not np.allclose(d, d[0]):
                raise TypeError("only constant diagonal (identity) matrix terms are accepted")
            self.extra_diag += complex(d[0])
            self.mat = None
            return
        raise TypeError("Unsupported term type: expected a TermBlock or a diagonal matrix")

    # ------------------------------------------------------------------ build
    def build(self, format="gpu", force_complex=False):
        if self.sector is None:
            raise ValueError("the device Hamiltonian needs a symmetry sector")
        if format not in ("gpu", "sparse", "linear", "dense"):
            raise ValueError(f"format must be 'gpu' (or the aliases 'sparse'/'linear'), or 'dense', got {format}")
        ed = self.extra_diag
        self.mat = assemble_blocks(self.sector, self.blocks, phase_weights=self.phase_weights,
                                   force_complex=force_complex, extra_diag=ed if ed != 0 else None)
        self.Ham_type = "gpu"
        # spectra of an earlier matrix no longer apply
        self._evecs = None
        self._evals_total = None
        self._thermal = None
        logger.info(f"SPARSITY: {(self.mat.nnz + self.shape[0]) / self.shape[0] ** 2:.3e}")

    def to_scipy(self):
        if self.mat is None:
            self.build()
        return self.mat.to_scipy()

    # -------------------------------------------------------------- phases
    def _row_phase(self):
        """i**e(row) of the real form's gauge transform (None if not used)."""
        w = self.mat.phase_weights if self.mat is not None else None
        if w is None:
            return None
        cfg = torch.from_numpy(self.sector.configs.astype(np.int64)).to(self.sector.device)
        wt = torch.from_numpy(np.asarray(w, dtype=np.int64)).to(self.sector.device)
        e = wt[torch.arange(cfg.shape[1], device=cfg.device)[None, :], cfg].sum(dim=1) % 4
        table = torch.tensor([1, 1j, -1, -1j], dtype=torch.complex128, device=cfg.device)
        return table[e]

    def to_original_basis(self, psi: torch.Tensor) -> torch.Tensor:
        """Map a real-form vector back to the reference (complex) basis."""
        ph = self._row_phase()
        if ph is None:
            return psi
        return ph * psi.to(torch.complex128)

    def from_original_basis(self, psi: torch.Tensor) -> torch.Tensor:
        ph = self._row_phase()
        if ph is None:
            return psi
        return torch.conj(ph) * psi.to(torch.complex128)

    # -------------------------------------------------------- diagonalize
    def diagonalize(self, n_eigs, format="gpu", loc_dims=None, print_results=False, tol=1e-12, precision="fp64",
                    max_iter=None):
        from ..solvers import lanczos, lanczos_mixed

        if self.mat is None:
            self.build(format)
        n = self.shape[0]
        if isinstance(n_eigs, str) and n_eigs == "full":
            k = n
        elif isinstance(n_eigs, int):
            if n_eigs > n:
                raise ValueError(f"n_eigs must be < H.shape[0]={n}, got {n_eigs}")
            k = n_eigs
        else:
            raise ValueError(f"n_eigs must be int or 'full', not {n_eigs}.")
        self.loc_dims = loc_dims
        self.n_eigs = k
        if format == "dense" or (isinstance(n_eigs, str) and n_eigs == "full"):
            self._diagonalize_dense(k, loc_dims, print_results)
            return
        if k > 16:
            raise NotImplementedError("the device Lanczos returns at most 16 eigenpairs")
        if max_iter is None:
            max_iter = min(n, 600)
        if precision == "mixed":
            r64, _ = lanczos_mixed(self.mat, k=k, tol=tol, max_iter=max_iter)
            evals = r64.evals[0][:1]
            vecs = r64.evecs[:, :, 0].T
            if k > 1:
                raise NotImplementedError("mixed precision refines the ground state only")
        else:
            evals, vecs, _ = lanczos(self.mat, k=k, tol=tol, max_iter=max_iter)
        n_sites = int(np.prod(self.lvals))
        if print_results:
            for e in evals:
                logger.info(f"{e:.10f}  {e / n_sites:.10f}")
        self.Nenergies = np.asarray(evals) / n_sites
        self.Npsi = [QMB_state(self.to_original_basis(vecs[:, i]), self.lvals, loc_dims) for i in range(k)]
        self.GSenergy = self.Nenergies[0]
        self.GSpsi = self.Npsi[0]

    def convert_hamiltonian(self, format):
        """Select the representation used by diagonalize / time_evolution:
        "dense" (full diagonalisation, exact evolution) or the device sparse
        matrix ("gpu", alias "sparse" / "linear") (qmb_hamiltonian.py:227-258)."""
        if format not in ("gpu", "sparse", "linear", "dense"):
            raise ValueError(f"Invalid format: {format}. Use 'dense', 'sparse', 'linear' or 'gpu'.")
        if self.mat is None:
            self.build(format)
        self.Ham_type = "dense" if format == "dense" else "gpu"

    def get_sparsity(self):
        """Stored entries over shape[0]^2 (qmb_hamiltonian.py:614-618)."""
        if self.mat is None:
            self.build()
        pres = int(self.mat.diag_present.sum().item()) if self.mat.diag_present is not None else self.shape[0]
        sparsity = (self.mat.nnz + pres) / float(self.shape[0]) ** 2
        logger.info(f"SPARSITY: {round(sparsity, 16)}")
        return sparsity

    def print_energy(self, en_state):
        logger.info("====================================================")
        logger.info(f"{en_state} ENERGY: {round(float(self.Nenergies[en_state]), 16)}")

    # ------------------------------------------------------ full spectrum
    DENSE_MAX = 32768

    def _diagonalize_dense(self, k, loc_dims, print_results):
        """All eigenpairs of the dense sector matrix (array_eigh after
        convert_hamiltonian("dense"), qmb_hamiltonian.py:227-258, 300-302):
        the matrix is densified on the device (``edg_csr_to_dense``) and
        diagonalised by the library Hermitian solver."""
        dense = self._densify()
        w, v = torch.linalg.eigh(dense)
        del dense
        ph = self._row_phase()
        if ph is not None:
            v = ph[:, None] * v.to(torch.complex128)
        self._evecs = v
        self._evals_total = w.cpu().numpy()
        n_sites = int(np.prod(self.lvals))
        if print_results:
            for e in self._evals_total[:k]:
                logger.info(f"{e:.10f}  {e / n_sites:.10f}")
        # as the reference's dense branch: every energy density, the first k states
        self.Nenergies = self._evals_total / n_sites
        self.Npsi = [QMB_state(v[:, i], self.lvals, loc_dims) for i in range(k)]
        self.GSenergy = self.Nenergies[0]
        self.GSpsi = self.Npsi[0]
        self.Ham_type = "dense"

    def _densify(self, original_basis=False):
        """The sector matrix as a dense device array (``edg_csr_to_dense``), in
        the assembled (possibly real) form, or with the real form's phases put
        back: H = D H' D^dagger, the reference's basis."""
        from .._lib import check, lib, ptr, stream_handle

        n = self.shape[0]
        if n > self.DENSE_MAX:
            raise ValueError(f"dense matrices limited to {self.DENSE_MAX} states, the sector has {n}")
        if self.mat is None:
            self.build()
        mat = self.mat
        dt = torch.complex128 if mat.is_complex else torch.float64
        dense = torch.empty((n, n), dtype=dt, device=self.sector.device)
        flag = torch.empty(1, dtype=torch.int32, device=self.sector.device)
        check(lib.edg_csr_to_dense(2 if mat.is_complex else 0, n, ptr(mat.rowptr), ptr(mat.cols) if mat.nnz else None,
                                   ptr(mat.vals) if mat.nnz else None, ptr(mat.diag), ptr(dense), ptr(flag),
                                   stream_handle()), "edg_csr_to_dense")
        if original_basis:
            ph = self._row_phase()
            if ph is not None:
                dense = ph[:, None] * dense.to(torch.complex128) * ph.conj()[None, :]
        return dense

    def _full(self):
        return getattr(self, "_evecs", None) is not None and self.n_eigs == self.shape[0]

    def _thermal_system(self, vectors=False, square=False):
        """Eigen-system behind the traces of exp(-beta H) that the reference
        takes of the sparse matrix exponential when fewer than all eigenpairs
        were computed (qmb_hamiltonian.py:446-452, 486-489, 505-508, 545-551;
        quantum_model.py:904-938): Tr f(H) exp(-beta H) is a sum over the
        eigenvalues.  Returns (total eigenvalues (host), eigenvectors in the
        reference basis (device) or None, per-eigenstate weights
        v^dagger (H o H) v of the elementwise-squared matrix or None).

        Uses the stored spectrum when every eigenvalue is there (the dense
        format); otherwise the densified matrix is diagonalised once on the
        device by the library Hermitian solver and kept until the matrix
        changes."""
        n = self.shape[0]
        c = getattr(self, "_thermal", None)
        if c is None or c["mat"] is not self.mat:
            c = {"mat": self.mat, "w": None, "v": None, "sq": None}
            self._thermal = c
        ev = getattr(self, "_evals_total", None)
        if c["w"] is None and getattr(self, "_evecs", None) is not None and ev is not None and len(ev) == n:
            c["w"], c["v"] = np.asarray(ev), self._evecs
        need_v = vectors or square
        if c["w"] is None or (need_v and c["v"] is None):
            dense = self._densify(original_basis=True)
            if need_v:
                w, v = torch.linalg.eigh(dense)
                c["v"] = v
            else:
                w = torch.linalg.eigvalsh(dense)
            c["w"] = w.cpu().numpy()
            del dense
        if square and c["sq"] is None:
            h = self._densify(original_basis=True)
            v = c["v"]
            if h.is_complex() or v.is_complex():
                h, v = h.to(torch.complex128), v.to(torch.complex128)
            g = (h * h) @ v
            c["sq"] = torch.sum(v.conj() * g, dim=0).real.cpu().numpy()
            del h, g
        return c["w"], c["v"], c["sq"]

    def _h2_weights(self):
        """Per-eigenstate weights of the Tr(H^2 exp(-beta H)) term: lambda^2
        for the sparse formats (the reference's csc matrix power), and
        v^dagger (H o H) v for the dense format (its dense array is squared
        elementwise, qmb_hamiltonian.py:505-508)."""
        if self.Ham_type == "dense":
            return self._thermal_system(square=True)[2]
        w = self._thermal_system()[0]
        return w * w

    def energy_of(self, state):
        """<state| H |state> (total energy) for a vector in the original basis."""
        x = state if isinstance(state, torch.Tensor) else torch.from_numpy(np.asarray(state, dtype=np.complex128))
        x = self.from_original_basis(x.to(self.sector.device))
        hx = self._apply(x)
        return float(torch.vdot(x.to(torch.complex128), hx.to(torch.complex128)).real)

    def _apply(self, x):
        if self.mat.is_complex or not x.is_complex():
            return self.mat.matvec(x)
        return torch.complex(self.mat.matvec(x.real.contiguous()), self.mat.matvec(x.imag.contiguous()))

    def partition_function(self, beta):
        """QMB_hamiltonian.partition_function (qmb_hamiltonian.py:428-452):
        with the full spectrum, the sum over the stored energy densities;
        otherwise Tr exp(-beta H) of the sector matrix (the reference's sparse
        expm branch), summed over its eigenvalues."""
        if self._full():
            Z = float(np.sum(np.exp(-beta * self.Nenergies)))
        else:
            w = self._thermal_system()[0]
            Z = float(np.sum(np.exp(-beta * w)))
        if Z <= 0:
            raise ValueError(f"Z must be positive, not {Z}.")
        return Z

    def free_energy(self, beta):
        return -1 / beta * np.log(self.partition_function(beta))

    def thermal_average(self, beta):
        """Energy density average (full spectrum) or Tr(H exp(-beta H)) / Z
        (qmb_hamiltonian.py:471-489)."""
        Z = self.partition_function(beta)
        if self._full():
            return float(self.Nenergies.dot(np.exp(-beta * self.Nenergies)) / Z)
        w = self._thermal_system()[0]
        return float(w.dot(np.exp(-beta * w)) / Z)

    def F_prime(self, beta):
        """-<H^2> - <H>^2 of qmb_hamiltonian.py:491-508, with the same two
        branches as partition_function."""
        Z = self.partition_function(beta)
        if self._full():
            exph2 = np.square(self.Nenergies).dot(np.exp(-beta * self.Nenergies)) / Z
        else:
            w = self._thermal_system()[0]
            exph2 = self._h2_weights().dot(np.exp(-beta * w)) / Z
        return float(-exph2 - self.thermal_average(beta) ** 2)

    def get_beta(self, state, threshold=1e-10, max_iter=1000):
        """Newton solve of QMB_hamiltonian.get_beta (qmb_hamiltonian.py:510-564)
        against the state's total energy <state|H|state>: with the full
        spectrum, on the energy densities (as the reference); otherwise on
        the traces of exp(-beta H) of the sector matrix."""
        e_state = self.energy_of(state)
        if self._full():
            E, H2 = self.Nenergies, np.square(self.Nenergies)
        else:
            E, H2 = self._thermal_system()[0], self._h2_weights()
        beta, accuracy, it = 1e-7, 1.0, 0
        while accuracy > threshold and it < max_iter:
            it += 1
            wgt = np.exp(-beta * E)
            Z = np.sum(wgt)
            Em = E.dot(wgt) / Z
            F = Em - e_state
            Fp = -H2.dot(wgt) / Z - Em ** 2
            prev = beta
            beta = beta - F / Fp
            accuracy = abs(beta - prev)
        if it >= max_iter:
            logger.warning("Maximum iterations reached without convergence.")
        return beta

    def get_r_value(self):
        """Adjacent-gap ratios of the full spectrum and their bulk mean
        (qmb_hamiltonian.py:566-601)."""
        if self.Ham_type != "dense" or not hasattr(self, "Nenergies"):
            raise ValueError("The Hamiltonian has to be fully diagonalized.")
        dE = np.diff(np.sort(self.Nenergies))
        r = np.minimum(dE[:-1], dE[1:]) / np.maximum(dE[:-1], dE[1:])
        lo, hi = int(0.1 * len(r)), int(0.9 * len(r))
        self.r_value = float(np.mean(r[lo:hi]))
        return r

    # ------------------------------------------------------- time evolution
    def _exact_time_evolution(self, initial_state, time_line, loc_dims):
        """exact_time_evolution (qmb_hamiltonian.py:791-835) on the device:
        psi(t) = V exp(-i E t) V^dagger psi0, all times as one product."""
        dev = self.sector.device
        v = self._evecs.to(torch.complex128)
        psi0 = initial_state if isinstance(initial_state, torch.Tensor) else torch.from_numpy(
            np.asarray(initial_state, dtype=np.complex128))
        psi0 = psi0.to(dev).to(torch.complex128)
        c = v.conj().T @ psi0
        e = torch.from_numpy(self._evals_total.astype(np.float64)).to(dev)
        t = torch.from_numpy(np.asarray(time_line, dtype=np.float64)).to(dev)
        coeff = torch.exp(-1j * e[:, None] * t[None, :]) * c[:, None]
        states = v @ coeff
        self.loc_dims = loc_dims
        self.psi_time = [QMB_state(states[:, j], self.lvals, loc_dims) for j in range(len(time_line))]

    def time_evolution(self, initial_state, time_line, loc_dims=None, m_krylov=30, precision="c128",
                       observables=None, reorth_passes=1):
        from ..dynamics import krylov_evolve

        if self.Ham_type == "dense" and self._full():
            return self._exact_time_evolution(initial_state, time_line, loc_dims)
        if self.mat is None:
            self.build()
        self.loc_dims = loc_dims
        psi0 = initial_state if isinstance(initial_state, torch.Tensor) else torch.from_numpy(
            np.asarray(initial_state, dtype=np.complex128)).to(self.sector.device)
        psi0 = self.from_original_basis(psi0)
        obs = None
        if observables is not None:
            obs = {name: (self.sector, op) for name, op in observables.items()}
        states = krylov_evolve(self.mat, psi0, np.asarray(time_line, dtype=float), m=m_krylov, precision=precision,
                               keep_states=observables is None, observables=obs, reorth_passes=reorth_passes)
        if observables is None:
            self.psi_time = [QMB_state(self.to_original_basis(s), self.lvals, loc_dims) for s in states]
        else:
            self.obs_time = states
