"""Hamiltonian term builders.

Mirrors ``edlgt.modeling`` (``LocalTerm`` local_term.py:25-117, ``TwoBodyTerm``
twobody_term.py:26-158, ``PlaquetteTerm`` plaquette_term.py:25-163,
``NBodyTerm`` nbody_term.py:66-162): the same constructor arguments and the
same site loops (linear site order, OBC/PBC geometry, masks), but
``get_Hamiltonian`` returns a :class:`TermBlock` -- the list of operator
instances with their coupling -- instead of host triplets.  The device
assembler turns all blocks of a Hamiltonian into one canonical matrix.
"""

from __future__ import annotations

import logging
from math import prod

import numpy as np

from ..lattice import neighbor_sites, plaquette_sites, zig_zag

__all__ = ["TermBlock", "LocalTerm", "TwoBodyTerm", "PlaquetteTerm", "NBodyTerm"]

logger = logging.getLogger(__name__)


class TermBlock:
    """Operator instances of one ``get_Hamiltonian`` call.

    ``ops``: list of ``(n_sites, d, d)`` site-resolved operator tensors, one per
    factor; ``sites``: ``(n_inst, n_ops)`` site tuples; ``strength``: scalar
    coupling; ``add_dagger``: add the Hermitian conjugate of every instance;
    ``diagonal``: single-factor term of which only the diagonal is used (as
    ``localbody_data_par`` does).
    """

    def __init__(self, ops, sites, strength, add_dagger=False, diagonal=False, name=""):
        self.ops = [np.asarray(o) for o in ops]
        self.sites = np.asarray(sites, dtype=np.int64).reshape(-1, len(self.ops))
        self.strength = complex(strength)
        self.add_dagger = bool(add_dagger)
        self.diagonal = bool(diagonal)
        self.name = name

    @property
    def n_instances(self):
        return self.sites.shape[0]


class QMBTerm:
    def __init__(self, lvals, has_obc, operator=None, op_name=None, op_list=None, op_names_list=None,
                 sector_configs=None, loc_dims=None, staggered_basis=False, gauge_basis=None, momentum_basis=None,
                 sector=None, phase_weights=None, **_):
        self.lvals = list(lvals)
        self.dimensions = "xyz"[: len(lvals)]
        self.has_obc = list(has_obc)
        self.loc_dims = loc_dims
        self.staggered_basis = staggered_basis
        self.gauge_basis = gauge_basis
        self.op = operator
        self.op_name = op_name
        self.op_list = op_list
        self.op_names_list = op_names_list
        self.sector_configs = sector_configs
        # a momentum sector is applied to the assembled sector matrix when the
        # Hamiltonian is diagonalised, so the terms themselves stay in the sector
        self.momentum_basis = momentum_basis
        self.sector = sector
        self.phase_weights = phase_weights
        self.n_sites = prod(self.lvals)

    def _mask_ok(self, coords, mask):
        return mask is None or bool(np.asarray(mask)[tuple(coords)])

    def get_staggered_conditions(self, coords, stag_label):
        """even / odd sublattice selection by (-1)^sum(coords) (qmb_term.py:105-127)."""
        stag = (-1) ** int(sum(coords))
        return stag_label is None or (stag_label == "even" and stag > 0) or (stag_label == "odd" and stag < 0)

    def get_mask_conditions(self, coords, mask):
        return self._mask_ok(coords, mask)

    def _device_psi(self, psi):
        import torch

        from .hamiltonian import QMB_state

        if self.sector is None:
            raise ValueError("expectation values need the model's symmetry sector (build the term from def_params)")
        if not isinstance(psi, QMB_state):
            raise TypeError(f"psi must be instance of class:QMB_state not {type(psi)}")
        x = psi.device(self.sector.device)
        if x.shape[0] != len(self.sector):
            raise ValueError("the state does not live in the sector basis (momentum-basis states are not supported)")
        return x if isinstance(x, torch.Tensor) else torch.from_numpy(np.asarray(x)).to(self.sector.device)

    def _instances_expval(self, blocks, psi, component):
        """<psi| O_inst |psi> for each single-instance block, assembled once."""
        import torch

        from .assembly import assemble_blocks

        if not hasattr(self, "_inst_mats"):
            self._inst_mats = [assemble_blocks(self.sector, [b], phase_weights=self.phase_weights, force_complex=True)
                               for b in blocks]
        x = self._device_psi(psi).to(torch.complex128)
        vals = []
        for m in self._inst_mats:
            z = torch.vdot(x, m.matvec(x)).item()
            vals.append(z.real if component == "real" else z.imag)
        return np.array(vals)

    def _split_instances(self, block):
        out = []
        for inst in block.sites:
            b = TermBlock(block.ops, np.array([inst]), 1.0, add_dagger=False, diagonal=block.diagonal, name=block.name)
            out.append(b)
        return out


class LocalTerm(QMBTerm):
    """Single-site (diagonal) term summed over the (masked) lattice sites."""

    def __init__(self, operator, op_name, **kwargs):
        super().__init__(operator=operator, op_name=op_name, **kwargs)

    def get_Hamiltonian(self, strength, mask=None):
        if not np.isscalar(strength):
            raise TypeError(f"strength must be SCALAR not a {type(strength)}")
        sites = [ii for ii in range(self.n_sites) if self._mask_ok(zig_zag(self.lvals, ii), mask)]
        return TermBlock([self.op], np.array(sites).reshape(-1, 1), strength, diagonal=True, name=self.op_name)

    def get_expval(self, psi, stag_label=None, print_values=True, get_variance=False):
        """Per-site <psi| op_s |psi> in ``self.obs`` and their average over the
        selected sublattice in ``self.avg`` (LocalTerm.get_expval,
        edlgt/modeling/local_term.py:119-237), one device reduction."""
        from ..models.quantum_model import site_expval_device

        x = self._device_psi(psi)
        self.obs = site_expval_device(self.sector, self.op, x).cpu().numpy()
        if get_variance:
            op2 = np.array([np.asarray(self.op[s]) @ np.asarray(self.op[s]) for s in range(self.op.shape[0])])
            self.var = site_expval_device(self.sector, op2, x).cpu().numpy() - self.obs ** 2
        sel = [ii for ii in range(self.n_sites) if self.get_staggered_conditions(zig_zag(self.lvals, ii), stag_label)]
        self.avg = float(np.mean(self.obs[sel]))
        self.std = float(np.sqrt(np.abs(np.sum(self.var[sel])) / len(sel))) if get_variance else 0.0
        if print_values:
            logger.info(f"{self.op_name} {self.avg:.16f}")


class TwoBodyTerm(QMBTerm):
    """Nearest-neighbour product ``op0[i] op1[i+axis]``."""

    def __init__(self, axis, op_list, op_names_list, **kwargs):
        super().__init__(op_list=op_list, op_names_list=op_names_list, **kwargs)
        if axis not in self.dimensions:
            raise ValueError(f"axis should be in {self.dimensions}: got {axis}")
        self.axis = axis

    def get_Hamiltonian(self, strength, add_dagger=False, mask=None):
        if not np.isscalar(strength):
            raise TypeError(f"strength must be SCALAR, not {type(strength)}")
        inst = []
        for ii in range(self.n_sites):
            coords = zig_zag(self.lvals, ii)
            sl = neighbor_sites(coords, self.lvals, self.axis, self.has_obc)
            if sl is None or not self._mask_ok(coords, mask):
                continue
            inst.append(sl)
        return TermBlock(self.op_list, np.array(inst).reshape(-1, 2), strength, add_dagger=add_dagger,
                         name="-".join(self.op_names_list or []))

    def get_expval(self, psi):
        """Correlator matrix Re <psi| A_i B_j |psi> over all pairs i < j in
        ``self.corr`` (TwoBodyTerm.get_expval, twobody_term.py:160-209)."""
        from ..models.quantum_model import twobody_corr_device

        self.corr = twobody_corr_device(self.sector, self.op_list[0], self.op_list[1],
                                        self._device_psi(psi)).cpu().numpy()


class PlaquetteTerm(QMBTerm):
    """Four-site plaquette product ``op0[o] op1[o+a] op2[o+b] op3[o+a+b]``."""

    def __init__(self, axes, op_list, op_names_list, print_plaq=True, **kwargs):
        super().__init__(op_list=op_list, op_names_list=op_names_list, **kwargs)
        self.axes = list(axes)
        self.print_plaq = print_plaq

    def get_Hamiltonian(self, strength, add_dagger=False, mask=None):
        if not np.isscalar(strength):
            raise TypeError(f"strength must be scalar, not {type(strength)}")
        inst = []
        for ii in range(self.n_sites):
            coords = zig_zag(self.lvals, ii)
            sl = plaquette_sites(coords, self.lvals, self.axes, self.has_obc)
            if sl is None or not self._mask_ok(coords, mask):
                continue
            inst.append(sl)
        return TermBlock(self.op_list, np.array(inst).reshape(-1, 4), strength, add_dagger=add_dagger,
                         name="-".join(self.op_names_list or []))

    def get_expval(self, psi, component="real", stag_label=None):
        """Per-plaquette <psi| P |psi> (real or imaginary part) in ``self.obs``,
        their mean in ``self.avg`` (PlaquetteTerm.get_expval,
        plaquette_term.py:165-263), plaquettes of the selected sublattice."""
        if component not in ("real", "imag"):
            raise ValueError(f"component must be 'real' or 'imag': got {component}")
        block = self.get_Hamiltonian(1.0)
        keep = [k for k, inst in enumerate(block.sites)
                if self.get_staggered_conditions(zig_zag(self.lvals, int(inst[0])), stag_label)]
        block.sites = block.sites[keep]
        self.obs = self._instances_expval(self._split_instances(block), psi, component)
        self.avg = float(np.mean(self.obs))


class NBodyTerm(QMBTerm):
    """Product of operators at fixed relative distances from each site.

    ``distances`` lists, for every factor after the first, the displacement
    vector from the first site (``edlgt/modeling/nbody_term.py:66-162``); sites
    outside an OBC lattice drop the instance, PBC wraps.
    """

    def __init__(self, op_list, op_names_list, distances, **kwargs):
        super().__init__(op_list=op_list, op_names_list=op_names_list, **kwargs)
        self.distances = [tuple(d) for d in distances]
        if len(self.distances) != len(op_list) - 1:
            raise ValueError("need one distance vector per factor after the first")

    def get_Hamiltonian(self, strength, add_dagger=False, mask=None):
        from ..lattice import inverse_zig_zag

        inst = []
        for ii in range(self.n_sites):
            coords = zig_zag(self.lvals, ii)
            if not self._mask_ok(coords, mask):
                continue
            sites = [ii]
            ok = True
            for dist in self.distances:
                c = list(coords)
                for ax, dd in enumerate(dist):
                    c[ax] += dd
                    if c[ax] < 0 or c[ax] >= self.lvals[ax]:
                        if self.has_obc[ax]:
                            ok = False
                            break
                        c[ax] %= self.lvals[ax]
                if not ok:
                    break
                sites.append(inverse_zig_zag(self.lvals, c))
            if ok:
                inst.append(sites)
        return TermBlock(self.op_list, np.array(inst).reshape(-1, len(self.op_list)), strength,
                         add_dagger=add_dagger, name="-".join(self.op_names_list or []))

    def get_expval(self, psi, component="real"):
        """<psi| prod_j op_j |psi> for every starting site whose pattern stays on
        the lattice, in ``self.obs`` (NBodyTerm.get_expval, nbody_term.py:164-220)."""
        self.obs = self._instances_expval(self._split_instances(self.get_Hamiltonian(1.0)), psi, component)
