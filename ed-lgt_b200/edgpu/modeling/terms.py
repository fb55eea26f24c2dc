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

from math import prod

import numpy as np

from ..lattice import neighbor_sites, plaquette_sites, zig_zag

__all__ = ["TermBlock", "LocalTerm", "TwoBodyTerm", "PlaquetteTerm", "NBodyTerm"]


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
                 **_):
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
        self.momentum_basis = momentum_basis
        if momentum_basis is not None:
            raise NotImplementedError("momentum-projected terms are not part of the device engine yet")
        self.n_sites = prod(self.lvals)

    def _mask_ok(self, coords, mask):
        return mask is None or bool(np.asarray(mask)[tuple(coords)])


class LocalTerm(QMBTerm):
    """Single-site (diagonal) term summed over the (masked) lattice sites."""

    def __init__(self, operator, op_name, **kwargs):
        super().__init__(operator=operator, op_name=op_name, **kwargs)

    def get_Hamiltonian(self, strength, mask=None):
        if not np.isscalar(strength):
            raise TypeError(f"strength must be SCALAR not a {type(strength)}")
        sites = [ii for ii in range(self.n_sites) if self._mask_ok(zig_zag(self.lvals, ii), mask)]
        return TermBlock([self.op], np.array(sites).reshape(-1, 1), strength, diagonal=True, name=self.op_name)


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
