"""Lattice geometry for hypercubic lattices: site linearisation, neighbours,
plaquettes, border labels, staggered masks and link pairs.

Conventions follow ed-lgt so that site indices, border labels and term
ordering agree with the reference:

* linear site index: mixed radix with the x coordinate fastest
  (``edlgt/modeling/lattice_mappings.py:20-98``);
* neighbour along an axis, with periodic wrap only for PBC axes
  (``edlgt/modeling/lattice_geometry.py:110-163``);
* plaquette corners ``[origin, +a, +b, +a+b]``
  (``edlgt/modeling/lattice_geometry.py:166-222``);
* site labels ``{even|odd|site}[_m<ax>|_p<ax>]...`` for OBC borders
  (``edlgt/modeling/lattice_geometry.py:22-74``);
* staggered parity ``(-1)**sum(coords)`` (``edlgt/modeling/masks.py:18-44``).
"""

from __future__ import annotations

from itertools import product
from math import prod

import numpy as np

__all__ = [
    "AXES",
    "zig_zag",
    "inverse_zig_zag",
    "neighbor_sites",
    "plaquette_sites",
    "site_label",
    "lattice_labels",
    "staggered_mask",
    "site_is_even",
    "link_site_pairs",
    "origin_surfaces",
    "border_labels",
]

AXES = "xyz"


def _strides(lvals):
    strides = [1] * len(lvals)
    for ax in range(1, len(lvals)):
        strides[ax] = strides[ax - 1] * int(lvals[ax - 1])
    return strides


def zig_zag(lvals, index):
    """Linear site index -> coordinates (x fastest)."""
    n = prod(lvals)
    if not 0 <= int(index) < n:
        raise ValueError(f"site index must be in [0, {n - 1}], got {index}")
    return tuple((int(index) // s) % int(l) for l, s in zip(lvals, _strides(lvals)))


def inverse_zig_zag(lvals, coords):
    """Coordinates -> linear site index (x fastest)."""
    if len(coords) != len(lvals):
        raise ValueError("coords and lvals must have the same length")
    for c, l in zip(coords, lvals):
        if not 0 <= int(c) < int(l):
            raise ValueError(f"coordinate {c} outside [0, {l - 1}]")
    return int(sum(int(c) * s for c, s in zip(coords, _strides(lvals))))


def neighbor_sites(coords, lvals, axis, has_obc):
    """Return ``[i, j]`` for the link leaving ``coords`` along ``axis`` or None."""
    ax = AXES.index(axis)
    c = list(coords)
    if c[ax] < lvals[ax] - 1 or (c[ax] == lvals[ax] - 1 and not has_obc[ax]):
        c2 = list(c)
        c2[ax] = (c2[ax] + 1) % lvals[ax]
        return [inverse_zig_zag(lvals, c), inverse_zig_zag(lvals, c2)]
    return None


def plaquette_sites(coords, lvals, axes, has_obc):
    """Return the four plaquette corners ``[o, o+a, o+b, o+a+b]`` or None."""
    ia, ib = AXES.index(axes[0]), AXES.index(axes[1])
    for ax in (ia, ib):
        c = coords[ax]
        if not (c < lvals[ax] - 1 or (c == lvals[ax] - 1 and not has_obc[ax])):
            return None
    base = list(coords)
    c1 = list(base)
    c1[ia] = (c1[ia] + 1) % lvals[ia]
    c2 = list(base)
    c2[ib] = (c2[ib] + 1) % lvals[ib]
    c3 = list(base)
    c3[ia] = (c3[ia] + 1) % lvals[ia]
    c3[ib] = (c3[ib] + 1) % lvals[ib]
    return [inverse_zig_zag(lvals, x) for x in (base, c1, c2, c3)]


def site_is_even(coords):
    return sum(coords) % 2 == 0


def site_label(coords, lvals, has_obc, staggered_basis):
    """Basis label of a site: staggering plus OBC border suffixes."""
    if staggered_basis:
        label = "even" if site_is_even(coords) else "odd"
    else:
        label = "site"
    for ax, c in enumerate(coords):
        if has_obc[ax]:
            if c == 0:
                label += f"_m{AXES[ax]}"
            elif c == lvals[ax] - 1:
                label += f"_p{AXES[ax]}"
    return label


def lattice_labels(lvals, has_obc, staggered_basis):
    """Per-site labels in linear site order."""
    return [
        site_label(zig_zag(lvals, ii), lvals, has_obc, staggered_basis)
        for ii in range(prod(lvals))
    ]


def staggered_mask(lvals, stag_label):
    """Boolean lattice-shaped mask of even or odd sites."""
    if stag_label not in ("even", "odd"):
        raise ValueError(f"stag_label must be 'even' or 'odd', got {stag_label}")
    mask = np.zeros(tuple(lvals), dtype=bool)
    for coords in product(*[range(l) for l in lvals]):
        even = site_is_even(coords)
        mask[coords] = even if stag_label == "even" else not even
    return mask


def link_site_pairs(lvals, has_obc):
    """Per-axis arrays of linked site pairs, in linear site order."""
    out = []
    for axis in AXES[: len(lvals)]:
        pairs = []
        for ii in range(prod(lvals)):
            s = neighbor_sites(zig_zag(lvals, ii), lvals, axis, has_obc)
            if s is not None:
                pairs.append(s)
        out.append(np.array(pairs, dtype=np.int32).reshape(-1, 2))
    return out


def origin_surfaces(lvals):
    """Sites on the lines (2D) or faces (3D) through the origin."""
    if len(lvals) == 2:
        lx, ly = lvals
        return {
            "x": [inverse_zig_zag(lvals, (x, 0)) for x in range(lx)],
            "y": [inverse_zig_zag(lvals, (0, y)) for y in range(ly)],
        }
    if len(lvals) == 3:
        lx, ly, lz = lvals
        return {
            "yz": [inverse_zig_zag(lvals, (0, y, z)) for y in range(ly) for z in range(lz)],
            "xz": [inverse_zig_zag(lvals, (x, 0, z)) for x in range(lx) for z in range(lz)],
            "xy": [inverse_zig_zag(lvals, (x, y, 0)) for x in range(lx) for y in range(ly)],
        }
    raise ValueError("origin surfaces exist only in 2D and 3D")


def border_labels(lattice_dim):
    """All border/corner suffixes a dressed-site basis is split into."""
    if lattice_dim == 1:
        return ["mx", "px"]
    if lattice_dim == 2:
        return ["mx", "px", "my", "py", "mx_my", "mx_py", "px_my", "px_py"]
    if lattice_dim == 3:
        single = ["mx", "px", "my", "py", "mz", "pz"]
        pairs = [
            "mx_my", "mx_py", "mx_mz", "mx_pz", "px_my", "px_py", "px_mz", "px_pz",
            "my_mz", "my_pz", "py_mz", "py_pz",
        ]
        triples = [f"{a}_{b}_{c}" for a in ("mx", "px") for b in ("my", "py") for c in ("mz", "pz")]
        return single + pairs + triples
    raise ValueError("lattice_dim must be 1, 2 or 3")
