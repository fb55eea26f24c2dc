"""Bipartitions of a sector, reduced density matrices and entanglement
entropies on the device.

Mirrors ``QuantumModel._get_partition`` with ``_unique_configs_with_inverse``
(edlgt/models/quantum_model.py:715-791, 73-117) and
``QMB_state._get_psi_matrix`` / ``reduced_density_matrix`` /
``entanglement_entropy`` (edlgt/modeling/qmb_state.py:159-291, with
build_psi_matrix :596-627).  The
partition maps and the state matrix come from ``edg_part_map`` and
``edg_psi_matrix``; the matrix product rho = M M^dagger and its
eigenvalues are library calls (cuBLAS, cuSOLVER through torch).

One difference: for large sparse state matrices the reference estimates the
entropy from a truncated ``svds`` (stopping once 99 % of the norm is
captured); here the spectrum is always exact.  The state matrix is dense on
the device, so ``subsys_dim * env_dim`` is limited by
``MAX_STATE_MATRIX_BYTES``.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = ["partition_map", "get_partition", "psi_matrix", "reduced_density_matrix", "entanglement_entropy",
           "MAX_STATE_MATRIX_BYTES"]

MAX_STATE_MATRIX_BYTES = 16 << 30
_PSI_CODES = {torch.float64: 0, torch.float32: 1, torch.complex128: 2, torch.complex64: 3}


def partition_map(sector, sites):
    """(index, unique_configs, dim) of the part made of ``sites`` (any order;
    used ascending): index[r] is row r's position among the distinct part
    configurations (a device int64 tensor), unique_configs their uint16 table
    in ascending lexicographic order (host)."""
    sector.require_narrow("partition map")
    sites = sorted(int(s) for s in sites)
    dev = sector.device
    n = len(sector)
    dims = [int(sector.loc_dims[s]) for s in sites]
    spec = _lib.PartSpec()
    spec.n_part = len(sites)
    space = 1
    for d in dims:
        space *= d
    spec.key_space = space
    run = 1
    for k in range(len(sites) - 1, -1, -1):
        spec.part_stride[k] = run
        run *= dims[k]
    for k, s in enumerate(sites):
        spec.src_stride[k] = int(sector.strides[s])
        spec.dim[k] = dims[k]
    ns = lib.edg_part_scratch_elems(space)
    if ns < 0:
        raise ValueError(f"part key space {space} above 2^34: this partition needs a sort-based map")
    scratch = torch.empty(ns, dtype=torch.int64, device=dev)
    index = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    cap = min(space, max(n, 1))
    ukeys = torch.empty(cap, dtype=torch.int64, device=dev)
    n_unique = ctypes.c_int64(0)
    check(lib.edg_part_map(ptr(sector.keys), n, ctypes.byref(spec), ptr(index), ptr(ukeys), cap,
                           ctypes.byref(n_unique), ptr(scratch), ns, stream_handle()), "edg_part_map")
    m = int(n_unique.value)
    if len(sites) == 0:
        configs = np.empty((1 if n else 0, 0), dtype=np.uint16)
    else:
        ld = torch.from_numpy(np.asarray(dims, dtype=np.int32)).to(dev)
        out = torch.empty((max(m, 1), len(sites)), dtype=torch.int16, device=dev)
        check(lib.edg_keys_to_configs(ptr(ukeys), m, len(sites), ptr(ld), ptr(out), stream_handle()),
              "edg_keys_to_configs")
        configs = out[:m].cpu().numpy().view(np.uint16)
    return index[:n], configs, m


def get_partition(sector, n_sites, keep_indices):
    """The partition record of ``QuantumModel._get_partition``: host maps and
    unique configurations as in the reference, plus the device maps."""
    keep = np.array(sorted(int(i) for i in keep_indices), dtype=np.int64)
    env = np.array([i for i in range(n_sites) if i not in set(keep.tolist())], dtype=np.int64)
    sub_idx, sub_cfg, sub_dim = partition_map(sector, keep)
    env_idx, env_cfg, env_dim = partition_map(sector, env)
    return {
        "subsys_indices": keep,
        "env_indices": env,
        "unique_subsys_configs": sub_cfg,
        "unique_env_configs": env_cfg,
        "subsys_dim": sub_dim,
        "env_dim": env_dim,
        "subsys_map": sub_idx.cpu().numpy(),
        "env_map": env_idx.cpu().numpy(),
        "subsys_map_dev": sub_idx,
        "env_map_dev": env_idx,
    }


def _record(keep_indices, partitions_dict):
    key = tuple(sorted(int(i) for i in keep_indices))
    if key not in partitions_dict:
        raise ValueError(f"{key} partition not yet implemented on the model")
    return partitions_dict[key]


def psi_matrix(psi, part):
    """Dense (subsys_dim, env_dim) complex128 state matrix on the device."""
    sub_dim, env_dim = int(part["subsys_dim"]), int(part["env_dim"])
    if sub_dim * env_dim * 16 > MAX_STATE_MATRIX_BYTES:
        raise ValueError(f"state matrix {sub_dim} x {env_dim} exceeds {MAX_STATE_MATRIX_BYTES} bytes")
    sub, env = part["subsys_map_dev"], part["env_map_dev"]
    p = psi if psi.dtype in _PSI_CODES else psi.to(torch.complex128)
    p = p.contiguous()
    out = torch.empty((sub_dim, env_dim), dtype=torch.complex128, device=sub.device)
    flag = torch.empty(1, dtype=torch.int32, device=sub.device)
    check(lib.edg_psi_matrix(ptr(p), _PSI_CODES[p.dtype], int(p.shape[0]), ptr(sub), ptr(env), sub_dim, env_dim,
                             ptr(out), 2, ptr(flag), stream_handle()), "edg_psi_matrix")
    return out


def reduced_density_matrix(psi, keep_indices, partitions_dict):
    """rho = M M^dagger on the subsystem (host complex128 array)."""
    m = psi_matrix(psi, _record(keep_indices, partitions_dict))
    return (m @ m.conj().T).cpu().numpy()


def entanglement_entropy(psi, keep_indices, partitions_dict):
    """Von Neumann entropy in bits of the subsystem: -sum l log2 l over the
    squared singular values l > 1e-10 of M, taken as the eigenvalues of the
    smaller of M M^dagger and M^dagger M."""
    m = psi_matrix(psi, _record(keep_indices, partitions_dict))
    if min(m.shape) == 1:
        return 0.0
    rho = m @ m.conj().T if m.shape[0] <= m.shape[1] else m.conj().T @ m
    lam = torch.linalg.eigvalsh(rho)
    lam = lam[lam > 1e-10]
    return float(-(lam * torch.log2(lam)).sum().item())
