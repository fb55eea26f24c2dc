"""Sectors whose key space exceeds 63 bits (two-word keys) on the device:
pure-gauge 4x4 QED lattices (spin 1 periodic, spin 2 open; product of the
local dimensions 2^68 and 2^68.9) against the reference's sector tables,
canonical matrices and energies (fixtures from tests/golden/make_golden.py
wide), plus a 25.5-million-state open QED chain of 30 sites (2^67) checked
through its properties.

Tolerances: sector tables and matrix patterns bit-exact; weighted value sums
1e-10 relative; energies per site 1e-10 absolute (the reference's own
validation tolerance); observables 1e-10."""

import hashlib

import numpy as np
import pytest

from cases import WIDE_CASES, build_wide

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def _lex_increasing(keys):
    """Two-word keys (low, high) strictly increasing as 128-bit numbers."""
    lo, hi = keys[:, 0], keys[:, 1]
    return bool(np.all((hi[1:] > hi[:-1]) | ((hi[1:] == hi[:-1]) & (lo[1:] > lo[:-1]))))


@pytest.mark.parametrize("name", sorted(WIDE_CASES))
def test_wide_sector_and_lookup(name, golden_wide, dev):
    from oracle import edlgt_oracle as O

    model, _ = build_wide(name, device=dev)
    sec = model.sector
    assert sec.wide and sec.keys.shape == (int(golden_wide[f"{name}/dim"]), 2)
    cfg = sec.configs
    assert hashlib.sha256(np.ascontiguousarray(cfg).tobytes()).hexdigest() == str(golden_wide[f"{name}/configs_sha"])
    keys = sec.host_keys()
    assert _lex_increasing(keys)
    assert int(keys[:, 0].max()) < sec.lo_space
    # encode -> keys is the identity on the sector; lookups of sampled rows
    assert np.array_equal(sec.encode(cfg).cpu().numpy().view(np.uint64), keys)
    rows = golden_wide[f"{name}/sample_rows"]
    assert np.array_equal(sec.index_of(golden_wide[f"{name}/sample_configs"]), rows)
    # random configurations: hits and misses agree with the oracle's search
    rng = np.random.default_rng(11)
    q = np.stack([rng.integers(0, d, 3000) for d in model.loc_dims], axis=1).astype(np.uint16)
    q[::3] = cfg[rng.integers(0, len(cfg), len(q[::3]))]
    got = sec.index_of(q)
    assert np.array_equal(got, O.config_to_index(q, cfg, model.loc_dims))
    assert (got >= 0).sum() >= len(q[::3])


@pytest.mark.parametrize("name", sorted(WIDE_CASES))
def test_wide_assembly_energies_observables(name, golden_wide, dev):
    from oracle import edlgt_oracle as O

    model, g = build_wide(name, device=dev)
    for b in model.hamiltonian_blocks(g):
        model.H.add_term(b)
    model.H.build(force_complex=True)
    m = model.H.mat.to_scipy()
    rows = np.repeat(np.arange(m.shape[0], dtype=np.int64), np.diff(m.indptr))
    cols = m.indices.astype(np.int64)
    assert m.nnz == int(golden_wide[f"{name}/H_nnz"])
    assert hashlib.sha256(np.stack([rows, cols]).tobytes()).hexdigest() == str(golden_wide[f"{name}/H_pattern_sha"])
    w = 1.0 / (1.0 + ((rows * 7919 + cols * 104729) % 1009))
    ref = complex(golden_wide[f"{name}/H_wsum"])
    assert abs(np.sum(m.data * w) - ref) <= 1e-10 * abs(ref)
    # the model API: build and diagonalise on the device
    model.build_Hamiltonian(g)
    e_ref = golden_wide[f"{name}/energies"]
    model.diagonalize_Hamiltonian(len(e_ref))
    assert np.allclose(np.asarray(model.H.Nenergies)[: len(e_ref)], e_ref, atol=1e-10, rtol=0)
    # a local observable on the ground state (two-word key decode)
    psi = model.H.Npsi[0]
    psi_h = psi.psi if hasattr(psi, "psi") else psi
    psi_h = np.asarray(psi_h.cpu().numpy() if hasattr(psi_h, "cpu") else psi_h)
    got = np.asarray(model.local_expval(model.ops["E2"], psi))
    want = O.local_expval(psi_h, model.ops["E2"], model.sector.configs)
    assert np.allclose(got, want, atol=1e-10, rtol=0)


def test_wide_chain_30_sites(dev):
    """QED spin-1 open chain with matter, 30 sites: 2^67 key space,
    25,532,994 states (the oracle's sector_configs count for this
    lattice).  Keys strictly increasing, every configuration decodes and
    encodes back to its key, and sampled rows are found at their index."""
    import torch

    from edgpu.models import QED_Model

    model = QED_Model(spin=1, pure_theory=False, lvals=[30], has_obc=[True], device=dev)
    sec = model.sector
    assert sec.wide and len(sec) == 25_532_994
    keys = sec.host_keys()
    assert _lex_increasing(keys)
    cfg = sec.configs
    back = sec.encode(cfg)
    assert torch.equal(back, sec.keys)
    rng = np.random.default_rng(5)
    rows = np.sort(rng.choice(len(sec), 5000, replace=False))
    assert np.array_equal(sec.index_of(cfg[rows]), rows)
