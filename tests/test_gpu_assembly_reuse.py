"""Coupling sweeps reuse the off-diagonal part of the sector matrix: builds
in the same sector whose off-diagonal instances are unchanged share the CSR
and recompute only the diagonal, and give the matrix a build in a fresh
sector gives (pattern and off-diagonal values bit-exact, diagonal 1e-13).
A change of an off-diagonal coefficient (the QED plaquette term follows g)
rebuilds it."""

import numpy as np
import pytest

from cases import build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def _fresh(name, g, m, dev):
    model, _, _ = build(name, device=dev)
    model.build_Hamiltonian(g, m)
    return model.H.mat


def _same(a, b):
    import torch

    assert a.n == b.n and a.is_complex == b.is_complex
    assert torch.equal(a.rowptr, b.rowptr) and torch.equal(a.cols, b.cols) and torch.equal(a.vals, b.vals)
    assert torch.equal(a.diag_present, b.diag_present)
    d = (a.diag - b.diag).abs().max().item() if a.n else 0.0
    assert d <= 1e-13 * max(1.0, b.diag.abs().max().item())


def test_su2_sweep_shares_offdiagonal(dev):
    name = "su2_1d_L10_pbc"
    model, _, _ = build(name, device=dev)
    mats = []
    for g in (0.5, 1.0, 2.0):
        model.build_Hamiltonian(g, 0.5)
        mats.append(model.H.mat)
    assert not mats[0].offdiag_reused and mats[1].offdiag_reused and mats[2].offdiag_reused
    assert mats[1].vals.data_ptr() == mats[0].vals.data_ptr()
    for g, mat in zip((0.5, 1.0, 2.0), mats):
        _same(mat, _fresh(name, g, 0.5, dev))
    # a later solve sees the right couplings
    e = []
    for g in (0.5, 2.0):
        model.build_Hamiltonian(g, 0.5)
        model.diagonalize_Hamiltonian(1)
        e.append(model.H.Nenergies[0])
    assert abs(e[0] - e[1]) > 1e-3


def test_qed_plaquette_change_rebuilds(dev):
    name = "qed2d_3x2_q0"
    model, _, _ = build(name, device=dev)
    model.build_Hamiltonian(0.7, 0.4)
    a = model.H.mat
    model.build_Hamiltonian(1.3, 0.4)  # the plaquette coefficient follows g
    b = model.H.mat
    assert not b.offdiag_reused
    _same(b, _fresh(name, 1.3, 0.4, dev))
    model.build_Hamiltonian(1.3, 0.9)  # mass only: diagonal
    c = model.H.mat
    assert c.offdiag_reused
    _same(c, _fresh(name, 1.3, 0.9, dev))
    _same(a, _fresh(name, 0.7, 0.4, dev))
