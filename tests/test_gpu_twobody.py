"""Two-body correlators on the device against the reference's fixtures and
the oracle (TwoBodyTerm.get_expval, edlgt/modeling/twobody_term.py:160-264)."""

import numpy as np
import pytest

from cases import TWOBODY_CASES, build
from oracle import edlgt_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


@pytest.mark.parametrize("name", sorted(TWOBODY_CASES))
def test_twobody_matches_reference_on_its_state(name, golden_twobody, dev):
    """The reference's own ground state: the device matrix equals the
    reference's correlator matrix (f64 accumulation, tolerance 1e-12)."""
    import torch

    model, _, _ = build(name, device=dev)
    assert np.array_equal(model.sector.host_keys(), golden_twobody[f"{name}/keys"])
    psi = torch.from_numpy(golden_twobody[f"{name}/psi"]).to(dev)
    for a, b in TWOBODY_CASES[name]:
        corr = model.twobody_expval(model.ops[a], model.ops[b], psi)
        ref = golden_twobody[f"{name}/{a}_{b}"]
        assert np.max(np.abs(corr - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), (a, b)


@pytest.mark.parametrize("name", sorted(TWOBODY_CASES))
def test_twobody_through_measure_observables(name, golden_twobody, dev):
    """get_observables(twobody_obs=...) + measure_observables on the device
    ground state; expectation values do not depend on the state's phase."""
    model, g, m = build(name, device=dev)
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(1)
    pairs = TWOBODY_CASES[name]
    model.get_observables([], twobody_obs=pairs)
    model.measure_observables(0)
    for a, b in pairs:
        ref = golden_twobody[f"{name}/{a}_{b}"]
        got = model.res[f"{a}_{b}"]
        assert got.shape == ref.shape
        assert np.max(np.abs(got - ref)) <= 1e-8 * max(1.0, np.max(np.abs(ref))), (a, b)


def _product_space(loc_dims, dev):
    """The whole product space as one sector: every local operator keeps it."""
    import torch

    from edgpu.symmetries import Sector

    n = int(np.prod(loc_dims))
    return Sector(torch.arange(n, dtype=torch.int64, device=dev), loc_dims, device=dev)


def _random_ops(rng, loc_dims, dmax, density=0.6):
    ops = np.zeros((len(loc_dims), dmax, dmax), dtype=np.complex128)
    for s, d in enumerate(loc_dims):
        m = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
        m[rng.random((d, d)) > density] = 0
        ops[s, :d, :d] = m
    return ops


@pytest.mark.parametrize("dtype", ["complex128", "complex64", "float64", "float32"])
def test_twobody_offdiagonal_complex_operators(dtype, dev):
    """Off-diagonal complex operators on a product space (kets move on both
    sites), every psi storage type, against the oracle on the same psi."""
    import torch

    from edgpu.models.quantum_model import twobody_corr_device

    rng = np.random.default_rng(11)
    loc_dims = np.array([3, 4, 2, 5, 3, 4])
    sector = _product_space(loc_dims, dev)
    op_a = _random_ops(rng, loc_dims, 5)
    op_b = _random_ops(rng, loc_dims, 5)
    n = len(sector)
    psi = rng.normal(size=n) + (1j * rng.normal(size=n) if dtype.startswith("complex") else 0)
    psi /= np.linalg.norm(psi)
    psi = psi.astype(dtype)
    corr = twobody_corr_device(sector, op_a, op_b, torch.from_numpy(psi).to(dev)).cpu().numpy()
    cfg = sector.configs
    ref = O.twobody_expval(psi.astype(np.complex128), op_a, op_b, cfg, loc_dims)
    tol = 1e-12 if dtype in ("complex128", "float64") else 2e-6
    assert np.max(np.abs(corr - ref)) <= tol * max(1.0, np.max(np.abs(ref)))
    assert np.all(np.diag(corr) == 0) and np.array_equal(corr, corr.T)


def test_twobody_pair_subset_and_empty(dev):
    """An explicit pair list fills only those entries; no pairs gives zeros."""
    import torch

    from edgpu.models.quantum_model import twobody_corr_device

    rng = np.random.default_rng(3)
    loc_dims = np.array([2, 3, 2, 3, 2])
    sector = _product_space(loc_dims, dev)
    op_a = _random_ops(rng, loc_dims, 3)
    psi = rng.normal(size=len(sector)) + 1j * rng.normal(size=len(sector))
    full = O.twobody_expval(psi, op_a, op_a, sector.configs, loc_dims)
    t = torch.from_numpy(psi).to(dev)
    pairs = [(0, 3), (2, 4)]
    got = twobody_corr_device(sector, op_a, op_a, t, pairs=pairs).cpu().numpy()
    want = np.zeros_like(full)
    for i, j in pairs:
        want[i, j] = want[j, i] = full[i, j]
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(full)))
    none = twobody_corr_device(sector, op_a, op_a, t, pairs=np.zeros((0, 2), dtype=np.int32)).cpu().numpy()
    assert np.all(none == 0)


def test_twobody_missing_ket_is_an_error(dev):
    """An operator that changes the charge takes configurations out of the
    sector: the device call reports it instead of reading a wrong amplitude."""
    import torch

    from edgpu._lib import EdgError

    model, _, _ = build("qed1d_L8_obc", device=dev)
    psi = torch.ones(len(model.sector), dtype=torch.float64, device=dev)
    with pytest.raises(EdgError, match="MISSING_KET"):
        model.twobody_expval(model.ops["Q_px_dag"], model.ops["N"], psi)


@pytest.mark.parametrize("kind", ["real", "complex", "mixed"])
def test_twobody_diagonal_operators(kind, dev):
    """Diagonal operators take the per-row |psi_r|^2 a b paths (real: the
    real-diagonal block path; complex or one off-diagonal factor: the
    transition-table path); all against the oracle."""
    import torch

    from edgpu.models.quantum_model import twobody_corr_device

    rng = np.random.default_rng(5)
    loc_dims = np.array([4, 3, 5, 2, 4, 3, 2])
    sector = _product_space(loc_dims, dev)
    dmax = 5

    def diag_ops(cplx):
        ops = np.zeros((len(loc_dims), dmax, dmax), dtype=np.complex128)
        for s, d in enumerate(loc_dims):
            v = rng.normal(size=d) + (1j * rng.normal(size=d) if cplx else 0)
            v[rng.random(d) < 0.3] = 0
            ops[s, np.arange(d), np.arange(d)] = v
        return ops

    op_a = diag_ops(kind == "complex")
    op_b = diag_ops(kind == "complex") if kind != "mixed" else _random_ops(rng, loc_dims, dmax)
    psi = rng.normal(size=len(sector)) + 1j * rng.normal(size=len(sector))
    psi /= np.linalg.norm(psi)
    got = twobody_corr_device(sector, op_a, op_b, torch.from_numpy(psi).to(dev)).cpu().numpy()
    ref = O.twobody_expval(psi, op_a, op_b, sector.configs, loc_dims)
    assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
