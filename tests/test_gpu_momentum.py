"""Momentum sectors on the device against the reference's projectors and
spectra (set_momentum_sector / get_momentum_basis,
edlgt/symmetries/translational_sym.py:508-949, 1307-1358) and the oracle."""

import numpy as np
import pytest

from cases import MOMENTUM_CASES, build_momentum_case
from oracle import edlgt_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def _tag(name, k):
    return f"{name}/k" + "_".join(str(x) for x in k)


@pytest.mark.parametrize("name", sorted(MOMENTUM_CASES))
def test_projector_and_spectrum_match_reference(name, golden_momentum, dev):
    """B bit-exact in pattern (CSC and CSR), values to 1e-13; the two lowest
    energies of B^dagger H B to 1e-10."""
    model, g, m, ucs, ks = build_momentum_case(name, device=dev)
    assert np.array_equal(model.sector.host_keys(), golden_momentum[f"{name}/keys"])
    model.build_Hamiltonian(g, m)
    for k in ks:
        tag = _tag(name, k)
        model.set_momentum_sector(ucs, k, TC_symmetry=name.endswith("_tc"))
        mb = model.momentum_basis
        cp, ri, dv = (golden_momentum[f"{tag}/{x}"] for x in ("L_col_ptr", "L_row_idx", "L_data"))
        assert mb["n_cols"] == len(cp) - 1
        assert np.array_equal(mb["L_col_ptr"], cp) and np.array_equal(mb["L_row_idx"], ri)
        assert np.max(np.abs(mb["L_data"] - dv), initial=0.0) <= 1e-13
        from scipy.sparse import csc_matrix

        B = csc_matrix((dv, ri, cp), shape=(mb["n_rows"], mb["n_cols"])).tocsr()
        B.sort_indices()
        assert np.array_equal(mb["R_row_ptr"], B.indptr) and np.array_equal(mb["R_col_idx"], B.indices)
        assert np.max(np.abs(mb["R_data"] - B.data), initial=0.0) <= 1e-13
        model.diagonalize_Hamiltonian(2)
        e_ref = golden_momentum[f"{tag}/energies"]
        assert np.allclose(model.H.Nenergies, e_ref, atol=1e-10, rtol=0), (k, model.H.Nenergies, e_ref)


def test_projected_matvec_and_lanczos(dev, monkeypatch):
    """H_k x against the oracle's dense B^dagger H B x (1e-12), and the
    Lanczos path (forced by a small dense limit) against the dense one."""
    import torch

    from edgpu import momentum

    model, g, m, ucs, _ = build_momentum_case("su2_1d_L8_pbc_uc2", device=dev)
    model.build_Hamiltonian(g, m)
    cfg = model.sector_configs
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims).toarray()
    for k in ([1], [0]):
        model.set_momentum_sector(ucs, k)
        cp, ri, data, n_cols = O.momentum_basis(cfg, model.loc_dims, model.lvals, ucs, k)
        Bd = np.zeros((len(cfg), n_cols), dtype=np.complex128)
        for c in range(n_cols):
            Bd[ri[cp[c]:cp[c + 1]], c] = data[cp[c]:cp[c + 1]]
        mom = model._momentum
        mom.bind(model.H)
        rng = np.random.default_rng(3)
        x = rng.normal(size=n_cols) + 1j * rng.normal(size=n_cols)
        y = mom.matvec(torch.from_numpy(x).to(dev)).cpu().numpy()
        ref = Bd.conj().T @ (H @ (Bd @ x))
        assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref))
        e_dense = np.linalg.eigvalsh(Bd.conj().T @ H @ Bd)[0]
        monkeypatch.setattr(momentum, "DENSE_MAX", 16)
        w, v = mom.lowest(1, tol=1e-12)
        monkeypatch.undo()
        assert abs(w[0] - e_dense) <= 1e-9 * abs(e_dense)
        r = mom.matvec(v[:, 0]) - w[0] * v[:, 0]
        assert float(torch.linalg.vector_norm(r)) <= 1e-5


def test_larger_sector_against_oracle(dev):
    """SU(2) L=10 PBC, unit cell 1: B against the oracle at k = 0 and k = 5."""
    from edgpu.models import SU2_Model

    model = SU2_Model(spin=0.5, pure_theory=False, lvals=[10], has_obc=[False], sectors=[10], device=dev)
    cfg = model.sector_configs
    for k in ([0], [5]):
        model.set_momentum_sector([1], k)
        mb = model.momentum_basis
        cp, ri, data, n_cols = O.momentum_basis(cfg, model.loc_dims, model.lvals, [1], k)
        assert mb["n_cols"] == n_cols
        assert np.array_equal(mb["L_col_ptr"], cp) and np.array_equal(mb["L_row_idx"], ri)
        assert np.max(np.abs(mb["L_data"] - data), initial=0.0) <= 1e-13


def test_sector_not_closed_under_translation_is_an_error(dev):
    """QED with staggered matter has different site bases on even and odd
    sites: a one-site translation leaves the sector, which is reported (the
    reference's binary search would return -1 and index with it)."""
    from edgpu._lib import EdgError
    from edgpu.models import QED_Model

    model = QED_Model(spin=1, pure_theory=False, lvals=[6], has_obc=[False], device=dev)
    with pytest.raises(EdgError, match="MISSING_KET"):
        model.set_momentum_sector([1], [0])
    obc, _, _, _, _ = build_momentum_case("su2_1d_L6_pbc", device=dev)
    obc.has_obc = [True]
    with pytest.raises(ValueError):
        obc.set_momentum_sector([1], [0])


def test_time_evolution_in_momentum_sector(dev):
    """Krylov evolution with the projected matvec against the dense
    exp(-i H_k t) of the oracle's B^dagger H B (1e-9), at absolute times."""
    import torch
    from scipy.linalg import expm

    model, g, m, ucs, _ = build_momentum_case("su2_1d_L6_pbc", device=dev)
    model.build_Hamiltonian(g, m)
    cfg = model.sector_configs
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims).toarray()
    model.set_momentum_sector(ucs, [1])
    cp, ri, data, n_cols = O.momentum_basis(cfg, model.loc_dims, model.lvals, ucs, [1])
    Bd = np.zeros((len(cfg), n_cols), dtype=np.complex128)
    for c in range(n_cols):
        Bd[ri[cp[c]:cp[c + 1]], c] = data[cp[c]:cp[c + 1]]
    Hk = Bd.conj().T @ H @ Bd
    rng = np.random.default_rng(9)
    psi0 = rng.normal(size=n_cols) + 1j * rng.normal(size=n_cols)
    psi0 /= np.linalg.norm(psi0)
    times = np.array([0.0, 0.1, 0.5, 1.5])
    model.time_evolution_Hamiltonian(torch.from_numpy(psi0).to(dev), times)
    for j, t in enumerate(times):
        ref = expm(-1j * t * Hk) @ psi0
        assert np.max(np.abs(model.H.psi_time[j].psi - ref)) <= 1e-9, t


def test_pair_mode_projection_and_state_projection(golden_momentum, dev):
    """set_momentum_pair arrays against the single-sector fixtures, the
    check_momentum_pair norms, momentum_basis_projection of H (spectrum of the
    reference) and of a state (B^dagger psi)."""
    from scipy.sparse import csc_matrix

    model, g, m, ucs, _ = build_momentum_case("su2_1d_L6_pbc", device=dev)
    model.build_Hamiltonian(g, m)
    model.set_momentum_pair([0], [1], ucs, False)
    mb = model.momentum_basis
    assert mb["pair_mode"]
    assert np.array_equal(mb["L_col_ptr"], golden_momentum["su2_1d_L6_pbc/k0/L_col_ptr"])
    right = csc_matrix((golden_momentum["su2_1d_L6_pbc/k1/L_data"], golden_momentum["su2_1d_L6_pbc/k1/L_row_idx"],
                        golden_momentum["su2_1d_L6_pbc/k1/L_col_ptr"]), shape=(mb["n_rows_full"], mb["n_cols_R"]))
    right = right.tocsr()
    right.sort_indices()
    assert np.array_equal(mb["R_row_ptr"], right.indptr) and np.array_equal(mb["R_col_idx"], right.indices)
    nl, nr, mix = model.check_momentum_pair()
    assert nl <= 1e-10 and nr <= 1e-10 and mix <= 1e-10
    model.set_momentum_sector(ucs, [3])
    model.momentum_basis_projection("H")
    e = np.linalg.eigvalsh(model.H.Ham.toarray())[:2] / model.n_sites
    assert np.allclose(e, golden_momentum["su2_1d_L6_pbc/k3/energies"], atol=1e-10, rtol=0)
    rng = np.random.default_rng(2)
    psi = rng.normal(size=len(model.sector)) + 1j * rng.normal(size=len(model.sector))
    cp = golden_momentum["su2_1d_L6_pbc/k3/L_col_ptr"]
    B = csc_matrix((golden_momentum["su2_1d_L6_pbc/k3/L_data"], golden_momentum["su2_1d_L6_pbc/k3/L_row_idx"], cp),
                   shape=(len(psi), len(cp) - 1))
    assert np.max(np.abs(model._project_state_with_basis(psi) - B.conj().T @ psi)) <= 1e-12


def test_hamiltonian_utilities_and_fullspace_projector(dev):
    from cases import build

    model, g, m = build("qed1d_L8_obc", device=dev)
    model.build_Hamiltonian(g, m)
    sp = model.H.get_sparsity()
    mat = model.H.to_scipy()
    assert abs(sp - mat.nnz / mat.shape[0] ** 2) <= 1e-15
    model.H.convert_hamiltonian("dense")
    assert model.H.Ham_type == "dense"
    P = model.build_projector_from_sector_to_fullspace([0, 1])
    ref = O.partition(model.sector_configs, model.loc_dims, [0, 1])["unique_subsys_configs"].astype(np.int64)
    dims = np.asarray(model.loc_dims)[[0, 1]]
    assert P.shape == (int(np.prod(dims)), len(ref))
    assert np.array_equal(P.tocsc().indices, ref[:, 0] * dims[1] + ref[:, 1])
