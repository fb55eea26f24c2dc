"""Full diagonalisation on the device (dense path), thermal functions,
ensemble averages and exact time evolution against the reference
(QMB_hamiltonian.diagonalize('full', 'dense'), partition_function ... get_beta,
get_r_value, exact_time_evolution; QuantumModel.canonical_avg,
microcanonical_avg, diagonal_avg: edlgt/modeling/qmb_hamiltonian.py:260-620,
791-835, edlgt/models/quantum_model.py:864-1156)."""

import numpy as np
import pytest

from cases import build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


@pytest.fixture(scope="module")
def full_model(dev):
    model, _, _ = build("su2_1d_L6_pbc", device=dev)
    model.build_Hamiltonian(1.0, 5.0)
    model.diagonalize_Hamiltonian("full", "dense")
    return model


def test_full_spectrum_and_thermal_functions(full_model, golden_full):
    g = golden_full
    m = full_model
    assert np.array_equal(m.sector.host_keys(), g["keys"])
    assert np.allclose(m.H.Nenergies, g["energies"], atol=1e-10, rtol=0)
    assert len(m.H.Npsi) == len(g["energies"])
    m.H.get_r_value()
    assert abs(m.H.r_value - float(g["r_value"])) <= 1e-6
    beta = float(g["beta"])
    assert np.isclose(m.H.partition_function(beta), g["Z"], rtol=1e-10)
    assert np.isclose(m.H.free_energy(beta), g["F"], rtol=1e-10)
    assert np.isclose(m.H.thermal_average(beta), g["E_thermal"], rtol=1e-10)
    assert np.isclose(m.H.F_prime(beta), g["F_prime"], rtol=1e-9)
    state = m.get_qmb_state_from_configs([g["config"]])
    assert np.isclose(m.get_thermal_beta(state, 1e-10), g["beta_state"], rtol=1e-9)


def test_ensemble_averages(full_model, golden_full):
    g = golden_full
    m = full_model
    state = m.get_qmb_state_from_configs([g["config"]])
    assert np.isclose(m.canonical_avg("N_tot", float(g["beta"])), g["canonical_N_tot"], rtol=1e-10)
    psi_th, me = m.microcanonical_avg(["N_tot", "T2_px"], state)
    assert abs(np.linalg.norm(psi_th) - 1.0) <= 1e-10  # eigenvector phases are arbitrary: only its norm compares
    for name in ("N_tot", "T2_px"):
        assert abs(me[f"ME_{name}"] - float(g[f"ME_{name}"])) <= 1e-10, name
    de = m.diagonal_avg(["N_tot", "T2_px"], state)
    for name in ("N_tot", "T2_px"):
        assert abs(de[f"DE_{name}"] - float(g[f"DE_{name}"])) <= 1e-10, name
    assert np.isclose(m.measure_fidelity(m.H.Npsi[3].psi, 3), 1.0, atol=1e-12)


def test_exact_time_evolution(full_model, golden_full):
    g = golden_full
    m = full_model
    state = m.get_qmb_state_from_configs([g["config"]])
    m.time_evolution_Hamiltonian(state, g["time"])
    for j in range(len(g["time"])):
        assert np.max(np.abs(m.H.psi_time[j].psi - g["psi_time"][j])) <= 1e-10, j


def test_dense_limit_and_partial_spectrum(dev):
    """An integer n_eigs with the dense format keeps every energy and the
    first n_eigs states (the reference's dense branch); thermal functions
    then take the reference's expm branch: Tr exp(-beta H) over the total
    energies, not the energy densities."""
    model, g, mass = build("qed1d_L8_obc", device=dev)
    model.build_Hamiltonian(g, mass)
    model.diagonalize_Hamiltonian(3, "dense")
    assert len(model.H.Nenergies) == model.H.shape[0] and len(model.H.Npsi) == 3
    e_tot = np.asarray(model.H.Nenergies) * model.n_sites
    assert np.isclose(model.H.partition_function(1.0), np.sum(np.exp(-e_tot)), rtol=1e-12, atol=0)
