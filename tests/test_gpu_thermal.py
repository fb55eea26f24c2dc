"""Thermal functions after a partial diagonalisation (two eigenpairs): the
reference's sparse-expm branches of partition_function, free_energy,
thermal_average, F_prime and get_beta (edlgt/modeling/qmb_hamiltonian.py:
428-564) and the canonical average (edlgt/models/quantum_model.py:904-938),
on SU(2) L=6 PBC (g=1, m=5, dim 282).  Fixtures: make_golden.py thermal.

The "sparse" format takes Tr(H^2 exp(-beta H)) by matrix power, the "dense"
format by the elementwise square of the dense array, as the reference does.
Tolerances: relative 1e-10 (1e-9 for F_prime and beta)."""

import numpy as np
import pytest

from cases import build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


@pytest.mark.parametrize("fmt", ["sparse", "dense"])
def test_thermal_functions_without_full_spectrum(fmt, golden_thermal, dev):
    g = golden_thermal
    model, _, _ = build("su2_1d_L6_pbc", device=dev)
    model.build_Hamiltonian(1.0, 5.0)
    model.diagonalize_Hamiltonian(2, fmt)
    assert not model.H._full()
    ref_e = g[f"{fmt}/energies"]
    assert np.allclose(np.asarray(model.H.Nenergies)[:2], ref_e[:2], atol=1e-10, rtol=0)
    for beta in (0.3, 0.7):
        q = f"{fmt}/b{beta}/"
        assert np.isclose(model.H.partition_function(beta), g[q + "Z"], rtol=1e-10, atol=0)
        assert np.isclose(model.H.free_energy(beta), g[q + "F"], rtol=1e-10, atol=0)
        assert np.isclose(model.H.thermal_average(beta), g[q + "E_thermal"], rtol=1e-10, atol=0)
        assert np.isclose(model.H.F_prime(beta), g[q + "F_prime"], rtol=1e-9, atol=0)
        assert np.isclose(model.canonical_avg("T2_px", beta), g[q + "canonical_T2_px"], rtol=1e-10, atol=0)
    if fmt == "sparse":
        state = model.get_qmb_state_from_configs([g["sparse/config"]])
        assert np.isclose(model.get_thermal_beta(state, 1e-10), g["sparse/beta_state"], rtol=1e-9, atol=0)


def test_thermal_cache_follows_the_matrix(golden_thermal, dev):
    """A rebuilt Hamiltonian drops the eigen-system of the previous one."""
    model, _, _ = build("su2_1d_L6_pbc", device=dev)
    model.build_Hamiltonian(2.0, 1.0)
    model.diagonalize_Hamiltonian(1, "sparse")
    z_other = model.H.partition_function(0.7)
    model.build_Hamiltonian(1.0, 5.0)
    model.diagonalize_Hamiltonian(1, "sparse")
    z = model.H.partition_function(0.7)
    assert np.isclose(z, golden_thermal["sparse/b0.7/Z"], rtol=1e-10, atol=0)
    assert not np.isclose(z, z_other, rtol=1e-6)
