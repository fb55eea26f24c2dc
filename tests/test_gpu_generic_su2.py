"""The generic SU(2) model (j_max = 1, 3/2, and j_max = 1/2 with
use_generic_model) on the device: sector keys bit-exact, the faithful
assembly against the reference's canonical matrix, and Lanczos energies
(f64 and mixed precision) against the reference's (fixtures from
edlgt/models/SU2_model.py:357-472 run by tests/golden/make_golden.py
generic)."""

import numpy as np
import pytest

from cases import SU2_GEN_CASES, build_generic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def _gold_csr(g, name):
    from scipy.sparse import csr_matrix

    n = int(g[f"{name}/dim"])
    return csr_matrix((g[f"{name}/H_data"], g[f"{name}/H_indices"], g[f"{name}/H_indptr"]), shape=(n, n))


@pytest.mark.parametrize("name", sorted(SU2_GEN_CASES))
def test_generic_su2_on_device(name, golden_generic, dev):
    model, g, m = build_generic(name, device=dev)
    assert np.array_equal(model.sector.host_keys(), golden_generic[f"{name}/keys"])
    for b in model.hamiltonian_blocks(g, m):
        model.H.add_term(b)
    model.H.build(force_complex=True)
    got = model.H.mat.to_scipy()
    ref = _gold_csr(golden_generic, name)
    assert np.array_equal(got.indptr, ref.indptr)
    assert np.array_equal(got.indices, ref.indices)
    assert np.max(np.abs(got.data - ref.data)) <= 1e-13 * max(1.0, np.max(np.abs(ref.data)))
    # the model API path: build (real form where the gauge phases allow it)
    # and diagonalise on the device
    model.build_Hamiltonian(g, m)
    e_ref = golden_generic[f"{name}/energies"]
    model.diagonalize_Hamiltonian(len(e_ref))
    assert np.allclose(np.asarray(model.H.Nenergies)[: len(e_ref)], e_ref, atol=1e-10, rtol=0)


def test_generic_su2_mixed_precision(golden_generic, dev):
    """Mixed-precision ground state of the largest 1D j_max = 1 case against
    the reference at 1e-9 relative."""
    from edgpu.solvers import lanczos_mixed

    name = "su2gen_1d_L6_obc_j1"
    model, g, m = build_generic(name, device=dev)
    model.build_Hamiltonian(g, m)
    mat = model.H.mat
    if mat.is_complex:
        pytest.skip("the gauge phases do not give a real form here")
    r64, _ = lanczos_mixed(mat)
    ref = golden_generic[f"{name}/energies"][0]
    assert abs(r64.evals[0, 0] / model.n_sites - ref) <= 1e-9 * abs(ref)
