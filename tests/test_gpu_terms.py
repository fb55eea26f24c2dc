"""Term-level expectation values (LocalTerm / TwoBodyTerm / PlaquetteTerm /
NBodyTerm .get_expval) and the reference's momentum workflow order
(set_momentum_sector, default_params, build_Hamiltonian, diagonalize) on the
device, against the reference's fixtures."""

import numpy as np
import pytest

from cases import NBODY_CASES, TWOBODY_CASES, build, build_momentum_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def test_term_expvals_match_reference(golden_twobody, golden_nbody, golden_pins, dev):
    import torch

    from edgpu.modeling import LocalTerm, NBodyTerm, PlaquetteTerm, QMB_state, TwoBodyTerm

    name = "su2_1d_L8_obc"
    model, _, _ = build(name, device=dev)
    st = QMB_state(torch.from_numpy(golden_twobody[f"{name}/psi"]).to(dev))
    a, b = TWOBODY_CASES[name][0]
    t = TwoBodyTerm("x", [model.ops[a], model.ops[b]], [a, b], **model.def_params)
    t.get_expval(st)
    assert np.max(np.abs(t.corr - golden_twobody[f"{name}/{a}_{b}"])) <= 1e-12
    lt = LocalTerm(model.ops["N_tot"], "N_tot", **model.def_params)
    lt.get_expval(st, get_variance=True)
    assert np.allclose(lt.obs, model.local_expval(model.ops["N_tot"], st), atol=1e-14)
    assert abs(lt.avg - np.mean(lt.obs)) <= 1e-15 and lt.std >= 0
    lt.get_expval(st, stag_label="even")
    assert abs(lt.avg - np.mean(lt.obs[0::2])) <= 1e-15
    ops, dists = NBODY_CASES[name]
    st_nb = QMB_state(torch.from_numpy(golden_nbody[f"{name}/psi"]).to(dev))
    nt = NBodyTerm([model.ops[o] for o in ops[0]], ops[0], dists[0], **model.def_params)
    nt.get_expval(st_nb)
    assert np.max(np.abs(nt.obs - golden_nbody[f"{name}/{'_'.join(ops[0])}"])) <= 1e-12
    model, g, m = build("qed2d_3x2_bg", device=dev)
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(1)
    names = ["C_px,py", "C_py,mx", "C_my,px", "C_mx,my"]
    pt = PlaquetteTerm(["x", "y"], [model.ops[o] for o in names], names, **model.def_params)
    pt.get_expval(model.H.GSpsi)
    assert abs(pt.avg - golden_pins["qed2d_3x2_bg/plaq"]) < 1e-10


def test_momentum_in_reference_workflow_order(golden_momentum, dev):
    """set_momentum_sector before default_params and build_Hamiltonian, as the
    reference's workflows call them."""
    model, g, m, ucs, _ = build_momentum_case("su2_1d_L6_pbc", device=dev)
    model.set_momentum_sector(ucs, [3])
    model.default_params()
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(2)
    assert np.allclose(model.H.Nenergies, golden_momentum["su2_1d_L6_pbc/k3/energies"], atol=1e-10, rtol=0)


@pytest.mark.parametrize("R0", [3, 6])
def test_local_hamiltonian_matches_reference(R0, golden_local, dev):
    """SU2_Model.build_local_Hamiltonian against the reference's matrix (in
    the reference basis, 1e-13)."""
    from scipy.sparse import csr_matrix, diags

    model, _, _ = build("su2_1d_L8_obc", device=dev)
    model.build_local_Hamiltonian(1.0, 0.5, R0)
    model.Hlocal.build()
    h = model.Hlocal.to_scipy()
    ph = model.Hlocal._row_phase()
    if ph is not None:
        p = diags(ph.cpu().numpy())
        h = p @ h @ p.conj()
    n = h.shape[0]
    ref = csr_matrix((golden_local[f"R{R0}/data"], golden_local[f"R{R0}/indices"], golden_local[f"R{R0}/indptr"]),
                     shape=(n, n))
    assert abs(h - ref).max() <= 1e-13


@pytest.mark.parametrize("name", ["qedint_L4", "qedint_L8_bg", "qedint_L10"])
def test_integrated_qed_on_device(name, golden_integrated, dev):
    """Integrated-gauge 1D QED built on the device: sector keys bit-exact, the
    matrix in the reference basis to 1e-12, energies to 1e-10."""
    from scipy.sparse import csr_matrix, diags

    from cases import INTEGRATED_CASES
    from edgpu.models import QED_Model

    lvals, bg, g, m = INTEGRATED_CASES[name]
    model = QED_Model(spin="integrated", pure_theory=False, lvals=lvals, has_obc=[True], bg_list=bg, device=dev)
    assert np.array_equal(model.sector.host_keys(), golden_integrated[f"{name}/keys"])
    model.build_Hamiltonian(g, m)
    h = model.H.to_scipy()
    ph = model.H._row_phase()
    if ph is not None:
        p = diags(ph.cpu().numpy())
        h = p @ h @ p.conj()
    n = h.shape[0]
    ref = csr_matrix((golden_integrated[f"{name}/H_data"], golden_integrated[f"{name}/H_indices"],
                      golden_integrated[f"{name}/H_indptr"]), shape=(n, n))
    assert abs(h - ref).max() <= 1e-12
    model.diagonalize_Hamiltonian(2)
    assert np.allclose(model.H.Nenergies, golden_integrated[f"{name}/energies"], atol=1e-10, rtol=0)
