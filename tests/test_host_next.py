"""Host-side pieces of the momentum, n-body and partition paths (CPU only):
the translation tables and phase tables the device kernels receive, and the
n-body pattern instances, against the oracle's restatements."""

import numpy as np
import pytest

from cases import nbody_instances
from oracle import edlgt_oracle as O


@pytest.mark.parametrize("lvals,ucs", [([6], [1]), ([8], [2]), ([4, 2], [1, 1]), ([4, 4], [2, 1]),
                                       ([2, 2, 2], [1, 1, 1])])
def test_translation_sources_match_oracle(lvals, ucs):
    from edgpu.momentum import translation_sources

    src, R = translation_sources(lvals, ucs)
    ref, R_ref = O.translation_sources(lvals, ucs)
    assert np.array_equal(src, ref) and np.array_equal(R, R_ref)
    n = int(np.prod(lvals))
    assert np.array_equal(src[0], np.arange(n))  # shift 0 is the identity
    for s in range(src.shape[0]):
        assert np.array_equal(np.sort(src[s]), np.arange(n))  # every shift permutes the sites


def test_translation_sources_reject_bad_cells():
    from edgpu.momentum import translation_sources

    with pytest.raises(ValueError):
        translation_sources([6], [4])
    with pytest.raises(ValueError):
        translation_sources([4, 2], [1])


def test_phase_table_is_the_bloch_phase():
    from edgpu.momentum import _phase_table

    R = np.array([6, 4], dtype=np.int32)
    tab = _phase_table(np.array([5, -1]), R)
    for d in range(2):
        k = [5, -1][d] % R[d]
        want = np.exp(-2j * np.pi * k * np.arange(R[d]) / R[d])
        assert np.max(np.abs(tab[d, : R[d]] - want)) <= 1e-14


@pytest.mark.parametrize("lvals,obc,dist", [([8], [True], [[1], [2]]), ([8], [False], [[3]]),
                                            ([3, 2], [True, True], [[1, 1]]), ([4, 3], [False, True], [[1, 0], [0, 1]])])
def test_nbody_instances_match_the_term(lvals, obc, dist):
    from edgpu.modeling import NBodyTerm

    ops = [np.zeros((int(np.prod(lvals)), 2, 2))] * (len(dist) + 1)
    term = NBodyTerm(ops, ["a"] * len(ops), dist, lvals=lvals, has_obc=obc)
    got = term.get_Hamiltonian(1.0).sites.tolist()
    assert got == nbody_instances(lvals, obc, dist)


def test_oracle_partition_edges():
    """Empty subsystem and empty environment give one unique configuration on
    the empty side (the reference's _unique_configs_with_inverse)."""
    cfg = np.array([[0, 1, 2], [1, 0, 2], [1, 1, 0]], dtype=np.uint16)
    loc = np.array([2, 2, 3])
    p = O.partition(cfg, loc, [])
    assert p["subsys_dim"] == 1 and p["unique_subsys_configs"].shape == (1, 0)
    assert np.array_equal(p["subsys_map"], [0, 0, 0]) and p["env_dim"] == 3
    p = O.partition(cfg, loc, [0, 1, 2])
    assert p["env_dim"] == 1 and np.array_equal(p["subsys_map"], [0, 1, 2])
    p = O.partition(cfg, loc, [0])
    assert np.array_equal(p["subsys_map"], [0, 1, 1]) and p["subsys_dim"] == 2


OVERLAP_MODELS = {
    "su2_1d_L6_pbc": ("SU2", dict(spin=0.5, pure_theory=False, lvals=[6], has_obc=[False], sectors=[6])),
    "su2_1d_L8_obc": ("SU2", dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[True], sectors=[8])),
    "su2_2d_2x2_obc": ("SU2", dict(spin=0.5, pure_theory=False, lvals=[2, 2], has_obc=[True, True], sectors=[4])),
    "su2_2d_2x2_pbc": ("SU2", dict(spin=0.5, pure_theory=False, lvals=[2, 2], has_obc=[False, False], sectors=[4])),
    "su2_2d_2x2_pure_pbc": ("SU2", dict(spin=0.5, pure_theory=True, lvals=[2, 2], has_obc=[False, False])),
    "qed1d_L8_obc": ("QED", dict(spin=1, pure_theory=False, lvals=[8], has_obc=[True])),
    "qed1d_L6_pbc": ("QED", dict(spin=1, pure_theory=False, lvals=[6], has_obc=[False])),
}


@pytest.mark.parametrize("name", sorted(OVERLAP_MODELS))
def test_named_states_match_reference(name, golden_overlap):
    """overlap_QMB_state configurations against the reference's tables."""
    from edgpu.models import QED_Model, SU2_Model

    kind, kw = OVERLAP_MODELS[name]
    model = (SU2_Model if kind == "SU2" else QED_Model)(**kw, device="cpu")
    labels = [k.split("/", 1)[1] for k in golden_overlap.files if k.startswith(name + "/")]
    assert labels
    for lab in labels:
        assert np.array_equal(model.overlap_QMB_state(lab), golden_overlap[f"{name}/{lab}"]), lab


def test_state_post_processing_matches_reference(golden_state):
    """QMB_state participation entropies, large-amplitude configurations
    (with the threshold relaxation) and dense expectation values on the
    reference's SU(2) L=8 ground state."""
    from cases import build
    from edgpu.modeling import QMB_state

    g = golden_state
    model, _, _ = build("su2_1d_L8_obc")
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), g["keys"])
    st = QMB_state(g["psi"], model.lvals, model.loc_dims)
    for a in (0.5, 2, 3):
        assert abs(st.participation_renyi_entropy(a) - float(g[f"PE_{a}"])) <= 1e-12
    with pytest.raises(ValueError):
        st.participation_renyi_entropy(1)
    cfgs, vals = st.get_state_configurations(1e-2, cfg, return_configs=True)
    assert np.array_equal(cfgs, g["cfgs"]) and np.array_equal(vals, g["vals"])
    cfgs, vals = st.get_state_configurations(0.9, cfg, return_configs=True)
    assert np.array_equal(cfgs, g["cfgs_relaxed"]) and np.array_equal(vals, g["vals_relaxed"])
    rng = np.random.default_rng(21)
    n = len(g["psi"])
    m = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    m = m + m.conj().T
    assert abs(st.expectation_value(m, "real") - float(g["ev_dense_real"])) <= 1e-10
    assert abs(st.expectation_value(1j * m, "imag") - float(g["ev_dense_imag"])) <= 1e-10
    from scipy.sparse import coo_matrix

    mc = coo_matrix(m)
    assert abs(st.expectation_value((mc.row, mc.col, mc.data)) - float(g["ev_dense_real"])) <= 1e-10


def test_state_normalize_and_truncate():
    from edgpu.modeling import QMB_state

    st = QMB_state(np.array([3.0, 4.0j, 1e-15]))
    assert np.array_equal(st.truncate(1e-14), np.array([3.0, 4.0j, 0]))
    assert st.normalize() == 5.0
    assert abs(st.get_norm() - 1.0) <= 1e-15
    assert st.normalize() == pytest.approx(1.0)


def test_dtype_mode_normalisation():
    from edgpu.models.quantum_model import QuantumModel

    n = QuantumModel._normalize_dtype_mode
    assert n(True) == "complex" and n(False) == "real" and n(None) == "auto" and n(" Real ") == "real"
    with pytest.raises(ValueError):
        n(None, allow_auto=False)
    with pytest.raises(ValueError):
        n("half")
    with pytest.raises(TypeError):
        n(3)
    m = QuantumModel([4], [True], device="cpu")
    assert m.configure_dtype_mode() == "complex" and m._resolve_dtype_mode("auto") == "complex"
    assert m._resolve_dtype_mode("real") == "real"
    assert m.configure_dtype_mode("real") == "real" and m._resolve_dtype_mode(None) == "real"
