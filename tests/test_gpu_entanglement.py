"""Bipartitions, reduced density matrices and entanglement entropies on the
device against the reference's fixtures and the oracle
(QuantumModel._get_partition, QMB_state.reduced_density_matrix /
entanglement_entropy: edlgt/models/quantum_model.py:715-791,
edlgt/modeling/qmb_state.py:159-291)."""

import numpy as np
import pytest

from cases import ENTROPY_CASES, build
from oracle import edlgt_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def _tag(name, keep):
    return f"{name}/" + "-".join(str(i) for i in keep)


@pytest.mark.parametrize("name", sorted(ENTROPY_CASES))
def test_partition_maps_and_entropy_match_reference(name, golden_entropy, dev):
    """Maps and unique configurations bit-exact; on the reference's state the
    entropy to 1e-10 (eigenvalues of rho instead of an SVD of M) and rho to
    1e-12."""
    import torch

    from edgpu.modeling import QMB_state

    model, _, _ = build(name, device=dev)
    assert np.array_equal(model.sector.host_keys(), golden_entropy[f"{name}/keys"])
    st = QMB_state(torch.from_numpy(golden_entropy[f"{name}/psi"]).to(dev))
    for keep in ENTROPY_CASES[name]:
        tag = _tag(name, keep)
        part = model._get_partition(keep)
        for k in ("subsys_map", "env_map", "unique_subsys_configs", "unique_env_configs"):
            assert np.array_equal(part[k], golden_entropy[f"{tag}/{k}"]), (keep, k)
        assert [part["subsys_dim"], part["env_dim"]] == list(golden_entropy[f"{tag}/dims"])
        s = st.entanglement_entropy(keep, model._partition_cache)
        assert abs(s - float(golden_entropy[f"{tag}/entropy"])) <= 1e-10, keep
        if f"{tag}/rdm" in golden_entropy:
            rho = st.reduced_density_matrix(keep, model._partition_cache)
            assert np.max(np.abs(rho - golden_entropy[f"{tag}/rdm"])) <= 1e-12


@pytest.mark.parametrize("name", sorted(ENTROPY_CASES))
def test_entropy_of_device_ground_state(name, golden_entropy, dev):
    model, g, m = build(name, device=dev)
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(1)
    for keep in ENTROPY_CASES[name]:
        model._get_partition(keep)
        s = model.H.Npsi[0].entanglement_entropy(keep, model._partition_cache)
        assert abs(s - float(golden_entropy[f"{_tag(name, keep)}/entropy"])) <= 1e-8, keep


@pytest.mark.parametrize("dtype", ["complex64", "float64", "float32"])
def test_entropy_state_dtypes_and_larger_sector(dtype, dev):
    """SU(2) L=12 OBC (73,789 states): half-chain and scattered partitions
    against the oracle, for a seeded random state in each storage type."""
    import torch

    from edgpu.modeling import QMB_state
    from edgpu.models import SU2_Model

    model = SU2_Model(spin=0.5, pure_theory=False, lvals=[12], has_obc=[True], sectors=[12], device=dev)
    cfg = model.sector_configs
    rng = np.random.default_rng(17)
    n = len(cfg)
    psi = rng.normal(size=n) + (1j * rng.normal(size=n) if dtype.startswith("complex") else 0)
    psi = (psi / np.linalg.norm(psi)).astype(dtype)
    st = QMB_state(torch.from_numpy(psi).to(dev))
    tol = 1e-10 if dtype == "float64" else 2e-5
    for keep in ([0, 1, 2, 3, 4, 5], [0, 3, 7, 11]):
        part = model._get_partition(keep)
        ref = O.partition(cfg, model.loc_dims, keep)
        for k in ("subsys_map", "env_map", "unique_subsys_configs", "unique_env_configs"):
            assert np.array_equal(part[k], ref[k]), (keep, k)
        s = st.entanglement_entropy(keep, model._partition_cache)
        assert abs(s - O.entanglement_entropy(psi.astype(np.complex128), ref)) <= tol, keep


def test_trivial_partitions_and_missing_partition(dev):
    """All sites kept (empty environment) or none kept: one unique
    configuration on the empty side, zero entropy; an unregistered partition
    raises as in the reference."""
    import torch

    from edgpu.modeling import QMB_state

    model, _, _ = build("qed1d_L8_obc", device=dev)
    cfg = model.sector_configs
    psi = torch.ones(len(cfg), dtype=torch.float64, device=dev) / np.sqrt(len(cfg))
    st = QMB_state(psi)
    for keep in (list(range(8)), []):
        part = model._get_partition(keep)
        ref = O.partition(cfg, model.loc_dims, keep)
        for k in ("subsys_map", "env_map"):
            assert np.array_equal(part[k], ref[k]), (keep, k)
        assert part["unique_subsys_configs"].shape == ref["unique_subsys_configs"].shape
        assert part["unique_env_configs"].shape == ref["unique_env_configs"].shape
        assert st.entanglement_entropy(keep, model._partition_cache) == 0.0
    with pytest.raises(ValueError):
        st.entanglement_entropy([0, 5], model._partition_cache)
