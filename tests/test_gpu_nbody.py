"""N-body correlators on the device (NBodyTerm.get_expval,
edlgt/modeling/nbody_term.py:164-257) against the reference's fixtures and
the oracle."""

import numpy as np
import pytest

from cases import NBODY_CASES, build, nbody_instances
from oracle import edlgt_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


@pytest.mark.parametrize("name", sorted(NBODY_CASES))
def test_nbody_matches_reference(name, golden_nbody, dev):
    """On the reference's state to 1e-12; through get_observables /
    measure_observables on the device ground state to 1e-8; the imaginary
    parts against the oracle."""
    import torch

    model, g, m = build(name, device=dev)
    assert np.array_equal(model.sector.host_keys(), golden_nbody[f"{name}/keys"])
    psi = golden_nbody[f"{name}/psi"]
    ops, dists = NBODY_CASES[name]
    cfg = model.sector_configs
    for names, dist in zip(ops, dists):
        ref = golden_nbody[f"{name}/{'_'.join(names)}"]
        got = model.nbody_expval(names, dist, torch.from_numpy(psi).to(dev))
        assert got.shape == ref.shape and np.max(np.abs(got - ref)) <= 1e-12, names
        im = model.nbody_expval(names, dist, torch.from_numpy(psi).to(dev), component="imag")
        im_ref = []
        for sites in nbody_instances(model.lvals, model.has_obc, dist):
            rows, cols, v = O.nbody_triplets([model.ops[o] for o in names], sites, cfg, model.loc_dims)
            im_ref.append(np.imag(np.sum(np.conj(psi[rows]) * v * psi[cols])))
        assert np.max(np.abs(im - np.array(im_ref))) <= 1e-12, names
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(1)
    model.get_observables([], nbody_obs=ops, nbody_dist=dists)
    model.measure_observables(0)
    for names in ops:
        ref = golden_nbody[f"{name}/{'_'.join(names)}"]
        assert np.max(np.abs(model.res["_".join(names)] - ref)) <= 1e-8, names
