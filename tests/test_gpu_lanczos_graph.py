"""The device-driven Lanczos driver (edg_lanczos): the step index, the
convergence checks and their schedule live on the device, and the steps run
as replays of a CUDA graph.  The same solve launched one kernel at a time
(the instrumented path, with CUDA events around every phase), or with the
host synchronising once per replay instead of polling pinned progress words,
must give bit-identical results: the kernels and their order are the same."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def su2_l10(golden_small):
    import torch

    from cases import build

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    model, g, m = build("su2_1d_L10_obc", device="cuda")
    diags = []
    for gg in (0.5, 1.0, 2.0):
        model.build_Hamiltonian(gg, 0.5)
        diags.append(model.H.mat.diag.clone())
    model.build_Hamiltonian(g, m)
    return model, diags


@pytest.mark.parametrize("dtype", [0, 1])
def test_graph_replay_matches_one_by_one(su2_l10, dtype, golden_small):
    import torch

    from edgpu.solvers import run_lanczos, stack_diagonals

    model, diags = su2_l10
    mat = model.H.mat
    tdt = torch.float64 if dtype == 0 else torch.float32
    vals = mat.vals.to(tdt)
    diag = stack_diagonals(diags, tdt)
    kw = dict(nvec=3, k=2, max_iter=300, tol=1e-12 if dtype == 0 else 1e-6, check_every=5)
    runs = []
    for stats, poll in ((None, True), (np.zeros(6), True), (None, False)):
        r = run_lanczos(dtype, mat.n, mat.nnz, mat.rowptr, mat.cols, vals, diag, stats=stats, poll_host=poll, **kw)
        runs.append((r.evals.copy(), r.iters.copy(), r.evecs.cpu().numpy()))
    for ev, it, vec in runs[1:]:
        assert np.array_equal(ev, runs[0][0])
        assert np.array_equal(it, runs[0][1])
        assert np.array_equal(vec, runs[0][2])
    if dtype == 0:
        # the g^2 = 1 problem is the reference's fixture case
        ref = golden_small["su2_1d_L10_obc/energies"][0]
        assert abs(runs[0][0][1, 0] / model.n_sites - ref) < 1e-10


def test_graph_replay_stops_at_the_krylov_limit(su2_l10):
    """An unconverged solve stops at max_iter with the not-converged status
    (the device's last check), in both launch modes."""
    from edgpu import _lib
    from edgpu.solvers import run_lanczos

    model, _ = su2_l10
    mat = model.H.mat
    for stats in (None, np.zeros(6)):
        with pytest.raises(_lib.EdgError) as exc:
            run_lanczos(0, mat.n, mat.nnz, mat.rowptr, mat.cols, mat.vals, mat.diag, nvec=1, k=1, max_iter=9,
                        tol=1e-14, check_every=5, stats=stats)
        assert exc.value.status == -5
        r = run_lanczos(0, mat.n, mat.nnz, mat.rowptr, mat.cols, mat.vals, mat.diag, nvec=1, k=1, max_iter=9,
                        tol=1e-14, check_every=5, stats=stats, allow_unconverged=True)
        assert r.iters[0] == 9 and np.isfinite(r.evals[0, 0])
