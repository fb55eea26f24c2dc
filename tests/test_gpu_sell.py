"""The SELL-32-sigma layout and matvec of the f32 Krylov path (sell.cu)
against the CSR matvec (the restatement of the reference's csr_spmv,
edlgt/modeling/qmb_hamiltonian.py:705-730) on the same f32 matrix: both
accumulate in f64 and differ only in summation order (relative 1e-12)."""

import numpy as np
import pytest

from cases import build

pytestmark = pytest.mark.gpu


def _mat(name, dev, g=None, m=None):
    model, g0, m0 = build(name, device=dev)
    model.build_Hamiltonian(g0 if g is None else g, m0 if m is None else m)
    return model


@pytest.mark.parametrize("name", ["su2_1d_L10_obc", "su2_1d_L10_pbc", "qed2d_3x2_q0", "qed1d_L8_obc"])
@pytest.mark.parametrize("nvec", [1, 2, 3, 4])
@pytest.mark.parametrize("window", [32, 4096])
def test_sell_matvec_matches_csr(name, nvec, window):
    import torch

    from edgpu._lib import check, lib, ptr, stream_handle
    from edgpu.solvers import SellLayout

    dev = "cuda"
    mat = _mat(name, dev).H.mat
    if mat.is_complex:
        pytest.skip("complex matrix")
    n = mat.n
    v32 = mat.vals.to(torch.float32)
    lay = SellLayout(mat, v32, window)
    # perm: a permutation of the rows, slice padding marked -1; rows sorted by
    # length (descending, stable) inside the windows
    perm = lay.perm.cpu().numpy()
    assert np.array_equal(np.sort(perm[perm >= 0]), np.arange(n))
    assert np.all(perm[n:] == -1) if len(perm) > n else True
    lens = np.diff(mat.rowptr.cpu().numpy())
    for w0 in range(0, n, window):
        seg = perm[w0: min(w0 + window, n)]
        assert np.all(np.diff(lens[seg]) <= 0)
        same = np.diff(lens[seg]) == 0
        assert np.all(np.diff(seg)[same] > 0)  # stable
    assert lay.pairs >= mat.nnz
    g = torch.Generator(device="cpu").manual_seed(7)
    x = torch.rand((n, nvec), generator=g, dtype=torch.float32).to(dev)
    diag = torch.rand((n, nvec), generator=g, dtype=torch.float32).to(dev)
    y_csr = torch.empty((n, nvec), dtype=torch.float32, device=dev)
    y_sell = torch.empty((nvec, n), dtype=torch.float64, device=dev)
    check(lib.edg_spmv(1, n, mat.nnz, ptr(mat.rowptr), ptr(mat.cols), ptr(v32), ptr(diag), nvec, ptr(x), ptr(y_csr),
                       stream_handle()), "edg_spmv")
    check(lib.edg_spmv_sell(n, nvec, ptr(lay.perm), ptr(lay.width), ptr(lay.off), ptr(lay.entries), ptr(diag), ptr(x),
                            nvec, ptr(y_sell), n, stream_handle()), "edg_spmv_sell")
    # exact product in f64 from the same f32 inputs, for the comparison
    H = mat.to_scipy(include_diag=False).astype(np.float32).astype(np.float64)
    xd = x.cpu().numpy().astype(np.float64)
    ref = H @ xd + diag.cpu().numpy().astype(np.float64) * xd
    ys = y_sell.cpu().numpy().T
    assert np.allclose(ys, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    # the CSR kernel rounds its output to f32
    assert np.allclose(y_csr.cpu().numpy(), ref, rtol=2e-7, atol=2e-7 * np.abs(ref).max())


def test_mixed_lanczos_on_sell_matches_reference(golden_small):
    """SU(2) L=10 periodic chain: mixed-precision ground states with the SELL
    matvec against the reference's energy (1e-9 relative) and against the
    same solve on the CSR matvec."""
    from edgpu.solvers import lanczos_mixed

    model = _mat("su2_1d_L10_pbc", "cuda")
    mat = model.H.mat
    r_sell, _ = lanczos_mixed(mat, sell=True)
    r_csr, _ = lanczos_mixed(mat, sell=False, group32=4)
    ref = golden_small["su2_1d_L10_pbc/energies"][0]
    e = r_sell.evals[0, 0] / model.n_sites
    assert abs(e - ref) <= 1e-9 * abs(ref)
    assert abs(r_sell.evals[0, 0] - r_csr.evals[0, 0]) <= 1e-9 * abs(r_csr.evals[0, 0])
