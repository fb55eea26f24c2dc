"""The dictionary-packed tiled layout (packed.cu) of the off-diagonal matrix:
one 32-bit word per entry slot (column | value index << colbits), the
distinct values in a table, tiles of 16 rows stored k-major and padded to
their longest row.  Its matvec computes the CSR product of the reference
(csr_spmv, edlgt/modeling/qmb_hamiltonian.py:705-730).  In f64 it forms the
same sums in the same order as the CSR kernel with two threads a row, so the
outputs are compared bit for bit (and to a host f64 product at 1e-12
relative).  In f32 (the f32 Krylov phase) each half row's products are summed
in f32: the bound checked is 1e-6 of the row's sum of |terms|."""

import numpy as np
import pytest

from cases import build

pytestmark = pytest.mark.gpu


def _model(name, dev):
    model, g0, m0 = build(name, device=dev)
    model.build_Hamiltonian(g0, m0)
    return model


def _decode(lay):
    """Host decoding of the tile layout back to CSR order: tile t is (its
    word count) / 16 wide, entry k of its row s at tile_off[t] + 16 k + s,
    padding words all ones."""
    w = lay.words.cpu().numpy().view(np.uint32)
    off = lay.tile_off.cpu().numpy().astype(np.int64)
    n = lay.n
    pad = np.uint32(0xFFFFFFFF)
    per_row, lens = [], np.zeros(n, dtype=np.int64)
    for t in range((n + 15) // 16):
        assert (off[t + 1] - off[t]) % 16 == 0 and off[t] % 16 == 0
        blk = w[off[t]: off[t + 1]].reshape(-1, 16)  # [k][s]
        for s_ in range(16):
            col = blk[:, s_]
            real = col != pad
            ln = int(real.sum())
            assert real[:ln].all() and not real[ln:].any()  # padding only after the row's entries
            if 16 * t + s_ < n:
                per_row.append(col[:ln])
                lens[16 * t + s_] = ln
            else:
                assert ln == 0
        assert blk.shape[0] == lens[16 * t: 16 * t + 16].max(initial=0)  # as wide as its longest row
    words = np.concatenate(per_row) if per_row else np.zeros(0, np.uint32)
    assert np.all(w[lay.total:] == pad)
    mask = np.uint32((1 << lay.colbits) - 1)
    return (words & mask).astype(np.int64), (words >> np.uint32(lay.colbits)).astype(np.int64), lens


@pytest.mark.parametrize("name", ["su2_1d_L10_obc", "su2_1d_L10_pbc", "qed2d_3x2_q0", "qed1d_L8_obc"])
def test_layout_decodes_to_the_matrix(name):
    import torch

    from edgpu.solvers import PackedLayout

    mat = _model(name, "cuda").H.mat
    if mat.is_complex:
        pytest.skip("complex matrix")
    lay = PackedLayout.build(mat)
    assert lay is not None
    table = lay.table64.cpu().numpy()
    assert np.all(np.diff(table) >= 0) and lay.count == len(np.unique(mat.vals.cpu().numpy()))
    assert (1 << lay.colbits) > mat.n and (lay.count - 1) >> (32 - lay.colbits) == 0
    cols, idx, lens = _decode(lay)
    assert np.array_equal(lens, np.diff(mat.rowptr.cpu().numpy()))
    assert np.array_equal(cols, mat.cols.cpu().numpy())
    assert np.array_equal(table[idx], mat.vals.cpu().numpy())  # bit-exact values
    assert lay.total >= lay.nnz
    assert torch.equal(lay.table32, lay.table64.to(torch.float32))


def _csr_planar(mat, dtype, v, diag, x, nvec, xs):
    """The CSR kernel with two threads a row, f64 planar output."""
    import torch

    from edgpu._lib import check, lib, ptr, stream_handle

    n = mat.n
    y = torch.empty((nvec, n), dtype=torch.float64, device=x.device)
    if dtype == 1:
        check(lib.edg_spmv_f32_planar(n, mat.nnz, ptr(mat.rowptr), ptr(mat.cols), ptr(v), ptr(diag), nvec, ptr(x), xs,
                                      ptr(y), n, 2, stream_handle()), "edg_spmv_f32_planar")
    else:  # f64 CSR kernel, interleaved output
        yi = torch.empty((n, nvec), dtype=torch.float64, device=x.device)
        assert xs == nvec
        check(lib.edg_spmv_group(0, n, mat.nnz, ptr(mat.rowptr), ptr(mat.cols), ptr(v), ptr(diag), nvec, ptr(x),
                                 ptr(yi), 2, stream_handle()), "edg_spmv_group")
        y.copy_(yi.T)
    return y


def _packed(lay, dtype, diag, x, nvec, xs):
    import torch

    y = torch.empty((nvec, lay.n), dtype=torch.float64, device=x.device)
    err = torch.zeros(1, dtype=torch.int32, device=x.device)
    lay.launch(dtype, nvec, diag, x, xs, y, lay.n, err)
    assert int(err.item()) == 0
    return y


@pytest.mark.parametrize("name", ["su2_1d_L10_obc", "su2_1d_L10_pbc", "qed2d_3x2_q0", "qed1d_L8_obc"])
@pytest.mark.parametrize("nvec,xs", [(1, 1), (2, 2), (3, 3), (3, 4), (4, 4)])
@pytest.mark.parametrize("dtype", [1, 0])
def test_packed_matvec_matches_csr(name, nvec, xs, dtype):
    import torch

    from edgpu.solvers import PackedLayout

    mat = _model(name, "cuda").H.mat
    if mat.is_complex:
        pytest.skip("complex matrix")
    if dtype == 0 and xs != nvec:
        pytest.skip("the f64 CSR kernel takes unpadded rows")
    tdt = torch.float32 if dtype == 1 else torch.float64
    lay = PackedLayout.build(mat)
    n = mat.n
    g = torch.Generator(device="cpu").manual_seed(11 + nvec)
    x = (torch.rand((n, xs), generator=g, dtype=torch.float64) - 0.5).to(tdt).to("cuda")
    diag = torch.rand((n, nvec), generator=g, dtype=torch.float64).to(tdt).to("cuda")
    v = mat.vals.to(tdt)
    y_csr = _csr_planar(mat, dtype, v, diag, x, nvec, xs)
    y_pk = _packed(lay, dtype, diag, x, nvec, xs)
    H = mat.to_scipy(include_diag=False).astype(np.float64)
    if dtype == 1:
        H.data = H.data.astype(np.float32).astype(np.float64)
    xd = x.cpu().numpy().astype(np.float64)[:, :nvec]
    dd = diag.cpu().numpy().astype(np.float64)
    ref = (H @ xd + dd * xd).T
    if dtype == 0:
        assert torch.equal(y_pk, y_csr)
        assert np.allclose(y_pk.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    else:
        absH = H.copy()
        absH.data = np.abs(absH.data)
        scale = (absH @ np.abs(xd) + np.abs(dd * xd)).T
        assert np.all(np.abs(y_pk.cpu().numpy() - ref) <= 1e-6 * scale + 1e-300)


def _synthetic(n, row_len, n_values, seed, dev):
    """A DeviceMatrix with given row lengths and values drawn from n_values
    distinct numbers (one f64 diagonal)."""
    import torch

    from edgpu.modeling.assembly import DeviceMatrix

    rng = np.random.default_rng(seed)
    lens = np.asarray(row_len, dtype=np.int64)
    rowptr = np.concatenate([[0], np.cumsum(lens)])
    cols = np.concatenate([np.sort(rng.choice(n, size=l, replace=False)) for l in lens]).astype(np.int32)
    pool = rng.standard_normal(n_values)
    vals = pool[rng.integers(0, n_values, size=int(rowptr[-1]))]
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dt).to(dev)
    return DeviceMatrix(n, t(rowptr, torch.int64), t(cols, torch.int32), t(vals, torch.float64),
                        t(rng.standard_normal(n), torch.float64), None, False)


def test_long_tiles_and_ragged_ends():
    """Tiles whose entries exceed the shared-memory stage (rows of 100 to 600
    entries) read the stream directly; empty rows, rows of equal length (the
    tile order's ties), a last tile of 5 rows and zero values of both signs
    are handled."""
    import torch

    from edgpu.solvers import PackedLayout

    n = 16 * 70 + 5
    rng = np.random.default_rng(3)
    lens = rng.integers(0, 12, size=n)
    lens[16:32] = rng.integers(100, 600, size=16)  # a tile of long rows
    lens[40:44] = 0
    lens[48:64] = 7  # a tile of equal lengths
    mat = _synthetic(n, lens, 9, 5, "cuda")
    v = mat.vals.cpu().numpy()
    v[:3] = [0.0, -0.0, 0.0]
    mat.vals = torch.from_numpy(v).to("cuda")
    lay = PackedLayout.build(mat)
    assert lay is not None
    cols, idx, lens = _decode(lay)
    assert np.array_equal(lens, np.diff(mat.rowptr.cpu().numpy()))
    assert np.array_equal(lay.table64.cpu().numpy()[idx].view(np.int64), v.view(np.int64))
    for nvec in (1, 3):
        x = torch.rand((n, nvec), dtype=torch.float64, device="cuda")
        diag = torch.rand((n, nvec), dtype=torch.float64, device="cuda")
        y_pk = _packed(lay, 0, diag, x, nvec, nvec)
        y_csr = _csr_planar(mat, 0, mat.vals, diag, x, nvec, nvec)
        assert torch.equal(y_pk, y_csr)


def test_matrices_that_do_not_pack():
    """More distinct values than the index bits or the table hold: no layout."""
    from edgpu.solvers import PackedLayout

    mat = _synthetic(5000, np.full(5000, 6), 30000, 8, "cuda")  # ~30000 values > 4096
    assert PackedLayout.build(mat) is None


def test_mixed_lanczos_on_packed_matches_reference(golden_small):
    """SU(2) L=10 periodic chain: mixed-precision ground state with the
    packed matvec (f32 phase and f64 refinement) against the reference's
    energy (1e-9 relative) and against the solve on the CSR matvec."""
    from edgpu.solvers import lanczos_mixed

    model = _model("su2_1d_L10_pbc", "cuda")
    mat = model.H.mat
    r_pk, r32 = lanczos_mixed(mat, sell=False, packed=True)
    r_csr, _ = lanczos_mixed(mat, sell=False, group32=2)
    ref = golden_small["su2_1d_L10_pbc/energies"][0]
    assert abs(r_pk.evals[0, 0] / model.n_sites - ref) <= 1e-9 * abs(ref)
    assert abs(r_pk.evals[0, 0] - r_csr.evals[0, 0]) <= 1e-9 * abs(r_csr.evals[0, 0])
    assert r32.iters[0] > 5


@pytest.mark.parametrize("window32,refine_iter", [(4, 5), (6, 8), (7, 6), (0, 5)])
@pytest.mark.parametrize("packed", [True, False])
def test_short_window_reorthogonalisation_matches_reference(golden_small, window32, refine_iter, packed):
    """The one-launch reorthogonalisation of short windows, both of its
    instantiations (up to 5 and up to 8 vectors: windows 4, 6 and 7 of the
    f32 phase; refinements of 5, 6 and 8 f64 steps), against the reference's
    ground-state energy (1e-9 relative) on the SU(2) L=10 periodic chain with
    three couplings; window 0 runs the f32 phase through the ring passes."""
    import torch

    from edgpu.solvers import lanczos_mixed, stack_diagonals

    model = _model("su2_1d_L10_pbc", "cuda")
    mat = model.H.mat
    r64, r32 = lanczos_mixed(mat, window32=window32, refine_iter=refine_iter, sell=False, packed=packed or None,
                             group32=0 if packed else 2)
    ref = golden_small["su2_1d_L10_pbc/energies"][0]
    assert abs(r64.evals[0, 0] / model.n_sites - ref) <= 1e-9 * abs(ref)
    # a batch of three diagonals (couplings) sharing the off-diagonal part
    d = mat.diag
    diags = [d, d + 0.25 * torch.ones_like(d), d - 0.5 * torch.ones_like(d)]
    rb, _ = lanczos_mixed(mat, diags=diags, window32=window32, refine_iter=refine_iter, sell=False,
                          packed=packed or None, group32=0 if packed else 2)
    e = rb.evals[:, 0]
    assert abs(e[0] - r64.evals[0, 0]) <= 1e-9 * abs(e[0])
    # a constant shift of the diagonal shifts the ground-state energy by it
    assert abs((e[1] - e[0]) - 0.25) <= 1e-9 * abs(e[0])
    assert abs((e[2] - e[0]) + 0.5) <= 1e-9 * abs(e[0])


@pytest.mark.parametrize("precision,tol", [("c128", 1e-11), ("c64", 2e-5)])
def test_krylov_evolution_on_packed_matches_csr(precision, tol):
    """Krylov time evolution with the packed matvec (a complex vector as two
    real right-hand sides of the real-form matrix) against the CSR matvec:
    the same states (complex128: both accumulate in f64; complex64: the
    packed kernel sums half rows in f32) and a unit norm."""
    import torch

    from edgpu.dynamics import KrylovEvolver

    model = _model("su2_1d_L10_pbc", "cuda")
    mat = model.H.mat
    assert not mat.is_complex
    n = mat.n
    g = torch.Generator(device="cpu").manual_seed(3)
    psi0 = torch.randn(n, dtype=torch.complex128, generator=g).to("cuda")
    psi0 /= torch.linalg.vector_norm(psi0)
    states = {}
    for matvec in ("auto", "csr"):
        ev = KrylovEvolver(mat, m=30, precision=precision, reorth_passes=0, matvec=matvec)
        assert (ev.packed is not None) == (matvec == "auto")
        psi = psi0.to(ev.vdtype).clone()
        for _ in range(5):
            ev.step(psi, 0.05)
        ev.check_status()
        states[matvec] = psi.to(torch.complex128)
    a, b = states["auto"], states["csr"]
    assert abs(float(torch.linalg.vector_norm(a)) - 1.0) < tol
    assert float(torch.max(torch.abs(a - b))) < tol
