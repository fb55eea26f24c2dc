"""GPU parity of the matrix-free Z_n engine against the CPU oracle.

Basis (representative keys, bit-exact), orbit table (representative, sign and
stabiliser of every Gauss-law state), matvec (f64 to 1e-12, f32 to 1e-6),
the interleaved vector kernels against torch f64, and lowest eigenvalues of
the batched thick-restart Lanczos (fp64 and mixed) to 1e-9 relative.
"""

import numpy as np
import pytest
import torch

from oracle.zn_oracle import ZnOracle

pytestmark = pytest.mark.gpu

CASES = [(2, 2, 3), (2, 3, 3), (2, 2, 2), (2, 3, 2), (4, 2, 2), (2, 2, 4)]
COUPLINGS = [(1.0, 0.5, 1.0), (1.0, 0.0, 0.7), (0.8, 1.2, 1.6), (1.0, 0.3, 0.4)]


def _engine(lx, ly, n, momentum=True):
    from edgpu.models.zn_model import ZnLattice
    from edgpu.zn import ZnEngine

    eng = ZnEngine(ZnLattice((lx, ly), n, momentum=momentum))
    eng.build_basis()
    return eng


def _coup(t, m, g):
    return [t, m, g * g / 2, -1.0 / (2 * g * g)]


_ORACLES = {}


def _oracle(lx, ly, n, momentum=True):
    key = (lx, ly, n, momentum)
    if key not in _ORACLES:
        _ORACLES[key] = ZnOracle(lx, ly, n, momentum=momentum)
    return _ORACLES[key]


@pytest.mark.parametrize("momentum", [True, False])
@pytest.mark.parametrize("lx,ly,n", CASES)
def test_representatives_bit_exact(lx, ly, n, momentum):
    eng = _engine(lx, ly, n, momentum)
    o = _oracle(lx, ly, n, momentum)
    rep_keys = o.momentum_basis()[1] if momentum else o.keys
    gk = eng.host_keys()
    assert eng.n_rows == len(rep_keys)
    assert np.array_equal(np.sort(gk), np.sort(rep_keys))
    g = np.array([eng.L.gauss_index(int(k)) for k in gk])
    assert np.all(np.diff(g) > 0), "rows must be in ascending Gauss index"


@pytest.mark.parametrize("lx,ly,n", CASES)
def test_orbit_table_matches_projector(lx, ly, n):
    eng = _engine(lx, ly, n)
    o = _oracle(lx, ly, n)
    B, rep_keys, stab = o.momentum_basis()
    G = len(o.group())
    gk = eng.host_keys()
    row_of_key = {int(k): r for r, k in enumerate(gk)}
    col_of_key = {int(k): c for c, k in enumerate(rep_keys)}
    orbit = eng.orbit.cpu().numpy().view(np.uint32)
    Bc = B.tocsr()
    for i in range(o.dim):
        e = int(orbit[eng.L.gauss_index(int(o.keys[i]))])
        row = Bc.getrow(i)
        if row.nnz == 0:
            assert e == 0xFFFFFFFF
            continue
        c, val = int(row.indices[0]), float(row.data[0])
        r = e & 0x0FFFFFFF
        assert int(gk[r]) == int(rep_keys[c])
        s_div = eng.L.divisors()[(e >> 28) & 7]
        assert s_div == stab[c]
        sign = -1.0 if e >> 31 else 1.0
        # projector entry of an orbit member: sign * sqrt(|Stab| / |G|)
        assert np.isclose(val, sign * np.sqrt(stab[c] / G), rtol=1e-12)
        assert row_of_key[int(rep_keys[c])] == r and col_of_key[int(gk[r])] == c


def _oracle_matrix_in_gpu_order(eng, o, coup, momentum=True):
    t, m, g = coup
    H = o.hamiltonian(t, m, g, momentum=momentum)
    keys = o.momentum_basis()[1] if momentum else o.keys
    pos = {int(k): i for i, k in enumerate(keys)}
    perm = np.array([pos[int(k)] for k in eng.host_keys()])
    return H[perm][:, perm]


@pytest.mark.parametrize("nvec", [1, 2, 4, 8])
@pytest.mark.parametrize("lx,ly,n", CASES)
def test_matvec_matches_oracle(lx, ly, n, nvec):
    eng = _engine(lx, ly, n)
    o = _oracle(lx, ly, n)
    rng = np.random.default_rng(7)
    cps = [COUPLINGS[i % len(COUPLINGS)] for i in range(nvec)]
    N = eng.n_rows
    x = rng.standard_normal((N, nvec))
    want = np.stack([_oracle_matrix_in_gpu_order(eng, o, cps[v]) @ x[:, v] for v in range(nvec)], axis=1)
    coup = torch.tensor([_coup(*c) for c in cps], dtype=torch.float64, device="cuda")
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 2e-6)):
        xd = torch.from_numpy(x).to("cuda", dt).contiguous()
        y = torch.zeros_like(xd)
        eng.matvec(xd, y, coup, nvec)
        got = y.double().cpu().numpy()
        scale = np.abs(want).max()
        assert np.abs(got - want).max() <= tol * scale * (1 if dt == torch.float64 else 10)


@pytest.mark.parametrize("lx,ly,n", [(2, 3, 3), (4, 2, 2)])
def test_matvec_full_sector_matches_oracle(lx, ly, n):
    eng = _engine(lx, ly, n, momentum=False)
    o = _oracle(lx, ly, n, momentum=False)
    x = np.random.default_rng(3).standard_normal((eng.n_rows, 1))
    want = _oracle_matrix_in_gpu_order(eng, o, COUPLINGS[0], momentum=False) @ x[:, 0]
    coup = torch.tensor([_coup(*COUPLINGS[0])], dtype=torch.float64, device="cuda")
    xd = torch.from_numpy(x).cuda().contiguous()
    y = torch.zeros_like(xd)
    eng.matvec(xd, y, coup, 1)
    assert np.abs(y.cpu().numpy()[:, 0] - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("m", [7, 20])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("nvec", [1, 2, 4, 8])
def test_interleaved_vector_kernels(nvec, dt, m):
    from edgpu._lib import lib, ptr, stream_handle

    dtype = 0 if dt == torch.float64 else 1
    rng = np.random.default_rng(nvec)
    n_rows = 1001
    n_pad = (n_rows + 3) // 4 * 4
    E = n_pad * nvec
    # an orthonormal basis per instance plus one more random vector (what a
    # delayed Gram-Schmidt step sees: Q orthonormal, u not yet orthogonalised)
    Vh = np.zeros((m, n_pad, nvec))
    for v in range(nvec):
        Vh[: m - 1, :n_rows, v] = np.linalg.qr(rng.standard_normal((n_rows, m - 1)))[0].T
    Vh[m - 1, :n_rows] = rng.standard_normal((n_rows, nvec)) / np.sqrt(n_rows)
    wh = np.zeros((n_pad, nvec))
    wh[:n_rows] = rng.standard_normal((n_rows, nvec))
    V = torch.from_numpy(Vh.reshape(m, E)).to("cuda", dt).contiguous()
    w = torch.from_numpy(wh.reshape(E)).to("cuda", dt).contiguous()
    Vr = V.double().cpu().numpy().reshape(m, n_pad, nvec)
    wr = w.double().cpu().numpy().reshape(n_pad, nvec)
    h = torch.zeros((m, nvec), dtype=torch.float64, device="cuda")
    scratch = torch.empty(lib.edg_iv_scratch_elems(E, m), dtype=torch.float64, device="cuda")
    st = stream_handle()
    assert lib.edg_iv_dots(dtype, E, nvec, ptr(V), E, m, ptr(w), ptr(h), ptr(scratch), st) == 0
    want_h = np.einsum("irv,rv->iv", Vr, wr)
    assert np.allclose(h.cpu().numpy(), want_h, rtol=1e-12, atol=1e-9)
    # two right-hand-side dots and one delayed Gram-Schmidt step with u = V[m-1]
    hu = torch.zeros((m, nvec), dtype=torch.float64, device="cuda")
    hw = torch.zeros((m, nvec), dtype=torch.float64, device="cuda")
    assert lib.edg_iv_dots2(dtype, E, nvec, ptr(V), E, m, ptr(V[m - 1]), ptr(w), ptr(hu), ptr(hw),
                            ptr(scratch), st) == 0
    assert np.allclose(hu.cpu().numpy(), np.einsum("irv,rv->iv", Vr, Vr[m - 1]), rtol=1e-12, atol=1e-9)
    assert np.allclose(hw.cpu().numpy(), want_h, rtol=1e-12, atol=1e-9)
    Vd, wd = V.clone(), w.clone()
    sqd = torch.zeros(nvec, dtype=torch.float64, device="cuda")
    j = m - 1
    assert lib.edg_iv_dcgs_update(dtype, E, nvec, ptr(Vd), E, j, ptr(hu), ptr(hw), ptr(wd), ptr(sqd),
                                  ptr(scratch), st) == 0
    hun, hwn = hu.cpu().numpy(), hw.cpu().numpy()
    s_, z_ = hun[:j], hwn[:j]
    r = np.sqrt(hun[j] - (s_ * s_).sum(axis=0))
    q = (Vr[j] - np.einsum("irv,iv->rv", Vr[:j], s_)) / r
    c = (hwn[j] - (s_ * z_).sum(axis=0)) / r
    want_wd = wr - np.einsum("irv,iv->rv", Vr[:j], z_) - q * c
    got_q = Vd[j].double().cpu().numpy().reshape(n_pad, nvec)
    got_w = wd.double().cpu().numpy().reshape(n_pad, nvec)
    tq = 1e-12 if dtype == 0 else 2e-6
    assert np.abs(got_q - q).max() <= tq * np.abs(q).max()
    assert np.abs(got_w - want_wd).max() <= tq * 10 * np.abs(want_wd).max()
    assert np.allclose(sqd.cpu().numpy(), (got_w**2).sum(axis=0), rtol=1e-11)
    assert torch.equal(Vd[:j], V[:j])
    # fused second pass on a copy: w1 = w - V h, sq = |w1|^2
    w1 = w.clone()
    sq1 = torch.zeros(nvec, dtype=torch.float64, device="cuda")
    assert lib.edg_iv_update_norm(dtype, E, nvec, ptr(V), E, m, ptr(h), ptr(w1), ptr(sq1), ptr(scratch), st) == 0
    w1r = w1.double().cpu().numpy().reshape(n_pad, nvec)
    want_w1 = wr - np.einsum("irv,iv->rv", Vr, h.cpu().numpy())
    tol = 1e-12 if dtype == 0 else 1e-5
    assert np.abs(w1r - want_w1).max() <= tol * np.abs(want_w1).max()
    assert np.allclose(sq1.cpu().numpy(), (w1r**2).sum(axis=0), rtol=1e-11)
    assert lib.edg_iv_update(dtype, E, nvec, ptr(V), E, m, ptr(h), ptr(w), st) == 0
    want_w = wr - np.einsum("irv,iv->rv", Vr, want_h)
    tol = 1e-12 if dtype == 0 else 1e-4
    assert np.abs(w.double().cpu().numpy().reshape(n_pad, nvec) - want_w).max() <= tol * np.abs(want_w).max()
    sq = torch.tensor(np.arange(1, nvec + 1, dtype=float), device="cuda")
    out = torch.empty_like(w)
    assert lib.edg_iv_scale(dtype, E, nvec, ptr(w), ptr(sq), ptr(out), st) == 0
    ww = w.double().cpu().numpy().reshape(n_pad, nvec)
    assert np.allclose(out.double().cpu().numpy().reshape(n_pad, nvec), ww / np.sqrt(np.arange(1, nvec + 1)),
                       rtol=1e-6 if dtype else 1e-14)
    k = 3
    S = rng.standard_normal((nvec, m, k))
    Sd = torch.from_numpy(S).cuda()
    V0 = V.double().cpu().numpy().reshape(m, n_pad, nvec)
    assert lib.edg_iv_combine(dtype, E, nvec, ptr(V), E, m, ptr(Sd), k, st) == 0
    want_c = np.einsum("irv,viq->qrv", V0, S)
    got_c = V[:k].double().cpu().numpy().reshape(k, n_pad, nvec)
    assert np.abs(got_c - want_c).max() <= (1e-12 if dtype == 0 else 1e-5) * np.abs(want_c).max()
    x = torch.empty(E, dtype=dt, device="cuda")
    assert lib.edg_iv_random(dtype, n_rows, E, nvec, 5, ptr(x), st) == 0
    xr = x.double().cpu().numpy().reshape(n_pad, nvec)
    assert np.all(xr[n_rows:] == 0) and np.abs(xr[:n_rows]).max() <= 1 and np.abs(xr[:n_rows]).min() > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("lx,ly,n", [(2, 3, 3), (4, 2, 2), (2, 2, 4), (2, 3, 2)])
def test_lowest_energies_match_oracle(lx, ly, n, precision):
    from edgpu.zn import zn_lowest

    eng = _engine(lx, ly, n)
    o = _oracle(lx, ly, n)
    cps = COUPLINGS[:3]  # the fourth set has near-degenerate pairs (gaps ~3e-6)
    res = zn_lowest(eng, [_coup(*c) for c in cps], k=2, precision=precision, m=20)
    for v, (t, m, g) in enumerate(cps):
        want = o.lowest(t, m, g, k=2)
        rel = np.abs(res.evals[v] - want) / np.abs(want)
        assert rel.max() <= 1e-9, (v, res.evals[v], want)


def test_ground_state_vector_is_eigenvector():
    from edgpu.zn import zn_lowest

    eng = _engine(2, 3, 3)
    o = _oracle(2, 3, 3)
    t, m, g = COUPLINGS[0]
    res = zn_lowest(eng, [_coup(t, m, g)], k=1, precision="mixed", m=16)
    n = eng.n_rows
    x = res.evecs.view(-1, 1)[:n, 0].cpu().numpy()
    H = _oracle_matrix_in_gpu_order(eng, o, (t, m, g))
    r = H @ x - res.evals[0, 0] * x
    assert np.linalg.norm(r) <= 1e-6 * abs(res.evals[0, 0]) * np.linalg.norm(x)


def test_matvec_rejects_bad_arguments():
    from edgpu._lib import EdgError

    eng = _engine(2, 2, 3)
    coup = torch.tensor([_coup(*COUPLINGS[0])] * 3, dtype=torch.float64, device="cuda")
    x = torch.zeros((eng.n_rows, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(EdgError):
        eng.matvec(x, torch.zeros_like(x), coup, 3)
