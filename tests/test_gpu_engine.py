"""Device engine parity: sector, lookup, assembly, matvec, Lanczos and local
observables against the reference's fixtures and the CPU oracle."""

import hashlib

import numpy as np
import pytest

from cases import ALL_CASES, BIG_CASES, build
from oracle import edlgt_oracle as O

pytestmark = pytest.mark.gpu


def _gold_csr(g, name):
    from scipy.sparse import csr_matrix

    n = int(g[f"{name}/dim"])
    return csr_matrix((g[f"{name}/H_data"], g[f"{name}/H_indices"], g[f"{name}/H_indptr"]), shape=(n, n))


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_sector_bit_exact(name, golden_small, dev):
    model, _, _ = build(name, device=dev)
    keys = model.sector.host_keys()
    assert np.array_equal(keys, golden_small[f"{name}/keys"])
    cfg = model.sector_configs
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), keys)


@pytest.mark.parametrize("name", sorted(BIG_CASES))
def test_sector_bit_exact_large(name, golden_big, dev):
    model = build(name, device=dev, big=True)
    keys = model.sector.host_keys()
    assert len(keys) == int(golden_big[f"{name}/dim"])
    assert hashlib.sha256(keys.tobytes()).hexdigest() == str(golden_big[f"{name}/keys_sha"])
    assert np.all(keys[1:] > keys[:-1])


def test_lookup_hits_and_misses(dev):
    model, _, _ = build("su2_1d_L10_obc", device=dev)
    cfg = model.sector_configs
    rng = np.random.default_rng(7)
    hits = cfg[rng.integers(0, len(cfg), 500)]
    rand = np.stack([rng.integers(0, d, 500) for d in model.loc_dims], axis=1).astype(np.uint16)
    q = np.concatenate([hits, rand])
    got = model.sector.index_of(q)
    ref = O.config_to_index(q, cfg, model.loc_dims)
    assert np.array_equal(got, ref)
    assert np.all(got[:500] >= 0)
    assert np.any(got[500:] < 0)


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_assembly_matches_reference(name, golden_small, dev):
    """Faithful (complex) assembly: canonical pattern bit-exact, values 1e-13."""
    model, g, m = build(name, device=dev)
    for b in model.hamiltonian_blocks(g, m):
        model.H.add_term(b)
    model.H.build(force_complex=True)
    got = model.H.mat.to_scipy()
    ref = _gold_csr(golden_small, name)
    assert np.array_equal(got.indptr, ref.indptr)
    assert np.array_equal(got.indices, ref.indices)
    assert np.max(np.abs(got.data - ref.data)) <= 1e-13 * max(1.0, np.max(np.abs(ref.data)))


@pytest.mark.parametrize("name", ["qed1d_L8_obc", "qed2d_3x2_bg", "su2_1d_L10_obc", "su2_1d_L10_pbc", "su2_1d_L8_obc_bg"])
def test_real_form_is_gauge_equivalent(name, golden_small, dev):
    """The real form equals D^dagger H D with D the diagonal gauge phases."""
    model, g, m = build(name, device=dev)
    model.build_Hamiltonian(g, m)
    mat = model.H.mat
    assert not mat.is_complex
    w = mat.phase_weights
    cfg = model.sector_configs
    e = w[np.arange(cfg.shape[1])[None, :], cfg.astype(np.int64)].sum(axis=1) % 4
    ph = np.power(1j, e)
    ref = _gold_csr(golden_small, name).tocoo()
    rot = np.conj(ph[ref.row]) * ref.data * ph[ref.col]
    assert np.max(np.abs(rot.imag)) < 1e-12
    got = mat.to_scipy().tocoo()
    from scipy.sparse import coo_matrix

    diff = coo_matrix((rot.real, (ref.row, ref.col)), shape=ref.shape).tocsr() - got.tocsr()
    assert abs(diff).max() <= 1e-13 * max(1.0, np.max(np.abs(ref.data)))


@pytest.mark.parametrize("name", ["su2_1d_L12_obc", "su2_1d_L14_obc"])
def test_assembly_large_digest(name, golden_big, dev):
    model = build(name, device=dev, big=True)
    for b in model.hamiltonian_blocks(1.0, 0.5):
        model.H.add_term(b)
    model.H.build(force_complex=True)
    m = model.H.mat.to_scipy()
    rows = np.repeat(np.arange(m.shape[0], dtype=np.int64), np.diff(m.indptr))
    cols = m.indices.astype(np.int64)
    assert m.nnz == int(golden_big[f"{name}/H_nnz"])
    assert hashlib.sha256(np.stack([rows, cols]).tobytes()).hexdigest() == str(golden_big[f"{name}/H_pattern_sha"])
    w = 1.0 / (1.0 + ((rows * 7919 + cols * 104729) % 1009))
    ws = np.sum(m.data * w)
    ref = complex(golden_big[f"{name}/H_wsum"])
    assert abs(ws - ref) <= 1e-10 * abs(ref)


def test_spmv_matches_scipy(golden_small, dev):
    import torch

    name = "su2_1d_L10_obc"
    model, g, m = build(name, device=dev)
    model.build_Hamiltonian(g, m)
    H = model.H.mat.to_scipy()
    rng = np.random.default_rng(3)
    x = rng.standard_normal(H.shape[0])
    y = model.H.mat.matvec(torch.from_numpy(x).to(dev)).cpu().numpy()
    assert np.max(np.abs(y - H @ x)) <= 1e-12 * np.max(np.abs(H @ x))


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_lanczos_energies(name, golden_small, dev):
    model, g, m = build(name, device=dev)
    model.build_Hamiltonian(g, m)
    e_ref = golden_small[f"{name}/energies"]
    model.diagonalize_Hamiltonian(len(e_ref), "gpu")
    assert np.allclose(model.H.Nenergies, e_ref, atol=1e-10, rtol=0)


def test_lanczos_large_and_sweep(golden_big, dev):
    import torch

    from edgpu.solvers import lanczos_mixed

    model = build("su2_1d_L14_obc", device=dev, big=True)
    e = {}
    diags = []
    for g in (0.5, 1.0, 2.0):
        model.build_Hamiltonian(g, 0.5)
        model.diagonalize_Hamiltonian(1)
        e[g] = model.H.Nenergies[0]
        assert abs(e[g] - golden_big[f"su2_1d_L14_obc/sweep_g{g}"][0]) < 1e-10
        diags.append(model.H.mat.diag.clone())
    # mixed precision, three couplings batched in one matvec (shared hopping)
    r64, r32 = lanczos_mixed(model.H.mat, diags=diags)
    for i, g in enumerate((0.5, 1.0, 2.0)):
        e_mix = r64.evals[i, 0] / 14
        assert abs(e_mix - e[g]) <= 1e-9 * abs(e[g])
    del torch


def test_local_observables_pins(golden_pins, dev):
    model, g, m = build("qed1d_L4_obc", device=dev)
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(1)
    psi = model.H.GSpsi
    e2 = model.local_expval(model.ops["E2_px"], psi)
    n_ev = model.local_expval(model.ops["N"], psi)
    nz = model.local_expval(model.ops["N_zero"], psi)
    assert abs(np.mean(e2[:3]) - golden_pins["qed1d_L4_obc/E2"]) < 1e-10
    assert abs(0.5 * np.mean(n_ev[0::2]) + 0.5 * np.mean(nz[1::2]) - golden_pins["qed1d_L4_obc/N"]) < 1e-10
    model, g, m = build("qed2d_3x2_bg", device=dev)
    model.build_Hamiltonian(g, m)
    model.diagonalize_Hamiltonian(1)
    assert abs(model.H.GSenergy - golden_pins["qed2d_3x2_bg/energy"]) < 1e-10
    names = ["C_px,py", "C_py,mx", "C_my,px", "C_mx,my"]
    model.get_observables(["E2_px", "E2_py"], plaquette_obs=[names])
    model.measure_observables(0)
    assert abs(model.res["_".join(names)] - golden_pins["qed2d_3x2_bg/plaq"]) < 1e-10
    assert abs(model.link_avg("E2") - golden_pins["qed2d_3x2_bg/E2"]) < 1e-10


def test_missing_ket_is_an_error(dev):
    """A term leaving the sector (a lone matter hop changes the charge) raises."""
    from edgpu._lib import EdgError
    from edgpu.modeling import TwoBodyTerm

    model, g, m = build("qed1d_L8_obc", device=dev)
    t = TwoBodyTerm("x", [model.ops["Q_px_dag"], model.ops["N"]], ["Q_px_dag", "N"], **model.def_params)
    model.H.add_term(t.get_Hamiltonian(1.0))
    with pytest.raises(EdgError, match="MISSING_KET"):
        model.H.build()


def test_tridiagonal_solver(dev):
    import ctypes

    import torch

    from edgpu import _lib

    rng = np.random.default_rng(11)
    m, k = 120, 4
    a = rng.standard_normal(m)
    b = np.concatenate([[0.0], rng.uniform(0.1, 1.0, m - 1)])
    T = np.diag(a) + np.diag(b[1:], 1) + np.diag(b[1:], -1)
    w, v = np.linalg.eigh(T)
    A = torch.from_numpy(a).to(dev)
    B = torch.from_numpy(b).to(dev)
    ev = torch.empty(k, dtype=torch.float64, device=dev)
    S = torch.empty((k, m), dtype=torch.float64, device=dev)
    work = torch.empty(6 * m, dtype=torch.float64, device=dev)
    _lib.check(_lib.lib.edg_tridiag_lowest(_lib.ptr(A), _lib.ptr(B), m, k, _lib.ptr(ev), _lib.ptr(S), _lib.ptr(work),
                                           _lib.stream_handle()))
    assert np.allclose(ev.cpu().numpy(), w[:k], atol=1e-12)
    Sv = S.cpu().numpy()
    for q in range(k):
        assert abs(abs(Sv[q] @ v[:, q]) - 1) < 1e-10
    del ctypes


@pytest.mark.parametrize("key,case", [("su2_1d_L6_pbc_V", "su2_1d_L6_pbc"), ("su2_1d_L10_obc_pair", None)])
@pytest.mark.parametrize("precision,tol", [("c128", 1e-9), ("c64", 2e-5)])
def test_krylov_dynamics_matches_reference(key, case, precision, tol, golden_dyn, dev):
    """Quench observables vs the reference's expm_multiply trajectories."""
    from edgpu.models import SU2_Model

    g = float(golden_dyn[f"{key}/g"])
    m = float(golden_dyn[f"{key}/m"])
    if case is not None:
        model, _, _ = build(case, device=dev)
    else:
        model = SU2_Model(spin=0.5, pure_theory=False, lvals=[10], has_obc=[True], sectors=[10],
                          bg_list=[0, 0, 0, 0.5, 0, 0, 0.5, 0, 0, 0], device=dev)
    model.build_Hamiltonian(g, m)
    psi0 = model.get_qmb_state_from_configs([golden_dyn[f"{key}/config"]])
    t = golden_dyn[f"{key}/time"]
    model.time_evolution_Hamiltonian(psi0, t, precision=precision,
                                     observables={"T2_px": model.ops["T2_px"], "N_pair": model.ops["N_pair"]})
    res = model.H.obs_time
    assert np.max(np.abs(res["T2_px"] - golden_dyn[f"{key}/T2_px"])) < tol
    assert np.max(np.abs(res["N_pair"] - golden_dyn[f"{key}/N_pair"])) < tol


def test_krylov_states_are_unitary_and_match_dense(dev):
    """Stored states (reference basis) agree with dense exp(-iHt) on a small case."""
    import scipy.linalg as sla

    model, g, m = build("su2_1d_L6_pbc", device=dev)
    model.build_Hamiltonian(g, m)
    cfg = model.sector_configs
    psi0 = model.get_qmb_state_from_configs([cfg[17]])
    t = np.linspace(0.0, 0.4, 9)
    model.time_evolution_Hamiltonian(psi0, t)
    H = model.H.mat.to_scipy().toarray()
    # the stored states are in the reference basis; map the real form back
    ph = model.H._row_phase().cpu().numpy()
    Hc = ph[:, None] * H * np.conj(ph)[None, :]
    for k, tk in enumerate(t):
        ref = sla.expm(-1j * tk * Hc) @ psi0
        got = model.H.psi_time[k].psi
        assert abs(np.vdot(got, got) - 1) < 1e-12
        assert np.max(np.abs(got - ref)) < 1e-10


def _c3_instances(dev, n_coupling=64, seed=0):
    """QED 3x2 OBC instances: couplings in the Q = 0 sector plus Q = -2..2."""
    from cases import build as _b

    rng = np.random.default_rng(seed)
    gs = np.exp(rng.uniform(np.log(0.1), np.log(5.0), n_coupling))
    ms = rng.uniform(0.0, 2.0, n_coupling)
    model, _, _ = _b("qed2d_3x2_q0", device=dev)
    mats, meta = [], []
    for g, m in zip(gs, ms):
        model.build_Hamiltonian(float(g), float(m))
        mats.append(model.H.mat)
        meta.append(("qed2d_3x2_q0", float(g), float(m)))
    for q in (-2, -1, 1, 2):
        name = f"qed2d_3x2_Q{q:+d}"
        mq, g, m = _b(name, device=dev)
        mq.build_Hamiltonian(g, m)
        mats.append(mq.H.mat)
        meta.append((name, g, m))
    return mats, meta


def test_batched_small_instances_match_oracle(golden_small, dev):
    from edgpu.batch import SmallBatch

    mats, meta = _c3_instances(dev)
    batch = SmallBatch(mats, k=2, want_vectors=True)
    batch.capture()
    e_graph = batch.solve(use_graph=True).cpu().numpy().copy()
    e_direct = batch.solve(use_graph=False).cpu().numpy()
    assert np.array_equal(e_graph, e_direct)
    for i, (name, g, m) in enumerate(meta):
        H = mats[i].to_scipy().toarray()
        w = np.linalg.eigvalsh(H)
        assert np.allclose(e_direct[i], w[:2], atol=1e-10, rtol=0), (i, name)
        if name.startswith("qed2d_3x2_Q"):
            assert abs(e_direct[i, 0] / 6 - golden_small[f"{name}/energies"][0]) < 1e-10
    # ground-state vectors: normalised and H x = E x
    ev = batch.evecs.cpu().numpy()
    off = 0
    for i, mat in enumerate(mats):
        x = ev[off: off + mat.n]
        off += mat.n
        H = mat.to_scipy()
        assert abs(np.linalg.norm(x) - 1) < 1e-12
        assert np.linalg.norm(H @ x - e_direct[i, 0] * x) < 1e-8
