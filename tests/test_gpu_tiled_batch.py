"""The (instance, row-tile) batched Lanczos (edg_lanczos_tiled_batch) on
instances of uneven dimension, against the reference's energies (fixtures
made by running ed-lgt's eigsh per instance) and the dense CPU eigen-solve.

Tolerances: energy densities 1e-10 absolute for the f64 solver (the
reference's own validation tolerance), relative 1e-9 for mixed precision."""

import numpy as np
import pytest

from cases import ALL_CASES, build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def _fixture_instances(golden_small, dev, with_l12=None):
    """Every real fixture case (dims 6 .. 17,906), optionally the L=12 open
    chain (73,789 rows): (matrix, n_sites, reference energy densities)."""
    mats, meta = [], []
    for name in sorted(ALL_CASES):
        model, g, m = build(name, device=dev)
        model.build_Hamiltonian(g, m)
        if model.H.mat.is_complex:
            continue
        mats.append(model.H.mat)
        meta.append((name, model.n_sites, np.asarray(golden_small[f"{name}/energies"])))
    if with_l12 is not None:
        model = build("su2_1d_L12_obc", device=dev, big=True)
        model.build_Hamiltonian(1.0, 0.5)
        mats.append(model.H.mat)
        meta.append(("su2_1d_L12_obc", model.n_sites, np.asarray(with_l12["su2_1d_L12_obc/energies"])))
    return mats, meta


def test_tiled_fp64_matches_reference(golden_small, dev):
    from edgpu.batch import TiledBatch

    mats, meta = _fixture_instances(golden_small, dev)
    assert len(mats) >= 14
    dims = [m.n for m in mats]
    assert min(dims) <= 10 and max(dims) >= 17000
    # small tiles: the large instances spread over tens of items
    tb = TiledBatch(mats, k=2, precision="fp64", tile_rows=512, lanes=4)
    e = tb.solve(use_graph=False).cpu().numpy()
    tb.check_status()
    for i, (name, ns, ref) in enumerate(meta):
        kk = min(len(ref), 2, mats[i].n)
        assert np.allclose(e[i, :kk] / ns, ref[:kk], atol=1e-10, rtol=0), (name, e[i, :kk] / ns, ref[:kk])
    # the same solve replayed from a CUDA graph gives the same numbers
    tb.capture()
    e2 = tb.solve(use_graph=True).cpu().numpy()
    tb.check_status()
    assert np.array_equal(np.nan_to_num(e2), np.nan_to_num(e))


def test_tiled_mixed_matches_reference(golden_small, golden_big, dev):
    from edgpu.batch import TiledBatch

    mats, meta = _fixture_instances(golden_small, dev, with_l12=golden_big)
    assert max(m.n for m in mats) == 73789
    tb = TiledBatch(mats, k=1, precision="mixed", want_vectors=True)  # autotuned tiles and lanes
    e = tb.solve(use_graph=False).cpu().numpy()[:, 0]
    tb.check_status()
    iters32 = tb.iters32.cpu().numpy()
    assert np.all(iters32 >= 1)
    for i, (name, ns, ref) in enumerate(meta):
        rel = abs(e[i] / ns - ref[0]) / abs(ref[0])
        assert rel <= 1e-9, (name, e[i] / ns, ref[0], rel)
    # ground-state vectors: normalised, Rayleigh quotient = E (to the energy
    # tolerance) and a small residual (the short f64 refinement converges the
    # eigenvalue quadratically faster than the vector)
    ev = tb.evecs.cpu().numpy()
    off = 0
    for i, mat in enumerate(mats):
        x = ev[off: off + mat.n]
        off += mat.n
        assert abs(np.linalg.norm(x) - 1.0) < 1e-10
        H = mat.to_scipy()
        hx = H @ x
        assert abs(float(x @ hx) - e[i]) <= 1e-9 * abs(e[i]), meta[i][0]
        assert np.linalg.norm(hx - e[i] * x) < 1e-4 * max(1.0, abs(e[i])), meta[i][0]


def _c3_instances(dev):
    """QED 3x2 open lattice: 64 couplings (g log-uniform in [0.1, 5], m
    uniform in [0, 2], seed 0) in Q = 0 plus the Q = -2..2 charge sectors."""
    from cases import QED_CHARGE
    from edgpu.models import QED_Model

    rng = np.random.default_rng(0)
    gs = np.exp(rng.uniform(np.log(0.1), np.log(5.0), 64))
    ms = rng.uniform(0.0, 2.0, 64)
    model = QED_Model(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True], device=dev)
    mats = []
    for g, m in zip(gs, ms):
        model.build_Hamiltonian(float(g), float(m))
        mats.append(model.H.mat)
    for q, bg in QED_CHARGE.items():
        mq = QED_Model(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True], bg_list=bg, charge=q,
                       device=dev)
        mq.build_Hamiltonian(1.0, 1.0)
        mats.append(mq.H.mat)
    return mats


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tiled_c3_batch_matches_dense(precision, dev):
    from edgpu.batch import TiledBatch

    mats = _c3_instances(dev)
    tb = TiledBatch(mats, k=1, precision=precision)
    tb.capture()
    e = tb.solve().cpu().numpy()[:, 0]
    tb.check_status()
    for i, mat in enumerate(mats):
        w = np.linalg.eigvalsh(mat.to_scipy().toarray())[0]
        if precision == "fp64":
            assert abs(e[i] - w) < 1e-10 * max(1.0, abs(w)), (i, e[i], w)
        else:
            assert abs(e[i] - w) <= 1e-9 * abs(w), (i, e[i], w)


def test_tiled_single_row_and_tiny_instances(dev):
    """Dimension 1..5 instances (Krylov caps below the check interval) finish
    with exact eigenvalues, alone and beside a larger one."""
    import torch

    from edgpu.batch import TiledBatch
    from edgpu.modeling.assembly import DeviceMatrix

    rng = np.random.default_rng(5)
    mats, dense = [], []
    for n in (1, 2, 3, 5, 300):
        A = rng.standard_normal((n, n))
        A = (A + A.T) / 2
        off = A - np.diag(np.diag(A))
        rows, cols = np.nonzero(off)
        rowptr = np.zeros(n + 1, dtype=np.int64)
        np.add.at(rowptr, rows + 1, 1)
        rowptr = np.cumsum(rowptr)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)  # noqa: E731
        mats.append(DeviceMatrix(n, t(rowptr, np.int64), t(cols, np.int32), t(off[rows, cols], np.float64),
                                 t(np.diag(A), np.float64), t(np.ones(n), np.uint8), False))
        dense.append(np.linalg.eigvalsh(A))
    tb = TiledBatch(mats, k=1, precision="fp64", tile_rows=256, lanes=2, max_iter=300)
    e = tb.solve(use_graph=False).cpu().numpy()[:, 0]
    tb.check_status()
    for i, w in enumerate(dense):
        assert abs(e[i] - w[0]) < 1e-10 * max(1.0, abs(w[0])), (i, e[i], w[0])
