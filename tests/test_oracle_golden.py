"""The CPU oracle (restatement of the reference) pinned against fixtures
produced by the reference itself; the operator factories and term lists of
the package feed both, so these tests also pin the host model layer."""

import numpy as np
import pytest

from cases import (ALL_CASES, ENTROPY_CASES, MOMENTUM_CASES, NBODY_CASES, TC_MAP, TC_SIGN, TWOBODY_CASES, build,
                   build_momentum_case, nbody_instances)
from oracle import edlgt_oracle as O


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_sector_matches_reference(name, golden_small):
    model, g, m = build(name)
    cfg = O.sector_configs(**model.sector_inputs)
    keys = O.keys_of(cfg, model.loc_dims)
    assert np.array_equal(model.loc_dims, golden_small[f"{name}/loc_dims"])
    assert np.array_equal(keys, golden_small[f"{name}/keys"])


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_matrix_and_energies_match_reference(name, golden_small):
    model, g, m = build(name)
    cfg = O.sector_configs(**model.sector_inputs)
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims)
    assert np.array_equal(H.indptr, golden_small[f"{name}/H_indptr"])
    assert np.array_equal(H.indices, golden_small[f"{name}/H_indices"])
    ref = golden_small[f"{name}/H_data"]
    assert np.max(np.abs(H.data - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
    e_ref = golden_small[f"{name}/energies"]
    w, _ = O.lowest_eigs(H, len(e_ref))
    assert np.allclose(w / model.n_sites, e_ref, atol=1e-10, rtol=0)


def test_validation_pins(golden_pins):
    """Energies and observables pinned by the reference's validation suite."""
    # QED 1D L=4 OBC/PBC (validation/qed/test_qed_1d_matter.py)
    for name in ("qed1d_L4_obc", "qed1d_L4_pbc"):
        model, g, m = build(name)
        cfg = O.sector_configs(**model.sector_inputs)
        H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims)
        w, v = O.lowest_eigs(H, 1)
        assert abs(w[0] / 4 - golden_pins[f"{name}/energy"]) < 1e-10
        e2 = O.local_expval(v[:, 0], model.ops["E2_px"], cfg)
        n_ev = O.local_expval(v[:, 0], model.ops["N"], cfg)
        nz = O.local_expval(v[:, 0], model.ops["N_zero"], cfg)
        links = [s for s in range(4) if (s < 3 or not model.has_obc[0])]
        assert abs(np.mean(e2[links]) - golden_pins[f"{name}/E2"]) < 1e-10
        n_val = 0.5 * np.mean(n_ev[0::2]) + 0.5 * np.mean(nz[1::2])
        assert abs(n_val - golden_pins[f"{name}/N"]) < 1e-10
    # SU(2) L=6 PBC (validation/su2/test_su2_spectrum.py)
    model, g, m = build("su2_1d_L6_pbc")
    cfg = O.sector_configs(**model.sector_inputs)
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims)
    w, v = O.lowest_eigs(H, 1)
    assert abs(w[0] / 6 - golden_pins["su2_1d_L6_pbc/energy"]) < 1e-10
    # staggered densities as edlgt/workflows/su2.py:211-218 combines them
    ev = {k: O.local_expval(v[:, 0], model.ops[k], cfg) for k in ("N_single", "N_pair", "N_zero", "T2_px")}
    single = np.mean(ev["N_single"])
    pair = 0.5 * np.mean(ev["N_pair"][0::2]) + 0.5 * np.mean(ev["N_zero"][1::2])
    zero = 0.5 * np.mean(ev["N_zero"][0::2]) + 0.5 * np.mean(ev["N_pair"][1::2])
    got = {"N_single": single, "N_pair": pair, "N_zero": zero, "N_tot": single + 2 * pair,
           "E2": np.mean(ev["T2_px"])}
    for k, val in got.items():
        assert abs(val - golden_pins[f"su2_1d_L6_pbc/{k}"]) < 1e-10, k


def test_charge_sector_dimensions(golden_small):
    dims = {q: int(golden_small[f"qed2d_3x2_Q{q:+d}/dim"]) for q in (-2, -1, 1, 2)}
    dims[0] = int(golden_small["qed2d_3x2_q0/dim"])
    assert dims == {-2: 26, -1: 52, 0: 90, 1: 67, 2: 26}


def test_dynamics_oracle(golden_dyn):
    """expm_multiply restatement reproduces the reference's quench observables."""
    for name, key in (("su2_1d_L6_pbc", "su2_1d_L6_pbc_V"),):
        model, _, _ = build(name)
        g = float(golden_dyn[f"{key}/g"])
        m = float(golden_dyn[f"{key}/m"])
        cfg = O.sector_configs(**model.sector_inputs)
        H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims)
        idx = O.config_to_index(golden_dyn[f"{key}/config"][None, :], cfg, model.loc_dims)[0]
        psi0 = np.zeros(H.shape[0], complex)
        psi0[idx] = 1
        t = golden_dyn[f"{key}/time"]
        psi_t = O.evolve(H, psi0, t)
        T2 = np.array([O.local_expval(p, model.ops["T2_px"], cfg) for p in psi_t])
        assert np.max(np.abs(T2 - golden_dyn[f"{key}/T2_px"])) < 1e-9


@pytest.mark.parametrize("name", sorted(TWOBODY_CASES))
def test_twobody_oracle(name, golden_twobody):
    """Correlator matrices of the reference's TwoBodyTerm on its own ground
    state, recomputed by the oracle from the package's projected operators."""
    model, _, _ = build(name)
    loc = golden_twobody[f"{name}/loc_dims"]
    assert np.array_equal(model.loc_dims, loc)
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, loc), golden_twobody[f"{name}/keys"])
    psi = golden_twobody[f"{name}/psi"]
    for a, b in TWOBODY_CASES[name]:
        corr = O.twobody_expval(psi, model.ops[a], model.ops[b], cfg, loc)
        ref = golden_twobody[f"{name}/{a}_{b}"]
        assert np.max(np.abs(corr - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), (a, b)


@pytest.mark.parametrize("name", sorted(ENTROPY_CASES))
def test_partition_and_entropy_oracle(name, golden_entropy):
    """Bipartition maps bit-exact, entropies and reduced density matrices of
    the reference's ground state to 1e-12, recomputed by the oracle."""
    model, _, _ = build(name)
    loc = golden_entropy[f"{name}/loc_dims"]
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, loc), golden_entropy[f"{name}/keys"])
    psi = golden_entropy[f"{name}/psi"]
    for keep in ENTROPY_CASES[name]:
        tag = f"{name}/" + "-".join(str(i) for i in keep)
        part = O.partition(cfg, loc, keep)
        for k in ("subsys_map", "env_map", "unique_subsys_configs", "unique_env_configs"):
            assert np.array_equal(part[k], golden_entropy[f"{tag}/{k}"]), (keep, k)
        assert [part["subsys_dim"], part["env_dim"]] == list(golden_entropy[f"{tag}/dims"])
        assert abs(O.entanglement_entropy(psi, part) - float(golden_entropy[f"{tag}/entropy"])) <= 1e-12
        if f"{tag}/rdm" in golden_entropy:
            assert np.max(np.abs(O.reduced_density_matrix(psi, part) - golden_entropy[f"{tag}/rdm"])) <= 1e-13


@pytest.mark.parametrize("name", sorted(MOMENTUM_CASES))
def test_momentum_basis_oracle(name, golden_momentum):
    """Momentum projectors B (CSC pattern exact, values to 1e-13) and the two
    lowest energies of B^dagger H B against the reference's
    set_momentum_sector / build_Hamiltonian / diagonalize_Hamiltonian."""
    model, g, m, ucs, ks = build_momentum_case(name)
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), golden_momentum[f"{name}/keys"])
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims).toarray()
    for k in ks:
        tag = f"{name}/k" + "_".join(str(x) for x in k)
        tc = dict(local_map=TC_MAP, label_sign=TC_SIGN) if name.endswith("_tc") else {}
        cp, ri, data, n_cols = O.momentum_basis(cfg, model.loc_dims, model.lvals, ucs, k, **tc)
        assert np.array_equal(cp, golden_momentum[f"{tag}/L_col_ptr"])
        assert np.array_equal(ri, golden_momentum[f"{tag}/L_row_idx"])
        assert np.max(np.abs(data - golden_momentum[f"{tag}/L_data"]), initial=0.0) <= 1e-13
        B = np.zeros((len(cfg), n_cols), dtype=np.complex128)
        for c in range(n_cols):
            B[ri[cp[c]:cp[c + 1]], c] = data[cp[c]:cp[c + 1]]
        e = np.linalg.eigvalsh(B.conj().T @ H @ B)[:2] / model.n_sites
        assert np.allclose(e, golden_momentum[f"{tag}/energies"], atol=1e-10, rtol=0), (k, e)


def test_full_spectrum_oracle(golden_full):
    """SU(2) L=6 PBC full spectrum and its thermal and ensemble quantities,
    restated with numpy on the oracle's matrix, against the reference."""
    g = golden_full
    model, _, _ = build("su2_1d_L6_pbc")
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), g["keys"])
    H = O.assemble(model.hamiltonian_blocks(1.0, 5.0), cfg, model.loc_dims).toarray()
    w, V = np.linalg.eigh(H)
    n = model.n_sites
    E = w / n
    assert np.allclose(E, g["energies"], atol=1e-10, rtol=0)
    beta = float(g["beta"])
    Z = np.sum(np.exp(-beta * E))
    assert np.isclose(Z, g["Z"], rtol=1e-10)
    assert np.isclose(-np.log(Z) / beta, g["F"], rtol=1e-10)
    assert np.isclose(E.dot(np.exp(-beta * E)) / Z, g["E_thermal"], rtol=1e-10)
    idx = np.searchsorted(O.keys_of(cfg, model.loc_dims), O.keys_of(g["config"][None, :], model.loc_dims))
    state = np.zeros(len(cfg), dtype=np.complex128)
    state[idx] = 1.0
    d_rows = lambda name: np.real(np.array([np.diagonal(model.ops[name][s]) for s in range(n)]))[  # noqa: E731
        np.arange(n)[None, :], cfg.astype(np.int64)]
    eig_obs = lambda name: (np.abs(V) ** 2).T @ d_rows(name)  # noqa: E731
    wt = np.exp(-beta * (w - w.min()))
    assert np.isclose(wt.dot(eig_obs("N_tot").sum(axis=1)) / (wt.sum() * n), g["canonical_N_tot"], rtol=1e-10)
    c = V.conj().T @ state
    block = np.concatenate([[0], np.cumsum(np.abs(np.diff(E)) >= 1e-10)])
    for name in ("N_tot", "T2_px"):
        de = 0.0
        for b in range(block[-1] + 1):
            psi_b = V[:, block == b] @ c[block == b]
            if np.vdot(psi_b, psi_b).real >= 1e-14:
                de += np.mean(np.abs(psi_b) ** 2 @ d_rows(name))
        assert np.isclose(de, g[f"DE_{name}"], atol=1e-10), name
    for j, t in enumerate(g["time"]):
        psi_t = V @ (np.exp(-1j * w * t) * c)
        assert np.max(np.abs(psi_t - g["psi_time"][j])) <= 1e-10


@pytest.mark.parametrize("name", sorted(NBODY_CASES))
def test_nbody_oracle(name, golden_nbody):
    """NBodyTerm.get_expval of the reference's ground state, recomputed from
    the oracle's n-site triplets (real part, 1e-12)."""
    model, _, _ = build(name)
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), golden_nbody[f"{name}/keys"])
    psi = golden_nbody[f"{name}/psi"]
    for names, dist in zip(*NBODY_CASES[name]):
        vals = []
        for sites in nbody_instances(model.lvals, model.has_obc, dist):
            rows, cols, v = O.nbody_triplets([model.ops[o] for o in names], sites, cfg, model.loc_dims)
            vals.append(np.real(np.sum(np.conj(psi[rows]) * v * psi[cols])))
        ref = golden_nbody[f"{name}/{'_'.join(names)}"]
        assert len(vals) == len(ref) and np.max(np.abs(np.array(vals) - ref)) <= 1e-12, names


@pytest.mark.parametrize("name", ["qedint_L4", "qedint_L8_bg", "qedint_L10"])
def test_integrated_qed_oracle(name, golden_integrated):
    """Integrated-gauge 1D QED: sector keys bit-exact, the matrix of the
    package's term list (oracle assembly plus the constant) against the
    reference's to 1e-12, energies to 1e-10."""
    from cases import INTEGRATED_CASES
    from edgpu.models import QED_Model
    from scipy.sparse import csr_matrix

    lvals, bg, g, m = INTEGRATED_CASES[name]
    model = QED_Model(spin="integrated", pure_theory=False, lvals=lvals, has_obc=[True], bg_list=bg, device="cpu")
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), golden_integrated[f"{name}/keys"])
    blocks, const = model.integrated_blocks(g, m)
    H = O.assemble(blocks, cfg, model.loc_dims).toarray() + const * np.eye(len(cfg))
    n = len(cfg)
    ref = csr_matrix((golden_integrated[f"{name}/H_data"], golden_integrated[f"{name}/H_indices"],
                      golden_integrated[f"{name}/H_indptr"]), shape=(n, n)).toarray()
    assert np.max(np.abs(H - ref)) <= 1e-12
    e = np.linalg.eigvalsh(H)[:2] / model.n_sites
    assert np.allclose(e, golden_integrated[f"{name}/energies"], atol=1e-10, rtol=0)


def test_integrated_e2_reconstruction():
    """reconstruct_integrated_E2_from_N from oracle-measured <N_k>, <N_k N_l>
    of the integrated ground state against <E_n^2> evaluated directly in the
    sector basis (the electric field is diagonal there)."""
    from cases import INTEGRATED_CASES
    from edgpu.models import QED_Model

    lvals, bg, g, m = INTEGRATED_CASES["qedint_L8_bg"]
    model = QED_Model(spin="integrated", pure_theory=False, lvals=lvals, has_obc=[True], bg_list=bg, device="cpu")
    cfg = O.sector_configs(**model.sector_inputs)
    blocks, const = model.integrated_blocks(g, m)
    H = O.assemble(blocks, cfg, model.loc_dims).toarray() + const * np.eye(len(cfg))
    w, V = np.linalg.eigh(H)
    p = np.abs(V[:, 0]) ** 2
    n_site = (cfg == 0).astype(float)  # basis index 0 is the occupied state
    model.res["N"] = p @ n_site
    model.res["N_N"] = (n_site * p[:, None]).T @ n_site
    e2 = model.reconstruct_integrated_E2_from_N(print_values=False)
    q = np.asarray(bg, dtype=float)
    k = np.arange(model.n_sites)
    field = np.cumsum(q + 0.5 * ((-1.0) ** k - 1.0) + n_site, axis=1)[:, :-1]
    assert np.allclose(e2, p @ field ** 2, atol=1e-12)
    assert abs(model.res["E2_avg"] - np.mean(e2)) <= 1e-15


def test_string_constraint_sectors_oracle(golden_string):
    """Site-resolved string constraints (the reference's
    iterative_sitebased_sym_sector_configs1): the oracle reproduces the
    reference's keys from the same inputs, including the empty sector."""
    from cases import string_case_inputs, string_case_names

    names = string_case_names(golden_string)
    assert len(names) >= 8
    for name in names:
        a = string_case_inputs(golden_string, name)
        cfg = O.sector_configs(a["loc_dims"], a["glob_op_diags"], a["glob_sectors"], "U", a["link_op_diags"],
                               a["link_sectors"], a["pair_list"], a["string_op_diags"], a["string_sectors"])
        keys = O.keys_of(cfg, a["loc_dims"]) if len(cfg) else np.zeros(0, dtype=np.uint64)
        assert np.array_equal(keys, golden_string[f"{name}/keys"]), name
        assert len(keys) <= int(golden_string[f"{name}/base_dim"])


@pytest.mark.parametrize("name", sorted(__import__("cases").SU2_GEN_CASES))
def test_generic_su2_matches_reference(name, golden_generic):
    """The generic SU(2) model (j_max = 1, 3/2, and j_max = 1/2 with
    use_generic_model): the package's operator factory and term list fed to
    the oracle reproduce the reference's sector keys (bit-exact), canonical
    matrix (pattern bit-exact, values 1e-13) and energies (1e-10)."""
    from cases import build_generic

    model, g, m = build_generic(name)
    assert np.array_equal(model.loc_dims, golden_generic[f"{name}/loc_dims"])
    cfg = O.sector_configs(**model.sector_inputs)
    assert np.array_equal(O.keys_of(cfg, model.loc_dims), golden_generic[f"{name}/keys"])
    H = O.assemble(model.hamiltonian_blocks(g, m), cfg, model.loc_dims)
    assert np.array_equal(H.indptr, golden_generic[f"{name}/H_indptr"])
    assert np.array_equal(H.indices, golden_generic[f"{name}/H_indices"])
    ref = golden_generic[f"{name}/H_data"]
    assert np.max(np.abs(H.data - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
    e_ref = golden_generic[f"{name}/energies"]
    w, _ = O.lowest_eigs(H, len(e_ref))
    assert np.allclose(w / model.n_sites, e_ref, atol=1e-10, rtol=0)


def _digest(H):
    import hashlib

    rows = np.repeat(np.arange(H.shape[0], dtype=np.int64), np.diff(H.indptr))
    cols = H.indices.astype(np.int64)
    w = 1.0 / (1.0 + ((rows * 7919 + cols * 104729) % 1009))
    return H.nnz, hashlib.sha256(np.stack([rows, cols]).tobytes()).hexdigest(), complex(np.sum(H.data * w))


def test_two_word_key_layout():
    """Key spaces above 63 bits split into a high word (leading sites) and a
    low word (the longest trailing run below 2^63); the 128-bit number
    hi * 2^64 + lo orders configurations lexicographically."""
    from edgpu.symmetries import compute_strides, key_layout

    assert key_layout([19] * 14) == (1, 0, 19**14)
    words, n_hi, lo_space = key_layout([19] * 16)
    assert (words, n_hi, lo_space) == (2, 2, 19**14)
    dims = [5, 19, 19, 5, 19, 85, 85, 19, 19, 85, 85, 19, 5, 19, 19, 5]
    words, n_hi, lo_space = key_layout(dims)
    assert words == 2 and lo_space < 2**63 and lo_space * dims[n_hi - 1] >= 2**63
    assert np.prod(np.asarray(dims[:n_hi], dtype=object)) < 2**63
    st = compute_strides(dims, n_hi)
    assert st[n_hi - 1] == 1 and st[-1] == 1
    rng = np.random.default_rng(0)
    cfg = np.stack([rng.integers(0, d, 4000) for d in dims], axis=1)
    cfg = cfg[np.lexsort(cfg.T[::-1])]
    big = [(int(sum(int(c[s]) * int(st[s]) for s in range(n_hi))) << 64)
           + int(sum(int(c[s]) * int(st[s]) for s in range(n_hi, len(dims)))) for c in cfg]
    assert all(a <= b for a, b in zip(big, big[1:]))
    with pytest.raises(OverflowError):
        key_layout([255] * 17)


@pytest.mark.parametrize("name", sorted(__import__("cases").WIDE_CASES))
def test_wide_sector_matches_reference(name, golden_wide):
    """Pure-gauge 4x4 QED lattices with a key space above 63 bits: the
    oracle's sector table equals the reference's (sha256 of the uint16
    table, sampled rows), the lookup finds every sampled row, and (periodic
    lattice) the canonical matrix digest and two lowest energies match."""
    import hashlib

    from cases import build_wide

    model, g = build_wide(name)
    assert np.array_equal(model.loc_dims, golden_wide[f"{name}/loc_dims"])
    assert model.sector_spec.key_words == 2
    cfg = O.sector_configs(**model.sector_inputs)
    assert cfg.shape[0] == int(golden_wide[f"{name}/dim"])
    assert hashlib.sha256(np.ascontiguousarray(cfg).tobytes()).hexdigest() == str(golden_wide[f"{name}/configs_sha"])
    rows = golden_wide[f"{name}/sample_rows"]
    assert np.array_equal(cfg[rows], golden_wide[f"{name}/sample_configs"])
    assert np.array_equal(O.config_to_index(cfg[rows], cfg, model.loc_dims), rows)
    if name.endswith("pbc_s1"):
        H = O.assemble(model.hamiltonian_blocks(g), cfg, model.loc_dims)
        nnz, pat, ws = _digest(H)
        assert nnz == int(golden_wide[f"{name}/H_nnz"])
        assert pat == str(golden_wide[f"{name}/H_pattern_sha"])
        ref = complex(golden_wide[f"{name}/H_wsum"])
        assert abs(ws - ref) <= 1e-10 * abs(ref)
        e_ref = golden_wide[f"{name}/energies"]
        w, _ = O.lowest_eigs(H, len(e_ref))
        assert np.allclose(w / model.n_sites, e_ref, atol=1e-10, rtol=0)


def test_thermal_expm_branches_match_reference(golden_thermal):
    """The traces the reference takes of expm(-beta H) after a partial
    diagonalisation, restated on the oracle's matrix of SU(2) L=6 PBC:
    Tr(H^2 e^-bH) by matrix power in the sparse format and by the elementwise
    square in the dense format (qmb_hamiltonian.py:446-452, 486-489,
    505-508)."""
    from scipy.linalg import expm

    model, _, _ = build("su2_1d_L6_pbc")
    cfg = O.sector_configs(**model.sector_inputs)
    H = O.assemble(model.hamiltonian_blocks(1.0, 5.0), cfg, model.loc_dims).toarray()
    for beta in (0.3, 0.7):
        M = expm(-beta * H)
        Z = np.real(np.trace(M))
        E = np.real(np.trace(H @ M)) / Z
        for fmt, H2 in (("sparse", H @ H), ("dense", H * H)):
            q = f"{fmt}/b{beta}/"
            assert np.isclose(Z, golden_thermal[q + "Z"], rtol=1e-10, atol=0)
            assert np.isclose(E, golden_thermal[q + "E_thermal"], rtol=1e-10, atol=0)
            fp = -np.real(np.trace(H2 @ M)) / Z - E**2
            assert np.isclose(fp, golden_thermal[q + "F_prime"], rtol=1e-9, atol=0)
