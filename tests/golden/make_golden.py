"""Generate golden fixtures by running ed-lgt (the reference) itself.

Run in a container that has the reference checkout (EDLGT_PATH, required)
and numba/scipy/sympy:

    python tests/golden/make_golden.py [group ...]

Groups: small, pins, dynamics, big, twobody, entropy, momentum, full,
nbody, overlap, state, local, integrated, string, generic, wide, thermal.  Output: .npz files next to
this script.  Nothing here is imported by the library or by the GPU tests;
the tests only read the .npz files.

Digests.  A sector is stored as its sorted uint64 keys (key = sum_s c_s *
stride_s, last site fastest) or, when large, as (dimension, sha256 of the key
bytes).  A matrix is the reference's triplets summed into canonical CSR
(scipy sum_duplicates), stored whole when small or as (nnz, sha256 of the
(row, col) pattern, weighted value sums) when large.
"""

from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402,F401

import logging  # noqa: E402

logging.disable(logging.INFO)

from scipy.sparse import coo_matrix  # noqa: E402

import edlgt.models.SU2_model as _su2mod  # noqa: E402
from edlgt.models import QED_Model, SU2_Model  # noqa: E402

# the reference's SU(2) static-charge path formats floats with ':d' in a log
# helper; silence that helper so the path can run.
_su2mod.format_loc_dims = lambda *a, **k: None


def keys_of(configs, loc_dims):
    loc_dims = np.asarray(loc_dims, dtype=np.uint64)
    strides = np.ones(len(loc_dims), dtype=np.uint64)
    for k in range(len(loc_dims) - 2, -1, -1):
        strides[k] = strides[k + 1] * loc_dims[k + 1]
    return (np.asarray(configs, dtype=np.uint64) * strides[None, :]).sum(axis=1, dtype=np.uint64)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canonical(model):
    H = model.H
    H._materialize_triplets()
    n = H.shape[0]
    m = coo_matrix((H.value_list, (H.row_list.astype(np.int64), H.col_list.astype(np.int64))), shape=(n, n)).tocsr()
    m.sum_duplicates()
    m.sort_indices()
    return m


def value_weights(rows, cols):
    return 1.0 / (1.0 + ((rows * 7919 + cols * 104729) % 1009))


def matrix_record(m, prefix, store_full):
    rows = np.repeat(np.arange(m.shape[0], dtype=np.int64), np.diff(m.indptr))
    cols = m.indices.astype(np.int64)
    vals = np.asarray(m.data, dtype=np.complex128)
    out = {
        f"{prefix}nnz": np.int64(len(vals)),
        f"{prefix}pattern_sha": np.array(sha(np.stack([rows, cols]))),
        f"{prefix}wsum": np.complex128(np.sum(vals * value_weights(rows, cols))),
        f"{prefix}abssum": np.float64(np.sum(np.abs(vals))),
    }
    if store_full:
        out |= {f"{prefix}indptr": m.indptr.astype(np.int64), f"{prefix}indices": cols.astype(np.int32),
                f"{prefix}data": vals}
    return out


def sector_record(model, prefix, store_full):
    cfg = model.sector_configs
    keys = keys_of(cfg, model.loc_dims)
    out = {f"{prefix}dim": np.int64(len(keys)), f"{prefix}keys_sha": np.array(sha(keys)),
           f"{prefix}loc_dims": np.asarray(model.loc_dims, dtype=np.int64)}
    if store_full:
        out[f"{prefix}keys"] = keys
    return out


# ---------------------------------------------------------------------------
QED_CASES = {
    # name: (kwargs, g, m)
    "qed1d_L4_obc": (dict(spin=1, pure_theory=False, lvals=[4], has_obc=[True]), 1.0, 1.0),
    "qed1d_L4_pbc": (dict(spin=1, pure_theory=False, lvals=[4], has_obc=[False]), 1.0, 1.0),
    "qed1d_L8_obc": (dict(spin=1, pure_theory=False, lvals=[8], has_obc=[True]), 1.0, 1.0),
    "qed2d_3x2_bg": (dict(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True],
                          bg_list=[-1, 0, 0, 0, 0, 1]), 1.0, 1.0),
    "qed2d_3x2_q0": (dict(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True]), 0.7, 0.4),
    "qed2d_2x2_pure_pbc": (dict(spin=1, pure_theory=True, lvals=[2, 2], has_obc=[False, False]), 1.3, None),
    "qed2d_3x2_pure_obc": (dict(spin=1, pure_theory=True, lvals=[3, 2], has_obc=[True, True]), 0.8, None),
}
# charge sectors of the 3x2 lattice: static charges summing to -Q, N = 3 + Q
QED_CHARGE = {-2: [1, 0, 0, 0, 0, 1], -1: [1, 0, 0, 0, 0, 0], 1: [-1, 0, 0, 0, 0, 0], 2: [-1, 0, 0, 0, 0, -1]}

SU2_CASES = {
    "su2_1d_L6_pbc": (dict(spin=0.5, pure_theory=False, lvals=[6], has_obc=[False], sectors=[6]), 1.0, 5.0),
    "su2_1d_L8_obc": (dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[True], sectors=[8]), 1.0, 0.5),
    "su2_1d_L10_obc": (dict(spin=0.5, pure_theory=False, lvals=[10], has_obc=[True], sectors=[10]), 1.0, 0.5),
    "su2_1d_L10_pbc": (dict(spin=0.5, pure_theory=False, lvals=[10], has_obc=[False], sectors=[10]), 2.0, 0.5),
    "su2_1d_L8_obc_bg": (dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[True], sectors=[8],
                              bg_list=[0, 0, 0.5, 0, 0, 0.5, 0, 0]), 1.0, 1.0),
    "su2_2d_2x2_pure_pbc": (dict(spin=0.5, pure_theory=True, lvals=[2, 2], has_obc=[False, False]), 1.0, None),
    "su2_2d_2x2_obc": (dict(spin=0.5, pure_theory=False, lvals=[2, 2], has_obc=[True, True], sectors=[4]), 1.0, 1.0),
}


def qed_model(kwargs):
    return QED_Model(**kwargs)


def su2_model(kwargs):
    m = SU2_Model(**kwargs)
    m.default_params()
    return m


def qed_charge_model(q):
    m = QED_Model(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True], bg_list=QED_CHARGE[q])
    link_ops = [[m.ops[f"E_p{d}"], -m.ops[f"E_m{d}"]] for d in m.directions]
    m.get_abelian_symmetry_sector(global_ops=[m.ops["N"]], global_sectors=[3 + q], link_ops=link_ops,
                                  link_sectors=[0, 0])
    m.default_params()
    return m


def gen_small(store_spectra=True):
    out = {}
    t0 = time.time()
    for name, (kw, g, mass) in QED_CASES.items():
        model = qed_model(kw)
        out |= sector_record(model, f"{name}/", True)
        model.build_Hamiltonian(g, mass)
        out |= matrix_record(canonical(model), f"{name}/H_", True)
        out[f"{name}/g"] = np.float64(g)
        out[f"{name}/m"] = np.float64(np.nan if mass is None else mass)
        if store_spectra:
            k = 2 if len(model.sector_configs) > 3 else 1
            model.diagonalize_Hamiltonian(k, "sparse")
            out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
        print(name, len(model.sector_configs), f"{time.time() - t0:.1f}s", flush=True)
    for q, bg in QED_CHARGE.items():
        name = f"qed2d_3x2_Q{q:+d}"
        model = qed_charge_model(q)
        out |= sector_record(model, f"{name}/", True)
        model.build_Hamiltonian(1.0, 1.0)
        out |= matrix_record(canonical(model), f"{name}/H_", True)
        model.diagonalize_Hamiltonian(1, "sparse")
        out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
        print(name, len(model.sector_configs), flush=True)
    for name, (kw, g, mass) in SU2_CASES.items():
        model = su2_model(kw)
        out |= sector_record(model, f"{name}/", True)
        model.build_Hamiltonian(g, mass)
        out |= matrix_record(canonical(model), f"{name}/H_", True)
        out[f"{name}/g"] = np.float64(g)
        out[f"{name}/m"] = np.float64(np.nan if mass is None else mass)
        model.diagonalize_Hamiltonian(1, "sparse")
        out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
        print(name, len(model.sector_configs), f"{time.time() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **out)


def gen_validation_pins():
    """Known answers of the reference's own validation suite, re-run here."""
    from edlgt.workflows.qed import run_QED_spectrum
    from edlgt.workflows.su2 import run_SU2_spectrum

    out = {}
    par = {"model": {"lvals": [4], "has_obc": [True], "spin": 1, "pure_theory": False, "ham_format": "sparse",
                     "bg_list": None}, "hamiltonian": {"n_eigs": 1}, "observables": {"measure_obs": True},
           "g": 1.0, "m": 1.0}
    r = run_QED_spectrum(par)
    out |= {"qed1d_L4_obc/energy": r["energy"][0], "qed1d_L4_obc/E2": r["E2"][0], "qed1d_L4_obc/N": r["N"][0]}
    par["model"]["has_obc"] = [False]
    r = run_QED_spectrum(par)
    out |= {"qed1d_L4_pbc/energy": r["energy"][0], "qed1d_L4_pbc/E2": r["E2"][0], "qed1d_L4_pbc/N": r["N"][0]}
    par = {"model": {"lvals": [3, 2], "has_obc": [True, True], "spin": 1, "pure_theory": False,
                     "ham_format": "sparse", "bg_list": [-1, 0, 0, 0, 0, 1]}, "hamiltonian": {"n_eigs": 1},
           "observables": {"measure_obs": True}, "g": 1, "m": 1}
    r = run_QED_spectrum(par)
    out |= {"qed2d_3x2_bg/energy": r["energy"][0], "qed2d_3x2_bg/E2": r["E2"][0], "qed2d_3x2_bg/N": r["N"][0],
            "qed2d_3x2_bg/plaq": r["C_px,py_C_py,mx_C_my,px_C_mx,my"][0]}
    par = {"model": {"lvals": [6], "sectors": [6], "has_obc": [False], "spin": 0.5, "pure_theory": False,
                     "ham_format": "sparse"}, "hamiltonian": {"n_eigs": 1}, "observables": {"measure_obs": True},
           "g": 1, "m": 5}
    r = run_SU2_spectrum(par)
    for k in ("energy", "E2", "N_tot", "N_single", "N_pair", "N_zero"):
        out[f"su2_1d_L6_pbc/{k}"] = r[k][0]
    np.savez(os.path.join(HERE, "validation_pins.npz"), **{k: np.float64(v) for k, v in out.items()})
    print(out)


def gen_big():
    """Sector digests and matrix digests at the benchmark sizes."""
    out = {}
    for name, kw, g, mass, with_matrix in (
        ("su2_1d_L12_obc", dict(spin=0.5, pure_theory=False, lvals=[12], has_obc=[True], sectors=[12]), 1.0, 0.5,
         True),
        ("su2_1d_L14_obc", dict(spin=0.5, pure_theory=False, lvals=[14], has_obc=[True], sectors=[14]), 1.0, 0.5,
         True),
        ("su2_1d_L14_pbc", dict(spin=0.5, pure_theory=False, lvals=[14], has_obc=[False], sectors=[14]), 1.0, 0.5,
         False),
        ("su2_1d_L16_obc_pair", dict(spin=0.5, pure_theory=False, lvals=[16], has_obc=[True], sectors=[16],
                                     bg_list=[0] * 5 + [0.5] + [0] * 4 + [0.5] + [0] * 5), 1.0, 1.0, False),
    ):
        t0 = time.time()
        model = su2_model(kw)
        out |= sector_record(model, f"{name}/", len(model.sector_configs) <= 100_000)
        if with_matrix:
            model.build_Hamiltonian(g, mass)
            out |= matrix_record(canonical(model), f"{name}/H_", False)
            out[f"{name}/triplets"] = np.int64(len(model.H.row_list))
            t1 = time.time()
            model.diagonalize_Hamiltonian(1, "sparse")
            out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
            out[f"{name}/eigsh_seconds"] = np.float64(time.time() - t1)
        print(name, len(model.sector_configs), f"{time.time() - t0:.1f}s", flush=True)
    # the coupling sweep of the L=14 OBC benchmark: g^2 in {0.5, 1, 2}, m = 0.5
    model = su2_model(dict(spin=0.5, pure_theory=False, lvals=[14], has_obc=[True], sectors=[14]))
    for g in (0.5, 1.0, 2.0):
        model.default_params()
        model.build_Hamiltonian(g, 0.5)
        model.diagonalize_Hamiltonian(1, "sparse")
        out[f"su2_1d_L14_obc/sweep_g{g}"] = np.asarray(model.H.Nenergies)
        print("sweep", g, model.H.Nenergies, flush=True)
    np.savez_compressed(os.path.join(HERE, "big_cases.npz"), **out)


def gen_dynamics():
    """Quench observables from the reference's expm_multiply path."""
    out = {}
    # SU(2) L=6 PBC, bare vacuum, g=1, m=5, t in [0, 0.5] step 0.01 (the
    # reference's own golden-dynamics case), and L=10 OBC string state.
    for name, kw, g, mass, state, tline in (
        ("su2_1d_L6_pbc_V", dict(spin=0.5, pure_theory=False, lvals=[6], has_obc=[False], sectors=[6]), 1.0, 5.0,
         "V", np.arange(0.0, 0.5 + 0.01, 0.01)),
        ("su2_1d_L10_obc_pair", dict(spin=0.5, pure_theory=False, lvals=[10], has_obc=[True], sectors=[10],
                                     bg_list=[0, 0, 0, 0.5, 0, 0, 0.5, 0, 0, 0]), 1.0, 1.0, None,
         np.arange(0.0, 2.0 + 0.05, 0.05)),
    ):
        model = su2_model(kw)
        model.build_Hamiltonian(g, mass)
        if state is not None:
            config = model.overlap_QMB_state(state)
        else:
            # a string product state: the first sector configuration with the
            # most sites in the local state 0 of each site (deterministic)
            cfg = model.sector_configs
            config = cfg[np.argmax((cfg == 0).sum(axis=1))]
        psi0 = model.get_qmb_state_from_configs([config])
        model.time_evolution_Hamiltonian(psi0, tline)
        T2 = np.zeros((len(tline), model.n_sites))
        NP = np.zeros((len(tline), model.n_sites))
        from edlgt.modeling import LocalTerm

        lt = LocalTerm(model.ops["T2_px"], "T2_px", **model.def_params)
        lp = LocalTerm(model.ops["N_pair"], "N_pair", **model.def_params)
        for k in range(len(tline)):
            lt.get_expval(model.H.psi_time[k], print_values=False)
            lp.get_expval(model.H.psi_time[k], print_values=False)
            T2[k] = lt.obs
            NP[k] = lp.obs
        out |= {f"{name}/time": tline, f"{name}/config": np.asarray(config, dtype=np.int64), f"{name}/T2_px": T2,
                f"{name}/N_pair": NP, f"{name}/g": np.float64(g), f"{name}/m": np.float64(mass)}
        print(name, len(model.sector_configs), flush=True)
    np.savez_compressed(os.path.join(HERE, "dynamics_cases.npz"), **out)


TWOBODY_CASES = {
    # name: (factory, kwargs, g, m, [operator pairs])
    "qed1d_L8_obc": (qed_model, QED_CASES["qed1d_L8_obc"][0], 1.0, 1.0, [["N", "N"], ["E2_px", "N"]]),
    "qed2d_3x2_bg": (qed_model, QED_CASES["qed2d_3x2_bg"][0], 1.0, 1.0, [["N", "N"], ["E2_px", "E2_py"]]),
    "su2_1d_L8_obc": (su2_model, SU2_CASES["su2_1d_L8_obc"][0], 1.0, 0.5,
                      [["N_tot", "N_tot"], ["N_pair", "T2_px"]]),
}


def gen_twobody():
    """Two-body correlator matrices of the ground state through the
    reference's get_observables(twobody_obs=...) / measure_observables path,
    stored with the ground state and the sector keys they were measured on."""
    out = {}
    for name, (factory, kw, g, mass, pairs) in TWOBODY_CASES.items():
        model = factory(kw)
        model.build_Hamiltonian(g, mass)
        model.diagonalize_Hamiltonian(1, "sparse")
        model.get_observables([], pairs, [])
        model.measure_observables(0)
        out[f"{name}/keys"] = keys_of(model.sector_configs, model.loc_dims)
        out[f"{name}/loc_dims"] = np.asarray(model.loc_dims, dtype=np.int64)
        out[f"{name}/psi"] = np.asarray(model.H.Npsi[0].psi, dtype=np.complex128)
        for a, b in pairs:
            out[f"{name}/{a}_{b}"] = np.asarray(model.res[f"{a}_{b}"], dtype=np.float64)
        print(name, len(model.sector_configs), flush=True)
    np.savez_compressed(os.path.join(HERE, "twobody_cases.npz"), **out)


ENTROPY_CASES = {
    # name: (factory, kwargs, g, m, [subsystems])
    "qed1d_L8_obc": (qed_model, QED_CASES["qed1d_L8_obc"][0], 1.0, 1.0, [[0, 1, 2, 3], [1, 2, 5], [0, 1]]),
    "qed2d_3x2_bg": (qed_model, QED_CASES["qed2d_3x2_bg"][0], 1.0, 1.0, [[0, 1, 2], [0, 3], [4]]),
    "su2_1d_L8_obc": (su2_model, SU2_CASES["su2_1d_L8_obc"][0], 1.0, 0.5, [[0, 1, 2, 3], [2, 3, 6], [0, 1]]),
}


def gen_entropy():
    """Bipartition maps (_get_partition), reduced density matrices and
    entanglement entropies of the reference's ground state."""
    out = {}
    for name, (factory, kw, g, mass, parts) in ENTROPY_CASES.items():
        model = factory(kw)
        model.build_Hamiltonian(g, mass)
        model.diagonalize_Hamiltonian(1, "sparse")
        st = model.H.Npsi[0]
        out[f"{name}/keys"] = keys_of(model.sector_configs, model.loc_dims)
        out[f"{name}/loc_dims"] = np.asarray(model.loc_dims, dtype=np.int64)
        out[f"{name}/psi"] = np.asarray(st.psi, dtype=np.complex128)
        for keep in parts:
            tag = f"{name}/" + "-".join(str(i) for i in keep)
            part = model._get_partition(keep)
            for k in ("subsys_map", "env_map", "unique_subsys_configs", "unique_env_configs"):
                out[f"{tag}/{k}"] = np.asarray(part[k])
            out[f"{tag}/dims"] = np.array([part["subsys_dim"], part["env_dim"]], dtype=np.int64)
            out[f"{tag}/entropy"] = np.float64(st.entanglement_entropy(keep, model._partition_cache))
            if part["subsys_dim"] <= 64:
                out[f"{tag}/rdm"] = np.asarray(st.reduced_density_matrix(keep, model._partition_cache))
        print(name, len(model.sector_configs), flush=True)
    np.savez_compressed(os.path.join(HERE, "entropy_cases.npz"), **out)


MOMENTUM_CASES = {
    # name: (factory, kwargs, g, m, unit cell, [k vectors]); the SU(2) L=6 k=3 case is the
    # reference's own finite-momentum validation case
    "su2_1d_L6_pbc": (su2_model, SU2_CASES["su2_1d_L6_pbc"][0], 1.0, 5.0, [1], [[0], [1], [3]]),
    "su2_1d_L8_pbc_uc2": (su2_model, dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[False], sectors=[8]), 1.0,
                          0.5, [2], [[0], [1], [2]]),
    "qed1d_L6_pbc_uc2": (qed_model, dict(spin=1, pure_theory=False, lvals=[6], has_obc=[False]), 1.0, 1.0, [2],
                         [[0], [1]]),
    "qed2d_2x2_pure_pbc": (qed_model, QED_CASES["qed2d_2x2_pure_pbc"][0], 1.3, None, [1, 1],
                           [[0, 0], [1, 0], [1, 1]]),
    # translation combined with charge conjugation (TC_symmetry=True)
    "su2_1d_L6_pbc_tc": (su2_model, SU2_CASES["su2_1d_L6_pbc"][0], 1.0, 5.0, [1], [[0], [1], [3]]),
    "su2_1d_L8_pbc_tc": (su2_model, dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[False], sectors=[8]), 1.0,
                         0.5, [1], [[0], [2], [5]]),
}


def gen_momentum():
    """Momentum projectors (set_momentum_sector / get_momentum_basis) and the
    two lowest energies of the projected Hamiltonian, from the reference."""
    out = {}
    for name, (factory, kw, g, mass, ucs, ks) in MOMENTUM_CASES.items():
        for k in ks:
            tag = f"{name}/k" + "_".join(str(x) for x in k)
            model = factory(kw)
            model.set_momentum_sector(ucs, k, name.endswith("_tc"))
            model.default_params()
            if mass is None:
                model.build_Hamiltonian(g)
            else:
                model.build_Hamiltonian(g, mass)
            mb = model.momentum_basis
            model.diagonalize_Hamiltonian(2, "sparse")
            out[f"{tag}/L_col_ptr"] = np.asarray(mb["L_col_ptr"], dtype=np.int64)
            out[f"{tag}/L_row_idx"] = np.asarray(mb["L_row_idx"], dtype=np.int64)
            out[f"{tag}/L_data"] = np.asarray(mb["L_data"], dtype=np.complex128)
            out[f"{tag}/energies"] = np.asarray(model.H.Nenergies)
            out[f"{name}/keys"] = keys_of(model.sector_configs, model.loc_dims)
            print(tag, len(model.sector_configs), mb["n_cols"], model.H.Nenergies, flush=True)
    np.savez_compressed(os.path.join(HERE, "momentum_cases.npz"), **out)


NBODY_CASES = {
    # name: (factory, kwargs, g, m, [operator lists], [distance lists])
    "su2_1d_L8_obc": (su2_model, SU2_CASES["su2_1d_L8_obc"][0], 1.0, 0.5,
                      [["N_tot", "N_tot", "N_tot"], ["N_pair", "T2_px"]], [[[1], [2]], [[3]]]),
    "qed1d_L8_obc": (qed_model, QED_CASES["qed1d_L8_obc"][0], 1.0, 1.0, [["Q_px_dag", "Q_mx"], ["N", "E2_px", "N"]],
                     [[[1]], [[1], [2]]]),
    "qed2d_3x2_bg": (qed_model, QED_CASES["qed2d_3x2_bg"][0], 1.0, 1.0, [["N", "N"]], [[[1, 1]]]),
}


def gen_nbody():
    """N-body correlators (NBodyTerm.get_expval through get_observables /
    measure_observables) of the reference's ground state."""
    out = {}
    for name, (factory, kw, g, mass, ops, dists) in NBODY_CASES.items():
        model = factory(kw)
        model.build_Hamiltonian(g, mass)
        model.diagonalize_Hamiltonian(1, "sparse")
        model.get_observables([], [], [], nbody_obs=ops, nbody_dist=dists)
        model.measure_observables(0)
        out[f"{name}/psi"] = np.asarray(model.H.Npsi[0].psi, dtype=np.complex128)
        out[f"{name}/keys"] = keys_of(model.sector_configs, model.loc_dims)
        for names in ops:
            out[f"{name}/{'_'.join(names)}"] = np.asarray(model.res["_".join(names)], dtype=np.float64)
        print(name, {"_".join(n): model.res["_".join(n)] for n in ops}, flush=True)
    np.savez_compressed(os.path.join(HERE, "nbody_cases.npz"), **out)


OVERLAP_CASES = {
    # name: (factory, kwargs, labels)
    "su2_1d_L6_pbc": (SU2_Model, SU2_CASES["su2_1d_L6_pbc"][0], ["V", "PV", "T", "M", "B", "DW", "DW2", "X"]),
    "su2_1d_L8_obc": (SU2_Model, SU2_CASES["su2_1d_L8_obc"][0], ["V", "PV", "T", "M", "B", "DW", "DW2", "X"]),
    "su2_2d_2x2_obc": (SU2_Model, SU2_CASES["su2_2d_2x2_obc"][0], ["V", "PV1", "PV2"]),
    "su2_2d_2x2_pbc": (SU2_Model, dict(spin=0.5, pure_theory=False, lvals=[2, 2], has_obc=[False, False],
                                       sectors=[4]), ["V"]),
    "su2_2d_2x2_pure_pbc": (SU2_Model, SU2_CASES["su2_2d_2x2_pure_pbc"][0], ["V"]),
    "qed1d_L8_obc": (QED_Model, QED_CASES["qed1d_L8_obc"][0], ["V", "PV", "meson_center", "Meson Center"]),
    "qed1d_L6_pbc": (QED_Model, dict(spin=1, pure_theory=False, lvals=[6], has_obc=[False]), ["V", "meson_center"]),
}


def gen_overlap():
    """Named benchmark configurations (overlap_QMB_state) of the reference."""
    out = {}
    for name, (cls, kw, labels) in OVERLAP_CASES.items():
        model = cls(**kw)
        for lab in labels:
            out[f"{name}/{lab}"] = np.asarray(model.overlap_QMB_state(lab), dtype=np.int64)
        print(name, {lab: out[f"{name}/{lab}"].tolist() for lab in labels}, flush=True)
    np.savez_compressed(os.path.join(HERE, "overlap_cases.npz"), **out)


def gen_state():
    """QMB_state post-processing of the reference on the SU(2) L=8 OBC ground
    state: participation entropies, large-amplitude configurations and the
    expectation value of a seeded dense Hermitian matrix."""
    from edlgt.modeling.qmb_state import QMB_state

    kw = SU2_CASES["su2_1d_L8_obc"][0]
    model = su2_model(kw)
    model.build_Hamiltonian(1.0, 0.5)
    model.diagonalize_Hamiltonian(1, "sparse")
    psi = np.asarray(model.H.Npsi[0].psi, dtype=np.complex128)
    st = QMB_state(psi, model.lvals, model.loc_dims)
    out = {"psi": psi, "keys": keys_of(model.sector_configs, model.loc_dims)}
    for a in (0.5, 2, 3):
        out[f"PE_{a}"] = np.float64(st.participation_renyi_entropy(a))
    cfgs, vals = st.get_state_configurations(1e-2, model.sector_configs, return_configs=True)
    out["cfgs"], out["vals"] = np.asarray(cfgs, dtype=np.int64), np.asarray(vals)
    cfgs, vals = st.get_state_configurations(0.9, model.sector_configs, return_configs=True)
    out["cfgs_relaxed"], out["vals_relaxed"] = np.asarray(cfgs, dtype=np.int64), np.asarray(vals)
    rng = np.random.default_rng(21)
    n = len(psi)
    m = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    m = m + m.conj().T
    out["ev_dense_real"] = np.float64(st.expectation_value(m, "real"))
    out["ev_dense_imag"] = np.float64(st.expectation_value(1j * m, "imag"))
    np.savez_compressed(os.path.join(HERE, "state_cases.npz"), **out)
    print("state", {k: out[k] for k in out if k.startswith("PE") or k.startswith("ev")}, len(out["cfgs"]),
          len(out["cfgs_relaxed"]), flush=True)


def gen_local():
    """SU2_Model.build_local_Hamiltonian of the reference (SU(2) L=8 OBC,
    g^2 = 1, m = 0.5) around the interior sites 3 and 6, as canonical CSR (an
    open-chain edge site makes the reference concatenate an empty bond list)."""
    out = {}
    kw = SU2_CASES["su2_1d_L8_obc"][0]
    for R0 in (3, 6):
        model = su2_model(kw)
        model.build_local_Hamiltonian(1.0, 0.5, R0)
        H = model.Hlocal
        H._materialize_triplets()
        n = len(model.sector_configs)
        m = coo_matrix((H.value_list, (H.row_list.astype(np.int64), H.col_list.astype(np.int64))),
                       shape=(n, n)).tocsr()
        m.sum_duplicates()
        m.sort_indices()
        out[f"R{R0}/indptr"], out[f"R{R0}/indices"] = m.indptr.astype(np.int64), m.indices.astype(np.int64)
        out[f"R{R0}/data"] = np.asarray(m.data, dtype=np.complex128)
        print("local", R0, n, m.nnz, flush=True)
    np.savez_compressed(os.path.join(HERE, "local_hamiltonian_cases.npz"), **out)


INTEGRATED_CASES = {
    # name: (lvals, bg_list, g, m)
    "qedint_L4": ([4], None, 1.4, 0.7),
    "qedint_L8_bg": ([8], [1, 0, 0, 0, 0, 0, 0, -1], 1.0, 0.5),
    "qedint_L10": ([10], None, 0.8, 1.2),
}


def gen_integrated():
    """Integrated-gauge 1D QED (spin="integrated") through the reference's
    build_Hamiltonian: sector keys, canonical matrix and two lowest energies."""
    out = {}
    for name, (lvals, bg, g, mass) in INTEGRATED_CASES.items():
        model = QED_Model(spin="integrated", pure_theory=False, lvals=lvals, has_obc=[True], bg_list=bg)
        model.build_Hamiltonian(g, mass)
        out |= sector_record(model, f"{name}/", True)
        out |= matrix_record(canonical(model), f"{name}/H_", True)
        model.diagonalize_Hamiltonian(2, "sparse")
        out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
        print(name, len(model.sector_configs), model.H.Nenergies, flush=True)
    np.savez_compressed(os.path.join(HERE, "integrated_cases.npz"), **out)


def gen_full():
    """Full spectrum of SU(2) L=6 PBC (g=1, m=5, dim 282) through the
    reference's dense path: energies, r value, thermal functions, thermal beta
    and ensemble averages of the bare vacuum, exact time evolution."""
    kw = SU2_CASES["su2_1d_L6_pbc"][0]
    model = su2_model(kw)
    model.build_Hamiltonian(1.0, 5.0)
    model.diagonalize_Hamiltonian("full", "dense")
    out = {"energies": np.asarray(model.H.Nenergies)}
    out["r_array"] = np.asarray(model.H.get_r_value())
    out["r_value"] = np.float64(model.H.r_value)
    beta = 0.7
    out["beta"] = np.float64(beta)
    out["Z"] = np.float64(model.H.partition_function(beta))
    out["F"] = np.float64(model.H.free_energy(beta))
    out["E_thermal"] = np.float64(model.H.thermal_average(beta))
    out["F_prime"] = np.float64(model.H.F_prime(beta))
    config = model.overlap_QMB_state("V")
    state = model.get_qmb_state_from_configs([config])
    out["config"] = np.asarray(config, dtype=np.int64)
    out["beta_state"] = np.float64(model.get_thermal_beta(state, 1e-10))
    # canonical_avg itself hands the sector triplets of LocalTerm.get_Hamiltonian
    # to csc_matrix, which scipy rejects; its formula is evaluated here with the
    # reference's own pieces (compute_expH and the same triplets)
    from edlgt.modeling import LocalTerm

    rows, cols, vals = LocalTerm(model.ops["N_tot"], "N_tot", **model.def_params).get_Hamiltonian(1)
    n = len(model.sector_configs)
    op = coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
    expm_matrix = model.compute_expH(beta)
    Z = np.real(expm_matrix.trace())
    out["canonical_N_tot"] = np.float64(np.real(op.dot(expm_matrix).trace()) / (Z * model.n_sites))
    psi_th, me = model.microcanonical_avg(["N_tot", "T2_px"], state)
    out["ME_psi"] = np.asarray(psi_th)
    out["ME_N_tot"], out["ME_T2_px"] = np.float64(me["ME_N_tot"]), np.float64(me["ME_T2_px"])
    de = model.diagonal_avg(["N_tot", "T2_px"], state)
    out["DE_N_tot"], out["DE_T2_px"] = np.float64(de["DE_N_tot"]), np.float64(de["DE_T2_px"])
    tline = np.array([0.0, 0.25, 0.5, 1.0, 2.0])
    model.time_evolution_Hamiltonian(state, tline)
    out["time"] = tline
    out["psi_time"] = np.array([p.psi for p in model.H.psi_time])
    out["keys"] = keys_of(model.sector_configs, model.loc_dims)
    print("full", len(model.sector_configs), out["r_value"], out["beta_state"], me, de, flush=True)
    np.savez_compressed(os.path.join(HERE, "full_spectrum_cases.npz"), **out)


def _parity_string(s, k):
    return float(s % 2)


def _dyadic_string(s, k):
    return 0.25 * ((s + k) % 3)


def gen_string():
    """String (site-resolved background) constraints: the reference's
    symmetry_sector_configs with string_op_diags/string_sectors, which
    dispatches to iterative_sitebased_sym_sector_configs1
    (edlgt/symmetries/symmetry_sector.py:68-145, 970-1164).  Every input of
    the call is stored with the resulting sorted keys, so the test pins the
    builder directly.  String diagonals are model operators or synthetic
    per-site functions of the local state (any real diagonal is a valid
    input); targets are read off a configuration of the sector without
    strings, so the sector contains it.  One case has an infeasible target
    and an empty result."""
    from edlgt.modeling.lattice_geometry import get_lattice_link_site_pairs
    from edlgt.symmetries import get_symmetry_sector_generators, symmetry_sector_configs

    qed1 = (QED_Model, dict(spin=1, pure_theory=False, lvals=[8], has_obc=[True]), "N", 4, "E")
    qed32 = (QED_Model, dict(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True]), "N", 3, "E")
    qed42 = (QED_Model, dict(spin=1, pure_theory=False, lvals=[4, 2], has_obc=[True, True]), "N", 4, "E")
    su8p = (SU2_Model, dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[False], sectors=[8]), "N_tot", 8, "T2")
    su10 = (SU2_Model, dict(spin=0.5, pure_theory=False, lvals=[10], has_obc=[True], sectors=[10]), "N_tot", 10, "T2")
    su12 = (SU2_Model, dict(spin=0.5, pure_theory=False, lvals=[12], has_obc=[True], sectors=[12]), "N_tot", 12, "T2")
    cases = {
        "qed1d_L8_N_E2": (qed1, ["N", "E2_px"], 0.61),
        "qed2d_3x2_N": (qed32, ["N"], 0.5),
        "qed2d_4x2_N": (qed42, ["N"], 0.5),
        "qed2d_4x2_dyadic": (qed42, [_dyadic_string], 0.4),
        "su2_L8_pbc_Ntot_T2": (su8p, ["N_tot", "T2_px"], 0.7),
        "su2_L10_Npair": (su10, ["N_pair"], 0.45),
        "su2_L12_parity": (su12, [_parity_string], 0.4),
        "qed1d_L8_empty": (qed1, ["N"], None),
    }
    out = {}
    for name, ((cls, kw, gop, gsec, lname), sops, frac) in cases.items():
        m = cls(**kw)
        link_ops = [[m.ops[f"{lname}_p{d}"], -m.ops[f"{lname}_m{d}"]] for d in m.directions]
        gd = get_symmetry_sector_generators([m.ops[gop]], action="global")
        ld = get_symmetry_sector_generators(link_ops, action="link")
        pairs = get_lattice_link_site_pairs(m.lvals, m.has_obc)
        gs = np.array([gsec], dtype=float)
        lsec = [0 for _ in m.directions]
        base = symmetry_sector_configs(loc_dims=m.loc_dims, glob_op_diags=gd, glob_sectors=gs, sym_type_flag="U",
                                       link_op_diags=ld, link_sectors=lsec, pair_list=pairs)
        n_sites, dmax = gd.shape[1], gd.shape[2]
        rows = []
        for o in sops:
            if isinstance(o, str):
                rows.append(get_symmetry_sector_generators([m.ops[o]], action="global")[0])
            else:
                rows.append(np.array([[o(st, k) for st in range(dmax)] for k in range(n_sites)], dtype=float))
        sd = np.stack(rows)
        if frac is None:
            # every site occupied: infeasible with the global sector
            targets = np.ones((len(sops), n_sites))
        else:
            c = np.asarray(base[int(frac * (len(base) - 1))], dtype=np.int64)
            targets = np.array([[sd[k, s, c[s]] for s in range(n_sites)] for k in range(len(sops))])
        cfg = symmetry_sector_configs(loc_dims=m.loc_dims, glob_op_diags=gd, glob_sectors=gs, sym_type_flag="U",
                                      link_op_diags=ld, link_sectors=lsec, pair_list=pairs, string_op_diags=sd,
                                      string_sectors=targets)
        cfg = np.zeros((0, n_sites), dtype=np.uint16) if cfg is None else np.asarray(cfg)
        out[f"{name}/loc_dims"] = np.asarray(m.loc_dims, dtype=np.int64)
        out[f"{name}/glob_diags"] = np.asarray(gd)
        out[f"{name}/glob_sectors"] = gs
        out[f"{name}/link_diags"] = np.asarray(ld)
        out[f"{name}/link_sectors"] = np.asarray(lsec, dtype=float)
        out[f"{name}/n_dirs"] = np.int64(len(pairs))
        for d, pl in enumerate(pairs):
            out[f"{name}/pairs{d}"] = np.asarray(pl, dtype=np.int64)
        out[f"{name}/string_diags"] = sd
        out[f"{name}/string_sectors"] = targets
        out[f"{name}/keys"] = keys_of(cfg, m.loc_dims) if len(cfg) else np.zeros(0, dtype=np.uint64)
        out[f"{name}/base_dim"] = np.int64(len(base))
        print(name, len(base), "->", len(cfg), flush=True)
    np.savez_compressed(os.path.join(HERE, "string_cases.npz"), **out)


SU2_GEN_CASES = {
    "su2gen_1d_L4_obc_j1": (dict(spin=1, pure_theory=False, lvals=[4], has_obc=[True], sectors=[4]), 1.0, 1.0),
    "su2gen_1d_L6_obc_j1": (dict(spin=1, pure_theory=False, lvals=[6], has_obc=[True], sectors=[6]), 0.8, 0.5),
    "su2gen_1d_L4_pbc_j1": (dict(spin=1, pure_theory=False, lvals=[4], has_obc=[False], sectors=[4]), 1.3, 0.7),
    "su2gen_1d_L6_obc_j12": (dict(spin=0.5, pure_theory=False, lvals=[6], has_obc=[True], sectors=[6],
                                  use_generic_model=True), 1.0, 0.5),
    "su2gen_1d_L4_obc_j32": (dict(spin=1.5, pure_theory=False, lvals=[4], has_obc=[True], sectors=[4]), 1.0, 1.0),
    "su2gen_2d_2x2_pure_pbc_j1": (dict(spin=1, pure_theory=True, lvals=[2, 2], has_obc=[False, False]), 1.2, None),
    "su2gen_2d_2x2_obc_j1": (dict(spin=1, pure_theory=False, lvals=[2, 2], has_obc=[True, True], sectors=[4]),
                             1.0, 1.0),
}


def gen_generic_su2():
    """The generic SU(2) model (j_max >= 1, or use_generic_model): the
    reference's SU2_gen_dressed_site_operators and build_gen_Hamiltonian
    (edlgt/operators/SU2_operators.py:302-622, edlgt/models/SU2_model.py:
    357-472): sector keys, canonical matrices and the lowest energies."""
    out = {}
    for name, (kw, g, mass) in SU2_GEN_CASES.items():
        t0 = time.time()
        model = su2_model(kw)
        out |= sector_record(model, f"{name}/", True)
        model.build_Hamiltonian(g, mass)
        out |= matrix_record(canonical(model), f"{name}/H_", True)
        out[f"{name}/g"] = np.float64(g)
        out[f"{name}/m"] = np.float64(np.nan if mass is None else mass)
        k = 2 if len(model.sector_configs) > 3 else 1
        model.diagonalize_Hamiltonian(k, "sparse")
        out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
        print(name, len(model.sector_configs), list(model.loc_dims), f"{time.time() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "generic_su2_cases.npz"), **out)


def gen_thermal():
    """Thermal functions without the full spectrum: the reference's expm
    branches (edlgt/modeling/qmb_hamiltonian.py:446-452, 486-489, 505-508,
    545-551; edlgt/models/quantum_model.py:904-938) after a two-eigenvalue
    diagonalisation of SU(2) L=6 PBC (g=1, m=5, dim 282), in the "sparse"
    format (Tr(H^2 e^-bH) by matrix power) and the "dense" format (the
    elementwise square of the dense array)."""
    from edlgt.modeling import LocalTerm

    out = {}
    kw = SU2_CASES["su2_1d_L6_pbc"][0]
    for fmt in ("sparse", "dense"):
        model = su2_model(kw)
        model.build_Hamiltonian(1.0, 5.0)
        model.diagonalize_Hamiltonian(2, fmt)
        p = f"{fmt}/"
        for beta in (0.3, 0.7):
            q = f"{p}b{beta}/"
            out[q + "Z"] = np.float64(model.H.partition_function(beta))
            out[q + "F"] = np.float64(model.H.free_energy(beta))
            out[q + "E_thermal"] = np.float64(model.H.thermal_average(beta))
            out[q + "F_prime"] = np.float64(model.H.F_prime(beta))
            # canonical_avg's formula with the reference's own pieces (its
            # csc_matrix call on the LocalTerm triplets is rejected by scipy)
            rows, cols, vals = LocalTerm(model.ops["T2_px"], "T2_px", **model.def_params).get_Hamiltonian(1)
            n = len(model.sector_configs)
            op = coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
            expm_matrix = model.compute_expH(beta)
            Z = np.real(expm_matrix.trace())
            out[q + "canonical_T2_px"] = np.float64(np.real(op.dot(expm_matrix).trace()) / (Z * model.n_sites))
        out[p + "energies"] = np.asarray(model.H.Nenergies)
        if fmt == "sparse":
            # in the dense format the reference's Newton iteration (with the
            # elementwise square) runs away and exhausts the host memory, so
            # the thermal beta is pinned in the sparse format only
            config = model.overlap_QMB_state("V")
            state = model.get_qmb_state_from_configs([config])
            out[p + "config"] = np.asarray(config, dtype=np.int64)
            out[p + "beta_state"] = np.float64(model.get_thermal_beta(state, 1e-10))
        print("thermal", fmt, out[p + "b0.7/Z"], out[p + "b0.7/F_prime"], flush=True)
    np.savez_compressed(os.path.join(HERE, "thermal_cases.npz"), **out)


WIDE_CASES = {
    # name: (kwargs, g); pure gauge lattices whose key space exceeds 63 bits
    "qed2d_4x4_pure_pbc_s1": (dict(spin=1, pure_theory=True, lvals=[4, 4], has_obc=[False, False]), 1.1),
    "qed2d_4x4_pure_obc_s2": (dict(spin=2, pure_theory=True, lvals=[4, 4], has_obc=[True, True]), 0.9),
}


def gen_wide():
    """Sectors whose key space exceeds 63 bits (product of the local
    dimensions >= 2^63): the reference's uint16 sector tables (dimension,
    sha256 of the table bytes, every 997th row), the canonical matrix digest
    and the two lowest energies."""
    out = {}
    for name, (kw, g) in WIDE_CASES.items():
        t0 = time.time()
        model = qed_model(kw)
        cfg = np.ascontiguousarray(model.sector_configs, dtype=np.uint16)
        out[f"{name}/dim"] = np.int64(cfg.shape[0])
        out[f"{name}/configs_sha"] = np.array(sha(cfg))
        out[f"{name}/sample_rows"] = np.arange(0, cfg.shape[0], 997, dtype=np.int64)
        out[f"{name}/sample_configs"] = cfg[::997].copy()
        out[f"{name}/loc_dims"] = np.asarray(model.loc_dims, dtype=np.int64)
        out[f"{name}/g"] = np.float64(g)
        t1 = time.time()
        model.build_Hamiltonian(g)
        out |= matrix_record(canonical(model), f"{name}/H_", False)
        t2 = time.time()
        model.diagonalize_Hamiltonian(2, "sparse")
        out[f"{name}/energies"] = np.asarray(model.H.Nenergies)
        out[f"{name}/seconds"] = np.array([t1 - t0, t2 - t1, time.time() - t2])
        print(name, cfg.shape[0], f"bits {np.log2(np.prod(np.asarray(model.loc_dims, dtype=float))):.1f}",
              f"{time.time() - t0:.1f}s", model.H.Nenergies, flush=True)
    np.savez_compressed(os.path.join(HERE, "wide_cases.npz"), **out)


if __name__ == "__main__":
    groups = sys.argv[1:] or ["small", "pins", "dynamics", "big", "twobody", "entropy", "momentum", "full", "nbody",
                             "overlap", "state", "local", "integrated", "string", "generic", "wide", "thermal"]
    if "thermal" in groups:
        gen_thermal()
    if "wide" in groups:
        gen_wide()
    if "generic" in groups:
        gen_generic_su2()
    if "string" in groups:
        gen_string()
    if "integrated" in groups:
        gen_integrated()
    if "local" in groups:
        gen_local()
    if "state" in groups:
        gen_state()
    if "overlap" in groups:
        gen_overlap()
    if "nbody" in groups:
        gen_nbody()
    if "full" in groups:
        gen_full()
    if "momentum" in groups:
        gen_momentum()
    if "entropy" in groups:
        gen_entropy()
    if "twobody" in groups:
        gen_twobody()
    if "small" in groups:
        gen_small()
    if "pins" in groups:
        gen_validation_pins()
    if "dynamics" in groups:
        gen_dynamics()
    if "big" in groups:
        gen_big()
