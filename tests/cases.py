"""Model cases of the golden fixtures (same parameters as make_golden.py)."""

QED_CASES = {
    "qed1d_L4_obc": (dict(spin=1, pure_theory=False, lvals=[4], has_obc=[True]), 1.0, 1.0),
    "qed1d_L4_pbc": (dict(spin=1, pure_theory=False, lvals=[4], has_obc=[False]), 1.0, 1.0),
    "qed1d_L8_obc": (dict(spin=1, pure_theory=False, lvals=[8], has_obc=[True]), 1.0, 1.0),
    "qed2d_3x2_bg": (dict(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True],
                          bg_list=[-1, 0, 0, 0, 0, 1]), 1.0, 1.0),
    "qed2d_3x2_q0": (dict(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True]), 0.7, 0.4),
    "qed2d_2x2_pure_pbc": (dict(spin=1, pure_theory=True, lvals=[2, 2], has_obc=[False, False]), 1.3, None),
    "qed2d_3x2_pure_obc": (dict(spin=1, pure_theory=True, lvals=[3, 2], has_obc=[True, True]), 0.8, None),
}
QED_CHARGE = {-2: [1, 0, 0, 0, 0, 1], -1: [1, 0, 0, 0, 0, 0], 1: [-1, 0, 0, 0, 0, 0], 2: [-1, 0, 0, 0, 0, -1]}
for _q, _bg in QED_CHARGE.items():
    QED_CASES[f"qed2d_3x2_Q{_q:+d}"] = (dict(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True],
                                             bg_list=_bg, charge=_q), 1.0, 1.0)

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

ALL_CASES = {**QED_CASES, **SU2_CASES}

BIG_CASES = {
    "su2_1d_L12_obc": dict(spin=0.5, pure_theory=False, lvals=[12], has_obc=[True], sectors=[12]),
    "su2_1d_L14_obc": dict(spin=0.5, pure_theory=False, lvals=[14], has_obc=[True], sectors=[14]),
    "su2_1d_L14_pbc": dict(spin=0.5, pure_theory=False, lvals=[14], has_obc=[False], sectors=[14]),
    "su2_1d_L16_obc_pair": dict(spin=0.5, pure_theory=False, lvals=[16], has_obc=[True], sectors=[16],
                                bg_list=[0] * 5 + [0.5] + [0] * 4 + [0.5] + [0] * 5),
}


def build(name, device="cpu", big=False):
    from edgpu.models import QED_Model, SU2_Model

    if big:
        return SU2_Model(**BIG_CASES[name], device=device)
    kw, g, m = ALL_CASES[name]
    cls = QED_Model if name.startswith("qed") else SU2_Model
    return cls(**kw, device=device), g, m

# two-body correlator fixtures: case name -> operator pairs measured on the ground state
TWOBODY_CASES = {
    "qed1d_L8_obc": [["N", "N"], ["E2_px", "N"]],
    "qed2d_3x2_bg": [["N", "N"], ["E2_px", "E2_py"]],
    "su2_1d_L8_obc": [["N_tot", "N_tot"], ["N_pair", "T2_px"]],
}

# entanglement fixtures: case name -> subsystems measured on the ground state
ENTROPY_CASES = {
    "qed1d_L8_obc": [[0, 1, 2, 3], [1, 2, 5], [0, 1]],
    "qed2d_3x2_bg": [[0, 1, 2], [0, 3], [4]],
    "su2_1d_L8_obc": [[0, 1, 2, 3], [2, 3, 6], [0, 1]],
}

# momentum fixtures: name -> (model kwargs, g, m, unit cell, k vectors)
MOMENTUM_CASES = {
    "su2_1d_L6_pbc": (dict(spin=0.5, pure_theory=False, lvals=[6], has_obc=[False], sectors=[6]), 1.0, 5.0, [1],
                      [[0], [1], [3]]),
    "su2_1d_L8_pbc_uc2": (dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[False], sectors=[8]), 1.0, 0.5, [2],
                          [[0], [1], [2]]),
    "qed1d_L6_pbc_uc2": (dict(spin=1, pure_theory=False, lvals=[6], has_obc=[False]), 1.0, 1.0, [2], [[0], [1]]),
    "qed2d_2x2_pure_pbc": (dict(spin=1, pure_theory=True, lvals=[2, 2], has_obc=[False, False]), 1.3, None, [1, 1],
                           [[0, 0], [1, 0], [1, 1]]),
    "su2_1d_L6_pbc_tc": (dict(spin=0.5, pure_theory=False, lvals=[6], has_obc=[False], sectors=[6]), 1.0, 5.0, [1],
                         [[0], [1], [3]]),
    "su2_1d_L8_pbc_tc": (dict(spin=0.5, pure_theory=False, lvals=[8], has_obc=[False], sectors=[8]), 1.0, 0.5, [1],
                         [[0], [2], [5]]),
}
# the TC variant's fixed tables (six-state SU(2) j=1/2 dressed site)
TC_MAP = [4, 5, 2, 3, 0, 1]
TC_SIGN = [1.0, 1.0, 1.0, -1.0, 1.0, 1.0]


def build_momentum_case(name, device="cpu"):
    from edgpu.models import QED_Model, SU2_Model

    kw, g, m, ucs, ks = MOMENTUM_CASES[name]
    cls = QED_Model if name.startswith("qed") else SU2_Model
    return cls(**kw, device=device), g, m, ucs, ks

# n-body correlator fixtures: name -> ([operator lists], [distance lists])
NBODY_CASES = {
    "su2_1d_L8_obc": ([["N_tot", "N_tot", "N_tot"], ["N_pair", "T2_px"]], [[[1], [2]], [[3]]]),
    "qed1d_L8_obc": ([["Q_px_dag", "Q_mx"], ["N", "E2_px", "N"]], [[[1]], [[1], [2]]]),
    "qed2d_3x2_bg": ([["N", "N"]], [[[1, 1]]]),
}


def nbody_instances(lvals, has_obc, distances):
    """Site lists of an n-body pattern from every starting site (PBC wraps, a
    pattern leaving an open lattice is dropped), zig-zag site order."""
    from edgpu.lattice import inverse_zig_zag, zig_zag

    n = 1
    for L in lvals:
        n *= L
    out = []
    for ii in range(n):
        c0 = zig_zag(lvals, ii)
        sites = [ii]
        for d in distances:
            c = [c0[k] + d[k] for k in range(len(lvals))]
            c = [c[k] % lvals[k] if not has_obc[k] else c[k] for k in range(len(lvals))]
            if not all(0 <= c[k] < lvals[k] for k in range(len(lvals))):
                sites = None
                break
            sites.append(inverse_zig_zag(lvals, tuple(c)))
        if sites is not None:
            out.append(sites)
    return out

# integrated-gauge 1D QED fixtures: name -> (lvals, bg_list, g, m)
INTEGRATED_CASES = {
    "qedint_L4": ([4], None, 1.4, 0.7),
    "qedint_L8_bg": ([8], [1, 0, 0, 0, 0, 0, 0, -1], 1.0, 0.5),
    "qedint_L10": ([10], None, 0.8, 1.2),
}


# ---------------------------------------------------------------------------
# string (site-resolved) constraint cases, stored with every input of the
# reference's symmetry_sector_configs call (tests/golden/string_cases.npz)
def string_case_names(golden):
    return sorted({k.split("/")[0] for k in golden.files})


def string_case_inputs(golden, name):
    """Keyword inputs of a string case, in the reference's argument names."""
    pairs = [golden[f"{name}/pairs{d}"] for d in range(int(golden[f"{name}/n_dirs"]))]
    return dict(loc_dims=golden[f"{name}/loc_dims"], glob_op_diags=golden[f"{name}/glob_diags"],
                glob_sectors=golden[f"{name}/glob_sectors"], sym_type_flag="U",
                link_op_diags=golden[f"{name}/link_diags"], link_sectors=golden[f"{name}/link_sectors"],
                pair_list=pairs, string_op_diags=golden[f"{name}/string_diags"],
                string_sectors=golden[f"{name}/string_sectors"])


# generic SU(2) model cases (j_max >= 1, or use_generic_model), same
# parameters as tests/golden/make_golden.py's SU2_GEN_CASES
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


def build_generic(name, device="cpu"):
    from edgpu.models import SU2_Model

    kw, g, m = SU2_GEN_CASES[name]
    return SU2_Model(**kw, device=device), g, m


# lattices whose key space exceeds 63 bits (two-word keys); fixtures from
# tests/golden/make_golden.py wide
WIDE_CASES = {
    "qed2d_4x4_pure_pbc_s1": (dict(spin=1, pure_theory=True, lvals=[4, 4], has_obc=[False, False]), 1.1),
    "qed2d_4x4_pure_obc_s2": (dict(spin=2, pure_theory=True, lvals=[4, 4], has_obc=[True, True]), 0.9),
}


def build_wide(name, device="cpu"):
    from edgpu.models import QED_Model

    kw, g = WIDE_CASES[name]
    return QED_Model(**kw, device=device), g
