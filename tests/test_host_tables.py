"""Host-side transition tables of the assembly (edgpu/modeling/assembly.py):
the whole-array builders against a table-by-table, bra-by-bra restatement
(the per-table loops of _prepare_local_transition_data,
edlgt/symmetries/sym_qmb_operations.py:32-92, with the real form's common
phases).  No device work: the models are built with device="cpu"."""

import numpy as np
import pytest


def _loop_tables(blocks, phase_weights, force_complex, OP_TOL, uniform_phase, phase_vec):
    raw_tables, table_site, table_index, terms = [], [], {}, []
    for bi, b in enumerate(blocks):
        if b.diagonal:
            continue
        for dag in ([False, True] if b.add_dagger else [False]):
            for inst in b.sites:
                tabs = []
                for j, s in enumerate(inst):
                    key = (bi, j, int(s), dag)
                    if key not in table_index:
                        m = np.asarray(b.ops[j][int(s)], dtype=np.complex128)
                        if dag:
                            m = m.conj().T
                        table_index[key] = len(raw_tables)
                        raw_tables.append(m)
                        table_site.append(int(s))
                    tabs.append(table_index[key])
                coef = np.conj(b.strength) if dag else b.strength
                terms.append((tuple(int(s) for s in inst), tuple(tabs), complex(coef)))
    real_ok, tables_real, coefs_real = False, None, None
    if not force_complex:
        tabs_t, phases, ok = [], [], True
        for t, m in enumerate(raw_tables):
            if phase_weights is not None:
                phi = phase_vec(phase_weights[table_site[t]])
                m = np.conj(phi)[:, None] * m * phi[None, :]
            ph = uniform_phase(m)
            if ph is None:
                ok = False
                break
            tabs_t.append((m / ph).real)
            phases.append(ph)
        if ok:
            cr = []
            for _, tabs, coef in terms:
                z = coef
                for t in tabs:
                    z *= phases[t]
                if abs(z.imag) > 1e-12 * max(1.0, abs(z)):
                    ok = False
                    break
                cr.append(z.real)
        if ok:
            real_ok, tables_real, coefs_real = True, tabs_t, cr
    return raw_tables, terms, real_ok, tables_real, coefs_real


def _loop_arrays(raw_tables, dmax, is_complex, tables_real, OP_TOL):
    nt = max(len(raw_tables), 1)
    t_count = np.zeros((nt, dmax), dtype=np.int32)
    t_ket = np.zeros((nt, dmax, dmax), dtype=np.uint8)
    t_amp = np.zeros((nt, dmax, dmax, 2 if is_complex else 1), dtype=np.float64)
    for t, m0 in enumerate(raw_tables):
        mags = np.abs(m0)
        m = m0 if is_complex else tables_real[t]
        for bra in range(dmax):
            kets = np.nonzero(mags[bra] > OP_TOL)[0]
            t_count[t, bra] = len(kets)
            t_ket[t, bra, : len(kets)] = kets
            if is_complex:
                t_amp[t, bra, : len(kets), 0] = m[bra, kets].real
                t_amp[t, bra, : len(kets), 1] = m[bra, kets].imag
            else:
                t_amp[t, bra, : len(kets), 0] = m[bra, kets]
    return t_count, t_ket, t_amp


def _models():
    from edgpu.models import QED_Model, SU2_Model

    return {
        "su2_1d_L14_pbc": lambda: SU2_Model(spin=0.5, pure_theory=False, lvals=[14], has_obc=[False], sectors=[14],
                                            device="cpu"),
        "su2_2d_2x2_obc": lambda: SU2_Model(spin=0.5, pure_theory=False, lvals=[2, 2], has_obc=[True, True],
                                            sectors=[4], device="cpu"),
        "su2_spin1_1d_L4": lambda: SU2_Model(spin=1, pure_theory=False, lvals=[4], has_obc=[True], sectors=[4],
                                             device="cpu"),
        "su2_pure_2x2_pbc": lambda: SU2_Model(spin=0.5, pure_theory=True, lvals=[2, 2], has_obc=[False, False],
                                              device="cpu"),
        "qed_2d_3x2_obc": lambda: QED_Model(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True],
                                            device="cpu"),
        "qed_1d_L8_obc": lambda: QED_Model(spin=1, pure_theory=False, lvals=[8], has_obc=[True], device="cpu"),
    }


@pytest.mark.parametrize("name", list(_models().keys()))
@pytest.mark.parametrize("force_complex", [False, True])
def test_whole_array_tables_equal_the_loops(name, force_complex):
    from edgpu.modeling import assembly as A

    model = _models()[name]()
    blocks = model.hamiltonian_blocks(1.0, 0.5)
    dmax = max(b.ops[0].shape[-1] for b in blocks)
    pw = getattr(model, "phase_weights", None)
    got = A._offdiag_tables(blocks, pw, force_complex, dmax)
    want = _loop_tables(blocks, pw, force_complex, A.OP_TOL, A._uniform_phase, A._phase_vec)
    assert got[1] == want[1]  # instance records
    assert len(got[0]) == len(want[0]) and all(np.array_equal(a, b) for a, b in zip(got[0], want[0]))
    assert got[2] == want[2]  # real form admitted
    if got[2]:
        assert all(np.array_equal(a, b) for a, b in zip(got[3], want[3]))
        assert np.array_equal(np.asarray(got[4]), np.asarray(want[4]))
    for is_complex in ([False, True] if got[2] else [True]):
        arrays = A._table_arrays(got[0], got[1], dmax, is_complex, got[3], got[4])
        for a, b in zip(arrays[:3], _loop_arrays(want[0], dmax, is_complex, want[3], A.OP_TOL)):
            assert a.dtype == b.dtype and np.array_equal(a, b)
