"""Host-side logic: lattice geometry, exact integer constraint tables, term
instance lists (no device needed)."""

import numpy as np
import pytest

from edgpu import lattice as Lt
from edgpu.symmetries import SectorSpec, compute_strides


def test_site_linearisation_roundtrip():
    lvals = [3, 4, 2]
    for i in range(24):
        assert Lt.inverse_zig_zag(lvals, Lt.zig_zag(lvals, i)) == i
    assert Lt.zig_zag(lvals, 1) == (1, 0, 0)  # x fastest


@pytest.mark.parametrize("lvals,obc,count", [([8], [True], 7), ([8], [False], 8), ([3, 2], [True, True], 2 * 2 + 3 * 1)])
def test_link_pairs(lvals, obc, count):
    pairs = Lt.link_site_pairs(lvals, obc)
    assert sum(len(p) for p in pairs) == count


def test_plaquettes_and_labels():
    assert Lt.plaquette_sites((0, 0), [3, 2], ["x", "y"], [True, True]) == [0, 1, 3, 4]
    assert Lt.plaquette_sites((2, 0), [3, 2], ["x", "y"], [True, True]) is None
    labels = Lt.lattice_labels([3, 2], [True, True], True)
    assert labels[0] == "even_mx_my" and labels[1] == "odd_my" and labels[5] == "odd_px_py"


def test_strides_last_site_fastest():
    assert list(compute_strides([2, 5, 3])) == [15, 3, 1]


def test_dyadic_generators_become_integers():
    # SU(2) Casimir values 0 and 3/4 on the link: scaled by 4
    n, d = 3, 3
    link = np.zeros((1, 2, n, d))
    link[0, 0] = [0, 0.75, 0.75]
    link[0, 1] = [0, -0.75, -0.75]
    spec = SectorSpec([3, 3, 3], link_op_diags=link, link_sectors=[0], pair_list=[np.array([[0, 1], [1, 2]])])
    assert set(np.unique(spec.link_val)) <= {0, 3, -3}
    assert list(spec.pair_start) == [0, 0, 1, 2]


def test_non_dyadic_generator_rejected():
    g = np.full((1, 2, 2), 1.0 / 3.0)
    with pytest.raises(ValueError):
        SectorSpec([2, 2], glob_op_diags=g, glob_sectors=[2.0 / 3.0])


def test_z2_generator_bits():
    g = np.array([[[1.0, -1.0], [1.0, -1.0]]])
    spec = SectorSpec([2, 2], glob_op_diags=g, glob_sectors=[1.0], sym_type_flag="Z")
    assert spec.glob_val.tolist() == [[[0, 1], [0, 1]]] and spec.glob_target.tolist() == [0]
    with pytest.raises(ValueError):
        SectorSpec([2, 2], glob_op_diags=np.full((1, 2, 2), 0.5), glob_sectors=[1.0], sym_type_flag="Z")


def test_key_overflow_rejected():
    """Two-word keys cover up to 126 bits of key space; beyond it the spec
    is refused."""
    spec = SectorSpec([1000] * 8)
    assert (spec.key_words, spec.n_hi, spec.lo_space) == (2, 2, 1000**6)
    with pytest.raises(OverflowError):
        SectorSpec([1000] * 13)


def test_term_instances_follow_reference_loops():
    from cases import build

    model, g, m = build("su2_1d_L8_obc")
    blocks = model.hamiltonian_blocks(g, m)
    names = [b.name for b in blocks]
    assert names[0] == "E_square"
    hop = [b for b in blocks if b.name.startswith("Qpx_dag")]
    # even-masked and odd-masked hopping over the 7 links of an open chain
    assert [b.n_instances for b in hop] == [4, 3]
    assert all(b.add_dagger for b in hop)
    model2, g2, m2 = build("qed2d_3x2_bg")
    plaq = [b for b in model2.hamiltonian_blocks(g2, m2) if len(b.ops) == 4]
    assert len(plaq) == 1 and plaq[0].n_instances == 2
