"""Host-side checks of the Z_n engine's tables against the oracle (CPU only).

The device kernels translate packed keys by lane rotations, count fermion
signs with row masks, and decode a Gauss index by peeling the spanning tree.
These tests replay exactly that integer arithmetic in Python from the tables
the engine uploads, and compare it with the oracle's explicit site
permutations and its enumerated basis.
"""

import numpy as np
import pytest

from edgpu.models.zn_model import ZnLattice
from oracle.zn_oracle import ZnOracle

CASES = [(2, 2, 3), (2, 3, 3), (2, 2, 2), (2, 3, 2), (4, 2, 2), (2, 2, 4)]


def _translate(L, m, key):
    """Python replay of the device translate_key / translate_sign."""
    F, N, lx, ly = L.field_bits, L.n_sites, L.lx, L.ly
    R = 2 * L.link_bits * lx
    fmask, mmask = (1 << F) - 1, (1 << N) - 1
    f, o = key & fmask, (key >> F) & mmask
    if m["sf"]:
        f = ((f << m["sf"]) | (f >> (F - m["sf"]))) & fmask
    if m["sx"]:
        f = ((f << m["sx"]) & m["hif"]) | ((f >> (R - m["sx"])) & m["lof"])
    o2 = o
    if m["sm"]:
        o2 = ((o2 << m["sm"]) | (o2 >> (N - m["sm"]))) & mmask
    if m["smx"]:
        o2 = ((o2 << m["smx"]) & m["him"]) | ((o2 >> (lx - m["smx"])) & m["lom"])
    par = (bin(o & m["ylow"]).count("1") * bin(o & m["yhigh"]).count("1")) & 1
    if m["smx"]:
        for y in range(ly):
            row = o >> (lx * y)
            par ^= (bin(row & m["xhead"]).count("1") * bin(row & m["xtail"]).count("1")) & 1
    return f | (o2 << F), par


def _decode(L, g):
    """Python replay of the device decode (cotree digits, then peeling)."""
    rank_occ = L.lookup_tables()[2]
    r, d = divmod(g, L.pow_cot)
    occ = int(rank_occ[r])
    key = occ << L.field_bits
    b, mask = L.link_bits, (1 << L.link_bits) - 1
    for l in L.cotree:
        key |= (d % L.n) << (b * l)
        d //= L.n
    for v, pl, ps, others in L.peel:
        s = ((occ >> v) & 1) - ((L.odd_mask >> v) & 1)
        for l, sg in others:
            s -= sg * ((key >> (b * l)) & mask)
        key |= ((ps * s) % L.n) << (b * pl)
    return key


@pytest.mark.parametrize("lx,ly,n", CASES)
def test_translations_match_permutations(lx, ly, n):
    L = ZnLattice((lx, ly), n)
    o = ZnOracle(lx, ly, n)
    keys = [int(k) for k in o.keys]
    for (a, b) in L.group:
        m = L.translation_masks(a, b)
        o2, e2, sg = o.translate(a, b, o.occ, o.E)
        want = o.pack(o2, e2)
        for i in range(0, len(keys), max(1, len(keys) // 3000)):
            k2, par = _translate(L, m, keys[i])
            assert k2 == int(want[i])
            assert (1 - 2 * par) == int(sg[i])


@pytest.mark.parametrize("lx,ly,n", CASES)
def test_gauss_index_is_dense_and_decodes(lx, ly, n):
    L = ZnLattice((lx, ly), n)
    o = ZnOracle(lx, ly, n)
    assert L.n_gauss == o.dim
    g = np.array([L.gauss_index(int(k)) for k in o.keys])
    assert np.array_equal(np.sort(g), np.arange(L.n_gauss))
    for i in range(0, o.dim, max(1, o.dim // 2000)):
        assert _decode(L, int(g[i])) == int(o.keys[i])


@pytest.mark.parametrize("lx,ly,n", CASES)
def test_chunk_tables_reproduce_gauss_index(lx, ly, n):
    L = ZnLattice((lx, ly), n)
    chunk, occ_rank, _ = L.lookup_tables()
    o = ZnOracle(lx, ly, n)
    for i in range(0, o.dim, max(1, o.dim // 2000)):
        k = int(o.keys[i])
        g = int(occ_rank[k >> L.field_bits]) * L.pow_cot
        for c in range(chunk.shape[0]):
            g += int(chunk[c, (k >> (8 * c)) & 255])
        assert g == L.gauss_index(k)


def test_sector_sizes_full_lattice():
    """4x3 Z3 sector: 924 occupation sets times 3^13 cotree fields, |G| = 6."""
    L = ZnLattice((4, 3), 3)
    assert (L.n_fermions, L.n_cot, len(L.group)) == (6, 13, 6)
    assert L.n_gauss == 924 * 3**13 == 1_473_154_452
    assert L.field_bits + L.n_sites == 60


def test_lattice_rejects_bad_shapes():
    with pytest.raises(ValueError):
        ZnLattice((3, 2), 3)
    with pytest.raises(ValueError):
        ZnLattice((4, 4), 3)
    with pytest.raises(ValueError):
        ZnLattice((2, 2), 5)


@pytest.mark.parametrize("lx,ly,n", [(2, 2, 3), (2, 3, 3), (2, 2, 2), (2, 3, 2), (2, 2, 4)])
def test_oracle_pinned_by_reference_kernels(lx, ly, n):
    """The oracle's full Gauss-law sector Hamiltonian against the one ed-lgt's
    own sector builder and nbody_term produce from dressed-site Z_n tables
    (tests/golden/make_zn_golden.py): dimension, tr H, ||H||_F^2 and the three
    lowest eigenvalues, all basis independent."""
    import os

    from scipy.sparse.linalg import eigsh

    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "zn_cases.npz"))
    tag = f"{lx}x{ly}_z{n}"
    o = ZnOracle(lx, ly, n, momentum=False)
    assert o.dim == int(gold[f"{tag}_dim"])
    for i, (t, m, g) in enumerate(gold["couplings"]):
        H = o.hamiltonian(t, m, g, momentum=False)
        assert np.isclose(H.diagonal().sum(), gold[f"{tag}_trace"][i], rtol=1e-12, atol=1e-9)
        assert np.isclose((abs(H).power(2)).sum(), gold[f"{tag}_fro2"][i], rtol=1e-12)
        if o.dim <= 3000:
            e = np.linalg.eigvalsh(H.toarray())[:3]
        else:
            e = np.sort(eigsh(H, k=3, which="SA", tol=0, return_eigenvectors=False))
        assert np.allclose(e, gold[f"{tag}_energies"][i], rtol=1e-10, atol=1e-10)
