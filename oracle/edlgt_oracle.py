"""CPU oracle for the ED hot path -- TEST INFRASTRUCTURE ONLY.

A numpy/scipy restatement of ed-lgt's algorithms for the path that the
device engine replaces.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it, and only as the checker; the
engine never calls it.  Parity of this restatement with the reference itself
is pinned by the fixtures in ``tests/golden`` (generated by running the
reference, see ``tests/golden/make_golden.py``) and by
``tests/test_oracle_golden.py``.

Functions and the reference code they restate:

* :func:`sector_configs` -- iterative_sitebased_sym_sector_configs(1) and
  iterative_link_sector_configs(_plus)
  (edlgt/symmetries/symmetry_sector.py:785-967, 970-1164, 1237-1469): grow
  prefixes one site at a time, keep running U(1) sums with min/max
  reachability pruning, Z2 products checked at the last site, link pairs and
  n-body constraints checked when their last site is assigned, tolerance
  SYM_TOL = 1e-13;
* :func:`config_to_index` -- config_to_index_binarysearch
  (edlgt/symmetries/generate_configs.py:145-173) via mixed-radix keys
  (edlgt/tools/magic.py:41-140);
* :func:`nbody_triplets`, :func:`localbody_triplets` -- nbody_data /
  nbody_data_2sites / nbody_data_4sites / localbody_data_par
  (edlgt/symmetries/sym_qmb_operations.py:32-602), OP_TOL = 1e-10;
* :func:`assemble` -- the term site loops with their h.c. handling
  (edlgt/modeling/{local,twobody,plaquette}_term.py) and the summed sparse
  build (edlgt/modeling/qmb_hamiltonian.py:173-225);
* :func:`lowest_eigs` -- scipy.sparse.linalg.eigsh(H, k, which="SA") as in
  QMB_hamiltonian.diagonalize (qmb_hamiltonian.py:260-332);
* :func:`evolve` -- scipy expm_multiply(-iH, ...) as in
  QMB_hamiltonian.time_evolution (qmb_hamiltonian.py:334-426).
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix, csr_matrix
from scipy.sparse.linalg import eigsh, expm_multiply

SYM_TOL = 1e-13
OP_TOL = 1e-10

__all__ = [
    "strides_of",
    "keys_of",
    "sector_configs",
    "config_to_index",
    "nbody_triplets",
    "localbody_triplets",
    "assemble",
    "lowest_eigs",
    "evolve",
    "local_expval",
]


def strides_of(loc_dims):
    loc_dims = np.asarray(loc_dims, dtype=np.uint64)
    s = np.ones(len(loc_dims), dtype=np.uint64)
    for k in range(len(loc_dims) - 2, -1, -1):
        s[k] = s[k + 1] * loc_dims[k + 1]
    return s


def keys_of(configs, loc_dims):
    c = np.asarray(configs, dtype=np.uint64)
    return (c * strides_of(loc_dims)[None, :]).sum(axis=1, dtype=np.uint64)


def _narrow(loc_dims):
    return int(np.prod(np.asarray(loc_dims, dtype=object))) < 2**63


def searchable(configs, loc_dims):
    """Row keys whose order is the lexicographic order of the configurations:
    uint64 mixed-radix keys when the key space is below 2^63, else the
    configurations as big-endian byte strings (the comparison
    config_to_index_binarysearch makes element by element,
    edlgt/symmetries/generate_configs.py:145-173)."""
    c = np.ascontiguousarray(np.atleast_2d(configs), dtype=np.uint16)
    if _narrow(loc_dims):
        return keys_of(c, loc_dims)
    return np.ascontiguousarray(c.astype(">u2")).view(f"V{2 * c.shape[1]}").reshape(-1)


def sector_configs(loc_dims, glob_diags=None, glob_sectors=None, glob_type="U", link_diags=None, link_sectors=None,
                   pair_list=None, string_diags=None, string_sectors=None, nbody_diags=None, nbody_sectors=None,
                   nbody_sites=None, nbody_type="U"):
    """Lexicographically sorted uint16 (N, n_sites) sector table."""
    loc_dims = np.asarray(loc_dims, dtype=np.int64)
    n = len(loc_dims)
    g = None if glob_diags is None else np.asarray(glob_diags, dtype=float)
    gs = None if glob_sectors is None else np.asarray(glob_sectors, dtype=float).reshape(-1)
    ng = 0 if g is None else g.shape[0]
    if ng and glob_type == "U":
        mins = np.zeros((ng, n + 1))
        maxs = np.zeros((ng, n + 1))
        for s in range(n - 1, -1, -1):
            v = g[:, s, : loc_dims[s]]
            mins[:, s] = mins[:, s + 1] + v.min(axis=1)
            maxs[:, s] = maxs[:, s + 1] + v.max(axis=1)
    pairs_at = [[] for _ in range(n)]
    if pair_list is not None:
        for d, plist in enumerate(pair_list):
            for s0, s1 in np.asarray(plist, dtype=np.int64).reshape(-1, 2):
                pairs_at[max(s0, s1)].append((int(s0), int(s1), d))
    lv = None if link_diags is None else np.asarray(link_diags, dtype=float)
    lt = None if link_sectors is None else np.asarray(link_sectors, dtype=float).reshape(-1)
    nb_at = [[] for _ in range(n)]
    if nbody_sites is not None:
        for i, sites in enumerate(nbody_sites):
            nb_at[int(np.max(sites))].append(i)
    nv = None if nbody_diags is None else np.asarray(nbody_diags, dtype=float)
    nt = None if nbody_sectors is None else np.asarray(nbody_sectors, dtype=float).reshape(-1)
    cfg = np.zeros((1, 0), dtype=np.uint16)
    vals = np.zeros((1, ng)) if glob_type == "U" else np.ones((1, ng))
    for s in range(n):
        d = int(loc_dims[s])
        m = cfg.shape[0]
        new = np.empty((m * d, s + 1), dtype=np.uint16)
        new[:, :s] = np.repeat(cfg, d, axis=0)
        st = np.tile(np.arange(d, dtype=np.uint16), m)
        new[:, s] = st
        keep = np.ones(m * d, dtype=bool)
        if string_diags is not None:
            sd = np.asarray(string_diags, dtype=float)
            ss = np.asarray(string_sectors, dtype=float)
            for k in range(sd.shape[0]):
                keep &= np.abs(sd[k, s, st] - ss[k, s]) <= SYM_TOL
        nvals = np.repeat(vals, d, axis=0)
        for gi in range(ng):
            if glob_type == "U":
                nvals[:, gi] += g[gi, s, st]
                if s < n - 1:
                    keep &= gs[gi] >= nvals[:, gi] + mins[gi, s + 1] - SYM_TOL
                    keep &= gs[gi] <= nvals[:, gi] + maxs[gi, s + 1] + SYM_TOL
                else:
                    keep &= np.abs(nvals[:, gi] - gs[gi]) <= SYM_TOL
            else:
                nvals[:, gi] *= g[gi, s, st]
                if s == n - 1:
                    keep &= np.abs(nvals[:, gi] - gs[gi]) <= SYM_TOL
        for s0, s1, dd in pairs_at[s]:
            v = lv[dd, 0, s0, new[:, s0]] + lv[dd, 1, s1, new[:, s1]]
            keep &= np.abs(v - lt[dd]) <= SYM_TOL
        for i in nb_at[s]:
            sites = np.asarray(nbody_sites[i], dtype=np.int64)
            if nbody_type == "U":
                v = np.zeros(m * d)
                for q in sites:
                    v += nv[i, q, new[:, q]]
            else:
                v = np.ones(m * d)
                for q in sites:
                    v *= nv[i, q, new[:, q]]
            keep &= np.abs(v - nt[i]) <= SYM_TOL
        cfg = new[keep]
        vals = nvals[keep]
    return cfg


def config_to_index(queries, sector_cfg, loc_dims):
    """Row of each query configuration in the sorted table, -1 if absent."""
    keys = searchable(sector_cfg, loc_dims)
    q = searchable(np.atleast_2d(queries), loc_dims)
    pos = np.searchsorted(keys, q)
    pos_c = np.minimum(pos, len(keys) - 1)
    hit = (pos < len(keys)) & (keys[pos_c] == q)
    return np.where(hit, pos_c, -1).astype(np.int64)


def _transitions(op):
    """Nonzero (ket, amp) per bra of one site operator (|amp| > OP_TOL)."""
    out = []
    for bra in range(op.shape[0]):
        kets = np.nonzero(np.abs(op[bra]) > OP_TOL)[0]
        out.append((kets, op[bra, kets]))
    return out


def nbody_triplets(op_list, op_sites, cfg, loc_dims):
    """(row, col, val) of prod_j op_j[site_j] in the sector (rows in order)."""
    op_sites = [int(s) for s in op_sites]
    trans = [_transitions(np.asarray(op_list[j][op_sites[j]], dtype=np.complex128)) for j in range(len(op_sites))]
    narrow = _narrow(loc_dims)
    keys = searchable(cfg, loc_dims)
    strides = strides_of(loc_dims).astype(np.int64) if narrow else None
    bra_states = cfg[:, op_sites].astype(np.int64)
    rows_out, cols_out, vals_out = [], [], []
    # group rows by their local bra states on the acted sites
    uniq, inv = np.unique(bra_states, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    per_row = []
    for gi, b in enumerate(uniq):
        rows = np.nonzero(inv == gi)[0]
        combos = [[]]
        for j, bj in enumerate(b):
            kets, amps = trans[j][bj]
            combos = [c + [(int(k), complex(a))] for c in combos for k, a in zip(kets, amps)]
        if not combos or any(len(c) != len(b) for c in combos):
            continue
        for t, combo in enumerate(combos):
            amp = 1.0 + 0.0j
            for _, a in combo:
                amp *= a
            if narrow:
                delta = sum((k - int(b[j])) * int(strides[op_sites[j]]) for j, (k, _) in enumerate(combo))
                ket_keys = (keys[rows].astype(np.int64) + delta).astype(np.uint64)
            else:
                kc = cfg[rows].copy()
                for j, (k, _) in enumerate(combo):
                    kc[:, op_sites[j]] = k
                ket_keys = searchable(kc, loc_dims)
            pos = np.searchsorted(keys, ket_keys)
            pos_c = np.minimum(pos, len(keys) - 1)
            col = np.where((pos < len(keys)) & (keys[pos_c] == ket_keys), pos_c, -1)
            per_row.append((rows, t, col, amp))
    if not per_row:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.complex128)
    for rows, t, col, amp in per_row:
        rows_out.append(rows)
        cols_out.append(col)
        vals_out.append(np.full(len(rows), amp))
    r = np.concatenate(rows_out)
    c = np.concatenate(cols_out)
    v = np.concatenate(vals_out)
    order = np.argsort(r, kind="stable")
    return r[order], c[order], v[order]


def localbody_triplets(op, site, cfg):
    """Diagonal-only local term; entries with |op_cc| < OP_TOL are dropped."""
    op_site = np.asarray(op[int(site)], dtype=np.complex128)
    v = op_site[cfg[:, int(site)], cfg[:, int(site)]]
    keep = np.abs(v) >= OP_TOL
    r = np.nonzero(keep)[0]
    return r, r, v[keep]


def assemble(blocks, cfg, loc_dims):
    """Canonical (duplicates summed) complex CSR of the sum of term blocks.

    A block needs ``ops``, ``sites`` (instances x factors), ``strength``,
    ``add_dagger`` and ``diagonal`` attributes.
    """
    n = cfg.shape[0]
    R, Cc, V = [], [], []
    for b in blocks:
        rr, cc, vv = [], [], []
        for inst in np.asarray(b.sites, dtype=np.int64).reshape(-1, len(b.ops)):
            if b.diagonal:
                r, c, v = localbody_triplets(b.ops[0], inst[0], cfg)
            else:
                r, c, v = nbody_triplets(b.ops, inst, cfg, loc_dims)
            rr.append(r)
            cc.append(c)
            vv.append(v)
        if not rr:
            continue
        r = np.concatenate(rr)
        c = np.concatenate(cc)
        v = np.concatenate(vv) * complex(b.strength)
        if np.any(c < 0):
            raise ValueError("a ket is outside the sector")
        R.append(r)
        Cc.append(c)
        V.append(v)
        if b.add_dagger:
            R.append(c)
            Cc.append(r)
            V.append(np.conj(v))
    r = np.concatenate(R) if R else np.zeros(0, np.int64)
    c = np.concatenate(Cc) if Cc else np.zeros(0, np.int64)
    v = np.concatenate(V) if V else np.zeros(0, np.complex128)
    m = coo_matrix((v, (r, c)), shape=(n, n)).tocsr()
    m.sum_duplicates()
    m.sort_indices()
    return m


def lowest_eigs(H, k=1):
    """k lowest eigenvalues (ascending) and vectors of a Hermitian matrix."""
    n = H.shape[0]
    if n <= 64 or k >= n - 1:
        from scipy.linalg import eigh

        w, v = eigh(H.toarray() if hasattr(H, "toarray") else H)
        return w[:k], v[:, :k]
    w, v = eigsh(H, k=k, which="SA")
    o = np.argsort(w)
    return w[o], v[:, o]


def evolve(H, psi0, time_line):
    """psi(t_k) for a uniform time grid (rows), as QMB_hamiltonian does."""
    t = np.asarray(time_line, dtype=float)
    return expm_multiply(-1j * csr_matrix(H), np.asarray(psi0, dtype=np.complex128), start=t[0], stop=t[-1],
                         num=len(t), endpoint=True)


def local_expval(psi, op, cfg):
    """<psi| op_s |psi> per site using the operator diagonal (LocalTerm)."""
    p2 = np.abs(np.asarray(psi)) ** 2
    n_sites = cfg.shape[1]
    out = np.zeros(n_sites)
    for s in range(n_sites):
        d = np.real(np.diagonal(np.asarray(op[s])))
        out[s] = np.sum(p2 * d[cfg[:, s]])
    return out


def twobody_expval(psi, op_a, op_b, cfg, loc_dims):
    """corr[i, j] = corr[j, i] = Re <psi| A_i B_j |psi> for all pairs i < j, the
    loop of lattice_twobody_exp_val (edlgt/modeling/twobody_term.py:232-264)
    over the two-site triplets (nbody_data_2sites) and exp_val_data
    (edlgt/modeling/qmb_state.py:631-654)."""
    psi = np.asarray(psi, dtype=np.complex128)
    n = cfg.shape[1]
    corr = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            rows, cols, vals = nbody_triplets([op_a, op_b], [i, j], cfg, loc_dims)
            ok = cols >= 0
            e = np.sum(np.conj(psi[rows[ok]]) * vals[ok] * psi[cols[ok]])
            corr[i, j] = corr[j, i] = float(np.real(e))
    return corr


def partition(cfg, loc_dims, keep):
    """QuantumModel._get_partition with _unique_configs_with_inverse
    (edlgt/models/quantum_model.py:715-791, 73-117): distinct subsystem and
    environment rows (np.unique on their packed keys) and each row's index."""
    n = cfg.shape[1]
    keep = sorted(int(i) for i in keep)
    env = [i for i in range(n) if i not in keep]
    out = {"subsys_indices": np.array(keep), "env_indices": np.array(env)}
    for tag, cols in (("subsys", keep), ("env", env)):
        sub = cfg[:, cols]
        if len(cols) == 0:
            uniq, inv = np.empty((1, 0), dtype=cfg.dtype), np.zeros(cfg.shape[0], dtype=np.int64)
        else:
            k = keys_of(sub, np.asarray(loc_dims)[cols])
            _, first, inv = np.unique(k, return_index=True, return_inverse=True)
            uniq = sub[first]
        out[f"unique_{tag}_configs"] = uniq
        out[f"{tag}_map"] = inv.reshape(-1).astype(np.int64)
        out[f"{tag}_dim"] = uniq.shape[0]
    return out


def psi_matrix(psi, part):
    """build_psi_matrix (edlgt/modeling/qmb_state.py:596-627)."""
    m = np.zeros((part["subsys_dim"], part["env_dim"]), dtype=np.complex128)
    m[part["subsys_map"], part["env_map"]] = psi
    return m


def reduced_density_matrix(psi, part):
    """QMB_state.reduced_density_matrix, sector case (qmb_state.py:211-243)."""
    m = psi_matrix(psi, part)
    return m @ m.conj().T


def entanglement_entropy(psi, part):
    """QMB_state.entanglement_entropy with the dense SVD branch
    (qmb_state.py:245-291): -sum l log2 l over squared singular values > 1e-10."""
    m = psi_matrix(psi, part)
    if min(m.shape) == 1:
        return 0.0
    lam = np.linalg.svd(m, compute_uv=False) ** 2
    lam = lam[lam > 1e-10]
    return float(-np.sum(lam * np.log2(lam)))


def translation_sources(lvals, unit_cell):
    """source[s, dest]: the site whose state lands on ``dest`` under block
    shift s (row-major shifts and sites, as _prepare_translation_source_sites,
    edlgt/symmetries/translational_sym.py:508-560)."""
    lvals = np.asarray(lvals, dtype=np.int64)
    ucs = np.asarray(unit_cell, dtype=np.int64)
    R = lvals // ucs
    n_sites = int(np.prod(lvals))
    coords = np.array(np.unravel_index(np.arange(n_sites), tuple(lvals))).T  # row-major
    shifts = np.array(np.unravel_index(np.arange(int(np.prod(R))), tuple(R))).T
    src = np.empty((len(shifts), n_sites), dtype=np.int64)
    for s, t in enumerate(shifts):
        dest = np.ravel_multi_index(tuple(((coords + t * ucs) % lvals).T), tuple(lvals))
        src[s, dest] = np.arange(n_sites)
    return src, R


def momentum_basis(cfg, loc_dims, lvals, unit_cell, k_vals, local_map=None, label_sign=None):
    """get_momentum_basis (translational_sym.py:1307-1358) for the zero-k and
    finite-k projectors (:697-949): (col_ptr, row_idx, data complex128, n_cols).
    Translations (build_all_translations :567-617) by key search; one
    reference per orbit, its smallest row; axis periods and the k filter of
    select_references (:620-694); Bloch sums over the period box with
    duplicates summed, finite-k entries with |a| <= 1e-14 dropped, columns
    normalised, rows ascending.  ``local_map`` / ``label_sign``: the TC
    variant (:455-505, 952-1303): the map applied once per unit shift, and
    odd shifts weighted by the reference's product of label signs."""
    src, R = translation_sources(lvals, unit_cell)
    keys = keys_of(cfg, loc_dims)
    n, n_shifts, D = len(cfg), len(src), len(R)
    trans = np.empty((n, n_shifts), dtype=np.int64)
    for s in range(n_shifts):
        moved = cfg[:, src[s]].astype(np.int64)
        if local_map is not None:
            for _ in range(s):
                moved = np.asarray(local_map, dtype=np.int64)[moved]
        tk = keys_of(moved, loc_dims)
        pos = np.searchsorted(keys, tk)
        ok = (pos < n) & (keys[np.minimum(pos, n - 1)] == tk)
        if not np.all(ok):
            raise ValueError("the sector is not closed under these translations")
        trans[:, s] = pos
    strides = np.ones(D, dtype=np.int64)
    for d in range(D - 2, -1, -1):
        strides[d] = strides[d + 1] * R[d + 1]
    k_vals = np.asarray(k_vals, dtype=np.int64)
    zero_k = not np.any(k_vals != 0)
    phase = [np.exp(-2j * np.pi * (k_vals[d] % R[d]) * np.arange(R[d]) / R[d]) for d in range(D)]
    cols = []
    for r in range(n):
        if trans[r].min() < r:
            continue
        p = np.empty(D, dtype=np.int64)
        for d in range(D):
            p[d] = next((q for q in range(1, R[d] + 1) if trans[r, (q % R[d]) * strides[d]] == r), R[d])
        if any((k_vals[d] * p[d]) % R[d] != 0 for d in range(D)):
            continue
        sign = 1.0 if label_sign is None else float(np.prod(np.asarray(label_sign)[cfg[r].astype(np.int64)]))
        acc = {}
        for t in np.ndindex(*p):
            full = int(np.dot(t, strides))
            row = int(trans[r, full])
            ph = 1.0 + 0j if zero_k else np.prod([phase[d][t[d]] for d in range(D)])
            if full & 1:
                ph = ph * sign
            acc[row] = acc.get(row, 0) + ph
        rows = np.array(sorted(acc), dtype=np.int64)
        vals = np.array([acc[x] for x in rows], dtype=np.complex128)
        if not zero_k:
            keep = np.abs(vals) > 1e-14
            rows, vals = rows[keep], vals[keep]
        nrm = np.sqrt(np.sum(np.abs(vals) ** 2))
        if zero_k and nrm ** 2 <= 1e-8:
            cols.append((rows, np.zeros_like(vals)))  # a cancelled sign-twisted orbit
        elif len(vals) == 0 or nrm ** 2 <= (0 if zero_k else 1e-30):
            cols.append((rows[:0], vals[:0]))
        else:
            cols.append((rows, vals / nrm))
    col_ptr = np.zeros(len(cols) + 1, dtype=np.int64)
    col_ptr[1:] = np.cumsum([len(c[0]) for c in cols])
    row_idx = np.concatenate([c[0] for c in cols]) if cols else np.zeros(0, dtype=np.int64)
    data = np.concatenate([c[1] for c in cols]) if cols else np.zeros(0, dtype=np.complex128)
    return col_ptr, row_idx, data, len(cols)
