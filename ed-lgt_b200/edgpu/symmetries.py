"""Symmetry sectors on the device: generator diagonals, exact integer
constraint tables, level-by-level enumeration and config<->index lookup.

Public functions mirror ``edlgt.symmetries``:

* ``get_symmetry_sector_generators`` (``symmetry_sector.py:148-196``);
* ``symmetry_sector_configs`` (``symmetry_sector.py:68-145``),
  ``get_link_sector_configs`` (``:1167-1234``) and ``global_abelian_sector``
  (``global_abelian_sym.py:147-198``), all served by one GPU enumerator that
  returns a :class:`Sector` (sorted keys on the device, configurations on
  demand);
* ``config_to_index_binarysearch`` (``generate_configs.py:145-173``).

Generator diagonals of the gauge models are dyadic rationals; they are scaled
by the smallest power of two that makes every value an integer, which turns
the reference's float comparisons with tolerance 1e-13 into exact integer
tests.  A generator that cannot be scaled this way is rejected.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = [
    "Sector",
    "SectorSpec",
    "get_symmetry_sector_generators",
    "enumerate_sector",
    "symmetry_sector_configs",
    "get_link_sector_configs",
    "global_abelian_sector",
    "compute_strides",
    "key_layout",
    "config_to_index_binarysearch",
]

SYM_TOL = 1e-13


KEY_WORD_LIMIT = 2**63


def key_layout(loc_dims):
    """Key layout of a lattice: ``(key_words, n_hi, lo_space)``.

    One word (``(1, 0, prod d)``) when the product of the local dimensions is
    below 2^63.  Otherwise two words: the low word takes the longest run of
    trailing sites whose dimensions multiply to less than 2^63 (``lo_space``),
    the high word the ``n_hi`` leading sites, whose product must also stay
    below 2^63 (126 bits of key space in all).  The key is then the 128-bit
    number ``hi * 2**64 + lo``, ordered like the configurations."""
    dims = [int(d) for d in np.asarray(loc_dims, dtype=np.int64)]
    total = math.prod(dims)
    if total < KEY_WORD_LIMIT:
        return 1, 0, total
    lo_space, n_hi = 1, len(dims)
    while n_hi > 0 and lo_space * dims[n_hi - 1] < KEY_WORD_LIMIT:
        n_hi -= 1
        lo_space *= dims[n_hi]
    if math.prod(dims[:n_hi]) >= KEY_WORD_LIMIT:
        raise OverflowError("the product of local dimensions exceeds a two-word (126-bit) key")
    return 2, n_hi, lo_space


def compute_strides(loc_dims, n_hi: int = 0) -> np.ndarray:
    """Mixed-radix strides with the last site fastest (``tools/magic.py:41-80``).

    With ``n_hi > 0`` (two-word keys) the strides of sites ``[0, n_hi)`` are
    relative to the high word and restart at 1 on site ``n_hi - 1``."""
    loc_dims = np.asarray(loc_dims, dtype=np.int64)
    strides = np.empty(len(loc_dims), dtype=np.uint64)
    run = 1
    for k in range(len(loc_dims) - 1, -1, -1):
        if k == n_hi - 1:
            run = 1
        strides[k] = run
        run *= int(loc_dims[k])
    return strides


def get_symmetry_sector_generators(op_list, action: str) -> np.ndarray:
    """Site-resolved real diagonals of symmetry generators.

    ``action`` is ``"global"`` / ``"nbody"`` (list of ``(n_sites, d, d)``
    operators) or ``"link"`` (list over directions of pairs of operators).
    """
    if action in ("global", "nbody"):
        n_sites, dmax = op_list[0].shape[0], op_list[0].shape[1]
        out = np.zeros((len(op_list), n_sites, dmax))
        for i, op in enumerate(op_list):
            for s in range(n_sites):
                out[i, s] = np.real(np.diagonal(op[s]))
        return out
    if action == "link":
        n_dirs = len(op_list)
        n_sites, dmax = op_list[0][0].shape[0], op_list[0][0].shape[1]
        out = np.zeros((n_dirs, 2, n_sites, dmax))
        for d in range(n_dirs):
            for e in range(2):
                for s in range(n_sites):
                    out[d, e, s] = np.real(np.diagonal(op_list[d][e][s]))
        return out
    raise ValueError(f"action must be 'global', 'link' or 'nbody', got {action!r}")


def _dyadic_scale(values) -> int:
    parts = [np.ravel(np.asarray(v, dtype=float)) for v in values if v is not None and np.size(v)]
    if not parts:
        return 1
    vals = np.concatenate(parts)
    for k in range(0, 21):
        s = float(2**k)
        if np.all(np.abs(vals * s - np.round(vals * s)) < 1e-9):
            if np.max(np.abs(np.round(vals * s))) > 2**28:
                break
            return int(s)
    raise ValueError("symmetry generators are not dyadic rationals: no exact integer form")


class SectorSpec:
    """All constraints of a sector in the form the device enumerator takes."""

    def __init__(
        self,
        loc_dims,
        glob_op_diags=None,
        glob_sectors=None,
        sym_type_flag="U",
        link_op_diags=None,
        link_sectors=None,
        pair_list=None,
        string_op_diags=None,
        string_sectors=None,
        nbody_op_diags=None,
        nbody_sectors=None,
        nbody_sites_list=None,
        nbody_sym_type="U",
    ):
        self.loc_dims = np.asarray(loc_dims, dtype=np.int64)
        n = len(self.loc_dims)
        if not 0 < n <= _lib.MAX_SITES:
            raise ValueError(f"1..{_lib.MAX_SITES} sites supported, got {n}")
        self.key_words, self.n_hi, self.lo_space = key_layout(self.loc_dims)
        self.n_sites = n
        self.dmax = int(self.loc_dims.max())
        self.strides = compute_strides(self.loc_dims, self.n_hi)
        dm = self.dmax

        def pad(a, lead):
            a = np.asarray(a, dtype=float)
            out = np.zeros(lead + (n, dm))
            out[..., : a.shape[-1]] = a[..., :dm]
            return out

        # string (site-local) constraints -> allowed states
        allowed = np.zeros((n, dm), dtype=np.uint8)
        for s in range(n):
            allowed[s, : self.loc_dims[s]] = 1
        if string_op_diags is not None:
            sd = np.asarray(string_op_diags, dtype=float)
            st = np.asarray(string_sectors, dtype=float)
            for k in range(sd.shape[0]):
                for s in range(n):
                    for c in range(self.loc_dims[s]):
                        if abs(sd[k, s, c] - st[k, s]) > SYM_TOL:
                            allowed[s, c] = 0
        self.site_allowed = allowed
        # global symmetries
        self.glob_type = 0 if sym_type_flag in ("U", 0) else 1
        if glob_op_diags is not None:
            g = pad(glob_op_diags, (np.asarray(glob_op_diags).shape[0],))
            tg = np.asarray(glob_sectors, dtype=float).reshape(-1)
            if g.shape[0] > 4:
                raise ValueError("at most 4 global symmetries are supported")
        else:
            g = np.zeros((0, n, dm))
            tg = np.zeros(0)
        # link symmetries
        if link_op_diags is not None:
            lv = np.asarray(link_op_diags, dtype=float)
            lt = np.asarray(link_sectors, dtype=float).reshape(-1)
            lv = pad(lv, lv.shape[:2])
        else:
            lv = np.zeros((0, 2, n, dm))
            lt = np.zeros(0)
        # n-body symmetries
        self.nbody_type = 0 if nbody_sym_type in ("U", 0, None) else 1
        if nbody_op_diags is not None:
            nv = pad(nbody_op_diags, (np.asarray(nbody_op_diags).shape[0],))
            nt = np.asarray(nbody_sectors, dtype=float).reshape(-1)
            nsites = [np.asarray(x, dtype=np.int64) for x in nbody_sites_list]
        else:
            nv = np.zeros((0, n, dm))
            nt = np.zeros(0)
            nsites = []
        # exact integer forms
        if self.glob_type == 0:
            sg = _dyadic_scale([g[:, s, : self.loc_dims[s]] for s in range(n)] + [tg])
            self.glob_val = np.round(g * sg).astype(np.int32)
            self.glob_target = np.round(tg * sg).astype(np.int32)
        else:
            self.glob_val, self.glob_target = self._z2_bits(g, tg, "global")
        sl = _dyadic_scale([lv[:, :, s, : self.loc_dims[s]] for s in range(n)] + [lt])
        self.link_val = np.round(lv * sl).astype(np.int32)
        self.link_target = np.round(lt * sl).astype(np.int32)
        if self.nbody_type == 0:
            sn = _dyadic_scale([nv[:, s, : self.loc_dims[s]] for s in range(n)] + [nt])
            self.nb_val = np.round(nv * sn).astype(np.int32)
            self.nb_target = np.round(nt * sn).astype(np.int32)
        else:
            self.nb_val, self.nb_target = self._z2_bits(nv, nt, "n-body")
        # reachable min/max of the remaining sites (U(1) branch and bound)
        ng = self.glob_val.shape[0]
        rem_min = np.zeros((ng, n + 1), dtype=np.int64)
        rem_max = np.zeros((ng, n + 1), dtype=np.int64)
        for gi in range(ng):
            for s in range(n - 1, -1, -1):
                vals = self.glob_val[gi, s, : self.loc_dims[s]]
                rem_min[gi, s] = rem_min[gi, s + 1] + int(vals.min())
                rem_max[gi, s] = rem_max[gi, s + 1] + int(vals.max())
        self.glob_rem_min = rem_min.astype(np.int32)
        self.glob_rem_max = rem_max.astype(np.int32)
        # link pairs grouped by activation site (the later endpoint)
        pairs = []
        if pair_list is not None:
            for d, plist in enumerate(pair_list):
                for s0, s1 in np.asarray(plist, dtype=np.int64).reshape(-1, 2):
                    pairs.append((max(s0, s1), int(s0), int(s1), d))
        pairs.sort(key=lambda x: x[0])
        self.pair_start = np.zeros(n + 1, dtype=np.int32)
        for a, *_ in pairs:
            self.pair_start[a + 1] += 1
        self.pair_start = np.cumsum(self.pair_start).astype(np.int32)
        self.pair_s0 = np.array([p[1] for p in pairs], dtype=np.int32)
        self.pair_s1 = np.array([p[2] for p in pairs], dtype=np.int32)
        self.pair_dir = np.array([p[3] for p in pairs], dtype=np.int32)
        # n-body constraints grouped by activation
        acts = sorted((int(x.max()), i) for i, x in enumerate(nsites)) if nsites else []
        self.nb_start = np.zeros(n + 1, dtype=np.int32)
        for a, _ in acts:
            self.nb_start[a + 1] += 1
        self.nb_start = np.cumsum(self.nb_start).astype(np.int32)
        self.nb_id = np.array([i for _, i in acts], dtype=np.int32)
        self.nb_site_start = np.zeros(len(nsites) + 1, dtype=np.int32)
        for i, x in enumerate(nsites):
            self.nb_site_start[i + 1] = self.nb_site_start[i] + len(x)
        self.nb_sites = np.concatenate(nsites).astype(np.int32) if nsites else np.zeros(0, dtype=np.int32)
        self.has_nbody = len(nsites) > 0

    def _z2_bits(self, vals, targets, what):
        bits = np.zeros(vals.shape, dtype=np.int32)
        for i in range(vals.shape[0]):
            for s in range(self.n_sites):
                for c in range(self.loc_dims[s]):
                    v = vals[i, s, c]
                    if abs(v - 1) < 1e-10:
                        bits[i, s, c] = 0
                    elif abs(v + 1) < 1e-10:
                        bits[i, s, c] = 1
                    else:
                        raise ValueError(f"{what} Z2 generator has a diagonal entry {v} not in {{+1,-1}}")
        tb = np.zeros(len(targets), dtype=np.int32)
        for i, t in enumerate(targets):
            if abs(t - 1) < 1e-10:
                tb[i] = 0
            elif abs(t + 1) < 1e-10:
                tb[i] = 1
            else:
                tb[i] = -1  # unreachable target: empty sector
        return bits, tb


class _DeviceTables:
    """Device copies of a SectorSpec plus the ctypes struct pointing at them."""

    def __init__(self, spec: SectorSpec, device):
        def dev(a, dtype):
            a = np.ascontiguousarray(a)
            if a.size == 0:
                a = np.zeros(1, dtype=a.dtype)
            return torch.from_numpy(a.astype(dtype, copy=False)).to(device)

        self._keep = {
            "allowed": dev(spec.site_allowed, np.uint8),
            "gv": dev(spec.glob_val, np.int32),
            "gt": dev(spec.glob_target, np.int32),
            "gmin": dev(spec.glob_rem_min, np.int32),
            "gmax": dev(spec.glob_rem_max, np.int32),
            "lv": dev(spec.link_val, np.int32),
            "lt": dev(spec.link_target, np.int32),
            "ps": dev(spec.pair_start, np.int32),
            "p0": dev(spec.pair_s0, np.int32),
            "p1": dev(spec.pair_s1, np.int32),
            "pd": dev(spec.pair_dir, np.int32),
            "nv": dev(spec.nb_val, np.int32),
            "nt": dev(spec.nb_target, np.int32),
            "ns": dev(spec.nb_start, np.int32),
            "ni": dev(spec.nb_id, np.int32),
            "nss": dev(spec.nb_site_start, np.int32),
            "nsi": dev(spec.nb_sites, np.int32),
        }
        k = self._keep
        t = _lib.SectorTables()
        t.n_sites = spec.n_sites
        t.dmax = spec.dmax
        for s in range(spec.n_sites):
            t.loc_dims[s] = int(spec.loc_dims[s])
            t.strides[s] = int(spec.strides[s])
        t.site_allowed = ptr(k["allowed"])
        t.n_glob = spec.glob_val.shape[0]
        t.glob_type = spec.glob_type
        t.glob_val = ptr(k["gv"])
        t.glob_target = ptr(k["gt"])
        t.glob_rem_min = ptr(k["gmin"])
        t.glob_rem_max = ptr(k["gmax"])
        t.n_dirs = spec.link_val.shape[0]
        t.link_val = ptr(k["lv"])
        t.link_target = ptr(k["lt"])
        t.pair_start = ptr(k["ps"])
        t.pair_s0 = ptr(k["p0"])
        t.pair_s1 = ptr(k["p1"])
        t.pair_dir = ptr(k["pd"])
        t.nbody_type = spec.nbody_type
        t.nb_val = ptr(k["nv"])
        t.nb_target = ptr(k["nt"])
        t.nb_start = ptr(k["ns"]) if spec.has_nbody else None
        t.nb_id = ptr(k["ni"])
        t.nb_site_start = ptr(k["nss"])
        t.nb_sites = ptr(k["nsi"])
        t.key_words = spec.key_words
        t.n_hi = spec.n_hi
        self.struct = t


class Sector:
    """A symmetry sector: sorted keys on the device (int64 storage).

    One-word keys are a ``(N,)`` tensor; two-word keys (key space above 2^63,
    :func:`key_layout`) a ``(N, 2)`` tensor of (low, high) words.
    ``configs`` decodes the keys to the reference's ``(N, n_sites)`` uint16
    table on demand; ``index_of`` looks configurations up on the device.
    """

    def __init__(self, keys: torch.Tensor, loc_dims, device=None):
        self.keys = keys
        self.loc_dims = np.asarray(loc_dims, dtype=np.int64)
        self.n_sites = len(self.loc_dims)
        self.key_words, self.n_hi, self.lo_space = key_layout(self.loc_dims)
        if (keys.dim() == 2) != (self.key_words == 2):
            raise ValueError("key tensor shape does not match the key layout of loc_dims")
        self.strides = compute_strides(self.loc_dims, self.n_hi)
        self.device = keys.device if device is None else device
        self._configs = None
        self._lookup = None

    def __len__(self):
        return int(self.keys.shape[0])

    @property
    def dim(self) -> int:
        return len(self)

    @property
    def wide(self) -> bool:
        """True for two-word keys."""
        return self.key_words == 2

    def require_narrow(self, what: str):
        """Refuses callers that handle one-word keys only."""
        if self.wide:
            raise NotImplementedError(f"{what}: sectors whose key space exceeds 63 bits are not supported")

    # ------------------------------------------------------------------ lookup
    def lookup_table(self):
        """Bucket table over the top bits of the dense key (built once, kept
        on the device)."""
        if self._lookup is None:
            n = len(self)
            key_space = int(np.prod(self.loc_dims.astype(object)))
            key_bits = max(1, int(key_space - 1).bit_length())
            bucket_bits = max(1, min(key_bits, max(1, (max(n, 1) // 2).bit_length()), 24))
            shift = key_bits - bucket_bits
            n_buckets = ((key_space - 1) >> shift) + 1
            starts = torch.empty(n_buckets + 1, dtype=torch.int64, device=self.device)
            if self.wide:
                check(lib.edg_lookup_build_wide(ptr(self.keys), n, 2, self.lo_space, shift, n_buckets, ptr(starts),
                                                stream_handle()), "edg_lookup_build_wide")
            else:
                check(lib.edg_lookup_build(ptr(self.keys), n, shift, n_buckets, ptr(starts), stream_handle()),
                      "edg_lookup_build")
            t = _lib.LookupTable()
            t.keys = ptr(self.keys)
            t.n = n
            t.bucket_start = ptr(starts)
            t.shift = shift
            t.n_buckets = n_buckets
            t.key_words = self.key_words
            t.n_hi = self.n_hi
            t.lo_space = self.lo_space if self.wide else 0
            self._lookup = (t, starts)
        return self._lookup[0]

    def encode(self, configs) -> torch.Tensor:
        """(M, n_sites) configurations -> int64 keys on the device ((M,) or
        (M, 2) for two-word keys)."""
        c = torch.as_tensor(np.ascontiguousarray(np.asarray(configs, dtype=np.uint16)).reshape(-1, self.n_sites))
        c = c.to(self.device)
        strides = torch.from_numpy(self.strides.astype(np.int64)).to(self.device)
        m = c.shape[0]
        if self.wide:
            keys = torch.empty((m, 2), dtype=torch.int64, device=self.device)
            check(lib.edg_configs_to_keys_wide(ptr(c), m, self.n_sites, self.n_hi, ptr(strides), ptr(keys),
                                               stream_handle()), "edg_configs_to_keys_wide")
        else:
            keys = torch.empty(m, dtype=torch.int64, device=self.device)
            check(lib.edg_configs_to_keys(ptr(c), m, self.n_sites, ptr(strides), ptr(keys), stream_handle()),
                  "edg_configs_to_keys")
        return keys

    def index_of(self, configs) -> np.ndarray:
        """Row index of each configuration, -1 when not in the sector."""
        q = self.encode(configs)
        out = torch.empty(q.shape[0], dtype=torch.int64, device=self.device)
        check(lib.edg_lookup(self.lookup_table(), ptr(q), q.shape[0], ptr(out), stream_handle()), "edg_lookup")
        return out.cpu().numpy()

    @property
    def configs(self) -> np.ndarray:
        """The sector as the reference's lexicographically sorted uint16 table."""
        if self._configs is None:
            n = len(self)
            out = torch.empty((max(n, 1), self.n_sites), dtype=torch.int16, device=self.device)
            ld = torch.from_numpy(self.loc_dims.astype(np.int32)).to(self.device)
            if self.wide:
                check(lib.edg_keys_to_configs_wide(ptr(self.keys), n, self.n_sites, self.n_hi, ptr(ld), ptr(out),
                                                   stream_handle()), "edg_keys_to_configs_wide")
            else:
                check(lib.edg_keys_to_configs(ptr(self.keys), n, self.n_sites, ptr(ld), ptr(out), stream_handle()),
                      "edg_keys_to_configs")
            self._configs = out[:n].cpu().numpy().view(np.uint16)
        return self._configs

    def host_keys(self) -> np.ndarray:
        """uint64 keys on the host: (N,), or (N, 2) (low, high) words."""
        return self.keys.cpu().numpy().view(np.uint64)


def enumerate_sector(spec: SectorSpec, device=None) -> Sector:
    """Level-by-level enumeration on the device; returns the sorted sector."""
    device = torch.device("cuda") if device is None else torch.device(device)
    tables = _DeviceTables(spec, device)
    st = stream_handle()
    ng = spec.glob_val.shape[0]
    kshape = (lambda m: (m, 2)) if spec.key_words == 2 else (lambda m: (m,))
    prev_keys = torch.zeros(kshape(1), dtype=torch.int64, device=device)
    prev_sums = torch.zeros(max(ng, 1), dtype=torch.int32, device=device)
    n_prev = 1
    level_sizes = []
    for depth in range(spec.n_sites):
        n_cand = n_prev * int(spec.loc_dims[depth])
        nb = lib.edg_sector_level_blocks(n_cand)
        offsets = torch.empty(nb + 1, dtype=torch.int64, device=device)
        scratch = torch.empty(lib.edg_scan_scratch_elems(nb), dtype=torch.int64, device=device)
        check(lib.edg_sector_level_count(C_ref(tables.struct), depth, ptr(prev_keys), ptr(prev_sums), n_prev,
                                         ptr(offsets), ptr(scratch), st), "edg_sector_level_count")
        total = int(offsets[nb].item())
        next_keys = torch.empty(kshape(max(total, 1)), dtype=torch.int64, device=device)
        next_sums = torch.empty(max(total * ng, 1), dtype=torch.int32, device=device)
        if total > 0:
            check(lib.edg_sector_level_fill(C_ref(tables.struct), depth, ptr(prev_keys), ptr(prev_sums), n_prev,
                                            ptr(offsets), ptr(next_keys), ptr(next_sums), st), "edg_sector_level_fill")
        prev_keys, prev_sums, n_prev = next_keys, next_sums, total
        level_sizes.append(total)
        if total == 0:
            break
    keys = prev_keys[:n_prev].clone()
    sector = Sector(keys, spec.loc_dims, device)
    sector.level_sizes = level_sizes  # surviving prefixes per depth
    sector.n_glob = ng
    return sector


def C_ref(struct):
    import ctypes

    return ctypes.byref(struct)


# ---------------------------------------------------------------------------
# reference-shaped entry points
# ---------------------------------------------------------------------------
def symmetry_sector_configs(loc_dims, glob_op_diags, glob_sectors, sym_type_flag, link_op_diags, link_sectors,
                            pair_list, string_op_diags=None, string_sectors=None, return_sector=False):
    """Global + link (+ string) sector; uint16 (N, n_sites) sorted table."""
    spec = SectorSpec(loc_dims, glob_op_diags, glob_sectors, sym_type_flag, link_op_diags, link_sectors, pair_list,
                      string_op_diags, string_sectors)
    sec = enumerate_sector(spec)
    return sec if return_sector else sec.configs


def get_link_sector_configs(loc_dims, link_op_diags, link_sectors, pair_list, nbody_op_diags=None,
                            nbody_sectors=None, nbody_sites_list=None, nbody_sym_type="U", return_sector=False):
    """Link (+ n-body) sector; uint16 (N, n_sites) sorted table."""
    spec = SectorSpec(loc_dims, link_op_diags=link_op_diags, link_sectors=link_sectors, pair_list=pair_list,
                      nbody_op_diags=nbody_op_diags, nbody_sectors=nbody_sectors,
                      nbody_sites_list=nbody_sites_list, nbody_sym_type=nbody_sym_type)
    sec = enumerate_sector(spec)
    return sec if return_sector else sec.configs


def global_abelian_sector(loc_dims, sym_op_diags, sym_sectors, sym_type="U", return_sector=False):
    """Global-only sector; uint16 (N, n_sites) sorted table."""
    spec = SectorSpec(loc_dims, sym_op_diags, sym_sectors, sym_type)
    sec = enumerate_sector(spec)
    return sec if return_sector else sec.configs


def config_to_index_binarysearch(config, sector) -> int:
    """Row of ``config`` in the sector (-1 if absent)."""
    if not isinstance(sector, Sector):
        raise TypeError("config_to_index_binarysearch needs a Sector")
    return int(sector.index_of(np.asarray(config).reshape(1, -1))[0])
