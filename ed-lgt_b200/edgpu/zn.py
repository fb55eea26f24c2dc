"""Matrix-free Z_n engine: zero-momentum basis on the device, batched matvec,
and a batched thick-restart Lanczos over interleaved instance vectors.

The Hamiltonian of a :class:`~edgpu.models.zn_model.ZnLattice` is never
stored: ``edg_zn_matvec`` recomputes every element from the packed
representative keys and a 4-byte orbit table, for up to 8 coupling sets at
once (vectors interleaved [row][instance]).  The eigensolver replaces
``eigsh(H, k, which="SA")`` (edlgt/modeling/qmb_hamiltonian.py:313): a
thick-restart Lanczos (Wu and Simon, SIAM J. Matrix Anal. Appl. 22 (2000)
602) with delayed classical Gram-Schmidt reorthogonalisation against the
whole basis (two reads of the basis per step), the basis length chosen from
the free device memory, all inner products in f64.
``precision="mixed"`` runs the Krylov vectors and the matvec input/output in
f32, then refines the Ritz vectors with a short f64 thick-restart run started
from them; ``precision="fp64"`` is the plain f64 solver.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle

__all__ = ["ZnEngine", "ZnResult", "trlan_batched", "zn_lowest"]

_F64, _F32 = 0, 1


def _struct_of(L, luts):
    """ctypes edg_zn_lattice of a ZnLattice plus its device lookup tables."""
    s = _lib.ZnLattice()
    s.lx, s.ly, s.zn, s.link_bits = L.lx, L.ly, L.n, L.link_bits
    s.n_sites, s.n_links, s.field_bits, s.n_cot = L.n_sites, L.n_links, L.field_bits, L.n_cot
    s.n_gauss, s.pow_cot = L.n_gauss, L.pow_cot
    s.odd_mask = L.odd_mask
    s.even_mask = ((1 << L.n_sites) - 1) & ~L.odd_mask
    s.n_group = len(L.group)
    divs = L.divisors()
    if len(divs) > 8:
        raise ValueError("translation group has more than 8 stabiliser sizes")
    s.n_div = len(divs)
    for i, d in enumerate(divs):
        s.divisors[i] = d
    for gi, (a, b) in enumerate(L.group):
        m = L.translation_masks(a, b)
        t = s.group[gi]
        t.sf, t.sx, t.sm, t.smx = m["sf"], m["sx"], m["sm"], m["smx"]
        t.hif, t.lof, t.him, t.lom = m["hif"], m["lof"], m["him"], m["lom"]
        t.ylow, t.yhigh, t.xhead, t.xtail = m["ylow"], m["yhigh"], m["xhead"], m["xtail"]
    for c, l in enumerate(L.cotree):
        s.cot_link[c] = l
    for k, (v, pl, ps, others) in enumerate(L.peel):
        s.peel_site[k], s.peel_link[k], s.peel_sign[k] = v, pl, ps
        if len(others) != 3:
            raise ValueError("every site must have four incident links")
        for o, (l, sg) in enumerate(others):
            s.peel_other[k][o] = l
            s.peel_osign[k][o] = sg
    for l in range(L.n_links):
        ta, he = int(L.link_from[l]), int(L.link_to[l])
        s.link_tail[l], s.link_head[l] = ta, he
        s.link_eta[l] = L.link_eta(l)
        lo, hi = min(ta, he), max(ta, he)
        s.link_between[l] = sum(1 << k for k in range(lo + 1, hi))
    for p in range(L.n_sites):
        for i in range(4):
            s.plaq[p][i] = int(L.plaquettes[p][i])
    esq = L_esq(L.n)
    for i in range(4):
        s.esq[i] = esq[i] if i < L.n else 0.0
    s.chunk_lut, s.occ_rank, s.rank_occ = ptr(luts[0]), ptr(luts[1]), ptr(luts[2])
    return s


def L_esq(n):
    """E^2 on the symmetric representative E in (-n/2, n/2] of each Z_n value."""
    v = np.arange(n)
    sym = np.where(v > n // 2, v - n, v)
    return (sym**2).astype(float)


class ZnEngine:
    """Device state of one Z_n lattice: lookup tables, representative keys,
    orbit table; ``matvec`` applies H for interleaved instance vectors."""

    def __init__(self, lattice, device="cuda"):
        self.L = lattice
        self.device = torch.device(device)
        chunk, occ_rank, rank_occ = lattice.lookup_tables()
        self.luts = (
            torch.from_numpy(chunk.view(np.int64)).to(self.device),
            torch.from_numpy(occ_rank.view(np.int32)).to(self.device),
            torch.from_numpy(rank_occ.view(np.int32)).to(self.device),
        )
        self.struct = _struct_of(lattice, self.luts)
        self.keys = None
        self.orbit = None
        self.n_rows = None
        self.build_ms = {}

    def build_basis(self):
        """Representatives (ascending Gauss index) and the orbit table."""
        L, dev, st = self.L, self.device, stream_handle()
        sref = ctypes.byref(self.struct)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        words = lib.edg_zn_bitmap_words(sref)
        if words < 0:
            raise _lib.EdgError(-1, _lib.last_error())
        bitmap = torch.empty(words, dtype=torch.int64, device=dev)
        counts = torch.empty(words, dtype=torch.int64, device=dev)
        offsets = torch.empty(words, dtype=torch.int64, device=dev)
        scratch = torch.empty(max(1, lib.edg_scan_scratch_elems(words)), dtype=torch.int64, device=dev)
        ev[0].record()
        check(lib.edg_zn_mark(sref, ptr(bitmap), ptr(counts), st), "edg_zn_mark")
        check(lib.edg_scan_i64(ptr(counts), ptr(offsets), words, ptr(scratch), st), "edg_scan_i64")
        ev[1].record()
        n_rows = int(offsets[-1].item() + counts[-1].item())
        self.n_rows = n_rows
        self.keys = torch.empty(max(n_rows, 1), dtype=torch.int64, device=dev)
        check(lib.edg_zn_fill(sref, ptr(bitmap), ptr(offsets), ptr(self.keys), st), "edg_zn_fill")
        ev[2].record()
        del bitmap, counts, offsets, scratch
        self.orbit = torch.empty(L.n_gauss, dtype=torch.int32, device=dev)
        check(lib.edg_zn_orbit_table(sref, ptr(self.keys), n_rows, ptr(self.orbit), st), "edg_zn_orbit_table")
        ev[3].record()
        ev[3].synchronize()
        self.build_ms = {"mark": ev[0].elapsed_time(ev[1]), "fill": ev[1].elapsed_time(ev[2]),
                         "orbit": ev[2].elapsed_time(ev[3])}
        self.basis = _lib.ZnBasis(n_rows, ptr(self.keys), ptr(self.orbit))
        return n_rows

    def host_keys(self):
        return self.keys[: self.n_rows].cpu().numpy().view(np.uint64)

    def matvec(self, x, y, couplings, nvec):
        """y = H x (interleaved [row][nvec], f32 or f64); couplings: device
        f64 [nvec][4] = (t, m, g^2/2, -1/(2 g^2))."""
        dt = _F64 if x.dtype == torch.float64 else _F32
        check(lib.edg_zn_matvec(ctypes.byref(self.struct), ctypes.byref(self.basis), ptr(couplings), nvec, dt,
                                ptr(x), ptr(y), stream_handle()), "edg_zn_matvec")

    def time_matvec(self, nvec=8, dtype=torch.float32, reps=3, warmup=2, g=1.0, m=0.5):
        """Average device time (ms) of one batched matvec on random vectors,
        measured with CUDA events after warm-up launches."""
        cp = np.tile([1.0, m, g * g / 2, -1.0 / (2 * g * g)], (nvec, 1))
        coup = torch.from_numpy(cp).to(self.device)
        x = torch.rand((self.n_rows, nvec), dtype=dtype, device=self.device)
        y = torch.empty_like(x)
        for _ in range(warmup):
            self.matvec(x, y, coup, nvec)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            self.matvec(x, y, coup, nvec)
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / max(reps, 1)


# --------------------------------------------------------------- eigensolver
@dataclass
class ZnResult:
    evals: np.ndarray                 # [n_instances, k]
    residuals: np.ndarray             # [n_instances, k] relative residual estimates
    evecs: torch.Tensor | None = None  # interleaved [n_pad][nvec] ground states (f64)
    matvecs: int = 0
    cycles: int = 0
    stats: dict = field(default_factory=dict)


def _ivec(op, *args):
    check(getattr(lib, op)(*args), op)


def trlan_batched(apply, n_rows, nvec, dtype, m, k_keep, k_want, tol, max_cycles, v0=None, seed=1, stats=None):
    """Batched thick-restart Lanczos on interleaved vectors.

    Orthogonalisation is delayed classical Gram-Schmidt with
    reorthogonalisation (DCGS2: Swirydowicz, Langou, Ananthan, Yang, Thomas,
    Numer. Linear Algebra Appl. 28 (2021) e2343): step j takes the matvec of
    the candidate u_j that has had one Gram-Schmidt pass, and in one read of
    the basis (``edg_iv_dots2``) gets u_j's second-pass coefficients s and the
    projections z of w = H u_j; one more read (``edg_iv_dcgs_update``)
    finishes q_j = (u_j - Q s) / r and projects w against Q and q_j.  The
    projected matrix follows from the recorded dots without further passes:
    T[:j, j] = (z - T s) / r, T[j, j] = (omega - 2 z.s + s.T s) / r^2.

    apply(x, y): y = H x for all instances.  Returns (theta [nvec, k_want],
    residual estimates [nvec, k_want] relative to |theta|, Ritz vectors
    (tensor [k_want, n_elems]), matvec count, cycles, converged flags)."""
    dev = torch.device("cuda")
    tdt = torch.float64 if dtype == _F64 else torch.float32
    n_pad = (n_rows + 3) // 4 * 4
    E = n_pad * nvec
    m = int(min(m, max(2, n_rows - 1)))
    k_keep = int(min(k_keep, m - 1))
    k_want = int(min(k_want, k_keep))
    V = torch.zeros((m + 1, E), dtype=tdt, device=dev)
    w = torch.zeros(E, dtype=tdt, device=dev)
    rec = torch.zeros((m, 3, m + 1, nvec), dtype=torch.float64, device=dev)
    scratch = torch.empty(lib.edg_iv_scratch_elems(E, m + 1), dtype=torch.float64, device=dev)
    st = stream_handle()
    launches = 0
    if v0 is None:
        _ivec("edg_iv_random", dtype, n_rows, E, nvec, seed, ptr(V[0]), st)
        launches += 1
    else:
        V[0].copy_(v0)
    T = np.zeros((nvec, m, m))
    j0 = 0
    n_mv = 0
    mv_events = []
    converged = np.zeros(nvec, dtype=bool)
    theta = np.zeros((nvec, k_want))
    th_keep = np.zeros((nvec, k_keep))
    res = np.full((nvec, k_want), np.inf)
    S_all = np.zeros((nvec, m, m))
    cycles = 0
    for cycles in range(1, max_cycles + 1):
        for j in range(j0, m):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            apply(V[j], w)
            e1.record()
            mv_events.append((e0, e1, e2))
            n_mv += 1
            hu, hw, sq = rec[j, 0], rec[j, 1], rec[j, 2, 0]
            _ivec("edg_iv_dots2", dtype, E, nvec, ptr(V), E, j + 1, ptr(V[j]), ptr(w), ptr(hu), ptr(hw),
                  ptr(scratch), st)
            _ivec("edg_iv_dcgs_update", dtype, E, nvec, ptr(V), E, j, ptr(hu), ptr(hw), ptr(w), ptr(sq),
                  ptr(scratch), st)
            _ivec("edg_iv_scale", dtype, E, nvec, ptr(w), ptr(sq), ptr(V[j + 1]), st)
            e2.record()
            launches += 6  # matvec, dots2 + reduce, update + reduce, scale
        R = rec.cpu().numpy()
        beta = np.zeros((m, nvec))
        for j in range(j0, m):
            s_, alpha = R[j, 0, :j], R[j, 0, j]       # [j, nvec], [nvec]
            z, omega = R[j, 1, :j], R[j, 1, j]
            r = np.sqrt(np.maximum(alpha - np.einsum("iv,iv->v", s_, s_), 1e-300))
            Ts = np.einsum("vik,kv->iv", T[:, :j, :j], s_)  # [j, nvec]
            col = (z - Ts) / r
            T[:, :j, j] = col.T
            T[:, j, :j] = col.T
            T[:, j, j] = (omega - 2 * np.einsum("iv,iv->v", z, s_) + np.einsum("iv,iv->v", s_, Ts)) / r**2
            beta[j] = np.sqrt(np.maximum(R[j, 2, 0], 0.0)) / r
        for v in range(nvec):
            # an invariant subspace ends the recurrence early for this instance
            scale = max(np.abs(np.diag(T[v])).max(), 1e-300)
            tiny = np.nonzero(beta[j0:m, v] <= 1e-12 * scale)[0]
            me = j0 + int(tiny[0]) + 1 if len(tiny) else m
            th, S = np.linalg.eigh(T[v, :me, :me])
            S_all[v] = 0.0
            S_all[v, :me, :me] = S
            theta[v] = th[:k_want]
            th_keep[v, : min(k_keep, me)] = th[:k_keep]
            bv = 0.0 if me < m else beta[m - 1, v]
            res[v] = bv * np.abs(S[me - 1, :k_want]) / np.maximum(np.abs(th[:k_want]), 1e-300)
            converged[v] = bool(np.all(res[v] <= tol)) or me < m
        if converged.all() or cycles == max_cycles:
            break
        # thick restart: keep the k_keep lowest Ritz vectors, continue from the
        # candidate V[m] (its second Gram-Schmidt pass happens in the next step)
        Sk = torch.from_numpy(np.ascontiguousarray(S_all[:, :, :k_keep])).to(dev)
        _ivec("edg_iv_combine", dtype, E, nvec, ptr(V), E, m, ptr(Sk), k_keep, st)
        launches += 1
        V[k_keep].copy_(V[m])
        T[:] = 0.0
        for v in range(nvec):
            T[v, :k_keep, :k_keep] = np.diag(th_keep[v])
        rec.zero_()
        j0 = k_keep
    Sk = torch.from_numpy(np.ascontiguousarray(S_all[:, :, :k_want])).to(dev)
    _ivec("edg_iv_combine", dtype, E, nvec, ptr(V), E, m, ptr(Sk), k_want, st)
    launches += 1
    torch.cuda.synchronize()
    mv_ms = sum(a.elapsed_time(b) for a, b, _ in mv_events)
    ro_ms = sum(b.elapsed_time(c) for _, b, c in mv_events)
    if stats is not None:
        stats["matvec_ms"] = stats.get("matvec_ms", 0.0) + mv_ms
        stats["reorth_ms"] = stats.get("reorth_ms", 0.0) + ro_ms
        stats["matvecs"] = stats.get("matvecs", 0) + n_mv
        stats["launches"] = stats.get("launches", 0) + launches
    out = V[:k_want].clone()
    return theta, res, out, n_mv, cycles, converged


def _auto_m(vec_bytes, cap, reserve_vectors=3):
    """Basis length that fits the free device memory (w, a copy and a margin
    besides the basis), at most cap."""
    torch.cuda.empty_cache()  # blocks cached by torch count as free here
    free, _ = torch.cuda.mem_get_info()
    fit = int((free - (1 << 30)) // max(vec_bytes, 1)) - reserve_vectors
    return max(4, min(cap, fit))


def zn_lowest(engine, couplings, k=1, precision="mixed", m=None, k_keep=None, tol32=2e-6, tol64=1e-8,
              max_cycles=400, refine_m=6, refine_cycles=30, seed=1):
    """Lowest k eigenvalues of H(t, m, g) for up to 8 coupling sets at once.

    couplings: array [n_inst, 4] of (t, m, g^2/2, -1/(2 g^2)).
    Returns a ZnResult with the f64 ground-state vectors (interleaved)."""
    cp = np.atleast_2d(np.asarray(couplings, dtype=np.float64))
    n_inst = len(cp)
    if n_inst > 8:
        raise ValueError("at most 8 coupling sets per batch")
    nvec = next(v for v in (1, 2, 4, 8) if v >= n_inst)
    cpad = np.concatenate([cp, np.repeat(cp[-1:], nvec - n_inst, axis=0)])
    dev = engine.device
    coup = torch.from_numpy(np.ascontiguousarray(cpad)).to(dev)
    n = engine.n_rows
    n_pad = (n + 3) // 4 * 4
    E = n_pad * nvec

    def apply(x, y):
        engine.matvec(x, y, coup, nvec)

    stats = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    if precision == "fp64":
        m64 = m or _auto_m(E * 8, 24)
        kk = k_keep or max(k + 1, m64 // 2)
        th, res, X, nmv, cyc, conv = trlan_batched(apply, n, nvec, _F64, m64, kk, k, tol64, max_cycles, seed=seed,
                                                   stats=stats)
        ev[1].record()
        ev[2].record()
        stats.update(m=m64, k_keep=kk, matvecs64=nmv, cycles64=cyc)
        cycles = cyc
    elif precision == "mixed":
        m32 = m or _auto_m(E * 4, 24)
        kk = k_keep or max(k + 1, m32 // 2)
        s32 = {}
        th32, res32, X32, nmv32, cyc32, conv32 = trlan_batched(apply, n, nvec, _F32, m32, kk, k, tol32, max_cycles,
                                                               seed=seed, stats=s32)
        ev[1].record()
        # start the f64 refinement from the sum of the wanted Ritz vectors
        x32 = X32.sum(dim=0) if k > 1 else X32[0]
        v0 = torch.empty(E, dtype=torch.float64, device=dev)
        check(lib.edg_convert(1, ptr(x32), 0, ptr(v0), E, stream_handle()), "edg_convert")
        del X32, x32
        s64 = {}
        rm = max(refine_m, k + 2)
        th, res, X, nmv64, cyc64, conv = trlan_batched(apply, n, nvec, _F64, rm, max(k + 1, rm // 2), k, tol64,
                                                       refine_cycles, v0=v0, stats=s64)
        ev[2].record()
        stats.update(m=m32, k_keep=kk, matvecs32=nmv32, cycles32=cyc32, matvec32_ms=s32.get("matvec_ms", 0.0),
                     matvecs64=nmv64, cycles64=cyc64, matvec64_ms=s64.get("matvec_ms", 0.0),
                     theta32=th32[:n_inst].copy(), res32=res32[:n_inst].copy())
        stats["matvec_ms"] = s32.get("matvec_ms", 0.0) + s64.get("matvec_ms", 0.0)
        stats["reorth_ms"] = s32.get("reorth_ms", 0.0) + s64.get("reorth_ms", 0.0)
        stats["reorth32_ms"] = s32.get("reorth_ms", 0.0)
        stats["matvecs"] = nmv32 + nmv64
        stats["launches"] = s32.get("launches", 0) + s64.get("launches", 0) + 1  # + convert
        cycles = cyc32 + cyc64
    else:
        raise ValueError("precision must be 'mixed' or 'fp64'")
    torch.cuda.synchronize()
    stats["phase1_ms"] = ev[0].elapsed_time(ev[1])
    stats["phase2_ms"] = ev[1].elapsed_time(ev[2])
    stats["total_ms"] = ev[0].elapsed_time(ev[2])
    stats["converged"] = conv[:n_inst].copy()
    return ZnResult(evals=th[:n_inst], residuals=res[:n_inst], evecs=X[0], matvecs=stats.get("matvecs", 0),
                    cycles=cycles, stats=stats)
