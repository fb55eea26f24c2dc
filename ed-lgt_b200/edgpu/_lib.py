"""ctypes binding of libedgpu (the C ABI declared in include/edgpu.h).

The library is the only compute path: loading fails loudly when the shared
object is missing, and every call's status is turned into an exception.
Device buffers are torch CUDA tensors passed by ``data_ptr()``.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

from ._build import LIB_PATH

__all__ = ["lib", "check", "EdgError", "MAX_SITES", "MAX_OPS", "SectorTables", "LookupTable", "Assembly",
           "LanczosProblem", "SiteDims", "KrylovProblem", "SmallBatch", "ZnTranslation", "ZnLattice", "ZnBasis",
           "ZN_MAX_SITES", "ZN_MAX_GROUP", "EXPORTED_SYMBOLS", "ptr", "stream_handle"]

MAX_SITES = 64
MAX_OPS = 4
PACK_MAX_VALUES = 4096  # EDG_PACK_MAX_VALUES
ZN_MAX_SITES = 14
ZN_MAX_GROUP = 32

EDG_OK = 0
STATUS_NAMES = {
    -1: "EDG_ERR_ARG",
    -2: "EDG_ERR_CUDA",
    -3: "EDG_ERR_OVERFLOW",
    -4: "EDG_ERR_MISSING_KET",
    -5: "EDG_ERR_NOT_CONVERGED",
    -6: "EDG_ERR_BREAKDOWN",
    -7: "EDG_ERR_TIMEOUT",
}


class EdgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
U64 = C.c_uint64
U32 = C.c_uint32
F64 = C.c_double


class SectorTables(C.Structure):
    _fields_ = [
        ("n_sites", I32),
        ("dmax", I32),
        ("loc_dims", I32 * MAX_SITES),
        ("strides", U64 * MAX_SITES),
        ("site_allowed", P),
        ("n_glob", I32),
        ("glob_type", I32),
        ("glob_val", P),
        ("glob_target", P),
        ("glob_rem_min", P),
        ("glob_rem_max", P),
        ("n_dirs", I32),
        ("link_val", P),
        ("link_target", P),
        ("pair_start", P),
        ("pair_s0", P),
        ("pair_s1", P),
        ("pair_dir", P),
        ("nbody_type", I32),
        ("nb_val", P),
        ("nb_target", P),
        ("nb_start", P),
        ("nb_id", P),
        ("nb_site_start", P),
        ("nb_sites", P),
        ("key_words", I32),
        ("n_hi", I32),
    ]


class LookupTable(C.Structure):
    _fields_ = [
        ("keys", P),
        ("n", I64),
        ("bucket_start", P),
        ("shift", I32),
        ("n_buckets", I64),
        ("key_words", I32),
        ("n_hi", I32),
        ("lo_space", U64),
    ]


class Assembly(C.Structure):
    _fields_ = [
        ("n_sites", I32),
        ("dmax", I32),
        ("loc_dims", I32 * MAX_SITES),
        ("strides", U64 * MAX_SITES),
        ("sector", LookupTable),
        ("complex_values", I32),
        ("t_count", P),
        ("t_ket", P),
        ("t_amp", P),
        ("n_terms", I32),
        ("term_nops", P),
        ("term_site", P),
        ("term_table", P),
        ("term_coef", P),
        ("n_dterms", I32),
        ("dterm_site", P),
        ("dterm_diag", P),
        ("dterm_coef", P),
    ]


class SiteDims(C.Structure):
    _fields_ = [("d", I32 * MAX_SITES)]


class LanczosProblem(C.Structure):
    _fields_ = [
        ("dtype", I32),
        ("n_rows", I64),
        ("nnz", I64),
        ("rowptr", P),
        ("cols", P),
        ("vals", P),
        ("diag", P),
        ("nvec", I32),
        ("k", I32),
        ("max_iter", I32),
        ("tol", F64),
        ("check_every", I32),
        ("seed", U64),
        ("v0", P),
        ("spmv_group", I32),
        ("stats", P),
        ("host_progress", P),
        ("sell_perm", P),
        ("sell_width", P),
        ("sell_off", P),
        ("sell_entries", P),
        ("reorth_window", I32),
        ("pk_tile_off", P),
        ("pk_words", P),
        ("pk_table", P),
        ("pk_count", I32),
        ("pk_colbits", I32),
    ]


class KrylovProblem(C.Structure):
    _fields_ = [
        ("vec_dtype", I32),
        ("mat_dtype", I32),
        ("n_rows", I64),
        ("nnz", I64),
        ("rowptr", P),
        ("cols", P),
        ("vals", P),
        ("diag", P),
        ("m", I32),
        ("reorth_passes", I32),
        ("spmv_group", I32),
        ("pk_tile_off", P),
        ("pk_words", P),
        ("pk_table", P),
        ("pk_count", I32),
        ("pk_colbits", I32),
        ("status", P),
    ]


class SmallBatch(C.Structure):
    _fields_ = [
        ("n_inst", I32),
        ("max_dim", I32),
        ("dims", P),
        ("row_off", P),
        ("rowptr_off", P),
        ("rowptr", P),
        ("cols", P),
        ("vals", P),
        ("diag", P),
        ("work", P),
        ("work_off", P),
        ("k", I32),
        ("max_iter", I32),
        ("check_every", I32),
        ("tol", F64),
        ("seed", U64),
        ("evals", P),
        ("evecs", P),
        ("iters", P),
    ]


class TiledBatch(C.Structure):
    _fields_ = [
        ("dtype", I32),
        ("n_inst", I32),
        ("n_items", I32),
        ("tile_rows", I32),
        ("lanes", I32),
        ("k", I32),
        ("max_iter", I32),
        ("reserved", I32),
        ("tol", F64),
        ("seed", U64),
        ("inst", P),
        ("item_inst", P),
        ("check_at", P),
        ("rowptr", P),
        ("cols", P),
        ("vals", P),
        ("diag", P),
        ("v0", P),
        ("workspace", P),
        ("evals", P),
        ("resid", P),
        ("iters", P),
        ("evecs", P),
        ("status", P),
    ]


class ZnTranslation(C.Structure):
    _fields_ = [
        ("sf", I32), ("sx", I32), ("sm", I32), ("smx", I32),
        ("hif", U64), ("lof", U64),
        ("him", U32), ("lom", U32),
        ("ylow", U32), ("yhigh", U32),
        ("xhead", U32), ("xtail", U32),
    ]


class ZnLattice(C.Structure):
    _fields_ = [
        ("lx", I32), ("ly", I32), ("zn", I32), ("link_bits", I32),
        ("n_sites", I32), ("n_links", I32), ("field_bits", I32), ("n_cot", I32),
        ("n_gauss", I64), ("pow_cot", I64),
        ("odd_mask", U32), ("even_mask", U32),
        ("n_group", I32), ("n_div", I32),
        ("divisors", I32 * 8),
        ("group", ZnTranslation * ZN_MAX_GROUP),
        ("cot_link", I32 * (2 * ZN_MAX_SITES)),
        ("peel_site", I32 * ZN_MAX_SITES), ("peel_link", I32 * ZN_MAX_SITES), ("peel_sign", I32 * ZN_MAX_SITES),
        ("peel_other", (I32 * 3) * ZN_MAX_SITES), ("peel_osign", (I32 * 3) * ZN_MAX_SITES),
        ("link_tail", I32 * (2 * ZN_MAX_SITES)), ("link_head", I32 * (2 * ZN_MAX_SITES)),
        ("link_eta", I32 * (2 * ZN_MAX_SITES)),
        ("link_between", U32 * (2 * ZN_MAX_SITES)),
        ("plaq", (I32 * 4) * ZN_MAX_SITES),
        ("esq", F64 * 4),
        ("chunk_lut", P), ("occ_rank", P), ("rank_occ", P),
    ]


class ZnBasis(C.Structure):
    _fields_ = [("n_rows", I64), ("keys", P), ("orbit", P)]


class MomentumGroup(C.Structure):
    _fields_ = [
        ("lattice_dim", I32),
        ("n_shifts", I32),
        ("shifts_per_dir", I32 * 4),
        ("shift_strides", I32 * 4),
        ("k_vals", I32 * 4),
    ]


class PartSpec(C.Structure):
    _fields_ = [
        ("n_part", I32),
        ("reserved", I32),
        ("key_space", U64),
        ("src_stride", U64 * MAX_SITES),
        ("dim", U64 * MAX_SITES),
        ("part_stride", U64 * MAX_SITES),
    ]


_SIGS = {
    "edg_get_last_error": (I32, [C.c_char_p, I32]),
    "edg_version": (I32, []),
    "edg_scan_scratch_elems": (I64, [I64]),
    "edg_scan_i64": (I32, [P, P, I64, P, P]),
    "edg_sector_level_blocks": (I64, [I64]),
    "edg_sector_level_count": (I32, [C.POINTER(SectorTables), I32, P, P, I64, P, P, P]),
    "edg_sector_level_fill": (I32, [C.POINTER(SectorTables), I32, P, P, I64, P, P, P, P]),
    "edg_keys_to_configs": (I32, [P, I64, I32, P, P, P]),
    "edg_configs_to_keys": (I32, [P, I64, I32, P, P, P]),
    "edg_lookup_build": (I32, [P, I64, I32, I64, P, P]),
    "edg_lookup_build_wide": (I32, [P, I64, I32, U64, I32, I64, P, P]),
    "edg_keys_to_configs_wide": (I32, [P, I64, I32, I32, P, P, P]),
    "edg_configs_to_keys_wide": (I32, [P, I64, I32, I32, P, P, P]),
    "edg_lookup": (I32, [C.POINTER(LookupTable), P, I64, P, P]),
    "edg_assemble_count": (I32, [C.POINTER(Assembly), P, P]),
    "edg_assemble_fill": (I32, [C.POINTER(Assembly), P, P, P, P, P, P, P, P]),
    "edg_assemble_compact": (I32, [I64, I32, P, P, P, P, P, P, P]),
    "edg_spmv": (I32, [I32, I64, I64, P, P, P, P, I32, P, P, P]),
    "edg_convert": (I32, [I32, P, I32, P, I64, P]),
    "edg_sell_slices": (I64, [I64]),
    "edg_sell_order": (I32, [P, I64, I32, P, P, P, P]),
    "edg_sell_fill": (I32, [I32, P, P, P, I64, P, P, P, P, P]),
    "edg_spmv_sell": (I32, [I64, I32, P, P, P, P, P, P, I32, P, I64, P]),
    "edg_spmv_f32_planar": (I32, [I64, I64, P, P, P, P, I32, P, I32, P, I64, I32, P]),
    "edg_pack_collect": (I32, [I32, P, I64, P, I32, P, P]),
    "edg_pack_tiles": (I64, [I64]),
    "edg_pack_tile_counts": (I32, [I64, P, P, P]),
    "edg_pack_encode": (I32, [I32, I64, I64, P, P, P, P, I32, I32, P, P, P, P, P]),
    "edg_spmv_packed": (I32, [I32, I64, I32, P, P, P, I32, I32, P, P, I32, P, I64, P, P]),
    "edg_spmv_group": (I32, [I32, I64, I64, P, P, P, P, I32, P, P, I32, P]),
    "edg_lanczos_workspace_bytes": (I64, [C.POINTER(LanczosProblem)]),
    "edg_lanczos": (I32, [C.POINTER(LanczosProblem), P, I64, P, P, P, P, P]),
    "edg_tridiag_lowest": (I32, [P, P, I32, I32, P, P, P, P]),
    "edg_tridiag_lowest_noalloc": (I32, [P, P, I32, I32, P, P, P]),
    "edg_local_expval": (I32, [P, I64, C.POINTER(SiteDims), I32, P, I32, I64, P, I32, P, P]),
    "edg_local_expval_wide": (I32, [P, I64, I32, C.POINTER(SiteDims), I32, P, I32, I64, P, I32, P, P]),
    "edg_small_batch_work_elems": (I64, [I64, I32, I32]),
    "edg_lanczos_small_batched": (I32, [C.POINTER(SmallBatch), P, P]),
    "edg_ctx_create": (P, []),
    "edg_ctx_destroy": (None, [P]),
    "edg_ctx_put": (I32, [P, U64, P, I32]),
    "edg_ctx_get": (I32, [P, U64, P, I32]),
    "edg_ctx_size": (I64, [P]),
    "edg_tiled_batch_plan": (I32, [I32, P, I32, I32, I32, I32, I32, P, P, P, P, P]),
    "edg_tiled_batch_header_bytes": (I32, [I32]),
    "edg_lanczos_tiled_batch": (I32, [C.POINTER(TiledBatch), P]),
    "edg_krylov_workspace_bytes": (I64, [C.POINTER(KrylovProblem)]),
    "edg_krylov_step": (I32, [C.POINTER(KrylovProblem), P, F64, P, I64, P, P]),
    "edg_twobody_scratch_elems": (I64, [I32]),
    "edg_twobody_expval": (I32, [C.POINTER(LookupTable), P, P, I32, P, P, P, I32, P, P, I32, P, I32, I64, P, P, I64, P]),
    "edg_csr_to_dense": (I32, [I32, I64, P, P, P, P, P, P, P]),
    "edg_momentum_translations": (I32, [C.POINTER(LookupTable), P, P, I32, P, I32, P, I32, P, P, P, P, P]),
    "edg_momentum_scratch_elems": (I64, [I64]),
    "edg_momentum_references": (I32, [P, I64, C.POINTER(MomentumGroup), P, P, C.POINTER(I64), P, I64, P]),
    "edg_momentum_columns": (I32, [P, P, I64, P, C.POINTER(MomentumGroup), P, I32, I32, P, P, C.POINTER(I64), P, P,
                                   P, I64, P]),
    "edg_momentum_rowmap": (I32, [P, P, P, I64, I64, P, P, P, P]),
    "edg_momentum_expand": (I32, [I64, P, P, P, P, P]),
    "edg_momentum_reduce": (I32, [I64, P, P, P, P, P, P]),
    "edg_part_scratch_elems": (I64, [U64]),
    "edg_part_map": (I32, [P, I64, C.POINTER(PartSpec), P, P, I64, C.POINTER(I64), P, I64, P]),
    "edg_psi_matrix": (I32, [P, I32, I64, P, P, I64, I64, P, I32, P, P]),
    "edg_zn_bitmap_words": (I64, [C.POINTER(ZnLattice)]),
    "edg_zn_mark": (I32, [C.POINTER(ZnLattice), P, P, P]),
    "edg_zn_fill": (I32, [C.POINTER(ZnLattice), P, P, P, P]),
    "edg_zn_orbit_table": (I32, [C.POINTER(ZnLattice), P, I64, P, P]),
    "edg_zn_matvec": (I32, [C.POINTER(ZnLattice), C.POINTER(ZnBasis), P, I32, I32, P, P, P]),
    "edg_iv_scratch_elems": (I64, [I64, I32]),
    "edg_iv_dots": (I32, [I32, I64, I32, P, I64, I32, P, P, P, P]),
    "edg_iv_update": (I32, [I32, I64, I32, P, I64, I32, P, P, P]),
    "edg_iv_scale": (I32, [I32, I64, I32, P, P, P, P]),
    "edg_iv_update_norm": (I32, [I32, I64, I32, P, I64, I32, P, P, P, P, P]),
    "edg_iv_dots2": (I32, [I32, I64, I32, P, I64, I32, P, P, P, P, P, P]),
    "edg_iv_dcgs_update": (I32, [I32, I64, I32, P, I64, I32, P, P, P, P, P, P]),
    "edg_iv_combine": (I32, [I32, I64, I32, P, I64, I32, P, I32, P]),
    "edg_iv_random": (I32, [I32, I64, I64, I32, U64, P, P]),
}

EXPORTED_SYMBOLS = tuple(_SIGS)


def _load():
    path = Path(LIB_PATH)
    if not path.exists():
        raise ImportError(
            f"libedgpu.so not found at {path}; build it with `python ed-lgt_b200/edgpu/_build.py` "
            "(there is no CPU fallback for the engine)"
        )
    handle = C.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    return handle


lib = _load()


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib.edg_get_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(status: int, what: str = ""):
    if status != EDG_OK:
        raise EdgError(status, f"{what}: {last_error()}" if what else last_error())
    return status


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(stream=None) -> int | None:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
