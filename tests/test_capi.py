"""The C-ABI library loads and exports every entry point of include/edgpu.h
(no device work: argument validation and size queries run on the host)."""

import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, "include", "edgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(edg_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    from edgpu import _lib

    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(_lib.lib, n), f"{n} missing from libedgpu.so"
        assert n in _lib.EXPORTED_SYMBOLS, f"{n} has no ctypes signature"


def test_version_and_error_buffer():
    from edgpu import _lib

    assert _lib.lib.edg_version() == 100
    st = _lib.lib.edg_scan_i64(None, None, -1, None, None)
    assert st == -1
    assert "negative" in _lib.last_error()


def test_size_queries():
    from edgpu import _lib

    assert _lib.lib.edg_sector_level_blocks(1) == 1
    assert _lib.lib.edg_sector_level_blocks(2048) == 1
    assert _lib.lib.edg_sector_level_blocks(2049) == 2
    assert _lib.lib.edg_scan_scratch_elems(4096) == 2
    p = _lib.LanczosProblem()
    p.dtype, p.n_rows, p.nnz, p.nvec, p.k, p.max_iter, p.tol, p.check_every = 1, 1000, 0, 3, 1, 50, 1e-8, 5
    p.rowptr = p.diag = 1  # any non-null value: only the layout is computed
    wb = _lib.lib.edg_lanczos_workspace_bytes(ctypes.byref(p))
    assert wb >= 51 * 1000 * 3 * 4
    p.k = 99
    assert _lib.lib.edg_lanczos_workspace_bytes(ctypes.byref(p)) == -1


def test_struct_layouts_match_header():
    """ctypes struct sizes agree with the C compiler's view of the header."""
    import subprocess
    import tempfile

    from edgpu import _lib

    src = r'''
#include <stdio.h>
#include "edgpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(edg_sector_tables), sizeof(edg_lookup_table),
         sizeof(edg_assembly), sizeof(edg_lanczos_problem), sizeof(edg_site_dims), sizeof(edg_krylov_problem),
         sizeof(edg_small_batch), sizeof(edg_zn_translation), sizeof(edg_zn_lattice), sizeof(edg_zn_basis),
         sizeof(edg_part_spec), sizeof(edg_momentum_group), sizeof(edg_tiled_batch));
  return 0;
}
'''
    cuda_inc = "/usr/local/cuda/include"
    if not os.path.isdir(cuda_inc):
        pytest.skip("CUDA headers not available")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", c, "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, "-o", exe], check=True)
        sizes = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert sizes == [ctypes.sizeof(_lib.SectorTables), ctypes.sizeof(_lib.LookupTable), ctypes.sizeof(_lib.Assembly),
                     ctypes.sizeof(_lib.LanczosProblem), ctypes.sizeof(_lib.SiteDims),
                     ctypes.sizeof(_lib.KrylovProblem), ctypes.sizeof(_lib.SmallBatch),
                     ctypes.sizeof(_lib.ZnTranslation), ctypes.sizeof(_lib.ZnLattice), ctypes.sizeof(_lib.ZnBasis),
                     ctypes.sizeof(_lib.PartSpec), ctypes.sizeof(_lib.MomentumGroup),
                     ctypes.sizeof(_lib.TiledBatch)]


def test_tuning_context_roundtrip():
    """edg_ctx: an explicit, caller-owned store of tuning choices."""
    from edgpu.context import Context

    a, b = Context(), Context()
    assert len(a) == 0 and a.get(7, 2) is None
    a.put(7, (512, 8))
    a.put(2**64 - 1, (3,))
    assert a.get(7, 2) == (512, 8)
    assert a.get(7, 1) == (512,)
    assert a.get(2**64 - 1, 4) == (3,)
    assert len(a) == 2 and len(b) == 0  # no shared state between contexts
    from edgpu import _lib

    assert _lib.lib.edg_ctx_put(a.handle, 1, None, 0) == -1
    assert _lib.lib.edg_ctx_size(None) == -1


def test_tiled_batch_plan():
    """Host-side plan of the (instance, row-tile) batched solver: tiles,
    items, Krylov caps, check schedule and workspace size."""
    import numpy as np

    from edgpu import _lib

    dims = np.array([26, 90, 5, 1000, 4096], dtype=np.int64)
    n_items, wb = ctypes.c_int32(0), ctypes.c_int64(0)
    inst = np.zeros((5, 8), dtype=np.int64)
    items = np.zeros(64, dtype=np.int32)
    chk = np.zeros(120, dtype=np.uint8)
    st = _lib.lib.edg_tiled_batch_plan(5, dims.ctypes.data, 1, 120, 1, 256, 8, inst.ctypes.data, items.ctypes.data,
                                       chk.ctypes.data, ctypes.byref(n_items), ctypes.byref(wb))
    assert st == 0
    pad = (dims + 3) // 4 * 4
    tiles = (pad + 255) // 256
    assert np.array_equal(inst[:, 0], dims)                                   # dim
    assert np.array_equal(inst[:, 1], np.concatenate([[0], np.cumsum(dims)[:-1]]))          # row offset
    assert np.array_equal(inst[:, 2], np.concatenate([[0], np.cumsum(dims + 1)[:-1]]))      # rowptr offset
    assert np.array_equal(inst[:, 5], tiles)
    assert np.array_equal(inst[:, 6], np.concatenate([[0], np.cumsum(tiles)[:-1]]))
    assert np.array_equal(inst[:, 7], np.minimum(dims, 120))                  # Krylov cap
    assert n_items.value == tiles.sum()
    assert np.array_equal(items[: n_items.value], np.repeat(np.arange(5), tiles))
    # arenas are 256-byte aligned and disjoint; the V arena of the last
    # instance ends inside the workspace
    assert np.all(inst[:, 3] % 256 == 0) and np.all(inst[:, 4] % 256 == 0)
    assert inst[-1, 3] + (inst[-1, 7] + 1) * pad[-1] * 4 <= wb.value
    # checks every 8 steps, at the last step and at every instance's cap
    want = {j for j in range(120) if (j + 1) % 8 == 0} | {119} | {int(c) - 1 for c in inst[:, 7]}
    assert set(np.nonzero(chk)[0].tolist()) == want
    # invalid arguments
    assert _lib.lib.edg_tiled_batch_plan(5, dims.ctypes.data, 1, 120, 1, 250, 8, None, None, None,
                                         ctypes.byref(n_items), ctypes.byref(wb)) == -1
    assert _lib.lib.edg_tiled_batch_plan(5, dims.ctypes.data, 1, 120, 9, 256, 8, None, None, None,
                                         ctypes.byref(n_items), ctypes.byref(wb)) == -1


def test_packed_layout_argument_checks():
    """The dictionary-packed layout's entry points refuse bad shapes on the
    host, before any device work (status EDG_ERR_ARG and a message)."""
    from edgpu import _lib

    L = _lib.lib
    assert L.edg_pack_tiles(0) == 0 and L.edg_pack_tiles(16) == 1 and L.edg_pack_tiles(17) == 2
    assert L.edg_pack_tiles(-1) == -1
    assert L.edg_pack_tile_counts(-1, None, None, None) == -1
    assert "negative" in _lib.last_error()
    # the value set: dtype, slot count, null pointers
    assert L.edg_pack_collect(2, None, 10, 1, 10, 1, None) == -1
    assert L.edg_pack_collect(1, None, 10, 1, 30, 1, None) == -1 and "log2_slots" in _lib.last_error()
    assert L.edg_pack_collect(1, None, 10, None, 10, None, None) == -1
    # encode: the column bits must leave room for the all-ones padding column
    assert L.edg_pack_encode(0, 16, 100, 1, 1, 1, 1, 4, 4, 1, 1, 1, 1, None) == -1
    assert "padding column" in _lib.last_error()
    # encode: more values than the index bits hold (5 column bits leave 27)
    # or than the table limit
    assert L.edg_pack_encode(0, 16, 100, 1, 1, 1, 1, _lib.PACK_MAX_VALUES + 1, 5, 1, 1, 1, 1, None) == -1
    assert L.edg_pack_encode(0, 16, 100, 1, 1, 1, 1, 9, 30, 1, 1, 1, 1, None) == -1
    assert "index bits" in _lib.last_error()
    assert L.edg_pack_encode(0, 16, 2**31, 1, 1, 1, 1, 4, 5, 1, 1, 1, 1, None) == -1
    # matvec: dtype, nvec, x stride, colbits, table size, null pointers
    args = dict(tile_off=1, words=1, table=1, count=4, colbits=5, diag=1, x=1, xs=3, y=1)

    def mv(dtype=1, n=16, nvec=3, **kw):
        a = {**args, **kw}
        return L.edg_spmv_packed(dtype, n, nvec, a["tile_off"], a["words"], a["table"], a["count"], a["colbits"],
                                 a["diag"], a["x"], a["xs"], a["y"], 0, None, None)

    assert mv(dtype=2) == -1
    assert mv(nvec=5) == -1
    assert mv(xs=5) == -1 and "x_stride" in _lib.last_error()
    assert mv(n=32) == -1 and "colbits" in _lib.last_error()
    assert mv(count=0) == -1
    assert mv(words=None) == -1 and "null" in _lib.last_error()
    assert mv(n=0) == 0  # an empty matrix is a no-op


def test_lanczos_problem_rejects_an_incomplete_packed_layout():
    """edg_lanczos_problem: a packed layout without its tile offsets or with
    column bits that leave no padding column is refused."""
    from edgpu import _lib

    p = _lib.LanczosProblem()
    p.dtype, p.n_rows, p.nnz, p.nvec, p.k, p.max_iter, p.tol, p.check_every = 1, 1000, 0, 3, 1, 50, 1e-8, 5
    p.rowptr = p.diag = 1
    assert _lib.lib.edg_lanczos_workspace_bytes(ctypes.byref(p)) > 0
    p.pk_words, p.pk_table, p.pk_count, p.pk_colbits = 1, 1, 4, 11
    assert _lib.lib.edg_lanczos_workspace_bytes(ctypes.byref(p)) == -1  # no tile offsets
    p.pk_tile_off = 1
    assert _lib.lib.edg_lanczos_workspace_bytes(ctypes.byref(p)) > 0
    p.pk_colbits = 9  # 2^9 rows: fewer than the 1000 rows
    assert _lib.lib.edg_lanczos_workspace_bytes(ctypes.byref(p)) == -1
