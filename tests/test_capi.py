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
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(edg_sector_tables), sizeof(edg_lookup_table),
         sizeof(edg_assembly), sizeof(edg_lanczos_problem), sizeof(edg_site_dims), sizeof(edg_krylov_problem),
         sizeof(edg_small_batch), sizeof(edg_zn_translation), sizeof(edg_zn_lattice), sizeof(edg_zn_basis),
         sizeof(edg_part_spec), sizeof(edg_momentum_group));
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
                     ctypes.sizeof(_lib.PartSpec), ctypes.sizeof(_lib.MomentumGroup)]
