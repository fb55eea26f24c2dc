"""The allocation-free tridiagonal eigensolver entry point.

edg_tridiag_lowest_noalloc serves callers that cannot allocate device
memory (no cudaMalloc available or allowed where they run): its scratch is a
static device array inside the library.  Its results must equal those of the
allocating entry point, call after call, since every call reuses the same
array.  This file is collected last on purpose.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(fn_name, a, b, k, dev, with_work):
    import torch

    from edgpu import _lib

    m = len(a)
    A = torch.from_numpy(a).to(dev)
    B = torch.from_numpy(b).to(dev)
    ev = torch.empty(k, dtype=torch.float64, device=dev)
    S = torch.empty((k, m), dtype=torch.float64, device=dev)
    args = [_lib.ptr(A), _lib.ptr(B), m, k, _lib.ptr(ev), _lib.ptr(S)]
    if with_work:
        work = torch.empty(6 * m, dtype=torch.float64, device=dev)
        args.append(_lib.ptr(work))
    _lib.check(getattr(_lib.lib, fn_name)(*args, _lib.stream_handle()), fn_name)
    torch.cuda.synchronize()
    return ev.cpu().numpy(), S.cpu().numpy()


def test_noalloc_matches_allocating_entry_on_consecutive_calls():
    import torch

    assert torch.cuda.is_available()
    dev = "cuda"
    rng = np.random.default_rng(2024)
    # calls in a row with different sizes; the last one is the largest size
    # the static array holds (m = 4096), after smaller calls left their
    # contents in it
    for call, (m, k) in enumerate([(300, 4), (97, 3), (4096, 2)]):
        a = rng.standard_normal(m)
        b = np.concatenate([[0.0], rng.uniform(0.05, 1.0, m - 1)])
        e_ref, s_ref = _solve("edg_tridiag_lowest", a, b, k, dev, with_work=True)
        e_new, s_new = _solve("edg_tridiag_lowest_noalloc", a, b, k, dev, with_work=False)
        assert np.allclose(e_new, e_ref, rtol=0, atol=1e-12), call
        for q in range(k):
            assert abs(abs(float(s_new[q] @ s_ref[q])) - 1.0) < 1e-10, (call, q)
        from scipy.linalg import eigvalsh_tridiagonal

        w = eigvalsh_tridiagonal(a, b[1:])
        assert np.allclose(e_new, w[:k], rtol=0, atol=1e-12), call


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    from edgpu import _lib

    m = 4097
    st = _lib.lib.edg_tridiag_lowest_noalloc(None, None, m, 1, None, None, None)
    assert st == -1
    assert "static scratch limit" in _lib.last_error()
