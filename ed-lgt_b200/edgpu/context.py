"""Tuning context: an explicit handle (``edg_ctx``) that holds autotuner
choices, keyed by a hash of the problem shape.

The library keeps no global tuning state; callers pass a :class:`Context`
to the tuned entry points (``ctx=``).  Without one, the package uses one
default context per device, created on first use and owned by this module.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import EdgError, check, last_error, lib

__all__ = ["Context", "default_context"]


class Context:
    """Owner of one ``edg_ctx`` handle (destroyed with the object)."""

    def __init__(self):
        h = lib.edg_ctx_create()
        if not h:
            raise EdgError(-2, "edg_ctx_create: out of host memory")
        self._h = h

    @property
    def handle(self):
        return self._h

    def put(self, key: int, params):
        a = np.ascontiguousarray(params, dtype=np.int32)
        check(lib.edg_ctx_put(self._h, int(key) & 0xFFFFFFFFFFFFFFFF, a.ctypes.data, len(a)), "edg_ctx_put")

    def get(self, key: int, n: int):
        """The stored values (tuple of n ints) or None when absent."""
        a = np.zeros(n, dtype=np.int32)
        got = lib.edg_ctx_get(self._h, int(key) & 0xFFFFFFFFFFFFFFFF, a.ctypes.data, n)
        if got < 0:
            raise EdgError(got, last_error())
        return tuple(int(x) for x in a[:got]) if got > 0 else None

    def __len__(self):
        return int(lib.edg_ctx_size(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.edg_ctx_destroy(ctypes.c_void_p(h))
            self._h = None


_DEFAULT = {}


def default_context(device=None) -> Context:
    """The package's context for a device (index or torch.device)."""
    idx = getattr(device, "index", device)
    idx = 0 if idx is None else int(idx)
    if idx not in _DEFAULT:
        _DEFAULT[idx] = Context()
    return _DEFAULT[idx]
