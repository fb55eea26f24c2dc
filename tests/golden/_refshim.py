"""Import shim that lets ed-lgt (the reference) run in this container.

Used only by make_golden.py to produce fixtures.  It stubs the modules the
reference imports but that are absent here (matplotlib and two edlgt.tools
submodules that are not in the snapshot), without touching the reference
tree.  Set EDLGT_PATH to the reference checkout (required).
"""

import os
import sys
import types

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_edlgt")


class _Any:
    def __getattr__(self, k):
        return _Any()

    def __call__(self, *a, **k):
        return _Any()


def _stub(name, **attrs):
    m = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(m, k, v)
    m.__getattr__ = lambda k: _Any()
    sys.modules[name] = m
    return m


_stub("matplotlib", use=lambda *a, **k: None, rcParams={})
_stub("matplotlib.pyplot", FuncFormatter=lambda f: f)
_stub("matplotlib.colors")
_stub("matplotlib.cm")
for _n in ("edlgt.tools.wannier", "edlgt.tools.tensor_networks"):
    _m = types.ModuleType(_n)
    _m.__all__ = []
    sys.modules[_n] = _m
if "EDLGT_PATH" not in os.environ:
    raise SystemExit("set EDLGT_PATH to an ed-lgt checkout (the directory that holds the edlgt package)")
sys.path.insert(0, os.environ["EDLGT_PATH"])
