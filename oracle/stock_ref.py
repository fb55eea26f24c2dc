"""Runs the unmodified reference (ed-lgt) through its own public model API.

Benchmark infrastructure, not part of the engine: ``bench.py`` starts this
file as a child process for its CPU baseline and for its reference arm, so
that the thread settings below are in place before numpy, SciPy and Numba
load, and so that the process never maps the engine's ``libedgpu.so``
(checked at exit through ``/proc/self/maps``).  Nothing in ``ed-lgt_b200/``
imports it.

The reference is the ``edlgt`` package installed, unmodified, into
``baseline/_ref`` at the repository root (``pip install --no-deps --target
baseline/_ref <checkout>``; set ``EDLGT_PATH`` to use another copy).  The
only shim is for modules its package imports but that are absent here:
matplotlib (plotting helpers) and two ``edlgt.tools`` submodules that are
not in its snapshot.

Stock path timed (ed-lgt 0.2.3):
* ``SU2_Model(...)`` constructor: operator tables and the symmetry sector
  (``edlgt/models/SU2_model.py:31-169``, whose ``get_abelian_symmetry_sector``
  is ``edlgt/models/quantum_model.py:504-604``);
* ``default_params`` + ``build_Hamiltonian(g, m)``: sector Hamiltonian
  assembly (``SU2_model.py:171-355``, ``modeling/qmb_hamiltonian.py:173-225``);
* ``diagonalize_Hamiltonian(1, fmt)``: ARPACK ``eigsh(k=1, "SA")`` on the
  Numba CSR matvec (``fmt="linear"``) or on SciPy CSR (``fmt="sparse"``)
  (``modeling/qmb_hamiltonian.py:260-332``).

    python oracle/stock_ref.py --L 14 --pbc --g 1.0 --m 0.5 --steps K --warmup W

prints one JSON object with the per-phase seconds of every timed step.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _threads_env():
    n = str(os.cpu_count() or 1)
    for k in ("NUMBA_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS", "OPENBLAS_NUM_THREADS"):
        os.environ.setdefault(k, n)
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join("/tmp", "numba_cache_edlgt_stock"))
    return int(os.environ["NUMBA_NUM_THREADS"])


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


def load_reference():
    """Put the installed reference on sys.path behind the module stubs and
    return its ``edlgt.models`` module."""
    path = os.environ.get("EDLGT_PATH", os.path.join(ROOT, "baseline", "_ref"))
    if not os.path.isdir(os.path.join(path, "edlgt")):
        raise FileNotFoundError(f"no edlgt package under {path}")
    _stub("matplotlib", use=lambda *a, **k: None, rcParams={})
    _stub("matplotlib.pyplot", FuncFormatter=lambda f: f)
    _stub("matplotlib.colors")
    _stub("matplotlib.cm")
    for n in ("edlgt.tools.wannier", "edlgt.tools.tensor_networks"):
        m = types.ModuleType(n)
        m.__all__ = []
        sys.modules[n] = m
    sys.path.insert(0, path)
    import logging

    logging.disable(logging.INFO)
    import edlgt.models as models

    return models


def engine_loaded():
    """True when this process has the engine's shared library mapped."""
    try:
        with open("/proc/self/maps") as f:
            return any("libedgpu" in line for line in f)
    except OSError:
        return False


def pipeline(models, L, pbc, g, m, fmt):
    """One ground state through the stock model API; returns phase seconds."""
    t0 = time.perf_counter()
    model = models.SU2_Model(spin=0.5, pure_theory=False, lvals=[L], has_obc=[not pbc], sectors=[L])
    t1 = time.perf_counter()
    model.default_params()
    model.build_Hamiltonian(g, m)
    t2 = time.perf_counter()
    model.diagonalize_Hamiltonian(1, fmt)
    t3 = time.perf_counter()
    return {"sector_s": t1 - t0, "assembly_s": t2 - t1, "solve_s": t3 - t2, "total_s": t3 - t0,
            "energy_density": float(model.H.Nenergies[0]), "dim": int(len(model.sector_configs)), "format": fmt}


def main(argv=None):
    threads = _threads_env()
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=14)
    ap.add_argument("--pbc", action="store_true")
    ap.add_argument("--g", type=float, nargs="+", default=[1.0])
    ap.add_argument("--m", type=float, default=0.5)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--warm-L", type=int, default=6)
    ap.add_argument("--format", default="auto", choices=["auto", "linear", "sparse"])
    a = ap.parse_args(argv)
    models = load_reference()
    # Warm-up: the first warm-up steps compile the Numba kernels on a short
    # chain (both matvec formats); with --format auto, two full-size warm-up
    # solves then pick the faster of the reference's "linear" (Numba CSR) and
    # "sparse" (SciPy) formats for the timed steps.
    warm = []
    t0 = time.perf_counter()
    pipeline(models, a.warm_L, a.pbc, a.g[0], a.m, "linear")
    pipeline(models, a.warm_L, a.pbc, a.g[0], a.m, "sparse")
    fmt = a.format
    choice = {}
    if fmt == "auto":
        for f in ("sparse", "linear"):
            choice[f] = pipeline(models, a.L, a.pbc, a.g[0], a.m, f)
            warm.append(choice[f])
        fmt = min(choice, key=lambda f: choice[f]["solve_s"])
    for _ in range(max(a.warmup - 1 - len(choice), 0)):
        pipeline(models, a.warm_L, a.pbc, a.g[0], a.m, fmt)
    warm_s = time.perf_counter() - t0
    steps = [pipeline(models, a.L, a.pbc, a.g[i % len(a.g)], a.m, fmt) for i in range(a.steps)]
    import numpy as np

    out = {"threads": threads, "cpu_count": os.cpu_count(), "format": fmt,
           "format_trial_solve_s": {f: c["solve_s"] for f, c in choice.items()},
           "format_trials": list(choice.values()),
           "warmup_s": warm_s, "steps": steps, "engine_loaded": engine_loaded(),
           "numpy": np.__version__, "reference_path": os.environ.get("EDLGT_PATH", "baseline/_ref")}
    try:
        with open("/proc/cpuinfo") as f:
            out["cpu_model"] = next(line.split(":", 1)[1].strip() for line in f if line.startswith("model name"))
    except (OSError, StopIteration):
        out["cpu_model"] = None
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
