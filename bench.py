#!/usr/bin/env python
"""Benchmark: Lanczos ground-state time-to-solution and matvec bandwidth,
mixed-precision batched vs plain FP64 on the GPU, for the SU(2) coupling
sweep workload (1D SU(2) Yang-Mills + staggered matter, j_max = 1/2, periodic
chain L = 14, N_tot = 14 sector of dimension 1,232,454, g^2 in {0.5, 1, 2},
m = 0.5).  One step solves the three ground states.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl edgpu|reference]

Arms.
* edgpu (default): the sector Hamiltonian is assembled once on the device;
  a step is one batched mixed-precision Lanczos over the three couplings
  (f32 Krylov vectors and matvec, f64 recurrence / reorthogonalisation /
  tridiagonal solve) plus the f64 refinement.  ``value`` = ground states per
  second with the matrix resident in HBM; ``e2e`` = the same through the
  public model API from host inputs (sector enumeration, assembly, solve,
  eigenvectors copied back to the host) every step.  The plain FP64 path
  (three sequential f64 Lanczos solves) is timed beside it, and the sector
  enumeration and assembly phases are timed on their own.
* reference: the unmodified ed-lgt (``baseline/_ref``) through its own model
  API -- ``SU2_Model(...)`` (sector), ``build_Hamiltonian`` (assembly),
  ``diagonalize_Hamiltonian(1, fmt)`` (ARPACK on the faster of its "linear"
  Numba CSR and "sparse" SciPy formats) -- one coupling per step, on all host
  cores, in a child process that never loads this engine
  (``oracle/stock_ref.py``).  Under torchrun only rank 0 runs it.

Other workloads (``--workload``), each printing its own JSON line: ``batch``
(QED 3x2 instance batch), ``quench`` (SU(2) L=16 Krylov dynamics), ``z3``
(Z3 4x3 zero-momentum matrix-free batch), ``corr`` (two-body correlator
matrices, SU(2) L=16), ``entropy`` (half-chain entanglement, SU(2) L=14) and
``momentum`` (zero-momentum ground state, SU(2) L=14 PBC).

Multi-GPU: one process per GPU (torchrun); every rank solves its own replica
of the sweep (independent instances, no data exchange: weak scaling);
timings are the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "ed-lgt_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

L = 14
PBC = True
SWEEP = (0.5, 1.0, 2.0)
MASS = 0.5
WINDOW32 = 4  # local reorthogonalisation window of the f32 phase (the f64 refinement is full)
METRIC = "Lanczos GS time-to-solution & matvec GB/s: mixed/batched vs plain FP64 GPU at 1e-9 rel."
# DRAM traffic of the headline kernels from one ncu capture each on this
# workload (summaries kept under profiles/): the one-launch reorthogonalisation
# of a full window (5 vectors) moved 146.00 + 15.95 MB against 251.42 MB
# algorithmic (its update phase re-reads the dots phase's rows from L2); one
# dictionary-packed matvec launch moved 112.87 + 14.91 MB; one CSR matvec
# launch (2 lanes a row) moved 179.21 + 21.61 MB
REORTH_TRAFFIC_RATIO = (146.00 + 15.95) / 251.42
PACKED_MATVEC_TRAFFIC_BYTES = (112.87 + 14.91) * 1e6
MATVEC_TRAFFIC_BYTES = (179.21 + 21.61) * 1e6
UNIT = "ground_states/s"
REF_MAX_PIPELINES = 6  # timed pipelines of the reference arm (about 12 s each on 16 host cores)
WORKLOAD = (f"SU(2) 1D Yang-Mills + staggered matter, j_max=1/2, {'periodic' if PBC else 'open'} chain L={L}, "
            f"N_tot={L} sector; ground states for g^2 in {list(SWEEP)}, m={MASS}")


def model_kwargs():
    return dict(spin=0.5, pure_theory=False, lvals=[L], has_obc=[not PBC], sectors=[L])


def stock_reference(steps, warmup, fmt="auto", couplings=SWEEP, timeout=3000):
    """Run the unmodified ed-lgt through its model API in a child process
    (oracle/stock_ref.py, which never loads this engine); returns its JSON."""
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "stock_ref.py"), "--L", str(L), "--m", str(MASS),
           "--steps", str(steps), "--warmup", str(warmup), "--format", fmt, "--g", *[str(g) for g in couplings]]
    if PBC:
        cmd.append("--pbc")
    env = dict(os.environ)
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "LOCAL_WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"stock reference failed (rc {out.returncode}): {out.stderr[-2000:]}")
    res = json.loads(out.stdout.strip().splitlines()[-1])
    if res["engine_loaded"]:
        raise RuntimeError("the reference process mapped libedgpu.so")
    return res


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world, device):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        # nvidia-smi numbers GPUs by PCI order, not by CUDA_VISIBLE_DEVICES:
        # name the device by its UUID so the samples describe this process's GPU
        self.gpu = str(gpu_index)
        try:
            import torch

            self.gpu = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
        except Exception:
            pass
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"edgpu_clocks_rank{gpu_index}_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = np.array([float(r[1]) for r in rows])
        smax = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, nm in enumerate(names):
            if any(r[5 + k].lower() == "active" for r in rows):
                reasons.append(nm)
        loaded = sm[sm > 0.5 * np.max(sm)] if np.any(sm > 0) else sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def run_reference(args):
    """The reference arm: stock ed-lgt on the host cores, rank 0 only (no
    process group is created, so other ranks exit at once)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    # a reference pipeline takes about 12 s on 16 host cores: at most
    # REF_MAX_PIPELINES of them are timed (the rate is their mean), so the arm
    # ends within a few minutes whatever --steps asks
    timed = max(1, min(args.steps, REF_MAX_PIPELINES))
    res = stock_reference(timed, args.warmup)
    steps = res["steps"]
    ms = 1e3 * float(np.mean([st["total_s"] for st in steps]))
    value = 1e3 / ms
    phases = {k: 1e3 * float(np.mean([st[k] for st in steps])) for k in ("sector_s", "assembly_s", "solve_s")}
    sample = (f"one coupling per step (cycling g^2 over {list(SWEEP)}): SU2_Model(...) sector, build_Hamiltonian, "
              f"diagonalize_Hamiltonian(1, '{res['format']}') = ARPACK eigsh; {timed} of the {args.steps} "
              "requested steps timed (each a full ground-state pipeline)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "steps_timed": timed, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128", "data": "synthetic (model Hamiltonian; no dataset)",
        "config": {"workload": WORKLOAD, "sector_dim": steps[0]["dim"] if steps else None, "instances_per_step": 1,
                   "sample": sample},
        "phases_ms_per_step": {"sector": phases["sector_s"], "assembly": phases["assembly_s"],
                               "solve": phases["solve_s"]},
        "format_trial_solve_s": res["format_trial_solve_s"],
        "energies_per_site": [st["energy_density"] for st in steps[:3]],
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["threads"], "kind": "reference",
                         "cpu_model": res.get("cpu_model"), "sample": sample,
                         "reference": "edlgt 0.2.3, unmodified, from baseline/_ref; Numba/SciPy/ARPACK threads = "
                                      "host cores; warm JIT; engine library not loaded"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def setup_phases(dev, reps=3):
    """Sector enumeration and assembly on the device, each timed on its own
    (host clock around synchronised calls: the enumeration reads each level's
    size back to the host).  Returns timings and the compulsory bytes."""
    import torch

    from edgpu.models import SU2_Model

    def once():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m = SU2_Model(**model_kwargs(), device=dev)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        m.build_Hamiltonian(SWEEP[1], MASS)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        return m, t1 - t0, t2 - t1

    once()  # warm-up: host caches, kernel loads
    ts_sec, ts_asm = [], []
    for _ in range(reps):
        m, a, b = once()
        ts_sec.append(a)
        ts_asm.append(b)
    sec = m.sector
    ng = getattr(sec, "n_glob", 1)
    rec = 8 + 4 * max(ng, 1)  # a prefix: its key and its running global sums
    parents = [1] + list(sec.level_sizes[:-1])
    # every level reads its parents twice (count, fill) and writes its survivors
    enum_bytes = sum(2 * p * rec + c * rec for p, c in zip(parents, sec.level_sizes))
    mat = m.H.mat
    n, nnz = mat.n, mat.nnz
    # compulsory assembly bytes: sector keys in; canonical CSR (rowptr, cols,
    # f64 values), f64 diagonal and the diagonal-present bytes out
    asm_bytes = 8 * n + 8 * (n + 1) + nnz * (4 + 8) + 8 * n + n
    sec_ms, asm_ms = 1e3 * float(np.median(ts_sec)), 1e3 * float(np.median(ts_asm))
    return {
        "sector_enumeration": {"ms": sec_ms, "levels": len(sec.level_sizes), "algorithmic_bytes": int(enum_bytes),
                               "GBps": enum_bytes / (sec_ms * 1e-3) / 1e9,
                               "includes": "model construction (operator tables) + level-by-level enumeration, "
                                           "one host read of each level's size"},
        "assembly": {"ms": asm_ms, "raw_entries": int(getattr(mat, "raw_entries", 0)), "nnz": nnz,
                     "algorithmic_bytes": int(asm_bytes), "GBps": asm_bytes / (asm_ms * 1e-3) / 1e9,
                     "includes": "build_Hamiltonian(g^2=1): term tables, count, scan, fill (key search per "
                                 "transition), per-row merge, compaction"},
    }


def run_edgpu(args, world, rank, local):
    import torch

    from edgpu import _lib
    from edgpu.models import SU2_Model
    from edgpu.solvers import lanczos_mixed, run_lanczos, stack_diagonals

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    # ---------------- setup phases, timed on their own -----------------------
    phases_setup = setup_phases(dev)
    # ---------------- setup (untimed): sector, assembly, f32 copies ----------
    model = SU2_Model(**model_kwargs(), device=dev)
    diags = []
    mat = None
    for g in SWEEP:
        model.build_Hamiltonian(g, MASS)
        diags.append(model.H.mat.diag.clone())
        mat = model.H.mat
    n, nnz = mat.n, mat.nnz
    vals32 = mat.vals.to(torch.float32)
    diag32 = stack_diagonals(diags, torch.float32)
    diag64 = stack_diagonals(diags, torch.float64)
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    from edgpu.solvers import tune_spmv_group

    g64s = args.spmv_group or tune_spmv_group(mat, 1, 0, vals=mat.vals)
    # ---------------- plain FP64 GPU path: three sequential solves -----------
    e64 = []
    t64 = []
    stats_fp64 = np.zeros(6)

    def fp64_solve(i, stats=None):
        return run_lanczos(0, n, nnz, mat.rowptr, mat.cols, mat.vals, diags[i], nvec=1, k=1, max_iter=400,
                           tol=1e-12, check_every=5, stats=stats, group=g64s)

    for rep in range(2):  # first repetition warms up
        e64.clear()
        t64.clear()
        for i in range(3):
            flush.zero_()
            torch.cuda.synchronize()
            a, b = ev(), ev()
            a.record()
            r = fp64_solve(i)
            b.record()
            torch.cuda.synchronize()
            t64.append(a.elapsed_time(b))
            e64.append(r.evals[0, 0])
    fp64_ms = float(np.sum(t64))
    for i in range(3):  # phase timings: one instrumented solve per coupling (outside the timed runs)
        st = np.zeros(6)
        fp64_solve(i, st)
        stats_fp64 += st

    # ---------------- mixed batched: warm-up + timed steps --------------------
    # matvec threads-per-row: the autotuner's choice (or --spmv-group), fixed
    # before the timed region
    from edgpu.solvers import sell_layout, tune_matvec32

    # f32 matvec layout (SELL or CSR) and threads per row: the autotuner's
    # choices (or --spmv-group, which forces CSR), fixed before the timed region
    from edgpu.solvers import packed_layout

    if args.matvec_layout == "auto":
        fmt32, param = ("csr", args.spmv_group) if args.spmv_group else tune_matvec32(mat, 3, vals32)
    elif args.matvec_layout == "sell":
        fmt32, param = "sell", args.sell_window
    elif args.matvec_layout == "packed":
        fmt32, param = "packed", 2
    else:
        fmt32, param = "csr", args.spmv_group or tune_spmv_group(mat, 3, 1, vals=vals32)
    sell32 = sell_layout(mat, vals32, param) if fmt32 == "sell" else False
    pk32 = packed_layout(mat) if fmt32 == "packed" else None
    if fmt32 == "packed" and pk32 is None:
        raise SystemExit("--matvec-layout packed: the matrix does not pack")
    g32 = param if fmt32 in ("csr", "packed") else tune_spmv_group(mat, 3, 1, vals=vals32)
    g64 = args.spmv_group or tune_spmv_group(mat, 3, 0, vals=mat.vals)

    def mixed_step(s32, s64):
        return lanczos_mixed(mat, diags=diags, vals32=vals32, diag32=diag32, diag64=diag64, stats32=s32, stats64=s64,
                             group32=g32, group64=g64, sell=sell32, window32=WINDOW32, packed=pk32)

    for _ in range(args.warmup):
        mixed_step(None, None)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    step_ms = []
    emix = None
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between steps (512 MB > 126 MB L2), outside the step events
        a, b = ev(), ev()
        a.record()
        r64, r32 = mixed_step(None, None)
        b.record()
        torch.cuda.synchronize()
        step_ms.append(a.elapsed_time(b))
        emix = r64.evals[:, 0]
        iters32 = r32.iters.tolist()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    # phase timings: one instrumented sweep (steps launched one by one with
    # CUDA events around each phase), outside the timed steps
    agg32, agg64 = np.zeros(6), np.zeros(6)
    flush.zero_()
    mixed_step(agg32, agg64)
    ms = max_over_ranks(float(np.mean(step_ms)), world, dev)
    value = 3 * world / (ms * 1e-3)
    rel = float(np.max(np.abs(np.array(emix) - np.array(e64)) / np.abs(np.array(e64))))

    # ---------------- rooflines (CUDA events inside the timed steps) -----------
    hbm, peak_kind = peaks()
    nv = 3
    n_pad = (n + 3) // 4 * 4
    # matvec: entries + row index + x (f32) + y (f64) + diagonal (f32); an
    # entry is a value and a column (8 B) for CSR and SELL; the
    # dictionary-packed tiles read one 4-byte word per slot (entries and the
    # tiles' padding) plus one int32 offset per tile of 16 rows (their value
    # table, a few bytes, once per CTA); the row index is rowptr (8 B a row)
    # for CSR, the row permutation (4 B a row) plus a width and an offset per
    # slice of 32 rows (12 B) for SELL
    if fmt32 == "packed":
        stream = pk32.stream_bytes
    else:
        stream = nnz * 8 + (8 * (n + 1) if fmt32 == "csr" else 4 * n + 12 * ((n + 31) // 32))
    spmv_bytes = stream + n * nv * 4 + n * nv * 8 + n * nv * 4
    spmv_ms = agg32[0] / max(agg32[1], 1)  # agg32/agg64: the one instrumented sweep
    spmv_achieved = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    # reorthogonalisation of step j (delayed Gram-Schmidt over the window
    # V[lo..j), lo = max(0, j - WINDOW32)), per row of every problem: the dots
    # read V[lo..j] (f32, the candidate u = V[j] among them) and w (f64) once;
    # the update reads V[lo..j), u and w and writes q_j = V[j], the next
    # candidate V[j+1] and the matvec input
    steps = int(round(agg32[4]))

    def lo_of(j):
        return j - WINDOW32 if (WINDOW32 and j > WINDOW32) else 0

    reorth_bytes = sum(n_pad * nv * (4 * (j + 1 - lo_of(j)) + 8 + 4 * (j - lo_of(j)) + 4 + 8 + 4 + 4 + 4)
                       for j in range(steps))
    reorth_ms_step = agg32[2]
    reorth_achieved = reorth_bytes / (reorth_ms_step * 1e-3) / 1e9
    reorth_ms = agg32[2] / max(agg32[4], 1)
    fp64_spmv_bytes = nnz * (8 + 4) + 8 * (n + 1) + n * 8 * 3
    fp64_spmv_ms = stats_fp64[0] / max(stats_fp64[1], 1)

    # ---------------- e2e through the public API with host inputs ------------
    e2e_ms = []
    d2h = h2d = 0
    for it in range(args.steps + 1):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m2 = SU2_Model(**model_kwargs(), device=dev)
        dg = []
        tables_bytes = 0
        for g in SWEEP:
            m2.build_Hamiltonian(g, MASS)
            dg.append(m2.H.mat.diag.clone())
            tables_bytes += sum(t.numel() * t.element_size() for t in m2.H.mat._keep)
        r64e, _ = lanczos_mixed(m2.H.mat, diags=dg, window32=WINDOW32)
        gs_host = torch.empty(r64e.evecs[0].shape, dtype=r64e.evecs[0].dtype, pin_memory=True)
        gs_host.copy_(r64e.evecs[0])  # ground states to pinned host memory
        gs = gs_host.numpy()
        energies = r64e.evals[:, 0] / L
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if it > 0:  # first iteration warms the host-side caches
            e2e_ms.append(1e3 * dt)
        d2h = gs.nbytes + energies.nbytes
        spec = m2.sector_spec
        spec_bytes = sum(np.asarray(getattr(spec, a)).nbytes for a in (
            "site_allowed", "glob_val", "glob_target", "glob_rem_min", "glob_rem_max", "link_val", "link_target",
            "pair_start", "pair_s0", "pair_s1", "pair_dir"))
        h2d = spec_bytes + tables_bytes
        del m2
    e2e = 3 * world / (max_over_ranks(float(np.mean(e2e_ms)), world, dev) * 1e-3)
    # phase split of one more pipeline, synchronised after every phase
    # (outside the timed pipelines)
    from edgpu.solvers import packed_layout as _packed_layout

    marks = [("start", time.perf_counter())]

    def mark(name):
        torch.cuda.synchronize()
        marks.append((name, time.perf_counter()))

    m2 = SU2_Model(**model_kwargs(), device=dev)
    mark("model_and_sector")
    dg = []
    for g in SWEEP:
        m2.build_Hamiltonian(g, MASS)
        dg.append(m2.H.mat.diag.clone())
    mark("assembly_x3")
    _packed_layout(m2.H.mat)
    mark("matvec_layout")
    r64e, _ = lanczos_mixed(m2.H.mat, diags=dg, window32=WINDOW32)
    mark("solve")
    gs_host = torch.empty(r64e.evecs[0].shape, dtype=r64e.evecs[0].dtype, pin_memory=True)
    gs_host.copy_(r64e.evecs[0])
    mark("d2h_ground_states")
    e2e_phases = {marks[i][0]: 1e3 * (marks[i][1] - marks[i - 1][1]) for i in range(1, len(marks))}
    del m2

    # ---------------- CPU baseline (rank 0, bounded sample) ------------------
    cpu = None
    if rank == 0 and not args.no_cpu:
        # the format trial of the stock runner: one full pipeline per matvec
        # format; the faster one is the sample
        res = stock_reference(0, 1, fmt="auto", couplings=(1.0,))
        st0 = min(res["format_trials"], key=lambda t: t["total_s"])
        cpu = {"value": 1.0 / st0["total_s"], "unit": UNIT, "cores": res["threads"], "kind": "reference",
               "cpu_model": res.get("cpu_model"),
               "sample": "one ground state (g^2=1) through the unmodified ed-lgt model API: SU2_Model(...) sector, "
                         f"build_Hamiltonian, diagonalize_Hamiltonian(1, '{st0['format']}') (the faster of its "
                         "'linear' and 'sparse' formats, both run)",
               "phases_s": {k: st0[k] for k in ("sector_s", "assembly_s", "solve_s")},
               "energy_matches_gpu": bool(abs(st0["energy_density"] * L - e64[1]) < 1e-8 * abs(e64[1]))}
    # the largest configuration (C5), on one GPU only: it holds most of HBM
    largest = None
    if world == 1 and not args.no_largest:
        del model, mat, vals32, diag32, diag64, diags, flush
        torch.cuda.empty_cache()
        clk_l = ClockSampler(local)
        clk_l.start()
        largest = largest_config(dev, args.warmup)
        largest["clocks"] = clk_l.stop()
    if rank != 0:
        return
    launches = int(agg32[3] + agg64[3]) + 1  # + the f32->f64 start-vector conversion
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "step_ms_spread": {"min": float(np.min(step_ms)), "median": float(np.median(step_ms)),
                           "max": float(np.max(step_ms))},
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 Krylov/matvec + f64 recurrence (mixed)",
        "data": "synthetic (model Hamiltonian, no dataset)",
        "config": {"workload": WORKLOAD, "sector_dim": n, "offdiag_nnz": nnz, "instances_per_step": 3,
                   "l2": "512 MB memset between steps (L2 is 126 MB), outside the step events",
                   "parallelism": f"replicas x{world} (independent sweeps per GPU)"},
        "fp64_gpu": {"ms_per_sweep": fp64_ms, "speedup_mixed_vs_fp64": fp64_ms / ms,
                     "steps_total": int(stats_fp64[4]), "spmv_ms": fp64_spmv_ms,
                     "spmv_GBps": fp64_spmv_bytes / (fp64_spmv_ms * 1e-3) / 1e9},
        "accuracy": {"max_rel_dE_vs_fp64": rel, "f32_lanczos_steps": iters32, "target": 1e-9,
                     "energies_per_site": [float(x) / L for x in emix]},
        "phases_ms_per_step": {"f32_matvec": agg32[0], "f32_reorth": agg32[2], "f32_checks": agg32[5],
                               "f32_steps": agg32[4], "f64_refine_total": agg64[0] + agg64[2] + agg64[5],
                               "f64_matvec": agg64[0], "f64_reorth": agg64[2], "f64_checks": agg64[5],
                               "f64_steps": agg64[4],
                               "source": "one instrumented sweep (CUDA events around every phase of every step)"},
        "setup_phases": phases_setup,
        "roofline": {"kernel": f"f32 delayed Gram-Schmidt reorthogonalisation over a window of {WINDOW32} vectors "
                               "(reorth_small_k<float,3,5>: one cooperative launch per Lanczos step -- dots, grid "
                               "barrier, coefficients in every CTA, update in reverse row order)",
                     "bound": "hbm",
                     "achieved": reorth_achieved, "peak": hbm, "unit": "GB/s", "frac": reorth_achieved / hbm,
                     "peak_source": peak_kind, "algorithmic_bytes_per_solve": reorth_bytes,
                     "ms_per_solve": reorth_ms_step, "ms_per_lanczos_step": reorth_ms,
                     "traffic": REORTH_TRAFFIC_RATIO * reorth_bytes,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch with a "
                                       f"full window on this workload = {REORTH_TRAFFIC_RATIO:.4f} x its algorithmic "
                                       "bytes (L2 reuse between its phases), applied per solve"},
        "roofline_matvec": {"kernel": ("batched f32 SELL-32-sigma + diag matvec (sell_spmv_k<float,3,4>), "
                                       f"sort window {sell32.window}, slice padding {sell32.padding:.3f} of the "
                                       "stored pairs"
                                       if fmt32 == "sell" else
                                       "batched f32 dictionary-packed tiled matvec (packed_spmv_k<float,3,4>): "
                                       f"{pk32.count} distinct values, {pk32.colbits}-bit columns, tiles of 16 rows, "
                                       f"padding {pk32.padding:.3f} of the words"
                                       if fmt32 == "packed" else
                                       f"batched f32 CSR+diag matvec (spmv_k<float,float,double,3,{g32},4>)"),
                            "layout_choice": fmt32,
                            "bound": "hbm", "achieved": spmv_achieved, "peak": hbm, "unit": "GB/s",
                            "frac": spmv_achieved / hbm, "peak_source": peak_kind,
                            "algorithmic_bytes_per_launch": spmv_bytes, "avg_launch_ms": spmv_ms,
                            "traffic": (PACKED_MATVEC_TRAFFIC_BYTES if fmt32 == "packed" and n == 1232454 else
                                        MATVEC_TRAFFIC_BYTES if fmt32 == "csr" and g32 == 2 and n == 1232454
                                        else None),
                            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                                              + ("packed_spmv_k<float, 3, 4>" if fmt32 == "packed" else
                                                 "spmv_k<float, float, double, 3, 2, 4>") + " on this matrix"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": float(np.mean(e2e_ms)), "steps": len(e2e_ms),
                "phases_ms": e2e_phases, "phases_source": "one extra pipeline, synchronised after every phase"},
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": cpu,
        "largest_config": largest,
    }
    print(json.dumps(line), flush=True)
    del _lib


# ---------------------------------------------------------------------------
# other workloads of the same path (not the headline line)
def run_batch(args, world, rank, local):
    """QED 3x2 OBC: 64 couplings (g log-uniform in [0.1, 5], m uniform in
    [0, 2], seed 0) in the Q = 0 sector plus the Q = -2, -1, 1, 2 sectors,
    then the same batch with SU(2) chains of L = 10 and 12 (dims 8,953 and
    73,789) added.  Each solve is one (instance, row-tile) batched launch per
    precision phase, replayed from a CUDA graph; mixed precision and f64."""
    import torch

    from edgpu.batch import TiledBatch
    from edgpu.models import QED_Model, SU2_Model

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(0)
    gs = np.exp(rng.uniform(np.log(0.1), np.log(5.0), 64))
    ms = rng.uniform(0.0, 2.0, 64)
    charge_bg = {-2: [1, 0, 0, 0, 0, 1], -1: [1, 0, 0, 0, 0, 0], 1: [-1, 0, 0, 0, 0, 0], 2: [-1, 0, 0, 0, 0, -1]}

    def build_c3():
        mats = []
        base = QED_Model(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True], device=dev)
        for g, m in zip(gs, ms):
            base.build_Hamiltonian(float(g), float(m))
            mats.append(base.H.mat)
        for q, bg in charge_bg.items():
            mq = QED_Model(spin=1, pure_theory=False, lvals=[3, 2], has_obc=[True, True], bg_list=bg, charge=q,
                           device=dev)
            mq.build_Hamiltonian(1.0, 1.0)
            mats.append(mq.H.mat)
        return mats

    def build_su2():
        mats = []
        for L_ in (10, 12):
            m2 = SU2_Model(spin=0.5, pure_theory=False, lvals=[L_], has_obc=[True], sectors=[L_], device=dev)
            m2.build_Hamiltonian(1.0, 0.5)
            mats.append(m2.H.mat)
        return mats

    c3 = build_c3()
    mixed_batch = c3 + build_su2()
    out = {}
    for label, mats in (("c3", c3), ("c3_plus_su2_L10_L12", mixed_batch)):
        for prec in ("mixed", "fp64"):
            tb = TiledBatch(mats, k=1, precision=prec)
            tb.capture()
            for _ in range(args.warmup):
                tb.solve()
            torch.cuda.synchronize()
            ts = []
            for _ in range(args.steps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                tb.solve()
                b.record()
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
            tb.check_status()
            ms_step = max_over_ranks(float(np.mean(ts)), world, dev)
            out[f"{label}/{prec}"] = {"ms_per_solve": ms_step, "instances_per_s": len(mats) * world / (ms_step * 1e-3),
                                     "tile_rows": tb.tile_rows, "lanes": tb.lanes,
                                     "energies_first": tb.evals[:3, 0].cpu().numpy().tolist()}
        e_m = TiledBatch(mats, precision="mixed").solve(use_graph=False).cpu().numpy()[:, 0]
        e_d = TiledBatch(mats, precision="fp64").solve(use_graph=False).cpu().numpy()[:, 0]
        out[f"{label}/max_rel_dE_mixed_vs_fp64"] = float(np.max(np.abs(e_m - e_d) / np.abs(e_d)))
        out[f"{label}/instances"] = len(mats)
        out[f"{label}/dims"] = sorted({int(m.n) for m in mats})
    # beside it: the one-CTA-per-instance f64 kernel (instances up to 4096
    # rows, no grid-wide waits), for the small-instance batch
    from edgpu.batch import SmallBatch

    sb = SmallBatch(c3, k=1)
    sb.capture()
    for _ in range(args.warmup):
        sb.solve()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        sb.solve()
    b.record()
    torch.cuda.synchronize()
    sb_ms = a.elapsed_time(b) / args.steps
    out["c3/one_cta_per_instance_fp64"] = {"ms_per_solve": sb_ms, "instances_per_s": len(c3) / (sb_ms * 1e-3)}
    # e2e: instances from host couplings to energies on the host
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mats2 = build_c3()
    tb2 = TiledBatch(mats2, k=1, precision="mixed")
    tb2.launch()
    e_host = tb2.evals.cpu().numpy()
    e2e_ms = 1e3 * (time.perf_counter() - t0)
    # CPU: scipy eigsh (the reference's solver, ARPACK) on each instance's
    # canonical matrix in a loop
    from scipy.sparse.linalg import eigsh

    def cpu_loop(ms_):
        Hs = [m.to_scipy() for m in ms_]
        t0_ = time.perf_counter()
        for H in Hs:
            if H.shape[0] > 3:
                eigsh(H, k=1, which="SA")
        return time.perf_counter() - t0_

    cpu_c3 = cpu_loop(c3)
    cpu_mixed = cpu_loop(mixed_batch)
    if rank == 0:
        head = out["c3/mixed"]
        print(json.dumps({
            "metric": METRIC, "workload": "batch", "value": head["instances_per_s"], "unit": "instances/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_solve"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 Krylov/matvec + f64 dots, recurrence, eigen-solve; f64 refinement",
            "data": "synthetic (model Hamiltonians)",
            "config": {"workload": "QED 2D 3x2 OBC spin 1 with matter: 64 (g, m) in Q=0 (dim 90) + Q=-2..2 sectors "
                                   "(dims 26, 52, 67, 26); and the same plus SU(2) L=10, 12 open chains; one "
                                   "(instance, row-tile) batched launch per precision phase (CUDA graph)",
                       "instances_per_step": out["c3/instances"]},
            "batches": out,
            "e2e": {"value": out["c3/instances"] / (e2e_ms * 1e-3), "unit": "instances/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": int(e_host.nbytes)},
            "cpu_baseline": {"value": out["c3/instances"] / cpu_c3, "unit": "instances/s", "cores": 1, "kind": "port",
                             "sample": "scipy eigsh(k=1, SA) on each instance's canonical matrix in a loop",
                             "c3_plus_su2_instances_per_s": out["c3_plus_su2_L10_L12/instances"] / cpu_mixed},
        }), flush=True)


def run_quench(args, world, rank, local):
    """SU(2) 1D L=16 OBC with a j=1/2 static pair at sites 5 and 10 (sector
    dim 7,133,222): complex64 Krylov (m = 30) from the string state for
    t in [0, T] with dt = 0.05, observables E^2 per link and pair density at
    every step, checked against a complex128 evolution over the first steps."""
    import torch

    from edgpu.dynamics import KrylovEvolver
    from edgpu.models import SU2_Model
    from edgpu.models.quantum_model import site_expval_device

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bg = [0] * 5 + [0.5] + [0] * 4 + [0.5] + [0] * 5
    model = SU2_Model(spin=0.5, pure_theory=False, lvals=[16], has_obc=[True], sectors=[16], bg_list=bg, device=dev)
    model.build_Hamiltonian(1.0, 1.0)
    cfg = model.sector_configs
    c0 = cfg[np.argmax((cfg == 0).sum(axis=1))]
    psi0 = model.H.from_original_basis(torch.from_numpy(model.get_qmb_state_from_configs([c0])).to(dev))
    dt, T = 0.05, args.quench_time
    n_t = int(round(T / dt))
    ops = {"T2_px": model.ops["T2_px"], "N_pair": model.ops["N_pair"]}

    layout = {}

    def evolve(prec, steps, matvec="auto"):
        ev = KrylovEvolver(model.H.mat, m=30, precision=prec, reorth_passes=0, matvec=matvec)
        layout[(prec, matvec)] = "packed" if ev.packed is not None else "csr"
        psi = psi0.to(ev.vdtype).clone()
        out = {k: torch.zeros((steps + 1, 16), dtype=torch.float64, device=dev) for k in ops}
        for k in ops:
            site_expval_device(model.sector, ops[k], psi, out=out[k][0])
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for t in range(1, steps + 1):
            ev.step(psi, dt)
            for k in ops:
                site_expval_device(model.sector, ops[k], psi, out=out[k][t])
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b), {k: v.cpu().numpy() for k, v in out.items()}

    evolve("c64", 2)  # warm-up
    t64, obs64 = evolve("c64", n_t)
    n_chk = min(n_t, args.steps * 10)
    t128, obs128 = evolve("c128", n_chk)
    dev_max = max(float(np.max(np.abs(obs64[k][: n_chk + 1] - obs128[k]))) for k in ops)
    # the same complex64 evolution on the CSR matvec, for comparison
    evolve("c64", 2, "csr")
    t64c, obs64c = evolve("c64", n_chk, "csr")
    dev_csr = max(float(np.max(np.abs(obs64[k][: n_chk + 1] - obs64c[k]))) for k in ops)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "workload": "quench", "value": n_t / (t64 * 1e-3), "unit": "time_steps/s",
            "n_gpus": world, "steps": n_t, "warmup": 1, "ms_per_step": t64 / n_t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex64 Krylov + f64 recurrence",
            "data": "synthetic (model Hamiltonian)",
            "config": {"workload": f"SU(2) 1D L=16 OBC, static pair at sites 5,10, dim {len(model.sector)}, "
                                   f"nnz {model.H.mat.nnz}; t in [0,{T}], dt={dt}, m_krylov=30",
                       "c128_check_steps": n_chk},
            "c128_ms_per_step": t128 / max(n_chk, 1),
            "max_observable_deviation_c64_vs_c128": dev_max,
            "matvec_layout": layout[("c64", "auto")],
            "c64_csr_ms_per_step": t64c / max(n_chk, 1),
            "max_observable_deviation_c64_layout_vs_csr": dev_csr,
        }), flush=True)


def run_corr(args, world, rank, local):
    """Two-body correlator matrices (TwoBodyTerm.get_expval) in the SU(2) 1D
    L=16 OBC sector with a j=1/2 static pair at sites 5 and 10 (dim
    7,133,222): one step is <N_pair_i N_pair_j> and <T2_px_i T2_px_j> over all
    120 site pairs on a seeded, normalised complex128 state."""
    import torch

    from edgpu.models import SU2_Model
    from edgpu.models.quantum_model import twobody_corr_device

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bg = [0] * 5 + [0.5] + [0] * 4 + [0.5] + [0] * 5
    model = SU2_Model(spin=0.5, pure_theory=False, lvals=[16], has_obc=[True], sectors=[16], bg_list=bg, device=dev)
    n = len(model.sector)
    gen = torch.Generator(device=dev).manual_seed(1234 + rank)
    psi = torch.randn(n, dtype=torch.complex128, device=dev, generator=gen)
    psi /= torch.linalg.vector_norm(psi)
    names = [("N_pair", "N_pair"), ("T2_px", "T2_px")]
    ops = [(model.ops[a], model.ops[b]) for a, b in names]
    n_pairs = 16 * 15 // 2

    def step(x):
        return [twobody_corr_device(model.sector, oa, ob, x) for oa, ob in ops]

    for _ in range(args.warmup):
        step(psi)
    torch.cuda.synchronize()
    barrier(world)
    clock = ClockSampler(local)
    clock.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    a0, b0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for k in range(args.steps):
        evs[k][0].record()
        out = step(psi)
        evs[k][1].record()
    b0.record()
    torch.cuda.synchronize()
    clocks = clock.stop()
    barrier(world)
    ms = max_over_ranks(a0.elapsed_time(b0) / args.steps, world, dev)
    per_launch = float(np.mean([e[0].elapsed_time(e[1]) for e in evs])) / len(ops)
    corr = [c.cpu().numpy() for c in out]
    # e2e: pinned host state in, both correlator matrices out, every step
    host = psi.cpu().pin_memory()
    outs = [torch.empty((16, 16), dtype=torch.float64).pin_memory() for _ in ops]
    torch.cuda.synchronize()
    a1, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a1.record()
    for _ in range(args.steps):
        x = host.to(dev, non_blocking=True)
        for o, c in zip(outs, step(x)):
            o.copy_(c, non_blocking=True)
    b1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(a1.elapsed_time(b1) / args.steps, world, dev)
    # parity on a sample of pairs: the oracle on the same state
    from oracle import edlgt_oracle as O

    cfg = model.sector_configs
    psi_h = psi.cpu().numpy()
    t0 = time.perf_counter()
    sample = [(0, 15), (7, 8)]
    dev_max = 0.0
    for i, j in sample:
        rows, cols, vals = O.nbody_triplets([ops[0][0], ops[0][1]], [i, j], cfg, model.loc_dims)
        ok = cols >= 0
        e = float(np.real(np.sum(np.conj(psi_h[rows[ok]]) * vals[ok] * psi_h[cols[ok]])))
        dev_max = max(dev_max, abs(e - corr[0][i, j]))
    cpu_s = time.perf_counter() - t0
    hbm, src = peaks()
    bytes_launch = n * (8 + 16)
    ach = bytes_launch / (per_launch * 1e-3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": "twobody_correlators", "workload": "corr", "value": world * n_pairs * len(ops) / (ms * 1e-3),
            "unit": "pair_correlators/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128 state, f64 accumulation", "data": "synthetic (seeded random normalised state)",
            "config": {"workload": f"SU(2) 1D L=16 OBC, static pair at sites 5,10, dim {n}; correlators "
                                   f"{['_'.join(x) for x in names]} over all {n_pairs} pairs",
                       "l2": "inputs larger than L2 (keys 57 MB + state 114 MB per launch)"},
            "ms_per_matrix": per_launch,
            "oracle_check": {"pairs": sample, "max_abs_dev": dev_max},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                         "traffic": None, "peak_source": src, "kernel": "twobody_k<2>",
                         "bytes_model": "per row: key 8 + complex128 amplitude 16, read once for all pairs"},
            "e2e": {"value": world * n_pairs * len(ops) / (e2e_ms * 1e-3), "unit": "pair_correlators/s",
                    "ms_per_step": e2e_ms, "h2d_bytes_per_step": int(host.nbytes),
                    "d2h_bytes_per_step": int(sum(o.nbytes for o in outs))},
            "cpu_baseline": {"value": len(sample) / cpu_s, "unit": "pair_correlators/s", "cores": 1, "kind": "port",
                             "sample": f"oracle two-site triplets + contraction for {len(sample)} pairs of N_pair"},
            "gpu_launches": 2 * len(ops),
            "clocks": clocks,
        }), flush=True)


def run_entropy(args, world, rank, local):
    """Half-chain entanglement in the SU(2) 1D L=14 periodic chain's N_tot=14
    sector (dim 1,232,454) of a seeded, normalised complex128 state: one step
    is the bipartition maps
    (QuantumModel._get_partition, both parts), the state matrix, rho = M M^dagger
    and its spectrum (QMB_state.entanglement_entropy)."""
    import torch

    from edgpu.entanglement import entanglement_entropy, get_partition
    from edgpu.models import SU2_Model

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    model = SU2_Model(**model_kwargs(), device=dev)
    n = len(model.sector)
    gen = torch.Generator(device=dev).manual_seed(4321 + rank)
    psi = torch.randn(n, dtype=torch.complex128, device=dev, generator=gen)
    psi /= torch.linalg.vector_norm(psi)
    keep = tuple(range(7))

    def step():
        cache = {keep: get_partition(model.sector, model.n_sites, keep)}
        t1 = torch.cuda.Event(enable_timing=True)
        t1.record()
        s = entanglement_entropy(psi, keep, cache)
        return s, cache[keep], t1

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clock = ClockSampler(local)
    clock.start()
    a0, b0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    spec_ms = []
    a0.record()
    for _ in range(args.steps):
        s, part, t1 = step()
        t2 = torch.cuda.Event(enable_timing=True)
        t2.record()
        torch.cuda.synchronize()
        spec_ms.append(t1.elapsed_time(t2))
    b0.record()
    torch.cuda.synchronize()
    clocks = clock.stop()
    barrier(world)
    ms = max_over_ranks(a0.elapsed_time(b0) / args.steps, world, dev)
    # the oracle on the same state: maps and entropy
    from oracle import edlgt_oracle as O

    cfg = model.sector_configs
    psi_h = psi.cpu().numpy()
    t0 = time.perf_counter()
    ref = O.partition(cfg, model.loc_dims, keep)
    s_ref = O.entanglement_entropy(psi_h, ref)
    cpu_s = time.perf_counter() - t0
    maps_ok = bool(np.array_equal(ref["subsys_map"], part["subsys_map"]) and
                   np.array_equal(ref["env_map"], part["env_map"]))
    if rank == 0:
        print(json.dumps({
            "metric": "entanglement_entropy", "workload": "entropy", "value": world / (ms * 1e-3),
            "unit": "entropies/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128 state and matrix, f64 spectrum", "data": "synthetic (seeded random normalised state)",
            "config": {"workload": f"SU(2) 1D L={L} {'periodic' if PBC else 'open'} chain, N_tot={L} sector, dim {n}; "
                                   "subsystem sites 0-6 "
                                   f"({part['subsys_dim']} x {part['env_dim']} state matrix)"},
            "phase_ms": {"maps_and_matrix": ms - float(np.mean(spec_ms)), "rho_and_spectrum": float(np.mean(spec_ms))},
            "oracle_check": {"maps_bit_exact": maps_ok, "abs_dS": abs(s - s_ref), "entropy": s},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "entropies/s", "cores": 1, "kind": "port",
                             "sample": "oracle partition (np.unique on packed keys) + dense SVD of the state matrix"},
            "gpu_launches": 19,  # per step: 2 x (mark, popcount, 4 scan, rank, list, decode) + state matrix
            "clocks": clocks,
        }), flush=True)


def run_momentum(args, world, rank, local):
    """Zero-momentum sector of the SU(2) 1D L=14 PBC chain (N_tot = 14 sector,
    dim 1,232,454; unit cell 1): one step builds the projector B on the
    device and finds the ground state of B^dagger H B by Lanczos on the
    matrix-free projected matvec (g^2 = 1, m = 0.5)."""
    import torch

    from edgpu.models import SU2_Model

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    model = SU2_Model(spin=0.5, pure_theory=False, lvals=[14], has_obc=[False], sectors=[14], device=dev)
    model.build_Hamiltonian(1.0, 0.5)
    n = len(model.sector)

    def step():
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        model.set_momentum_sector([1], [0])
        b.record()
        model.diagonalize_Hamiltonian(1, tol=1e-10)
        c.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b), b.elapsed_time(c)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clock = ClockSampler(local)
    clock.start()
    t_basis, t_solve = [], []
    a0, b0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for _ in range(args.steps):
        tb, ts = step()
        t_basis.append(tb)
        t_solve.append(ts)
    b0.record()
    torch.cuda.synchronize()
    clocks = clock.stop()
    barrier(world)
    ms = max_over_ranks(a0.elapsed_time(b0) / args.steps, world, dev)
    e_k0 = float(model.H.Nenergies[0])
    m_cols = model._momentum.n_cols
    matvecs = model._momentum.last_matvecs
    # the full-sector ground state beside it (B has orthonormal columns: E_k0 >= E_full)
    model._momentum = None
    model.diagonalize_Hamiltonian(1, tol=1e-10)
    e_full = float(model.H.Nenergies[0])
    from oracle import edlgt_oracle as O

    cfg = model.sector_configs
    t0 = time.perf_counter()
    cp, _, _, n_cols_cpu = O.momentum_basis(cfg, model.loc_dims, [14], [1], [0])
    cpu_s = time.perf_counter() - t0
    if rank == 0:
        print(json.dumps({
            "metric": "momentum_ground_states", "workload": "momentum", "value": world / (ms * 1e-3),
            "unit": "ground_states/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128 momentum vectors, f64 sector matrix", "data": "synthetic (model Hamiltonian)",
            "config": {"workload": f"SU(2) 1D L=14 PBC, N_tot=14 sector dim {n}, unit cell 1, k=0: "
                                   f"{m_cols} momentum states; g^2=1, m=0.5"},
            "phase_ms": {"basis": float(np.mean(t_basis)), "solve": float(np.mean(t_solve))},
            "energy_density_k0": e_k0, "energy_density_full_sector": e_full,
            "oracle_check": {"n_cols_match": int(n_cols_cpu) == int(m_cols)},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "bases/s", "cores": 1, "kind": "port",
                             "sample": "oracle momentum projector (translations, references, Bloch sums) only"},
            # per step: basis 14 (translations, references + scan + list, column count + scan + fill,
            # row map), solve 3 per projected matvec (expand, sector matvec, reduce)
            "gpu_launches": 14 + 3 * int(matvecs),
            "clocks": clocks,
        }), flush=True)


Z3_G = tuple(float(g) for g in np.geomspace(0.7, 1.6, 8))
Z3_MASS = 0.5


def largest_config(dev, warmup=2):
    """The largest configuration: 2D Z3 lattice gauge theory with staggered
    matter on the 4x3 periodic lattice, Gauss law + zero charge + zero
    momentum (245,518,920 representatives of 1,473,154,452 Gauss-law
    states), matrix-free; 8 couplings g in geomspace(0.7, 1.6, 8), t = 1,
    m = 0.5, batched.  Mixed-precision time-to-solution (f32 thick-restart
    Lanczos + f64 refinement) and the plain f64 solver's, both on this GPU,
    plus the batched matvec timed alone.  Returns a dict."""
    import torch

    from edgpu.models.zn_model import ZnModel

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    model = ZnModel((4, 3), 3, momentum=True, device=dev)
    eng = model.engine
    cp = model.build_Hamiltonian(np.array(Z3_G), Z3_MASS)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    nvec = 8
    coup = torch.from_numpy(np.ascontiguousarray(cp)).to(dev)
    n = eng.n_rows
    mv = {}
    for dt in (torch.float32, torch.float64):
        x = torch.rand((n, nvec), dtype=dt, device=dev)
        y = torch.empty_like(x)
        for _ in range(warmup):
            eng.matvec(x, y, coup, nvec)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(3):
            eng.matvec(x, y, coup, nvec)
        b.record()
        b.synchronize()
        mv[dt] = a.elapsed_time(b) / 3
        del x, y
    # images per row: hops across links with unequal occupations + 2 per plaquette
    L = eng.L
    occ = (eng.keys[:n] >> L.field_bits) & ((1 << L.n_sites) - 1)
    hops = torch.zeros(n, dtype=torch.int64, device=dev)
    for l in range(L.n_links):
        hops += ((occ >> int(L.link_from[l])) ^ (occ >> int(L.link_to[l]))) & 1
    images = float(hops.double().mean().item()) + 2 * L.n_sites
    del occ, hops
    torch.cuda.empty_cache()
    res_mixed = model.diagonalize_Hamiltonian(1, precision="mixed")
    e_mixed = res_mixed.evals[:, 0].copy()
    res_mixed.evecs = None  # free the f64 vectors for the f64 solver's basis
    res64 = model.diagonalize_Hamiltonian(1, precision="fp64")
    e64 = res64.evals[:, 0].copy()
    res64.evecs = None
    t_mixed, t64 = res_mixed.stats["total_ms"], res64.stats["total_ms"]
    hbm, src = peaks()
    # compulsory bytes of one batched matvec (matrix-free): keys + x + y
    comp32 = n * (8 + 2 * 4 * nvec)
    comp64 = n * (8 + 2 * 8 * nvec)
    # with the gathers: per row its own orbit entry; per image an orbit entry
    # and an x row
    gath32 = comp32 + n * 4 + n * images * (4 + 4 * nvec)
    out = {
        "workload": f"Z3 LGT + staggered matter, 4x3 periodic, Gauss law + zero charge + zero momentum, {n} rows "
                    f"({L.n_gauss} Gauss-law states), matrix-free; g in {[round(g, 4) for g in Z3_G]}, t=1, "
                    f"m={Z3_MASS}; 8 ground states",
        "rows": n, "setup_s": setup_s, "basis_build_ms": eng.build_ms,
        "mixed_ms": t_mixed, "fp64_ms": t64, "speedup_mixed_vs_fp64": t64 / t_mixed,
        "ground_states_per_s_mixed": nvec / (t_mixed * 1e-3),
        "max_rel_dE_mixed_vs_fp64": float(np.max(np.abs(e_mixed - e64) / np.abs(e64))), "target": 1e-9,
        "energies_mixed": e_mixed.tolist(), "energies_fp64": e64.tolist(),
        "solver_mixed": {k: res_mixed.stats[k] for k in ("m", "k_keep", "matvecs32", "cycles32", "matvecs64",
                                                          "cycles64", "phase1_ms", "phase2_ms", "matvec_ms",
                                                          "reorth_ms")},
        "solver_fp64": {k: res64.stats[k] for k in ("m", "k_keep", "matvecs64", "cycles64", "matvec_ms",
                                                     "reorth_ms")},
        "matvec": {"kernel": "zn_matvec_k<3, T, 8>", "ms_f32_x8": mv[torch.float32], "ms_f64_x8": mv[torch.float64],
                   "images_per_row": images,
                   "compulsory_bytes_f32": comp32, "compulsory_GBps_f32": comp32 / (mv[torch.float32] * 1e-3) / 1e9,
                   "compulsory_frac_f32": comp32 / (mv[torch.float32] * 1e-3) / 1e9 / hbm,
                   "compulsory_bytes_f64": comp64, "compulsory_frac_f64": comp64 / (mv[torch.float64] * 1e-3) / 1e9 / hbm,
                   "with_gathers_bytes_f32": gath32,
                   "with_gathers_frac_f32": gath32 / (mv[torch.float32] * 1e-3) / 1e9 / hbm,
                   "peak": hbm, "peak_source": src,
                   "bytes": "compulsory = rows x (8 key + 32 x + 32 y) [f32 x8]; with gathers adds the row's own "
                            "4-byte orbit entry and, per image, a 4-byte orbit entry and a 32-byte x row"},
        "cpu_baseline": None,
        "cpu_baseline_note": "no CPU reference at this size: ed-lgt has no Z3 model with matter and its int32 "
                             "triplets overflow here; the oracle covers lattices up to 4x2",
    }
    del model, eng, coup, res_mixed, res64
    torch.cuda.empty_cache()
    return out


def run_z3(args, world, rank, local):
    """The largest configuration on its own line (see largest_config)."""
    import torch

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    clock = ClockSampler(local)
    clock.start()
    blk = largest_config(dev, args.warmup)
    clocks = clock.stop()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "workload": "z3", "value": blk["ground_states_per_s_mixed"] * world,
            "unit": "ground_states/s", "n_gpus": world, "steps": 1, "warmup": args.warmup,
            "ms_per_step": blk["mixed_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 Krylov/matvec + f64 dots, recurrence, refinement",
            "data": "synthetic (model Hamiltonian; no reference run exists for Z3 with matter)",
            "config": {"workload": blk["workload"]}, "largest_config": blk, "clocks": clocks,
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)  # ~0.8 s timed: several 200 ms clock samples
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="edgpu", choices=["edgpu", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-largest", action="store_true",
                    help="skip the largest-configuration block (Z3 4x3, about 6 minutes; run at N=1 only)")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "batch", "quench", "z3", "corr", "entropy", "momentum"],
                    help="sweep: SU(2) L=14 coupling sweep (the headline); batch: QED 3x2 instance batch; "
                         "quench: SU(2) L=16 Krylov dynamics; z3: Z3 4x3 zero-momentum matrix-free batch; "
                         "corr: SU(2) L=16 two-body correlator matrices; entropy: SU(2) L=14 half-chain entanglement; "
                         "momentum: SU(2) L=14 PBC zero-momentum ground state")
    ap.add_argument("--quench-time", type=float, default=20.0)
    ap.add_argument("--matvec-layout", default="auto", choices=["auto", "sell", "csr", "packed"],
                    help="f32 matvec layout of the headline solve; auto = the autotuner's choice")
    ap.add_argument("--sell-window", type=int, default=32, help="SELL sort window with --matvec-layout sell")
    ap.add_argument("--spmv-group", type=int, default=0,
                    help="matvec threads per row (2/4/8/16/32); 0 = autotune before the timed region")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.workload == "batch":
            run_batch(args, world, rank, local)
        elif args.workload == "quench":
            run_quench(args, world, rank, local)
        elif args.workload == "z3":
            run_z3(args, world, rank, local)
        elif args.workload == "corr":
            run_corr(args, world, rank, local)
        elif args.workload == "entropy":
            run_entropy(args, world, rank, local)
        elif args.workload == "momentum":
            run_momentum(args, world, rank, local)
        else:
            run_edgpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
