"""UW12 energy + Fock benchmark: split precision + adjoint vs FP64 (one JSON line
on rank 0).

Workload (default ``--config c1``): N=500 AO, M=1500 DF, R=2000 RI, UHF with
n_alpha=40, n_beta=38, all-electron, scale factors (1.0, 0.5) -- the largest
benchmark configuration whose inputs (28.6 GB) fit one GPU; the N=1200 one
(395 GB of inputs) runs integral-direct with ``--config c2 --direct``.
Seeded synthetic inputs (libuw12_b200.workload: three-index N(0,1)
exp(-|m-n|/30), metrics B B^T + 1e-6 I, S-orthonormal orbitals), generated
once on the host; the reference arm generates the identical bytes.

One step = the metric's subject: energy + Fock (dE/dD) and the gradient of
the energy with respect to every stored integral (dE/d(P|mn) of W, V, WV,
dE/d(P_ri|mn) of W, V, dE/d(P|Q) of W, V, WV), same-spin terms included, with
every large contraction in split precision (int8 tensor-core residue products,
``--moduli`` moduli, default 14: FP64-level accuracy).

* ``value``: s/step with the integrals resident in HBM and the gradients
  written to device buffers (CUDA events on the library's stream around
  exactly ``--steps`` steps after ``--warmup`` untimed ones; no profiling in
  the timed loop; max over ranks).  Inputs exceed the 126 MB L2.
* ``fp64``: the same step in FP64 (DMMA tensor cores), ``speedup`` = FP64 /
  split, and the split result's error against it (energy in Eh and relative,
  Fock and every gradient relative); ``fp64_forward``: energy + Fock only,
  the plain libuw12 computation in FP64.
* ``roofline``: the dominant kernel of the step (``k_i8_mma``, int8
  tcgen05.mma) from a separate profiled step; ``roofline_fp64`` the FP64 GEMM
  kernel of the forward pass.
* ``e2e``: the same step through the public API from pinned host buffers:
  integral upload, metric and overlap eigensolves, forward + backward, Fock and
  all gradients read back to pinned host memory, per step.
* ``cpu_baseline``: libuw12 itself (its unmodified sources compiled by
  oracle/ref.mk, OpenMP on every host core) on the same inputs: one
  sampled evaluation of energy + Fock (libuw12 has no adjoint), every loop
  over aux functions or orbital pairs timed on a sample of its iterations and
  extrapolated (oracle/refshim/timing/utils/parallel.hpp; checked against full
  evaluations by oracle/validate_sampler.py).

With N > 1 ranks every rank evaluates its own copy (replicas; ``value`` =
max-over-ranks time / (steps x ranks)).  ``--impl reference`` runs the
reference arm alone on rank 0: warm-up steps on the c0 system plus one
priming evaluation, then ``--steps`` rotated samples of the workload (each
measures every ``--ref-rotation``-th loop, the others at their last
estimate).  ``--gemm m,n,k[,beta]`` times one GEMM shape instead;
``--batched`` adds the 64-molecule batch.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

# The CPU baseline (libuw12 from its own sources) calls BLAS inside its OpenMP
# loops, one BLAS call per thread: its BLAS runs single-threaded, which has to
# be set before any BLAS library of this process is loaded (the sampler's
# validation, oracle/validate_sampler.py, runs the same way).
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "UW12 energy+Fock s/eval: split-prec+adjoint vs FP64 GPU at |ΔE|≤1e-6 Eh; TFLOP/s"
SEED = 11


# --------------------------------------------------------------------------
# canonical FLOPs (algorithmic work of one forward evaluation, dense GEMMs)
# --------------------------------------------------------------------------
def canonical_flops(N, M, R, occ, act, same_spin=True, fock=True):
    Rp = N + R
    Np = N * (N + 1) // 2
    tot = 0.0
    for o, a in zip(occ, act):
        f = 2 * (2 * N * N * o * M + 2 * N * o * M * M)          # T1, W and V
        f += 2 * (2 * R * N * a * M + 2 * R * a * M * M)         # T2
        f += 2 * (2 * a * N * o * M)                             # T3
        f += 4 * Np * M                                          # 2-el direct
        f += 2 * M * M * a * o                                   # 4-el t
        f += 2 * Rp * Rp * a * M + 2 * M * M * Rp * a            # 3-el X_AB
        if fock:
            f += 2 * N * o * M * M + 2 * N * N * o * M + (2 * N * N * a * M if a < o else 0)
            f += 2 * N * o * M * M + 2 * N * N * o * M + (2 * N * N * a * M if a < o else 0)
            f += 4 * M ** 3 + 2 * (Np + R * N) * M * M + 2 * Rp * Rp * N * M + 2 * N * N * Rp * M
        if same_spin:
            f += 4 * N * N * a * M + 2 * N * a * M * M + 2 * a * a * N * M
            f += 4 * (a * o) ** 2 * M + (4 * N * o * a * o * M + 2 * N * N * a * a * o
                                          + (2 * N * N * o * o * a if a < o else 0) if fock else 0)
            f += 4 * Rp * a * a * o * M + 2 * Rp * a * a * o
            if fock:
                f += 2 * Rp * Rp * a * M + 2 * (4 * N * Rp * a * o * M + 2 * N * N * Rp * a * o
                                                 + 2 * a * o * M * M)
                f += 4 * Rp * a * a * N * M + 2 * N * N * Rp * a * a
        tot += f
    return float(tot)


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# peaks measured in the run (MEASURED_PEAKS.json has no FP64 or int8 figure)
# --------------------------------------------------------------------------
def _best_of(fn, reps=5):
    import torch
    for _ in range(2):
        fn()
    best = 1e30
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return best


def fp64_peak_tflops(device) -> float:
    """cuBLAS DGEMM 8192^3 burst (best of 5)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    t = _best_of(lambda: a @ b)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / t / 1e12


def int8_peak_tops(device):
    """Dense int8 tensor-core throughput of a library GEMM (torch._int_mm, 8192^3,
    best of 5); (value, source).  Without an int8 library GEMM: twice the
    measured bf16 peak, else twice the 1.59 PFLOP/s bf16 fallback."""
    import torch
    n = 8192
    try:
        a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=device)
        b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=device)
        t = _best_of(lambda: torch._int_mm(a, b))
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / t / 1e12, "torch._int_mm int8 8192^3 burst measured in this run"
    except Exception as exc:
        p = ROOT / "MEASURED_PEAKS.json"
        if p.exists():
            return (2.0 * json.loads(p.read_text())["bf16_tflops"],
                    f"2 x MEASURED_PEAKS bf16 burst ({type(exc).__name__})")
        return 2.0 * 1590.0, f"2 x 1.59 PFLOP/s bf16 fallback ({type(exc).__name__})"


def read_traffic(name: str, key: str):
    """Per-unit DRAM traffic of a kernel from its committed ncu summary."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


# --------------------------------------------------------------------------
# inputs
# --------------------------------------------------------------------------
def workload_of(args):
    from libuw12_b200 import workload as WL
    return WL.CONFIGS[args.config]


def config_dict(args):
    """The workload (identical in both arms)."""
    w = workload_of(args)
    return {"workload": f"uw12 {args.config}: N={w.n_ao} AO, M={w.n_df} DF, R={w.n_ri} RI, "
                        f"n_occ={list(w.n_occ)} "
                        f"({'UHF' if w.n_spin == 2 else 'closed shell'}), all-electron, "
                        f"scales (s_os, s_ss)=({args.s_os}, {args.s_ss})",
            "n_ao": w.n_ao, "n_df": w.n_df, "n_ri": w.n_ri, "n_occ": list(w.n_occ),
            "decay": w.decay, "seed": SEED, "s_os": args.s_os, "s_ss": args.s_ss,
            "inputs": "counter-based seeded generators (libuw12_b200.workload == oracle.synth, "
                      "identical bytes in both arms)",
            "l2": "inputs exceed the 126 MB L2 (no flush needed)"}


def host_inputs(w, pinned: bool):
    """Three-index tensors (in pinned host memory when asked, filled in place)
    and the small inputs, all from the seeded generators."""
    from libuw12_b200 import workload as WL
    h = WL.make_small(w, SEED)
    if pinned:
        import torch
    for nm in WL.THREE_INDEX:
        rows, cols = WL.tensor_shape(w, nm)
        if pinned:
            t = torch.empty(rows * cols, dtype=torch.float64, pin_memory=True)
            h["_pinned_" + nm] = t
            buf = t.numpy()
        else:
            buf = np.empty(rows * cols)
        WL.make_three_index(w, nm, SEED, out=buf)
        h[nm] = buf.reshape((rows, cols), order="F")
    return h


def reference_inputs(w):
    """The workload's inputs from the oracle's generators (oracle/synth.py): the
    same formulas, element for element, as libuw12_b200.workload, so the
    reference arm evaluates the GPU arm's bytes (tests/test_workload.py)."""
    from oracle import synth as S
    N, M, R = w.n_ao, w.n_df, w.n_ri
    h = {nm: S.three_index_ao(SEED, nm, N, M, w.decay) for nm in ("W3", "V3", "WV3")}
    h.update({nm: S.three_index_ri(SEED, nm, N, R, M, w.decay) for nm in ("W3_ri", "V3_ri")})
    h.update({nm: S.metric(SEED, nm, M) for nm in ("W2", "V2", "WV2")})
    h["S"] = S.overlap(SEED, N, R)
    h["orbitals"] = [S.orbitals(SEED, h["S"][:N, :N], max(o, 1), f"C{s}")[:, :max(o, 1)]
                     for s, o in enumerate(w.n_occ)]
    per = 2.0 if w.n_spin == 1 else 1.0
    h["occ"] = [np.full(o, per) for o in w.n_occ]
    return h


# --------------------------------------------------------------------------
# CPU baseline: libuw12 itself, sampled (timing build of oracle/ref.mk)
# --------------------------------------------------------------------------
def cpu_reference_problem(w, h):
    from oracle import ref_lib as R
    if not R.available(timing=True):
        R.build()
    cores = os.cpu_count() or 1
    R.set_threads(cores, 1, timing=True)
    p = R.RefProblem(h["W3"], h["W2"], h["W3_ri"], h["V3"], h["V2"], h["V3_ri"], h["WV3"],
                     h["WV2"], h["S"], w.n_ao, w.n_df, w.n_ri, timing=True)
    return p, cores


def cpu_reference_args(w, h, s_os, s_ss):
    n_orb = max(max(o.shape[1] for o in h["orbitals"]), 1)
    C = np.asfortranarray(np.concatenate(
        [np.concatenate([o, np.zeros((w.n_ao, n_orb - o.shape[1]))], axis=1)
         for o in h["orbitals"]], axis=1))
    return (C, n_orb, w.n_spin, np.concatenate(h["occ"]), list(w.n_occ), list(w.n_occ), s_os,
            s_ss)


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, rank, world):
    """The reference arm: libuw12 (timing build) on the host cores, rank 0 only."""
    if rank != 0:
        return
    from oracle import ref_lib as R, synth
    w = workload_of(args)
    t0 = time.perf_counter()
    h = reference_inputs(w)
    t_gen = time.perf_counter() - t0
    p, cores = cpu_reference_problem(w, h)
    a = cpu_reference_args(w, h, args.s_os, args.s_ss)
    del h
    # warm-up: the c0 system, then one priming sample of the workload
    c0 = synth.Config("c0", 24, 84, 116, (5,), 8.0)
    i0 = synth.make_inputs(c0, SEED)
    p0 = R.RefProblem.from_inputs(i0, timing=True)
    for _ in range(args.warmup):
        p0.evaluate(i0.C, i0.n_orb, 1, i0.occ, [5], [5], args.s_os, args.s_ss)
    p0.close()
    S = max(1, args.ref_rotation)
    prime = p.timed_evaluate(1, *a, rotation=S, phase=0)
    ests, walls = [], []
    for k in range(args.steps):
        est, sec, nloops, _ = p.timed_evaluate(1, *a, rotation=S, phase=(k + 1) % S)
        ests.append(est)
        walls.append(sec)
    value = float(statistics.median(ests))
    sample = (f"{args.config} energy + Fock (libuw12 has no adjoint), libuw12's unmodified "
              f"sources (oracle/ref.mk, OpenMP, BLAS single-threaded inside its loops); every "
              f"top-level loop over aux functions / orbital pairs sampled on every thread at "
              f"once (the first two iterations of its static-schedule block, the rest at the "
              f"warm iteration's time; the loop as its slowest block), loops "
              f"rotated over {S} steps (each step measures every {S}-th loop, the others at "
              f"their last estimate; primed by one full sample of {prime[1]:.1f} s); value = "
              f"median of {args.steps} step estimates (min {min(ests):.0f}, max "
              f"{max(ests):.0f} s); wall time per step {statistics.median(walls):.1f} s; "
              f"setup (deep copies + metric and overlap eigensolves, {p.setup_seconds:.1f} s) "
              f"and input generation ({t_gen:.1f} s) excluded")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s/eval",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators, the GPU arm's inputs byte for byte)",
        "config": config_dict(args),
        "cpu_baseline": {"value": value, "unit": "s/eval", "cores": cores, "kind": "reference",
                         "cpu_model": cpu_model(), "sample": sample},
        "e2e": {"value": value, "unit": "s/eval", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step_estimates_s": ests,
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GEMM probe
# --------------------------------------------------------------------------
def gemm_probe(args):
    """One GEMM shape on both paths: `--warmup` untimed and `--steps` timed calls
    each, CUDA events on the library's stream, kernel-class times of the split
    path (one JSON line)."""
    import torch
    import libuw12_b200 as L
    dims = [int(x) for x in args.gemm.split(",")]
    m, n, k = dims[:3]
    beta = float(dims[3]) if len(dims) > 3 else 0.0
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    L.lib()
    stream = torch.cuda.current_stream(device)
    L.set_stream(stream.cuda_stream)
    g = torch.Generator(device=device)
    g.manual_seed(3)
    A = torch.randn(m * k, dtype=torch.float64, device=device, generator=g)
    B = torch.randn(k * n, dtype=torch.float64, device=device, generator=g)
    C = torch.zeros(m * n, dtype=torch.float64, device=device)
    gargs = (m, n, k, 1.0, A.data_ptr(), m, False, B.data_ptr(), k, False, beta, C.data_ptr(), m)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        return e0.elapsed_time(e1) / args.steps

    flops = 2.0 * m * n * k
    out = {"gemm": [m, n, k], "beta": beta, "fp64_ms": timed(lambda: L.dgemm(*gargs))}
    out["fp64_tflops"] = flops / out["fp64_ms"] / 1e9
    Lm = args.moduli
    for _ in range(args.warmup):
        L.dgemm_split(*gargs, n_moduli=Lm)
    torch.cuda.synchronize(device)
    L.profile_enable(True)
    out[f"split{Lm}_ms"] = timed(lambda: L.dgemm_split(*gargs, n_moduli=Lm))
    n_calls = args.steps + args.warmup
    for kind in ("i8_mma", "split_prep", "split_crt"):
        r = L.profile_read_kind(kind)
        out[f"split{Lm}_{kind}"] = {"ms_per_call": r["ms"] / n_calls,
                                    "work_per_s": r["work"] / (r["ms"] / 1e3) if r["ms"] else None}
    L.profile_enable(False)
    out["speedup"] = out["fp64_ms"] / out[f"split{Lm}_ms"]
    # accuracy of one split call against the FP64 kernel (same C on input)
    C0 = torch.randn(m * n, dtype=torch.float64, device=device, generator=g)
    C.copy_(C0)
    L.dgemm(*gargs)
    ref = C.clone()
    C.copy_(C0)
    L.dgemm_split(*gargs, n_moduli=Lm)
    torch.cuda.synchronize(device)
    out[f"split{Lm}_max_rel_err"] = float((C - ref).abs().max() / ref.abs().max())
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------
# 64-molecule batch (--batched)
# --------------------------------------------------------------------------
def batched_report(L, args, moduli):
    import torch
    from libuw12_b200 import workload as WL
    mols = []
    for w, seed in WL.batch_molecules():
        sm = WL.make_small(w, seed)
        t3 = {nm: WL.make_three_index(w, nm, seed) for nm in WL.THREE_INDEX}
        mols.append({"W": L.setup_base_integrals(t3["W3"], sm["W2"], t3["W3_ri"]),
                     "V": L.setup_base_integrals(t3["V3"], sm["V2"], t3["V3_ri"]),
                     "WV": L.setup_base_integrals(t3["WV3"], sm["WV2"]),
                     "abs": L.setup_abs_projectors(sm["S"], w.n_ao, w.n_ri),
                     "orbitals": sm["orbitals"], "occ": sm["occ"], "n_active": list(w.n_occ),
                     "n_ao": w.n_ao})
    indirect = abs(args.s_ss) > 4 * np.finfo(float).eps
    out = {"workload": "64 molecules, N ~ U[20,300], M = 3N, R = 4N, n_occ = round(N/10), half "
                       "closed shell, half UHF (n_beta = n_alpha - 1), energy + Fock",
           "n_ao_range": [min(m["n_ao"] for m in mols), max(m["n_ao"] for m in mols)]}
    for n_streams in (1, 8):
        L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=n_streams)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.batched_steps):
            L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=n_streams)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.batched_steps
        out[f"s_per_batch_{n_streams}_streams"] = dt
    ref = L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
    # split-K autotuner: one batch on one stream tunes every new GEMM class
    # (timed, so not counted), then the batch runs from the table
    L.autotune_clear()
    L.autotune(L.AUTOTUNE_TUNE)
    t0 = time.perf_counter()
    L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t0
    L.autotune(L.AUTOTUNE_USE)
    tuned = {"classes": L.autotune_size(), "tuning_batch_s": tune_s}
    for n_streams in (1, 8):
        L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=n_streams)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.batched_steps):
            res = L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=n_streams)
        torch.cuda.synchronize()
        tuned[f"s_per_batch_{n_streams}_streams"] = (time.perf_counter() - t0) / args.batched_steps
    tuned["max_energy_rel_diff_vs_rule"] = max(abs(r[0] - q[0]) / abs(q[0])
                                               for r, q in zip(res, ref))
    L.autotune(L.AUTOTUNE_OFF)
    L.autotune_clear()
    out["autotuned_split_k"] = tuned
    L.set_precision(moduli)
    L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.batched_steps):
        res = L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
    torch.cuda.synchronize()
    L.set_precision(0)
    out["split"] = {"n_moduli": moduli,
                    "s_per_batch_1_stream": (time.perf_counter() - t0) / args.batched_steps,
                    "max_energy_rel_err_vs_fp64": max(abs(r[0] - q[0]) / abs(q[0])
                                                      for r, q in zip(res, ref))}
    for m in mols:
        for k in ("W", "V", "WV", "abs"):
            m[k].close()
    return out


# --------------------------------------------------------------------------
# main arm
# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c1s", "c2"])
    ap.add_argument("--s-os", dest="s_os", type=float, default=1.0)
    ap.add_argument("--s-ss", dest="s_ss", type=float, default=0.5)
    ap.add_argument("--moduli", type=int, default=14,
                    help="moduli of the split-precision products (14: FP64-level accuracy)")
    ap.add_argument("--extra-moduli", default="10",
                    help="further moduli counts reported beside the headline ('' = none)")
    ap.add_argument("--fp64-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-rotation", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--direct", action="store_true",
                    help="integral-direct: no three-index tensor stored, each regenerated on "
                         "the device by the library's synthetic producer at every use (inputs "
                         "larger than device memory, --config c2); three-index gradients "
                         "streamed in aux blocks to a squared-norm sink")
    ap.add_argument("--no-fp64-forward", action="store_true",
                    help="skip the FP64 energy + Fock arm")
    ap.add_argument("--no-profile", action="store_true",
                    help="skip the profiled pass (roofline and phase split)")
    ap.add_argument("--batched", action="store_true", help="add the 64-molecule batch")
    ap.add_argument("--batched-steps", type=int, default=2)
    ap.add_argument("--batched-only", action="store_true",
                    help="only the 64-molecule batch (FP64, autotuned split-K, split precision)")
    ap.add_argument("--gemm", default="",
                    help="instead of the workload: time one GEMM shape 'm,n,k[,beta]' on the "
                         "FP64 path and the split path with --moduli (kernel profiling probe)")
    args = ap.parse_args()
    if args.gemm:
        gemm_probe(args)
        return
    if args.direct:
        args.no_e2e = args.no_cpu_baseline = True

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=device)

    import libuw12_b200 as L
    from libuw12_b200 import workload as WL
    L.lib()
    stream = torch.cuda.current_stream(device)
    L.set_stream(stream.cuda_stream)
    if args.batched_only:
        if rank == 0:
            print(json.dumps({"batched": batched_report(L, args, args.moduli)}))
        return

    w = workload_of(args)
    N, M, R, occ = w.n_ao, w.n_df, w.n_ri, list(w.n_occ)
    act = list(occ)
    indirect = abs(args.s_ss) > 4 * np.finfo(float).eps
    t_gen = time.perf_counter()
    host = host_inputs(w, pinned=True) if not args.direct else WL.make_small(w, SEED)
    t_gen = time.perf_counter() - t_gen
    orbs, occs = host["orbitals"], host["occ"]
    fp64_peak = fp64_peak_tflops(device)
    i8_peak, i8_src = int8_peak_tops(device)

    # ---- handles with the integrals resident in HBM
    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order="F"))).to(device)

    small = {nm: dev(host[nm]) for nm in ("W2", "V2", "WV2", "S")}
    if args.direct:
        specs = {nm: L.SynthSpec(1 if nm.endswith("_ri") else 0, N, R, SEED, WL.tag(nm), w.decay)
                 for nm in WL.THREE_INDEX}
        fp = L.synth_producer()

        def produced(ao, ri, met):
            return L.setup_base_integrals_callback(
                small[met].data_ptr(), fp, fp if ri else None, n_ao=N, n_df=M,
                n_ri=R if ri else 0, store_ao=False, store_ri=False, device=True,
                user=ctypes.addressof(specs[ao]), user_ri=ctypes.addressof(specs[ri]) if ri else 0)

        W, V, WV = produced("W3", "W3_ri", "W2"), produced("V3", "V3_ri", "V2"), \
            produced("WV3", None, "WV2")
    else:
        def handle(x3, x2, x3ri):
            t3 = host["_pinned_" + x3].to(device, non_blocking=True)
            tri = host["_pinned_" + x3ri].to(device, non_blocking=True) if x3ri else None
            torch.cuda.synchronize(device)
            hd = L.setup_base_integrals(t3.data_ptr(), small[x2].data_ptr(),
                                        tri.data_ptr() if tri is not None else None, n_ao=N,
                                        n_df=M, n_ri=R if x3ri else 0, device=True)
            del t3, tri
            return hd

        W, V, WV = handle("W3", "W2", "W3_ri"), handle("V3", "V2", "V3_ri"), \
            handle("WV3", "WV2", None)
        torch.cuda.empty_cache()
    A = L.setup_abs_projectors(small["S"].data_ptr(), N, R, device=True)

    shapes = {"W3": (N * (N + 1) // 2, M), "V3": (N * (N + 1) // 2, M),
              "WV3": (N * (N + 1) // 2, M), "W3_ri": (R * N, M), "V3_ri": (R * N, M),
              "W2": (M, M), "V2": (M, M), "WV2": (M, M)}
    streamed = set(WL.THREE_INDEX) if args.direct else set()
    grad_bytes = int(sum(a * b for a, b in shapes.values()) * 8)

    def grad_buffers():
        return {k: torch.empty(a * b, dtype=torch.float64, device=device)
                for k, (a, b) in shapes.items() if k not in streamed}

    norms = torch.zeros(len(WL.THREE_INDEX), dtype=torch.float64, device=device)

    def step(gb):
        """energy + Fock + every gradient (device buffers / norm sinks)."""
        if not streamed:
            return L.fock_backward(W, V, WV, A, orbs, occs, act, args.s_os, args.s_ss,
                                   calculate_fock=True, indirect_term=indirect,
                                   device_out={k: b.data_ptr() for k, b in gb.items()})
        norms.zero_()
        e, f, t, mg = L.fock_backward_blocks(
            W, V, WV, A, orbs, occs, act, args.s_os, args.s_ss,
            {k: L.sink_norm2() for k in WL.THREE_INDEX}, calculate_fock=True, device=True,
            users={k: norms.data_ptr() + 8 * i for i, k in enumerate(WL.THREE_INDEX)},
            indirect_term=indirect)
        for k, v in mg.items():
            gb[k].copy_(torch.from_numpy(np.ascontiguousarray(v.reshape(-1, order="F"))))
        return e, f, t, {}

    def timed(fn, n_warm, n):
        for _ in range(n_warm):
            out = fn()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        if world > 1:
            dist.barrier()
        el = e0.elapsed_time(e1) / 1e3
        if world > 1:
            tt = torch.tensor([el], dtype=torch.float64, device=device)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el = float(tt.item())
        return el, out

    # ---- headline: split precision forward + adjoint, uninstrumented
    g_split = grad_buffers()
    L.set_precision(args.moduli)
    for _ in range(args.warmup):
        step(g_split)
    clocks = ClockSampler(local)
    clocks.start()
    n0 = L.launch_count()
    elapsed, (e_split, f_split, t_split, _) = timed(lambda: step(g_split), 0, args.steps)
    launches = L.launch_count() - n0
    clk = clocks.stop()
    norms_split = norms.clone()
    L.set_precision(0)
    value = elapsed / (args.steps * world)

    # ---- the same step in FP64, and the error of the split result against it
    g64 = grad_buffers()
    n64 = max(1, min(args.fp64_steps, args.steps))
    el64, (e64, f64, t64, _) = timed(lambda: step(g64), 1, n64)
    s64 = el64 / n64
    norms64 = norms.clone()

    def max_rel(a, b, chunk=1 << 26):
        d = max(float((a[i:i + chunk] - b[i:i + chunk]).abs().max())
                for i in range(0, a.numel(), chunk))
        r = max(float(b[i:i + chunk].abs().max()) for i in range(0, b.numel(), chunk))
        return d / r if r > 0 else d

    fs, fr = np.concatenate(f_split, axis=1), np.concatenate(f64, axis=1)
    accuracy = {"energy_fp64": e64, "energy_split": e_split,
                "energy_abs_err_Eh": abs(e_split - e64),
                "energy_rel_err": abs(e_split - e64) / abs(e64),
                "fock_max_rel_err": float(np.max(np.abs(fs - fr)) / np.max(np.abs(fr))),
                "gradient_max_rel_err": {k: max_rel(g_split[k], g64[k]) for k in g64}}
    if streamed:
        a_, b_ = norms_split.cpu().numpy(), norms64.cpu().numpy()
        accuracy["streamed_gradient_norm_rel_err"] = {
            k: abs(math.sqrt(a_[i]) - math.sqrt(b_[i])) / math.sqrt(b_[i])
            for i, k in enumerate(WL.THREE_INDEX)}
    del g64
    torch.cuda.empty_cache()

    # ---- FP64 forward only (energy + Fock: the plain libuw12 computation)
    fock_dev = torch.empty(N * N * len(occ), dtype=torch.float64, device=device)

    def forward():
        return L.form_fock(W, V, WV, A, orbs, occs, act, indirect, True, args.s_os, args.s_ss,
                           fock_out=fock_dev.data_ptr())[0]

    s_fwd, e_fwd = None, None
    if not args.no_fp64_forward:
        nf = max(1, min(3, args.steps))
        elf, e_fwd = timed(forward, 1, nf)
        s_fwd = elf / nf

    # ---- further moduli counts
    extra = []
    nx = max(1, min(3, args.steps))
    for Lm in [int(x) for x in args.extra_moduli.split(",") if x.strip()]:
        L.set_precision(Lm)
        elx, (ex, fx, _, _) = timed(lambda: step(g_split), 1, nx)
        L.set_precision(0)
        extra.append({"n_moduli": Lm, "s_per_step": elx / nx, "speedup_vs_fp64": s64 / (elx / nx),
                      "energy_abs_err_Eh": abs(ex - e64), "energy_rel_err": abs(ex - e64) / abs(e64),
                      "fock_max_rel_err": float(np.max(np.abs(np.concatenate(fx, axis=1) - fr)) /
                                                np.max(np.abs(fr)))})

    # ---- profiled pass (separate from every timed loop): kernel classes
    roofline = roofline_fp64 = phases_split = phases_fwd = None
    if not args.no_profile:
        L.set_precision(args.moduli)
        L.profile_enable(True)
        for kind in L.PROFILE_KINDS:
            L.profile_read_kind(kind)
        L.profile_phases()
        L.profile_read()
        step(g_split)
        torch.cuda.synchronize(device)
        kinds = {k: L.profile_read_kind(k) for k in L.PROFILE_KINDS}
        phases_split = L.profile_phases()
        L.set_precision(0)
        L.profile_read()
        forward()
        torch.cuda.synchronize(device)
        prof64 = L.profile_read()
        phases_fwd = L.profile_phases()
        L.profile_enable(False)
        i8 = kinds["i8_mma"]
        i8_tops = i8["work"] / (i8["ms"] / 1e3) / 1e12 if i8["ms"] else None
        bpg = read_traffic("i8_mma_traffic.txt", "traffic_bytes_per_gop")
        roofline = {"bound": "tensor", "kernel": "k_i8_mma (tcgen05.mma kind::i8, TMA-fed)",
                    "achieved": i8_tops, "peak": i8_peak, "unit": "TOPS",
                    "frac": i8_tops / i8_peak if i8_tops else None, "peak_source": i8_src,
                    "traffic": (bpg * i8["work"] / max(1, i8["launches"]) / 1e9) if bpg else None,
                    "launches": i8["launches"], "kernel_ms": i8["ms"],
                    "share_of_step": i8["ms"] / 1e3 / (elapsed / args.steps) if elapsed > 0 else None,
                    "ms_per_step_by_class": {"i8_mma": i8["ms"],
                                             "operand_prep": kinds["split_prep"]["ms"],
                                             "crt": kinds["split_crt"]["ms"],
                                             "fp64_dmma": kinds["dgemm"]["ms"],
                                             "producer": kinds["producer"]["ms"]}}
        gemm_tf = prof64["flops"] / (prof64["ms"] / 1e3) / 1e12 if prof64["ms"] > 0 else None
        bpg64 = read_traffic("dgemm_dmma_traffic.txt", "traffic_bytes_per_gflop")
        roofline_fp64 = {"bound": "tensor", "kernel": "dgemm_dmma (mma.sync m16n8k4 f64)",
                         "achieved": gemm_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": gemm_tf / fp64_peak if gemm_tf else None,
                         "peak_source": "cuBLAS DGEMM 8192^3 burst measured in this run",
                         "traffic": (bpg64 * prof64["flops"] / max(1, prof64["launches"]) / 1e9)
                         if bpg64 else None,
                         "launches": prof64["launches"], "kernel_ms": prof64["ms"],
                         "share_of_forward": prof64["ms"] / 1e3 / s_fwd if s_fwd else None}

    # ---- end to end through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        for hd in (W, V, WV, A):
            hd.close()
        del g_split
        torch.cuda.empty_cache()
        L.trim_memory()
        gh = {k: torch.empty(a * b, dtype=torch.float64, pin_memory=True)
              for k, (a, b) in shapes.items()}
        host_out = {k: t.numpy().reshape(shapes[k], order="F") for k, t in gh.items()}
        h2d = sum(host[nm].nbytes for nm in WL.THREE_INDEX) + \
            sum(host[nm].nbytes for nm in ("W2", "V2", "WV2", "S")) + sum(o.nbytes for o in orbs)
        d2h = grad_bytes + N * N * len(occ) * 8

        def e2e_step():
            We = L.setup_base_integrals(host["W3"], host["W2"], host["W3_ri"])
            Ve = L.setup_base_integrals(host["V3"], host["V2"], host["V3_ri"])
            WVe = L.setup_base_integrals(host["WV3"], host["WV2"])
            Ae = L.setup_abs_projectors(host["S"], N, R)
            r = L.fock_backward(We, Ve, WVe, Ae, orbs, occs, act, args.s_os, args.s_ss,
                                calculate_fock=True, indirect_term=indirect, host_out=host_out)
            for hd in (We, Ve, WVe, Ae):
                hd.close()
            return r[0]

        L.set_precision(args.moduli)
        ele, e_e2e = timed(e2e_step, 1, args.e2e_steps)
        L.set_precision(0)
        e2e = {"value": ele / (args.e2e_steps * world), "unit": "s/eval",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "includes": "H2D of all integrals from pinned host memory, metric and overlap "
                           "eigensolves, split-precision forward + adjoint, Fock and all "
                           "gradients D2H into pinned host memory",
               "energy_rel_diff_vs_value_arm": abs(e_e2e - e_split) / abs(e_split)}
        del gh, host_out

    # ---- CPU baseline: libuw12 itself on the same inputs (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        p, cores = cpu_reference_problem(w, host)
        est, wall, nloops, _ = p.timed_evaluate(1, *cpu_reference_args(w, host, args.s_os,
                                                                       args.s_ss))
        p.close()
        cpu = {"value": est, "unit": "s/eval", "cores": cores, "kind": "reference",
               "cpu_model": cpu_model(),
               "sample": f"{args.config} energy + Fock (libuw12 has no adjoint) by libuw12's "
                         f"unmodified sources (oracle/ref.mk, OpenMP on {cores} threads): one "
                         f"evaluation with each of its {nloops} top-level loops over aux "
                         f"functions / orbital pairs sampled (the first two iterations of "
                         f"every thread's static-schedule block, the rest at the warm "
                         f"iteration's time; {wall:.1f} s measured); setup excluded"}

    batched = batched_report(L, args, args.moduli) if args.batched and world == 1 else None

    flops_fwd = canonical_flops(N, M, R, occ, act, same_spin=indirect, fock=True)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "s/eval", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": f"f64 in, int8 residue products ({args.moduli} moduli) out to f64",
            "data": "synthetic (seeded generators)",
            "config": config_dict(args),
            "parallelism": "single GPU" if world == 1 else f"{world} replicas (one per GPU)",
            "step": "energy + Fock + all 8 integral gradients, same-spin terms included, "
                    "split precision" + (", integral-direct" if args.direct else ""),
            "fp64": {"s_per_step": s64, "speedup": s64 / (elapsed / args.steps),
                     "accuracy_of_split": accuracy},
            "fp64_forward": ({"s_per_eval": s_fwd, "energy": e_fwd,
                              "tflops_canonical": flops_fwd / s_fwd / 1e12} if s_fwd else None),
            "extra_moduli": extra,
            "canonical_flops_forward": flops_fwd,
            "tflops_canonical_forward_per_step": flops_fwd / (elapsed / args.steps) / 1e12,
            "gradient_bytes": grad_bytes,
            "roofline": roofline,
            "roofline_fp64": roofline_fp64,
            "phases_ms_split_step": phases_split,
            "phases_ms_fp64_forward": phases_fwd,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk,
            "input_generation_s": t_gen,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
