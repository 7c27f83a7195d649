"""UW12 energy + Fock benchmark (one JSON line on rank 0).

Workload: the unrestricted medium system N=500 AO, M=1500 DF, R=2000 RI,
n_alpha=40, n_beta=38 (all-electron), scale factors (1.0, 0.5), seeded
synthetic inputs (three-index N(0,1) exp(-|m-n|/30), metrics B B^T + 1e-6 I,
S-orthonormal orbitals), FP64 throughout.  One step = one energy + Fock
evaluation (uw12 form_fock with the integrals resident in HBM).

``value`` is seconds per evaluation (max-over-ranks device time / steps).
With N > 1 ranks one evaluation is split over the ranks (strong scaling):
each rank holds the full integrals, evaluates its shard (a contiguous part of
the aux functions of the t~ dX Fock term and of the occupied orbitals of the
same-spin three-electron terms; the rest on rank 0) and one NCCL all-reduce
sums the partial Fock matrices and energies.  ``e2e`` is the same metric
through the C-ABI from pinned host buffers: integral upload, on-device metric
and overlap eigensolves, evaluation (and all-reduce) and Fock read-back per
step.

Beside the headline the JSON line reports the split-precision arms
(``--split-moduli``), forward + backward (``adjoint``) and a 64-molecule batch
(``batched``).  ``--config c2 --direct`` evaluates N=1200, M=3600, R=4800
(closed shell, 100 occupied) integral-direct: no three-index tensor stored,
each regenerated on the device by the library's synthetic producer at every
use, the three-index gradients streamed in aux blocks to a squared-norm sink.
``--gemm m,n,k[,beta]`` times one GEMM shape on the FP64 and split paths
instead (a kernel profiling probe).

``--impl reference`` times the CPU restatement of libuw12's algorithm (the
oracle; libuw12 itself cannot be built here) on the host cores for the same
workload: every heavy loop of the reference (its parallel_for /
parallel_sum / parallel_sum_2d over aux functions and orbital pairs) runs a
bounded number of iterations and its time is extrapolated to the full count.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "UW12 energy+Fock s/eval (FP64 plain GPU path vs reference CPU algorithm)"
CONFIGS = {
    # name: N, M, R, n_occ per spin, decay
    "c0": (24, 84, 116, (5,), 8.0),
    "c1": (500, 1500, 2000, (40, 38), 30.0),
    # reduced c1 shape used for single-kernel ncu captures (inputs ~2 GB)
    "c1s": (200, 600, 800, (16, 15), 30.0),
    "c2": (1200, 3600, 4800, (100,), 30.0),
}


# --------------------------------------------------------------------------
# canonical FLOPs (algorithmic work of one evaluation, dense-GEMM FLOPs)
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
# clocks
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
# inputs
# --------------------------------------------------------------------------
def _tag(name: str) -> int:
    import hashlib
    return int.from_bytes(hashlib.sha256(name.encode()).digest()[:8], "little")


def make_device_inputs(cfg, seed, device, three_index=True):
    """Three-index tensors generated on the device (library synth kernel; left
    out when three_index is false); metrics, overlap and orbitals generated with
    torch on the device."""
    import torch
    import libuw12_b200 as L
    N, M, R, occ, L_decay = cfg
    np_ = N * (N + 1) // 2
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    t = {}
    for nm in ("W3", "V3", "WV3") if three_index else ():
        t[nm] = torch.empty(np_ * M, dtype=torch.float64, device=device)
        L.synth_three_index(t[nm].data_ptr(), 0, N, 0, M, seed, _tag(nm), L_decay)
    for nm in ("W3_ri", "V3_ri") if three_index else ():
        t[nm] = torch.empty(R * N * M, dtype=torch.float64, device=device)
        L.synth_three_index(t[nm].data_ptr(), 1, N, R, M, seed, _tag(nm), L_decay)
    for nm in ("W2", "V2", "WV2"):
        B = torch.randn(M, M, dtype=torch.float64, device=device, generator=g) / math.sqrt(M)
        J = B @ B.T + 1e-6 * torch.eye(M, dtype=torch.float64, device=device)
        t[nm] = (0.5 * (J + J.T)).contiguous()  # symmetric: row/column-major agree
    n = N + R
    A = torch.randn(n, n, dtype=torch.float64, device=device, generator=g) / math.sqrt(n)
    S = A @ A.T + 0.1 * torch.eye(n, dtype=torch.float64, device=device)
    t["S"] = (0.5 * (S + S.T)).contiguous()
    Sao = t["S"][:N, :N]
    orbs = []
    for s, o in enumerate(occ):
        C = torch.randn(N, o, dtype=torch.float64, device=device, generator=g)
        G = C.T @ Sao @ C
        Lc = torch.linalg.cholesky(0.5 * (G + G.T))
        C = torch.linalg.solve_triangular(Lc, C.T, upper=False).T
        orbs.append(np.asfortranarray(C.cpu().numpy()))
    torch.cuda.synchronize(device)
    per = 2.0 if len(occ) == 1 else 1.0
    occs = [np.full(o, per) for o in occ]
    return t, orbs, occs


def fp64_peak_tflops(device) -> float:
    """cuBLAS DGEMM 8192^3 burst (best of 5), the FP64 roofline denominator."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def read_profile_traffic():
    """Per-launch DRAM traffic of the GEMM kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "dgemm_dmma_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_gflop:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


# --------------------------------------------------------------------------
# CPU baseline (oracle restatement of libuw12's algorithm, sampled loops)
# --------------------------------------------------------------------------
def cpu_reference_eval(host, cfg, s_os, s_ss, max_iters):
    """One sampled evaluation of the reference algorithm; returns
    (extrapolated seconds per eval, measured seconds, description)."""
    from oracle import uw12_oracle as O
    N, M, R, occ, _ = cfg
    samp = O.Sampler(max_iters)
    t0 = time.perf_counter()
    W = O.BaseIntegrals(host["W3"], host["W2"], host["W3_ri"])
    V = O.BaseIntegrals(host["V3"], host["V2"], host["V3_ri"])
    WV = O.BaseIntegrals(host["WV3"], host["WV2"])
    absp = O.calculate_abs_projectors(host["S"], N, R)
    t_setup = time.perf_counter() - t0
    t1 = time.perf_counter()
    O.uw12_fock(W, V, WV, absp, host["orbitals"], host["occ"], list(occ), s_os, s_ss,
                sampler=samp)
    t_eval = time.perf_counter() - t1
    return t_eval + samp.extra_seconds, t_setup, t_eval, samp


def host_inputs_numpy(cfg, seed):
    from oracle import synth
    N, M, R, occ, Ld = cfg
    h = {}
    for nm in ("W3", "V3", "WV3"):
        h[nm] = synth.fast_three_index(seed, nm, N * (N + 1) // 2, M, synth.ao_damping(N, Ld))
    for nm in ("W3_ri", "V3_ri"):
        h[nm] = synth.fast_three_index(seed, nm, R * N, M, synth.ri_damping(N, R, Ld))
    for nm in ("W2", "V2", "WV2"):
        h[nm] = synth.metric(seed, nm, M)
    h["S"] = synth.overlap(seed, N, R)
    h["orbitals"] = [synth.orbitals(seed, h["S"][:N, :N], o, f"C{s}") for s, o in enumerate(occ)]
    per = 2.0 if len(occ) == 1 else 1.0
    h["occ"] = [np.full(o, per) for o in occ]
    return h


def run_reference(args, rank, world):
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    N, M, R, occ, _ = cfg
    cores = os.cpu_count() or 1
    t_gen = time.perf_counter()
    host = host_inputs_numpy(cfg, 11)
    t_gen = time.perf_counter() - t_gen
    small = host_inputs_numpy(CONFIGS["c0"], 11)
    for _ in range(args.warmup):  # warm BLAS threads / imports on the small case
        cpu_reference_eval(small, CONFIGS["c0"], 1.0, 0.5, None)
    vals, setups = [], []
    for _ in range(args.steps):
        v, ts, te, samp = cpu_reference_eval(host, cfg, args.s_os, args.s_ss, args.ref_iters)
        vals.append(v)
        setups.append(ts)
    value = float(np.median(vals))
    sample = (f"{args.config}: every reference loop over aux functions / orbital pairs capped at "
              f"{args.ref_iters} iterations, loop time extrapolated to full counts; setup "
              f"(3 metric eigensolves + ABS projectors, {np.median(setups):.1f} s) excluded")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s/eval",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, numpy PCG64 streams)",
        "config": config_dict(args),
        "cpu_baseline": {"value": value, "unit": "s/eval", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "s/eval", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "notes": f"input generation {t_gen:.1f} s (untimed)",
    }
    print(json.dumps(line), flush=True)


def batched_workload(device, n_mol=64, seed=2024):
    """64 molecules, N ~ U[20, 300], M = 3N, R = 4N, n_occ = round(N/10), even
    index closed shell and odd index UHF with n_beta = n_alpha - 1, decay 8;
    inputs generated per molecule with a seed derived from (seed, index)."""
    import torch
    import libuw12_b200 as L
    rng = np.random.default_rng(seed)
    mols = []
    for i in range(n_mol):
        N = int(rng.integers(20, 301))
        o = max(1, int(round(N / 10)))
        occ = (o,) if i % 2 == 0 else (o, max(1, o - 1))
        cfg = (N, 3 * N, 4 * N, occ, 8.0)
        t, orbs, occs = make_device_inputs(cfg, seed * 1000 + i, device)
        mols.append({
            "W": L.setup_base_integrals(t["W3"].data_ptr(), t["W2"].data_ptr(),
                                        t["W3_ri"].data_ptr(), n_ao=N, n_df=3 * N, n_ri=4 * N,
                                        device=True),
            "V": L.setup_base_integrals(t["V3"].data_ptr(), t["V2"].data_ptr(),
                                        t["V3_ri"].data_ptr(), n_ao=N, n_df=3 * N, n_ri=4 * N,
                                        device=True),
            "WV": L.setup_base_integrals(t["WV3"].data_ptr(), t["WV2"].data_ptr(), None, n_ao=N,
                                         n_df=3 * N, device=True),
            "abs": L.setup_abs_projectors(t["S"].data_ptr(), N, 4 * N, device=True),
            "orbitals": orbs, "occ": occs, "n_active": list(occ), "n_ao": N})
        del t
        torch.cuda.empty_cache()  # the handles hold their own copies
    return mols


def int8_peak_tops(device):
    """Dense int8 tensor-core throughput of a library GEMM (torch._int_mm,
    8192^3, best of 5), the roofline denominator of the split-precision int8
    kernel; (value, source)."""
    import torch
    n = 8192
    try:
        a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=device)
        b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=device)
        for _ in range(2):
            torch._int_mm(a, b)
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / best / 1e12, "torch._int_mm int8 8192^3 burst measured in this run"
    except Exception as exc:  # no int8 library GEMM: twice the measured bf16 peak
        peaks = json.loads((Path(__file__).parent / "MEASURED_PEAKS.json").read_text())
        return 2.0 * peaks["bf16_tflops"], f"2 x MEASURED_PEAKS bf16 burst ({type(exc).__name__})"


def config_dict(args):
    N, M, R, occ, Ld = CONFIGS[args.config]
    return {"workload": f"uw12 energy+Fock {args.config}: N={N} AO, M={M} DF, R={R} RI, "
                        f"n_occ={list(occ)} ({'UHF' if len(occ) == 2 else 'closed shell'}), "
                        f"all-electron, scales (s_os, s_ss)=({args.s_os}, {args.s_ss})",
            "n_ao": N, "n_df": M, "n_ri": R, "n_occ": list(occ), "decay": Ld,
            "precision": "fp64", "l2": "inputs (28.6 GB at c1) exceed the 126 MB L2",
            "integrals": ("integral-direct: no three-index tensor stored, each regenerated "
                          "on the device (library synthetic producer) in aux blocks at every use"
                          if getattr(args, "direct", False) else "stored on the device")}


# --------------------------------------------------------------------------
# main arm
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
    moduli = [int(x) for x in args.split_moduli.split(",") if x.strip()] or [14]
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
    Lm = moduli[0]
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
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=sorted(CONFIGS))
    ap.add_argument("--s-os", dest="s_os", type=float, default=1.0)
    ap.add_argument("--s-ss", dest="s_ss", type=float, default=0.5)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-iters", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--direct", action="store_true",
                    help="integral-direct three-index tensors: regenerated on the device by "
                         "the library's synthetic producer at every use instead of stored (for "
                         "workloads whose inputs exceed device memory, e.g. --config c2)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched many-molecule report")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the forward+backward (adjoint) report")
    ap.add_argument("--split-moduli", default="14,10",
                    help="moduli counts of the split-precision runs reported beside the FP64 "
                         "headline ('' = none)")
    ap.add_argument("--gemm", default="",
                    help="instead of the workload: time one GEMM shape 'm,n,k[,beta]' (A m x k "
                         "m-contiguous, B k x n k-contiguous, FP64 N(0,1)) on the FP64 path and "
                         "the split path with the first --split-moduli count (kernel profiling "
                         "probe)")
    args = ap.parse_args()
    if args.gemm:
        gemm_probe(args)
        return
    if args.direct:  # the host-side arms need every tensor in memory
        args.no_e2e = args.no_cpu_baseline = args.no_batched = True

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
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=device)

    import libuw12_b200 as L
    L.lib()
    stream = torch.cuda.current_stream(device)
    L.set_stream(stream.cuda_stream)

    cfg = CONFIGS[args.config]
    N, M, R, occ, _ = cfg
    act = list(occ)
    t, orbs, occs = make_device_inputs(cfg, 11, device, three_index=not args.direct)
    peak = fp64_peak_tflops(device)

    if args.direct:
        # the same synthetic tensors from the library's device producer,
        # nothing stored: every three-index tensor is regenerated in aux
        # blocks at every use
        decay = cfg[4]
        specs = {nm: L.SynthSpec(kind, N, R, 11, _tag(nm), decay)
                 for nm, kind in (("W3", 0), ("V3", 0), ("WV3", 0), ("W3_ri", 1), ("V3_ri", 1))}
        fp = L.synth_producer()

        def produced(ao, ri, met):
            return L.setup_base_integrals_callback(
                t[met].data_ptr(), fp, fp if ri else None, n_ao=N, n_df=M, n_ri=R if ri else 0,
                store_ao=False, store_ri=False, device=True,
                user=ctypes.addressof(specs[ao]), user_ri=ctypes.addressof(specs[ri]) if ri else 0)

        W = produced("W3", "W3_ri", "W2")
        V = produced("V3", "V3_ri", "V2")
        WV = produced("WV3", None, "WV2")
    else:
        W = L.setup_base_integrals(t["W3"].data_ptr(), t["W2"].data_ptr(), t["W3_ri"].data_ptr(),
                                   n_ao=N, n_df=M, n_ri=R, device=True)
        V = L.setup_base_integrals(t["V3"].data_ptr(), t["V2"].data_ptr(), t["V3_ri"].data_ptr(),
                                   n_ao=N, n_df=M, n_ri=R, device=True)
        WV = L.setup_base_integrals(t["WV3"].data_ptr(), t["WV2"].data_ptr(), None, n_ao=N,
                                    n_df=M, device=True)
    A = L.setup_abs_projectors(t["S"].data_ptr(), N, R, device=True)
    fock_dev = torch.empty(N * N * len(occ), dtype=torch.float64, device=device)
    indirect = abs(args.s_ss) > 4 * np.finfo(float).eps

    from libuw12_b200.distributed import form_fock_sharded

    def evaluate(Wh, Vh, WVh, Ah, fock):
        if world > 1:
            return form_fock_sharded(Wh, Vh, WVh, Ah, orbs, occs, act, indirect, True, args.s_os,
                                     args.s_ss, fock)[0]
        return L.form_fock(Wh, Vh, WVh, Ah, orbs, occs, act, indirect, True, args.s_os,
                           args.s_ss, fock_out=fock.data_ptr())[0]

    def step():
        return evaluate(W, V, WV, A, fock_dev)

    for _ in range(args.warmup):
        energy = step()
    torch.cuda.synchronize(device)

    clocks = ClockSampler(local)
    clocks.start()
    L.profile_enable(True)
    n0 = L.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(device)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        energy = step()
    ev1.record(stream)
    torch.cuda.synchronize(device)
    if world > 1:
        dist.barrier()
    launches = L.launch_count() - n0
    prof = L.profile_read()
    producer = L.profile_read_kind("producer")
    phases = {k: v / args.steps for k, v in L.profile_phases().items()}
    L.profile_enable(False)
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    if world > 1:
        tt = torch.tensor([elapsed], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed = float(tt.item())
    s_per_eval = elapsed / args.steps

    # ---- split precision (int8 tensor-core GEMMs), same workload and timing
    split = []
    moduli = [int(x) for x in args.split_moduli.split(",") if x.strip()]
    if moduli:
        fock64 = fock_dev.clone()
        i8_peak, i8_src = int8_peak_tops(device)
        for Lm in moduli:
            L.set_precision(Lm)
            for _ in range(max(1, args.warmup - 1)):
                e_split = step()
            torch.cuda.synchronize(device)
            L.profile_enable(True)
            for kind in L.PROFILE_KINDS:
                L.profile_read_kind(kind)
            L.profile_phases()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize(device)
            sv0, sv1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            sv0.record(stream)
            for _ in range(args.steps):
                e_split = step()
            sv1.record(stream)
            torch.cuda.synchronize(device)
            kinds = {k: L.profile_read_kind(k) for k in L.PROFILE_KINDS}
            L.profile_phases()
            L.profile_enable(False)
            L.set_precision(0)
            t_split = sv0.elapsed_time(sv1) / 1e3
            if world > 1:
                tt = torch.tensor([t_split], dtype=torch.float64, device=device)
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                t_split = float(tt.item())
            t_split /= args.steps
            i8 = kinds["i8_mma"]
            i8_tops = i8["work"] / (i8["ms"] / 1e3) / 1e12 if i8["ms"] else None
            split.append({
                "n_moduli": Lm, "bits_per_element_k1500": L.split_bits(Lm, 1500),
                "s_per_eval": t_split, "speedup_vs_fp64": s_per_eval / t_split,
                "energy": e_split, "energy_abs_err_vs_fp64_Eh": abs(e_split - energy),
                "energy_rel_err_vs_fp64": abs(e_split - energy) / abs(energy),
                "fock_max_rel_err_vs_fp64": float((fock_dev - fock64).abs().max() /
                                                  fock64.abs().max()),
                "ms_per_step": {"split_gemms": kinds["split_gemm"]["ms"] / args.steps,
                                "i8_mma": i8["ms"] / args.steps,
                                "operand_prep": kinds["split_prep"]["ms"] / args.steps,
                                "crt": kinds["split_crt"]["ms"] / args.steps,
                                "fp64_dmma_gemms": kinds["dgemm"]["ms"] / args.steps},
                "roofline_i8_mma": {"bound": "tensor", "kernel": "k_i8_mma (tcgen05.mma kind::i8)",
                                    "achieved": i8_tops, "peak": i8_peak, "unit": "TOPS",
                                    "frac": i8_tops / i8_peak if i8_tops else None,
                                    "peak_source": i8_src},
            })
        fock_dev.copy_(fock64)
        del fock64

    # ---- reverse mode: forward + backward of the direct terms (s_ss = 0), FP64
    # and split precision, all gradients written to device buffers
    adjoint = None
    if not args.no_adjoint and world == 1:
        shapes = {"W3": N * (N + 1) // 2 * M, "V3": N * (N + 1) // 2 * M,
                  "WV3": N * (N + 1) // 2 * M, "W3_ri": R * N * M, "V3_ri": R * N * M,
                  "W2": M * M, "V2": M * M, "WV2": M * M}
        # integral-direct: the three-index gradients (as large as the unstored
        # tensors) are streamed in aux blocks into the library's squared-norm
        # device sink; the metric gradients come back whole
        streamed = ("W3", "V3", "WV3", "W3_ri", "V3_ri") if args.direct else ()
        gbuf = {k: torch.empty(v, dtype=torch.float64, device=device) for k, v in shapes.items()
                if k not in streamed}
        gptr = {k: b.data_ptr() for k, b in gbuf.items()}
        norms = torch.zeros(max(1, len(streamed)), dtype=torch.float64, device=device)
        sink_users = {k: norms.data_ptr() + 8 * i for i, k in enumerate(streamed)}
        metric_host = {}

        def backward():
            if not streamed:
                return L.fock_backward(W, V, WV, A, orbs, occs, act, args.s_os, 0.0,
                                       calculate_fock=True, device_out=gptr)[0]
            norms.zero_()
            e, _, _, mg = L.fock_backward_blocks(
                W, V, WV, A, orbs, occs, act, args.s_os, 0.0,
                {k: L.sink_norm2() for k in streamed}, calculate_fock=True, device=True,
                users=sink_users)
            metric_host.clear()
            metric_host.update(mg)
            return e

        def fwd_direct():
            return L.form_fock(W, V, WV, A, orbs, occs, act, False, True, args.s_os, 0.0,
                               fock_out=fock_dev.data_ptr())[0]

        def max_rel_diff(a, b, chunk=1 << 26):
            """max|a - b| / max|b| without full-size temporaries."""
            d = max(float((a[i:i + chunk] - b[i:i + chunk]).abs().max())
                    for i in range(0, a.numel(), chunk))
            r = max(float(b[i:i + chunk].abs().max()) for i in range(0, b.numel(), chunk))
            return d / r if r > 0 else d

        def timed(fn, n):
            # same free memory (and so the same automatic chunk budget) for every arm
            torch.cuda.empty_cache()
            L.trim_memory()
            fn()
            torch.cuda.synchronize(device)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(n):
                val = fn()
            a1.record(stream)
            torch.cuda.synchronize(device)
            return a0.elapsed_time(a1) / 1e3 / n, val

        t_fwd, e_fwd = timed(fwd_direct, args.steps)
        t_bwd, e_bwd = timed(backward, args.steps)
        ref_g = {k: b.clone() for k, b in gbuf.items()}
        ref_norms = norms.cpu().numpy().copy()
        ref_metric = {k: v.copy() for k, v in metric_host.items()}
        adjoint = {"scales": [args.s_os, 0.0], "terms": "direct (indirect_term = 0)",
                   "fp64": {"forward_s": t_fwd, "forward_backward_s": t_bwd, "energy": e_bwd,
                            "energy_equals_forward": e_bwd == e_fwd},
                   "gradients": sorted(shapes),
                   "gradients_streamed_in_blocks": list(streamed),
                   "gradient_bytes": int(sum(v for v in shapes.values()) * 8)}
        splits = []
        for Lm in moduli:
            L.set_precision(Lm)
            t_s, e_s = timed(backward, args.steps)
            L.set_precision(0)
            errs = {k: max_rel_diff(gbuf[k], ref_g[k]) for k in ref_g}
            for k, v in metric_host.items():
                errs[k] = float(np.max(np.abs(v - ref_metric[k])) / np.max(np.abs(ref_metric[k])))
            entry = {"n_moduli": Lm, "forward_backward_s": t_s,
                     "speedup_vs_fp64_forward_backward": t_bwd / t_s,
                     "energy_rel_err_vs_fp64": abs(e_s - e_bwd) / abs(e_bwd),
                     "gradient_max_rel_err_vs_fp64": errs}
            if streamed:
                got = norms.cpu().numpy()
                entry["gradient_norm_rel_err_vs_fp64"] = {
                    k: abs(float(np.sqrt(got[i])) - float(np.sqrt(ref_norms[i]))) /
                    float(np.sqrt(ref_norms[i])) for i, k in enumerate(streamed)}
            splits.append(entry)
        adjoint["split_precision"] = splits
        del gbuf, ref_g
        torch.cuda.empty_cache()

    # ---- end to end through the C-ABI from pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = {k: torch.empty(v.numel(), dtype=torch.float64, pin_memory=True)
                for k, v in t.items()}
        for k, v in t.items():
            host[k].copy_(v.reshape(-1))
        h2d = sum(v.numel() * 8 for v in t.values()) + sum(o.nbytes for o in orbs)
        d2h = N * N * len(occ) * 8
        # free the device inputs and handles so the e2e arm holds its own copies
        for h in (W, V, WV, A):
            h.close()
        del t
        torch.cuda.empty_cache()
        np_ = N * (N + 1) // 2
        hp = {k: v.numpy() for k, v in host.items()}
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        stages = {}
        for _ in range(args.e2e_steps):
            ts = time.perf_counter()
            We = L.setup_base_integrals(hp["W3"].reshape((np_, M), order="F"),
                                        hp["W2"].reshape((M, M)),
                                        hp["W3_ri"].reshape((R * N, M), order="F"))
            stages["setup_W_s"] = time.perf_counter() - ts
            ts = time.perf_counter()
            Ve = L.setup_base_integrals(hp["V3"].reshape((np_, M), order="F"),
                                        hp["V2"].reshape((M, M)),
                                        hp["V3_ri"].reshape((R * N, M), order="F"))
            stages["setup_V_s"] = time.perf_counter() - ts
            ts = time.perf_counter()
            WVe = L.setup_base_integrals(hp["WV3"].reshape((np_, M), order="F"),
                                         hp["WV2"].reshape((M, M)))
            stages["setup_WV_s"] = time.perf_counter() - ts
            ts = time.perf_counter()
            Ae = L.setup_abs_projectors(hp["S"].reshape((N + R, N + R)), N, R)
            stages["setup_abs_s"] = time.perf_counter() - ts
            ts = time.perf_counter()
            if world > 1:
                e_e2e = evaluate(We, Ve, WVe, Ae, fock_dev)
                fock_host = fock_dev.cpu()
            else:
                e_e2e, fock_host = L.uw12_fock(We, Ve, WVe, Ae, orbs, occs, act, args.s_os,
                                               args.s_ss)
            stages["fock_s"] = time.perf_counter() - ts
            for h in (We, Ve, WVe, Ae):
                h.close()
        torch.cuda.synchronize(device)
        te = time.perf_counter() - t0
        if world > 1:
            tt = torch.tensor([te], dtype=torch.float64, device=device)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt.item())
        e2e = {"value": te / args.e2e_steps, "unit": "s/eval",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "includes": "H2D of all integrals from pinned host memory, metric/overlap "
                           "eigensolves, evaluation, Fock D2H",
               "energy_rel_diff_vs_value_arm": abs(e_e2e - energy) / abs(energy),
               "last_step_stages": stages}

    # ---- CPU baseline on a bounded sample (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.no_e2e:
        hostd = {k: hp[k] for k in hp}
        hb = {"W3": hostd["W3"].reshape((N * (N + 1) // 2, M), order="F"),
              "V3": hostd["V3"].reshape((N * (N + 1) // 2, M), order="F"),
              "WV3": hostd["WV3"].reshape((N * (N + 1) // 2, M), order="F"),
              "W3_ri": hostd["W3_ri"].reshape((R * N, M), order="F"),
              "V3_ri": hostd["V3_ri"].reshape((R * N, M), order="F"),
              "W2": hostd["W2"].reshape((M, M)), "V2": hostd["V2"].reshape((M, M)),
              "WV2": hostd["WV2"].reshape((M, M)), "S": hostd["S"].reshape((N + R, N + R)),
              "orbitals": orbs, "occ": occs}
        v, ts, te_, samp = cpu_reference_eval(hb, cfg, args.s_os, args.s_ss, args.ref_iters)
        cpu = {"value": v, "unit": "s/eval", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"{args.config}: reference loops over aux functions / orbital pairs capped "
                         f"at {args.ref_iters} iterations each, loop time extrapolated "
                         f"(measured {te_:.1f} s); numpy/OpenBLAS on all host threads"}

    # ---- batched evaluation of 64 molecules of uneven size (one call), after
    # the c1 workload has left the device
    batched = None
    if not args.no_batched and world == 1:
        if args.no_e2e:  # the end-to-end arm has not released them
            for h in (W, V, WV, A):
                h.close()
            del t
        torch.cuda.empty_cache()
        L.trim_memory()
        mols = batched_workload(device)
        batched = {"workload": "64 molecules, N ~ U[20,300], M = 3N, R = 4N, n_occ = round(N/10),"
                               " half closed shell, half UHF (n_beta = n_alpha - 1), scales "
                               f"({args.s_os}, {args.s_ss}), energy + Fock, FP64 and split "
                               "precision",
                   "n_ao_range": [min(m["n_ao"] for m in mols), max(m["n_ao"] for m in mols)]}
        for n_streams in (1, 8):
            L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=n_streams)
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=n_streams)
            torch.cuda.synchronize(device)
            dt = (time.perf_counter() - t0) / args.steps
            batched[f"s_per_batch_{n_streams}_streams"] = dt
            batched[f"molecules_per_s_{n_streams}_streams"] = len(mols) / dt
        batched["speedup_8_vs_1_stream"] = (batched["s_per_batch_1_streams"] /
                                            batched["s_per_batch_8_streams"])
        # the same batch in split precision (the calling thread's setting applies
        # to every molecule), energies against the FP64 batch
        ref = L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
        split_b = []
        for Lm in moduli:
            L.set_precision(Lm)
            L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                res = L.fock_batched(mols, indirect, True, args.s_os, args.s_ss, n_streams=1)
            torch.cuda.synchronize(device)
            L.set_precision(0)
            dt = (time.perf_counter() - t0) / args.steps
            split_b.append({"n_moduli": Lm, "s_per_batch_1_stream": dt,
                            "speedup_vs_fp64_1_stream": batched["s_per_batch_1_streams"] / dt,
                            "max_energy_rel_err_vs_fp64": max(
                                abs(r[0] - q[0]) / abs(q[0]) for r, q in zip(res, ref))})
        batched["split_precision"] = split_b
        for m in mols:
            for k in ("W", "V", "WV", "abs"):
                m[k].close()
        del mols
        L.trim_memory()

    flops = canonical_flops(N, M, R, occ, act, same_spin=indirect, fock=True)
    gemm_tf = prof["flops"] / (prof["ms"] / 1e3) / 1e12 if prof["ms"] > 0 else None
    bpg = read_profile_traffic()
    avg_launch_flops = prof["flops"] / max(1, prof["launches"])
    roof = {"bound": "tensor", "kernel": "dgemm_dmma (mma.sync m16n8k4 f64)",
            "achieved": gemm_tf, "peak": peak, "unit": "TFLOP/s",
            "frac": (gemm_tf / peak) if gemm_tf else None,
            "peak_source": "cuBLAS DGEMM 8192^3 burst measured in this run (MEASURED_PEAKS.json "
                           "has no FP64 figure)",
            "traffic": (bpg * avg_launch_flops / 1e9) if bpg else None,
            "launches": prof["launches"], "kernel_ms": prof["ms"],
            "share_of_step": (prof["ms"] / 1e3) / elapsed if elapsed > 0 else None}
    if rank == 0:
        line = {
            "metric": METRIC, "value": s_per_eval, "unit": "s/eval", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generators; integrals generated on device)",
            "config": dict(config_dict(args), parallelism=(
                "single GPU" if world == 1 else
                f"{world}-way sharded evaluation + NCCL all-reduce of Fock and energy")),
            "tflops_canonical": flops / s_per_eval / 1e12,
            "canonical_flops_per_eval": flops,
            "energy": energy,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "phases_ms_per_step": phases,
            "producer": ({"ms_per_step": producer["ms"] / args.steps,
                          "calls_per_step": producer["launches"] / args.steps,
                          "gb_per_step": producer["work"] / args.steps / 1e9,
                          "note": "integral generation, reported separately; it is inside "
                                  "value (the timed evaluation)"}
                         if args.direct else None),
            "gpu_launches": int(launches),
            "clocks": clk,
            "split_precision": split,
            "adjoint": adjoint,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
