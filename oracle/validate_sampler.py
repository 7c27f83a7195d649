"""Checks the sampled CPU-baseline timer against full evaluations -- TEST
INFRASTRUCTURE ONLY.

    python oracle/validate_sampler.py --config c1s --reps 3 [--rounds 1] [--rotation 8]

For one workload shape (the c1 generators at a reduced size) this times, on
all host threads, in separate processes:
  * full evaluations of libuw12 built with its own loop dispatcher
    (oracle/_ref/libuw12_ref.so, every loop iteration run);
  * sampled evaluations of the timing build (oracle/_ref/libuw12_ref_timing.so:
    every thread runs the first max(2, rounds) iterations of its own block of
    each top-level loop's static schedule, the rest of the block is
    extrapolated at the warm iterations' time, the loop is its slowest block);
  * with --rotation S, the estimator bench.py's reference arm uses: one primed
    sampled evaluation, then S evaluations each measuring every S-th loop
    (the others at their last estimate), reporting every step's estimate;
and prints one JSON line: medians, the estimate's ratio to the full time, the
host's CPU model and thread count.  Every child runs with OPENBLAS_NUM_THREADS=1
(BLAS single-threaded inside libuw12's OpenMP loops), as bench.py does.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import statistics
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHAPES = {
    # name: N, M, R, n_occ per spin, decay (the c1 generators at reduced size)
    "c1s": (200, 600, 800, (16, 15), 30.0),
    "c1m": (300, 900, 1200, (24, 23), 30.0),
    "c1": (500, 1500, 2000, (40, 38), 30.0),
}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def child(args):
    sys.path.insert(0, ROOT)
    import numpy as np
    from oracle import ref_lib as R, synth
    N, M, Rr, occ, L = SHAPES[args.config]
    cfg = synth.Config(args.config, N, M, Rr, occ, L)
    inp = synth.make_inputs(cfg, 11)
    timing = args.mode != "full"
    threads = os.cpu_count() or 1
    R.set_threads(threads, 1, timing=timing)
    p = R.RefProblem.from_inputs(inp, timing=timing)
    a = (inp.C, inp.n_orb, cfg.n_spin, inp.occ, cfg.n_occ, cfg.active, args.s_os, args.s_ss)
    if args.mode == "full":
        e, _, _, sec = p.evaluate(*a)
        out = {"mode": "full", "seconds": sec, "energy": e}
    elif args.mode.startswith("rot"):
        S = int(args.mode[3:])
        p.timed_evaluate(1, *a, rotation=S, phase=0)  # primes every loop estimate
        steps = [p.timed_evaluate(1, *a, rotation=S, phase=q) for q in range(1, S + 1)]
        out = {"mode": args.mode, "estimates": [x[0] for x in steps],
               "measured": [x[1] for x in steps], "measured_loops": [x[2] for x in steps]}
    else:
        est, sec, ns, nf = p.timed_evaluate(int(args.mode), *a)
        out = {"mode": f"sampled{args.mode}", "estimate": est, "measured": sec,
               "sampled_loops": ns, "full_loops": nf}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c1s", choices=sorted(SHAPES))
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--rounds", default="1")
    ap.add_argument("--rotation", type=int, default=8)
    ap.add_argument("--s-os", dest="s_os", type=float, default=1.0)
    ap.add_argument("--s-ss", dest="s_ss", type=float, default=0.5)
    ap.add_argument("--mode", default="")
    args = ap.parse_args()
    if args.mode:
        child(args)
        return
    runs = {}
    modes = ["full"] + [r.strip() for r in args.rounds.split(",") if r.strip()]
    if args.rotation > 0:
        modes.append(f"rot{args.rotation}")
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    for _ in range(args.reps):
        for m in modes:
            cmd = [sys.executable, __file__, "--config", args.config, "--mode", m,
                   "--s-os", str(args.s_os), "--s-ss", str(args.s_ss)]
            r = subprocess.run(cmd, capture_output=True, text=True, env=env, check=True)
            runs.setdefault(m, []).append(json.loads(r.stdout.strip().splitlines()[-1]))
    full = statistics.median(x["seconds"] for x in runs["full"])
    rec = {"config": args.config, "shape": SHAPES[args.config], "scales": [args.s_os, args.s_ss],
           "cpu_model": cpu_model(), "threads": os.cpu_count(), "reps": args.reps,
           "full_seconds": [x["seconds"] for x in runs["full"]], "full_median": full}
    for m in modes[1:]:
        if m.startswith("rot"):
            ests = [e for x in runs[m] for e in x["estimates"]]
            rec[m] = {"estimates": ests, "measured": [t for x in runs[m] for t in x["measured"]],
                      "estimate_median": statistics.median(ests),
                      "ratio_to_full": statistics.median(ests) / full}
            continue
        est = statistics.median(x["estimate"] for x in runs[m])
        rec[f"sampled{m}"] = {"estimates": [x["estimate"] for x in runs[m]],
                              "measured": [x["measured"] for x in runs[m]],
                              "estimate_median": est, "ratio_to_full": est / full,
                              "sampled_loops": runs[m][0]["sampled_loops"]}
    print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
