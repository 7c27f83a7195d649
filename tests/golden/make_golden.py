"""Writes tests/golden/reference_goldens.npz from the compiled libuw12 reference.

Run from the repository root after building the reference:

    make -f oracle/ref.mk REF=<libuw12 source tree>
    python tests/golden/make_golden.py

Every case of ``tests/golden_cases.py`` is evaluated by libuw12 itself
(``uw12::setup_base_integrals``, ``setup_abs_projectors``, ``uw12_fock`` and the
term calls of ``uw12::form_fock``, through ``oracle/refshim/ref_capi.cpp``).
Inputs are regenerated from their seeds by ``tests/parity_cases.make_case``;
the fixture stores the outputs, a few input checksums (so a test notices if the
generators drift) and the SHA-256 of every reference source compiled.

Keys: ``<case>|<s_os>,<s_ss>|energy`` (scalar), ``...|terms`` (two-, three-,
four-electron energies), ``...|fock`` (n_ao x n_ao*n_spin, Fortran order);
``<case>|checksum`` (sums of the three-index inputs and the metric);
``abs|<name>|S`` / ``|ri_ri`` / ``|ri_ao`` / ``|ao_ri`` / ``|ao_ao`` / ``|n_kept``;
``error|<name>|class`` (1 runtime_error, 2 logic_error) and ``|message``.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_lib as R  # noqa: E402
from tests import golden_cases as G  # noqa: E402
from tests.parity_cases import make_case  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "reference_goldens.npz")


def pack_orbitals(orbitals):
    """libuw12's setup_orbitals layout: n_ao x (n_orb * n_spin), every spin
    padded with zero columns to the same n_orb (only the occupied leading
    columns are read)."""
    n_ao = orbitals[0].shape[0]
    n_orb = max(max(o.shape[1] for o in orbitals), 1)
    cols = []
    for o in orbitals:
        pad = np.zeros((n_ao, n_orb - o.shape[1]))
        cols.append(np.concatenate([o, pad], axis=1))
    return np.asfortranarray(np.concatenate(cols, axis=1)), n_orb


def checksum(d):
    return np.array([d.W3.sum(), d.V3.sum(), d.WV3.sum(), d.W3_ri.sum(), d.V3_ri.sum(),
                     d.W2.sum(), d.S.sum()])


def problem(d):
    c = d.case
    return R.RefProblem(d.W3, d.W2, d.W3_ri, d.V3, d.V2, d.V3_ri, d.WV3, d.WV2, d.S,
                        c.n_ao, c.n_df, c.n_ri)


def evaluate(p, d, s_os, s_ss, want_fock=True):
    c = d.case
    C, n_orb = pack_orbitals(d.orbitals)
    occ = np.concatenate(d.occ)
    n_spin = len(c.n_occ)
    e, F, _, _ = p.evaluate(C, n_orb, n_spin, occ, c.n_occ, c.n_active, s_os, s_ss,
                            fock=want_fock, terms=False)
    e_t, _, T, _ = p.evaluate(C, n_orb, n_spin, occ, c.n_occ, c.n_active, s_os, s_ss,
                              fock=False, terms=True)
    # the two calls differ only in OpenMP reduction order; with same-spin
    # scaling the direct and exchange parts of a term cancel by up to 1e-8 on
    # the unit-test shapes, so the check is loose (a consistency check of the
    # two entry points, not a parity bound)
    assert abs(e - e_t) <= 1e-7 * max(1.0, abs(e), float(np.max(np.abs(T)))), (e, e_t, T)
    return e, F, T


def key(name, s_os, s_ss, what):
    return f"{name}|{s_os:g},{s_ss:g}|{what}"


def main():
    if not R.available():
        R.build()
    R.set_threads(os.cpu_count() or 1, 1)
    out = {}
    t0 = time.time()
    for case, scales in G.PARITY:
        d = make_case(case)
        p = problem(d)
        out[f"{case.name}|checksum"] = checksum(d)
        for s_os, s_ss in scales:
            e, F, T = evaluate(p, d, s_os, s_ss)
            out[key(case.name, s_os, s_ss, "energy")] = np.array(e)
            out[key(case.name, s_os, s_ss, "terms")] = T
            out[key(case.name, s_os, s_ss, "fock")] = F
        p.close()
    print(f"parity cases {time.time() - t0:.1f} s", flush=True)

    d = make_case(G.C1S)
    p = problem(d)
    out[f"{G.C1S.name}|checksum"] = checksum(d)
    for s_os, s_ss in G.C1S_SCALES:
        t = time.time()
        e, F, T = evaluate(p, d, s_os, s_ss)
        out[key(G.C1S.name, s_os, s_ss, "energy")] = np.array(e)
        out[key(G.C1S.name, s_os, s_ss, "terms")] = T
        if (s_os, s_ss) == G.C1S_SCALES[0]:
            out[key(G.C1S.name, s_os, s_ss, "fock")] = F
        print(f"c1s ({s_os}, {s_ss}) {time.time() - t:.1f} s", flush=True)
    p.close()
    del d

    for i, case in G.c4_subset():
        d = make_case(case)
        p = problem(d)
        out[f"{case.name}|checksum"] = checksum(d)
        e, F, T = evaluate(p, d, 1.0, 0.5)
        out[key(case.name, 1.0, 0.5, "energy")] = np.array(e)
        out[key(case.name, 1.0, 0.5, "terms")] = T
        out[key(case.name, 1.0, 0.5, "fock")] = F
        p.close()
    print(f"c4 subset {[c.name for _, c in G.c4_subset()]}", flush=True)

    for e in G.ABS_EDGE:
        S, lam = G.abs_edge_overlap(e)
        blocks, kept = R.abs_blocks(S, e.n_ao, e.n_ri)
        out[f"abs|{e.name}|S"] = S
        for nm, b in zip(("ri_ri", "ri_ao", "ao_ri", "ao_ao"), blocks):
            out[f"abs|{e.name}|{nm}"] = b
        out[f"abs|{e.name}|n_kept"] = np.array(kept)

    for name, what, arg in G.ERRORS:
        dd = make_case(G.ERROR_CASE)
        n_active = list(G.ERROR_CASE.n_active)
        if what == "n_active":
            n_active = arg
        elif what == "occ_alpha_negative":
            dd.occ = [-dd.occ[0], dd.occ[1]]
        elif what == "W2_asymmetric":
            dd.W2 = dd.W2 + np.triu(np.ones_like(dd.W2), 1)
        status, msg = 0, ""
        try:
            p = problem(dd)
            C, n_orb = pack_orbitals(dd.orbitals)
            c = dd.case
            p.evaluate(C, n_orb, len(c.n_occ), np.concatenate(dd.occ), c.n_occ, n_active,
                       1.0, 0.5, fock=True, terms=False)
        except R.RefRuntimeError as ex:
            status, msg = 1, str(ex)
        except R.RefLogicError as ex:
            status, msg = 2, str(ex)
        out[f"error|{name}|class"] = np.array(status)
        out[f"error|{name}|message"] = np.array(msg)
        print(f"error {name}: {status} {msg}", flush=True)

    srcs = {}
    for dirpath, _, files in os.walk(os.path.join(R.REFERENCE_TREE, "src")):
        for f in sorted(files):
            if f.endswith((".cpp", ".hpp")):
                pth = os.path.join(dirpath, f)
                srcs[os.path.relpath(pth, R.REFERENCE_TREE)] = hashlib.sha256(
                    open(pth, "rb").read()).hexdigest()
    for f in ("libuw12.cpp", "libuw12.hpp"):
        srcs[f] = hashlib.sha256(open(os.path.join(R.REFERENCE_TREE, f), "rb").read()).hexdigest()
    out["meta|sources"] = np.array(json.dumps(srcs, sort_keys=True))
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e6:.2f} MB, {len(out)} keys, "
          f"{time.time() - t0:.1f} s)")


if __name__ == "__main__":
    main()
