"""The C++ drop-in header (include/libuw12.hpp) compiled into a small program
that uses libuw12's API the way its callers do; its energy and Fock match the
CPU oracle, the callback-built BaseIntegrals give the same energy, stored or
integral-direct (shells produced at every use), the error paths throw the
reference's exception classes, and the uw12::b200 gradient extensions give
the same gradients whole and in blocks."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.parity_cases import Case, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def program(uw12lib, tmp_path_factory):
    out = tmp_path_factory.mktemp("cpp") / "drop_in_check"
    lib_dir = uw12lib.library_path().parent
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}",
           str(ROOT / "tests" / "cpp" / "drop_in_check.cpp"), "-o", str(out),
           f"-L{lib_dir}", "-luw12_b200", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("case", [
    Case("cpp_closed", 24, 84, 116, (5,), (4,), "baseline", 11, 8.0),
    Case("cpp_open", 10, 17, 13, (4, 3), (3, 2), "baseline", 5, 4.0),
], ids=lambda c: c.name)
def test_cpp_drop_in_matches_oracle(program, tmp_path, case):
    d = make_case(case)
    n_spin = len(case.n_occ)
    n_orb = max(o.shape[1] for o in d.orbitals)
    C = np.zeros((case.n_ao, n_orb * n_spin), order="F")
    for s, o in enumerate(d.orbitals):
        C[:, s * n_orb:s * n_orb + o.shape[1]] = o
    occ = np.concatenate(d.occ)
    act = list(case.n_active) + [0] * (2 - n_spin)
    nocc = list(case.n_occ) + [0] * (2 - n_spin)
    hdr = np.array([case.n_ao, case.n_df, case.n_ri, n_spin, n_orb, nocc[0], nocc[1], act[0],
                    act[1]], dtype=np.int64)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(hdr.tobytes())
        for a in (d.W3, d.W2, d.W3_ri, d.V3, d.V2, d.V3_ri, d.WV3, d.WV2, d.S, C, occ,
                  np.array([1.0, 0.5])):
            f.write(np.asfortranarray(a).tobytes(order="F"))
    outp = tmp_path / "out.bin"
    r = subprocess.run([str(program), str(inp), str(outp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr + r.stdout
    raw = np.fromfile(outp, dtype=np.float64)
    e_fock, e_only, e_cb, errors, e_direct, fock_direct_diff, grad_diff = raw[:7]
    fock = raw[7:].reshape((case.n_ao, case.n_ao * n_spin), order="F")
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    fr = np.concatenate(f_ref, axis=1)
    assert abs(e_fock - e_ref) <= 1e-9 * abs(e_ref)
    assert np.max(np.abs(fock - fr)) <= 1e-8 * np.max(np.abs(fr))
    assert abs(e_only - e_fock) <= 1e-12 * abs(e_fock)
    assert abs(e_cb - e_fock) <= 1e-9 * abs(e_fock)
    # integral-direct W and V (shells produced in aux blocks at every use)
    assert abs(e_direct - e_fock) <= 1e-12 * abs(e_fock)
    assert fock_direct_diff <= 1e-12 * np.max(np.abs(fr))
    # uw12::b200 extensions: gradients in blocks equal the whole gradients
    assert grad_diff <= 1e-12
    assert errors == 5
