"""libuw12's regression run (tests/test_water.cpp of the reference) through the
C++ drop-in: fixture directories in libuw12's test_data CSV layout, written from
the parity cases with the oracle's energy and Fock as the expected results, are
read by libuw12_b200/examples/fixture_regression.cpp and must agree within
libuw12's regression tolerances (1e-8 Eh energy, 1e-7 Eh Fock, relative to
max(1, |value|)); a wrong expected energy must be reported."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.fixture_io import write_fixture
from tests.parity_cases import CASES, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def driver(uw12lib, tmp_path_factory):
    lib_dir = uw12lib.library_path().parent
    out = tmp_path_factory.mktemp("drv") / "fixture_regression"
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}",
                        str(ROOT / "libuw12_b200" / "examples" / "fixture_regression.cpp"), "-o",
                        str(out), f"-L{lib_dir}", "-luw12_b200", f"-Wl,-rpath,{lib_dir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("name", ["unit_closed", "unit_open", "unit_tiles"])
def test_fixture_regression_matches_oracle(driver, cuda_device, tmp_path, name):
    case = [c for c in CASES if c.name == name][0]
    d = make_case(case)
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    write_fixture(d, tmp_path / "data", "neutral", e_ref, f_ref)
    r = subprocess.run([str(driver), str(tmp_path / "data"), "neutral", str(len(d.orbitals))],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    energy = float([ln for ln in r.stdout.splitlines() if ln.startswith("energy ")][0].split()[1])
    assert abs(energy - e_ref) <= 1e-8 * max(1.0, abs(e_ref))


def test_wrong_expected_energy_is_reported(driver, cuda_device, tmp_path):
    case = [c for c in CASES if c.name == "unit_open"][0]
    d = make_case(case)
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    write_fixture(d, tmp_path / "data", "cation", e_ref + 1e-3, f_ref)
    r = subprocess.run([str(driver), str(tmp_path / "data"), "cation", "2"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "FAIL" in r.stdout
