"""The C-ABI library loads on a machine without a GPU and exports every
function declared in include/uw12_c.h (no compute calls)."""
import ctypes
import re

import pytest
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "uw12_c.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(uw12c_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("uw12c_integrals_create", "uw12c_abs_create", "uw12c_fock", "uw12c_energy",
                 "uw12c_form_fock", "uw12c_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol(uw12lib):
    lib = ctypes.CDLL(str(uw12lib.library_path()))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_state_without_gpu(uw12lib):
    L = uw12lib.lib()
    assert b"sm_100a" in L.uw12c_version()
    buf = ctypes.create_string_buffer(64)
    assert L.uw12c_last_error(buf, 64) == 0


def test_cpp_drop_in_header_compiles(uw12lib, tmp_path):
    """include/libuw12.hpp (libuw12's C++ API over the C-ABI) compiles and links."""
    import subprocess
    lib_dir = uw12lib.library_path().parent
    out = tmp_path / "drop_in_check"
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
                        str(ROOT / "tests" / "cpp" / "drop_in_check.cpp"), "-o", str(out),
                        f"-L{lib_dir}", "-luw12_b200"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_invalid_arguments_are_rejected_without_touching_the_device(uw12lib):
    L = uw12lib.lib()
    out = ctypes.c_void_p()
    # bad mem_kind and null output handle are argument errors (status 5)
    assert L.uw12c_integrals_create(None, None, None, 3, 4, 0, 7, ctypes.byref(out)) == 5
    assert L.uw12c_abs_create(None, 3, 4, 0, None) == 5
    buf = ctypes.create_string_buffer(256)
    assert L.uw12c_last_error(buf, 256) == 5 and buf.value


def test_shard_arguments_are_validated_without_touching_the_device(uw12lib):
    L = uw12lib.lib()
    assert L.uw12c_set_shard(2, 2) == 5
    assert L.uw12c_set_shard(0, 0) == 5
    with pytest.raises(uw12lib.UW12Error):
        uw12lib.set_shard(3, 2)
    assert L.uw12c_set_shard(1, 2) == 0
    assert L.uw12c_set_shard(0, 1) == 0


def _compile(uw12lib, src, out):
    import subprocess
    lib_dir = uw12lib.library_path().parent
    return subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
                           str(src), "-o", str(out), f"-L{lib_dir}", "-luw12_b200",
                           f"-Wl,-rpath,{lib_dir}"], capture_output=True, text=True)


def test_fixture_regression_driver_compiles(uw12lib, tmp_path):
    r = _compile(uw12lib, ROOT / "libuw12_b200" / "examples" / "fixture_regression.cpp",
                 tmp_path / "fixture_regression")
    assert r.returncode == 0, r.stderr


def test_load_csv_reads_libuw12_csv_files(uw12lib, tmp_path):
    """load_csv of the C++ drop-in: libuw12's CSV format (one row per line,
    %.16e cells), blank lines, and the error on ragged or unparsable files
    (no device needed)."""
    import subprocess
    import numpy as np
    exe = tmp_path / "csv_check"
    r = _compile(uw12lib, ROOT / "tests" / "cpp" / "csv_check.cpp", exe)
    assert r.returncode == 0, r.stderr
    rng = np.random.default_rng(4)
    a = rng.standard_normal((7, 5)) * np.exp(rng.uniform(-30, 30, (7, 5)))
    f = tmp_path / "a.csv"
    np.savetxt(f, a, delimiter=",", fmt="%.16e")
    f.write_text(f.read_text() + "\n")
    out = subprocess.run([str(exe), str(f)], capture_output=True, text=True).stdout.split()
    assert out[:2] == ["7", "5"]
    assert np.array_equal(np.array([float(x) for x in out[2:]]), a.reshape(-1, order="F"))
    bad = tmp_path / "bad.csv"
    bad.write_text("1.0,2.0\n3.0\n")
    r = subprocess.run([str(exe), str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot read data from file" in r.stdout
    r = subprocess.run([str(exe), str(tmp_path / "missing.csv")], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot read data from file" in r.stdout
