"""ctypes access to the compiled libuw12 reference -- TEST INFRASTRUCTURE ONLY.

``oracle/ref.mk`` compiles libuw12's unmodified sources (``src/**/*.cpp``,
``libuw12.cpp``) over the project's Armadillo-subset header and scipy's
OpenBLAS into ``oracle/_ref/libuw12_ref.so``; ``oracle/refshim/ref_capi.cpp``
exposes libuw12's public calls (``setup_base_integrals``,
``setup_abs_projectors``, ``uw12_fock`` / ``uw12_energy``, and the term calls
of ``uw12::form_fock``) as a small C-ABI.  This module loads it.  Only
``tests/``, the golden-fixture script and ``bench.py``'s CPU-baseline legs use
it, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libuw12_ref.so")
TIMING_LIB_PATH = os.path.join(HERE, "_ref", "libuw12_ref_timing.so")
REFERENCE_TREE = os.environ.get("UW12_REFERENCE_TREE", "/root/reference")

_libs = {}
_dp = C.POINTER(C.c_double)
_sp = C.POINTER(C.c_size_t)


class RefRuntimeError(RuntimeError):
    """libuw12 threw ``std::runtime_error``."""


class RefLogicError(ValueError):
    """libuw12 threw ``std::logic_error``."""


def build(quiet: bool = True) -> bool:
    """Compile the reference when its source tree is present; True if the
    library exists afterwards."""
    if os.path.isdir(REFERENCE_TREE):
        out = subprocess.run(
            ["make", "-f", os.path.join(HERE, "ref.mk"), f"REF={REFERENCE_TREE}", "-j8", "all"],
            capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError("reference build failed:\n" + out.stdout[-2000:] + out.stderr[-4000:])
        if not quiet:
            print(out.stdout[-500:])
    return os.path.exists(LIB_PATH)


def available(timing: bool = False) -> bool:
    return os.path.exists(TIMING_LIB_PATH if timing else LIB_PATH)


def lib(timing: bool = False):
    """The parity build (libuw12's own loop dispatcher) or, with ``timing``,
    the timing build (same sources, loops run in full or sampled)."""
    path = TIMING_LIB_PATH if timing else LIB_PATH
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -f oracle/ref.mk)")
        L = C.CDLL(path)
        L.uw12ref_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.uw12ref_set_threads.argtypes = [C.c_int, C.c_int]
        L.uw12ref_max_threads.restype = C.c_int
        L.uw12ref_create.argtypes = [_dp] * 9 + [C.c_size_t] * 3 + [C.POINTER(C.c_void_p), _dp]
        L.uw12ref_destroy.argtypes = [C.c_void_p]
        L.uw12ref_evaluate.argtypes = [C.c_void_p, _dp, C.c_size_t, C.c_size_t, _dp, _sp, _sp,
                                       C.c_size_t, C.c_double, C.c_double, _dp, _dp, _dp, _dp]
        L.uw12ref_abs_blocks.argtypes = [_dp, C.c_size_t, C.c_size_t, _dp, _dp, _dp, _dp, _sp]
        if timing:
            L.uw12ref_timing_set.argtypes = [C.c_int]
            L.uw12ref_timing_read.argtypes = [_dp, C.POINTER(C.c_long), C.POINTER(C.c_long)]
            L.uw12ref_timing_rotation.argtypes = [C.c_int, C.c_int]
            L.uw12ref_timing_loops.argtypes = [_dp, C.c_long]
            L.uw12ref_timing_loops.restype = C.c_long
        _libs[path] = L
    return _libs[path]


def _check(status: int, timing: bool = False):
    if status == 0:
        return
    buf = C.create_string_buffer(4096)
    lib(timing).uw12ref_last_error(buf, 4096)
    msg = buf.value.decode()
    if status == 1:
        raise RefRuntimeError(msg)
    if status == 2:
        raise RefLogicError(msg)
    raise RuntimeError(msg)


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _f64(a: Optional[np.ndarray]) -> Optional[np.ndarray]:
    if a is None:
        return None
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def set_threads(omp_threads: int, blas_threads: int = 1, timing: bool = False) -> None:
    lib(timing).uw12ref_set_threads(int(omp_threads), int(blas_threads))


def max_threads(timing: bool = False) -> int:
    return int(lib(timing).uw12ref_max_threads())


class RefProblem:
    """libuw12's ``BaseIntegrals`` W, V, WV and ``ABSProjectors`` built by its own
    setup calls (deep copies; the arrays may be dropped afterwards)."""

    def __init__(self, W3, W2, W3_ri, V3, V2, V3_ri, WV3, WV2, S, n_ao, n_df, n_ri,
                 timing: bool = False):
        self.timing = timing
        self._L = lib(timing)
        arrs = [_f64(x) for x in (W3, W2, W3_ri, V3, V2, V3_ri, WV3, WV2, S)]
        h = C.c_void_p()
        t = C.c_double(0.0)
        _check(self._L.uw12ref_create(*[_ptr(a) for a in arrs], n_ao, n_df, n_ri, C.byref(h),
                                      C.byref(t)), timing)
        self._h = h
        self.n_ao = n_ao
        self.setup_seconds = t.value

    @classmethod
    def from_inputs(cls, inp, timing: bool = False):
        cfg = inp.cfg
        return cls(inp.W3, inp.W2, inp.W3_ri, inp.V3, inp.V2, inp.V3_ri, inp.WV3, inp.WV2,
                   inp.S, cfg.n_ao, cfg.n_df, cfg.n_ri, timing=timing)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.uw12ref_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def evaluate(self, C_orb, n_orb: int, n_spin: int, occ, n_occ: Sequence[int],
                 n_active: Sequence[int], s_os: float, s_ss: float, fock: bool = True,
                 terms: bool = False):
        """Returns (energy, fock n_ao x n_ao*n_spin or None, terms (2,3,4-el) or None,
        seconds)."""
        Cm = _f64(C_orb)
        occ = np.ascontiguousarray(np.asarray(occ, dtype=np.float64))
        no = (C.c_size_t * 2)(*list(n_occ) + [0] * (2 - len(n_occ)))
        na = (C.c_size_t * max(1, len(n_active)))(*list(n_active))
        F = np.zeros((self.n_ao, self.n_ao * n_spin), order="F") if fock else None
        T = np.zeros(3) if terms else None
        e = C.c_double(0.0)
        sec = C.c_double(0.0)
        _check(self._L.uw12ref_evaluate(self._h, _ptr(Cm), n_orb, n_spin, _ptr(occ), no, na,
                                        len(n_active), float(s_os), float(s_ss), _ptr(F),
                                        C.byref(e), _ptr(T), C.byref(sec)), self.timing)
        return e.value, F, T, sec.value

    def timed_evaluate(self, rounds: int, *args, rotation: int = 0, phase: int = 0, **kw):
        """Timing build only: one evaluation with every top-level loop sampled
        at ``rounds`` iterations per thread (0 = every iteration); with
        ``rotation`` S > 0 only the loops q with q % S == phase are measured,
        the others booked at their last estimate (``rotation=0`` clears those).
        Returns (estimated seconds, measured seconds, measured loops, full loops)."""
        if not self.timing:
            raise ValueError("timed_evaluate needs the timing build")
        self._L.uw12ref_timing_rotation(int(rotation), int(phase))
        self._L.uw12ref_timing_set(int(rounds))
        _, _, _, sec = self.evaluate(*args, **kw)
        extra = C.c_double(0.0)
        ns, nf = C.c_long(0), C.c_long(0)
        self._L.uw12ref_timing_read(C.byref(extra), C.byref(ns), C.byref(nf))
        buf = np.zeros(3 * 4096)
        n = self._L.uw12ref_timing_loops(buf.ctypes.data_as(_dp), 4096)
        self.loop_log = buf[:3 * min(n, 4096)].reshape(-1, 3)
        self._L.uw12ref_timing_set(0)
        return sec + extra.value, sec, int(ns.value), int(nf.value)


def abs_blocks(S: np.ndarray, n_ao: int, n_ri: int):
    """libuw12's ABS projector blocks (ri_ri, ri_ao, ao_ri, ao_ao) and the kept
    eigenvector count."""
    S = _f64(S)
    rr = np.zeros((n_ri, n_ri), order="F")
    ra = np.zeros((n_ri, n_ao), order="F")
    ar = np.zeros((n_ao, n_ri), order="F")
    aa = np.zeros((n_ao, n_ao), order="F")
    k = C.c_size_t(0)
    _check(lib().uw12ref_abs_blocks(_ptr(S), n_ao, n_ri, _ptr(rr), _ptr(ra), _ptr(ar), _ptr(aa),
                                    C.byref(k)))
    return (rr, ra, ar, aa), int(k.value)
