"""libuw12_b200 -- B200-native UW12 energy + Fock behind libuw12's API.

The compute lives in ``_lib/libuw12_b200.so`` (hand-written sm_100a CUDA
behind the C-ABI declared in ``include/uw12_c.h``).  This module is a thin
ctypes mirror of libuw12's public C++ API (``libuw12.hpp``) for Python
callers and tests: ``setup_base_integrals``, ``setup_abs_projectors``,
``setup_orbitals``, ``setup_occupations``, ``uw12_energy``, ``uw12_fock`` and
the lower-level ``form_fock`` (``src/uw12.hpp:129-142``).  There is no CPU
path: if the shared library is missing or no CUDA device is usable, calls
raise.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

__all__ = [
    "UW12Error", "UW12RuntimeError", "UW12LogicError", "UW12CudaError",
    "BaseIntegrals", "ABSProjectors", "setup_base_integrals", "setup_abs_projectors",
    "setup_orbitals", "setup_occupations", "uw12_energy", "uw12_fock", "form_fock",
    "lib", "library_path",
]

_HERE = Path(__file__).resolve().parent
_LIB_PATH = Path(os.environ.get("UW12_LIB_PATH", _HERE / "_lib" / "libuw12_b200.so"))
_lib = None

OK, ERR_RUNTIME, ERR_LOGIC, ERR_CUDA, ERR_ALLOC, ERR_INVALID = range(6)
MEM_HOST, MEM_DEVICE = 0, 1


class UW12Error(Exception):
    """Base class of errors reported by the CUDA library."""


class UW12RuntimeError(UW12Error, RuntimeError):
    """libuw12 raises std::runtime_error (user-input errors)."""


class UW12LogicError(UW12Error, ValueError):
    """libuw12 raises std::logic_error (shape errors)."""


class UW12CudaError(UW12Error):
    """CUDA / cuSOLVER failure or invalid argument."""


def library_path() -> Path:
    return _LIB_PATH


def lib():
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} not found: build it with `python -m libuw12_b200.build` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(str(_LIB_PATH))
    c_d = ctypes.c_double
    c_sz = ctypes.c_size_t
    P = ctypes.c_void_p
    PD = ctypes.POINTER(c_d)
    PSZ = ctypes.POINTER(c_sz)
    L.uw12c_last_error.argtypes = [ctypes.c_char_p, c_sz]
    L.uw12c_last_error.restype = ctypes.c_int
    L.uw12c_version.restype = ctypes.c_char_p
    L.uw12c_integrals_create.argtypes = [P, P, P, c_sz, c_sz, c_sz, ctypes.c_int,
                                         ctypes.POINTER(P)]
    L.uw12c_integrals_create_eigenbasis.argtypes = [P, P, c_sz, c_sz, ctypes.c_int,
                                                    ctypes.POINTER(P)]
    L.uw12c_integrals_destroy.argtypes = [P]
    L.uw12c_integrals_dims.argtypes = [P, PSZ, PSZ, PSZ]
    L.uw12c_integrals_df_vals.argtypes = [P, PD]
    L.uw12c_abs_create.argtypes = [P, c_sz, c_sz, ctypes.c_int, ctypes.POINTER(P)]
    L.uw12c_abs_destroy.argtypes = [P]
    L.uw12c_abs_blocks.argtypes = [P, P, P, P, P]
    L.uw12c_form_fock.argtypes = [P, P, P, P, c_sz, c_sz, ctypes.POINTER(P), PSZ, PSZ,
                                  ctypes.POINTER(P), PSZ, PSZ, ctypes.c_int, ctypes.c_int, c_d,
                                  c_d, c_sz, PD, PD, P, ctypes.c_int]
    L.uw12c_fock.argtypes = [P, P, P, P, P, P, c_sz, c_sz, c_sz, P, c_sz, c_sz, PSZ, c_d, c_d,
                             c_sz, PD]
    L.uw12c_integrals_create_callback.argtypes = [P, ctypes.c_int, BLOCK_FN, P, BLOCK_FN, P,
                                                  c_sz, c_sz, c_sz, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.POINTER(P)]
    L.uw12c_fock_batched.argtypes = [P, c_sz, ctypes.c_int, ctypes.c_int, c_d, c_d, c_sz,
                                     ctypes.POINTER(ctypes.c_int)]
    L.uw12c_fock_backward.argtypes = [P, P, P, P, c_sz, c_sz, ctypes.POINTER(P), PSZ, PSZ,
                                      ctypes.POINTER(P), PSZ, PSZ, ctypes.c_int, c_d, c_d, PD,
                                      PD, P,
                                      ctypes.c_int, ctypes.POINTER(P), ctypes.POINTER(P),
                                      ctypes.POINTER(P), ctypes.c_int]
    L.uw12c_fock_backward_blocks.argtypes = [P, P, P, P, c_sz, c_sz, ctypes.POINTER(P), PSZ,
                                             PSZ, ctypes.POINTER(P), PSZ, PSZ, ctypes.c_int, c_d,
                                             c_d, PD, PD,
                                             P, ctypes.c_int, ctypes.POINTER(P),
                                             ctypes.POINTER(P), ctypes.POINTER(P),
                                             ctypes.POINTER(P), ctypes.c_int, ctypes.POINTER(P),
                                             ctypes.c_int]
    L.uw12c_energy.argtypes = [P, P, P, P, P, c_sz, c_sz, c_sz, P, c_sz, c_sz, PSZ, c_d, c_d,
                               c_sz, PD]
    L.uw12c_set_stream.argtypes = [P]
    L.uw12c_set_memory_budget.argtypes = [c_sz]
    L.uw12c_set_shard.argtypes = [c_sz, c_sz]
    L.uw12c_set_allreduce.argtypes = [ALLREDUCE_FN, P]
    L.uw12c_launch_count.restype = ctypes.c_ulonglong
    L.uw12c_profile_enable.argtypes = [ctypes.c_int]
    L.uw12c_profile_read.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), PD, PD]
    L.uw12c_profile_phases.argtypes = [ctypes.c_char_p, c_sz]
    LL = ctypes.c_longlong
    L.uw12c_dgemm.argtypes = [LL, LL, LL, c_d, P, LL, ctypes.c_int, P, LL, ctypes.c_int, c_d, P,
                              LL, LL, LL, ctypes.POINTER(LL), LL, LL, ctypes.POINTER(LL),
                              ctypes.c_int]
    L.uw12c_synth_three_index.argtypes = [P, ctypes.c_int, c_sz, c_sz, c_sz, ctypes.c_ulonglong,
                                          ctypes.c_ulonglong, c_d]
    L.uw12c_dgemm_split.argtypes = L.uw12c_dgemm.argtypes
    L.uw12c_set_precision.argtypes = [ctypes.c_int]
    L.uw12c_set_split_threshold.argtypes = [c_d]
    L.uw12c_split_bits.argtypes = [ctypes.c_int, LL, ctypes.POINTER(ctypes.c_int)]
    L.uw12c_profile_read_kind.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                          ctypes.POINTER(c_d), ctypes.POINTER(c_d)]
    L.uw12c_autotune.argtypes = [ctypes.c_int, ctypes.c_char_p]
    L.uw12c_autotune_save.argtypes = [ctypes.c_char_p]
    L.uw12c_autotune_size.argtypes = [ctypes.POINTER(LL)]
    L.uw12c_autotune_lookup.argtypes = [LL, LL, LL, LL, LL, ctypes.POINTER(ctypes.c_int)]
    _lib = L
    return L


def _check(status: int):
    if status == OK:
        return
    buf = ctypes.create_string_buffer(1024)
    lib().uw12c_last_error(buf, 1024)
    msg = buf.value.decode(errors="replace")
    if status == ERR_RUNTIME:
        raise UW12RuntimeError(msg)
    if status == ERR_LOGIC:
        raise UW12LogicError(msg)
    raise UW12CudaError(f"status {status}: {msg}")


def _fptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


def _col_major(a, rows: int, cols: int) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape((rows, cols), order="F")
    if a.shape != (rows, cols):
        raise UW12LogicError(f"expected a {rows} x {cols} matrix, got {a.shape}")
    return np.asfortranarray(a)


class BaseIntegrals:
    """Device-resident ``BaseIntegrals`` (src/integrals/base_integrals.hpp:46-293)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        n_ao, n_df, n_ri = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib().uw12c_integrals_dims(self._h, ctypes.byref(n_ao), ctypes.byref(n_df),
                                          ctypes.byref(n_ri)))
        self.n_ao, self.n_df, self.n_ri = n_ao.value, n_df.value, n_ri.value

    def get_number_ao(self) -> int:
        return self.n_ao

    def get_number_df(self) -> int:
        return self.n_df

    def get_number_ri(self) -> int:
        return self.n_ri

    def get_df_vals(self) -> np.ndarray:
        out = np.empty(self.n_df)
        _check(lib().uw12c_integrals_df_vals(self._h, out.ctypes.data_as(
            ctypes.POINTER(ctypes.c_double))))
        return out

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().uw12c_integrals_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ABSProjectors:
    """Device-resident ABS+ projectors (src/three_electron/ri_utils.hpp:20-29)."""

    def __init__(self, handle: ctypes.c_void_p, n_ao: int, n_ri: int):
        self._h = handle
        self.n_ao, self.n_ri = n_ao, n_ri

    @property
    def handle(self):
        return self._h

    def blocks(self):
        """(s_inv_ri_ri, s_inv_ri_ao, s_inv_ao_ri, s_inv_ao_ao) as host arrays."""
        N, R = self.n_ao, self.n_ri
        rr = np.zeros((R, R), order="F")
        ra = np.zeros((R, N), order="F")
        ar = np.zeros((N, R), order="F")
        aa = np.zeros((N, N), order="F")
        _check(lib().uw12c_abs_blocks(self._h, _fptr(rr), _fptr(ra), _fptr(ar), _fptr(aa)))
        return rr, ra, ar, aa

    def close(self):
        if self._h:
            lib().uw12c_abs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setup_base_integrals(X3, X2, X3_ri=None, n_ao: Optional[int] = None,
                         n_df: Optional[int] = None, n_ri: int = 0,
                         device: bool = False) -> BaseIntegrals:
    """``uw12::setup_base_integrals`` (libuw12.hpp:42-70).

    With ``device=True`` the arguments are raw device pointers (ints) and the
    sizes must be given; otherwise they are host arrays (column-major).
    """
    h = ctypes.c_void_p()
    if device:
        if n_ao is None or n_df is None:
            raise UW12LogicError("n_ao and n_df are required for device pointers")
        st = lib().uw12c_integrals_create(ctypes.c_void_p(X3), ctypes.c_void_p(X2),
                                          ctypes.c_void_p(X3_ri or 0), n_ao, n_df,
                                          n_ri if X3_ri else 0, MEM_DEVICE, ctypes.byref(h))
        _check(st)
        return BaseIntegrals(h)
    X2 = np.asarray(X2, dtype=np.float64)
    if n_df is None:
        n_df = X2.shape[0]
    X3 = np.asarray(X3, dtype=np.float64)
    if n_ao is None:
        rows = X3.shape[0] if X3.ndim == 2 else X3.size // n_df
        n_ao = int((np.sqrt(8 * rows + 1) - 1) / 2)
    np_ = n_ao * (n_ao + 1) // 2
    X3 = _col_major(X3, np_, n_df)
    X2 = _col_major(X2, n_df, n_df)
    if X3_ri is not None:
        X3_ri = np.asarray(X3_ri, dtype=np.float64)
        if not n_ri:
            rows = X3_ri.shape[0] if X3_ri.ndim == 2 else X3_ri.size // n_df
            n_ri = rows // n_ao
        X3_ri = _col_major(X3_ri, n_ri * n_ao, n_df)
    st = lib().uw12c_integrals_create(_fptr(X3), _fptr(X2), _fptr(X3_ri) if X3_ri is not None
                                      else ctypes.c_void_p(0), n_ao, n_df,
                                      n_ri if X3_ri is not None else 0, MEM_HOST, ctypes.byref(h))
    _check(st)
    return BaseIntegrals(h)


BLOCK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                            ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


class SynthSpec(ctypes.Structure):
    """``uw12c_synth_spec``: the synthetic tensors of ``synth_three_index``."""
    _fields_ = [("kind", ctypes.c_int), ("n_ao", ctypes.c_size_t), ("n_ri", ctypes.c_size_t),
                ("seed", ctypes.c_ulonglong), ("tag", ctypes.c_ulonglong),
                ("decay", ctypes.c_double)]


def setup_base_integrals_callback(X2, three_index, three_index_ri=None, n_ao: int = 0,
                                  n_df: int = 0, n_ri: int = 0, store_ao: bool = True,
                                  store_ri: bool = True, device: bool = False,
                                  user: int = 0, user_ri: int = 0) -> BaseIntegrals:
    """``BaseIntegrals`` from producers of the three-index integrals
    (``uw12c_integrals_create_callback``; the callback constructors of
    src/integrals/base_integrals.hpp:52-72).

    ``three_index`` / ``three_index_ri`` are Python callables
    ``f(first, count, out_ptr, ld, stream_ptr)`` writing aux functions
    [first, first + count) as columns of ``out`` (device memory when
    ``device``, else host memory), or raw function pointers (ints) of C
    producers called with ``user`` / ``user_ri`` (the library's own
    ``synth_producer()`` is a device producer).  Unstored tensors are produced
    again at every use (integral-direct mode).  ``X2`` is the metric: a host
    array, or a device pointer (int).
    """
    keep = []

    def as_fn(f):
        if f is None:
            return BLOCK_FN()
        if isinstance(f, int):
            return ctypes.cast(ctypes.c_void_p(f), BLOCK_FN)

        def tramp(_user, first, count, out, ld, stream):
            try:
                f(first, count, out or 0, ld, stream or 0)
                return 0
            except Exception:  # reported to the library as a failed producer
                return 1

        cf = BLOCK_FN(tramp)
        keep.append(cf)
        return cf

    x2_device = isinstance(X2, int)
    if x2_device:
        x2 = ctypes.c_void_p(X2)
    else:
        X2 = _col_major(np.asarray(X2, dtype=np.float64), n_df, n_df)
        keep.append(X2)
        x2 = _fptr(X2)
    h = ctypes.c_void_p()
    if isinstance(three_index, int) and not device:
        raise UW12LogicError("native producers write device memory: pass device=True")
    _check(lib().uw12c_integrals_create_callback(
        x2, MEM_DEVICE if x2_device else MEM_HOST, as_fn(three_index), ctypes.c_void_p(user),
        as_fn(three_index_ri), ctypes.c_void_p(user_ri), n_ao, n_df,
        n_ri if three_index_ri is not None else 0, int(store_ao), int(store_ri),
        MEM_DEVICE if device else MEM_HOST, ctypes.byref(h)))
    out = BaseIntegrals(h)
    out._producers = keep  # the producers must outlive the handle
    return out


def synth_producer() -> int:
    """Address of ``uw12c_synth_block``, a native device producer (user = SynthSpec*)."""
    return ctypes.cast(lib().uw12c_synth_block, ctypes.c_void_p).value


def base_integrals_eigenbasis(J3, df_vals) -> BaseIntegrals:
    """``BaseIntegrals(J3, df_vals)`` (src/integrals/base_integrals.hpp:104): three-index
    integrals already in the metric eigenbasis (J3 = J3_0 P2) and the eigenvalues; no RI."""
    df_vals = np.ascontiguousarray(np.asarray(df_vals, dtype=np.float64).reshape(-1))
    n_df = df_vals.size
    J3 = np.asarray(J3, dtype=np.float64)
    rows = J3.shape[0] if J3.ndim == 2 else J3.size // n_df
    n_ao = int((np.sqrt(8 * rows + 1) - 1) / 2)
    J3 = _col_major(J3, n_ao * (n_ao + 1) // 2, n_df)
    h = ctypes.c_void_p()
    _check(lib().uw12c_integrals_create_eigenbasis(_fptr(J3), _fptr(df_vals), n_ao, n_df,
                                                   MEM_HOST, ctypes.byref(h)))
    return BaseIntegrals(h)


def setup_abs_projectors(S, n_ao: int, n_ri: int, device: bool = False) -> ABSProjectors:
    """``uw12::setup_abs_projectors`` (libuw12.hpp:80)."""
    h = ctypes.c_void_p()
    if device:
        st = lib().uw12c_abs_create(ctypes.c_void_p(S), n_ao, n_ri, MEM_DEVICE, ctypes.byref(h))
    else:
        S = _col_major(S, n_ao + n_ri, n_ao + n_ri)
        st = lib().uw12c_abs_create(_fptr(S), n_ao, n_ri, MEM_HOST, ctypes.byref(h))
    _check(st)
    return ABSProjectors(h, n_ao, n_ri)


def setup_orbitals(C, n_ao: int, n_orb: int, n_spin: int) -> List[np.ndarray]:
    """``uw12::setup_orbitals`` (libuw12.cpp:58-77): alpha columns then beta."""
    if n_spin not in (1, 2):
        raise UW12RuntimeError("Number of spin channels must be 1 or 2")
    C1 = _col_major(C, n_ao, n_orb * n_spin)
    if n_spin == 1:
        return [C1]
    return [np.asfortranarray(C1[:, :n_orb]), np.asfortranarray(C1[:, n_orb:])]


def setup_occupations(occ, n_occ_alpha: int, n_occ_beta: Optional[int] = None):
    """``uw12::setup_occupations`` closed (n_occ) and open (n_alpha, n_beta) forms
    (libuw12.cpp:79-112)."""
    occ = np.asarray(occ, dtype=np.float64).reshape(-1)
    if n_occ_beta is None:
        return [occ[:n_occ_alpha].copy()]
    return [occ[:n_occ_alpha].copy(), occ[n_occ_alpha:n_occ_alpha + n_occ_beta].copy()]


def _nearly_zero(x: float) -> bool:
    return abs(x) <= 4 * np.finfo(np.float64).eps


def form_fock(W: BaseIntegrals, V: BaseIntegrals, WV: BaseIntegrals, abs_p: ABSProjectors,
              orbitals: Sequence[np.ndarray], occupations: Sequence[np.ndarray],
              n_active: Sequence[int], indirect_term: bool, calculate_fock: bool,
              scale_opp_spin: float, scale_same_spin: float, print_level: int = 0,
              fock_out=None) -> Tuple[float, Optional[List[np.ndarray]], Tuple[float, float, float]]:
    """``uw12::form_fock`` (src/uw12.hpp:129-142).

    Returns ``(energy, fock, (E2, E3, E4))`` with ``fock`` a list of n_ao x n_ao
    arrays per spin (None when ``calculate_fock`` is false).  ``fock_out`` may
    be a device pointer (int) receiving the n_ao x n_ao*n_spin Fock matrix.
    """
    n_spin = len(orbitals)
    if n_spin < 1 or n_spin > 2:
        raise UW12LogicError("invalid number of spin channels")
    if len(occupations) != n_spin:
        if len(occupations) < 1 or len(occupations) > 2:
            raise UW12LogicError("invalid number of spin channels")
        raise UW12RuntimeError("Different number of spin channels for orbitals and occupations")
    if len(n_active) != n_spin:
        if len(n_active) < 1 or len(n_active) > 2:
            raise UW12LogicError("invalid number of spin channels")
        raise UW12RuntimeError("Different number of spin channels in n_active and orbitals")
    n_ao = W.n_ao
    Cs = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in orbitals]
    for c in Cs:
        if c.ndim != 2 or c.shape[0] != n_ao:
            raise UW12RuntimeError("Inconsistent number of atomic orbitals")
    occs = [np.ascontiguousarray(np.asarray(o, dtype=np.float64).reshape(-1)) for o in occupations]
    P = ctypes.c_void_p
    c_ptrs = (P * n_spin)(*[_fptr(c) for c in Cs])
    ldc = (ctypes.c_size_t * n_spin)(*[max(1, c.shape[0]) for c in Cs])
    norb = (ctypes.c_size_t * n_spin)(*[c.shape[1] for c in Cs])
    o_ptrs = (P * n_spin)(*[_fptr(o) for o in occs])
    nocc = (ctypes.c_size_t * n_spin)(*[o.size for o in occs])
    nact = (ctypes.c_size_t * n_spin)(*[int(a) for a in n_active])
    energy = ctypes.c_double()
    terms = (ctypes.c_double * 3)()
    fock = None
    if fock_out is not None:
        fptr, fmem = ctypes.c_void_p(fock_out), MEM_DEVICE
    elif calculate_fock:
        fock = np.zeros((n_ao, n_ao * n_spin), order="F")
        fptr, fmem = _fptr(fock), MEM_HOST
    else:
        fptr, fmem = ctypes.c_void_p(0), MEM_HOST
    st = lib().uw12c_form_fock(W.handle, V.handle, WV.handle, abs_p.handle, n_ao, n_spin, c_ptrs,
                               ldc, norb, o_ptrs, nocc, nact, int(bool(indirect_term)),
                               int(bool(calculate_fock)), float(scale_opp_spin),
                               float(scale_same_spin), int(print_level), ctypes.byref(energy),
                               terms, fptr, fmem)
    _check(st)
    focks = None
    if fock is not None:
        focks = [np.array(fock[:, s * n_ao:(s + 1) * n_ao]) for s in range(n_spin)]
    return energy.value, focks, (terms[0], terms[1], terms[2])


class _Molecule(ctypes.Structure):
    _fields_ = [("W", ctypes.c_void_p), ("V", ctypes.c_void_p), ("WV", ctypes.c_void_p),
                ("abs", ctypes.c_void_p), ("n_ao", ctypes.c_size_t), ("n_spin", ctypes.c_size_t),
                ("C", ctypes.c_void_p), ("ldc", ctypes.c_void_p), ("n_orb", ctypes.c_void_p),
                ("occ", ctypes.c_void_p), ("n_occ", ctypes.c_void_p),
                ("n_active", ctypes.c_void_p), ("energy", ctypes.c_void_p),
                ("terms", ctypes.c_void_p), ("fock", ctypes.c_void_p),
                ("fock_mem_kind", ctypes.c_int)]


def fock_batched(molecules: Sequence[dict], indirect_term: bool, calculate_fock: bool,
                 scale_opp_spin: float, scale_same_spin: float, n_streams: int = 8):
    """``uw12c_fock_batched``: ``form_fock`` for many molecules in one call.

    Each molecule is a dict with W, V, WV (BaseIntegrals), abs (ABSProjectors),
    orbitals, occ and n_active as for ``form_fock``.  Returns a list of
    ``(energy, fock, (E2, E3, E4))`` in input order.
    """
    keep = []  # ctypes arrays and numpy buffers alive until the call returns
    arr = (_Molecule * max(1, len(molecules)))()
    outs = []
    P = ctypes.c_void_p
    for i, m in enumerate(molecules):
        n_spin = len(m["orbitals"])
        n_ao = m["W"].n_ao
        Cs = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in m["orbitals"]]
        occs = [np.ascontiguousarray(np.asarray(o, dtype=np.float64).reshape(-1))
                for o in m["occ"]]
        c_ptrs = (P * n_spin)(*[_fptr(c) for c in Cs])
        ldc = (ctypes.c_size_t * n_spin)(*[max(1, c.shape[0]) for c in Cs])
        norb = (ctypes.c_size_t * n_spin)(*[c.shape[1] for c in Cs])
        o_ptrs = (P * n_spin)(*[_fptr(o) for o in occs])
        nocc = (ctypes.c_size_t * n_spin)(*[o.size for o in occs])
        nact = (ctypes.c_size_t * n_spin)(*[int(a) for a in m["n_active"]])
        energy = ctypes.c_double()
        terms = (ctypes.c_double * 3)()
        fock = np.zeros((n_ao, n_ao * n_spin), order="F") if calculate_fock else None
        keep += [Cs, occs, c_ptrs, ldc, norb, o_ptrs, nocc, nact, energy, terms, fock]
        arr[i] = _Molecule(m["W"].handle, m["V"].handle, m["WV"].handle, m["abs"].handle, n_ao,
                           n_spin, ctypes.cast(c_ptrs, P), ctypes.cast(ldc, P),
                           ctypes.cast(norb, P), ctypes.cast(o_ptrs, P), ctypes.cast(nocc, P),
                           ctypes.cast(nact, P), ctypes.cast(ctypes.pointer(energy), P),
                           ctypes.cast(terms, P), _fptr(fock) if fock is not None else P(0),
                           MEM_HOST)
        outs.append((energy, fock, terms, n_ao, n_spin))
    statuses = (ctypes.c_int * max(1, len(molecules)))()
    _check(lib().uw12c_fock_batched(ctypes.cast(arr, P), len(molecules),
                                    int(bool(indirect_term)), int(bool(calculate_fock)),
                                    float(scale_opp_spin), float(scale_same_spin),
                                    int(n_streams), statuses))
    res = []
    for energy, fock, terms, n_ao, n_spin in outs:
        focks = None
        if fock is not None:
            focks = [np.array(fock[:, s * n_ao:(s + 1) * n_ao]) for s in range(n_spin)]
        res.append((energy.value, focks, (terms[0], terms[1], terms[2])))
    return res


GRADIENT_NAMES = ("W3", "V3", "WV3", "W3_ri", "V3_ri", "W2", "V2", "WV2")


def fock_backward(W: BaseIntegrals, V: BaseIntegrals, WV: BaseIntegrals, abs_p: ABSProjectors,
                  orbitals: Sequence[np.ndarray], occupations: Sequence[np.ndarray],
                  n_active: Sequence[int], scale_opp_spin: float, scale_same_spin: float,
                  gradients: Sequence[str] = GRADIENT_NAMES, calculate_fock: bool = True,
                  device_out: Optional[dict] = None, indirect_term: bool = False,
                  host_out: Optional[dict] = None):
    """Reverse mode of ``form_fock`` (``uw12c_fock_backward``).

    Returns ``(energy, fock, (E2, E3, E4), grads)``: the energy, per-spin Fock
    and terms of ``form_fock(..., indirect_term, ...)`` (the direct terms only
    by default; with ``indirect_term`` and ``scale_same_spin != 0`` the
    same-spin terms too, the energy of ``uw12_energy``) and a dict of the
    requested gradients of that energy with respect to the stored integrals
    ("W3", "V3", "WV3" packed n_ao(n_ao+1)/2 x n_df; "W3_ri", "V3_ri"
    (n_ri n_ao) x n_df; "W2", "V2", "WV2" n_df x n_df).  With ``device_out``
    (name -> device pointer) the gradients are written to device memory and
    the dict is empty; with ``host_out`` (name -> Fortran-ordered float64 host
    array of the gradient's shape, e.g. a view of pinned memory) those arrays
    are filled and returned instead of new ones.
    """
    n_spin = len(orbitals)
    if n_spin < 1 or n_spin > 2 or len(occupations) != n_spin or len(n_active) != n_spin:
        raise UW12LogicError("invalid number of spin channels")
    n_ao = W.n_ao
    Cs = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in orbitals]
    occs = [np.ascontiguousarray(np.asarray(o, dtype=np.float64).reshape(-1)) for o in occupations]
    P = ctypes.c_void_p
    c_ptrs = (P * n_spin)(*[_fptr(c) for c in Cs])
    ldc = (ctypes.c_size_t * n_spin)(*[max(1, c.shape[0]) for c in Cs])
    norb = (ctypes.c_size_t * n_spin)(*[c.shape[1] for c in Cs])
    o_ptrs = (P * n_spin)(*[_fptr(o) for o in occs])
    nocc = (ctypes.c_size_t * n_spin)(*[o.size for o in occs])
    nact = (ctypes.c_size_t * n_spin)(*[int(a) for a in n_active])
    shapes = {"W3": (W.n_ao * (W.n_ao + 1) // 2, W.n_df), "V3": (V.n_ao * (V.n_ao + 1) // 2, V.n_df),
              "WV3": (WV.n_ao * (WV.n_ao + 1) // 2, WV.n_df),
              "W3_ri": (W.n_ri * W.n_ao, W.n_df), "V3_ri": (V.n_ri * V.n_ao, V.n_df),
              "W2": (W.n_df, W.n_df), "V2": (V.n_df, V.n_df), "WV2": (WV.n_df, WV.n_df)}
    grads, ptr = {}, {}
    for name in GRADIENT_NAMES:
        if device_out is not None:
            ptr[name] = P(device_out[name]) if name in device_out else P(0)
        elif host_out is not None and name in host_out:
            arr = host_out[name]
            if (arr.shape != shapes[name] or arr.dtype != np.float64
                    or not arr.flags.f_contiguous):
                raise UW12LogicError(f"host_out[{name!r}] must be float64 F-ordered {shapes[name]}")
            grads[name] = arr
            ptr[name] = _fptr(arr)
        elif name in gradients:
            grads[name] = np.zeros(shapes[name], order="F")
            ptr[name] = _fptr(grads[name])
        else:
            ptr[name] = P(0)
    d3 = (P * 3)(ptr["W3"], ptr["V3"], ptr["WV3"])
    d3ri = (P * 2)(ptr["W3_ri"], ptr["V3_ri"])
    d2 = (P * 3)(ptr["W2"], ptr["V2"], ptr["WV2"])
    energy = ctypes.c_double()
    terms = (ctypes.c_double * 3)()
    fock = np.zeros((n_ao, n_ao * n_spin), order="F") if calculate_fock else None
    _check(lib().uw12c_fock_backward(W.handle, V.handle, WV.handle, abs_p.handle, n_ao, n_spin,
                                     c_ptrs, ldc, norb, o_ptrs, nocc, nact,
                                     int(bool(indirect_term)), float(scale_opp_spin),
                                     float(scale_same_spin), ctypes.byref(energy), terms,
                                     _fptr(fock) if fock is not None else P(0), MEM_HOST, d3,
                                     d3ri, d2, MEM_DEVICE if device_out is not None else MEM_HOST))
    focks = None
    if fock is not None:
        focks = [np.array(fock[:, s * n_ao:(s + 1) * n_ao]) for s in range(n_spin)]
    return energy.value, focks, (terms[0], terms[1], terms[2]), grads


SINK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                           ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
BLOCK_GRADIENT_NAMES = ("W3", "V3", "WV3", "W3_ri", "V3_ri")


def sink_norm2() -> int:
    """Address of ``uw12c_sink_norm2``, a native device sink (user = device
    double that accumulates the squared norm of the blocks)."""
    return ctypes.cast(lib().uw12c_sink_norm2, ctypes.c_void_p).value


def fock_backward_blocks(W: BaseIntegrals, V: BaseIntegrals, WV: BaseIntegrals,
                         abs_p: ABSProjectors, orbitals: Sequence[np.ndarray],
                         occupations: Sequence[np.ndarray], n_active: Sequence[int],
                         scale_opp_spin: float, scale_same_spin: float, sinks: dict,
                         metric_gradients: Sequence[str] = ("W2", "V2", "WV2"),
                         calculate_fock: bool = True, device: bool = False,
                         users: Optional[dict] = None, indirect_term: bool = False):
    """``uw12c_fock_backward_blocks``: the three-index gradients delivered in aux
    blocks (``indirect_term`` as for ``fock_backward``).  ``sinks`` maps names of
    ``BLOCK_GRADIENT_NAMES`` to Python callables
    ``f(first, count, block)`` (``block`` a host ``rows x count`` array, valid
    during the call; ``device=False``) or to C function pointers (ints) with
    ``users[name]`` as their user pointer (``device=True`` passes device
    blocks).  Returns ``(energy, fock, (E2, E3, E4), metric_grads)``."""
    n_spin = len(orbitals)
    if n_spin < 1 or n_spin > 2 or len(occupations) != n_spin or len(n_active) != n_spin:
        raise UW12LogicError("invalid number of spin channels")
    n_ao = W.n_ao
    Cs = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in orbitals]
    occs = [np.ascontiguousarray(np.asarray(o, dtype=np.float64).reshape(-1)) for o in occupations]
    P = ctypes.c_void_p
    c_ptrs = (P * n_spin)(*[_fptr(c) for c in Cs])
    ldc = (ctypes.c_size_t * n_spin)(*[max(1, c.shape[0]) for c in Cs])
    norb = (ctypes.c_size_t * n_spin)(*[c.shape[1] for c in Cs])
    o_ptrs = (P * n_spin)(*[_fptr(o) for o in occs])
    nocc = (ctypes.c_size_t * n_spin)(*[o.size for o in occs])
    nact = (ctypes.c_size_t * n_spin)(*[int(a) for a in n_active])
    users = users or {}
    keep = []  # callbacks stay alive for the call

    def as_sink(name):
        f = sinks.get(name)
        if f is None:
            return P(0)
        if isinstance(f, int):
            return P(f)

        def cb(user, first, count, block, ld, stream):
            try:
                view = np.ctypeslib.as_array(ctypes.cast(block, ctypes.POINTER(ctypes.c_double)),
                                             shape=(ld * count,)).reshape((ld, count), order="F")
                f(int(first), int(count), view)
                return 0
            except Exception:  # reported by the library as a runtime error
                return 1
        c = SINK_FN(cb)
        keep.append(c)
        return ctypes.cast(c, P)

    s3 = (P * 3)(*[as_sink(n) for n in ("W3", "V3", "WV3")])
    s3ri = (P * 2)(*[as_sink(n) for n in ("W3_ri", "V3_ri")])
    u3 = (P * 3)(*[P(users.get(n, 0)) for n in ("W3", "V3", "WV3")])
    u3ri = (P * 2)(*[P(users.get(n, 0)) for n in ("W3_ri", "V3_ri")])
    shapes = {"W2": (W.n_df, W.n_df), "V2": (V.n_df, V.n_df), "WV2": (WV.n_df, WV.n_df)}
    grads = {n: np.zeros(shapes[n], order="F") for n in metric_gradients}
    d2 = (P * 3)(*[_fptr(grads[n]) if n in grads else P(0) for n in ("W2", "V2", "WV2")])
    energy = ctypes.c_double()
    terms = (ctypes.c_double * 3)()
    fock = np.zeros((n_ao, n_ao * n_spin), order="F") if calculate_fock else None
    _check(lib().uw12c_fock_backward_blocks(
        W.handle, V.handle, WV.handle, abs_p.handle, n_ao, n_spin, c_ptrs, ldc, norb, o_ptrs,
        nocc, nact, int(bool(indirect_term)), float(scale_opp_spin), float(scale_same_spin),
        ctypes.byref(energy), terms, _fptr(fock) if fock is not None else P(0), MEM_HOST, s3, u3,
        s3ri, u3ri,
        MEM_DEVICE if device else MEM_HOST, d2, MEM_HOST))
    focks = None
    if fock is not None:
        focks = [np.array(fock[:, s * n_ao:(s + 1) * n_ao]) for s in range(n_spin)]
    return energy.value, focks, (terms[0], terms[1], terms[2]), grads


def uw12_fock(W, V, WV, abs_p, orbitals, occ, n_active, scale_opp_spin, scale_same_spin,
              print_level: int = 0) -> Tuple[float, np.ndarray]:
    """``uw12::uw12_fock`` (libuw12.hpp:157-169): returns (energy, fock) with
    fock of shape n_ao x (n_ao * n_spin)."""
    indirect = not _nearly_zero(scale_same_spin)
    e, f, _ = form_fock(W, V, WV, abs_p, orbitals, occ, n_active, indirect, True, scale_opp_spin,
                        scale_same_spin, print_level)
    return e, np.concatenate(f, axis=1)


def uw12_energy(W, V, WV, abs_p, orbitals, occ, n_active, scale_opp_spin, scale_same_spin,
                print_level: int = 0) -> float:
    """``uw12::uw12_energy`` (libuw12.hpp:129-140)."""
    indirect = not _nearly_zero(scale_same_spin)
    return form_fock(W, V, WV, abs_p, orbitals, occ, n_active, indirect, False, scale_opp_spin,
                     scale_same_spin, print_level)[0]


def set_stream(stream_ptr: int):
    _check(lib().uw12c_set_stream(ctypes.c_void_p(stream_ptr)))


def set_shard(shard: int, n_shards: int):
    """Evaluate only part `shard` of `n_shards` in subsequent calls on this thread
    (partial energies and Fock matrices sum to the full result; a sharded
    evaluation needs an all-reduce, set_allreduce)."""
    _check(lib().uw12c_set_shard(int(shard), int(n_shards)))


# fn(data, count, stream, user) -> 0: sums `count` doubles at device address
# `data` over the shards, ordered on the cudaStream_t `stream`
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                ctypes.c_void_p)
_allreduce_keep = threading.local()


def set_allreduce(fn: Optional[Callable[[int, int, int], None]]):
    """The all-reduce of sharded evaluations on this host thread
    (uw12c_set_allreduce): ``fn(data_ptr, count, stream_ptr)`` replaces the
    ``count`` float64 values at device address ``data_ptr`` by their sum over
    the shards, ordered on the CUDA stream ``stream_ptr``; an exception fails
    the evaluation.  None removes it."""
    if fn is None:
        _check(lib().uw12c_set_allreduce(ALLREDUCE_FN(), None))
        _allreduce_keep.cb = None
        return

    def tramp(data, count, stream, user):
        try:
            fn(int(data or 0), int(count), int(stream or 0))
            return 0
        except Exception as exc:  # reported through the evaluation's status
            _allreduce_keep.error = exc
            return 1

    cb = ALLREDUCE_FN(tramp)
    _check(lib().uw12c_set_allreduce(cb, None))
    _allreduce_keep.cb = cb  # the C side holds only the pointer


def trim_memory():
    """Return the device memory the library keeps reserved between calls."""
    _check(lib().uw12c_trim_memory())


def set_memory_budget(nbytes: int):
    _check(lib().uw12c_set_memory_budget(int(nbytes)))


def launch_count() -> int:
    return int(lib().uw12c_launch_count())


def profile_enable(on: bool):
    _check(lib().uw12c_profile_enable(1 if on else 0))


def profile_read():
    n = ctypes.c_ulonglong()
    ms = ctypes.c_double()
    fl = ctypes.c_double()
    _check(lib().uw12c_profile_read(ctypes.byref(n), ctypes.byref(ms), ctypes.byref(fl)))
    return {"launches": n.value, "ms": ms.value, "flops": fl.value}


def dgemm(m, n, k, alpha, A, lda, a_kcontig, B, ldb, b_ncontig, beta, C, ldc, nbo1=1, nbo2=1,
          so=(0, 0, 0, 0, 0, 0), nbr1=1, nbr2=1, sr=(0, 0, 0, 0), split=0):
    """The FP64 tensor-core GEMM engine on device pointers (see uw12_c.h)."""
    LLa = ctypes.c_longlong * 6
    LLr = ctypes.c_longlong * 4
    _check(lib().uw12c_dgemm(m, n, k, alpha, ctypes.c_void_p(A), lda, int(a_kcontig),
                             ctypes.c_void_p(B), ldb, int(b_ncontig), beta, ctypes.c_void_p(C),
                             ldc, nbo1, nbo2, LLa(*so), nbr1, nbr2, LLr(*sr), int(split)))


def dgemm_split(m, n, k, alpha, A, lda, a_kcontig, B, ldb, b_ncontig, beta, C, ldc, nbo1=1,
                nbo2=1, so=(0, 0, 0, 0, 0, 0), nbr1=1, nbr2=1, sr=(0, 0, 0, 0), n_moduli=14):
    """``dgemm`` computed by the split-precision (int8 tensor-core, CRT) GEMM."""
    LLa = ctypes.c_longlong * 6
    LLr = ctypes.c_longlong * 4
    _check(lib().uw12c_dgemm_split(m, n, k, alpha, ctypes.c_void_p(A), lda, int(a_kcontig),
                                   ctypes.c_void_p(B), ldb, int(b_ncontig), beta,
                                   ctypes.c_void_p(C), ldc, nbo1, nbo2, LLa(*so), nbr1, nbr2,
                                   LLr(*sr), int(n_moduli)))


def set_precision(n_moduli: int):
    """Split-precision GEMMs with ``n_moduli`` moduli in subsequent evaluations on
    this thread (0 = FP64)."""
    _check(lib().uw12c_set_precision(int(n_moduli)))


def form_fock_split(W: BaseIntegrals, V: BaseIntegrals, WV: BaseIntegrals,
                    abs_p: ABSProjectors, orbitals: Sequence[np.ndarray],
                    occupations: Sequence[np.ndarray], n_active: Sequence[int],
                    indirect_term: bool, calculate_fock: bool, scale_opp_spin: float,
                    scale_same_spin: float, n_moduli: int = 14):
    """``form_fock`` in split precision (``n_moduli`` moduli) with the error of
    its result against the FP64 evaluation stated in Hartree.

    Returns ``(energy, fock, (E2, E3, E4), errors)`` where ``errors`` holds
    ``energy_Eh`` = |E_split - E_FP64|, ``terms_Eh`` (the same per term),
    ``fock_max_Eh`` = max |F_split - F_FP64| over both spins (None without
    Fock) and ``n_moduli``.  The FP64 result is the plain GPU path on the same
    handles (libuw12's arithmetic in FP64), so the call costs one evaluation of
    each kind.  The calling thread is left in FP64 mode (precision 0).
    """
    args = (W, V, WV, abs_p, orbitals, occupations, n_active, indirect_term, calculate_fock,
            scale_opp_spin, scale_same_spin)
    set_precision(n_moduli)
    try:
        e, f, t = form_fock(*args)
    finally:
        set_precision(0)
    e64, f64, t64 = form_fock(*args)
    errors = {"energy_Eh": abs(e - e64),
              "terms_Eh": tuple(abs(a - b) for a, b in zip(t, t64)),
              "fock_max_Eh": (max(float(np.max(np.abs(a - b))) for a, b in zip(f, f64))
                              if f is not None else None),
              "n_moduli": int(n_moduli)}
    return e, f, t, errors


def set_split_threshold(min_flops: float):
    """GEMMs below ``min_flops`` stay FP64 in split-precision mode (default 2e9)."""
    _check(lib().uw12c_set_split_threshold(float(min_flops)))


def split_bits(n_moduli: int, k_total: int) -> int:
    """Bits kept per operand element by a split-precision GEMM."""
    b = ctypes.c_int()
    _check(lib().uw12c_split_bits(int(n_moduli), int(k_total), ctypes.byref(b)))
    return b.value


AUTOTUNE_OFF, AUTOTUNE_TUNE, AUTOTUNE_USE = 0, 1, 2


def autotune(mode: int, path: Optional[str] = None):
    """Split-K autotuner of the FP64 GEMM engine (``uw12c_autotune``): mode 0
    the wave rule, 1 time every candidate split of each new shape class and
    keep the fastest, 2 use the table only; ``path`` (a table written by
    ``autotune_save``) is merged into the table first when it exists."""
    _check(lib().uw12c_autotune(int(mode), os.fsencode(path) if path else None))


def autotune_save(path: str):
    _check(lib().uw12c_autotune_save(os.fsencode(path)))


def autotune_clear():
    _check(lib().uw12c_autotune_clear())


def autotune_size() -> int:
    n = ctypes.c_longlong()
    _check(lib().uw12c_autotune_size(ctypes.byref(n)))
    return n.value


def autotune_lookup(m: int, n: int, k: int, nbo: int = 1, nbr: int = 1) -> int:
    """The table's split for a GEMM of this shape (0: not in the table)."""
    s = ctypes.c_int()
    _check(lib().uw12c_autotune_lookup(int(m), int(n), int(k), int(nbo), int(nbr),
                                       ctypes.byref(s)))
    return s.value


PROFILE_KINDS = ("dgemm", "split_gemm", "i8_mma", "split_prep", "split_crt", "producer")


def profile_read_kind(kind: str) -> dict:
    """Launches, milliseconds and work (FLOPs, int8 ops or bytes) of a kernel class."""
    n, ms, w = ctypes.c_ulonglong(), ctypes.c_double(), ctypes.c_double()
    _check(lib().uw12c_profile_read_kind(PROFILE_KINDS.index(kind), ctypes.byref(n),
                                         ctypes.byref(ms), ctypes.byref(w)))
    return {"launches": n.value, "ms": ms.value, "work": w.value}


def profile_phases() -> dict:
    """Device milliseconds per evaluation phase since the last read."""
    buf = ctypes.create_string_buffer(4096)
    _check(lib().uw12c_profile_phases(buf, 4096))
    out = {}
    for item in buf.value.decode().split(";"):
        if "=" in item:
            k, v = item.split("=", 1)
            out[k] = float(v)
    return out


def synth_three_index(out_ptr: int, kind: int, n_ao: int, n_ri: int, n_df: int, seed: int,
                      tag: int, decay: float):
    _check(lib().uw12c_synth_three_index(ctypes.c_void_p(out_ptr), kind, n_ao, n_ri, n_df,
                                         seed & (2**64 - 1), tag & (2**64 - 1), decay))
