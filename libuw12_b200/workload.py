"""Seeded synthetic UW12 workloads (the benchmark configurations).

No public dataset exists for this path; the configurations are described by
generators: AO+RI overlap ``A A^T + 0.1 I`` (A ~ N(0, 1/(N+R))), occupied
orbitals S-orthonormalised (``C^T S C = I``), three-index tensors
``N(0,1) exp(-|m-n|/L)`` in libuw12's layouts (packed ``Np x M`` with row
``i(i+1)/2 + j``, RI ``(R N) x M`` with row ``nu + R mu``), metrics
``B B^T + 1e-6 I`` (B ~ N(0, 1/M)).  Every value is a pure function of
(seed, tensor name, element index):

    key = mix(mix(seed) ^ tag(name)),   h_k = mix(key + 2 e + k)   (k = 0, 1)
    u1 = ((h_0 >> 11) + 1) 2^-53,  u2 = (h_1 >> 11) 2^-53
    g  = sqrt(-2 ln u1) cos(2 pi u2)

with ``mix`` the SplitMix64 finaliser and ``tag`` the first 8 bytes of the
name's SHA-256, so the benchmark's host inputs, the library's device producer
``uw12c_synth_three_index`` (same formula on the GPU) and any other consumer
of the same seed see the same tensors.  Arrays can be filled in place
(``out=``), e.g. straight into pinned host buffers.
"""
from __future__ import annotations

import hashlib
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

import numpy as np

_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_U64 = (1 << 64) - 1


def _mix_int(x: int) -> int:
    z = (x + 0x9E3779B97F4A7C15) & _U64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _U64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _U64
    return z ^ (z >> 31)


def tag(name: str) -> int:
    """64-bit tag of a tensor name (the first 8 bytes of its SHA-256, little endian)."""
    return int.from_bytes(hashlib.sha256(name.encode()).digest()[:8], "little")


def key_of(seed: int, name: str) -> int:
    return _mix_int(_mix_int(seed & _U64) ^ tag(name))


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = z + _GOLD
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def gaussians(key: int, start: int, count: int) -> np.ndarray:
    """The standard normals of elements start .. start + count - 1 of a stream."""
    e = np.arange(start, start + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = np.uint64(key) + np.uint64(2) * e
        h0 = _mix(base)
        h1 = _mix(base + np.uint64(1))
    u1 = ((h0 >> np.uint64(11)).astype(np.float64) + 1.0) * float(2.0 ** -53)
    u2 = (h1 >> np.uint64(11)).astype(np.float64) * float(2.0 ** -53)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def _fill(flat: np.ndarray, fn, chunk: int = 1 << 22) -> None:
    n = flat.size
    starts = list(range(0, n, chunk))
    if len(starts) <= 1:
        if n:
            fn(0, n)
        return
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        list(ex.map(lambda s: fn(s, min(n, s + chunk)), starts))


def _column_major(rows: int, cols: int, out: Optional[np.ndarray]) -> np.ndarray:
    if out is None:
        return np.empty(rows * cols, dtype=np.float64)
    flat = out.reshape(-1, order="F") if out.ndim > 1 else out
    if flat.size != rows * cols or flat.dtype != np.float64 or not flat.flags.c_contiguous:
        raise ValueError("out must be a contiguous float64 buffer of rows x cols")
    return flat


def three_index_ao(seed: int, name: str, n_ao: int, n_df: int, decay: float,
                   out: Optional[np.ndarray] = None) -> np.ndarray:
    """Packed (P|mn), ``Np x M`` column-major: g * exp(-|m-n|/decay)."""
    npk = n_ao * (n_ao + 1) // 2
    r, c = np.tril_indices(n_ao)
    damp = np.exp(-np.abs(r - c).astype(np.float64) / decay)
    key = key_of(seed, name)
    flat = _column_major(npk, n_df, out)

    def fill(s, e):
        flat[s:e] = gaussians(key, s, e - s) * damp[np.arange(s, e) % npk]

    _fill(flat, fill)
    return flat.reshape((npk, n_df), order="F")


def three_index_ri(seed: int, name: str, n_ao: int, n_ri: int, n_df: int, decay: float,
                   out: Optional[np.ndarray] = None) -> np.ndarray:
    """(P|nu mu), ``(R N) x M`` column-major, row nu + R mu: g * exp(-|nu-mu|/decay)."""
    nr = n_ri * n_ao
    nu = np.arange(nr) % n_ri
    mu = np.arange(nr) // n_ri
    damp = np.exp(-np.abs(nu - mu).astype(np.float64) / decay)
    key = key_of(seed, name)
    flat = _column_major(nr, n_df, out)

    def fill(s, e):
        flat[s:e] = gaussians(key, s, e - s) * damp[np.arange(s, e) % nr]

    _fill(flat, fill)
    return flat.reshape((nr, n_df), order="F")


def gaussian_matrix(seed: int, name: str, n_rows: int, n_cols: int,
                    scale: float = 1.0) -> np.ndarray:
    return (gaussians(key_of(seed, name), 0, n_rows * n_cols) * scale).reshape(
        (n_rows, n_cols), order="F")


def metric(seed: int, name: str, n_df: int) -> np.ndarray:
    """(P|Q) = B B^T + 1e-6 I, B ~ N(0, 1/M) (condition number up to ~1e6)."""
    B = gaussian_matrix(seed, name, n_df, n_df, 1.0 / np.sqrt(n_df))
    J2 = B @ B.T + 1e-6 * np.eye(n_df)
    return 0.5 * (J2 + J2.T)


def overlap(seed: int, n_ao: int, n_ri: int) -> np.ndarray:
    """Combined AO + RI overlap A A^T + 0.1 I, AO block first."""
    n = n_ao + n_ri
    A = gaussian_matrix(seed, "S", n, n, 1.0 / np.sqrt(n))
    S = A @ A.T + 0.1 * np.eye(n)
    return 0.5 * (S + S.T)


def orbitals(seed: int, S_ao: np.ndarray, n_orb: int, name: str) -> np.ndarray:
    """C ~ N(0, 1), orthonormalised so that C^T S C = I (Cholesky of C^T S C)."""
    C = gaussian_matrix(seed, name, S_ao.shape[0], n_orb)
    if n_orb == 0:
        return C
    G = C.T @ S_ao @ C
    L = np.linalg.cholesky(0.5 * (G + G.T))
    return np.linalg.solve(L, C.T).T


@dataclass
class Workload:
    name: str
    n_ao: int
    n_df: int
    n_ri: int
    n_occ: Tuple[int, ...]   # per spin: (n,) closed shell, (n_alpha, n_beta) open
    decay: float

    @property
    def n_spin(self) -> int:
        return len(self.n_occ)


CONFIGS: Dict[str, Workload] = {
    "c0": Workload("c0", 24, 84, 116, (5,), 8.0),
    "c1": Workload("c1", 500, 1500, 2000, (40, 38), 30.0),
    "c1s": Workload("c1s", 200, 600, 800, (16, 15), 30.0),
    "c2": Workload("c2", 1200, 3600, 4800, (100,), 30.0),
    "c3": Workload("c3", 2000, 6000, 8000, (170, 170), 30.0),
}

THREE_INDEX = ("W3", "V3", "WV3", "W3_ri", "V3_ri")
TWO_INDEX = ("W2", "V2", "WV2")


def tensor_shape(w: Workload, name: str) -> Tuple[int, int]:
    N, M, R = w.n_ao, w.n_df, w.n_ri
    if name in ("W3", "V3", "WV3"):
        return N * (N + 1) // 2, M
    if name in ("W3_ri", "V3_ri"):
        return R * N, M
    if name in TWO_INDEX:
        return M, M
    raise KeyError(name)


def make_three_index(w: Workload, name: str, seed: int = 11,
                     out: Optional[np.ndarray] = None) -> np.ndarray:
    if name.endswith("_ri"):
        return three_index_ri(seed, name, w.n_ao, w.n_ri, w.n_df, w.decay, out)
    return three_index_ao(seed, name, w.n_ao, w.n_df, w.decay, out)


def make_small(w: Workload, seed: int = 11) -> dict:
    """Metrics, overlap, orbitals (per spin, n_occ[s] columns) and occupations
    (2 closed shell, 1 open shell)."""
    N, R = w.n_ao, w.n_ri
    out = {nm: metric(seed, nm, w.n_df) for nm in TWO_INDEX}
    out["S"] = overlap(seed, N, R)
    out["orbitals"] = [orbitals(seed, out["S"][:N, :N], max(o, 1), f"C{s}")[:, :max(o, 1)]
                       for s, o in enumerate(w.n_occ)]
    per = 2.0 if w.n_spin == 1 else 1.0
    out["occ"] = [np.full(o, per) for o in w.n_occ]
    return out


def batch_molecules(n_mol: int = 64, seed: int = 2024) -> List[Tuple[Workload, int]]:
    """The 64-molecule batch: N ~ U[20, 300] (numpy default_rng(seed)), M = 3N,
    R = 4N, n_occ = round(N/10), even index closed shell, odd index UHF with
    n_beta = n_alpha - 1, decay 8; molecule i uses seed 1000 seed + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_mol):
        N = int(rng.integers(20, 301))
        o = max(1, int(round(N / 10)))
        occ = (o,) if i % 2 == 0 else (o, max(1, o - 1))
        out.append((Workload(f"mol{i}", N, 3 * N, 4 * N, occ, 8.0), seed * 1000 + i))
    return out
