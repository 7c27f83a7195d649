"""Seeded synthetic UW12 inputs -- TEST INFRASTRUCTURE ONLY.

The reference quotes no public dataset; its benchmark configurations are
described by generators (AO overlap ``S = A A^T + 0.1 I``, S-orthonormal
occupied orbitals, three-index tensors ``N(0,1) * exp(-|m-n|/L)`` symmetric in
``m,n``, metrics ``B B^T + 1e-6 I``).  This module restates those generators
with a counter-based RNG so that every tensor element is a pure function of
``(seed, tag, index)``:

    key   = mix(mix(seed) ^ tag)
    h_k   = mix(key + 2*index + k)                  k = 0, 1   (wrapping u64)
    u1    = ((h_0 >> 11) + 1) * 2**-53               in (0, 1]
    u2    =  (h_1 >> 11)      * 2**-53               in [0, 1)
    g     = sqrt(-2 ln u1) * cos(2 pi u2)            (Box-Muller)

``mix`` is the SplitMix64 finaliser.  ``libuw12_b200/csrc/synth.cu`` evaluates
the same formula on the GPU for the large benchmark tensors (values agree to
libm rounding, ~1e-15 relative).

Layouts are libuw12's: packed AO tensor ``Np x M`` with row
``i(i+1)/2 + j`` (j <= i) for pair (i, j); RI tensor ``(R*N) x M`` with row
``nu + R*mu``; everything column-major (``order='F'`` on the numpy side).
"""
from __future__ import annotations

import hashlib
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_2M53 = float(2.0 ** -53)


def _mix_scalar(x: int) -> int:
    m = (1 << 64) - 1
    z = (x + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def tag_of(name: str) -> int:
    """64-bit tag of a tensor name (first 8 bytes of its SHA-256)."""
    return int.from_bytes(hashlib.sha256(name.encode()).digest()[:8], "little")


def stream_key(seed: int, name: str) -> int:
    return _mix_scalar(_mix_scalar(seed & ((1 << 64) - 1)) ^ tag_of(name))


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = z + _GOLD
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def normals(key: int, start: int, count: int) -> np.ndarray:
    """Standard normals for counters ``start .. start+count-1`` of a stream."""
    idx = np.arange(start, start + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = np.uint64(key) + np.uint64(2) * idx
        h0 = _mix(base)
        h1 = _mix(base + np.uint64(1))
    u1 = ((h0 >> np.uint64(11)).astype(np.float64) + 1.0) * _2M53
    u2 = (h1 >> np.uint64(11)).astype(np.float64) * _2M53
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def _parallel_fill(out_flat: np.ndarray, fn, chunk: int = 1 << 22):
    n = out_flat.size
    starts = list(range(0, n, chunk))
    if len(starts) <= 1:
        if n:
            fn(0, n)
        return

    def work(s):
        fn(s, min(n, s + chunk))

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        list(ex.map(work, starts))


def three_index_ao(seed: int, name: str, n_ao: int, n_df: int, decay: float) -> np.ndarray:
    """Packed (P|mn): ``Np x M`` column-major, value g * exp(-|m-n|/L)."""
    np_ = n_ao * (n_ao + 1) // 2
    rows, cols = np.tril_indices(n_ao)
    damp = np.exp(-np.abs(rows - cols).astype(np.float64) / decay)
    key = stream_key(seed, name)
    out = np.empty(np_ * n_df, dtype=np.float64)

    def fill(s, e):
        out[s:e] = normals(key, s, e - s) * damp[np.arange(s, e) % np_]

    _parallel_fill(out, fill)
    return out.reshape((np_, n_df), order="F")


def three_index_ri(seed: int, name: str, n_ao: int, n_ri: int, n_df: int, decay: float) -> np.ndarray:
    """(P|nu mu): ``(R*N) x M`` column-major, row nu + R*mu, g * exp(-|nu-mu|/L)."""
    nr = n_ri * n_ao
    nu = np.arange(nr) % n_ri
    mu = np.arange(nr) // n_ri
    damp = np.exp(-np.abs(nu - mu).astype(np.float64) / decay)
    key = stream_key(seed, name)
    out = np.empty(nr * n_df, dtype=np.float64)

    def fill(s, e):
        out[s:e] = normals(key, s, e - s) * damp[np.arange(s, e) % nr]

    _parallel_fill(out, fill)
    return out.reshape((nr, n_df), order="F")


def fast_three_index(seed: int, name: str, n_rows: int, n_df: int, damp: np.ndarray) -> np.ndarray:
    """Same distribution as ``three_index_ao`` / ``three_index_ri`` (value
    g * damp[row]) from numpy's PCG64 streams, multithreaded; used only where
    benchmark-sized host inputs are needed quickly and exact values do not
    matter (CPU baseline timing)."""
    out = np.empty((n_rows, n_df), order="F")
    flat = out.reshape(-1, order="F")
    ss = np.random.SeedSequence([seed, tag_of(name) & 0xFFFFFFFF])
    chunk = 1 << 24
    starts = list(range(0, flat.size, chunk))
    children = ss.spawn(len(starts))

    def work(q):
        s = starts[q]
        e = min(flat.size, s + chunk)
        g = np.random.Generator(np.random.PCG64(children[q]))
        g.standard_normal(out=flat[s:e])
        flat[s:e] *= damp[np.arange(s, e) % n_rows]

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        list(ex.map(work, range(len(starts))))
    return out


def ao_damping(n_ao: int, decay: float) -> np.ndarray:
    rows, cols = np.tril_indices(n_ao)
    return np.exp(-np.abs(rows - cols).astype(np.float64) / decay)


def ri_damping(n_ao: int, n_ri: int, decay: float) -> np.ndarray:
    nr = n_ri * n_ao
    return np.exp(-np.abs(np.arange(nr) % n_ri - np.arange(nr) // n_ri).astype(np.float64) / decay)


def gaussian_matrix(seed: int, name: str, n_rows: int, n_cols: int, scale: float = 1.0) -> np.ndarray:
    key = stream_key(seed, name)
    return (normals(key, 0, n_rows * n_cols) * scale).reshape((n_rows, n_cols), order="F")


def metric(seed: int, name: str, n_df: int) -> np.ndarray:
    """(P|Q) = B B^T + 1e-6 I with B ~ N(0, 1/M)."""
    B = gaussian_matrix(seed, name, n_df, n_df, 1.0 / np.sqrt(n_df))
    J2 = B @ B.T + 1e-6 * np.eye(n_df)
    return 0.5 * (J2 + J2.T)


def overlap(seed: int, n_ao: int, n_ri: int) -> np.ndarray:
    """Combined AO+RI overlap A A^T + 0.1 I, A ~ N(0, 1/(N+R)); AO block first."""
    n = n_ao + n_ri
    A = gaussian_matrix(seed, "S", n, n, 1.0 / np.sqrt(n))
    S = A @ A.T + 0.1 * np.eye(n)
    return 0.5 * (S + S.T)


def orbitals(seed: int, S_ao: np.ndarray, n_orb: int, name: str = "C") -> np.ndarray:
    """C ~ N(0,1), orthonormalised so that C^T S C = I (Cholesky of C^T S C)."""
    n_ao = S_ao.shape[0]
    C = gaussian_matrix(seed, name, n_ao, n_orb)
    if n_orb == 0:
        return C
    G = C.T @ S_ao @ C
    L = np.linalg.cholesky(0.5 * (G + G.T))
    return np.linalg.solve(L, C.T).T


@dataclass
class Config:
    name: str
    n_ao: int
    n_df: int
    n_ri: int
    n_occ: Tuple[int, ...]          # one entry (closed shell) or two (alpha, beta)
    decay: float
    n_active: Optional[Tuple[int, ...]] = None

    @property
    def n_spin(self) -> int:
        return len(self.n_occ)

    @property
    def active(self) -> Tuple[int, ...]:
        return self.n_active if self.n_active is not None else self.n_occ


# Benchmark configurations described by the reference's workload (sizes only).
CONFIGS = {
    "c0": Config("c0", 24, 84, 116, (5,), 8.0),
    "c1": Config("c1", 500, 1500, 2000, (40, 38), 30.0),
    "c2": Config("c2", 1200, 3600, 4800, (100,), 30.0),
    "c3": Config("c3", 2000, 6000, 8000, (170, 170), 30.0),
}


@dataclass
class Inputs:
    cfg: Config
    W3: np.ndarray
    W2: np.ndarray
    W3_ri: np.ndarray
    V3: np.ndarray
    V2: np.ndarray
    V3_ri: np.ndarray
    WV3: np.ndarray
    WV2: np.ndarray
    S: np.ndarray
    C: np.ndarray                  # n_ao x (n_orb * n_spin), alpha then beta
    occ: np.ndarray                # packed alpha || beta
    n_orb: int


def make_inputs(cfg: Config, seed: int = 11, with_ri: bool = True) -> Inputs:
    N, M, R, L = cfg.n_ao, cfg.n_df, cfg.n_ri, cfg.decay
    S = overlap(seed, N, R)
    n_orb = max(cfg.n_occ)
    Cs = [orbitals(seed, S[:N, :N], n_orb, f"C{s}") for s in range(cfg.n_spin)]
    per = 2.0 if cfg.n_spin == 1 else 1.0
    occ = np.concatenate([np.full(o, per) for o in cfg.n_occ])
    ri = (lambda name: three_index_ri(seed, name, N, R, M, L)) if with_ri else (lambda name: None)
    return Inputs(
        cfg=cfg,
        W3=three_index_ao(seed, "W3", N, M, L), W2=metric(seed, "W2", M), W3_ri=ri("W3_ri"),
        V3=three_index_ao(seed, "V3", N, M, L), V2=metric(seed, "V2", M), V3_ri=ri("V3_ri"),
        WV3=three_index_ao(seed, "WV3", N, M, L), WV2=metric(seed, "WV2", M),
        S=S, C=np.concatenate(Cs, axis=1), occ=occ, n_orb=n_orb,
    )


def random_pd(n: int, seed: int, name: str) -> np.ndarray:
    """Well-conditioned SPD matrix U diag(1+u) U^T (the reference tests' ``random_pd``
    shape, eigenvalues in [1, 2]); U is the orthogonal factor of a Gaussian matrix."""
    G = gaussian_matrix(seed, name, n, n)
    Q, Rr = np.linalg.qr(G)
    Q = Q * np.sign(np.diag(Rr))[None, :]
    key = stream_key(seed, name + ".eig")
    u = 0.5 * (1.0 + np.tanh(normals(key, 0, n)))
    A = (Q * (1.0 + u)[None, :]) @ Q.T
    return 0.5 * (A + A.T)


def uniform_matrix(seed: int, name: str, n_rows: int, n_cols: int) -> np.ndarray:
    """U(0,1)-like entries (the reference tests' ``random`` inputs), via tanh of normals."""
    return 0.5 * (1.0 + np.tanh(gaussian_matrix(seed, name, n_rows, n_cols)))
