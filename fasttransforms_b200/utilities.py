"""Seeded fills in the reference's coefficient layouts.

The reference's test utilities fill the triangular layouts with unseeded
``rand()`` (src/ftutilities.c:75-129).  These fills use a counter-based
splitmix64 generator instead, so the same (kind, n, seed) gives the same
matrix on every machine: the value at column-major linear index idx is
2u - 1 with u the top 53 bits of mix(seed + (idx + 1) * 0x9E3779B97F4A7C15)
divided by 2^53; entries outside the layout's triangle are zero.
"""
from __future__ import annotations

import numpy as np

__all__ = ["layout_cols", "sphrand", "trirand", "diskrand", "rectdiskrand", "tetrand", "rand_layout"]

_STEP = {"sph": 2, "tri": 1, "disk": 4, "rect": 1}


def layout_cols(kind: str, n: int) -> int:
    """Columns M of the layout for n rows: 2n-1 (sph), n (tri, rect), 4n-3 (disk)."""
    return {"sph": 2 * n - 1, "tri": n, "disk": 4 * n - 3, "rect": n}[kind]


def rand_layout(kind: str, n: int, seed: int) -> np.ndarray:
    """n x M float64 matrix, Fortran order, U(-1, 1) inside the layout's triangle."""
    M = layout_cols(kind, n)
    i = np.arange(n, dtype=np.int64)[:, None]
    j = np.arange(M, dtype=np.int64)[None, :]
    on = j < M - _STEP[kind] * i
    idx = (i + j * n).astype(np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return np.asfortranarray(np.where(on, 2.0 * u - 1.0, 0.0))


def sphrand(n: int, seed: int) -> np.ndarray:
    return rand_layout("sph", n, seed)


def trirand(n: int, seed: int) -> np.ndarray:
    return rand_layout("tri", n, seed)


def diskrand(n: int, seed: int) -> np.ndarray:
    return rand_layout("disk", n, seed)


def rectdiskrand(n: int, seed: int) -> np.ndarray:
    """The Dunkl-Xu layout of src/ftutilities.c:123-129: rows i, columns j < M - i (M = n)."""
    return rand_layout("rect", n, seed)


def tetrand(n: int, seed: int, L: int = None, M: int = None) -> np.ndarray:
    """n x L x M float64 tensor, Fortran order, in tetrand's layout (src/ftutilities.c:140-147):
    entry (i, l, m) with l < L - m and i < n - l - m is U(-1, 1) from the counter at its
    column-major index i + n l + n L m, the rest zero (L = M = n by default)."""
    L = n if L is None else L
    M = n if M is None else M
    i = np.arange(n, dtype=np.int64)[:, None, None]
    l = np.arange(L, dtype=np.int64)[None, :, None]
    m = np.arange(M, dtype=np.int64)[None, None, :]
    on = (l < L - m) & (i < n - l - m)
    e = i + n * l + n * L * m
    return np.asfortranarray(np.where(on, _u_pm1(seed, e), 0.0))


def _u_pm1(seed: int, idx: np.ndarray) -> np.ndarray:
    """2u - 1, u from splitmix64 at counter idx (see the module docstring)."""
    idx = idx.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return 2.0 * ((z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53) - 1.0


def spinsphrand(n: int, s: int, seed: int, m: int = None) -> np.ndarray:
    """n x M complex128 matrix, Fortran order, in the spin layout of the reference's
    spinsphrand (src/ftutilities.c:159-167): rows i < n - |s|, columns j < M - 2i, real and
    imaginary parts U(-1, 1) from the counter at the interleaved double index."""
    M = 2 * n - 1 if m is None else m
    i = np.arange(n, dtype=np.int64)[:, None]
    j = np.arange(M, dtype=np.int64)[None, :]
    on = (i < n - abs(s)) & (j < M - 2 * i)
    e = i + j * n
    re = np.where(on, _u_pm1(seed, 2 * e), 0.0)
    im = np.where(on, _u_pm1(seed, 2 * e + 1), 0.0)
    return np.asfortranarray(re + 1j * im)
