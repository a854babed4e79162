"""ctypes bindings for the two CPU oracles -- TEST INFRASTRUCTURE ONLY.

* ``Oracle``: the plain-C restatement in ``oracle/ft_oracle.c`` (built into
  ``oracle/_build/libft_oracle.so``).
* ``Reference``: the reference FastTransforms library compiled from its own
  sources by ``oracle/ref_build/Makefile`` into ``oracle/_ref/libft_ref.so``;
  absent when the reference sources were not available at build time.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module.  Arrays are numpy float64 in Fortran (column-major) order, N x M,
exactly the reference's layout (``src/fasttransforms.h:370-415``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libft_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libft_ref.so")

SPH, TRI, DISK, RECT = 0, 1, 2, 3
KIND = {"sph": SPH, "tri": TRI, "disk": DISK, "rect": RECT}


def layout_cols(kind: str, n: int) -> int:
    """Number of columns M of the reference layout for degree n-1."""
    return {"sph": 2 * n - 1, "tri": n, "disk": 4 * n - 3, "rect": n}[kind]


def fill(kind: str, n: int, seed: int) -> np.ndarray:
    """Seeded U(-1,1) fill in the reference's triangular layouts (src/ftutilities.c:75-113).

    Counter-based splitmix64 on the column-major linear index; identical to
    ``oracle_fill`` in ft_oracle.c and to ``fasttransforms_b200.utilities``.
    """
    M = layout_cols(kind, n)
    i = np.arange(n, dtype=np.int64)[:, None]
    j = np.arange(M, dtype=np.int64)[None, :]
    step = {"sph": 2, "tri": 1, "disk": 4, "rect": 1}[kind]
    on = j < M - step * i
    idx = (i + j * n).astype(np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    A = np.where(on, 2.0 * u - 1.0, 0.0)
    return np.asfortranarray(A)


def fill_spin(n: int, M: int, s: int, seed: int) -> np.ndarray:
    """Seeded complex fill in spinsphrand's layout (src/ftutilities.c:159-167); identical to
    ``oracle_fill_spin`` in ft_oracle.c and ``fasttransforms_b200.utilities.spinsphrand``."""
    from fasttransforms_b200.utilities import spinsphrand
    return spinsphrand(n, s, seed, M)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ptr3(a: np.ndarray):
    """float64 Fortran-order array of any rank as a double pointer."""
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _cptr(a: np.ndarray):
    """complex128 Fortran-order array as interleaved doubles (the ft_complex layout)."""
    assert a.dtype == np.complex128 and a.flags.f_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _OraclePlan(C.Structure):
    _fields_ = [("kind", C.c_int), ("n", C.c_int), ("s", C.POINTER(C.c_double)),
                ("c", C.POINTER(C.c_double)), ("P", C.POINTER(C.c_double) * 3),
                ("Pinv", C.POINTER(C.c_double) * 3), ("alpha", C.c_double),
                ("beta", C.c_double), ("gamma", C.c_double)]


class _OracleAnnPlan(C.Structure):
    _fields_ = [("disk", C.POINTER(_OraclePlan)), ("rd", C.POINTER(C.c_double)), ("ru", C.POINTER(C.c_double)),
                ("rho", C.c_double)]


class _OracleTetPlan(C.Structure):
    _fields_ = [("n", C.c_int), ("rp1", C.c_void_p), ("rp2", C.c_void_p),
                ("P", C.POINTER(C.c_double) * 3), ("Pinv", C.POINTER(C.c_double) * 3),
                ("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double), ("delta", C.c_double)]


class Oracle:
    """The C restatement."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library not built: {path} (run make -C oracle)")
        L = self.lib = C.CDLL(path)
        PP = C.POINTER(_OraclePlan)
        L.oracle_plan_sph2fourier.restype = PP
        L.oracle_plan_sph2fourier.argtypes = [C.c_int]
        L.oracle_plan_tri2cheb.restype = PP
        L.oracle_plan_tri2cheb.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.oracle_plan_disk2cxf.restype = PP
        L.oracle_plan_disk2cxf.argtypes = [C.c_int, C.c_double, C.c_double]
        L.oracle_plan_rectdisk2cheb.restype = PP
        L.oracle_plan_rectdisk2cheb.argtypes = [C.c_int, C.c_double]
        L.oracle_plan_rotations.restype = PP
        L.oracle_plan_rotations.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.oracle_destroy_plan.argtypes = [PP]
        L.oracle_execute.argtypes = [PP, C.c_int, C.c_char, C.POINTER(C.c_double), C.c_int, C.c_int]
        L.oracle_execute_sphv.argtypes = [PP, C.c_int, C.c_char, C.POINTER(C.c_double), C.c_int, C.c_int]
        for f in ("oracle_execute_hi2lo", "oracle_execute_lo2hi"):
            getattr(L, f).argtypes = [PP, C.POINTER(C.c_double), C.c_int]
        for f in ("oracle_kernel_hi2lo", "oracle_kernel_lo2hi"):
            getattr(L, f).argtypes = [PP, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int]
        L.oracle_set_fused.argtypes = [C.c_int]
        L.oracle_fill.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(C.c_double)]
        dp = C.POINTER(C.c_double)
        L.oracle_plan_legendre_to_chebyshev.restype = dp
        L.oracle_plan_legendre_to_chebyshev.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oracle_plan_chebyshev_to_legendre.restype = dp
        L.oracle_plan_chebyshev_to_legendre.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oracle_plan_ultraspherical_to_ultraspherical.restype = dp
        L.oracle_plan_ultraspherical_to_ultraspherical.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.oracle_plan_jacobi_to_jacobi.restype = dp
        L.oracle_plan_jacobi_to_jacobi.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_double] * 4
        self._libc = C.CDLL(None)
        self._libc.free.argtypes = [C.c_void_p]

        sp = C.c_void_p
        L.oracle_plan_spinsph2fourier.restype = sp
        L.oracle_plan_spinsph2fourier.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oracle_destroy_spin_plan.argtypes = [sp]
        L.oracle_execute_spin.argtypes = [sp, C.c_int, C.c_char, dp, C.c_int, C.c_int]
        for f in ("oracle_execute_spinsph_hi2lo", "oracle_execute_spinsph_lo2hi"):
            getattr(L, f).argtypes = [sp, dp, C.c_int]
        for f in ("oracle_kernel_spinsph_hi2lo", "oracle_kernel_spinsph_lo2hi"):
            getattr(L, f).argtypes = [sp, C.c_int, dp]
        L.oracle_kernel_tet.argtypes = [PP, C.c_int, C.c_int, dp, C.c_int]
        L.oracle_fill_spin.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, dp]
        AP = C.POINTER(_OracleAnnPlan)
        L.oracle_plan_ann2cxf.restype = AP
        L.oracle_plan_ann2cxf.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]
        L.oracle_destroy_ann_plan.argtypes = [AP]
        L.oracle_execute_ann.argtypes = [AP, C.c_int, C.c_char, dp, C.c_int, C.c_int]
        L.oracle_plan_tet2cheb.restype = sp
        L.oracle_plan_tet2cheb.argtypes = [C.c_int] + [C.c_double] * 4 + [C.c_int]
        L.oracle_destroy_tet_plan.argtypes = [sp]
        for f in ("oracle_execute_tet_hi2lo", "oracle_execute_tet_lo2hi"):
            getattr(L, f).argtypes = [sp, dp, C.c_int, C.c_int]
        L.oracle_execute_tet.argtypes = [sp, C.c_int, C.c_char, dp, C.c_int, C.c_int, C.c_int]
        L.oracle_fill_tet.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, dp]

    def set_fused(self, fused: bool):
        self.lib.oracle_set_fused(1 if fused else 0)

    # annulus harmonics (gamma = 0): float64 N x (4N - 3) arrays in Fortran order
    def ann_plan(self, n: int, alpha=0.0, beta=0.0, rho=0.5, connections: bool = True):
        return self.lib.oracle_plan_ann2cxf(n, alpha, beta, rho, 1 if connections else 0)

    def ann_destroy(self, P):
        self.lib.oracle_destroy_ann_plan(P)

    def ann_execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, M = A.shape
        self.lib.oracle_execute_ann(P, 1 if forward else 0, trans.encode(), _ptr(A), N, M)

    def ann_hi2lo(self, P, A: np.ndarray):
        self.lib.oracle_execute_hi2lo(P.contents.disk, _ptr(A), A.shape[1])

    def ann_lo2hi(self, P, A: np.ndarray):
        self.lib.oracle_execute_lo2hi(P.contents.disk, _ptr(A), A.shape[1])

    def ann_table(self, P):
        return self.tables(P.contents.disk)

    def ann_connection(self, P):
        p = P.contents.disk.contents
        n = p.n
        get = lambda q: np.ctypeslib.as_array(q, shape=(n * n,)).reshape(n, n, order="F").copy()
        return get(p.P[0]), get(p.Pinv[0])

    def ann_cholesky(self, P):
        p = P.contents
        n = p.disk.contents.n
        return np.ctypeslib.as_array(p.rd, shape=(n,)).copy(), np.ctypeslib.as_array(p.ru, shape=(max(n - 1, 1),))[: n - 1].copy()

    # tetrahedral harmonics: float64 N x L x M arrays in Fortran order
    def tet_plan(self, n: int, alpha=0.0, beta=0.0, gamma=0.0, delta=0.0, connections: bool = True):
        return self.lib.oracle_plan_tet2cheb(n, alpha, beta, gamma, delta, 1 if connections else 0)

    def tet_destroy(self, P):
        self.lib.oracle_destroy_tet_plan(P)

    def tet_connection(self, P):
        p = C.cast(C.c_void_p(P), C.POINTER(_OracleTetPlan)).contents
        n = p.n
        get = lambda q: np.ctypeslib.as_array(q, shape=(n * n,)).reshape(n, n, order="F").copy()
        return [get(p.P[i]) for i in range(3)], [get(p.Pinv[i]) for i in range(3)]

    def tet_execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, L, M = A.shape
        self.lib.oracle_execute_tet(P, 1 if forward else 0, trans.encode(), _ptr3(A), N, L, M)

    def tet_hi2lo(self, P, A: np.ndarray):
        self.lib.oracle_execute_tet_hi2lo(P, _ptr3(A), A.shape[1], A.shape[2])

    def tet_lo2hi(self, P, A: np.ndarray):
        self.lib.oracle_execute_tet_lo2hi(P, _ptr3(A), A.shape[1], A.shape[2])

    def tet_fill(self, N: int, L: int, M: int, seed: int) -> np.ndarray:
        A = np.zeros((N, L, M), order="F")
        self.lib.oracle_fill_tet(N, L, M, seed, _ptr3(A))
        return A

    # spin-weighted spherical harmonics: complex128 N x M arrays in Fortran order (the
    # interleaved (re, im) layout of ft_complex)
    def spin_plan(self, n: int, s: int, connections: bool = True):
        return self.lib.oracle_plan_spinsph2fourier(n, s, 1 if connections else 0)

    def spin_destroy(self, P):
        self.lib.oracle_destroy_spin_plan(P)

    def spin_execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, M = A.shape
        self.lib.oracle_execute_spin(P, 1 if forward else 0, trans.encode(), _cptr(A), N, M)

    def spin_hi2lo(self, P, A: np.ndarray):
        self.lib.oracle_execute_spinsph_hi2lo(P, _cptr(A), A.shape[1])

    def spin_lo2hi(self, P, A: np.ndarray):
        self.lib.oracle_execute_spinsph_lo2hi(P, _cptr(A), A.shape[1])

    def spin_kernel(self, P, hi2lo: bool, m: int, col: np.ndarray) -> np.ndarray:
        """One complex column of order m (src/rotations/rotations_default.c:87-117)."""
        a = np.ascontiguousarray(col, dtype=complex).copy()
        (self.lib.oracle_kernel_spinsph_hi2lo if hi2lo else self.lib.oracle_kernel_spinsph_lo2hi)(P, m, _cptr(a))
        return a

    def tet_kernel(self, RP, hi2lo: bool, L: int, m: int, A: np.ndarray) -> np.ndarray:
        """The n x L slab of order m with a triangle rotation plan (src/rotations.c:297-321)."""
        a = np.asfortranarray(A, dtype=np.float64).copy(order="F")
        self.lib.oracle_kernel_tet(RP, L, m, _ptr(a), 1 if hi2lo else 0)
        return a

    def spin_fill(self, n: int, M: int, s: int, seed: int) -> np.ndarray:
        A = np.zeros((n, M), dtype=complex, order="F")
        self.lib.oracle_fill_spin(n, M, s, seed, _cptr(A))
        return A

    def plan(self, kind: str, n: int, alpha=0.0, beta=0.0, gamma=0.0, rotations_only=False):
        L = self.lib
        if rotations_only:
            return L.oracle_plan_rotations(KIND[kind], n, alpha, beta, gamma)
        if kind == "sph":
            return L.oracle_plan_sph2fourier(n)
        if kind == "tri":
            return L.oracle_plan_tri2cheb(n, alpha, beta, gamma)
        if kind == "rect":
            return L.oracle_plan_rectdisk2cheb(n, beta)
        return L.oracle_plan_disk2cxf(n, alpha, beta)

    def destroy(self, P):
        self.lib.oracle_destroy_plan(P)

    def execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, M = A.shape
        self.lib.oracle_execute(P, 1 if forward else 0, trans.encode(), _ptr(A), N, M)

    def execute_sphv(self, P, forward: bool, trans: str, A: np.ndarray):
        """sph vector fields on a sph plan: sphv2fourier (forward) / fourier2sphv."""
        N, M = A.shape
        self.lib.oracle_execute_sphv(P, 1 if forward else 0, trans.encode(), _ptr(A), N, M)

    def hi2lo(self, P, A):
        self.lib.oracle_execute_hi2lo(P, _ptr(A), A.shape[1])

    def lo2hi(self, P, A):
        self.lib.oracle_execute_lo2hi(P, _ptr(A), A.shape[1])

    def kernel(self, P, hi2lo: bool, m1: int, m2: int, col: np.ndarray):
        a = np.asfortranarray(col.reshape(-1, 1))
        f = self.lib.oracle_kernel_hi2lo if hi2lo else self.lib.oracle_kernel_lo2hi
        f(P, m1, m2, _ptr(a), 1)
        return a.ravel()

    def tables(self, P):
        p = P.contents
        n = p.n
        ln = n * n if p.kind == DISK else n * (n + 1) // 2
        s = np.ctypeslib.as_array(p.s, shape=(ln,)).copy()
        c = np.ctypeslib.as_array(p.c, shape=(ln,)).copy()
        return s, c

    def connection(self, P):
        p = P.contents
        n = p.n
        get = lambda q: np.ctypeslib.as_array(q, shape=(n * n,)).reshape(n, n, order="F").copy()
        k = 3 if p.kind == RECT else 2
        return [get(p.P[i]) for i in range(k)], [get(p.Pinv[i]) for i in range(k)]

    def fill(self, kind: str, n: int, seed: int) -> np.ndarray:
        M = layout_cols(kind, n)
        A = np.zeros((n, M), order="F")
        self.lib.oracle_fill(KIND[kind], n, M, seed, _ptr(A))
        return A


class _RefHarmonicPlan(C.Structure):
    # src/fasttransforms.h:370-385
    _fields_ = [("RP", C.c_void_p), ("MP", C.c_void_p), ("B", C.c_void_p),
                ("P", C.POINTER(C.POINTER(C.c_double))), ("Pinv", C.POINTER(C.POINTER(C.c_double))),
                ("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double),
                ("delta", C.c_double), ("rho", C.c_double),
                ("NRP", C.c_int), ("NMP", C.c_int), ("NP", C.c_int)]


class Reference:
    """The reference library compiled from its own sources (oracle/_ref)."""

    _FWD = {"sph": "ft_execute_sph2fourier", "tri": "ft_execute_tri2cheb", "disk": "ft_execute_disk2cxf",
            "sphv": "ft_execute_sphv2fourier", "rect": "ft_execute_rectdisk2cheb"}
    _BWD = {"sph": "ft_execute_fourier2sph", "tri": "ft_execute_cheb2tri", "disk": "ft_execute_cxf2disk",
            "sphv": "ft_execute_fourier2sphv", "rect": "ft_execute_cheb2rectdisk"}

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference library not built: {path}")
        L = self.lib = C.CDLL(path)
        HP = C.POINTER(_RefHarmonicPlan)
        L.ft_plan_sph2fourier.restype = HP
        L.ft_plan_sph2fourier.argtypes = [C.c_int]
        L.ft_plan_tri2cheb.restype = HP
        L.ft_plan_tri2cheb.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.ft_plan_disk2cxf.restype = HP
        L.ft_plan_disk2cxf.argtypes = [C.c_int, C.c_double, C.c_double]
        L.ft_plan_rectdisk2cheb.restype = HP
        L.ft_plan_rectdisk2cheb.argtypes = [C.c_int, C.c_double]
        L.ft_destroy_harmonic_plan.argtypes = [HP]
        L.ft_plan_ann2cxf.restype = HP
        L.ft_plan_ann2cxf.argtypes = [C.c_int] + [C.c_double] * 4
        for f in ("ft_execute_ann2cxf", "ft_execute_cxf2ann"):
            getattr(L, f).argtypes = [C.c_char, HP, C.POINTER(C.c_double), C.c_int, C.c_int]
        L.ft_plan_rotannulus.restype = C.POINTER(C.POINTER(C.c_double))
        L.ft_plan_rotannulus.argtypes = [C.c_int] + [C.c_double] * 4
        for f in ("ft_execute_disk_hi2lo", "ft_execute_disk_lo2hi"):
            getattr(L, f).argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        L.ft_plan_tet2cheb.restype = HP
        L.ft_plan_tet2cheb.argtypes = [C.c_int] + [C.c_double] * 4
        for f in ("ft_execute_tet2cheb", "ft_execute_cheb2tet"):
            getattr(L, f).argtypes = [C.c_char, HP, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int]
        L.ft_plan_rottriangle.restype = C.c_void_p
        L.ft_plan_rottriangle.argtypes = [C.c_int] + [C.c_double] * 3
        for f in ("ft_execute_tet_hi2lo", "ft_execute_tet_lo2hi"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int]
        L.ft_plan_rotrectdisk.restype = C.c_void_p
        L.ft_plan_rotrectdisk.argtypes = [C.c_int, C.c_double]
        L.ft_destroy_rotation_plan.argtypes = [C.c_void_p]
        for f in ("ft_execute_rectdisk_hi2lo", "ft_execute_rectdisk_lo2hi"):
            getattr(L, f).argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        for f in list(self._FWD.values()) + list(self._BWD.values()):
            getattr(L, f).argtypes = [C.c_char, HP, C.POINTER(C.c_double), C.c_int, C.c_int]
        L.ft_set_num_threads.argtypes = [C.c_int]
        sp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.ft_plan_spinsph2fourier.restype = sp
        L.ft_plan_spinsph2fourier.argtypes = [C.c_int, C.c_int]
        L.ft_destroy_spin_harmonic_plan.argtypes = [sp]
        for f in ("ft_execute_spinsph2fourier", "ft_execute_fourier2spinsph"):
            getattr(L, f).argtypes = [C.c_char, sp, dp, C.c_int, C.c_int]
        L.ft_plan_rotspinsphere.restype = sp
        L.ft_plan_rotspinsphere.argtypes = [C.c_int, C.c_int]
        L.ft_destroy_spin_rotation_plan.argtypes = [sp]
        for f in ("ft_execute_spinsph_hi2lo", "ft_execute_spinsph_lo2hi"):
            getattr(L, f).argtypes = [sp, dp, dp, C.c_int]

    # spin-weighted spherical harmonics (complex128 Fortran arrays)
    def spin_plan(self, n: int, s: int):
        return self.lib.ft_plan_spinsph2fourier(n, s)

    def spin_destroy(self, P):
        self.lib.ft_destroy_spin_harmonic_plan(P)

    def spin_execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, M = A.shape
        f = self.lib.ft_execute_spinsph2fourier if forward else self.lib.ft_execute_fourier2spinsph
        f(trans.encode(), P, _cptr(A), N, M)

    def spin_rotations(self, n: int, s: int, hi2lo: bool, A: np.ndarray):
        """The rotation stage alone (ft_execute_spinsph_hi2lo / lo2hi, with a scratch array)."""
        SRP = self.lib.ft_plan_rotspinsphere(n, s)
        B = np.zeros_like(A)
        f = self.lib.ft_execute_spinsph_hi2lo if hi2lo else self.lib.ft_execute_spinsph_lo2hi
        f(SRP, _cptr(A), _cptr(B), A.shape[1])
        self.lib.ft_destroy_spin_rotation_plan(SRP)

    def rect_rotations(self, n: int, beta: float, hi2lo: bool, A: np.ndarray):
        """The Dunkl-Xu rotation stage alone (ft_execute_rectdisk_hi2lo / lo2hi)."""
        RP = self.lib.ft_plan_rotrectdisk(n, beta)
        B = np.zeros_like(A)
        f = self.lib.ft_execute_rectdisk_hi2lo if hi2lo else self.lib.ft_execute_rectdisk_lo2hi
        f(RP, _ptr(A), _ptr(B), A.shape[1])
        self.lib.ft_destroy_rotation_plan(RP)

    def ann_plan(self, n: int, alpha=0.0, beta=0.0, rho=0.5):
        return self.lib.ft_plan_ann2cxf(n, alpha, beta, 0.0, rho)

    def ann_execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, M = A.shape
        f = self.lib.ft_execute_ann2cxf if forward else self.lib.ft_execute_cxf2ann
        f(trans.encode(), P, _ptr(A), N, M)

    def ann_rotations(self, n: int, alpha: float, beta: float, rho: float, hi2lo: bool, A: np.ndarray):
        """The annulus rotation stage alone: ft_plan_rotannulus's table through the disk sweeps
        (ft_execute_disk_hi2lo / lo2hi), as ft_execute_ann2cxf runs it."""
        RP = self.lib.ft_plan_rotannulus(n, alpha, beta, 0.0, rho)
        B = np.zeros_like(A)
        f = self.lib.ft_execute_disk_hi2lo if hi2lo else self.lib.ft_execute_disk_lo2hi
        f(C.cast(RP, C.c_void_p), _ptr(A), _ptr(B), A.shape[1])
        self.lib.ft_destroy_rotation_plan(C.cast(RP, C.c_void_p))

    def ann_table(self, n: int, alpha: float, beta: float, rho: float):
        """ft_plan_rotannulus's sine and cosine tables (the disk packing, n^2 entries)."""
        RP = self.lib.ft_plan_rotannulus(n, alpha, beta, 0.0, rho)
        s = np.ctypeslib.as_array(RP[0], shape=(n * n,)).copy()
        c = np.ctypeslib.as_array(RP[1], shape=(n * n,)).copy()
        self.lib.ft_destroy_rotation_plan(C.cast(RP, C.c_void_p))
        return s, c

    def tet_plan(self, n: int, alpha=0.0, beta=0.0, gamma=0.0, delta=0.0):
        return self.lib.ft_plan_tet2cheb(n, alpha, beta, gamma, delta)

    def tet_execute(self, P, forward: bool, trans: str, A: np.ndarray):
        N, L, M = A.shape
        f = self.lib.ft_execute_tet2cheb if forward else self.lib.ft_execute_cheb2tet
        f(trans.encode(), P, _ptr3(A), N, L, M)

    def tet_rotations(self, n: int, params, hi2lo: bool, A: np.ndarray):
        """The tetrahedral rotation stage alone (ft_execute_tet_hi2lo / lo2hi) with the plan's two
        triangle tables (src/drivers.c:1176-1177)."""
        a, b, g, d = params
        RP1 = self.lib.ft_plan_rottriangle(n, a, b, g + d + 1.0)
        RP2 = self.lib.ft_plan_rottriangle(n, b, g, d)
        f = self.lib.ft_execute_tet_hi2lo if hi2lo else self.lib.ft_execute_tet_lo2hi
        f(RP1, RP2, _ptr3(A), A.shape[1], A.shape[2])
        self.lib.ft_destroy_rotation_plan(RP1)
        self.lib.ft_destroy_rotation_plan(RP2)

    def set_num_threads(self, t: int):
        self.lib.ft_set_num_threads(t)

    def plan(self, kind: str, n: int, alpha=0.0, beta=0.0, gamma=0.0):
        L = self.lib
        if kind in ("sph", "sphv"):
            return L.ft_plan_sph2fourier(n)
        if kind == "tri":
            return L.ft_plan_tri2cheb(n, alpha, beta, gamma)
        if kind == "rect":
            return L.ft_plan_rectdisk2cheb(n, beta)
        return L.ft_plan_disk2cxf(n, alpha, beta)

    def destroy(self, P):
        self.lib.ft_destroy_harmonic_plan(P)

    def execute(self, kind: str, P, forward: bool, trans: str, A: np.ndarray):
        N, M = A.shape
        f = getattr(self.lib, (self._FWD if forward else self._BWD)[kind])
        f(trans.encode(), P, _ptr(A), N, M)

    def connection(self, P, n: int):
        p = P.contents
        get = lambda q: np.ctypeslib.as_array(q, shape=(n * n,)).reshape(n, n, order="F").copy()
        return [get(p.P[i]) for i in range(p.NP)], [get(p.Pinv[i]) for i in range(p.NP)]


QUAD_SO = os.path.join(HERE, "_build", "libft_quad.so")


class Quad:
    """The __float128 restatement of the rotation tables, the default sweep kernels and (sph,
    disk) the forward transform 'N' (oracle/ft_quad.c), on selected columns."""

    KIND = {"sph": 0, "tri": 1, "disk": 2}

    @staticmethod
    def available(path: str = QUAD_SO) -> bool:
        return os.path.exists(path)

    def __init__(self, path: str = QUAD_SO):
        L = self.lib = C.CDLL(path)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.quad_columns.restype = C.c_int
        L.quad_columns.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp, C.c_longlong, ip, C.c_int,
                                   C.c_int, dp, dp, dp, dp]
        L.quad_table_column.restype = None
        L.quad_table_column.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, dp, dp, dp, dp]

    def columns(self, kind: str, A: np.ndarray, cols, params=(), hi2lo: bool = True, P=None):
        """Columns `cols` of A (N x M, Fortran order) through the rotation stage (P None) or the
        forward transform 'N' with connection matrices P = (P0, P1) (n x n, Fortran order).
        Returns (hi, lo), N x len(cols) each: the quad result rounded to double, and the rest."""
        n = A.shape[0]
        a = tuple(params) + (0.0,) * (3 - len(params))
        A = np.asfortranarray(A, dtype=np.float64)
        cc = (C.c_int * max(len(cols), 1))(*[int(c) for c in cols])
        hi = np.zeros((n, len(cols)), order="F")
        lo = np.zeros((n, len(cols)), order="F")
        p0 = p1 = None
        if P is not None:
            keep = (np.asfortranarray(P[0], dtype=np.float64), np.asfortranarray(P[1], dtype=np.float64))
            p0, p1 = _ptr(keep[0]), _ptr(keep[1])
        r = self.lib.quad_columns(self.KIND[kind], n, a[0], a[1], a[2], _ptr(A), n, cc, len(cols), 1 if hi2lo else 0,
                                  p0, p1, _ptr(hi), _ptr(lo))
        if r != 0:
            raise RuntimeError(f"quad_columns failed ({r})")
        return hi, lo

    def table_column(self, kind: str, n: int, j: int, length: int, params=()):
        a = tuple(params) + (0.0,) * (3 - len(params))
        out = [np.zeros(length, order="F") for _ in range(4)]
        self.lib.quad_table_column(self.KIND[kind], n, a[0], a[1], a[2], j, length, *[_ptr(o) for o in out])
        return out
