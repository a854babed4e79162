"""B200-native (sm_100a) harmonic-conversion path of FastTransforms.

Python mirror of the reference's C API for sph2fourier / fourier2sph,
tri2cheb / cheb2tri and disk2cxf / cxf2disk (src/fasttransforms.h:370-415), the
sphere's vector-field and spin-weighted transforms, the Dunkl-Xu, annulus and
tetrahedral transforms and the sphere, disk and triangle grids, over the C ABI
in include/ft_b200.h.  The compute runs in hand-written CUDA
kernels in ``_lib/libft_b200.so``; there is no CPU fallback: importing this
package fails if the library is missing, and planning fails without an sm_100
device.

Host arrays are numpy float64 in Fortran (column-major) order, N x M, exactly
the reference's layout; transforms run in place like the reference's.
Device entry points take raw device pointers (e.g. ``tensor.data_ptr()``).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from .utilities import diskrand, layout_cols, rand_layout, rectdiskrand, sphrand, spinsphrand, tetrand, trirand

__all__ = [
    "FTB200Error", "HarmonicPlan", "RotationPlan", "library_path", "lib",
    "plan_sph2fourier", "plan_tri2cheb", "plan_disk2cxf",
    "execute_sph2fourier", "execute_fourier2sph", "execute_tri2cheb", "execute_cheb2tri",
    "execute_disk2cxf", "execute_cxf2disk", "execute_sphv2fourier", "execute_fourier2sphv", "execute_sphv_dev",
    "plan_rotsphere", "plan_rottriangle", "plan_rotdisk",
    "execute_sph_hi2lo", "execute_sph_lo2hi", "execute_tri_hi2lo", "execute_tri_lo2hi",
    "execute_disk_hi2lo", "execute_disk_lo2hi",
    "execute_dev", "execute_shared_dev", "execute_shared_host", "FP64", "FP64_BLOCKED", "MIXED_BF16", "MIXED_BF16X4", "device_status", "execute_noalloc_dev", "NOALLOC_MAX_ELEMS", "execute_batched_dev", "rotations_dev", "kernel_launches", "profile", "profile_read", "set_rotation_config",
    "layout_cols", "rand_layout", "sphrand", "trirand", "diskrand",
    "SphereGridPlan", "plan_sph_synthesis", "plan_sph_analysis", "plan_sphv_synthesis", "plan_sphv_analysis",
    "execute_sph_synthesis", "execute_sph_analysis", "execute_sphv_synthesis", "execute_sphv_analysis",
    "execute_sph_grid_dev", "GRID_OPS",
    "SpinHarmonicPlan", "SpinRotationPlan", "plan_spinsph2fourier", "plan_rotspinsphere",
    "execute_spinsph2fourier", "execute_fourier2spinsph", "execute_spinsph_hi2lo", "execute_spinsph_lo2hi",
    "execute_spin_dev", "spin_rotations_dev", "spinsphrand", "kernel_column", "kernel_spin_column", "kernel_tet_slab",
    "execute_sphv_hi2lo", "execute_sphv_lo2hi",
    "SpinGridPlan", "plan_spinsph_synthesis", "plan_spinsph_analysis", "execute_spinsph_synthesis",
    "execute_spinsph_analysis", "execute_spinsph_grid_dev",
    "plan_rectdisk2cheb", "execute_rectdisk2cheb", "execute_cheb2rectdisk", "plan_rotrectdisk",
    "execute_rectdisk_hi2lo", "execute_rectdisk_lo2hi", "rectdiskrand",
    "TetPlan", "plan_tet2cheb", "execute_tet2cheb", "execute_cheb2tet", "execute_tet_hi2lo", "execute_tet_lo2hi",
    "execute_tet_dev", "tet_rotations_dev", "tetrand",
    "plan_ann2cxf", "execute_ann2cxf", "execute_cxf2ann", "plan_rotannulus",
    "plan_disk_synthesis", "plan_disk_analysis", "execute_disk_synthesis", "execute_disk_analysis", "execute_disk_grid_dev",
    "plan_tri_synthesis", "plan_tri_analysis", "execute_tri_synthesis", "execute_tri_analysis", "execute_tri_grid_dev",
    "plan_annulus_synthesis", "plan_annulus_analysis", "execute_annulus_synthesis", "execute_annulus_analysis",
    "execute_annulus_grid_dev", "plan_rectdisk_synthesis", "plan_rectdisk_analysis", "execute_rectdisk_synthesis",
    "execute_rectdisk_analysis", "execute_rectdisk_grid_dev",
    "plan_tet_synthesis", "plan_tet_analysis", "execute_tet_synthesis", "execute_tet_analysis", "execute_tet_grid_dev",
    "SPH", "TRI", "DISK",
]

SPH, TRI, DISK = 0, 1, 2
_KINDS = {"sph": SPH, "tri": TRI, "disk": DISK}

_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(_HERE, "_lib", "libft_b200.so")


class FTB200Error(RuntimeError):
    """A call into the CUDA library failed; ``status`` is the ft_b200 status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"ft_b200 status {status}: {message}")
        self.status = status


def _load() -> C.CDLL:
    if not os.path.exists(library_path):
        raise ImportError(f"{library_path} is not built (python fasttransforms_b200/build.py)")
    L = C.CDLL(library_path)
    vp, dp, i, d, ch = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_char
    sig = {
        "ft_b200_last_status": (i, []), "ft_b200_last_error": (C.c_char_p, []),
        "ft_b200_kernel_launches": (C.c_ulonglong, []),
        "ft_plan_sph2fourier": (vp, [i]), "ft_plan_tri2cheb": (vp, [i, d, d, d]), "ft_plan_disk2cxf": (vp, [i, d, d]),
        "ft_destroy_harmonic_plan": (None, [vp]),
        "ft_plan_rotsphere": (vp, [i]), "ft_plan_rottriangle": (vp, [i, d, d, d]), "ft_plan_rotdisk": (vp, [i, d, d]),
        "ft_destroy_rotation_plan": (None, [vp]),
        "ft_b200_execute_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_b200_execute_sphv_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_b200_rotations_dev": (i, [vp, i, vp, i, vp]),
        "ft_b200_execute_batched_dev": (i, [C.POINTER(vp), i, ch, C.POINTER(vp), C.POINTER(i), C.POINTER(i), i, vp]),
        "ft_b200_plan_kind": (i, [vp]), "ft_b200_plan_device": (i, [vp]),
        "ft_b200_execute_noalloc_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_b200_execute_shared_dev": (i, [vp, i, ch, C.POINTER(vp), i, i, vp]),
        "ft_b200_execute_shared_host": (i, [vp, i, C.POINTER(i), C.c_char_p, C.POINTER(vp), i, i]),
        "ft_b200_device_status": (i, [vp]),
        "ft_b200_profile": (i, [i]), "ft_b200_profile_read": (i, [i, C.POINTER(C.c_double), C.POINTER(i)]),
        "ft_b200_set_rotation_config": (None, [i]),
        "ft_plan_sph_synthesis": (vp, [i, i, C.c_uint]), "ft_plan_sph_analysis": (vp, [i, i, C.c_uint]),
        "ft_plan_sphv_synthesis": (vp, [i, i, C.c_uint]), "ft_plan_sphv_analysis": (vp, [i, i, C.c_uint]),
        "ft_destroy_sphere_fftw_plan": (None, [vp]),
        "ft_b200_execute_sph_grid_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_plan_rotspinsphere": (vp, [i, i]), "ft_destroy_spin_rotation_plan": (None, [vp]),
        "ft_execute_spinsph_hi2lo": (None, [vp, dp, dp, i]), "ft_execute_spinsph_lo2hi": (None, [vp, dp, dp, i]),
        "ft_plan_spinsph2fourier": (vp, [i, i]), "ft_destroy_spin_harmonic_plan": (None, [vp]),
        "ft_execute_spinsph2fourier": (None, [ch, vp, dp, i, i]), "ft_execute_fourier2spinsph": (None, [ch, vp, dp, i, i]),
        "ft_b200_execute_spin_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_b200_spin_rotations_dev": (i, [vp, i, vp, i, vp]),
        "ft_plan_rectdisk2cheb": (vp, [i, d]), "ft_plan_rotrectdisk": (vp, [i, d]),
        "ft_plan_tet2cheb": (vp, [i, d, d, d, d]),
        "ft_plan_ann2cxf": (vp, [i, d, d, d, d]), "ft_plan_rotannulus": (vp, [i, d, d, d, d]),
        "ft_plan_disk_synthesis": (vp, [i, i, C.c_uint]), "ft_plan_disk_analysis": (vp, [i, i, C.c_uint]),
        "ft_destroy_disk_fftw_plan": (None, [vp]),
        "ft_plan_tri_synthesis": (vp, [i, i, C.c_uint]), "ft_plan_tri_analysis": (vp, [i, i, C.c_uint]),
        "ft_destroy_triangle_fftw_plan": (None, [vp]),
        "ft_b200_execute_disk_grid_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_b200_execute_tri_grid_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_plan_annulus_synthesis": (vp, [i, i, d, C.c_uint]), "ft_plan_annulus_analysis": (vp, [i, i, d, C.c_uint]),
        "ft_destroy_annulus_fftw_plan": (None, [vp]), "ft_get_rho_annulus_fftw_plan": (d, [vp]),
        "ft_plan_rectdisk_synthesis": (vp, [i, i, C.c_uint]), "ft_plan_rectdisk_analysis": (vp, [i, i, C.c_uint]),
        "ft_destroy_rectdisk_fftw_plan": (None, [vp]),
        "ft_plan_tet_synthesis": (vp, [i, i, i, C.c_uint]), "ft_plan_tet_analysis": (vp, [i, i, i, C.c_uint]),
        "ft_destroy_tetrahedron_fftw_plan": (None, [vp]),
        "ft_execute_tet_synthesis": (None, [ch, vp, dp, i, i, i]), "ft_execute_tet_analysis": (None, [ch, vp, dp, i, i, i]),
        "ft_b200_execute_tet_grid_dev": (i, [vp, i, ch, vp, i, i, i, vp]),
        "ft_b200_execute_annulus_grid_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_b200_execute_rectdisk_grid_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_execute_tet2cheb": (None, [ch, vp, dp, i, i, i]), "ft_execute_cheb2tet": (None, [ch, vp, dp, i, i, i]),
        "ft_execute_tet_hi2lo": (None, [vp, vp, dp, i, i]), "ft_execute_tet_lo2hi": (None, [vp, vp, dp, i, i]),
        "ft_b200_execute_tet_dev": (i, [vp, i, ch, vp, i, i, i, vp]),
        "ft_b200_tet_rotations_dev": (i, [vp, i, vp, i, i, vp]),
        "ft_plan_spinsph_synthesis": (vp, [i, i, i, C.c_uint]), "ft_plan_spinsph_analysis": (vp, [i, i, i, C.c_uint]),
        "ft_destroy_spinsphere_fftw_plan": (None, [vp]), "ft_get_spin_spinsphere_fftw_plan": (i, [vp]),
        "ft_execute_spinsph_synthesis": (None, [ch, vp, dp, i, i]), "ft_execute_spinsph_analysis": (None, [ch, vp, dp, i, i]),
        "ft_b200_execute_spinsph_grid_dev": (i, [vp, i, ch, vp, i, i, vp]),
        "ft_kernel_spinsph_hi2lo": (None, [vp, i, dp, i]), "ft_kernel_spinsph_lo2hi": (None, [vp, i, dp, i]),
        "ft_kernel_tet_hi2lo": (None, [vp, i, i, dp]), "ft_kernel_tet_lo2hi": (None, [vp, i, i, dp]),
        "ft_set_num_threads": (None, [i]), "ft_fftw_init_threads": (i, []), "ft_fftw_plan_with_nthreads": (None, [i]),
        "ft_plan_sph_with_kind": (vp, [i, i, C.POINTER(i), C.c_uint]), "ft_plan_disk_with_kind": (vp, [i, i, C.POINTER(i), C.c_uint]),
        "ft_plan_tri_with_kind": (vp, [i, i, i, i, C.c_uint]),
        "ft_plan_annulus_with_kind": (vp, [i, i, d, C.POINTER(i), C.c_uint]),
        "ft_plan_rectdisk_with_kind": (vp, [i, i, C.POINTER(i), C.c_uint]),
        "ft_plan_tet_with_kind": (vp, [i, i, i, i, i, i, C.c_uint]),
        "ft_plan_spinsph_with_kind": (vp, [i, i, i, C.POINTER(i), i, C.c_uint]),
    }
    for name in ("sph_synthesis", "sph_analysis", "sphv_synthesis", "sphv_analysis", "disk_synthesis", "disk_analysis",
                 "tri_synthesis", "tri_analysis", "annulus_synthesis", "annulus_analysis", "rectdisk_synthesis",
                 "rectdisk_analysis"):
        sig["ft_execute_" + name] = (None, [ch, vp, dp, i, i])
    for name in ("sph2fourier", "fourier2sph", "tri2cheb", "cheb2tri", "disk2cxf", "cxf2disk", "sphv2fourier", "fourier2sphv",
                 "rectdisk2cheb", "cheb2rectdisk", "ann2cxf", "cxf2ann"):
        sig["ft_execute_" + name] = (None, [ch, vp, dp, i, i])
    for fam in ("sph", "tri", "disk", "rectdisk", "sphv"):
        for d_ in ("hi2lo", "lo2hi"):
            sig[f"ft_execute_{fam}_{d_}"] = (None, [vp, dp, dp, i])
            if fam != "sphv":
                sig[f"ft_kernel_{fam}_{d_}"] = (None, [vp, i, i, dp, i])
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


lib = _load()


def _check():
    st = lib.ft_b200_last_status()
    if st != 0:
        raise FTB200Error(st, lib.ft_b200_last_error().decode())


def set_rotation_config(cfg: int) -> None:
    """Force the rotation kernel's launch shape (0 .. 5; + 8 through the pass pipeline) or
    let the autotuner choose (-1)."""
    lib.ft_b200_set_rotation_config(int(cfg))


def profile(enable: bool) -> None:
    """Turn per-launch CUDA-event timing on (resetting the record) or off."""
    lib.ft_b200_profile(1 if enable else 0)


def profile_read(family: int):
    """(total ms, launches) recorded for a kernel family: 0 rotations, 1 trmm, 2 other, 3 blocked sweeps."""
    ms = C.c_double(0)
    cnt = C.c_int(0)
    if lib.ft_b200_profile_read(family, C.byref(ms), C.byref(cnt)) != 0:
        _check()
    return ms.value, cnt.value


def kernel_launches() -> int:
    """Kernels this library has launched since it was loaded."""
    return int(lib.ft_b200_kernel_launches())


class HarmonicPlan:
    """Owns an ``ft_harmonic_plan *`` of the CUDA library (reference: src/drivers.c:793-1021)."""

    def __init__(self, ptr: int, kind: str, n: int, params=()):
        self.ptr = ptr
        self.kind = kind
        self.n = n
        self.params = tuple(params)

    @property
    def M(self) -> int:
        return layout_cols(self.kind, self.n)

    def close(self):
        if self.ptr:
            lib.ft_destroy_harmonic_plan(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class RotationPlan(HarmonicPlan):
    """Owns an ``ft_rotation_plan *`` (reference: src/rotations.c:116-190)."""

    def close(self):
        if self.ptr:
            lib.ft_destroy_rotation_plan(self.ptr)
            self.ptr = None


def _plan(kind, n, ptr, params=()):
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return HarmonicPlan(ptr, kind, n, params)


def plan_sph2fourier(n: int) -> HarmonicPlan:
    return _plan("sph", n, lib.ft_plan_sph2fourier(n))


def plan_tri2cheb(n: int, alpha: float, beta: float, gamma: float) -> HarmonicPlan:
    return _plan("tri", n, lib.ft_plan_tri2cheb(n, alpha, beta, gamma), (alpha, beta, gamma))


def plan_disk2cxf(n: int, alpha: float, beta: float) -> HarmonicPlan:
    return _plan("disk", n, lib.ft_plan_disk2cxf(n, alpha, beta), (alpha, beta))


def plan_ann2cxf(n: int, alpha: float, beta: float, gamma: float, rho: float) -> HarmonicPlan:
    """Annulus plan (reference: src/drivers.c:1023-1071; gamma must be 0); the disk layout, M = 4n - 3."""
    return _plan("disk", n, lib.ft_plan_ann2cxf(n, alpha, beta, gamma, rho), (alpha, beta, gamma, rho))


def plan_rectdisk2cheb(n: int, beta: float) -> HarmonicPlan:
    """Dunkl-Xu (rectangularised disk) plan (reference: src/drivers.c:1123-1141); M = n."""
    return _plan("rect", n, lib.ft_plan_rectdisk2cheb(n, beta), (beta,))


class SphereGridPlan(HarmonicPlan):
    """Owns an ``ft_sphere_fftw_plan *``: synthesis / analysis on the sphere's N x M grid
    (reference: src/fftw.c:63-277; cuFFT and this library's kernels in place of FFTW)."""

    def __init__(self, ptr: int, kind: str, n: int, m: int):
        super().__init__(ptr, kind, n)
        self.m = m

    @property
    def M(self) -> int:
        return self.m

    def close(self):
        if self.ptr:
            lib.ft_destroy_sphere_fftw_plan(self.ptr)
            self.ptr = None


def _grid_plan(kind, n, m):
    m = 2 * n - 1 if m is None else m
    ptr = getattr(lib, "ft_plan_" + kind)(n, m, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return SphereGridPlan(ptr, kind, n, m)


def plan_sph_synthesis(n: int, m: int = None) -> SphereGridPlan: return _grid_plan("sph_synthesis", n, m)
def plan_sph_analysis(n: int, m: int = None) -> SphereGridPlan: return _grid_plan("sph_analysis", n, m)
def plan_sphv_synthesis(n: int, m: int = None) -> SphereGridPlan: return _grid_plan("sphv_synthesis", n, m)
def plan_sphv_analysis(n: int, m: int = None) -> SphereGridPlan: return _grid_plan("sphv_analysis", n, m)


GRID_OPS = {"sph_synthesis": 0, "sph_analysis": 1, "sphv_synthesis": 2, "sphv_analysis": 3}


class _FamilyGridPlan(SphereGridPlan):
    """A disk or triangle grid plan (reference: src/fftw.c:279-330, 404-532)."""

    _destroy = None

    def close(self):
        if self.ptr:
            getattr(lib, self._destroy)(self.ptr)
            self.ptr = None


class DiskGridPlan(_FamilyGridPlan):
    _destroy = "ft_destroy_disk_fftw_plan"


class TriGridPlan(_FamilyGridPlan):
    _destroy = "ft_destroy_triangle_fftw_plan"


class AnnulusGridPlan(_FamilyGridPlan):
    _destroy = "ft_destroy_annulus_fftw_plan"

    @property
    def rho(self) -> float:
        return lib.ft_get_rho_annulus_fftw_plan(self.ptr)


class RectdiskGridPlan(_FamilyGridPlan):
    _destroy = "ft_destroy_rectdisk_fftw_plan"


class TetGridPlan(_FamilyGridPlan):
    _destroy = "ft_destroy_tetrahedron_fftw_plan"


def plan_tet_synthesis(n: int) -> TetGridPlan:
    ptr = lib.ft_plan_tet_synthesis(n, n, n, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return TetGridPlan(ptr, "tet_synthesis", n, n)


def plan_tet_analysis(n: int) -> TetGridPlan:
    ptr = lib.ft_plan_tet_analysis(n, n, n, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return TetGridPlan(ptr, "tet_analysis", n, n)


def execute_tet_synthesis(trans, P, A): _exec_tet("ft_execute_tet_synthesis", trans, P, A)
def execute_tet_analysis(trans, P, A): _exec_tet("ft_execute_tet_analysis", trans, P, A)


def execute_tet_grid_dev(P: TetGridPlan, analysis: bool, trans: str, ptr: int, N: int, L: int, M: int, stream: int = 0) -> None:
    """The tetrahedron grid's synthesis (analysis = False) or analysis sequence with P's kind on a device tensor."""
    st = lib.ft_b200_execute_tet_grid_dev(P.ptr, 1 if analysis else 0, trans.encode(), C.c_void_p(ptr), N, L, M, C.c_void_p(stream))
    if st != 0:
        _check()


def plan_annulus_synthesis(n: int, rho: float, m: int = None) -> AnnulusGridPlan:
    m = 4 * n - 3 if m is None else m
    ptr = lib.ft_plan_annulus_synthesis(n, m, rho, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return AnnulusGridPlan(ptr, "annulus_synthesis", n, m)


def plan_annulus_analysis(n: int, rho: float, m: int = None) -> AnnulusGridPlan:
    m = 4 * n - 3 if m is None else m
    ptr = lib.ft_plan_annulus_analysis(n, m, rho, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return AnnulusGridPlan(ptr, "annulus_analysis", n, m)


def plan_rectdisk_synthesis(n: int, m: int = None) -> RectdiskGridPlan: return _family_plan(RectdiskGridPlan, "ft_plan_rectdisk_synthesis", n, n if m is None else m)
def plan_rectdisk_analysis(n: int, m: int = None) -> RectdiskGridPlan: return _family_plan(RectdiskGridPlan, "ft_plan_rectdisk_analysis", n, n if m is None else m)


def execute_annulus_grid_dev(P: AnnulusGridPlan, analysis: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """The annulus grid's synthesis (analysis = False) or analysis sequence with P's kind and rho."""
    st = lib.ft_b200_execute_annulus_grid_dev(P.ptr, 1 if analysis else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_rectdisk_grid_dev(P: RectdiskGridPlan, analysis: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """The rectangularised disk grid's synthesis (analysis = False) or analysis sequence with P's kinds."""
    st = lib.ft_b200_execute_rectdisk_grid_dev(P.ptr, 1 if analysis else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def _family_plan(cls, fname, n, m):
    ptr = getattr(lib, fname)(n, m, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return cls(ptr, fname[8:], n, m)


def plan_disk_synthesis(n: int, m: int = None) -> DiskGridPlan: return _family_plan(DiskGridPlan, "ft_plan_disk_synthesis", n, 4 * n - 3 if m is None else m)
def plan_disk_analysis(n: int, m: int = None) -> DiskGridPlan: return _family_plan(DiskGridPlan, "ft_plan_disk_analysis", n, 4 * n - 3 if m is None else m)
def plan_tri_synthesis(n: int, m: int = None) -> TriGridPlan: return _family_plan(TriGridPlan, "ft_plan_tri_synthesis", n, n if m is None else m)
def plan_tri_analysis(n: int, m: int = None) -> TriGridPlan: return _family_plan(TriGridPlan, "ft_plan_tri_analysis", n, n if m is None else m)


def execute_disk_grid_dev(P: DiskGridPlan, analysis: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """The disk grid's synthesis (analysis = False) or analysis sequence with P's kinds on a device matrix."""
    st = lib.ft_b200_execute_disk_grid_dev(P.ptr, 1 if analysis else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_tri_grid_dev(P: TriGridPlan, analysis: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """The triangle grid's synthesis (analysis = False) or analysis sequence with P's kinds on a device matrix."""
    st = lib.ft_b200_execute_tri_grid_dev(P.ptr, 1 if analysis else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_sph_grid_dev(P: SphereGridPlan, op: str, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """Grid synthesis / analysis (op: a key of GRID_OPS) on a device matrix, asynchronous."""
    st = lib.ft_b200_execute_sph_grid_dev(P.ptr, GRID_OPS[op], trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


class SpinRotationPlan(HarmonicPlan):
    """Owns an ``ft_spin_rotation_plan *`` (reference: src/rotations.c:431-478)."""

    def __init__(self, ptr: int, n: int, s: int):
        super().__init__(ptr, "spin", n)
        self.s = s

    def close(self):
        if self.ptr:
            lib.ft_destroy_spin_rotation_plan(self.ptr)
            self.ptr = None


class SpinHarmonicPlan(SpinRotationPlan):
    """Owns an ``ft_spin_harmonic_plan *`` (reference: src/drivers.c:1259-1361)."""

    def close(self):
        if self.ptr:
            lib.ft_destroy_spin_harmonic_plan(self.ptr)
            self.ptr = None


def plan_rotspinsphere(n: int, s: int) -> SpinRotationPlan:
    p = lib.ft_plan_rotspinsphere(n, s)
    if not p:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return SpinRotationPlan(p, n, s)


def plan_spinsph2fourier(n: int, s: int) -> SpinHarmonicPlan:
    p = lib.ft_plan_spinsph2fourier(n, s)
    if not p:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return SpinHarmonicPlan(p, n, s)


def _complex_matrix(A: np.ndarray) -> np.ndarray:
    if not (isinstance(A, np.ndarray) and A.dtype == np.complex128 and A.ndim == 2 and A.flags.f_contiguous and A.flags.writeable):
        raise TypeError("A must be a writeable 2-D complex128 numpy array in Fortran order")
    return A


def _exec_spin(fname: str, trans: str, P: SpinHarmonicPlan, A: np.ndarray, N=None, M=None):
    A = _complex_matrix(A)
    N = A.shape[0] if N is None else N
    M = A.shape[1] if M is None else M
    if N * M > A.size:
        raise ValueError("N x M exceeds the array")
    getattr(lib, fname)(trans.encode(), P.ptr, A.ctypes.data_as(C.POINTER(C.c_double)), N, M)
    _check()


def execute_spinsph2fourier(trans, P, A, N=None, M=None): _exec_spin("ft_execute_spinsph2fourier", trans, P, A, N, M)
def execute_fourier2spinsph(trans, P, A, N=None, M=None): _exec_spin("ft_execute_fourier2spinsph", trans, P, A, N, M)


def _exec_spin_rot(fname, SRP, A, M=None):
    A = _complex_matrix(A)
    M = A.shape[1] if M is None else M
    if A.shape[0] != SRP.n or M > A.shape[1]:
        raise ValueError("A must have the plan's n rows and at least M columns")
    getattr(lib, fname)(SRP.ptr, A.ctypes.data_as(C.POINTER(C.c_double)), None, M)
    _check()


def execute_spinsph_hi2lo(SRP, A, M=None): _exec_spin_rot("ft_execute_spinsph_hi2lo", SRP, A, M)
def execute_spinsph_lo2hi(SRP, A, M=None): _exec_spin_rot("ft_execute_spinsph_lo2hi", SRP, A, M)


class SpinGridPlan(_FamilyGridPlan):
    """Owns an ``ft_spinsphere_fftw_plan *`` (reference: src/fftw.c:743-960)."""

    _destroy = "ft_destroy_spinsphere_fftw_plan"

    @property
    def s(self) -> int:
        return lib.ft_get_spin_spinsphere_fftw_plan(self.ptr)


def _spin_grid_plan(fname, n, s, m):
    m = 2 * n - 1 if m is None else m
    ptr = getattr(lib, fname)(n, m, s, 0)
    if not ptr:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return SpinGridPlan(ptr, fname[8:], n, m)


def plan_spinsph_synthesis(n: int, s: int, m: int = None) -> SpinGridPlan:
    return _spin_grid_plan("ft_plan_spinsph_synthesis", n, s, m)


def plan_spinsph_analysis(n: int, s: int, m: int = None) -> SpinGridPlan:
    return _spin_grid_plan("ft_plan_spinsph_analysis", n, s, m)


def execute_spinsph_synthesis(trans, P, A, N=None, M=None): _exec_spin("ft_execute_spinsph_synthesis", trans, P, A, N, M)
def execute_spinsph_analysis(trans, P, A, N=None, M=None): _exec_spin("ft_execute_spinsph_analysis", trans, P, A, N, M)


def execute_spinsph_grid_dev(P: SpinGridPlan, analysis: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """The spin grid's synthesis (analysis = False) or analysis sequence with P's kinds on a device
    matrix of N x M interleaved complex doubles, asynchronous."""
    st = lib.ft_b200_execute_spinsph_grid_dev(P.ptr, 1 if analysis else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_spin_dev(P: SpinHarmonicPlan, forward: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """Spin-weighted transform on a device matrix of N x M interleaved complex doubles."""
    st = lib.ft_b200_execute_spin_dev(P.ptr, 1 if forward else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def spin_rotations_dev(SRP: SpinRotationPlan, hi2lo: bool, ptr: int, M: int, stream: int = 0) -> None:
    """The spin rotation stage alone on a device matrix (interleaved complex)."""
    st = lib.ft_b200_spin_rotations_dev(SRP.ptr, 1 if hi2lo else 0, C.c_void_p(ptr), M, C.c_void_p(stream))
    if st != 0:
        _check()


class TetPlan(HarmonicPlan):
    """Owns a tetrahedral ``ft_harmonic_plan *`` (reference: src/drivers.c:1173-1257); tensors are
    n x n x n float64 in Fortran order."""

    def __init__(self, ptr: int, n: int, params):
        super().__init__(ptr, "tet", n, params)
        self.RP = C.cast(C.c_void_p(ptr), C.POINTER(C.c_void_p))[0]   # the plan's RP member: its two rotation plans

    @property
    def M(self) -> int:
        return self.n


def plan_tet2cheb(n: int, alpha: float, beta: float, gamma: float, delta: float) -> TetPlan:
    p = lib.ft_plan_tet2cheb(n, alpha, beta, gamma, delta)
    if not p:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return TetPlan(p, n, (alpha, beta, gamma, delta))


def _tensor(A: np.ndarray) -> np.ndarray:
    if not (isinstance(A, np.ndarray) and A.dtype == np.float64 and A.ndim == 3 and A.flags.f_contiguous and A.flags.writeable):
        raise TypeError("A must be a writeable 3-D float64 numpy array in Fortran order")
    return A


def _exec_tet(fname: str, trans: str, P: TetPlan, A: np.ndarray):
    A = _tensor(A)
    N, L, M = A.shape
    getattr(lib, fname)(trans.encode(), P.ptr, A.ctypes.data_as(C.POINTER(C.c_double)), N, L, M)
    _check()


def execute_tet2cheb(trans, P, A): _exec_tet("ft_execute_tet2cheb", trans, P, A)
def execute_cheb2tet(trans, P, A): _exec_tet("ft_execute_cheb2tet", trans, P, A)


def _exec_tet_rot(fname, P: TetPlan, A: np.ndarray):
    """ft_execute_tet_hi2lo / lo2hi with the plan's two rotation plans."""
    A = _tensor(A)
    rp = C.cast(C.c_void_p(P.RP), C.POINTER(C.c_void_p))
    getattr(lib, fname)(rp[0], rp[1], A.ctypes.data_as(C.POINTER(C.c_double)), A.shape[1], A.shape[2])
    _check()


def execute_tet_hi2lo(P, A): _exec_tet_rot("ft_execute_tet_hi2lo", P, A)
def execute_tet_lo2hi(P, A): _exec_tet_rot("ft_execute_tet_lo2hi", P, A)


def execute_tet_dev(P: TetPlan, forward: bool, trans: str, ptr: int, N: int, L: int, M: int, stream: int = 0) -> None:
    """Tetrahedral transform on a device tensor (N x L x M, column-major), asynchronous."""
    st = lib.ft_b200_execute_tet_dev(P.ptr, 1 if forward else 0, trans.encode(), C.c_void_p(ptr), N, L, M, C.c_void_p(stream))
    if st != 0:
        _check()


def tet_rotations_dev(P: TetPlan, hi2lo: bool, ptr: int, L: int, M: int, stream: int = 0) -> None:
    """The plan's tetrahedral rotation stage alone on a device tensor."""
    st = lib.ft_b200_tet_rotations_dev(P.ptr, 1 if hi2lo else 0, C.c_void_p(ptr), L, M, C.c_void_p(stream))
    if st != 0:
        _check()


def _host_matrix(A: np.ndarray) -> np.ndarray:
    if not (isinstance(A, np.ndarray) and A.dtype == np.float64 and A.ndim == 2 and A.flags.f_contiguous and A.flags.writeable):
        raise TypeError("A must be a writeable 2-D float64 numpy array in Fortran order")
    return A


def _exec_host(fname: str, trans: str, P: HarmonicPlan, A: np.ndarray, N=None, M=None):
    A = _host_matrix(A)
    N = A.shape[0] if N is None else N
    M = A.shape[1] if M is None else M
    if N * M > A.size:
        raise ValueError("N x M exceeds the array")
    getattr(lib, fname)(trans.encode(), P.ptr, A.ctypes.data_as(C.POINTER(C.c_double)), N, M)
    _check()


def execute_sph2fourier(trans, P, A, N=None, M=None): _exec_host("ft_execute_sph2fourier", trans, P, A, N, M)
def execute_sph_synthesis(trans, P, A, N=None, M=None): _exec_host("ft_execute_sph_synthesis", trans, P, A, N, M)
def execute_sph_analysis(trans, P, A, N=None, M=None): _exec_host("ft_execute_sph_analysis", trans, P, A, N, M)
def execute_sphv_synthesis(trans, P, A, N=None, M=None): _exec_host("ft_execute_sphv_synthesis", trans, P, A, N, M)
def execute_sphv_analysis(trans, P, A, N=None, M=None): _exec_host("ft_execute_sphv_analysis", trans, P, A, N, M)
def execute_disk_synthesis(trans, P, A, N=None, M=None): _exec_host("ft_execute_disk_synthesis", trans, P, A, N, M)
def execute_disk_analysis(trans, P, A, N=None, M=None): _exec_host("ft_execute_disk_analysis", trans, P, A, N, M)
def execute_tri_synthesis(trans, P, A, N=None, M=None): _exec_host("ft_execute_tri_synthesis", trans, P, A, N, M)
def execute_tri_analysis(trans, P, A, N=None, M=None): _exec_host("ft_execute_tri_analysis", trans, P, A, N, M)
def execute_annulus_synthesis(trans, P, A, N=None, M=None): _exec_host("ft_execute_annulus_synthesis", trans, P, A, N, M)
def execute_annulus_analysis(trans, P, A, N=None, M=None): _exec_host("ft_execute_annulus_analysis", trans, P, A, N, M)
def execute_rectdisk_synthesis(trans, P, A, N=None, M=None): _exec_host("ft_execute_rectdisk_synthesis", trans, P, A, N, M)
def execute_rectdisk_analysis(trans, P, A, N=None, M=None): _exec_host("ft_execute_rectdisk_analysis", trans, P, A, N, M)
def execute_fourier2sph(trans, P, A, N=None, M=None): _exec_host("ft_execute_fourier2sph", trans, P, A, N, M)
def execute_tri2cheb(trans, P, A, N=None, M=None): _exec_host("ft_execute_tri2cheb", trans, P, A, N, M)
def execute_cheb2tri(trans, P, A, N=None, M=None): _exec_host("ft_execute_cheb2tri", trans, P, A, N, M)
def execute_disk2cxf(trans, P, A, N=None, M=None): _exec_host("ft_execute_disk2cxf", trans, P, A, N, M)
def execute_cxf2disk(trans, P, A, N=None, M=None): _exec_host("ft_execute_cxf2disk", trans, P, A, N, M)
def execute_sphv2fourier(trans, P, A, N=None, M=None): _exec_host("ft_execute_sphv2fourier", trans, P, A, N, M)
def execute_fourier2sphv(trans, P, A, N=None, M=None): _exec_host("ft_execute_fourier2sphv", trans, P, A, N, M)
def execute_rectdisk2cheb(trans, P, A, N=None, M=None): _exec_host("ft_execute_rectdisk2cheb", trans, P, A, N, M)
def execute_ann2cxf(trans, P, A, N=None, M=None): _exec_host("ft_execute_ann2cxf", trans, P, A, N, M)
def execute_cxf2ann(trans, P, A, N=None, M=None): _exec_host("ft_execute_cxf2ann", trans, P, A, N, M)
def execute_cheb2rectdisk(trans, P, A, N=None, M=None): _exec_host("ft_execute_cheb2rectdisk", trans, P, A, N, M)


def plan_rotsphere(n: int) -> RotationPlan:
    p = lib.ft_plan_rotsphere(n)
    if not p:
        _check()
    return RotationPlan(p, "sph", n)


def plan_rottriangle(n: int, alpha: float, beta: float, gamma: float) -> RotationPlan:
    p = lib.ft_plan_rottriangle(n, alpha, beta, gamma)
    if not p:
        _check()
    return RotationPlan(p, "tri", n, (alpha, beta, gamma))


def plan_rotdisk(n: int, alpha: float, beta: float) -> RotationPlan:
    p = lib.ft_plan_rotdisk(n, alpha, beta)
    if not p:
        _check()
    return RotationPlan(p, "disk", n, (alpha, beta))


def plan_rotannulus(n: int, alpha: float, beta: float, gamma: float, rho: float) -> RotationPlan:
    """A disk-kind rotation plan with the annulus table (use execute_disk_hi2lo / lo2hi)."""
    p = lib.ft_plan_rotannulus(n, alpha, beta, gamma, rho)
    if not p:
        _check()
        raise FTB200Error(-1, "plan creation failed")
    return RotationPlan(p, "disk", n, (alpha, beta, gamma, rho))


def plan_rotrectdisk(n: int, beta: float) -> RotationPlan:
    p = lib.ft_plan_rotrectdisk(n, beta)
    if not p:
        _check()
    return RotationPlan(p, "rect", n, (beta,))


def _exec_rot(fname, RP, A, M=None):
    A = _host_matrix(A)
    M = A.shape[1] if M is None else M
    getattr(lib, fname)(RP.ptr, A.ctypes.data_as(C.POINTER(C.c_double)), None, M)
    _check()


def execute_sph_hi2lo(RP, A, M=None): _exec_rot("ft_execute_sph_hi2lo", RP, A, M)
def execute_sph_lo2hi(RP, A, M=None): _exec_rot("ft_execute_sph_lo2hi", RP, A, M)
def execute_tri_hi2lo(RP, A, M=None): _exec_rot("ft_execute_tri_hi2lo", RP, A, M)
def execute_tri_lo2hi(RP, A, M=None): _exec_rot("ft_execute_tri_lo2hi", RP, A, M)
def execute_disk_hi2lo(RP, A, M=None): _exec_rot("ft_execute_disk_hi2lo", RP, A, M)
def execute_disk_lo2hi(RP, A, M=None): _exec_rot("ft_execute_disk_lo2hi", RP, A, M)
def execute_rectdisk_hi2lo(RP, A, M=None): _exec_rot("ft_execute_rectdisk_hi2lo", RP, A, M)
def execute_rectdisk_lo2hi(RP, A, M=None): _exec_rot("ft_execute_rectdisk_lo2hi", RP, A, M)
def execute_sphv_hi2lo(RP, A, M=None): _exec_rot("ft_execute_sphv_hi2lo", RP, A, M)
def execute_sphv_lo2hi(RP, A, M=None): _exec_rot("ft_execute_sphv_lo2hi", RP, A, M)


_KERNEL_FAMILY = {"sph": "sph", "tri": "tri", "disk": "disk", "rect": "rectdisk"}


def kernel_column(RP: "RotationPlan", hi2lo: bool, m1: int, m2: int, a: np.ndarray, S: int = 1) -> None:
    """ft_kernel_<family>_{hi2lo,lo2hi}(RP, m1, m2, a, S) on a writeable float64 host array, in
    place: the sweeps between orders m1 and m2 on the column a[0], a[S], a[2 S], .."""
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.ndim == 1 and a.flags.c_contiguous and a.flags.writeable):
        raise TypeError("a must be a writeable contiguous 1-D float64 array")
    if S < 1 or (a.size - 1) // S + 1 < RP.n:
        raise ValueError("a must hold the plan's n entries at stride S")
    fam = _KERNEL_FAMILY[RP.kind]
    getattr(lib, f"ft_kernel_{fam}_{'hi2lo' if hi2lo else 'lo2hi'}")(RP.ptr, m1, m2, a.ctypes.data_as(C.POINTER(C.c_double)), S)
    _check()


def kernel_spin_column(SRP: "SpinRotationPlan", hi2lo: bool, m: int, a: np.ndarray, S: int = 1) -> None:
    """ft_kernel_spinsph_{hi2lo,lo2hi}(SRP, m, a, S) on a writeable complex128 host array, in place:
    the column a[0], a[S], a[2 S], .. of order m."""
    if not (isinstance(a, np.ndarray) and a.dtype == np.complex128 and a.ndim == 1 and a.flags.c_contiguous and a.flags.writeable):
        raise TypeError("a must be a writeable contiguous 1-D complex128 array")
    if S < 1 or (a.size - 1) // S + 1 < SRP.n:
        raise ValueError("a must hold the plan's n entries at stride S")
    f = lib.ft_kernel_spinsph_hi2lo if hi2lo else lib.ft_kernel_spinsph_lo2hi
    f(SRP.ptr, m, a.ctypes.data_as(C.POINTER(C.c_double)), S)
    _check()


def kernel_tet_slab(RP: "RotationPlan", hi2lo: bool, L: int, m: int, a: np.ndarray) -> None:
    """ft_kernel_tet_{hi2lo,lo2hi}(RP, L, m, a) on the n x L slab a (float64, Fortran order), in place."""
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.ndim == 2 and a.flags.f_contiguous and a.flags.writeable):
        raise TypeError("a must be a writeable 2-D float64 array in Fortran order")
    if a.shape != (RP.n, L):
        raise ValueError("a must be n x L")
    f = lib.ft_kernel_tet_hi2lo if hi2lo else lib.ft_kernel_tet_lo2hi
    f(RP.ptr, L, m, a.ctypes.data_as(C.POINTER(C.c_double)))
    _check()


def execute_dev(P: HarmonicPlan, forward: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """Full transform on a device matrix (N x M, column-major) enqueued on ``stream``."""
    st = lib.ft_b200_execute_dev(P.ptr, 1 if forward else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_sphv_dev(P: HarmonicPlan, forward: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """sph vector-field transform (sphv2fourier / fourier2sphv) on a device matrix, sph plan."""
    st = lib.ft_b200_execute_sphv_dev(P.ptr, 1 if forward else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


NOALLOC_MAX_ELEMS = 1 << 20


def execute_noalloc_dev(P: HarmonicPlan, forward: bool, trans: str, ptr: int, N: int, M: int, stream: int = 0) -> None:
    """Like execute_dev, but the library allocates no device memory for the call.

    For callers that manage all device memory themselves and cannot let a
    library call cudaMalloc: the intermediate matrix lives in a fixed 8 MiB
    device array inside the library, so N*M is limited to NOALLOC_MAX_ELEMS and
    M must be the plan's default.  The array is shared by every call: calls that
    overlap on the GPU race and must be serialised by the caller.
    """
    st = lib.ft_b200_execute_noalloc_dev(P.ptr, 1 if forward else 0, trans.encode(), C.c_void_p(ptr), N, M, C.c_void_p(stream))
    if st != 0:
        _check()


FP64, FP64_BLOCKED, MIXED_BF16, MIXED_BF16X4 = 0, 1, 2, 3


def execute_shared_dev(P: HarmonicPlan, forward: bool, trans: str, ptrs: Sequence[int], precision: int = FP64,
                       stream: int = 0) -> None:
    """Transform every field of ``ptrs`` (device matrices sharing plan ``P``) in one call.

    precision FP64: the direct sweeps; FP64_BLOCKED: whole blocks of 32 sweeps
    applied as pre-multiplied 64 x 64 tile matrices on the FP64 tensor pipe
    (rounds differently from the direct sweeps, ~1e-14 relative); MIXED_BF16:
    the tile products and the connection multiply on the BF16 tensor cores
    from fixed-point BF16 slices (three per operand in the blocks, ~5e-7
    relative for sph at n = 4096); MIXED_BF16X4: four slices in the blocks and
    of the multiply's input (~1.4e-7 for sph at n = 2048).  All three
    families; the errors of tri and of generic disk parameters are larger (the
    connection multiplies amplify the sweeps' error).
    """
    nf = len(ptrs)
    aa = (C.c_void_p * nf)(*ptrs)
    st = lib.ft_b200_execute_shared_dev(P.ptr, 1 if forward else 0, trans.encode(), aa, nf, precision, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_shared_host(P: HarmonicPlan, ops: Sequence[tuple], arrays: Sequence, precision: int = FP64) -> None:
    """Host-pointer form of ``execute_shared_dev`` for a sequence of transforms.

    ``ops``: (forward, trans) pairs applied in order to every field; ``arrays``:
    N x M float64 host matrices in column-major order (numpy arrays in Fortran
    order, or the flat buffers of page-locked tensors as integer addresses),
    transformed in place.  Copies of one group of fields overlap the
    transforms of the previous group (page-locked memory only); the call
    returns when every result is back in host memory.
    """
    nops = len(ops)
    fw = (C.c_int * max(nops, 1))(*[1 if f else 0 for f, _ in ops])
    tr = "".join(t for _, t in ops).encode()
    ptrs = []
    for a in arrays:
        if isinstance(a, int):
            ptrs.append(a)
        else:
            if a.dtype != np.float64 or not a.flags.f_contiguous or a.shape != (P.n, P.M):
                raise ValueError(f"each field must be a float64 Fortran-order {P.n} x {P.M} array")
            ptrs.append(a.ctypes.data)
    nf = len(ptrs)
    aa = (C.c_void_p * max(nf, 1))(*ptrs)
    st = lib.ft_b200_execute_shared_host(P.ptr, nops, fw, tr, aa, nf, precision)
    if st != 0:
        _check()


def device_status(P: HarmonicPlan) -> int:
    """Read and clear the plan's device status word (nonzero: a tensor-core wait gave up)."""
    v = lib.ft_b200_device_status(P.ptr)
    if v < 0:
        _check()
    return v


def rotations_dev(RP: RotationPlan, hi2lo: bool, ptr: int, M: int, stream: int = 0) -> None:
    st = lib.ft_b200_rotations_dev(RP.ptr, 1 if hi2lo else 0, C.c_void_p(ptr), M, C.c_void_p(stream))
    if st != 0:
        _check()


def execute_batched_dev(plans: Sequence[HarmonicPlan], forward: bool, trans: str, ptrs: Sequence[int],
                        N: Sequence[int], M: Sequence[int], stream: int = 0) -> None:
    nf = len(plans)
    pa = (C.c_void_p * nf)(*[p.ptr for p in plans])
    aa = (C.c_void_p * nf)(*ptrs)
    na = (C.c_int * nf)(*N)
    ma = (C.c_int * nf)(*M)
    st = lib.ft_b200_execute_batched_dev(pa, 1 if forward else 0, trans.encode(), aa, na, ma, nf, C.c_void_p(stream))
    if st != 0:
        _check()
