"""Generate the golden fixtures in this directory from the reference library.

The reference FastTransforms library is compiled from its own sources by
oracle/ref_build/Makefile into oracle/_ref/libft_ref.so; this script runs it on
seeded inputs and stores inputs and outputs as compressed .npz files:

  * full transforms: forward and backward, TRANS 'N' and 'T', each applied to
    the same seeded input (sph, tri and disk families, small degrees, even and
    odd n, several Jacobi parameters); for sph also the vector-field transforms
    (ft_execute_sphv2fourier / ft_execute_fourier2sphv, keys "v_fwd_N" ...);
  * rotation stages alone (ft_execute_*_hi2lo / _lo2hi);
  * the four dense connection matrices of each plan;
  * spin-weighted transforms (ft_execute_spinsph2fourier / ft_execute_fourier2spinsph and
    the rotation stages ft_execute_spinsph_hi2lo / _lo2hi) on complex inputs in
    spinsphrand's layout, files spin_n<n>_s<s>.npz;
  * Dunkl-Xu (rectangularised disk) transforms (ft_execute_rectdisk2cheb /
    ft_execute_cheb2rectdisk, M = N), their rotation stages (ft_execute_rectdisk_hi2lo /
    _lo2hi) and the six connection matrices, files rect_n<n>_b<beta>.npz;
  * tetrahedral transforms (ft_execute_tet2cheb / ft_execute_cheb2tet, N = L = M), their
    rotation stages (ft_execute_tet_hi2lo / _lo2hi) and the six connection matrices, files
    tet_n<n>_<params>.npz;
  * annulus transforms (ft_execute_ann2cxf / ft_execute_cxf2ann, gamma = 0, M = 4N - 3), the
    annulus rotation table (ft_plan_rotannulus) and its sweeps through ft_execute_disk_hi2lo /
    _lo2hi, files ann_n<n>_<params>.npz.

    python tests/golden/make_golden.py [sph tri disk spin rect tet ann]   (default: all)
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.bind import Reference, _ptr, fill, fill_spin  # noqa: E402

CASES = [
    ("sph", 8, ()), ("sph", 17, ()), ("sph", 33, ()),
    ("tri", 16, (0.0, 0.0, 0.0)), ("tri", 17, (-0.5, -0.5, -0.5)), ("tri", 16, (0.5, 1.0, -0.25)),
    ("disk", 9, (0.0, 0.0)), ("disk", 16, (0.0, 0.0)), ("disk", 12, (0.5, -0.25)),
]
SPIN_CASES = [(8, -2), (17, 0), (17, 1), (16, 3), (33, -1), (12, 4)]
RECT_CASES = [(8, 0.0), (17, 0.5), (16, -0.25), (33, 1.5)]
ANN_CASES = [(8, (0.0, 0.0, 0.5773502691896257)), (13, (0.5, -0.25, 0.4)), (16, (0.0, 0.0, 0.0))]
TET_CASES = [(8, (0.0, 0.0, 0.0, 0.0)), (9, (-0.5, -0.5, -0.5, -0.5)), (12, (0.5, -0.25, 0.25, 1.0))]
SEED = 20261203


def case_name(kind, n, params):
    tag = "_".join(f"{p:+.2f}".replace(".", "p").replace("+", "p").replace("-", "m") for p in params)
    return f"{kind}_n{n}" + (f"_{tag}" if tag else "")


def main():
    R = Reference()
    R.set_num_threads(1)
    L = R.lib
    planner = {"sph": ("ft_plan_rotsphere", [C.c_int]), "tri": ("ft_plan_rottriangle", [C.c_int] + [C.c_double] * 3),
               "disk": ("ft_plan_rotdisk", [C.c_int] + [C.c_double] * 2)}
    for name, args in planner.values():
        getattr(L, name).restype = C.c_void_p
        getattr(L, name).argtypes = args
    for fam in ("sph", "tri", "disk"):
        for d in ("hi2lo", "lo2hi"):
            getattr(L, f"ft_execute_{fam}_{d}").argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
    L.ft_destroy_rotation_plan.argtypes = [C.c_void_p]
    families = set(sys.argv[1:]) or {"sph", "tri", "disk", "spin", "rect", "tet", "ann"}
    for kind, n, params in CASES:
        if kind not in families:
            continue
        A = fill(kind, n, SEED)
        P = R.plan(kind, n, *params)
        out = {"A": A, "params": np.array(params, dtype=np.float64)}
        for fwd in (True, False):
            for tr in "NT":
                B = A.copy(order="F")
                R.execute(kind, P, fwd, tr, B)
                out[("fwd" if fwd else "bwd") + "_" + tr] = B
                if kind == "sph":
                    V = A.copy(order="F")
                    R.execute("sphv", P, fwd, tr, V)
                    out["v_" + ("fwd" if fwd else "bwd") + "_" + tr] = V
        Ps, Pinvs = R.connection(P, n)
        out["P0"], out["P1"], out["Pinv0"], out["Pinv1"] = Ps[0], Ps[1], Pinvs[0], Pinvs[1]
        R.destroy(P)
        pname, _ = planner[kind]
        RP = getattr(L, pname)(n, *params[: 3 if kind == "tri" else 2]) if params else getattr(L, pname)(n)
        for d in ("hi2lo", "lo2hi"):
            B = A.copy(order="F")
            scratch = np.zeros_like(B, order="F")
            getattr(L, f"ft_execute_{kind}_{d}")(RP, _ptr(B), _ptr(scratch), A.shape[1])
            out["rot_" + d] = B
        L.ft_destroy_rotation_plan(RP)
        path = os.path.join(HERE, case_name(kind, n, params) + ".npz")
        np.savez_compressed(path, **out)
        print("wrote", os.path.relpath(path), A.shape)
    if "spin" in families:
        for n, sw in SPIN_CASES:
            M = 2 * n - 1
            A = fill_spin(n, M, sw, SEED)
            P = R.spin_plan(n, sw)
            out = {"A": A, "s": np.array(sw)}
            for fwd in (True, False):
                for tr in "NT":
                    B = A.copy(order="F")
                    R.spin_execute(P, fwd, tr, B)
                    out[("fwd" if fwd else "bwd") + "_" + tr] = B
            R.spin_destroy(P)
            for d in ("hi2lo", "lo2hi"):
                B = A.copy(order="F")
                R.spin_rotations(n, sw, d == "hi2lo", B)
                out["rot_" + d] = B
            path = os.path.join(HERE, f"spin_n{n}_s{sw}.npz".replace("-", "m"))
            np.savez_compressed(path, **out)
            print("wrote", os.path.relpath(path), A.shape)
    if "rect" in families:
        for n, beta in RECT_CASES:
            A = fill("rect", n, SEED)
            P = R.plan("rect", n, beta=beta)
            out = {"A": A, "beta": np.array(beta)}
            for fwd in (True, False):
                for tr in "NT":
                    B = A.copy(order="F")
                    R.execute("rect", P, fwd, tr, B)
                    out[("fwd" if fwd else "bwd") + "_" + tr] = B
            Ps, Pinvs = R.connection(P, n)
            for i in range(3):
                out[f"P{i}"], out[f"Pinv{i}"] = Ps[i], Pinvs[i]
            R.destroy(P)
            for d in ("hi2lo", "lo2hi"):
                B = A.copy(order="F")
                R.rect_rotations(n, beta, d == "hi2lo", B)
                out["rot_" + d] = B
            path = os.path.join(HERE, case_name("rect", n, (beta,)) + ".npz")
            np.savez_compressed(path, **out)
            print("wrote", os.path.relpath(path), A.shape)
    if "ann" in families:
        for n, (a, b, rho) in ANN_CASES:
            A = fill("disk", n, SEED)
            P = R.ann_plan(n, a, b, rho)
            out = {"A": A, "params": np.array((a, b, rho), dtype=np.float64)}
            for fwd in (True, False):
                for tr in "NT":
                    B = A.copy(order="F")
                    R.ann_execute(P, fwd, tr, B)
                    out[("fwd" if fwd else "bwd") + "_" + tr] = B
            R.destroy(P)
            out["s"], out["c"] = R.ann_table(n, a, b, rho)
            for d in ("hi2lo", "lo2hi"):
                B = A.copy(order="F")
                R.ann_rotations(n, a, b, rho, d == "hi2lo", B)
                out["rot_" + d] = B
            path = os.path.join(HERE, case_name("ann", n, (a, b, rho)) + ".npz")
            np.savez_compressed(path, **out)
            print("wrote", os.path.relpath(path), A.shape)
    if "tet" in families:
        from fasttransforms_b200.utilities import tetrand
        for n, params in TET_CASES:
            A = tetrand(n, SEED)
            P = R.tet_plan(n, *params)
            out = {"A": A, "params": np.array(params, dtype=np.float64)}
            for fwd in (True, False):
                for tr in "NT":
                    B = A.copy(order="F")
                    R.tet_execute(P, fwd, tr, B)
                    out[("fwd" if fwd else "bwd") + "_" + tr] = B
            Ps, Pinvs = R.connection(P, n)
            for i in range(3):
                out[f"P{i}"], out[f"Pinv{i}"] = Ps[i], Pinvs[i]
            R.destroy(P)
            for d in ("hi2lo", "lo2hi"):
                B = A.copy(order="F")
                R.tet_rotations(n, params, d == "hi2lo", B)
                out["rot_" + d] = B
            path = os.path.join(HERE, case_name("tet", n, params) + ".npz")
            np.savez_compressed(path, **out)
            print("wrote", os.path.relpath(path), A.shape)


if __name__ == "__main__":
    main()
