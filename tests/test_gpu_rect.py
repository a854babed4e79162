"""Dunkl-Xu (rectangularised disk) transforms on the GPU (ft_plan_rotrectdisk,
ft_execute_rectdisk_hi2lo / lo2hi, ft_plan_rectdisk2cheb, ft_execute_rectdisk2cheb /
cheb2rectdisk: src/rotations.c:270-287, src/drivers.c:488-508, 1123-1171), through the C ABI.

Against the oracle (oracle/ft_oracle.c, pinned to the compiled reference in
tests/test_oracle_rect.py) in its fused form: the rotation stage bit for bit, for every
launch shape of the rotation kernel; the transforms within 1e-14 relative 2-norm (or twice
the oracle's distance from the compiled reference where that is larger).  Against
the reference's golden fixtures: the plan's connection matrices bit for bit, the
transforms within 1e-14, the rotation stages within 1e-15 (the reference runs the unfused
scalar kernel).  The reference's round trips (test/test_drivers.c:1179-1200, 1230-1252)
within 4 sqrt(N) eps and 2N eps at its beta = 0, within twice the oracle's (the
reference algorithm's) own error at beta = 1/2."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "rect_*.npz")))
BETAS = [0.0, 0.5, -0.25, 1.5]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


def run_dev(ft, torch, fn, A):
    t = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()
    fn(t.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return t.cpu().numpy().reshape(A.shape, order="F")


def rot_dev(ft, torch, RP, hi2lo, A):
    return run_dev(ft, torch, lambda p, s: ft.rotations_dev(RP, hi2lo, p, A.shape[1], s), A)


def transform_dev(ft, torch, P, fwd, tr, A):
    n, m = A.shape
    return run_dev(ft, torch, lambda p, s: ft.execute_dev(P, fwd, tr, p, n, m, s), A)


class _Plan(C.Structure):
    # the public ft_harmonic_plan (include/ft_b200.h)
    _fields_ = [("RP", C.c_void_p), ("MP", C.c_void_p), ("B", C.c_void_p),
                ("P", C.POINTER(C.POINTER(C.c_double))), ("Pinv", C.POINTER(C.POINTER(C.c_double))),
                ("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double),
                ("delta", C.c_double), ("rho", C.c_double), ("NRP", C.c_int), ("NMP", C.c_int), ("NP", C.c_int)]


def host_connection(P, n):
    p = C.cast(C.c_void_p(P.ptr), C.POINTER(_Plan)).contents
    get = lambda q: np.ctypeslib.as_array(q, shape=(n * n,)).reshape(n, n, order="F").copy()
    return p.NP, [get(p.P[i]) for i in range(p.NP)], [get(p.Pinv[i]) for i in range(p.NP)]


@pytest.mark.parametrize("n,M", [(1, 1), (2, 2), (3, 3), (8, 8), (33, 33), (100, 100), (257, 257), (40, 3), (40, 57)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_rotations_bit_exact(env, n, M, beta):
    ft, torch, O = env
    A = np.asfortranarray(np.random.default_rng(n * 100 + M).uniform(-1, 1, (n, M)))
    RP = ft.plan_rotrectdisk(n, beta)
    Po = O.plan("rect", n, beta=beta, rotations_only=True)
    for hi2lo in (True, False):
        want = A.copy(order="F")
        (O.hi2lo if hi2lo else O.lo2hi)(Po, want)
        got = rot_dev(ft, torch, RP, hi2lo, A)
        assert np.array_equal(got, want), (n, M, hi2lo, rel2(got, want))
    O.destroy(Po)
    RP.close()


@pytest.mark.parametrize("cfg", [0, 2, 3, 4, 5, 8, 10, 11, 12, 13, 16, 19])
def test_every_launch_shape_bit_exact(env, cfg):
    """Forced launch shapes (and the pass pipeline, cfg + 8) give the oracle's bits."""
    ft, torch, O = env
    n, beta = 700, 0.5
    A = ft.rectdiskrand(n, 3)
    RP = ft.plan_rotrectdisk(n, beta)
    Po = O.plan("rect", n, beta=beta, rotations_only=True)
    try:
        ft.set_rotation_config(cfg)
        for hi2lo in (True, False):
            want = A.copy(order="F")
            (O.hi2lo if hi2lo else O.lo2hi)(Po, want)
            assert np.array_equal(rot_dev(ft, torch, RP, hi2lo, A), want), (cfg, hi2lo)
    finally:
        ft.set_rotation_config(-1)
        O.destroy(Po)
        RP.close()


@pytest.mark.parametrize("n", [1, 2, 8, 33, 128])
@pytest.mark.parametrize("beta", BETAS)
def test_transforms_vs_oracle(env, n, beta):
    """Within 1e-14, or within twice the oracle's own distance from the compiled reference
    where the transform amplifies rounding beyond that (beta = 3/2, rectdisk2cheb 'N' at
    n = 128: 1.8e-14 between the oracle and the reference)."""
    ft, torch, O = env
    from oracle.bind import Reference
    R = Reference() if Reference.available() else None
    A = ft.rectdiskrand(n, 9)
    P = ft.plan_rectdisk2cheb(n, beta)
    Po = O.plan("rect", n, beta=beta)
    Pr = R.plan("rect", n, beta=beta) if R else None
    for fwd in (True, False):
        for tr in "NT":
            want = A.copy(order="F")
            O.execute(Po, fwd, tr, want)
            tol = 1e-14
            if R:
                ref = A.copy(order="F")
                R.execute("rect", Pr, fwd, tr, ref)
                tol = max(tol, 2 * rel2(want, ref))
            got = transform_dev(ft, torch, P, fwd, tr, A)
            assert rel2(got, want) <= tol, (n, beta, fwd, tr, rel2(got, want), tol)
    if R:
        R.destroy(Pr)
    O.destroy(Po)
    P.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_vs_golden(env, path):
    ft, torch, O = env
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n = A.shape[0]
    beta = float(z["beta"])
    P = ft.plan_rectdisk2cheb(n, beta)
    NP, Ps, Pinvs = host_connection(P, n)
    assert NP == 3
    for i in range(3):
        assert np.array_equal(Ps[i], z[f"P{i}"]) and np.array_equal(Pinvs[i], z[f"Pinv{i}"]), i
    for fwd in (True, False):
        for tr in "NT":
            got = transform_dev(ft, torch, P, fwd, tr, A)
            assert rel2(got, z[("fwd" if fwd else "bwd") + "_" + tr]) <= 1e-14, (fwd, tr)
    P.close()
    RP = ft.plan_rotrectdisk(n, beta)
    for d in ("hi2lo", "lo2hi"):
        got = rot_dev(ft, torch, RP, d == "hi2lo", A)
        assert rel2(got, z["rot_" + d]) <= 1e-15, d
    RP.close()


@pytest.mark.parametrize("n", [64, 256, 1024])
def test_reference_round_trips(env, n):
    """test/test_drivers.c:1179-1200 and 1230-1252 on this library."""
    ft, torch, O = env
    A = ft.rectdiskrand(n, 5)
    st = torch.cuda.current_stream().cuda_stream
    for beta in (0.0, 0.5):
        RP = ft.plan_rotrectdisk(n, beta)
        t = torch.from_numpy(A.ravel(order="F").copy()).cuda()
        ft.rotations_dev(RP, True, t.data_ptr(), n, st)
        ft.rotations_dev(RP, False, t.data_ptr(), n, st)
        torch.cuda.synchronize()
        B = t.cpu().numpy().reshape((n, n), order="F")
        assert rel2(B, A) <= 4 * np.sqrt(n) * EPS
        RP.close()
        P = ft.plan_rectdisk2cheb(n, beta)
        t = torch.from_numpy(A.ravel(order="F").copy()).cuda()
        for tr in "NT":
            ft.execute_dev(P, True, tr, t.data_ptr(), n, n, st)
            ft.execute_dev(P, False, tr, t.data_ptr(), n, n, st)
        torch.cuda.synchronize()
        B = t.cpu().numpy().reshape((n, n), order="F")
        P.close()
        e2, einf = rel2(B, A), np.abs(B - A).max() / np.abs(A).max()
        if beta == 0.0:
            assert e2 <= 4 * np.sqrt(n) * EPS and einf <= 2 * n * EPS, (e2, einf)
        else:
            Po = O.plan("rect", n, beta=beta)
            C2 = A.copy(order="F")
            for tr in "NT":
                O.execute(Po, True, tr, C2)
                O.execute(Po, False, tr, C2)
            O.destroy(Po)
            assert e2 <= 2 * rel2(C2, A) and einf <= 2 * np.abs(C2 - A).max() / np.abs(A).max(), (e2, einf)


def test_host_entry_points(env):
    ft, torch, O = env
    n, beta = 45, 0.5
    A = ft.rectdiskrand(n, 17)
    P = ft.plan_rectdisk2cheb(n, beta)
    for fwd in (True, False):
        for tr in "NT":
            H = A.copy(order="F")
            (ft.execute_rectdisk2cheb if fwd else ft.execute_cheb2rectdisk)(tr, P, H)
            assert np.array_equal(H, transform_dev(ft, torch, P, fwd, tr, A)), (fwd, tr)
    P.close()
    RP = ft.plan_rotrectdisk(n, beta)
    for hi2lo in (True, False):
        H = A.copy(order="F")
        (ft.execute_rectdisk_hi2lo if hi2lo else ft.execute_rectdisk_lo2hi)(RP, H)
        assert np.array_equal(H, rot_dev(ft, torch, RP, hi2lo, A))
    RP.close()


def test_bad_arguments(env):
    ft, torch, O = env
    P = ft.plan_rectdisk2cheb(8, 0.0)
    A = ft.rectdiskrand(8, 1)
    with pytest.raises(ft.FTB200Error):
        ft.execute_rectdisk2cheb("X", P, A)
    with pytest.raises(ft.FTB200Error):
        ft.execute_rectdisk2cheb("N", P, np.asfortranarray(A[:, :7]))   # M != N
    with pytest.raises(ft.FTB200Error):
        ft.execute_rectdisk2cheb("N", P, np.asfortranarray(A[:7, :7]))  # N != n
    P.close()
