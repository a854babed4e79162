"""Tetrahedral harmonics on the GPU (ft_plan_tet2cheb, ft_execute_tet2cheb / cheb2tet,
ft_execute_tet_hi2lo / lo2hi: src/drivers.c:26-54, 510-528, 1173-1257, src/rotations.c:297-321),
through the C ABI.

Against the oracle (oracle/ft_oracle.c, pinned to the compiled reference in
tests/test_oracle_tet.py) in its fused form: the rotation stage bit for bit (for every launch
shape of the triangle sweeps, and for L < n, M != L); the transforms within 1e-14, or within
four times the oracle's own fused-versus-unfused spread where the transform amplifies rounding
beyond that (the rotation stage is bit-identical; the multiplies sum in another order).
Against the reference's golden fixtures: the plan's connection matrices bit for bit, the
transforms within the same bar, the rotation stages within 2n ulps.  The reference's own
round-trip tests (test/test_drivers.c:1282-1304, 1418-1447) with its own bounds."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "tet_*.npz")))
PARAMS = [(0.0, 0.0, 0.0, 0.0), (-0.5, -0.5, -0.5, -0.5), (0.5, -0.25, 0.25, 1.0)]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


def on_dev(torch, fn, A):
    t = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()
    fn(t.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return t.cpu().numpy().reshape(A.shape, order="F")


def rot_dev(ft, torch, P, hi2lo, A):
    return on_dev(torch, lambda p, s: ft.tet_rotations_dev(P, hi2lo, p, A.shape[1], A.shape[2], s), A)


def transform_dev(ft, torch, P, fwd, tr, A):
    N, L, M = A.shape
    return on_dev(torch, lambda p, s: ft.execute_tet_dev(P, fwd, tr, p, N, L, M, s), A)


def sensitivity(O, Po, fwd, tr, A):
    a, b = A.copy(order="F"), A.copy(order="F")
    O.tet_execute(Po, fwd, tr, a)
    O.set_fused(False)
    O.tet_execute(Po, fwd, tr, b)
    O.set_fused(True)
    return rel2(a, b)


class _Plan(C.Structure):
    # the public ft_harmonic_plan (include/ft_b200.h)
    _fields_ = [("RP", C.c_void_p), ("MP", C.c_void_p), ("B", C.c_void_p),
                ("P", C.POINTER(C.POINTER(C.c_double))), ("Pinv", C.POINTER(C.POINTER(C.c_double))),
                ("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double),
                ("delta", C.c_double), ("rho", C.c_double), ("NRP", C.c_int), ("NMP", C.c_int), ("NP", C.c_int)]


@pytest.mark.parametrize("n,L,M", [(1, 1, 1), (2, 2, 2), (3, 3, 3), (8, 8, 8), (17, 17, 17), (64, 64, 64),
                                   (130, 130, 130), (40, 30, 50), (40, 40, 3)])
@pytest.mark.parametrize("params", PARAMS[::2])
def test_rotations_bit_exact(env, n, L, M, params):
    ft, torch, O = env
    A = np.asfortranarray(np.random.default_rng(n + 7 * L + 31 * M).uniform(-1, 1, (n, L, M)))
    P = ft.plan_tet2cheb(n, *params)
    Po = O.tet_plan(n, *params, connections=False)
    for hi2lo in (True, False):
        want = A.copy(order="F")
        (O.tet_hi2lo if hi2lo else O.tet_lo2hi)(Po, want)
        got = rot_dev(ft, torch, P, hi2lo, A)
        assert np.array_equal(got, want), (n, L, M, hi2lo, rel2(got, want))
    O.tet_destroy(Po)
    P.close()


@pytest.mark.parametrize("cfg", [0, 2, 3, 4, 5])
def test_every_launch_shape_bit_exact(env, cfg):
    ft, torch, O = env
    n = 96
    A = ft.tetrand(n, 3)
    P = ft.plan_tet2cheb(n, 0.0, 0.0, 0.0, 0.0)
    Po = O.tet_plan(n, 0.0, 0.0, 0.0, 0.0, connections=False)
    try:
        ft.set_rotation_config(cfg)
        for hi2lo in (True, False):
            want = A.copy(order="F")
            (O.tet_hi2lo if hi2lo else O.tet_lo2hi)(Po, want)
            assert np.array_equal(rot_dev(ft, torch, P, hi2lo, A), want), (cfg, hi2lo)
    finally:
        ft.set_rotation_config(-1)
        O.tet_destroy(Po)
        P.close()


@pytest.mark.parametrize("n", [1, 2, 8, 17, 32, 64])
@pytest.mark.parametrize("params", PARAMS)
def test_transforms_vs_oracle(env, n, params):
    ft, torch, O = env
    A = ft.tetrand(n, 9)
    P = ft.plan_tet2cheb(n, *params)
    Po = O.tet_plan(n, *params)
    for fwd in (True, False):
        for tr in "NT":
            want = A.copy(order="F")
            O.tet_execute(Po, fwd, tr, want)
            tol = max(1e-14, 4 * sensitivity(O, Po, fwd, tr, A))
            got = transform_dev(ft, torch, P, fwd, tr, A)
            assert rel2(got, want) <= tol, (n, params, fwd, tr, rel2(got, want), tol)
    O.tet_destroy(Po)
    P.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_vs_golden(env, path):
    ft, torch, O = env
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n = A.shape[0]
    params = tuple(float(x) for x in z["params"])
    P = ft.plan_tet2cheb(n, *params)
    p = C.cast(C.c_void_p(P.ptr), C.POINTER(_Plan)).contents
    assert p.NP == 3 and p.NRP == 2
    get = lambda q: np.ctypeslib.as_array(q, shape=(n * n,)).reshape(n, n, order="F")
    for i in range(3):
        assert np.array_equal(get(p.P[i]), z[f"P{i}"]) and np.array_equal(get(p.Pinv[i]), z[f"Pinv{i}"]), i
    Po = O.tet_plan(n, *params)
    for fwd in (True, False):
        for tr in "NT":
            got = transform_dev(ft, torch, P, fwd, tr, A)
            tol = max(1e-14, 4 * sensitivity(O, Po, fwd, tr, A))
            assert rel2(got, z[("fwd" if fwd else "bwd") + "_" + tr]) <= tol, (fwd, tr)
    for d in ("hi2lo", "lo2hi"):
        got = rot_dev(ft, torch, P, d == "hi2lo", A)
        assert np.abs(got - z["rot_" + d]).max() <= 2 * n * EPS, d
    O.tet_destroy(Po)
    P.close()


@pytest.mark.parametrize("n", [16, 33, 64, 128])
def test_reference_round_trips(env, n):
    """test/test_drivers.c:1282-1304 and 1418-1447 on this library, with their bounds."""
    ft, torch, O = env
    A = ft.tetrand(n, 5)
    P = ft.plan_tet2cheb(n, 0.0, 0.0, 0.0, 0.0)
    st = torch.cuda.current_stream().cuda_stream
    einf = lambda B: np.abs(B - A).max() / np.abs(A).max()
    t = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    ft.tet_rotations_dev(P, True, t.data_ptr(), n, n, st)
    ft.tet_rotations_dev(P, False, t.data_ptr(), n, n, st)
    torch.cuda.synchronize()
    B = t.cpu().numpy().reshape(A.shape, order="F")
    assert rel2(B, A) <= 8 * n * EPS and einf(B) <= 4 * n * n * EPS
    t = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    ft.execute_tet_dev(P, True, "N", t.data_ptr(), n, n, n, st)
    ft.execute_tet_dev(P, False, "N", t.data_ptr(), n, n, n, st)
    torch.cuda.synchronize()
    B = t.cpu().numpy().reshape(A.shape, order="F")
    assert rel2(B, A) <= 8 * n * EPS and einf(B) <= 4 * n * n * EPS
    ft.execute_tet_dev(P, True, "T", t.data_ptr(), n, n, n, st)
    ft.execute_tet_dev(P, False, "T", t.data_ptr(), n, n, n, st)
    torch.cuda.synchronize()
    B = t.cpu().numpy().reshape(A.shape, order="F")
    assert rel2(B, A) <= 64 * n * n * EPS and einf(B) <= 32 * n ** 3 * EPS
    P.close()


def test_host_entry_points(env):
    ft, torch, O = env
    n = 21
    A = ft.tetrand(n, 17)
    P = ft.plan_tet2cheb(n, 0.5, -0.25, 0.25, 1.0)
    for fwd in (True, False):
        for tr in "NT":
            H = A.copy(order="F")
            (ft.execute_tet2cheb if fwd else ft.execute_cheb2tet)(tr, P, H)
            assert np.array_equal(H, transform_dev(ft, torch, P, fwd, tr, A)), (fwd, tr)
    for hi2lo in (True, False):
        H = A.copy(order="F")
        (ft.execute_tet_hi2lo if hi2lo else ft.execute_tet_lo2hi)(P, H)
        assert np.array_equal(H, rot_dev(ft, torch, P, hi2lo, A)), hi2lo
    P.close()


def test_bad_arguments(env):
    ft, torch, O = env
    P = ft.plan_tet2cheb(6, 0.0, 0.0, 0.0, 0.0)
    A = ft.tetrand(6, 1)
    with pytest.raises(ft.FTB200Error):
        ft.execute_tet2cheb("X", P, A)
    with pytest.raises(ft.FTB200Error):
        ft.execute_tet2cheb("N", P, np.asfortranarray(A[:, :5, :]))   # L != N
    with pytest.raises(ft.FTB200Error):
        ft.execute_tet2cheb("N", P, np.asfortranarray(A[:5, :5, :5]))  # N != n
    P.close()
