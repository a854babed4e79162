"""Annulus harmonics on the GPU (ft_plan_rotannulus, ft_plan_ann2cxf, ft_execute_ann2cxf /
cxf2ann: src/rotations.c:192-268, src/drivers.c:1023-1121), through the C ABI.

Against the oracle (oracle/ft_oracle.c, pinned to the compiled reference in
tests/test_oracle_ann.py) in its fused form: the plan's host table bit for bit (both restate the
recurrences without contraction), the rotation stage bit for bit, the transforms within 1e-14
relative 2-norm.  Against the reference's golden fixtures: the table within 2n ulps, the
transforms within 1e-14.  The reference's own round trips (test/test_drivers.c:985-1020,
1128-1150) with its bounds."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ann_*.npz")))
CASES = [(0.0, 0.0, float(np.sqrt(1 / 3))), (0.5, -0.25, 0.4), (0.0, 0.0, 0.0)]


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


def host_table(RPptr, n):
    """s, c of an ft_rotation_plan (its leading members, as in the reference's struct)."""
    p = C.cast(C.c_void_p(RPptr), C.POINTER(C.POINTER(C.c_double)))
    return (np.ctypeslib.as_array(p[0], shape=(n * n,)).copy(), np.ctypeslib.as_array(p[1], shape=(n * n,)).copy())


@pytest.mark.parametrize("n", [1, 2, 5, 16, 33, 100, 257])
@pytest.mark.parametrize("case", CASES, ids=["rho_test", "generic", "rho0"])
def test_table_and_rotations_bit_exact(env, n, case):
    ft, torch, O = env
    a, b, rho = case
    RP = ft.plan_rotannulus(n, a, b, 0.0, rho)
    Po = O.ann_plan(n, a, b, rho, connections=False)
    s, c = host_table(RP.ptr, n)
    so, co = O.ann_table(Po)
    assert np.array_equal(s, so) and np.array_equal(c, co)
    M = 4 * n - 3
    A = np.asfortranarray(np.random.default_rng(n).uniform(-1, 1, (n, M)))
    for hi2lo in (True, False):
        want = A.copy(order="F")
        (O.ann_hi2lo if hi2lo else O.ann_lo2hi)(Po, want)
        got = on_dev(torch, lambda p, st: ft.rotations_dev(RP, hi2lo, p, M, st), A)
        assert np.array_equal(got, want), (n, hi2lo, rel2(got, want))
    O.ann_destroy(Po)
    RP.close()


@pytest.mark.parametrize("n", [1, 2, 8, 33, 128])
@pytest.mark.parametrize("case", CASES, ids=["rho_test", "generic", "rho0"])
def test_transforms_vs_oracle(env, n, case):
    ft, torch, O = env
    a, b, rho = case
    A = ft.diskrand(n, 9)
    P = ft.plan_ann2cxf(n, a, b, 0.0, rho)
    Po = O.ann_plan(n, a, b, rho)
    M = A.shape[1]
    for fwd in (True, False):
        for tr in "NT":
            want = A.copy(order="F")
            O.ann_execute(Po, fwd, tr, want)
            got = on_dev(torch, lambda p, st: ft.execute_dev(P, fwd, tr, p, n, M, st), A)
            assert rel2(got, want) <= 1e-14, (n, case, fwd, tr, rel2(got, want))
    O.ann_destroy(Po)
    P.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_vs_golden(env, path):
    ft, torch, O = env
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n, M = A.shape
    a, b, rho = (float(x) for x in z["params"])
    P = ft.plan_ann2cxf(n, a, b, 0.0, rho)
    rp = C.cast(C.c_void_p(P.ptr), C.POINTER(C.POINTER(C.c_void_p))).contents[0]   # P->RP[0]
    s, c = host_table(rp, n)
    assert np.abs(s - z["s"]).max() <= 2 * n * EPS and np.abs(c - z["c"]).max() <= 2 * n * EPS
    for fwd in (True, False):
        for tr in "NT":
            got = on_dev(torch, lambda p, st: ft.execute_dev(P, fwd, tr, p, n, M, st), A)
            assert rel2(got, z[("fwd" if fwd else "bwd") + "_" + tr]) <= 1e-14, (fwd, tr)
    P.close()


@pytest.mark.parametrize("n", [64, 256, 1024])
def test_reference_round_trips(env, n):
    """test/test_drivers.c:985-1020 and 1128-1150 on this library, with their bounds."""
    ft, torch, O = env
    A = ft.diskrand(n, 5)
    M = A.shape[1]
    einf = lambda B: np.abs(B - A).max() / np.abs(A).max()
    for rho in (0.0, float(np.sqrt(1 / 3))):
        RP = ft.plan_rotannulus(n, 0.0, 0.0, 0.0, rho)
        B = on_dev(torch, lambda p, st: (ft.rotations_dev(RP, True, p, M, st), ft.rotations_dev(RP, False, p, M, st)), A)
        assert rel2(B, A) <= 6 * np.sqrt(n) * EPS and einf(B) <= 5 * n * EPS, rho
        RP.close()
    P = ft.plan_ann2cxf(n, 0.0, 0.0, 0.0, float(np.sqrt(1 / 3)))

    def trip(p, st):
        for tr in "NT":
            ft.execute_dev(P, True, tr, p, n, M, st)
            ft.execute_dev(P, False, tr, p, n, M, st)
    B = on_dev(torch, trip, A)
    assert rel2(B, A) <= 12 * np.sqrt(n) * EPS and einf(B) <= 6 * n * EPS
    P.close()


def test_host_entry_points(env):
    ft, torch, O = env
    n = 30
    A = ft.diskrand(n, 17)
    M = A.shape[1]
    P = ft.plan_ann2cxf(n, 0.5, -0.25, 0.0, 0.4)
    for fwd in (True, False):
        for tr in "NT":
            H = A.copy(order="F")
            (ft.execute_ann2cxf if fwd else ft.execute_cxf2ann)(tr, P, H)
            assert np.array_equal(H, on_dev(torch, lambda p, st: ft.execute_dev(P, fwd, tr, p, n, M, st), A)), (fwd, tr)
    P.close()


def test_bad_arguments(env):
    ft, torch, O = env
    with pytest.raises(ft.FTB200Error):
        ft.plan_ann2cxf(8, 0.0, 0.0, 0.5, 0.3)    # gamma != 0: not implemented in the reference either
    P = ft.plan_ann2cxf(8, 0.0, 0.0, 0.0, 0.3)
    A = ft.diskrand(8, 1)
    with pytest.raises(ft.FTB200Error):
        ft.execute_ann2cxf("X", P, A)
    with pytest.raises(ft.FTB200Error):
        ft.execute_ann2cxf("N", P, np.asfortranarray(A[:, :28]))   # even M
    P.close()
