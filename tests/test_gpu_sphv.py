"""sph vector-field transforms (ft_execute_sphv2fourier / ft_execute_fourier2sphv,
src/drivers.c:867-899) on the GPU, through the C ABI: the sph plan, order m's
sweeps on the column pair (2m+1, 2m+2), P[0] and P[1] swapped in the four
column classes.  Bars as for the scalar transforms: relative 2-norm <= 1e-14
against the oracle and against the reference's golden outputs; round trips
within the reference's own tolerances (test/test_drivers.c:478-483: 4 sqrt(N)
eps in the 2-norm, 2N eps in the max norm)."""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2, relinf

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sph_*.npz")))


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


def run_dev(ft, torch, P, A, fwd, tr):
    n, M = A.shape
    t = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()
    ft.execute_sphv_dev(P, fwd, tr, t.data_ptr(), n, M, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return t.cpu().numpy().reshape((n, M), order="F")


@pytest.mark.parametrize("n", [3, 4, 8, 17, 65, 256])
def test_sphv_vs_oracle(env, n):
    ft, torch, O = env
    P = ft.plan_sph2fourier(n)
    PO = O.plan("sph", n)
    A = ft.sphrand(n, 11)
    for fwd in (True, False):
        for tr in "NT":
            got = run_dev(ft, torch, P, A, fwd, tr)
            ref = A.copy(order="F")
            O.execute_sphv(PO, fwd, tr, ref)
            assert rel2(got, ref) <= 1e-14, (n, fwd, tr, rel2(got, ref))
    O.destroy(PO)
    P.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_sphv_vs_reference_golden(env, path):
    ft, torch, O = env
    z = np.load(path)
    A = z["A"]
    n = A.shape[0]
    P = ft.plan_sph2fourier(n)
    for fwd in (True, False):
        for tr in "NT":
            got = run_dev(ft, torch, P, A, fwd, tr)
            ref = z["v_" + ("fwd" if fwd else "bwd") + "_" + tr]
            assert rel2(got, ref) <= 1e-14, (fwd, tr, rel2(got, ref))
    P.close()


@pytest.mark.parametrize("n", [64, 257, 1024])
def test_sphv_round_trip_reference_tolerance(env, n):
    """The reference's test: N forward then backward, T forward then backward."""
    ft, torch, O = env
    P = ft.plan_sph2fourier(n)
    A = ft.sphrand(n, 12)
    B = run_dev(ft, torch, P, A, True, "N")
    B = run_dev(ft, torch, P, B, False, "N")
    B = run_dev(ft, torch, P, B, True, "T")
    B = run_dev(ft, torch, P, B, False, "T")
    assert rel2(B, A) <= 4 * np.sqrt(n) * EPS
    assert relinf(B, A) <= 2 * n * EPS
    P.close()


def test_sphv_host_entry_points(env):
    """ft_execute_sphv2fourier / ft_execute_fourier2sphv on host arrays equal the device path."""
    ft, torch, O = env
    n = 40
    P = ft.plan_sph2fourier(n)
    A = ft.sphrand(n, 13)
    for fwd, f in ((True, ft.execute_sphv2fourier), (False, ft.execute_fourier2sphv)):
        for tr in "NT":
            H = A.copy(order="F")
            f(tr, P, H)
            assert np.array_equal(H, run_dev(ft, torch, P, A, fwd, tr))
    P.close()


def test_sphv_rejects_other_families(env):
    ft, torch, O = env
    P = ft.plan_disk2cxf(8, 0.0, 0.0)
    t = torch.zeros(8 * P.M, dtype=torch.float64, device="cuda")
    with pytest.raises(ft.FTB200Error):
        ft.execute_sphv_dev(P, True, "N", t.data_ptr(), 8, P.M)
    P.close()


@pytest.mark.parametrize("n", [1, 3, 4, 17, 65])
def test_sphv_rotation_entry_points_bit_exact(env, n):
    """ft_execute_sphv_hi2lo / lo2hi (src/drivers.c:168-276) against the oracle's column loops:
    order m on the columns 2m + 1 and 2m + 2, m = 2 .. M/2 - 1, the other columns untouched."""
    ft, torch, O = env
    M = 2 * n - 1
    RP = ft.plan_rotsphere(n)
    Po = O.plan("sph", n, rotations_only=True)
    A = np.asfortranarray(np.random.default_rng(n).uniform(-1, 1, (n, M)))
    for hi2lo in (True, False):
        want = A.copy(order="F")
        for m in range(2, M // 2):
            for c in (2 * m + 1, 2 * m + 2):
                want[:, c] = O.kernel(Po, hi2lo, m % 2, m, A[:, c].copy())
        got = A.copy(order="F")
        (ft.execute_sphv_hi2lo if hi2lo else ft.execute_sphv_lo2hi)(RP, got)
        assert np.array_equal(got, want), (n, hi2lo)
    O.destroy(Po)
    RP.close()
