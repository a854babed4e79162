"""Spin-weighted spherical harmonics on the GPU (ft_plan_rotspinsphere,
ft_execute_spinsph_hi2lo / lo2hi, ft_plan_spinsph2fourier, ft_execute_spinsph2fourier /
fourier2spinsph: src/rotations.c:431-478, src/drivers.c:645-695, 1259-1361), through the
C ABI.

Against the oracle (oracle/ft_oracle.c, pinned to the compiled reference in
tests/test_oracle_spin.py) in its fused form: the rotation stage bit for bit (the GPU
kernels apply each rotation as the oracle's fused form does, in the same order per
element), the transforms within 1e-14 relative 2-norm; against the reference's golden
fixtures within 1e-14 (transforms) and 1e-15 (rotations).  The reference's own tests
(test/test_drivers.c:1479-1500, 1649-1671): hi2lo then lo2hi, and spinsph2fourier then
fourier2spinsph in 'N' then in 'T', return the input within 4 sqrt(N) eps (2-norm) and
2N eps (max norm)."""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "spin_*.npz")))
SPINS = [-4, -3, -2, -1, 0, 1, 2, 3, 4]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


def to_dev(torch, A):
    """complex128 N x M (Fortran) -> device tensor of 2 N M interleaved doubles."""
    return torch.from_numpy(np.asfortranarray(A).ravel(order="F").view(np.float64).copy()).cuda()


def from_dev(t, n, m):
    return t.cpu().numpy().view(np.complex128).reshape((n, m), order="F")


def run_rot(ft, torch, SRP, hi2lo, A):
    n, m = A.shape
    t = to_dev(torch, A)
    ft.spin_rotations_dev(SRP, hi2lo, t.data_ptr(), m, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return from_dev(t, n, m)


def run_spin(ft, torch, P, fwd, tr, A):
    n, m = A.shape
    t = to_dev(torch, A)
    ft.execute_spin_dev(P, fwd, tr, t.data_ptr(), n, m, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return from_dev(t, n, m)


@pytest.mark.parametrize("n", [1, 2, 3, 8, 33, 100, 257])
@pytest.mark.parametrize("s", SPINS)
def test_rotations_bit_exact(env, n, s):
    ft, torch, O = env
    A = ft.spinsphrand(n, s, 5)
    SRP = ft.plan_rotspinsphere(n, s)
    Po = O.spin_plan(n, s, False)
    for hi2lo in (True, False):
        want = A.copy(order="F")
        (O.spin_hi2lo if hi2lo else O.spin_lo2hi)(Po, want)
        got = run_rot(ft, torch, SRP, hi2lo, A)
        assert np.array_equal(got, want), (n, s, hi2lo, rel2(got, want))
    O.spin_destroy(Po)
    SRP.close()


@pytest.mark.parametrize("n", [1, 2, 8, 33, 128])
@pytest.mark.parametrize("s", SPINS)
def test_transforms_vs_oracle(env, n, s):
    ft, torch, O = env
    A = ft.spinsphrand(n, s, 9)
    P = ft.plan_spinsph2fourier(n, s)
    Po = O.spin_plan(n, s, True)
    for fwd in (True, False):
        for tr in "NT":
            want = A.copy(order="F")
            O.spin_execute(Po, fwd, tr, want)
            got = run_spin(ft, torch, P, fwd, tr, A)
            assert rel2(got, want) <= 1e-14, (n, s, fwd, tr, rel2(got, want))
    O.spin_destroy(Po)
    P.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_vs_golden(env, path):
    ft, torch, O = env
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n, M = A.shape
    s = int(z["s"])
    P = ft.plan_spinsph2fourier(n, s)
    for fwd in (True, False):
        for tr in "NT":
            got = run_spin(ft, torch, P, fwd, tr, A)
            assert rel2(got, z[("fwd" if fwd else "bwd") + "_" + tr]) <= 1e-14, (fwd, tr)
    SRP = ft.plan_rotspinsphere(n, s)
    for d in ("hi2lo", "lo2hi"):
        got = run_rot(ft, torch, SRP, d == "hi2lo", A)
        assert rel2(got, z["rot_" + d]) <= 1e-15, d
    SRP.close()
    P.close()


@pytest.mark.parametrize("n", [64, 256, 1024])
@pytest.mark.parametrize("s", [-3, 1, 4])
def test_reference_round_trips(env, n, s):
    """test/test_drivers.c:1479-1500 and 1649-1671 on this library."""
    ft, torch, O = env
    M = 2 * n - 1
    A = ft.spinsphrand(n, s, 3)
    st = torch.cuda.current_stream().cuda_stream
    SRP = ft.plan_rotspinsphere(n, s)
    t = to_dev(torch, A)
    ft.spin_rotations_dev(SRP, True, t.data_ptr(), M, st)
    ft.spin_rotations_dev(SRP, False, t.data_ptr(), M, st)
    torch.cuda.synchronize()
    B = from_dev(t, n, M)
    assert rel2(B, A) <= 4 * np.sqrt(n) * EPS
    assert np.abs(B - A).max() / np.abs(A).max() <= 2 * n * EPS
    SRP.close()
    P = ft.plan_spinsph2fourier(n, s)
    t = to_dev(torch, A)
    for tr in "NT":
        ft.execute_spin_dev(P, True, tr, t.data_ptr(), n, M, st)
        ft.execute_spin_dev(P, False, tr, t.data_ptr(), n, M, st)
    torch.cuda.synchronize()
    B = from_dev(t, n, M)
    assert rel2(B, A) <= 4 * np.sqrt(n) * EPS
    assert np.abs(B - A).max() / np.abs(A).max() <= 2 * n * EPS
    P.close()


def test_large_rotations_vs_oracle(env):
    """Degree 2047 with s = 2: the rotation stage bit for bit (many tasks, full sweeps)."""
    ft, torch, O = env
    n, s = 2048, 2
    A = ft.spinsphrand(n, s, 21)
    SRP = ft.plan_rotspinsphere(n, s)
    Po = O.spin_plan(n, s, False)
    for hi2lo in (True, False):
        want = A.copy(order="F")
        (O.spin_hi2lo if hi2lo else O.spin_lo2hi)(Po, want)
        got = run_rot(ft, torch, SRP, hi2lo, A)
        assert np.array_equal(got, want), hi2lo
    O.spin_destroy(Po)
    SRP.close()


def test_host_entry_points(env):
    ft, torch, O = env
    n, s = 40, -2
    A = ft.spinsphrand(n, s, 17)
    P = ft.plan_spinsph2fourier(n, s)
    for fwd in (True, False):
        for tr in "NT":
            H = A.copy(order="F")
            (ft.execute_spinsph2fourier if fwd else ft.execute_fourier2spinsph)(tr, P, H)
            assert np.array_equal(H, run_spin(ft, torch, P, fwd, tr, A)), (fwd, tr)
    SRP = ft.plan_rotspinsphere(n, s)
    for hi2lo in (True, False):
        H = A.copy(order="F")
        (ft.execute_spinsph_hi2lo if hi2lo else ft.execute_spinsph_lo2hi)(SRP, H)
        assert np.array_equal(H, run_rot(ft, torch, SRP, hi2lo, A))
    SRP.close()
    P.close()


def test_bad_arguments(env):
    ft, torch, O = env
    P = ft.plan_spinsph2fourier(8, 1)
    A = ft.spinsphrand(8, 1, 1)
    with pytest.raises(ft.FTB200Error):
        ft.execute_spinsph2fourier("X", P, A)
    with pytest.raises(ft.FTB200Error):
        ft.execute_spinsph2fourier("N", P, np.asfortranarray(A[:, :14]))   # even M
    with pytest.raises(ft.FTB200Error):
        ft.execute_spinsph2fourier("N", P, np.asfortranarray(A[:7, :]))    # N != n
    P.close()
