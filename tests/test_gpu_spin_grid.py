"""Spin-weighted sphere grid synthesis and analysis on the GPU (ft_plan_spinsph_synthesis ..
ft_execute_spinsph_analysis, src/fftw.c:743-960), through the C ABI.

Against the oracle (oracle/grid.py, pinned in tests/test_oracle_grid.py): both sequences, 'N'
and 'C', every plan with every sequence, spins of both parities, within 1e-14 relative 2-norm;
other TRANS values leave the matrix untouched, as the reference's.  The reference's own accuracy
test (test/test_fftw.c:481-516) with every stage on the GPU: spinsph2fourier, synthesis,
analysis, fourier2spinsph in 'N' then 'T' return the input within 4 sqrt(N) eps and 2N eps.  The host sequence and index maps are also
restated on the CPU in tests/test_device_schedules.py."""
import numpy as np
import pytest

from conftest import EPS, rel2

pytestmark = pytest.mark.gpu

OPS = ["spinsph_synthesis", "spinsph_analysis"]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    torch.cuda.set_device(0)
    return ft, torch


def run_dev(ft, torch, P, analysis, tr, X):
    n, m = X.shape
    t = torch.from_numpy(np.asfortranarray(X).ravel(order="F").copy()).cuda()
    ft.execute_spinsph_grid_dev(P, analysis, tr, t.data_ptr(), n, m, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return t.cpu().numpy().reshape((n, m), order="F")


@pytest.mark.parametrize("N,M", [(1, 1), (2, 3), (3, 5), (8, 15), (17, 33), (64, 127), (33, 21), (256, 511)])
@pytest.mark.parametrize("s", [0, 1, -2, 3])
def test_spin_grid_vs_oracle(env, N, M, s):
    ft, torch = env
    from oracle import grid as G
    rng = np.random.default_rng(N * 1000 + M + s)
    X = np.asfortranarray(rng.uniform(-1, 1, (N, M)) + 1j * rng.uniform(-1, 1, (N, M)))
    plans = {k: getattr(ft, "plan_" + k)(N, s, M) for k in OPS}
    try:
        for op in OPS:
            for tr in "NCT":
                for plan in OPS:   # every plan with every sequence (the reference's test crosses them)
                    got = run_dev(ft, torch, plans[plan], op == "spinsph_analysis", tr, X)
                    want = G.execute_spinsph(op, tr, plan, s, X)
                    assert rel2(got, want) <= 1e-14, (N, M, s, op, tr, plan, rel2(got, want))
    finally:
        for P in plans.values():
            P.close()


@pytest.mark.parametrize("N", [64, 128, 256])
@pytest.mark.parametrize("s", [-4, -1, 0, 2, 3])
def test_reference_round_trip_on_gpu(env, N, s):
    """test/test_fftw.c:481-516 on this library: every stage on the GPU."""
    ft, torch = env
    M = 2 * N - 1
    A = ft.spinsphrand(N, s, 5)
    SP = ft.plan_spinsph2fourier(N, s)
    US, UA = ft.plan_spinsph_synthesis(N, s), ft.plan_spinsph_analysis(N, s)
    st = torch.cuda.current_stream().cuda_stream
    t = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    p = t.data_ptr()
    ft.execute_spin_dev(SP, True, "N", p, N, M, st)
    ft.execute_spinsph_grid_dev(US, False, "N", p, N, M, st)
    ft.execute_spinsph_grid_dev(UA, True, "N", p, N, M, st)
    ft.execute_spin_dev(SP, False, "N", p, N, M, st)
    ft.execute_spin_dev(SP, True, "T", p, N, M, st)
    ft.execute_spinsph_grid_dev(UA, False, "T", p, N, M, st)   # a no-op, as in the reference
    ft.execute_spinsph_grid_dev(US, True, "T", p, N, M, st)
    ft.execute_spin_dev(SP, False, "T", p, N, M, st)
    torch.cuda.synchronize()
    B = t.cpu().numpy().reshape((N, M), order="F")
    for P in (SP, US, UA):
        P.close()
    assert rel2(B, A) <= 4 * np.sqrt(N) * EPS
    assert np.abs(B - A).max() / np.abs(A).max() <= 2 * N * EPS


def test_host_entry_points(env):
    ft, torch = env
    N, M, s = 20, 39, -3
    rng = np.random.default_rng(7)
    X = np.asfortranarray(rng.uniform(-1, 1, (N, M)) + 1j * rng.uniform(-1, 1, (N, M)))
    plans = {"spinsph_synthesis": ft.plan_spinsph_synthesis(N, s), "spinsph_analysis": ft.plan_spinsph_analysis(N, s)}
    try:
        assert plans["spinsph_synthesis"].s == s and plans["spinsph_analysis"].s == s
        for op in OPS:
            for tr in "NC":
                H = X.copy(order="F")
                getattr(ft, "execute_" + op)(tr, plans[op], H)
                assert np.array_equal(H, run_dev(ft, torch, plans[op], op == "spinsph_analysis", tr, X)), (op, tr)
    finally:
        for P in plans.values():
            P.close()


def test_bad_arguments(env):
    ft, torch = env
    with pytest.raises(ft.FTB200Error):
        ft.plan_spinsph_synthesis(8, 0, 14)   # even M
    P = ft.plan_spinsph_analysis(8, 1)
    X = np.zeros((8, 15), dtype=complex, order="F")
    with pytest.raises(ft.FTB200Error):
        ft.execute_spinsph_analysis("N", P, X, 7, 15)   # N != the plan's
    P.close()
