"""GPU parity of the CUDA library against the oracle restatement and the
reference's golden outputs, through the C ABI.

Bars:
  * rotation stage: bit-exact against the oracle's fused arithmetic (the
    kernels perform the same IEEE operations on every element in the same
    order);
  * full transforms: relative 2-norm <= 1e-14 against the oracle and against
    the reference's outputs (the triangular multiplies sum in another order);
  * round trips: the reference's own tolerances (test/test_drivers.c).
"""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2, relinf

pytestmark = pytest.mark.gpu

# the sph / tri / disk fixtures (the spin and Dunkl-Xu fixtures have their own tests)
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if os.path.basename(p).split("_")[0] in ("sph", "tri", "disk"))
TOL = {"sph": (4, 2), "tri": (32, 8), "disk": (8, 4)}
FAMILIES = [("sph", ()), ("tri", (0.0, 0.0, 0.0)), ("tri", (-0.5, -0.5, -0.5)), ("tri", (0.5, 1.0, -0.25)),
            ("disk", (0.0, 0.0)), ("disk", (0.5, -0.25))]


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
    return torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()


def to_host(t, n, M):
    return t.cpu().numpy().reshape((n, M), order="F")


def plan(ft, kind, n, params):
    return {"sph": ft.plan_sph2fourier, "tri": ft.plan_tri2cheb, "disk": ft.plan_disk2cxf}[kind](n, *params)


def rot_plan(ft, kind, n, params):
    return {"sph": ft.plan_rotsphere, "tri": ft.plan_rottriangle, "disk": ft.plan_rotdisk}[kind](n, *params)


def stream(torch):
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("kind,params", FAMILIES)
@pytest.mark.parametrize("n", [2, 3, 5, 16, 33, 64, 127, 256])
def test_rotation_stage_bitexact(env, kind, params, n):
    ft, torch, O = env
    A = ft.rand_layout(kind, n, 5 + n)
    M = A.shape[1]
    RP = rot_plan(ft, kind, n, params)
    PO = O.plan(kind, n, *params, rotations_only=True)
    for hi2lo in (True, False):
        d = to_dev(torch, A)
        ft.rotations_dev(RP, hi2lo, d.data_ptr(), M, stream(torch))
        got = to_host(d, n, M)
        ref = A.copy(order="F")
        (O.hi2lo if hi2lo else O.lo2hi)(PO, ref)
        assert np.array_equal(got, ref), (hi2lo, rel2(got, ref))
    O.destroy(PO)
    RP.close()


@pytest.mark.parametrize("kind,params", FAMILIES)
@pytest.mark.parametrize("n", [1, 2, 3, 8, 31, 64, 129])
def test_transforms_vs_oracle(env, kind, params, n):
    ft, torch, O = env
    if kind == "tri" and n < 2:
        pytest.skip("tri needs n >= 2 for a nontrivial transform")
    A = ft.rand_layout(kind, n, 100 + n)
    M = A.shape[1]
    P = plan(ft, kind, n, params)
    PO = O.plan(kind, n, *params)
    for fwd in (True, False):
        for tr in "NT":
            d = to_dev(torch, A)
            ft.execute_dev(P, fwd, tr, d.data_ptr(), n, M, stream(torch))
            got = to_host(d, n, M)
            ref = A.copy(order="F")
            O.execute(PO, fwd, tr, ref)
            assert rel2(got, ref) <= 1e-14, (fwd, tr, rel2(got, ref))
    O.destroy(PO)
    P.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_transforms_vs_reference_golden(env, path):
    ft, torch, O = env
    z = np.load(path)
    kind = os.path.basename(path).split("_")[0]
    A = z["A"]
    n, M = A.shape
    P = plan(ft, kind, n, tuple(z["params"]))
    for fwd in (True, False):
        for tr in "NT":
            d = to_dev(torch, A)
            ft.execute_dev(P, fwd, tr, d.data_ptr(), n, M, stream(torch))
            got = to_host(d, n, M)
            ref = z[("fwd" if fwd else "bwd") + "_" + tr]
            assert rel2(got, ref) <= 1e-14, (fwd, tr, rel2(got, ref))
    # the plan's host connection matrices are the reference's, bit for bit
    import ctypes as C
    from oracle.bind import _RefHarmonicPlan
    hp = C.cast(C.c_void_p(P.ptr), C.POINTER(_RefHarmonicPlan)).contents
    for i, name in enumerate(("P0", "P1")):
        got = np.ctypeslib.as_array(hp.P[i], shape=(n * n,)).reshape(n, n, order="F")
        assert np.array_equal(np.triu(got), np.triu(z[name]))
    for i, name in enumerate(("Pinv0", "Pinv1")):
        got = np.ctypeslib.as_array(hp.Pinv[i], shape=(n * n,)).reshape(n, n, order="F")
        assert np.array_equal(np.triu(got), np.triu(z[name]))
    P.close()


@pytest.mark.parametrize("kind,params", FAMILIES)
@pytest.mark.parametrize("n", [64, 255, 256])
def test_round_trip_reference_tolerance(env, kind, params, n):
    """test/test_drivers.c sequence: N forward, N backward, T forward, T backward.

    The bound is the reference's own tolerance (4 sqrt(N) eps etc.), or twice the
    round-trip error of the reference algorithm itself (the oracle) where that is
    larger: some Jacobi parameters are ill-conditioned in the reference too."""
    ft, torch, O = env
    A = ft.rand_layout(kind, n, 7)
    M = A.shape[1]
    P = plan(ft, kind, n, params)
    d = to_dev(torch, A)
    seq = ((True, "N"), (False, "N"), (True, "T"), (False, "T"))
    for fwd, tr in seq:
        ft.execute_dev(P, fwd, tr, d.data_ptr(), n, M, stream(torch))
    got = to_host(d, n, M)
    ref = A.copy(order="F")
    PO = O.plan(kind, n, *params)
    for fwd, tr in seq:
        O.execute(PO, fwd, tr, ref)
    O.destroy(PO)
    c2, ci = TOL[kind]
    assert rel2(got, A) < max(c2 * np.sqrt(n) * EPS, 2 * rel2(ref, A))
    assert relinf(got, A) < max(ci * n * EPS, 2 * relinf(ref, A))
    P.close()


@pytest.mark.parametrize("kind,params", [("sph", ()), ("tri", (0.0, 0.0, 0.0)), ("disk", (0.0, 0.0))])
def test_host_dropin_entry_points(env, kind, params):
    ft, torch, O = env
    n = 40
    A = ft.rand_layout(kind, n, 1)
    P = plan(ft, kind, n, params)
    PO = O.plan(kind, n, *params)
    fwd_fn = {"sph": ft.execute_sph2fourier, "tri": ft.execute_tri2cheb, "disk": ft.execute_disk2cxf}[kind]
    bwd_fn = {"sph": ft.execute_fourier2sph, "tri": ft.execute_cheb2tri, "disk": ft.execute_cxf2disk}[kind]
    for fn, fwd in ((fwd_fn, True), (bwd_fn, False)):
        for tr in "NT":
            B = A.copy(order="F")
            fn(tr, P, B)
            ref = A.copy(order="F")
            O.execute(PO, fwd, tr, ref)
            assert rel2(B, ref) <= 1e-14
    O.destroy(PO)
    P.close()


def test_host_rotation_entry_points(env):
    ft, torch, O = env
    for kind, params in (("sph", ()), ("tri", (0.0, 0.0, 0.0)), ("disk", (0.0, 0.0))):
        n = 37
        A = ft.rand_layout(kind, n, 2)
        RP = rot_plan(ft, kind, n, params)
        PO = O.plan(kind, n, *params, rotations_only=True)
        for d in ("hi2lo", "lo2hi"):
            B = A.copy(order="F")
            getattr(ft, f"execute_{kind}_{d}")(RP, B)
            ref = A.copy(order="F")
            (O.hi2lo if d == "hi2lo" else O.lo2hi)(PO, ref)
            assert np.array_equal(B, ref)
        O.destroy(PO)
        RP.close()


def test_errors(env):
    ft, torch, O = env
    P = ft.plan_sph2fourier(16)
    A = ft.sphrand(16, 3)
    B = A.copy(order="F")
    with pytest.raises(ft.FTB200Error) as e:
        ft.execute_sph2fourier("X", P, B)
    assert e.value.status == 1 and np.array_equal(A, B)
    with pytest.raises(ft.FTB200Error):
        ft.execute_sph2fourier("N", P, np.zeros((15, 29), order="F"))
    with pytest.raises(ft.FTB200Error):
        ft.plan_sph2fourier(0)
    T = ft.plan_tri2cheb(8, 0.0, 0.0, 0.0)
    with pytest.raises(ft.FTB200Error):
        ft.execute_tri2cheb("N", T, np.zeros((8, 7), order="F"))
    T.close()
    P.close()


@pytest.mark.parametrize("kind,params,n", [("sph", (), 1024), ("sph", (), 2048), ("tri", (0.0, 0.0, 0.0), 2048),
                                           ("disk", (0.0, 0.0), 1024)])
def test_large_properties(env, kind, params, n):
    """At full sizes: round trip, orthogonality of the rotation stage, linearity."""
    ft, torch, O = env
    A = ft.rand_layout(kind, n, 42)
    M = A.shape[1]
    P = plan(ft, kind, n, params)
    d = to_dev(torch, A)
    ft.execute_dev(P, True, "N", d.data_ptr(), n, M, stream(torch))
    F1 = to_host(d, n, M)
    ft.execute_dev(P, False, "N", d.data_ptr(), n, M, stream(torch))
    back = to_host(d, n, M)
    c2, _ = TOL[kind]
    assert rel2(back, A) < c2 * np.sqrt(n) * EPS
    # linearity: T(2A) = 2 T(A) exactly (scaling by 2 is exact), T(A + A') ~ T(A) + T(A')
    d2 = to_dev(torch, 2.0 * A)
    ft.execute_dev(P, True, "N", d2.data_ptr(), n, M, stream(torch))
    # exact up to gradual underflow: the sweeps leave subnormal entries where scaling by 2 is not exact
    assert rel2(to_host(d2, n, M), 2.0 * F1) <= 1e-15
    A2 = ft.rand_layout(kind, n, 43)
    dB = to_dev(torch, A2)
    ft.execute_dev(P, True, "N", dB.data_ptr(), n, M, stream(torch))
    dS = to_dev(torch, A + A2)
    ft.execute_dev(P, True, "N", dS.data_ptr(), n, M, stream(torch))
    assert rel2(to_host(dS, n, M), F1 + to_host(dB, n, M)) < c2 * np.sqrt(n) * EPS
    # rotation stage alone is orthogonal: norms preserved, lo2hi(hi2lo(A)) = A
    RP = rot_plan(ft, kind, n, params)
    dR = to_dev(torch, A)
    ft.rotations_dev(RP, True, dR.data_ptr(), M, stream(torch))
    R1 = to_host(dR, n, M)
    assert abs(np.linalg.norm(R1) / np.linalg.norm(A) - 1) < 1e-13
    ft.rotations_dev(RP, False, dR.data_ptr(), M, stream(torch))
    assert rel2(to_host(dR, n, M), A) < 4 * np.sqrt(n) * EPS
    RP.close()
    P.close()
