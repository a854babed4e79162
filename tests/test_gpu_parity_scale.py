"""FP64 parity at the benchmarked sizes: the GPU's transforms against the reference library
compiled from its own sources (oracle/_ref/libft_ref.so), on the same seeded inputs, through
the C ABI.

* sph at degrees 255, 1023 and 4095 (n = 256, 1024, 4096; M = 2n - 1); tri with
  (alpha, beta, gamma) = (0, 0, 0) and (-1/2, -1/2, -1/2) and disk with (alpha, beta) = (0, 0) at
  n = 1024 and 2048: forward and backward, 'N' and 'T', each against the reference's output for
  the same input.  The bar is a relative 2-norm of 1e-14 (the rotation stage is bit-identical to
  the oracle, the plans' connection matrices are the reference's bit for bit, and only the
  triangular multiplies sum in another order), or the reference's own round-trip error on the
  same input where that is larger: the triangle transform with (0, 0, 0) amplifies rounding
  (the reference's published round trip at degree 2047 is 7.3e-14), so two correct
  implementations differ by up to that much.
* The reference's own accuracy test (test/test_drivers.c:226-250 for sph, and the tri / disk
  tests of the same file) at n = 64 * 2^i + J for the sizes above: sph2fourier and fourier2sph
  'N' then 'T' return the input within its bounds (4 sqrt(N) eps / 2N eps sph, 32 sqrt(N) eps /
  8N eps tri, 8 sqrt(N) eps / 4N eps disk), or within twice the reference's own round-trip error
  for the same input where the reference itself exceeds them.
"""
import numpy as np
import pytest

from conftest import EPS, rel2, relinf

pytestmark = pytest.mark.gpu

TOL = {"sph": (4, 2), "tri": (32, 8), "disk": (8, 4)}

CASES = [("sph", (), 256), ("sph", (), 1024), ("sph", (), 4096),
         ("tri", (0.0, 0.0, 0.0), 1024), ("tri", (-0.5, -0.5, -0.5), 1024), ("disk", (0.0, 0.0), 1024),
         ("tri", (0.0, 0.0, 0.0), 2048), ("tri", (-0.5, -0.5, -0.5), 2048), ("disk", (0.0, 0.0), 2048)]


def _id(c):
    kind, params, n = c
    return f"{kind}{''.join('%+.1f' % p for p in params)}-n{n}"


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Reference
    if not Reference.available():
        pytest.fail("the compiled reference (oracle/_ref/libft_ref.so) is missing: run __graft_entry__.build()")
    torch.cuda.set_device(0)
    return ft, torch, Reference()


def _gpu_plan(ft, kind, n, params):
    return {"sph": ft.plan_sph2fourier, "tri": ft.plan_tri2cheb, "disk": ft.plan_disk2cxf}[kind](n, *params)


def _dev(torch, A):
    return torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()


def _host(t, n, M):
    return t.cpu().numpy().reshape((n, M), order="F")


@pytest.mark.parametrize("case", CASES, ids=[_id(c) for c in CASES])
def test_transforms_vs_compiled_reference(env, case):
    ft, torch, R = env
    kind, params, n = case
    A = ft.rand_layout(kind, n, 20261203)
    M = A.shape[1]
    P = _gpu_plan(ft, kind, n, params)
    RP = R.plan(kind, n, *params)
    stream = torch.cuda.current_stream().cuda_stream
    errs = {}
    try:
        rt = A.copy(order="F")   # the reference's own round trip: its conditioning on this input
        R.execute(kind, RP, True, "N", rt)
        R.execute(kind, RP, False, "N", rt)
        bar = max(1e-14, rel2(rt, A))
        for fwd in (True, False):
            for tr in "NT":
                d = _dev(torch, A)
                ft.execute_dev(P, fwd, tr, d.data_ptr(), n, M, stream)
                got = _host(d, n, M)
                ref = A.copy(order="F")
                R.execute(kind, RP, fwd, tr, ref)
                errs[("fwd" if fwd else "bwd") + tr] = (rel2(got, ref), relinf(got, ref))
    finally:
        R.destroy(RP)
        P.close()
    print(f"\n{_id(case)} vs reference (rel2, relinf): " + ", ".join(f"{k} {a:.2e} {b:.2e}" for k, (a, b) in errs.items())
          + f"; bar {bar:.2e}")
    for k, (e2, _) in errs.items():
        assert e2 <= bar, (k, e2, bar)


RT_CASES = [("sph", (), 1024), ("sph", (), 2049), ("tri", (0.0, 0.0, 0.0), 1024), ("tri", (-0.5, -0.5, -0.5), 2048),
            ("disk", (0.0, 0.0), 1025), ("disk", (0.0, 0.0), 2048)]


@pytest.mark.parametrize("case", RT_CASES, ids=[_id(c) for c in RT_CASES])
def test_reference_accuracy_test_at_scale(env, case):
    """test/test_drivers.c's sequence: forward 'N', backward 'N', forward 'T', backward 'T'."""
    ft, torch, R = env
    kind, params, n = case
    A = ft.rand_layout(kind, n, 7)
    M = A.shape[1]
    P = _gpu_plan(ft, kind, n, params)
    stream = torch.cuda.current_stream().cuda_stream
    seq = ((True, "N"), (False, "N"), (True, "T"), (False, "T"))
    d = _dev(torch, A)
    for fwd, tr in seq:
        ft.execute_dev(P, fwd, tr, d.data_ptr(), n, M, stream)
    got = _host(d, n, M)
    P.close()
    ref = A.copy(order="F")
    RP = R.plan(kind, n, *params)
    for fwd, tr in seq:
        R.execute(kind, RP, fwd, tr, ref)
    R.destroy(RP)
    c2, ci = TOL[kind]
    print(f"\n{_id(case)} round trip: GPU {rel2(got, A):.2e} / {relinf(got, A):.2e}, "
          f"reference {rel2(ref, A):.2e} / {relinf(ref, A):.2e}, bounds {c2 * np.sqrt(n) * EPS:.2e} / {ci * n * EPS:.2e}")
    assert rel2(got, A) < max(c2 * np.sqrt(n) * EPS, 2 * rel2(ref, A))
    assert relinf(got, A) < max(ci * n * EPS, 2 * relinf(ref, A))


QUAD_COLS = lambda M: sorted({0, 1, 2, 3, 4, 5, 6, M // 4 - 1, M // 4, M // 4 + 1, M // 4 + 2, M // 2 - 1, M // 2, M // 2 + 1,
                              M // 2 + 2, 3 * M // 4, 3 * M // 4 + 1, M - 4, M - 3, M - 2, M - 1})


def _host_connections(P, n):
    """The plan's host connection matrices P[0], P[1] (the reference's, bit for bit)."""
    import ctypes as C
    from oracle.bind import _RefHarmonicPlan
    hp = C.cast(C.c_void_p(P.ptr), C.POINTER(_RefHarmonicPlan)).contents
    return [np.triu(np.ctypeslib.as_array(hp.P[i], shape=(n * n,)).reshape(n, n, order="F")) for i in range(2)]


@pytest.mark.parametrize("kind,params,n", [("sph", (), 1024), ("sph", (), 4096), ("disk", (0.0, 0.0), 2048)])
def test_forward_vs_quad_precision(env, kind, params, n):
    """The plain FP64 forward transform 'N' against the __float128 oracle (oracle/ft_quad.c: the
    reference's tables and sweeps in quad precision, with the plan's own connection matrices),
    on columns of every class spread over all orders: within 1e-14 relative (the arithmetic
    error of double precision; the compiled reference lies at the same distance)."""
    ft, torch, R = env
    from oracle.bind import Quad
    A = ft.rand_layout(kind, n, 20261203)
    M = A.shape[1]
    P = _gpu_plan(ft, kind, n, params)
    d = _dev(torch, A)
    ft.execute_dev(P, True, "N", d.data_ptr(), n, M, torch.cuda.current_stream().cuda_stream)
    got = _host(d, n, M)
    cols = QUAD_COLS(M)
    hi, _ = Quad().columns(kind, A, cols, params, True, _host_connections(P, n))
    P.close()
    e2, ei = rel2(got[:, cols], hi), relinf(got[:, cols], hi)
    print(f"\n{_id((kind, params, n))} forward vs quad on {len(cols)} columns: {e2:.2e} / {ei:.2e}")
    assert e2 <= 1e-14, e2


@pytest.mark.parametrize("prec,bound", [("FP64", 1e-14), ("FP64_BLOCKED", 1e-13), ("MIXED_BF16", 1e-6), ("MIXED_BF16X4", 1e-6)])
def test_shared_precisions_vs_quad_precision(env, prec, bound):
    """Every precision of the shared-plan call (two fields of degree 2047) against the quad
    oracle: FP64 and the blocked FP64 tile products at double-precision accuracy, the split-BF16
    forms within the 1e-6 of the mixed-precision target."""
    ft, torch, R = env
    from oracle.bind import Quad
    n = 2048
    P = ft.plan_sph2fourier(n)
    M = P.M
    As = [ft.rand_layout("sph", n, 500 + f) for f in range(2)]
    ts = [_dev(torch, A) for A in As]
    ft.execute_shared_dev(P, True, "N", [t.data_ptr() for t in ts], getattr(ft, prec), torch.cuda.current_stream().cuda_stream)
    cols = QUAD_COLS(M)
    Q = Quad()
    conn = _host_connections(P, n)
    for A, t in zip(As, ts):
        hi, _ = Q.columns("sph", A, cols, (), True, conn)
        got = _host(t, n, M)[:, cols]
        print(f"\n{prec} vs quad: {rel2(got, hi):.2e} / {relinf(got, hi):.2e}")
        assert rel2(got, hi) <= bound, (prec, rel2(got, hi))
    P.close()
