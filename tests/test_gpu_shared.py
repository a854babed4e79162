"""Fields sharing one plan: ft_b200_execute_shared_dev, direct and blocked.

The blocked form applies whole blocks of 32 sweeps as pre-multiplied 64 x 64
tile matrices (FP64 tensor-core products); it rounds differently from the
direct sweeps, so it is held to 1e-13 relative against the oracle, while the
direct form is bit-identical to per-field execution."""
import numpy as np
import pytest

from conftest import EPS, rel2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


@pytest.mark.parametrize("n", [16, 65, 130, 257, 300])
def test_shared_direct_and_blocked_vs_oracle(env, n):
    ft, torch, O = env
    st = torch.cuda.current_stream().cuda_stream
    P = ft.plan_sph2fourier(n)
    PO = O.plan("sph", n)
    As = [ft.sphrand(n, 40 + f) for f in range(3)]
    for fwd in (True, False):
        for tr in "NT":
            for prec in (ft.FP64, ft.FP64_BLOCKED):
                ts = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in As]
                ft.execute_shared_dev(P, fwd, tr, [t.data_ptr() for t in ts], prec, st)
                for A, t in zip(As, ts):
                    ref = A.copy(order="F")
                    O.execute(PO, fwd, tr, ref)
                    got = t.cpu().numpy().reshape(A.shape, order="F")
                    bound = 1e-14 if prec == ft.FP64 else 1e-13
                    assert rel2(got, ref) <= bound, (n, fwd, tr, prec, rel2(got, ref))
    O.destroy(PO)
    P.close()


def test_blocked_round_trip_large(env):
    ft, torch, O = env
    st = torch.cuda.current_stream().cuda_stream
    n = 2048
    P = ft.plan_sph2fourier(n)
    As = [ft.sphrand(n, 90 + f) for f in range(2)]
    ts = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in As]
    direct = [t.clone() for t in ts]
    ft.execute_shared_dev(P, True, "N", [t.data_ptr() for t in ts], ft.FP64_BLOCKED, st)
    ft.execute_shared_dev(P, True, "N", [t.data_ptr() for t in direct], ft.FP64, st)
    for t, d in zip(ts, direct):
        assert rel2(t.cpu().numpy(), d.cpu().numpy()) <= 1e-13
    ft.execute_shared_dev(P, False, "N", [t.data_ptr() for t in ts], ft.FP64_BLOCKED, st)
    for A, t in zip(As, ts):
        assert rel2(t.cpu().numpy().reshape(A.shape, order="F"), A) < 4 * np.sqrt(n) * EPS * 10
    P.close()


@pytest.mark.parametrize("kind,params,n,nf", [("sph", (), 64, 10), ("sph", (), 257, 5), ("disk", (0.0, 0.0), 96, 7),
                                              ("tri", (0.0, 0.0, 0.0), 120, 3)])
def test_shared_host_pipeline_matches_device_call(env, kind, params, n, nf):
    """ft_b200_execute_shared_host (host fields in groups through three device buffers, copies
    overlapped with the transforms) gives the device call's results bit for bit, for a sequence
    of transforms, with uneven group sizes (10 fields: groups 2, 4, 2, 2), page-locked and
    pageable host memory."""
    ft, torch, O = env
    st = torch.cuda.current_stream().cuda_stream
    planner = {"sph": ft.plan_sph2fourier, "tri": ft.plan_tri2cheb, "disk": ft.plan_disk2cxf}[kind]
    P = planner(n, *params)
    As = [ft.rand_layout(kind, n, 300 + f) for f in range(nf)]
    ops = [(True, "N"), (False, "T"), (True, "T")]
    for prec in (ft.FP64, ft.MIXED_BF16):
        ts = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in As]
        for fwd, tr in ops:
            ft.execute_shared_dev(P, fwd, tr, [t.data_ptr() for t in ts], prec, st)
        want = [t.cpu().numpy() for t in ts]
        pageable = [A.copy(order="F") for A in As]
        ft.execute_shared_host(P, ops, pageable, prec)
        pinned = [torch.from_numpy(A.ravel(order="F").copy()).pin_memory() for A in As]
        ft.execute_shared_host(P, ops, [h.data_ptr() for h in pinned], prec)
        for f in range(nf):
            assert np.array_equal(pageable[f].ravel(order="F"), want[f]), (prec, f)
            assert np.array_equal(pinned[f].numpy(), want[f]), (prec, f)
    with pytest.raises(ft.FTB200Error):
        ft.execute_shared_host(P, [(True, "X")], [As[0].copy(order="F")], ft.FP64)
    P.close()
