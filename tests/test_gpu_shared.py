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
