"""Split-BF16 tensor-core paths of ft_b200_execute_shared_dev (sph fields
sharing one plan): whole blocks of 32 sweeps as tile products and the
connection multiply, both from fixed-point BF16 slices on the tcgen05 tensor
cores.  Checked against the oracle's FP64 transform; the bound is the
relative 2-norm error the slicing is built for: 1e-6 (measured about 1e-7 ..
5e-7 up to n = 4096 for both MIXED_BF16, three slices, and MIXED_BF16X4,
four slices)."""
import numpy as np
import pytest

from conftest import rel2

pytestmark = pytest.mark.gpu

TOL = {2: 1e-6, 3: 1e-6}   # precision -> bound on the relative 2-norm error


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


def run_shared(ft, torch, P, fields, fwd, tr, prec):
    ts = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in fields]
    ft.execute_shared_dev(P, fwd, tr, [t.data_ptr() for t in ts], prec, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return [t.cpu().numpy().reshape(A.shape, order="F") for t, A in zip(ts, fields)]


@pytest.mark.parametrize("prec", [2, 3])
@pytest.mark.parametrize("n,nf", [(64, 1), (65, 3), (200, 2), (513, 3)])
def test_mixed_vs_oracle(env, prec, n, nf):
    ft, torch, O = env
    P = ft.plan_sph2fourier(n)
    PO = O.plan("sph", n)
    fields = [ft.sphrand(n, 40 + f) for f in range(nf)]
    for fwd in (True, False):
        for tr in "NT":
            got = run_shared(ft, torch, P, fields, fwd, tr, prec)
            for A, g in zip(fields, got):
                ref = A.copy(order="F")
                O.execute(PO, fwd, tr, ref)
                assert rel2(g, ref) <= TOL[prec], (prec, n, fwd, tr, rel2(g, ref))
    assert ft.device_status(P) == 0
    O.destroy(PO)
    P.close()


@pytest.mark.parametrize("prec", [2, 3])
def test_mixed_large_and_round_trip(env, prec):
    """n = 2048, three fields: forward within 1e-6 of the oracle, the round
    trip within 2e-6 of the input, and two runs bit-identical."""
    ft, torch, O = env
    n = 2048
    P = ft.plan_sph2fourier(n)
    fields = [ft.sphrand(n, 70 + f) for f in range(3)]
    fw = run_shared(ft, torch, P, fields, True, "N", prec)
    fw2 = run_shared(ft, torch, P, fields, True, "N", prec)
    PO = O.plan("sph", n)
    for A, g, g2 in zip(fields, fw, fw2):
        assert np.array_equal(g, g2)
        ref = A.copy(order="F")
        O.execute(PO, True, "N", ref)
        assert rel2(g, ref) <= 1e-6
    back = run_shared(ft, torch, P, fw, False, "N", prec)
    for A, b in zip(fields, back):
        assert rel2(b, A) <= 2e-6
    assert ft.device_status(P) == 0
    O.destroy(PO)
    P.close()


def test_shared_rejects_unknown_precision(env):
    ft, torch, O = env
    P = ft.plan_tri2cheb(16, 0.0, 0.0, 0.0)
    t = torch.zeros(16 * 16, dtype=torch.float64, device="cuda")
    with pytest.raises(ft.FTB200Error):
        ft.execute_shared_dev(P, True, "N", [t.data_ptr()], 7)
    P.close()
