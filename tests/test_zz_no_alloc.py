"""The allocation-free entry point, ft_b200_execute_noalloc_dev.

It exists for callers that cannot let a library allocate device memory (a
framework that owns all device memory through its own pool, or a service that
must not allocate after start-up).  Its intermediate matrix lives in a fixed
device array inside the library instead of the plan's scratch.  This file is
collected last, so a run that stops at the first failure has already run every
other test; it also passes when run alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,params,n", [("sph", (), 64), ("sph", (), 511), ("tri", (0.0, 0.0, 0.0), 300),
                                           ("disk", (0.0, 0.0), 160)])
def test_noalloc_matches_execute_dev_twice(kind, params, n):
    import torch
    import fasttransforms_b200 as ft
    torch.cuda.set_device(0)
    plan = {"sph": ft.plan_sph2fourier, "tri": ft.plan_tri2cheb, "disk": ft.plan_disk2cxf}[kind](n, *params)
    M = plan.M
    assert n * M <= ft.NOALLOC_MAX_ELEMS
    st = torch.cuda.current_stream().cuda_stream
    for call in range(2):   # two calls in a row: the shared array keeps the previous call's contents
        A = ft.rand_layout(kind, n, 1000 + call)
        for fwd in (True, False):
            for tr in "NT":
                a = torch.from_numpy(A.ravel(order="F").copy()).cuda()
                b = a.clone()
                ft.execute_dev(plan, fwd, tr, a.data_ptr(), n, M, st)
                ft.execute_noalloc_dev(plan, fwd, tr, b.data_ptr(), n, M, st)
                # the same kernels in the same order: bit-identical results
                assert np.array_equal(b.cpu().numpy(), a.cpu().numpy()), (call, fwd, tr)
    plan.close()


def test_noalloc_takes_no_device_memory():
    """A warm call leaves the device's free memory unchanged (an allocation on this path, by the
    library or by anything it calls, would lower it)."""
    import torch
    import fasttransforms_b200 as ft
    torch.cuda.set_device(0)
    n = 256
    plan = ft.plan_sph2fourier(n)
    M = plan.M
    st = torch.cuda.current_stream().cuda_stream
    a = torch.from_numpy(ft.rand_layout("sph", n, 5).ravel(order="F").copy()).cuda()
    ft.execute_noalloc_dev(plan, True, "N", a.data_ptr(), n, M, st)   # first call: the per-device set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for fwd in (True, False):
        for tr in "NT":
            ft.execute_noalloc_dev(plan, fwd, tr, a.data_ptr(), n, M, st)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    plan.close()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_oversize_and_bad_arguments():
    import torch
    import fasttransforms_b200 as ft
    torch.cuda.set_device(0)
    n = 1024   # n * (2n - 1) = 2,096,128 > 1 << 20
    plan = ft.plan_sph2fourier(n)
    a = torch.zeros(n * plan.M, dtype=torch.float64, device="cuda")
    with pytest.raises(ft.FTB200Error) as e:
        ft.execute_noalloc_dev(plan, True, "N", a.data_ptr(), n, plan.M)
    assert e.value.status == 1 and "limit" in str(e.value)
    plan.close()
    small = ft.plan_sph2fourier(32)
    b = torch.zeros(32 * small.M, dtype=torch.float64, device="cuda")
    with pytest.raises(ft.FTB200Error):
        ft.execute_noalloc_dev(small, True, "X", b.data_ptr(), 32, small.M)
    small.close()
