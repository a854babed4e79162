"""The rotation kernel's launch shapes and the autotuner that picks among them
(ft_b200_set_rotation_config).  Every shape computes the same rotations in the
same order per element, so the transforms must agree bit for bit whichever
shape runs; the first out-of-place launch of a new shape times the candidates
(visible as extra kernel launches), later ones reuse the choice."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("sph", 200, ()), ("tri", 150, (0.0, 0.0, 0.0)), ("disk", 150, (0.0, 0.0))]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    torch.cuda.set_device(0)
    yield ft, torch
    ft.set_rotation_config(-1)


def make_plan(ft, kind, n, params):
    if kind == "sph":
        return ft.plan_sph2fourier(n)
    return ft.plan_tri2cheb(n, *params) if kind == "tri" else ft.plan_disk2cxf(n, *params)


def transform(ft, torch, P, A, fwd, tr):
    n, M = A.shape
    t = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    ft.execute_dev(P, fwd, tr, t.data_ptr(), n, M, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("kind,n,params", CASES, ids=[c[0] for c in CASES])
def test_every_shape_bit_identical(env, kind, n, params):
    ft, torch = env
    P = make_plan(ft, kind, n, params)
    A = ft.rand_layout(kind, n, 31)
    try:
        ft.set_rotation_config(-1)
        ref = {(fwd, tr): transform(ft, torch, P, A, fwd, tr) for fwd in (True, False) for tr in "NT"}
        for cfg in range(6):
            ft.set_rotation_config(cfg)
            for (fwd, tr), r in ref.items():
                assert np.array_equal(transform(ft, torch, P, A, fwd, tr), r), (kind, cfg, fwd, tr)
    finally:
        ft.set_rotation_config(-1)
        P.close()


def test_first_launch_of_a_shape_is_tuned(env):
    """A degree no other test uses: the first forward transform times the
    candidate shapes (several extra rotation launches), the second does not."""
    ft, torch = env
    ft.set_rotation_config(-1)
    n = 333
    P = ft.plan_sph2fourier(n)
    A = ft.sphrand(n, 32)
    c0 = ft.kernel_launches()
    first = transform(ft, torch, P, A, True, "N")
    c1 = ft.kernel_launches()
    second = transform(ft, torch, P, A, True, "N")
    c2 = ft.kernel_launches()
    assert np.array_equal(first, second)
    # six shapes for sph, one untimed and one timed launch each
    assert (c1 - c0) - (c2 - c1) == 12, (c1 - c0, c2 - c1)
    P.close()
