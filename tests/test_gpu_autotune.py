"""The rotation kernel's launch configurations (six shapes, each without the pass
pipeline and with its two queue modes) and the autotuner that picks among them
(ft_b200_set_rotation_config).  Every configuration computes the same rotations
in the same order per element, so the transforms must agree bit for bit
whichever runs; the first out-of-place launch of a new shape times the
candidates (visible as extra kernel launches), later ones reuse the choice."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("sph", 200, ()), ("tri", 150, (0.0, 0.0, 0.0)), ("disk", 150, (0.0, 0.0)), ("sph", 700, ())]


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


@pytest.mark.parametrize("kind,n,params", CASES, ids=[f"{c[0]}{c[1]}" for c in CASES])
def test_every_shape_bit_identical(env, kind, n, params):
    ft, torch = env
    P = make_plan(ft, kind, n, params)
    A = ft.rand_layout(kind, n, 31)
    try:
        ft.set_rotation_config(-1)
        ref = {(fwd, tr): transform(ft, torch, P, A, fwd, tr) for fwd in (True, False) for tr in "NT"}
        for cfg in [s + 8 * p for p in range(3) for s in range(6)]:
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
    # six shapes for sph, without the pipeline and in its two queue modes, one untimed and one
    # timed launch each
    assert (c1 - c0) - (c2 - c1) == 36, (c1 - c0, c2 - c1)
    P.close()


@pytest.mark.parametrize("kind,n,params", [("sph", 1024, ()), ("tri", 700, (0.0, 0.0, 0.0)), ("disk", 600, (0.0, 0.0))],
                         ids=["sph1024", "tri700", "disk600"])
def test_pass_pipeline_rotation_stage_bitexact(env, kind, n, params):
    """Pass r of a task runs on another SM behind pass r - 1 (the pass pipeline,
    forced: configurations 8, 10, 12).  Sizes with many passes per task, every
    pass length (64, 32 and 16 sweeps), three runs each: the rotation stage
    equals the oracle's bit for bit every time, and no pipeline wait ran out."""
    ft, torch = env
    from oracle.bind import Oracle
    O = Oracle()
    O.set_fused(True)
    A = ft.rand_layout(kind, n, 77)
    M = A.shape[1]
    RP = {"sph": ft.plan_rotsphere, "tri": ft.plan_rottriangle, "disk": ft.plan_rotdisk}[kind](n, *params)
    PO = O.plan(kind, n, *params, rotations_only=True)
    refs = {}
    for hi2lo in (True, False):
        r = A.copy(order="F")
        (O.hi2lo if hi2lo else O.lo2hi)(PO, r)
        refs[hi2lo] = r
    try:
        for cfg in (8, 10, 12, 16, 19):
            ft.set_rotation_config(cfg)
            for _ in range(3):
                for hi2lo in (True, False):
                    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
                    ft.rotations_dev(RP, hi2lo, d.data_ptr(), M, torch.cuda.current_stream().cuda_stream)
                    torch.cuda.synchronize()
                    got = d.cpu().numpy().reshape((n, M), order="F")
                    assert np.array_equal(got, refs[hi2lo]), (kind, cfg, hi2lo)
    finally:
        ft.set_rotation_config(-1)
        O.destroy(PO)
        RP.close()
    P = ft.plan_sph2fourier(8)
    assert ft.device_status(P) == 0
    P.close()
