"""Batched execution through ft_b200_execute_batched_dev: many fields of
different degrees in one launch per stage (the rotation kernel's longest-first
queue spans every field's tasks; one triangular-multiply launch covers every
field's column classes).  Results must equal per-field execution bit for bit
(same kernels, same arithmetic) and the oracle to 1e-14."""
import numpy as np
import pytest

from conftest import rel2

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


def make_fields(ft, torch, kind, degrees, params, seed0=500):
    planner = {"sph": ft.plan_sph2fourier, "tri": ft.plan_tri2cheb, "disk": ft.plan_disk2cxf}[kind]
    plans = {}
    fields = []
    for f, n in enumerate(degrees):
        if n not in plans:
            plans[n] = planner(n, *params)
        A = ft.rand_layout(kind, n, seed0 + f)
        fields.append((plans[n], A, torch.from_numpy(A.ravel(order="F").copy()).cuda()))
    return plans, fields


@pytest.mark.parametrize("kind,params,degrees", [
    ("sph", (), [15, 64, 33, 127, 64, 8, 2, 3]),
    ("disk", (0.0, 0.0), [9, 40, 40, 17]),
    ("tri", (0.0, 0.0, 0.0), [12, 30, 30]),
    ("tri", (-0.5, -0.5, -0.5), [7, 64, 33]),
    ("tri", (0.5, 1.0, -0.25), [16, 16]),
])
def test_batched_equals_per_field(env, kind, params, degrees):
    ft, torch, O = env
    st = torch.cuda.current_stream().cuda_stream
    plans, fields = make_fields(ft, torch, kind, degrees, params)
    for fwd in (True, False):
        for tr in "NT":
            batch = [t.clone() for _, _, t in fields]
            ft.execute_batched_dev([p for p, _, _ in fields], fwd, tr, [b.data_ptr() for b in batch],
                                   [p.n for p, _, _ in fields], [p.M for p, _, _ in fields], st)
            for (P, A, t), b in zip(fields, batch):
                single = t.clone()
                ft.execute_dev(P, fwd, tr, single.data_ptr(), P.n, P.M, st)
                got = b.cpu().numpy()
                assert np.array_equal(got, single.cpu().numpy()), (kind, P.n, fwd, tr)
                ref = A.copy(order="F")
                PO = O.plan(kind, P.n, *params)
                O.execute(PO, fwd, tr, ref)
                O.destroy(PO)
                assert rel2(got.reshape(A.shape, order="F"), ref) <= 1e-14
    for p in plans.values():
        p.close()


def test_batched_rejects_mixed_families(env):
    ft, torch, O = env
    a = ft.plan_sph2fourier(8)
    b = ft.plan_disk2cxf(8, 0.0, 0.0)
    ta = torch.zeros(8 * a.M, dtype=torch.float64, device="cuda")
    tb = torch.zeros(8 * b.M, dtype=torch.float64, device="cuda")
    with pytest.raises(ft.FTB200Error):
        ft.execute_batched_dev([a, b], True, "N", [ta.data_ptr(), tb.data_ptr()], [8, 8], [a.M, b.M])
    a.close()
    b.close()


def test_batched_fwd_bwd_in_cuda_graph(env):
    """fwd+bwd of an uneven batch captured once in a CUDA graph and replayed:
    equal to the eager batched result (the first, eager call builds the batch's
    tables and workspace outside the capture)."""
    ft, torch, O = env
    plans, fields = make_fields(ft, torch, "sph", [31, 64, 127, 64, 255], ())
    P = [p for p, _, _ in fields]
    Ns = [p.n for p in P]
    Ms = [p.M for p in P]
    work = [t.clone() for _, _, t in fields]
    ptrs = [w.data_ptr() for w in work]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):   # warm-up outside capture
        ft.execute_batched_dev(P, True, "N", ptrs, Ns, Ms, s.cuda_stream)
        ft.execute_batched_dev(P, False, "N", ptrs, Ns, Ms, s.cuda_stream)
    torch.cuda.current_stream().wait_stream(s)
    eager = [w.clone() for w in work]
    ft.execute_batched_dev(P, True, "N", [e.data_ptr() for e in eager], Ns, Ms, torch.cuda.current_stream().cuda_stream)
    ft.execute_batched_dev(P, False, "N", [e.data_ptr() for e in eager], Ns, Ms, torch.cuda.current_stream().cuda_stream)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cs = torch.cuda.current_stream().cuda_stream
        ft.execute_batched_dev(P, True, "N", ptrs, Ns, Ms, cs)
        ft.execute_batched_dev(P, False, "N", ptrs, Ns, Ms, cs)
    g.replay()
    torch.cuda.synchronize()
    for w, e in zip(work, eager):
        assert torch.equal(w, e)
    del g
    for p in plans.values():
        p.close()


def test_batched_tri_mixed_parameters(env):
    """tri plans whose parameters call for different multiplies in one batch."""
    ft, torch, O = env
    st = torch.cuda.current_stream().cuda_stream
    specs = [((0.0, 0.0, 0.0), 20), ((-0.5, -0.5, -0.5), 24), ((0.0, 0.0, 0.0), 9)]
    plans = [ft.plan_tri2cheb(n, *p) for p, n in specs]
    As = [ft.trirand(n, 7 + i) for i, (_, n) in enumerate(specs)]
    ts = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in As]
    ft.execute_batched_dev(plans, True, "N", [t.data_ptr() for t in ts], [p.n for p in plans], [p.M for p in plans], st)
    for (params, n), A, t in zip(specs, As, ts):
        ref = A.copy(order="F")
        PO = O.plan("tri", n, *params)
        O.execute(PO, True, "N", ref)
        O.destroy(PO)
        assert rel2(t.cpu().numpy().reshape(A.shape, order="F"), ref) <= 1e-14
    for p in plans:
        p.close()
