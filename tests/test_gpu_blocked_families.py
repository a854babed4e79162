"""Blocked forms of ft_b200_execute_shared_dev for the disk and tri families
(disk2cxf / cxf2disk, src/drivers.c:989-1021; tri2cheb / cheb2tri,
src/drivers.c:921-957), on fields sharing one plan.

FP64_BLOCKED: whole blocks of 32 sweeps as pre-multiplied 64 x 64 tile
matrices on the FP64 tensor pipe; rounds differently from the direct sweeps,
held to 1e-13 relative against the oracle (as for sph).
MIXED_BF16 / MIXED_BF16X4, disk: the same tiles on the tcgen05 tensor cores
from fixed-point BF16 slices, and the connection multiplies too.  The slicing
error of the sweeps (about 2e-7 relative) is amplified by the connection
multiplies that follow them, by a factor that depends on the family's
parameters: the bounds below are per family and precision, about three times
the largest relative 2-norm error measured against the FP64 transform for
n <= 1024 (measured at n = 2048, MIXED_BF16 / MIXED_BF16X4: disk (0, 0)
2.9e-7 / 1.7e-7, disk (1/2, -1/4) 3.1e-6 / 4.5e-7).
MIXED_BF16 / MIXED_BF16X4, tri: the sweeps stay in FP64 (the triangle's
multiplies amplify a sliced sweep's error to 3e-6 .. 3e-5), the two connection
multiplies run on the tensor cores from four slices of each operand (the
right one through two transposes), each 256-row chunk's exact level sums
recombined and added into the output in FP64 (with FP32 recombination the
transform's conditioning left 1.3e-6 at n = 1024 and 2.2e-6 at 2048 for
(0, 0, 0)).

The parameters are the reference's test choices (test/test_drivers.c): disk
(alpha, beta) = (0, 0) and a generic pair; tri (0, 0, 0), (-1/2, -1/2, -1/2)
(no right multiply: an odd number of multiplies, so the sweeps run out of
place) and a generic triple."""
import numpy as np
import pytest

from conftest import rel2

pytestmark = pytest.mark.gpu

FAMILIES = [
    ("disk", (0.0, 0.0)),
    ("disk", (0.5, -0.25)),
    ("tri", (0.0, 0.0, 0.0)),
    ("tri", (-0.5, -0.5, -0.5)),
    ("tri", (0.25, -0.125, 0.375)),
]
IDS = ["disk00", "disk_generic", "tri000", "tri_half", "tri_generic"]
# family -> bound on the relative 2-norm error for precision 1 (FP64_BLOCKED), 2, 3
TOL = {
    "disk00": {1: 1e-13, 2: 1e-6, 3: 1e-6},
    "disk_generic": {1: 1e-13, 2: 6e-6, 3: 1.5e-6},
    "tri000": {1: 1e-13, 2: 1e-6, 3: 1e-6},
    "tri_half": {1: 1e-13, 2: 1e-6, 3: 1e-6},
    "tri_generic": {1: 1e-13, 2: 2e-6, 3: 2e-6},
}


def tol(fam, prec):
    return TOL[IDS[FAMILIES.index(fam)]][prec]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, torch, O


def make_plan(ft, kind, n, params):
    return ft.plan_disk2cxf(n, *params) if kind == "disk" else ft.plan_tri2cheb(n, *params)


def rand(ft, kind, n, seed):
    return ft.diskrand(n, seed) if kind == "disk" else ft.trirand(n, seed)


def run_shared(ft, torch, P, fields, fwd, tr, prec):
    ts = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in fields]
    ft.execute_shared_dev(P, fwd, tr, [t.data_ptr() for t in ts], prec, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return [t.cpu().numpy().reshape(A.shape, order="F") for t, A in zip(ts, fields)]


@pytest.mark.parametrize("prec", [1, 2, 3])
@pytest.mark.parametrize("n,nf", [(40, 1), (65, 3), (130, 5), (257, 9)])
@pytest.mark.parametrize("fam", FAMILIES, ids=IDS)
def test_blocked_forms_vs_oracle(env, fam, n, nf, prec):
    ft, torch, O = env
    kind, params = fam
    P = make_plan(ft, kind, n, params)
    PO = O.plan(kind, n, *params)
    fields = [rand(ft, kind, n, 50 + f) for f in range(nf)]
    for fwd in (True, False):
        for tr in "NT":
            got = run_shared(ft, torch, P, fields, fwd, tr, prec)
            for A, g in zip(fields, got):
                ref = A.copy(order="F")
                O.execute(PO, fwd, tr, ref)
                assert rel2(g, ref) <= tol(fam, prec), (kind, params, n, fwd, tr, prec, rel2(g, ref))
    assert ft.device_status(P) == 0
    O.destroy(PO)
    P.close()


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("fam", [FAMILIES[0], FAMILIES[2], FAMILIES[3]], ids=["disk00", "tri000", "tri_half"])
def test_blocked_forms_large(env, fam, prec):
    """n = 1024, two fields: forward within the bound of the oracle, the round
    trip within twice the bound of the input, two runs bit-identical."""
    ft, torch, O = env
    kind, params = fam
    n = 1024
    P = make_plan(ft, kind, n, params)
    fields = [rand(ft, kind, n, 80 + f) for f in range(2)]
    fw = run_shared(ft, torch, P, fields, True, "N", prec)
    fw2 = run_shared(ft, torch, P, fields, True, "N", prec)
    PO = O.plan(kind, n, *params)
    for A, g, g2 in zip(fields, fw, fw2):
        assert np.array_equal(g, g2)
        ref = A.copy(order="F")
        O.execute(PO, True, "N", ref)
        assert rel2(g, ref) <= tol(fam, prec), (kind, prec, rel2(g, ref))
    back = run_shared(ft, torch, P, fw, False, "N", prec)
    for A, b in zip(fields, back):
        assert rel2(b, A) <= 2 * tol(fam, prec)
    assert ft.device_status(P) == 0
    O.destroy(PO)
    P.close()


def test_blocked_direct_agree_large_disk(env):
    """disk at n = 2048, the degree of the sibling benchmark: the split-BF16
    form against the direct FP64 form on the GPU (no oracle at this size)."""
    ft, torch, O = env
    n = 2048
    P = ft.plan_disk2cxf(n, 0.0, 0.0)
    fields = [ft.diskrand(n, 91)]
    d = run_shared(ft, torch, P, fields, True, "N", ft.FP64)
    for prec in (1, 2, 3):
        g = run_shared(ft, torch, P, fields, True, "N", prec)
        assert rel2(g[0], d[0]) <= tol(FAMILIES[0], prec), (prec, rel2(g[0], d[0]))
    assert ft.device_status(P) == 0
    P.close()


@pytest.mark.parametrize("kind", ["sph", "disk"])
def test_even_column_count_rejected(env, kind):
    """Order m occupies columns 2m-1 and 2m, m <= M/2: an even M >= 4 would reach
    column M, so it is rejected before anything runs."""
    ft, torch, O = env
    n = 16
    P = ft.plan_sph2fourier(n) if kind == "sph" else ft.plan_disk2cxf(n, 0.0, 0.0)
    M = P.M - 1
    t = torch.zeros(n * (M + 1), dtype=torch.float64, device="cuda")
    t[n * M:] = 7.0   # the column past the matrix
    with pytest.raises(ft.FTB200Error):
        ft.execute_dev(P, True, "N", t.data_ptr(), n, M)
    torch.cuda.synchronize()
    assert bool((t[n * M:] == 7.0).all())
    P.close()
