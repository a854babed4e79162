"""Pins the annulus part of the oracle (oracle/ft_oracle.c: plan_rotannulus with its Jacobi
tridiagonal, Givens QR, Jacobi similarity and tridiagonal Cholesky, oracle_plan_ann2cxf and the
transforms, restating src/rotations.c:192-268, src/drivers.c:1023-1121 and
src/banded_source.c:381-498, 1415-1458, 1609-1619, 1797-1830) against the reference compiled
from its own sources and against the golden fixtures it produced.  CPU only.

The table comes out of long chains of QR and similarity recurrences; the reference's build
contracts products and sums into FMAs there (gcc's default for C with an FMA target) and the
oracle's does not, so the tables agree to a few ulps, not bit for bit.  Bars: the table within
2n ulps; transforms within 1e-14 at the reference test's rho = sqrt(1/3) and at rho = 0.4, within
4e-14 at rho = 0 (t = 1, the unshifted limit, where the recurrences amplify those ulps most:
1.8e-14 at n = 64); the reference's own round trips (test/test_drivers.c:985-1020,
1128-1150: 6 sqrt(N) eps / 5N eps for the sweeps, 12 sqrt(N) eps / 6N eps for the transforms)."""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ann_*.npz")))
CASES = [(0.0, 0.0, np.sqrt(1 / 3)), (0.5, -0.25, 0.4), (0.0, 0.0, 0.0)]


@pytest.fixture(scope="module")
def oracles():
    from oracle.bind import Oracle, Reference
    O = Oracle()
    O.set_fused(True)
    return O, Reference()


@pytest.mark.parametrize("n", [1, 2, 5, 16, 33, 64])
@pytest.mark.parametrize("case", CASES, ids=["rho_test", "generic", "rho0"])
def test_ann_vs_reference(oracles, n, case):
    O, R = oracles
    from oracle.bind import fill
    a, b, rho = case
    Po = O.ann_plan(n, a, b, rho)
    so, co = O.ann_table(Po)
    sr, cr = R.ann_table(n, a, b, rho)
    assert np.abs(so - sr).max() <= 2 * n * EPS and np.abs(co - cr).max() <= 2 * n * EPS
    A = fill("disk", n, 7)
    P = R.ann_plan(n, a, b, rho)
    tol = 4e-14 if rho == 0.0 else 1e-14
    for fwd in (True, False):
        for tr in "NT":
            x, y = A.copy(order="F"), A.copy(order="F")
            R.ann_execute(P, fwd, tr, x)
            O.ann_execute(Po, fwd, tr, y)
            assert rel2(y, x) <= tol, (fwd, tr, rel2(y, x))
    R.destroy(P)
    O.ann_destroy(Po)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_ann_oracle_vs_golden(oracles, path):
    O, R = oracles
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n = A.shape[0]
    a, b, rho = (float(x) for x in z["params"])
    Po = O.ann_plan(n, a, b, rho)
    so, co = O.ann_table(Po)
    assert np.abs(so - z["s"]).max() <= 2 * n * EPS and np.abs(co - z["c"]).max() <= 2 * n * EPS
    for fwd in (True, False):
        for tr in "NT":
            y = A.copy(order="F")
            O.ann_execute(Po, fwd, tr, y)
            assert rel2(y, z[("fwd" if fwd else "bwd") + "_" + tr]) <= 1e-14
    for d in ("hi2lo", "lo2hi"):
        y = A.copy(order="F")
        (O.ann_hi2lo if d == "hi2lo" else O.ann_lo2hi)(Po, y)
        assert rel2(y, z["rot_" + d]) <= 1e-15 * n
    O.ann_destroy(Po)


@pytest.mark.parametrize("n", [64, 128])
def test_ann_round_trips(oracles, n):
    """test/test_drivers.c:985-1020 (sweeps with rho = 0 and rho = sqrt(1/3)) and 1128-1150."""
    O, R = oracles
    from oracle.bind import fill
    A = fill("disk", n, 5)
    einf = lambda B: np.abs(B - A).max() / np.abs(A).max()
    for rho in (0.0, np.sqrt(1 / 3)):
        Po = O.ann_plan(n, 0.0, 0.0, rho, connections=False)
        B = A.copy(order="F")
        O.ann_hi2lo(Po, B)
        O.ann_lo2hi(Po, B)
        assert rel2(B, A) <= 6 * np.sqrt(n) * EPS and einf(B) <= 5 * n * EPS
        O.ann_destroy(Po)
    Po = O.ann_plan(n, 0.0, 0.0, np.sqrt(1 / 3))
    B = A.copy(order="F")
    for tr in "NT":
        O.ann_execute(Po, True, tr, B)
        O.ann_execute(Po, False, tr, B)
    assert rel2(B, A) <= 12 * np.sqrt(n) * EPS and einf(B) <= 6 * n * EPS
    O.ann_destroy(Po)
