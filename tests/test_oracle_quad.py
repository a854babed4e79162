"""The __float128 oracle (oracle/ft_quad.c): the rotation tables and default sweep kernels of the
reference (src/rotations.c:116-190, src/rotations/rotations_default.c:31-71) and the sph / disk
forward transform 'N' (src/drivers.c:833-840, 989-994) in quad precision, on selected columns.

Pinned here on the CPU:
  * its tables round to the double-precision oracle's tables (the reference's formulas) within
    one unit in the last place;
  * an independent evaluation with mpmath at 50 digits of the sph and disk sweeps at small n
    agrees with it to 1e-30;
  * the double-precision oracle's rotation stage and the compiled reference's transforms lie
    within their own rounding (a few 1e-16 .. 1e-15) of it.
The GPU's distance to it is checked in tests/test_gpu_parity_scale.py and reported by bench.py."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel2


@pytest.fixture(scope="module")
def Q():
    from oracle.bind import Quad
    return Quad()


FAMS = [("sph", ()), ("tri", (0.0, 0.0, 0.0)), ("tri", (0.5, 1.0, -0.25)), ("disk", (0.0, 0.0)), ("disk", (0.5, -0.25))]


@pytest.mark.parametrize("kind,params", FAMS)
def test_tables_round_to_the_double_tables(Q, kind, params):
    from oracle.bind import Oracle, _OraclePlan
    O = Oracle()
    n = 97
    P = O.plan(kind, n, *params, rotations_only=True)
    p = C.cast(P, C.POINTER(_OraclePlan)).contents
    cols = 2 * n - 1 if kind == "disk" else n
    size = n * n if kind == "disk" else n * (n + 1) // 2
    s = np.ctypeslib.as_array(p.s, shape=(size,))
    c = np.ctypeslib.as_array(p.c, shape=(size,))
    base = 0
    for j in range(cols):
        length = n - (j + 1) // 2 if kind == "disk" else n - j
        sh, sl, ch, cl = Q.table_column(kind, n, j, length, params)
        for d, h, lo in ((s[base:base + length], sh, sl), (c[base:base + length], ch, cl)):
            # |double - exact| <= one ulp (the reference's sqrt(num / den) rounds twice)
            err = np.abs((d - h) - lo)
            assert np.all(err <= np.spacing(np.abs(h)) * 1.0001), (kind, j)
        base += length
    O.destroy(P)


def _mp_sweeps(kind, A, hi2lo=True):
    import mpmath as mp
    mp.mp.dps = 50
    n, M = A.shape
    X = [[mp.mpf(float(A[i, j])) for j in range(M)] for i in range(n)]
    for col in range(M):
        m = (col + 1) // 2
        js = list(range(m - 2, m % 2 - 1, -2))
        if not hi2lo:
            js = js[::-1]
        for j in js:
            K = n - 3 - j if kind == "sph" else n - 2 - (j + 1) // 2
            d = 2 if kind == "sph" else 1
            ks = range(K, -1, -1) if hi2lo else range(0, K + 1)
            for k in ks:
                if kind == "sph":
                    nums, numc, den = (k + 1) * (k + 2), (2 * j + 2) * (2 * k + 2 * j + 5), (k + 2 * j + 3) * (k + 2 * j + 4)
                    s, c = mp.sqrt(mp.mpf(nums) / den), mp.sqrt(mp.mpf(numc) / den)
                else:   # disk, alpha = beta = 0
                    nums, numc, den = (k + 1) * (k + 1), (j + 1) * (2 * k + j + 3), (k + j + 2) * (k + j + 2)
                    s, c = -mp.sqrt(mp.mpf(nums) / den), mp.sqrt(mp.mpf(numc) / den)
                x, y = X[k][col], X[k + d][col]
                if hi2lo:
                    X[k][col], X[k + d][col] = c * x + s * y, c * y - s * x
                else:
                    X[k][col], X[k + d][col] = c * x - s * y, c * y + s * x
    return X


@pytest.mark.parametrize("kind", ["sph", "disk"])
def test_sweeps_against_mpmath(Q, kind):
    import mpmath as mp
    from oracle.bind import fill
    n = 12
    A = fill(kind, n, 5)
    for hi2lo in (True, False):
        X = _mp_sweeps(kind, A, hi2lo)
        hi, lo = Q.columns(kind, A, list(range(A.shape[1])), (0.0, 0.0) if kind == "disk" else (), hi2lo)
        worst = 0.0
        for i in range(n):
            for j in range(A.shape[1]):
                worst = max(worst, abs(float((mp.mpf(float(hi[i, j])) + mp.mpf(float(lo[i, j]))) - X[i][j])))
        assert worst < 1e-30, (kind, hi2lo, worst)


@pytest.mark.parametrize("kind,params", FAMS)
@pytest.mark.parametrize("n", [64, 129])
def test_double_oracle_sweeps_within_rounding(Q, kind, params, n):
    from oracle.bind import Oracle, fill
    O = Oracle()
    A = fill(kind, n, 11)
    P = O.plan(kind, n, *params, rotations_only=True)
    cols = list(range(A.shape[1]))
    for hi2lo in (True, False):
        for fused in (True, False):
            O.set_fused(fused)
            R = A.copy(order="F")
            (O.hi2lo if hi2lo else O.lo2hi)(P, R)
            hi, _ = Q.columns(kind, A, cols, params, hi2lo)
            assert rel2(R, hi) < 2e-15, (kind, n, hi2lo, fused, rel2(R, hi))
    O.destroy(P)


@pytest.mark.parametrize("kind,params", [("sph", ()), ("disk", (0.0, 0.0)), ("disk", (0.5, -0.25))])
def test_compiled_reference_transform_within_rounding(Q, kind, params):
    from oracle.bind import Reference, fill
    if not Reference.available():
        pytest.skip("reference library not built")
    R = Reference()
    n = 256
    A = fill(kind, n, 13)
    P = R.plan(kind, n, *params)
    Ps, _ = R.connection(P, n)
    F = A.copy(order="F")
    R.execute(kind, P, True, "N", F)
    R.destroy(P)
    cols = [0, 1, 2, 3, 4, 5, 6, 100, 101, 102, 103, 254, 255, 256, 257, A.shape[1] - 2, A.shape[1] - 1]
    hi, _ = Q.columns(kind, A, cols, params, True, (np.triu(Ps[0]), np.triu(Ps[1])))
    assert rel2(F[:, cols], hi) < 1e-14, rel2(F[:, cols], hi)
