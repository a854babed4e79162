"""CPU restatement of the connection multiply's 8-bit integer form (fasttransforms_b200/csrc/
trmm_mixed.cu: digits16 / slice_matrix_s8_kernel / column_scale_kernel / slice_input_s8_kernel /
trmm_s8_kernel), checking its arithmetic claims with numpy:

* a row (column) scaled by the power of two that puts its largest entry below 64 cuts into
  balanced base-2^7 digits that all lie in [-64, 64] (one signed byte each) and rebuild the scaled
  value within half a unit of the last digit;
* the level sums of the digit products (levels a + b <= 4) are integers bounded by
  5 * 64 * 64 * K, so 32-bit accumulation is exact for K below 104 857;
* recombining the five level sums in FP64 and scaling back gives op(U) x within the digits'
  truncation, half a unit of the last digit of each row's and column's scale (about 2^-27 of a
  column's largest entry with four input digits, 2^-34 with five), well inside the multiply's
  share of the mixed forms' error budget."""
import numpy as np
import pytest


def scale_pow2(amax):
    """Power of two s with amax * s < 64 (1 for a zero row)."""
    if amax == 0:
        return 1.0
    ex = np.frexp(amax)[1]          # amax < 2^ex
    return 2.0 ** (6 - ex)


def digits(t, nd):
    """Balanced base-2^7 digits of t (|t| < 64), the kernels' rint / subtract / * 128 sequence."""
    out = np.zeros(t.shape + (nd,), dtype=np.int64)
    r = t.astype(np.float64).copy()
    for k in range(nd):
        i = np.rint(r)
        out[..., k] = i.astype(np.int64)
        r = (r - i) * 128.0
    return out


def recombine(levels):
    """FP64 recombination of the level sums, highest level first (the epilogue's fma chain)."""
    y = levels[-1].astype(np.float64)
    for lv in range(len(levels) - 2, -1, -1):
        y = y * 0.0078125 + levels[lv].astype(np.float64)
    return y


def s8_multiply(U, X, nu=5, nx=4, lmax=4):
    """Out = U X by the integer form: rows of U and columns of X scaled and cut into digits,
    products of levels a + b <= lmax summed exactly (int64 here, checked against the int32
    bound), recombined in FP64 and scaled back."""
    su = np.array([scale_pow2(np.abs(r).max()) for r in U])
    sx = np.array([scale_pow2(np.abs(c).max()) for c in X.T])
    du = digits(U * su[:, None], nu)            # rows x K x nu
    dx = digits(X * sx[None, :], nx)            # K x cols x nx
    assert du.min() >= -64 and du.max() <= 64 and dx.min() >= -64 and dx.max() <= 64
    levels = []
    for lv in range(lmax + 1):
        acc = np.zeros((U.shape[0], X.shape[1]), dtype=np.int64)
        for b in range(max(0, lv - (nx - 1)), min(lv, nu - 1) + 1):
            a = lv - b
            acc += du[:, :, b] @ dx[:, :, a]
        assert np.abs(acc).max() < 2 ** 31
        levels.append(acc)
    return recombine(levels) / su[:, None] / sx[None, :]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_digits_range_and_reconstruction(seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(4000) * 2.0 ** rng.integers(-40, 10, 4000)
    for v in x:
        t = np.array([v * scale_pow2(abs(v) * rng.uniform(1, 8))])
        assert abs(t[0]) < 64
        for nd in (4, 5):
            d = digits(t, nd)[0]
            assert d.min() >= -64 and d.max() <= 64
            rec = sum(int(d[k]) * 2.0 ** (-7 * k) for k in range(nd))
            assert abs(rec - t[0]) <= 0.5 * 2.0 ** (-7 * (nd - 1)) * (1 + 1e-12)


def test_int32_bound():
    # the worst level sum: 5 products of 64 x 64 per row of K
    kmax = (2 ** 31 - 1) // (5 * 64 * 64)
    assert kmax == 104857


# relative 2-norm bounds: four input digits leave the inputs' 2^-27 truncation, five leave the
# dropped levels (a + b >= 5, four products at 2^-35) of the same order as their 2^-34 truncation
@pytest.mark.parametrize("nx,bound", [(4, 2.0 ** -25), (5, 2.0 ** -29)])
def test_upper_triangular_multiply(nx, bound):
    rng = np.random.default_rng(7)
    n, m = 96, 40
    U = np.triu(rng.standard_normal((n, n)) / np.sqrt(np.arange(1, n + 1))[None, :])
    X = rng.standard_normal((n, m)) * np.exp(-np.arange(n) / 30.0)[:, None]   # decaying coefficients
    got = s8_multiply(U, X, nu=5, nx=nx)
    ref = U @ X
    # a digit cut leaves at most half a unit of the last digit of the scaled value, i.e. 2^(-7(nd-1)-6)
    # of the row's (column's) largest entry; the dropped levels (a + b >= 5) are far below that
    colmax, rowmax = np.abs(X).max(0), np.abs(U).max(1)
    elem = 1.01 * (np.abs(U).sum(1)[:, None] * colmax[None, :] * 2.0 ** (-7 * (nx - 1) - 6)
                   + rowmax[:, None] * np.abs(X).sum(0)[None, :] * 2.0 ** (-7 * 4 - 6)
                   + np.abs(U).sum(1)[:, None] * colmax[None, :] * 2.0 ** -35)
    assert np.all(np.abs(got - ref) <= elem)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= bound
