"""Oracle (test infrastructure, not the product): a CPU restatement of the
sphere, disk and triangle grid synthesis and analysis of the reference
(src/fftw.c:63-753: ft_plan_sph_with_kind, ft_execute_sph_synthesis / _analysis and the
sphv variants, ft_execute_disk_*, ft_execute_tri_*, ft_execute_tet_*, ft_execute_annulus_*,
ft_execute_rectdisk_* and ft_execute_spinsph_*; src/fftw.c:755-960) in numpy / scipy.

FFTW, which the reference calls for these transforms, is not available here, so
its one-dimensional transforms are restated from their published definitions
(FFTW manual, "What FFTW Really Computes"), all unnormalised:
  REDFT10 (DCT-II)  y_k = 2 sum_j x_j cos(pi (j + 1/2) k / N)
  REDFT01 (DCT-III) y_k = x_0 + 2 sum_{j>=1} x_j cos(pi j (k + 1/2) / N)
  RODFT10 (DST-II)  y_k = 2 sum_j x_j sin(pi (j + 1/2) (k + 1) / N)
  RODFT01 (DST-III) y_k = (-1)^k x_{N-1} + 2 sum_{j<N-1} x_j sin(pi (j + 1) (k + 1/2) / N)
  REDFT11 (DCT-IV)  y_k = 2 sum_j x_j cos(pi (j + 1/2) (k + 1/2) / N)
  c2r of length M   x_k = sum over the Hermitian-completed spectrum of Y_j e^{2 pi i jk / M}
  r2c of length M   Y_j = sum_k x_k e^{-2 pi i jk / M}
which scipy.fft's dct / dst of types 2 and 3 (norm=None) and numpy's rfft /
irfft (times M) compute.  tests/test_oracle_grid.py checks those identities
against the explicit sums, and pins the sequences and scalings through the
reference's own test (src/fftw.c round trip with the compiled reference's
sph2fourier / fourier2sph, test/test_fftw.c:43-73) and known harmonics.
"""
import numpy as np
import scipy.fft as sf

REDFT01, REDFT10, RODFT01, RODFT10, REDFT11 = "REDFT01", "REDFT10", "RODFT01", "RODFT10", "REDFT11"

# plan kinds (classes {0, 3}, classes {1, 2}): src/fftw.c:104-122
PLANS = {
    "sph_synthesis": (REDFT01, RODFT01),
    "sph_analysis": (REDFT10, RODFT10),
    "sphv_synthesis": (RODFT01, REDFT01),
    "sphv_analysis": (RODFT10, REDFT10),
}
# disk plan kinds (classes {0, 3}, classes {1, 2}): src/fftw.c:450-458
DISK_PLANS = {"disk_synthesis": (REDFT01, REDFT11), "disk_analysis": (REDFT10, REDFT11)}
# triangle plan kinds (both dimensions): src/fftw.c:289-290
TRI_PLANS = {"tri_synthesis": REDFT01, "tri_analysis": REDFT10}

# src/ftinternal.h:48-56
M_1_4_SQRT_PI = 0.141047395886939072
M_1_2_SQRT_PI = 0.282094791773878143
M_4_SQRT_PI = 7.089815403622064109
M_2_SQRT_PI = 3.544907701811032055
M_SQRT2 = 1.41421356237309504880
M_SQRT1_2 = 0.70710678118654752440


def r2r(x, kind):
    """FFTW's 1-d real transform `kind` down the columns of x (axis 0)."""
    if kind == REDFT10:
        return sf.dct(x, type=2, axis=0)
    if kind == REDFT01:
        return sf.dct(x, type=3, axis=0)
    if kind == RODFT10:
        return sf.dst(x, type=2, axis=0)
    if kind == RODFT01:
        return sf.dst(x, type=3, axis=0)
    if kind == REDFT11:
        return sf.dct(x, type=4, axis=0)
    raise ValueError(kind)


def theta(X, kinds):
    """plantheta1 .. 4 (src/fftw.c:85-95): column classes j mod 4 = 0, 3 take
    kinds[0], classes 1, 2 take kinds[1]."""
    Y = X.copy()
    for r, k in ((0, kinds[0]), (1, kinds[1]), (2, kinds[1]), (3, kinds[0])):
        if Y[:, r::4].shape[1]:
            Y[:, r::4] = r2r(X[:, r::4], k)
    return Y


def data_r2c(X):
    """src/fftw.c:40-49: column 0 -> frequency 0, (2j, 2j - 1) -> Re, -Im of frequency j."""
    N, M = X.shape
    Y = np.zeros((N, M // 2 + 1), dtype=complex)
    Y[:, 0] = X[:, 0]
    for j in range(1, M // 2 + 1):
        Y[:, j] = X[:, 2 * j] - 1j * X[:, 2 * j - 1]
    return Y


def data_c2r(Y, M):
    """src/fftw.c:51-60."""
    N = Y.shape[0]
    X = np.zeros((N, M))
    X[:, 0] = Y[:, 0].real
    for j in range(1, M // 2 + 1):
        X[:, 2 * j] = Y[:, j].real
        X[:, 2 * j - 1] = -Y[:, j].imag
    return X


def c2r(Y, M):
    return np.fft.irfft(Y, n=M, axis=1) * M


def r2c(X):
    return np.fft.rfft(X, axis=1)


def _ends(X, first, sph, f):
    """The end-entry factors of the sequences: first entries of columns
    {0, 3, 4, 7, 8, ..} (sph) or {1, 2, 5, 6, ..} (sphv); last entries of
    {1, 2, 5, 6, ..} (sph) or {0, 3, 4, 7, 8, ..} (sphv)."""
    N, M = X.shape
    row = 0 if first else N - 1
    if first == sph:
        cols = [0] + [c for j in range(3, M, 4) for c in (j, j + 1) if c < M]
    else:
        cols = [c for j in range(1, M, 4) for c in (j, j + 1) if c < M]
    for c in cols:
        X[row, c] *= f


def execute(op, trans, plan, X):
    """ft_execute_{sph,sphv}_{synthesis,analysis}(trans, P, X) with P a plan of
    kind `plan` (a key of PLANS).  op: "sph_synthesis", "sph_analysis",
    "sphv_synthesis", "sphv_analysis".  Returns the new X (N x M, column-major
    meaning: X[i, j] is row i, column j)."""
    X = np.array(X, dtype=float, copy=True)
    N, M = X.shape
    kinds = PLANS[plan]
    sph = op.startswith("sph_")
    nm2 = 2.0 * N * M
    if op.endswith("synthesis"):
        if trans == "N":                                # src/fftw.c:124-146, 202-219
            _ends(X, True, sph, 2.0)
            X = theta(X, kinds)
            X *= M_1_4_SQRT_PI
            X[:, 0] *= M_SQRT2
            return c2r(data_r2c(X), M)
        X = data_c2r(r2c(X), M)                         # :147-164, 220-237
        X *= M_1_2_SQRT_PI
        X[:, 0] *= M_SQRT1_2
        X = theta(X, kinds)
        _ends(X, False, sph, 0.5)
        return X
    if trans == "N":                                    # :166-183, 239-256
        X = data_c2r(r2c(X), M)
        X *= M_4_SQRT_PI / nm2
        X[:, 0] *= M_SQRT1_2
        X = theta(X, kinds)
        _ends(X, True, sph, 0.5)
        return X
    _ends(X, False, sph, 2.0)                           # :184-199, 257-276
    X = theta(X, kinds)
    X *= M_2_SQRT_PI / nm2
    X[:, 0] *= M_SQRT2
    return c2r(data_r2c(X), M)


def grid(N, M):
    """The points: theta_i = (i + 1/2) pi / N, phi_k = 2 pi k / M."""
    return (np.arange(N) + 0.5) * np.pi / N, 2 * np.pi * np.arange(M) / M


def execute_disk(op, trans, plan, X):
    """ft_execute_disk_{synthesis,analysis}(trans, P, X) with P a plan of kind `plan` (a key of
    DISK_PLANS), src/fftw.c:460-532: the sph sequences with the disk's kinds (classes 1, 2 a
    DCT-IV) and only the first-entry factors of columns {0, 3, 4, 7, 8, ..}."""
    X = np.array(X, dtype=float, copy=True)
    N, M = X.shape
    kinds = DISK_PLANS[plan]
    nm2 = 2.0 * N * M
    if op == "disk_synthesis":
        if trans == "N":
            _ends(X, True, True, 2.0)
            X = theta(X, kinds)
            X *= M_1_4_SQRT_PI
            X[:, 0] *= M_SQRT2
            return c2r(data_r2c(X), M)
        X = data_c2r(r2c(X), M)
        X *= M_1_2_SQRT_PI
        X[:, 0] *= M_SQRT1_2
        return theta(X, kinds)
    if trans == "N":
        X = data_c2r(r2c(X), M)
        X *= M_4_SQRT_PI / nm2
        X[:, 0] *= M_SQRT1_2
        X = theta(X, kinds)
        _ends(X, True, True, 0.5)
        return X
    X = theta(X, kinds)
    X *= M_2_SQRT_PI / nm2
    X[:, 0] *= M_SQRT2
    return c2r(data_r2c(X), M)


def _r2r_2d(X, kind):
    return r2r(r2r(X, kind).T, kind).T


def execute_tri(op, trans, plan, X):
    """ft_execute_tri_{synthesis,analysis}(trans, P, X), src/fftw.c:292-330: a 2-D transform of
    the plan's kind along both dimensions (N = M; nothing happens unless N, M > 1), with the
    first row and column factors and the 1/4 or 1/(N M) scalings."""
    X = np.array(X, dtype=float, copy=True)
    N, M = X.shape
    if N <= 1 or M <= 1:
        return X
    kind = TRI_PLANS[plan]
    if op == "tri_synthesis":
        if trans == "N":
            X[:, 0] *= 2.0
            X[0, :] *= 2.0
        X *= 0.25
        return _r2r_2d(X, kind)
    if trans == "N":
        X = _r2r_2d(X, kind)
        X[:, 0] *= 0.5
        X[0, :] *= 0.5
        return X / (N * M)
    return _r2r_2d(X / (N * M), kind)


# annulus plan kinds (all columns): src/fftw.c:573-581
ANN_PLANS = {"annulus_synthesis": REDFT01, "annulus_analysis": REDFT10}
# rectdisk plan kinds (even columns, odd columns, rows): src/fftw.c:687-695
RECT_PLANS = {"rectdisk_synthesis": (REDFT01, RODFT01, REDFT01), "rectdisk_analysis": (REDFT10, RODFT10, REDFT10)}


def annulus_weights(N, rho):
    """src/fftw.c:545-551: w_n = sqrt(2 (sin^2 t + rho^2 cos^2 t) / (1 - rho^2)), t = (N - n - 1/2) pi / 2N."""
    w = np.empty(N)
    for n in range(N):
        t = (N - n - 0.5) * np.pi / (2.0 * N)
        ct, st = np.sin(t), np.cos(t)
        w[n] = np.sqrt(2.0 * (ct * ct + rho * rho * st * st) / (1.0 - rho * rho))
    return w


def _ann_cols(M):
    return [c for j in range(1, M, 4) for c in (j, j + 1) if c < M]


def execute_annulus(op, trans, plan, X, rho):
    """ft_execute_annulus_{synthesis,analysis}(trans, P, X) with P a plan of kind `plan` (a key of
    ANN_PLANS) and radius ratio rho, src/fftw.c:583-658: the plan's cosine transform on every
    column, the columns of classes 1 and 2 weighted by w (divided in analysis), the sph phi stage
    and scalings, and the first-row factors."""
    X = np.array(X, dtype=float, copy=True)
    N, M = X.shape
    kind = ANN_PLANS[plan]
    w = annulus_weights(N, rho)[:, None]
    cols = _ann_cols(M)
    nm2 = 2.0 * N * M
    if op == "annulus_synthesis":
        if trans == "N":
            X[0, :] *= 2.0
            X = r2r(X, kind)
            X[:, cols] *= w
            X *= M_1_4_SQRT_PI
            X[:, 0] *= M_SQRT2
            return c2r(data_r2c(X), M)
        X = data_c2r(r2c(X), M)
        X *= M_1_2_SQRT_PI
        X[:, 0] *= M_SQRT1_2
        X[:, cols] *= w
        return r2r(X, kind)
    if trans == "N":
        X = data_c2r(r2c(X), M)
        X *= M_4_SQRT_PI / nm2
        X[:, 0] *= M_SQRT1_2
        X[:, cols] /= w
        X = r2r(X, kind)
        X[0, :] *= 0.5
        return X
    X = r2r(X, kind)
    X[:, cols] /= w
    X *= M_2_SQRT_PI / nm2
    X[:, 0] *= M_SQRT2
    return c2r(data_r2c(X), M)


def _rect_x(X, kinds):
    Y = X.copy()
    if Y[:, 0::2].shape[1]:
        Y[:, 0::2] = r2r(X[:, 0::2], kinds[0])
    if Y[:, 1::2].shape[1]:
        Y[:, 1::2] = r2r(X[:, 1::2], kinds[1])
    return Y


def _rect_y(X, kind):
    return r2r(X.T, kind).T


def execute_rectdisk(op, trans, plan, X):
    """ft_execute_rectdisk_{synthesis,analysis}(trans, P, X), src/fftw.c:697-753: the plan's first
    kind down the even columns and its second down the odd ones, its third along the rows, with
    the reference's end-entry factors and scalings."""
    X = np.array(X, dtype=float, copy=True)
    N, M = X.shape
    kinds = RECT_PLANS[plan]
    if op == "rectdisk_synthesis":
        if trans == "N":
            X[0, 0::2] *= 2.0
            X = _rect_x(X, kinds)
            X[:, 0] *= 2.0
            X *= 0.25
            return _rect_y(X, kinds[2])
        X = _rect_y(X, kinds[2])
        X *= 0.25
        X = _rect_x(X, kinds)
        X[N - 1, 1::2] *= 0.5
        return X
    if trans == "N":
        X = _rect_y(X, kinds[2])
        X /= N * M
        X[:, 0] *= 0.5
        X = _rect_x(X, kinds)
        X[0, 0::2] *= 0.5
        return X
    X[N - 1, 1::2] *= 2.0
    X = _rect_x(X, kinds)
    X = _rect_y(X, kinds[2])
    return X / (N * M)


# tetrahedron plan kinds (all three dimensions): src/fftw.c:348-349
TET_PLANS = {"tet_synthesis": REDFT01, "tet_analysis": REDFT10}


def _r2r_3d(X, kind):
    Y = r2r(X, kind)                                   # axis 0
    Y = np.moveaxis(r2r(np.moveaxis(Y, 1, 0), kind), 0, 1)
    return np.moveaxis(r2r(np.moveaxis(Y, 2, 0), kind), 0, 2)


def execute_tet(op, trans, plan, X):
    """ft_execute_tet_{synthesis,analysis}(trans, P, X), src/fftw.c:351-402: the plan's kind along
    all three dimensions of the N x L x M tensor (N = L = M; nothing happens unless all exceed 1),
    with the factors of the faces m = 0, i = 0, l = 0 and the 1/8 or 1/(N L M) scalings."""
    X = np.array(X, dtype=float, copy=True)
    N, L, M = X.shape
    if N <= 1 or L <= 1 or M <= 1:
        return X
    kind = TET_PLANS[plan]
    if op == "tet_synthesis":
        if trans == "N":
            X[:, :, 0] *= 2.0
            X[0, :, :] *= 2.0
            X[:, 0, :] *= 2.0
            X *= 0.125
            return _r2r_3d(X, kind)
        return _r2r_3d(X, kind) * 0.125
    if trans == "N":
        X = _r2r_3d(X, kind)
        X[:, :, 0] *= 0.5
        X[0, :, :] *= 0.5
        X[:, 0, :] *= 0.5
        return X / (N * L * M)
    return _r2r_3d(X / (N * L * M), kind)


# src/ftinternal.h:53-54
M_2_SQRT_2PI = 5.013256549262001005
M_1_2_SQRT_2PI = 0.199471140200716338


def spin_plan_kinds(op, s):
    """src/fftw.c:789-799: the (classes {0, 3}, classes {1, 2}) kinds of a spin plan, and the sign
    of its row DFT (+1: FFTW_BACKWARD, synthesis; -1: FFTW_FORWARD, analysis)."""
    if op == "spinsph_synthesis":
        return ((REDFT01, RODFT01) if s % 2 == 0 else (RODFT01, REDFT01)), +1
    return ((REDFT10, RODFT10) if s % 2 == 0 else (RODFT10, REDFT10)), -1


def _colswap(X):
    """src/fftw.c:6-21: column 0 stays, column 2j goes to j and column 2j - 1 to M - j."""
    N, M = X.shape
    Y = np.empty_like(X)
    Y[:, 0] = X[:, 0]
    for j in range(1, (M + 1) // 2):
        Y[:, j] = X[:, 2 * j]
        Y[:, M - j] = X[:, 2 * j - 1]
    return Y


def _colswap_t(Y):
    """src/fftw.c:23-38, the inverse permutation."""
    N, M = Y.shape
    X = np.empty_like(Y)
    X[:, 0] = Y[:, 0]
    for j in range(1, (M + 1) // 2):
        X[:, 2 * j] = Y[:, j]
        X[:, 2 * j - 1] = Y[:, M - j]
    return X


def _row_dft(X, sign):
    """FFTW's unnormalised DFT along the rows with exp(sign 2 pi i j k / M)."""
    M = X.shape[1]
    return np.fft.ifft(X, axis=1) * M if sign > 0 else np.fft.fft(X, axis=1)


def _spin_theta(X, kinds):
    return theta(X.real, kinds) + 1j * theta(X.imag, kinds)


def _spin_ends(X, row, even_set, f):
    """Entries of `row` in the columns {0, 3, 4, 7, 8, ..} (even_set) or {1, 2, 5, 6, ..}, both parts."""
    N, M = X.shape
    if even_set:
        cols = [0] + [c for j in range(3, M, 4) for c in (j, j + 1) if c < M]
    else:
        cols = [c for j in range(1, M, 4) for c in (j, j + 1) if c < M]
    X[row, cols] *= f


def execute_spinsph(op, trans, plan_op, s_plan, X):
    """ft_execute_spinsph_{synthesis,analysis}(trans, P, X) with P the plan of `plan_op` and spin
    s_plan (its kinds, sign and spin), src/fftw.c:801-960.  X: complex N x M.  The reference's
    routines act for TRANS 'N' and 'C' only; any other character leaves X untouched."""
    X = np.array(X, dtype=complex, copy=True)
    N, M = X.shape
    if trans not in ("N", "C"):
        return X
    kinds, sign = spin_plan_kinds(plan_op, s_plan)
    even = s_plan % 2 == 0
    nm2 = 2.0 * N * M
    if op == "spinsph_synthesis":
        if trans == "N":
            _spin_ends(X, 0, even, 2.0)
            X = _spin_theta(X, kinds) * M_1_2_SQRT_2PI
            return _row_dft(_colswap(X), sign)
        X = _colswap_t(_row_dft(X, sign)) * M_1_2_SQRT_2PI
        X = _spin_theta(X, kinds)
        _spin_ends(X, N - 1, not even, 0.5)
        return X
    if trans == "N":
        X = _colswap_t(_row_dft(X, sign)) * (M_2_SQRT_2PI / nm2)
        X = _spin_theta(X, kinds)
        _spin_ends(X, 0, even, 0.5)
        return X
    _spin_ends(X, N - 1, not even, 2.0)
    X = _spin_theta(X, kinds) * (M_2_SQRT_2PI / nm2)
    return _row_dft(_colswap(X), sign)
