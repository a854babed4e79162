"""CPU checks of two device designs, restated here in Python with the kernels' own index
formulas, against the oracle (these restatements are the specification the CUDA code follows;
the GPU tests then compare the kernels themselves with the oracle):

* the column wavefront of fasttransforms_b200/csrc/column.cu (the reference's ft_kernel_*,
  src/rotations/rotations_default.c:31-117): thread u of a chunk of consecutive sweeps applies
  rotation s - D u of its sweep at step s (D = 1 hi2lo, p + 1 lo2hi); every step's rotations touch
  disjoint entries and every entry sees its rotations in the sequential order, so the result is
  bit-identical to the sequential loops (checked here in the oracle's unfused mode, where Python's
  float arithmetic is the same);
* the spin grid sequence of fasttransforms_b200/csrc/grid.cu (run_spin, src/fftw.c:801-960): the
  split / merge index maps with the column permutation, the end-entry classes and the scalings
  around the theta stage on 2M real columns and the row DFT."""
import numpy as np
import pytest

SPH, TRI, DISK, SPIN, RECT = 0, 1, 2, 3, 4


def _cdiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b > 0) else -q


def _geo(kind):
    return (1 if kind in (TRI, DISK, SPIN) else 2), (1 if kind in (TRI, SPIN) else 2)


def _top(kind, n, j, d=0):
    if kind == TRI:
        return n - 2 - j
    if kind == DISK:
        return n - 2 - _cdiv(j + 1, 2)
    if kind == SPIN:
        return n - 2 - d - j
    return n - 3 - j


def _base(kind, n, j, d=0, a_s=0):
    if kind == SPIN:
        return j * n + d * a_s * n
    if kind == DISK:
        return j * n - _cdiv(j, 2) * _cdiv(j + 1, 2)
    return _cdiv(j * (2 * n + 1 - j), 2)


def _sweeps(kind, hi, m1, m2, n):
    st = _geo(kind)[1]
    cap = 2 * n + 4   # orders j >= 2n + 2 have no rotation: m2 brought below cap + st, residue kept
    if m2 > cap:
        m2 -= ((m2 - cap) // st) * st
    if hi:
        j0 = m2 - st
        return j0, (_cdiv(j0 - m1, st) + 1 if j0 >= m1 else 0)
    return m1, (_cdiv(m2 - 1 - m1, st) + 1 if m2 > m1 else 0)


def wavefront(col, s_tab, c_tab, kind, n, m1, m2, hi, fwd, B, d=0, a_s=0):
    """column_kernel<HI2LO> with blockDim.x = B on a real or complex column, unfused rotations."""
    col = col.copy()
    p, st = _geo(kind)
    D, sgn = (1, -1) if hi else (p + 1, 1)
    j0, T = _sweeps(kind, hi, m1, m2, n)
    for t0 in range(0, T, B):
        nb = min(B, T - t0)
        kmax = max(_top(kind, n, j0 + sgn * st * t0, d), _top(kind, n, j0 + sgn * st * (t0 + nb - 1), d))
        K = [_top(kind, n, j0 + sgn * st * (t0 + u), d) if u < nb else -1 for u in range(B)]
        base = [_base(kind, n, j0 + sgn * st * (t0 + u), d, a_s) if K[u] >= 0 else 0 for u in range(B)]
        for s in range(D * (nb - 1) + kmax + 1):
            touched, new = set(), {}
            for u in range(B):
                r = s - D * u
                if 0 <= r <= K[u]:
                    k = K[u] - r if hi else r
                    assert not ({k, k + p} & touched) and k + p < len(col)
                    touched |= {k, k + p}
                    sv, cv = s_tab[base[u] + k], c_tab[base[u] + k]
                    x, y = col[k], col[k + p]
                    new[k], new[k + p] = (cv * x + sv * y, cv * y - sv * x) if fwd else (cv * x - sv * y, cv * y + sv * x)
            for k, v in new.items():
                col[k] = v
    return col


@pytest.fixture(scope="module")
def O():
    from oracle.bind import Oracle
    o = Oracle()
    o.set_fused(False)
    yield o
    o.set_fused(True)


@pytest.mark.parametrize("name,kind,kw", [("sph", SPH, {}), ("tri", TRI, {"alpha": 0.0, "beta": -0.5, "gamma": 0.25}),
                                          ("disk", DISK, {"alpha": 0.5, "beta": -0.25}), ("rect", RECT, {"beta": 0.5})])
@pytest.mark.parametrize("n", [1, 3, 8, 13])
def test_column_wavefront_is_the_sequential_order(O, name, kind, kw, n):
    P = O.plan(name, n, rotations_only=True, **kw)
    s_tab, c_tab = O.tables(P)
    rng = np.random.default_rng(n + kind)
    mmax = 2 * n + 1 if kind == DISK else n + 2
    pairs = [(m1, m2) for m2 in range(mmax + 1) for m1 in range(m2 + 2)]
    pairs += [(m1, m2) for m2 in (10 * n + 7, 10 * n + 8) for m1 in (0, 1, n // 2, 3 * n)]   # m2 past the clamp
    for m1, m2 in pairs:
        col = rng.uniform(-1, 1, n)
        for hi in (True, False):
            want = O.kernel(P, hi, m1, m2, col.copy())
            for B in (1, 3, 32):
                got = wavefront(col, s_tab, c_tab, kind, n, m1, m2, hi, hi, B)
                assert np.array_equal(got, want), (name, n, m1, m2, hi, B)
    O.destroy(P)


@pytest.mark.parametrize("s", [-3, 0, 2])
def test_spin_column_stages_are_the_sequential_order(O, s):
    import ctypes as C

    class _SP(C.Structure):
        _fields_ = [("n", C.c_int), ("s", C.c_int), ("s2", C.POINTER(C.c_double)), ("c2", C.POINTER(C.c_double)), ("sph", C.c_void_p)]
    n, a_s = 9, abs(s)
    P = O.spin_plan(n, s, connections=False)
    sp = C.cast(P, C.POINTER(_SP)).contents
    s2 = np.ctypeslib.as_array(sp.s2, shape=(a_s * n * n,)) if a_s else np.zeros(1)
    c2 = np.ctypeslib.as_array(sp.c2, shape=(a_s * n * n,)) if a_s else np.zeros(1)
    Psph = O.plan("sph", n, rotations_only=True)   # the same sph table as the spin plan's
    s1, c1 = O.tables(Psph)
    rng = np.random.default_rng(a_s)
    for m in range(-(n + 1), n + 2):
        am = abs(m)
        d, mn, par = abs(am - a_s), min(am, a_s), (am + a_s) % 2
        col = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        for hi in (True, False):
            want = O.spin_kernel(P, hi, m, col)
            fwd1 = hi == (m * s >= 0)
            st1 = lambda c: wavefront(c, s2, c2, SPIN, n, 0, mn, hi, fwd1, 4, d, a_s)
            st2 = lambda c: wavefront(c, s1, c1, SPH, n, par, d, hi, hi, 4)
            got = st2(st1(col)) if hi else st1(st2(col))
            assert np.array_equal(got, want), (s, m, hi)
    O.destroy(Psph)
    O.spin_destroy(P)


def _spin_src(c, M, perm):
    if perm == 0 or c == 0:
        return c
    if perm == 1:
        return M - (c + 1) // 2 if c & 1 else c // 2
    return 2 * c if c <= (M - 1) // 2 else 2 * (M - c) - 1


def _split(X, perm, s, row, cls, f):
    N, M = X.shape
    W = np.empty((N, 2 * M))
    for c in range(M):
        v = X[:, _spin_src(c, M, perm)] * s
        re, im = v.real.copy(), v.imag.copy()
        if row >= 0 and (1 if (c & 3) in (1, 2) else 0) == cls:
            re[row] *= f
            im[row] *= f
        W[:, 2 * c], W[:, 2 * c + 1] = re, im
    return W


def _merge(W, perm, s, row, cls, f):
    N, M = W.shape[0], W.shape[1] // 2
    X = np.empty((N, M), complex)
    for c in range(M):
        q = _spin_src(c, M, perm)
        re, im = W[:, 2 * q] * s, W[:, 2 * q + 1] * s
        if row >= 0 and (1 if (c & 3) in (1, 2) else 0) == cls:
            re[row] *= f
            im[row] *= f
        X[:, c] = re + 1j * im
    return X


def test_spin_grid_sequence_is_the_reference_sequence():
    from oracle import grid as G
    c12, c2 = 0.199471140200716338, 5.013256549262001005

    def theta(W, kinds):
        out = np.empty_like(W)
        for j in range(W.shape[1]):
            k = kinds[0] if ((j >> 1) & 3) in (0, 3) else kinds[1]
            out[:, j] = G.theta(W[:, j:j + 1], (k, k))[:, 0]
        return out

    def run_spin(op, T, plan_op, S, X):
        N, M = X.shape
        if T not in "NC":
            return X.copy()
        kinds, sign = G.spin_plan_kinds(plan_op, S)
        dft = (lambda Y: np.fft.ifft(Y, axis=1) * M) if sign > 0 else (lambda Y: np.fft.fft(Y, axis=1))
        first = 0 if S % 2 == 0 else 1
        last, sa = 1 - first, c2 / (2.0 * N * M)
        if op == "spinsph_synthesis":
            if T == "N":
                return dft(_merge(theta(_split(X, 0, 1.0, 0, first, 2.0), kinds), 2, c12, -1, 0, 1.0))
            return _merge(theta(_split(dft(X), 1, c12, -1, 0, 1.0), kinds), 0, 1.0, N - 1, last, 0.5)
        if T == "N":
            return _merge(theta(_split(dft(X), 1, sa, -1, 0, 1.0), kinds), 0, 1.0, 0, first, 0.5)
        return dft(_merge(theta(_split(X, 0, 1.0, N - 1, last, 2.0), kinds), 2, sa, -1, 0, 1.0))

    rng = np.random.default_rng(1)
    for N, M in [(1, 1), (2, 3), (5, 9), (7, 13), (6, 5)]:
        for S in (-3, 0, 1, 2):
            X = rng.standard_normal((N, M)) + 1j * rng.standard_normal((N, M))
            for op in ("spinsph_synthesis", "spinsph_analysis"):
                for plan_op in ("spinsph_synthesis", "spinsph_analysis"):
                    for T in "NCT":
                        got = run_spin(op, T, plan_op, S, X)
                        want = G.execute_spinsph(op, T, plan_op, S, X)
                        assert np.abs(got - want).max() <= 1e-14 * max(np.abs(want).max(), 1.0), (N, M, S, op, plan_op, T)
