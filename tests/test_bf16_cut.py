"""CPU restatement of the blocked tensor-core sweeps' arithmetic (fasttransforms_b200/csrc/blocked.cu:
slice_scale, slice8, build_img_kernel, the level products and the recombination), checking its
claims with numpy:

* the window's scale puts every entry below 2^8, and each cut (one FMA that scales and adds
  1.5 * 2^23, one subtraction from 1.5 * 2^23) gives minus the nearest integer exactly, with the
  residual FMA exact and at most 1/2: the slices are integers |i| <= 256, which BF16 holds exactly,
  and the negated form gives the same residuals as rounding, subtracting and scaling in turn;
* the tile images' slices of 256 q are integers |j| <= 256 as well, stored negated, so every
  product (-i_a)(-j_b) is i_a j_b;
* a level's sum over the 64 positions of a window stays within 2^24, so FP32 accumulation is
  exact whatever order the tensor core adds in, and recombining the levels gives Q x to the
  slices' truncation.

Every multiplication in the cut is by a power of two (the scale, 512), so float32 numpy
operations reproduce the kernel's instructions bit for bit: a product is exact and the one
rounding is that of the addition or subtraction."""
import numpy as np
import pytest

MAGIC = np.float32(12582912.0)          # 1.5 * 2^23
WIN = 64


def slice_scale(amax):
    """2^(8 - (E - 126)) for the biased exponent E of amax (E >= 8), as a float32."""
    E = int((np.float32(amax).view(np.uint32) >> 23) & 0xFF)
    E = max(E, 8)
    return np.float32(2.0 ** (134 - E))


def cut(v, s, ns):
    """The kernel's cut of float32 values v at scale s: the stored (negated) slices and the
    residuals, each checked against the former positive form's on the way."""
    v = np.asarray(v, dtype=np.float32)
    t, m = v.copy(), np.float32(s)
    stored, resid_neg = [], []
    for a in range(ns):
        u = (t * m) + MAGIC                      # fma(t, m, magic): t * m is exact
        neg_i = MAGIC - u                        # -i_a, exact
        i = u - MAGIC                            # the former form's i_a
        assert np.array_equal(neg_i, -i)
        stored.append(neg_i)
        if a + 1 < ns:
            r_neg = (t * m) + neg_i              # fma(t, m, -i_a) as the kernel issues it
            r_pos = (t * m) - i
            assert np.array_equal(r_neg, r_pos)
            resid_neg.append(r_neg)
            t, m = r_neg, np.float32(512.0)
    return stored, resid_neg


def tile_slices(q, ns):
    """build_img_kernel: 256 q cut into ns integers (FP64), stored negated (a zero as +0)."""
    t = q.astype(np.float64) * 256.0
    out = []
    for _ in range(ns):
        j = np.rint(t)
        out.append(np.where(j == 0.0, 0.0, -j))
        t = (t - j) * 512.0
    return out


def bf16_exact(x):
    """x (float32) has at most 8 significant bits: its low 16 bits are zero."""
    return np.all((np.asarray(x, dtype=np.float32).view(np.uint32) & 0xFFFF) == 0)


def random_orthogonal(rng, n):
    qm, r = np.linalg.qr(rng.standard_normal((n, n)))
    return qm * np.sign(np.diag(r))[None, :]


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
@pytest.mark.parametrize("ns", [3, 4])
def test_window_cut(seed, ns):
    rng = np.random.default_rng(seed)
    for _ in range(200):
        v = (rng.standard_normal(WIN) * 2.0 ** rng.integers(-60, 30)).astype(np.float32)
        v[rng.integers(0, WIN, 5)] = 0.0
        s = slice_scale(np.abs(v).max())
        assert np.all(np.abs(v.astype(np.float64) * s) < 256.0)
        stored, resid = cut(v, s, ns)
        for a, sl in enumerate(stored):
            assert np.all(sl == np.rint(sl)) and np.abs(sl).max() <= 256.0, a
            assert bf16_exact(sl)
        for r in resid:
            assert np.abs(r).max() <= 0.5
        # -sum_a stored_a 2^(-9a) is s v to within half a unit of the last slice
        rec = -sum(sl.astype(np.float64) * 2.0 ** (-9 * a) for a, sl in enumerate(stored))
        assert np.abs(rec - v.astype(np.float64) * s).max() <= 0.5 * 2.0 ** (-9 * (ns - 1)) * (1 + 1e-12)


@pytest.mark.parametrize("ns,lv", [(3, 3), (4, 3)])
def test_levels_exact_and_tile_product(ns, lv):
    rng = np.random.default_rng(11)
    Q = random_orthogonal(rng, WIN)              # a tile: an orthogonal 64 x 64 matrix, |q| <= 1
    J = tile_slices(Q, ns)
    for b, jb in enumerate(J):
        assert np.all(np.abs(jb) <= 256.0) and bf16_exact(jb.astype(np.float32))
    worst = 0.0
    for _ in range(50):
        x = (rng.standard_normal(WIN) * np.exp(rng.uniform(-8, 8, WIN))).astype(np.float32)
        s = slice_scale(np.abs(x).max())
        I, _ = cut(x, s, ns)
        # products of levels 0 .. lv, one accumulator per level, over the window's positions
        levels = []
        for L in range(lv + 1):
            acc = np.zeros(WIN)
            for b in range(max(0, L - (ns - 1)), min(L, ns - 1) + 1):
                a = L - b
                acc += J[b] @ I[a].astype(np.float64)   # (-j_b)(-i_a) = i_a j_b, exact integers
            assert np.all(acc == np.rint(acc)) and np.abs(acc).max() <= 2.0 ** 24
            levels.append(acc)
        # every partial sum is an integer within 2^24 too: FP32 adds them exactly in any order
        y = levels[-1]
        for L in range(lv - 1, -1, -1):
            y = y * 2.0 ** -9 + levels[L]
        got = y * (2.0 ** -8 / float(s))
        ref = Q @ x.astype(np.float64)
        err = np.abs(got - ref).max() / np.abs(x).max()
        worst = max(worst, err)
    # bounds relative to the window's largest entry, summed over its 64 positions: the window's
    # and the tile's truncations (half a unit of the last slice) and, with four slices, the
    # products of levels 4 .. 6 left out (measured: 3.7e-8 and 4.4e-10)
    assert worst <= (64 * 2.0 ** -26 if ns == 3 else 64 * 2.0 ** -33), worst
