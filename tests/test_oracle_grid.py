"""Pins the grid oracle (oracle/grid.py, a restatement of src/fftw.c:63-330, 404-532: the
sphere's, the disk's and the triangle's grids; FFTW is not available here).  CPU only.

1. The one-dimensional transforms equal FFTW's published definitions (explicit
   sums) for every kind the plans use.
2. The reference's own accuracy test (test/test_fftw.c:43-73): the compiled
   reference's sph2fourier, the oracle's synthesis and analysis, the compiled
   reference's fourier2sph, in 'N' then 'T' (with the plans crossed, as there),
   return the input within 4 sqrt(N) eps (2-norm) and 2N eps (max norm).
3. Known harmonics: the reference's sph2fourier of a unit coefficient followed
   by the oracle's synthesis gives the real orthonormal spherical harmonic on the
   grid (Y_0^0, Y_1^0, and order 1 in columns 1 (sin phi) and 2 (cos phi))."""
import numpy as np
import pytest

from conftest import EPS
from oracle import grid as G


def explicit(x, kind):
    N = x.shape[0]
    k = np.arange(N)[:, None]
    j = np.arange(N)[None, :]
    if kind == G.REDFT10:
        A = 2 * np.cos(np.pi * (j + 0.5) * k / N)
    elif kind == G.REDFT01:
        A = 2 * np.cos(np.pi * j * (k + 0.5) / N)
        A[:, 0] = 1.0
    elif kind == G.RODFT10:
        A = 2 * np.sin(np.pi * (j + 0.5) * (k + 1) / N)
    elif kind == G.REDFT11:
        A = 2 * np.cos(np.pi * (j + 0.5) * (k + 0.5) / N)
    else:
        A = 2 * np.sin(np.pi * (j + 1) * (k + 0.5) / N)
        A[:, N - 1] = (-1.0) ** np.arange(N)
    return A @ x


@pytest.mark.parametrize("N", [1, 2, 5, 8, 13])
@pytest.mark.parametrize("kind", [G.REDFT10, G.REDFT01, G.RODFT10, G.RODFT01, G.REDFT11])
def test_kinds_are_fftws_definitions(N, kind):
    x = np.random.default_rng(N).standard_normal((N, 3))
    assert np.allclose(G.r2r(x, kind), explicit(x, kind), rtol=1e-13, atol=1e-13)


def test_phi_transforms_are_unnormalised_dfts():
    M = 9
    x = np.random.default_rng(3).standard_normal((2, M))
    Y = G.r2c(x)
    k = np.arange(M)
    for j in range(M // 2 + 1):
        assert np.allclose(Y[:, j], x @ np.exp(-2j * np.pi * j * k / M))
    back = G.c2r(Y, M)
    assert np.allclose(back, M * x)


@pytest.fixture(scope="module")
def ref():
    from oracle.bind import Reference
    return Reference()


@pytest.mark.parametrize("N", [64, 128])
def test_reference_round_trip(ref, N):
    from fasttransforms_b200.utilities import rand_layout
    A = rand_layout("sph", N, 5)
    P = ref.plan("sph", N)
    X = A.copy(order="F")
    ref.execute("sph", P, True, "N", X)
    X = G.execute("sph_synthesis", "N", "sph_synthesis", X)
    X = np.asfortranarray(G.execute("sph_analysis", "N", "sph_analysis", X))
    ref.execute("sph", P, False, "N", X)
    ref.execute("sph", P, True, "T", X)
    X = G.execute("sph_synthesis", "T", "sph_analysis", X)
    X = np.asfortranarray(G.execute("sph_analysis", "T", "sph_synthesis", X))
    ref.execute("sph", P, False, "T", X)
    ref.destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 4 * np.sqrt(N) * EPS
    assert np.abs(X - A).max() / np.abs(A).max() <= 2 * N * EPS


def test_known_harmonics(ref):
    N = 32
    M = 2 * N - 1
    P = ref.plan("sph", N)
    th, ph = G.grid(N, M)
    c1 = np.sqrt(3 / (4 * np.pi))
    cases = [(0, 0, np.full((N, M), 0.5 / np.sqrt(np.pi))),
             (1, 0, np.outer(c1 * np.cos(th), np.ones(M))),
             (0, 1, np.outer(c1 * np.sin(th), np.sin(ph))),
             (0, 2, np.outer(c1 * np.sin(th), np.cos(ph)))]
    for row, col, want in cases:
        A = np.zeros((N, M), order="F")
        A[row, col] = 1.0
        ref.execute("sph", P, True, "N", A)
        got = G.execute("sph_synthesis", "N", "sph_synthesis", A)
        assert np.abs(got - want).max() < 1e-14, (row, col)
    ref.destroy(P)


@pytest.mark.parametrize("N", [64, 128])
def test_disk_reference_round_trip(ref, N):
    """test/test_fftw.c:226-255: the compiled reference's disk2cxf / cxf2disk around the oracle's
    disk synthesis and analysis, 'N' then 'T' with the plans crossed: 8 sqrt(N) eps, 4N eps."""
    from fasttransforms_b200.utilities import rand_layout
    A = rand_layout("disk", N, 5)
    P = ref.plan("disk", N, 0.0, 0.0)
    X = A.copy(order="F")
    ref.execute("disk", P, True, "N", X)
    X = G.execute_disk("disk_synthesis", "N", "disk_synthesis", X)
    X = np.asfortranarray(G.execute_disk("disk_analysis", "N", "disk_analysis", X))
    ref.execute("disk", P, False, "N", X)
    ref.execute("disk", P, True, "T", X)
    X = G.execute_disk("disk_synthesis", "T", "disk_analysis", X)
    X = np.asfortranarray(G.execute_disk("disk_analysis", "T", "disk_synthesis", X))
    ref.execute("disk", P, False, "T", X)
    ref.destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 8 * np.sqrt(N) * EPS
    assert np.abs(X - A).max() / np.abs(A).max() <= 4 * N * EPS


@pytest.mark.parametrize("N", [64, 128])
def test_tri_reference_round_trip(ref, N):
    """test/test_fftw.c:164-195 (M = N): 32 sqrt(N) eps, 8N eps."""
    from fasttransforms_b200.utilities import rand_layout
    A = rand_layout("tri", N, 5)
    P = ref.plan("tri", N, 0.0, 0.0, 0.0)
    X = A.copy(order="F")
    ref.execute("tri", P, True, "N", X)
    X = G.execute_tri("tri_synthesis", "N", "tri_synthesis", X)
    X = np.asfortranarray(G.execute_tri("tri_analysis", "N", "tri_analysis", X))
    ref.execute("tri", P, False, "N", X)
    ref.execute("tri", P, True, "T", X)
    X = G.execute_tri("tri_synthesis", "T", "tri_analysis", X)
    X = np.asfortranarray(G.execute_tri("tri_analysis", "T", "tri_synthesis", X))
    ref.execute("tri", P, False, "T", X)
    ref.destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 32 * np.sqrt(N) * EPS
    assert np.abs(X - A).max() / np.abs(A).max() <= 8 * N * EPS


def test_tri_grid_is_a_2d_cosine_series():
    """Known answer: the triangle synthesis of a unit coefficient (i, j) (i, j > 0) is
    T_i(x) T_j(y) on the Chebyshev points x_k = cos((k + 1/2) pi / N) (FFTW's REDFT01 with the
    reference's 1/4 scaling)."""
    N = 9
    th = (np.arange(N) + 0.5) * np.pi / N
    for i, j in [(1, 2), (3, 1), (4, 4)]:
        A = np.zeros((N, N))
        A[i, j] = 1.0
        got = G.execute_tri("tri_synthesis", "N", "tri_synthesis", A)
        want = np.outer(np.cos(i * th), np.cos(j * th))
        assert np.abs(got - want).max() < 1e-14, (i, j)


@pytest.mark.parametrize("N", [64, 128])
def test_annulus_reference_round_trip(ref, N):
    """test/test_fftw.c:288-320 (rho = sqrt(1/3), plans crossed in 'T'): the compiled reference's
    ann2cxf / cxf2ann around the oracle's annulus synthesis and analysis: 8 sqrt(N) eps, 4N eps."""
    from fasttransforms_b200.utilities import rand_layout
    rho = np.sqrt(1 / 3)
    A = rand_layout("disk", N, 5)
    P = ref.ann_plan(N, 0.0, 0.0, rho)
    X = A.copy(order="F")
    ref.ann_execute(P, True, "N", X)
    X = G.execute_annulus("annulus_synthesis", "N", "annulus_synthesis", X, rho)
    X = np.asfortranarray(G.execute_annulus("annulus_analysis", "N", "annulus_analysis", X, rho))
    ref.ann_execute(P, False, "N", X)
    ref.ann_execute(P, True, "T", X)
    X = G.execute_annulus("annulus_synthesis", "T", "annulus_analysis", X, rho)
    X = np.asfortranarray(G.execute_annulus("annulus_analysis", "T", "annulus_synthesis", X, rho))
    ref.ann_execute(P, False, "T", X)
    ref.destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 8 * np.sqrt(N) * EPS
    assert np.abs(X - A).max() / np.abs(A).max() <= 4 * N * EPS


@pytest.mark.parametrize("N", [64, 128])
def test_rectdisk_reference_round_trip(ref, N):
    """test/test_fftw.c:350-380 (M = N, beta = 0, plans crossed in 'T'): 8 sqrt(N) eps, 4N eps."""
    from fasttransforms_b200.utilities import rand_layout
    A = rand_layout("rect", N, 5)
    P = ref.plan("rect", N, beta=0.0)
    X = A.copy(order="F")
    ref.execute("rect", P, True, "N", X)
    X = G.execute_rectdisk("rectdisk_synthesis", "N", "rectdisk_synthesis", X)
    X = np.asfortranarray(G.execute_rectdisk("rectdisk_analysis", "N", "rectdisk_analysis", X))
    ref.execute("rect", P, False, "N", X)
    ref.execute("rect", P, True, "T", X)
    X = G.execute_rectdisk("rectdisk_synthesis", "T", "rectdisk_analysis", X)
    X = np.asfortranarray(G.execute_rectdisk("rectdisk_analysis", "T", "rectdisk_synthesis", X))
    ref.execute("rect", P, False, "T", X)
    ref.destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 8 * np.sqrt(N) * EPS
    assert np.abs(X - A).max() / np.abs(A).max() <= 4 * N * EPS


def test_rectdisk_grid_is_a_chebyshev_product():
    """Known answer: the rectdisk synthesis of a unit coefficient in an even column j = 2q is
    T_i(x) T_j(y) (the plan's DCT-III down the even columns and along the rows, with the
    reference's factors) on the Chebyshev points."""
    N = 9
    th = (np.arange(N) + 0.5) * np.pi / N
    for i, j in [(1, 2), (3, 4), (2, 6)]:
        A = np.zeros((N, N))
        A[i, j] = 1.0
        got = G.execute_rectdisk("rectdisk_synthesis", "N", "rectdisk_synthesis", A)
        want = np.outer(np.cos(i * th), np.cos(j * th))
        assert np.abs(got - want).max() < 1e-14, (i, j)


@pytest.mark.parametrize("N", [16, 32])
def test_tet_reference_round_trip(ref, N):
    """test/test_fftw.c:412-447 (L = M = N, parameters 0, plans crossed in 'T'): after the 'N' pair
    8 (NLM)^(1/3) eps, 4 (NLM)^(2/3) eps; after the 'T' pair 64 (NLM)^(2/3) eps, 32 NLM eps."""
    from fasttransforms_b200.utilities import tetrand
    A = tetrand(N, 5)
    P = ref.tet_plan(N, 0.0, 0.0, 0.0, 0.0)
    X = A.copy(order="F")
    ref.tet_execute(P, True, "N", X)
    X = G.execute_tet("tet_synthesis", "N", "tet_synthesis", X)
    X = np.asfortranarray(G.execute_tet("tet_analysis", "N", "tet_analysis", X))
    ref.tet_execute(P, False, "N", X)
    einf = lambda B: np.abs(B - A).max() / np.abs(A).max()
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 8 * N * EPS and einf(X) <= 4 * N * N * EPS
    ref.tet_execute(P, True, "T", X)
    X = G.execute_tet("tet_synthesis", "T", "tet_analysis", X)
    X = np.asfortranarray(G.execute_tet("tet_analysis", "T", "tet_synthesis", X))
    ref.tet_execute(P, False, "T", X)
    ref.destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 64 * N * N * EPS and einf(X) <= 32 * N ** 3 * EPS


def test_tet_grid_is_a_chebyshev_product():
    """Known answer: the tet synthesis of a unit coefficient (i, l, m) (all > 0) is
    T_i(x) T_l(y) T_m(z) on the Chebyshev points."""
    N = 7
    th = (np.arange(N) + 0.5) * np.pi / N
    for i, l, m in [(1, 2, 3), (4, 1, 2)]:
        A = np.zeros((N, N, N))
        A[i, l, m] = 1.0
        got = G.execute_tet("tet_synthesis", "N", "tet_synthesis", A)
        want = np.einsum("a,b,c->abc", np.cos(i * th), np.cos(l * th), np.cos(m * th))
        assert np.abs(got - want).max() < 1e-14, (i, l, m)


@pytest.mark.parametrize("s", [-4, -1, 0, 1, 2, 3])
def test_spin_grid_reference_round_trip(ref, s):
    """test/test_fftw.c:481-516 (N = 64, M = 2N - 1): the compiled reference's spinsph2fourier /
    fourier2spinsph around the oracle's spin synthesis and analysis ('N'), then the 'T' pair, whose
    grid steps the reference's routines leave alone (they act for 'N' and 'C' only): 4 sqrt(N) eps,
    2N eps."""
    from fasttransforms_b200.utilities import spinsphrand
    N = 64
    A = spinsphrand(N, s, 5)
    P = ref.spin_plan(N, s)
    X = A.copy(order="F")
    ref.spin_execute(P, True, "N", X)
    X = G.execute_spinsph("spinsph_synthesis", "N", "spinsph_synthesis", s, X)
    X = np.asfortranarray(G.execute_spinsph("spinsph_analysis", "N", "spinsph_analysis", s, X))
    ref.spin_execute(P, False, "N", X)
    ref.spin_execute(P, True, "T", X)
    assert np.array_equal(G.execute_spinsph("spinsph_synthesis", "T", "spinsph_analysis", s, X), X)   # a no-op
    ref.spin_execute(P, False, "T", X)
    ref.spin_destroy(P)
    assert np.linalg.norm(X - A) / np.linalg.norm(A) <= 4 * np.sqrt(N) * EPS
    assert np.abs(X - A).max() / np.abs(A).max() <= 2 * N * EPS


@pytest.mark.parametrize("s", [0, 1, -2, 3])
def test_spin_grid_pairs_are_identities(s):
    """Synthesis then analysis ('N', own plans) and, with the plans crossed as the reference's
    tests cross them, 'C' synthesis then 'C' analysis both return arbitrary complex data to
    rounding: the sequences, kinds, signs, permutations and scalings fit together."""
    rng = np.random.default_rng(s + 10)
    N, M = 16, 31
    X = rng.standard_normal((N, M)) + 1j * rng.standard_normal((N, M))
    Y = G.execute_spinsph("spinsph_analysis", "N", "spinsph_analysis", s,
                          G.execute_spinsph("spinsph_synthesis", "N", "spinsph_synthesis", s, X))
    Z = G.execute_spinsph("spinsph_analysis", "C", "spinsph_synthesis", s,
                          G.execute_spinsph("spinsph_synthesis", "C", "spinsph_analysis", s, X))
    assert np.linalg.norm(Y - X) / np.linalg.norm(X) < 1e-15 * N
    assert np.linalg.norm(Z - X) / np.linalg.norm(X) < 1e-15 * N
