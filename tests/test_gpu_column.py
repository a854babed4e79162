"""One column's sweeps on the GPU (ft_kernel_{sph,tri,disk,rectdisk}_{hi2lo,lo2hi}:
src/rotations.c:135-141, 162-168, 262-268, 289-295; ft_kernel_spinsph_* and ft_kernel_tet_*:
src/rotations.c:297-321, 479-485), through the C ABI.

Against the oracle's sequential per-column loops (oracle/ft_oracle.c, oracle_kernel_hi2lo /
lo2hi, pinned to the compiled reference in tests/test_oracle_pin.py) in its fused form, bit for
bit: every family, orders m1 <= m2 of both parities, strides 1 and 3 (the entries between the
strided ones untouched), more than one chunk of 1024 sweeps, and a column past the shared-memory
size.  Consistency with the matrix form: the column kernel from order m down to m mod 2 on a
matrix's columns equals ft_execute_*_hi2lo on that matrix.  The schedule and index arithmetic
are also restated on the CPU in tests/test_device_schedules.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FAMILIES = {"sph": (), "tri": (0.0, -0.5, 0.25), "disk": (0.5, -0.25), "rect": (0.5,)}


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    from oracle.bind import Oracle
    torch.cuda.set_device(0)
    O = Oracle()
    O.set_fused(True)
    return ft, O


def plans(ft, O, fam, n):
    params = FAMILIES[fam]
    if fam == "sph":
        return ft.plan_rotsphere(n), O.plan("sph", n, rotations_only=True)
    if fam == "tri":
        return ft.plan_rottriangle(n, *params), O.plan("tri", n, alpha=params[0], beta=params[1], gamma=params[2], rotations_only=True)
    if fam == "disk":
        return ft.plan_rotdisk(n, *params), O.plan("disk", n, alpha=params[0], beta=params[1], rotations_only=True)
    return ft.plan_rotrectdisk(n, *params), O.plan("rect", n, beta=params[0], rotations_only=True)


@pytest.mark.parametrize("fam", list(FAMILIES))
@pytest.mark.parametrize("n", [1, 2, 5, 33, 300])
def test_column_vs_oracle_bit_exact(env, fam, n):
    ft, O = env
    RP, Po = plans(ft, O, fam, n)
    rng = np.random.default_rng(n)
    mmax = 2 * n + 1 if fam == "disk" else n + 2
    pairs = [(m1, m2) for m2 in range(mmax + 1) for m1 in range(m2 + 2)]
    if len(pairs) > 80:
        pairs = [pairs[i] for i in rng.choice(len(pairs), 80, replace=False)] + [(0, mmax), (1, mmax - 1)]
    for m1, m2 in pairs:
        for S in (1, 3):
            A = rng.uniform(-1, 1, n * S)
            for hi2lo in (True, False):
                want = O.kernel(Po, hi2lo, m1, m2, A[::S].copy())
                got = A.copy()
                ft.kernel_column(RP, hi2lo, m1, m2, got, S)
                assert np.array_equal(got[::S], want), (fam, n, m1, m2, S, hi2lo)
                mask = np.ones(n * S, bool)
                mask[::S] = False
                assert np.array_equal(got[mask], A[mask])
    O.destroy(Po)
    RP.close()


@pytest.mark.parametrize("fam,n", [("sph", 2600), ("tri", 1500), ("disk", 1100), ("sph", 25700)])
def test_long_columns_bit_exact(env, fam, n):
    """More than 1024 sweeps (several chunks), and (n = 25700, m1 = m2 mod 2) a column longer
    than the shared-memory column of 25600 entries, kept in global memory.

    The reference's sph table multiplies in int (src/rotations.c:122-124, den = (l + 2m + 3)
    (l + 2m + 4)), which overflows once l + 2m + 4 > 46340; the oracle restates that, while this
    library multiplies in 64 bits.  The sweeps compared therefore stay below that: for the long
    column the highest order is capped so that n + m2 + 1 <= 46340 (its column still spans
    n - 1 entries)."""
    ft, O = env
    RP, Po = plans(ft, O, fam, n)
    m2 = 2 * n - 2 if fam == "disk" else n - 1
    if fam == "sph":
        m2 = min(m2, 46340 - n - 1)
    A = np.random.default_rng(1).uniform(-1, 1, n)
    for m1 in (m2 % 2, m2 - 40):
        for hi2lo in (True, False):
            want = O.kernel(Po, hi2lo, m1, m2, A.copy())
            got = A.copy()
            ft.kernel_column(RP, hi2lo, m1, m2, got)
            assert np.array_equal(got, want), (fam, n, m1, hi2lo)
    O.destroy(Po)
    RP.close()


@pytest.mark.parametrize("fam", ["sph", "rect"])
def test_column_matches_matrix_form(env, fam):
    ft, O = env
    n = 64
    RP, Po = plans(ft, O, fam, n)
    M = 2 * n - 1 if fam == "sph" else n
    A = np.asfortranarray(np.random.default_rng(5).uniform(-1, 1, (n, M)))
    whole = A.copy(order="F")
    (ft.execute_sph_hi2lo if fam == "sph" else ft.execute_rectdisk_hi2lo)(RP, whole)
    cols = A.copy(order="F")
    if fam == "sph":   # order m on columns 2m - 1, 2m
        for m in range(2, M // 2 + 1):
            for c in (2 * m - 1, 2 * m):
                v = cols[:, c].copy()
                ft.kernel_column(RP, True, m % 2, m, v)
                cols[:, c] = v
    else:              # order m on column m
        for m in range(2, M):
            v = cols[:, m].copy()
            ft.kernel_column(RP, True, m % 2, m, v)
            cols[:, m] = v
    assert np.array_equal(cols, whole)
    O.destroy(Po)
    RP.close()


def test_bad_arguments(env):
    ft, O = env
    RP = ft.plan_rotsphere(8)
    a = np.zeros(8)
    with pytest.raises(ft.FTB200Error):
        ft.kernel_column(RP, True, -1, 4, a)     # m1 < 0
    with pytest.raises(ValueError):
        ft.kernel_column(RP, True, 0, 4, np.zeros(7))
    ft.kernel_column(RP, True, 4, 4, a)          # no sweep: a no-op
    RP.close()


@pytest.mark.parametrize("n", [1, 3, 24, 200])
@pytest.mark.parametrize("s", [-3, 0, 1, 4])
def test_spin_column_vs_oracle_bit_exact(env, n, s):
    """ft_kernel_spinsph_hi2lo / lo2hi (src/rotations.c:479-485) against the oracle's column
    kernel: every order -(n + 1) .. n + 1, strides 1 and 2."""
    ft, O = env
    SRP = ft.plan_rotspinsphere(n, s)
    P = O.spin_plan(n, s, connections=False)
    rng = np.random.default_rng(n + 10 * (s + 5))
    for m in range(-(n + 1), n + 2):
        for S in (1, 2):
            A = rng.uniform(-1, 1, n * S) + 1j * rng.uniform(-1, 1, n * S)
            for hi2lo in (True, False):
                want = O.spin_kernel(P, hi2lo, m, A[::S])
                got = A.copy()
                ft.kernel_spin_column(SRP, hi2lo, m, got, S)
                assert np.array_equal(got[::S], want), (n, s, m, S, hi2lo)
    O.spin_destroy(P)
    SRP.close()


@pytest.mark.parametrize("n,L", [(1, 1), (5, 5), (40, 40), (40, 17), (130, 130)])
def test_tet_slab_vs_oracle_bit_exact(env, n, L):
    """ft_kernel_tet_hi2lo / lo2hi (src/rotations.c:297-321) against the oracle's slab loops."""
    ft, O = env
    RP = ft.plan_rottriangle(n, 0.0, -0.5, 0.25)
    Po = O.plan("tri", n, alpha=0.0, beta=-0.5, gamma=0.25, rotations_only=True)
    rng = np.random.default_rng(n + L)
    for m in sorted({0, 1, L // 2, L - 1, L, n}):
        A = np.asfortranarray(rng.uniform(-1, 1, (n, L)))
        for hi2lo in (True, False):
            want = O.tet_kernel(Po, hi2lo, L, m, A)
            got = A.copy(order="F")
            ft.kernel_tet_slab(RP, hi2lo, L, m, got)
            assert np.array_equal(got, want), (n, L, m, hi2lo)
    O.destroy(Po)
    RP.close()
