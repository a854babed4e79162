"""Pins the spin-weighted part of the oracle (oracle/ft_oracle.c: ft_plan_rotspinsphere,
kernel_spinsph_*_default, execute_spinsph_*, ft_execute_spinsph2fourier /
fourier2spinsph restated) against the reference compiled from its own sources and
against the golden fixtures it produced.  CPU only.

Bars: the rotation stage within 1e-15 relative 2-norm of the reference's (the
reference runs its SIMD kernels, the oracle the fused scalar form), the transforms
within 1e-14; the fills of the C oracle and of numpy bit-identical."""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "spin_*.npz")))


@pytest.fixture(scope="module")
def oracles():
    from oracle.bind import Oracle, Reference
    O = Oracle()
    O.set_fused(True)
    return O, Reference()


def test_fills_agree(oracles):
    O, R = oracles
    from fasttransforms_b200.utilities import spinsphrand
    for n, s in ((9, 0), (16, -3), (7, 2)):
        assert np.array_equal(O.spin_fill(n, 2 * n - 1, s, 11), spinsphrand(n, s, 11))


@pytest.mark.parametrize("n", [16, 33, 64])
@pytest.mark.parametrize("s", [-4, -3, -2, -1, 0, 1, 2, 3, 4])
def test_spin_vs_reference(oracles, n, s):
    O, R = oracles
    M = 2 * n - 1
    A = O.spin_fill(n, M, s, 7)
    Po = O.spin_plan(n, s, False)
    for hi2lo in (True, False):
        a, b = A.copy(order="F"), A.copy(order="F")
        R.spin_rotations(n, s, hi2lo, a)
        (O.spin_hi2lo if hi2lo else O.spin_lo2hi)(Po, b)
        assert rel2(b, a) <= 1e-15, (hi2lo, rel2(b, a))
    O.spin_destroy(Po)
    P, Po = R.spin_plan(n, s), O.spin_plan(n, s, True)
    for fwd in (True, False):
        for tr in "NT":
            a, b = A.copy(order="F"), A.copy(order="F")
            R.spin_execute(P, fwd, tr, a)
            O.spin_execute(Po, fwd, tr, b)
            assert rel2(b, a) <= 1e-14, (fwd, tr, rel2(b, a))
    R.spin_destroy(P)
    O.spin_destroy(Po)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_spin_oracle_vs_golden(oracles, path):
    O, R = oracles
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n, M = A.shape
    s = int(z["s"])
    Po = O.spin_plan(n, s, True)
    for fwd in (True, False):
        for tr in "NT":
            b = A.copy(order="F")
            O.spin_execute(Po, fwd, tr, b)
            assert rel2(b, z[("fwd" if fwd else "bwd") + "_" + tr]) <= 1e-14
    for d in ("hi2lo", "lo2hi"):
        b = A.copy(order="F")
        (O.spin_hi2lo if d == "hi2lo" else O.spin_lo2hi)(Po, b)
        assert rel2(b, z["rot_" + d]) <= 1e-15
    O.spin_destroy(Po)


def test_spin_rotation_round_trip(oracles):
    """test/test_drivers.c:1479-1500: hi2lo then lo2hi within 4 sqrt(N) eps, 2N eps."""
    O, R = oracles
    for n in (64, 128):
        for s in (-2, 1, 4):
            A = O.spin_fill(n, 2 * n - 1, s, 3)
            Po = O.spin_plan(n, s, False)
            B = A.copy(order="F")
            O.spin_hi2lo(Po, B)
            O.spin_lo2hi(Po, B)
            O.spin_destroy(Po)
            assert rel2(B, A) <= 4 * np.sqrt(n) * EPS
            assert np.abs(B - A).max() / np.abs(A).max() <= 2 * n * EPS


@pytest.mark.parametrize("s", [-2, 0, 3])
def test_oracle_spin_column_kernel_matches_matrix_form(s):
    """The oracle's one-column kernel (the reference's ft_kernel_spinsph_hi2lo / lo2hi) on each
    column of a matrix, order 0 in column 0 and orders -m, m in columns 2m - 1, 2m, equals its
    matrix form: the checker of the device column kernels agrees with the pinned matrix sweeps."""
    from oracle.bind import Oracle
    O = Oracle()
    n = 24
    M = 2 * n - 1
    P = O.spin_plan(n, s, connections=False)
    A = O.spin_fill(n, M, s, 3)
    for hi2lo in (True, False):
        whole = A.copy(order="F")
        (O.spin_hi2lo if hi2lo else O.spin_lo2hi)(P, whole)
        cols = np.empty_like(A)
        for c in range(M):
            m = 0 if c == 0 else ((c + 1) // 2 if c % 2 == 0 else -((c + 1) // 2))
            cols[:, c] = O.spin_kernel(P, hi2lo, m, A[:, c])
        assert np.array_equal(cols, whole), hi2lo
    O.spin_destroy(P)
