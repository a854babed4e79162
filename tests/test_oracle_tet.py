"""Pins the tetrahedral part of the oracle (oracle/ft_oracle.c: oracle_plan_tet2cheb, the
slab sweeps, the execute loop and the transforms, restating src/rotations.c:297-321,
src/drivers.c:26-54, 510-528, 1173-1257) against the reference compiled from its own sources
and against the golden fixtures it produced.  CPU only.

The reference's tetrahedral transforms amplify rounding: its own round-trip test
(test/test_drivers.c:1418-1447) allows 8 (NLM)^(1/3) eps after the 'N' pair and
64 (NLM)^(2/3) eps after the 'T' pair, and rounding differences of a few ulps in the rotation
stage come out of the forward 'N' transform amplified by the connection multiplies.  So the
bars are: connection matrices bit-identical; the rotation stage within 2n ulps of the
input's scale (the reference mixes scalar, SSE2 and AVX kernels); the transforms within
1e-14, or within four times the oracle's own fused-versus-unfused spread (the rounding
sensitivity of the transform at that size) where that is larger; the reference's round trips
within its own bounds."""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "tet_*.npz")))
PARAMS = [(0.0, 0.0, 0.0, 0.0), (-0.5, -0.5, -0.5, -0.5), (0.5, -0.25, 0.25, 1.0)]


@pytest.fixture(scope="module")
def oracles():
    from oracle.bind import Oracle, Reference
    return Oracle(), Reference()


def sensitivity(O, Po, fwd, tr, A):
    """Relative 2-norm distance between the oracle's fused and unfused results."""
    a, b = A.copy(order="F"), A.copy(order="F")
    O.set_fused(True)
    O.tet_execute(Po, fwd, tr, a)
    O.set_fused(False)
    O.tet_execute(Po, fwd, tr, b)
    O.set_fused(True)
    return rel2(a, b)


def test_fills_agree(oracles):
    O, R = oracles
    from fasttransforms_b200.utilities import tetrand
    for n in (1, 5, 12):
        assert np.array_equal(O.tet_fill(n, n, n, 13), tetrand(n, 13))


@pytest.mark.parametrize("n", [1, 2, 8, 17, 32])
@pytest.mark.parametrize("params", PARAMS)
def test_tet_vs_reference(oracles, n, params):
    O, R = oracles
    from fasttransforms_b200.utilities import tetrand
    A = tetrand(n, 7)
    P, Po = R.tet_plan(n, *params), O.tet_plan(n, *params)
    Pr, Pir = R.connection(P, n)
    Pc, Pic = O.tet_connection(Po)
    for a, b in zip(Pr + Pir, Pc + Pic):
        assert np.array_equal(a, b)
    for fwd in (True, False):
        for tr in "NT":
            a, b = A.copy(order="F"), A.copy(order="F")
            R.tet_execute(P, fwd, tr, a)
            O.tet_execute(Po, fwd, tr, b)
            tol = max(1e-14, 4 * sensitivity(O, Po, fwd, tr, A))
            assert rel2(b, a) <= tol, (fwd, tr, rel2(b, a), tol)
    for hi2lo in (True, False):
        a, b = A.copy(order="F"), A.copy(order="F")
        R.tet_rotations(n, params, hi2lo, a)
        (O.tet_hi2lo if hi2lo else O.tet_lo2hi)(Po, b)
        assert np.abs(b - a).max() <= 2 * n * EPS * max(1.0, np.abs(A).max()), hi2lo
    R.destroy(P)
    O.tet_destroy(Po)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_tet_oracle_vs_golden(oracles, path):
    O, R = oracles
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n = A.shape[0]
    params = tuple(float(x) for x in z["params"])
    Po = O.tet_plan(n, *params)
    Pc, Pic = O.tet_connection(Po)
    for i in range(3):
        assert np.array_equal(Pc[i], z[f"P{i}"]) and np.array_equal(Pic[i], z[f"Pinv{i}"])
    for fwd in (True, False):
        for tr in "NT":
            b = A.copy(order="F")
            O.tet_execute(Po, fwd, tr, b)
            tol = max(1e-14, 4 * sensitivity(O, Po, fwd, tr, A))
            assert rel2(b, z[("fwd" if fwd else "bwd") + "_" + tr]) <= tol
    for d in ("hi2lo", "lo2hi"):
        b = A.copy(order="F")
        (O.tet_hi2lo if d == "hi2lo" else O.tet_lo2hi)(Po, b)
        assert np.abs(b - z["rot_" + d]).max() <= 2 * n * EPS
    O.tet_destroy(Po)


@pytest.mark.parametrize("n", [16, 33, 64])
def test_tet_round_trips(oracles, n):
    """The reference's own tests with its bounds (N = L = M = n, its parameters 0, 0, 0, 0):
    test/test_drivers.c:1282-1304, hi2lo then lo2hi within 8 n eps (2-norm) and 4 n^2 eps
    (max); :1418-1447, tet2cheb then cheb2tet 'N' within 8 n eps and 4 n^2 eps, then the 'T'
    pair as well within 64 n^2 eps and 32 n^3 eps."""
    O, R = oracles
    from fasttransforms_b200.utilities import tetrand
    A = tetrand(n, 5)
    Po = O.tet_plan(n, 0.0, 0.0, 0.0, 0.0)
    einf = lambda B: np.abs(B - A).max() / np.abs(A).max()
    B = A.copy(order="F")
    O.tet_hi2lo(Po, B)
    O.tet_lo2hi(Po, B)
    assert rel2(B, A) <= 8 * n * EPS and einf(B) <= 4 * n * n * EPS
    B = A.copy(order="F")
    O.tet_execute(Po, True, "N", B)
    O.tet_execute(Po, False, "N", B)
    assert rel2(B, A) <= 8 * n * EPS and einf(B) <= 4 * n * n * EPS
    O.tet_execute(Po, True, "T", B)
    O.tet_execute(Po, False, "T", B)
    assert rel2(B, A) <= 64 * n * n * EPS and einf(B) <= 32 * n ** 3 * EPS
    O.tet_destroy(Po)
