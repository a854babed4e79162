"""Pins the Dunkl-Xu (rectangularised disk) part of the oracle (oracle/ft_oracle.c:
plan_rotrectdisk, the rect kernels, execute loop, oracle_plan_rectdisk2cheb and the
rect transforms, restating src/rotations.c:270-287, src/rotations/rotations_default.c:73-85,
src/drivers.c:488-508, 1123-1171 and src/transforms.c:185-211) against the reference
compiled from its own sources and against the golden fixtures it produced.  CPU only.

Bars: connection matrices bit-identical; the rotation stage bit-identical in the unfused
form (the reference has only the scalar kernel for this family) and within 1e-15
(max-abs relative) in the fused form the GPU uses; transforms within 1e-14 relative
2-norm; the reference's own round-trip tests (test/test_drivers.c:1179-1200, 1230-1252)
within 4 sqrt(N) eps and 2N eps at the test's beta = 0 (twice the reference's own error
at beta = 1/2, where the reference exceeds those bounds)."""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "rect_*.npz")))
BETAS = [0.0, 0.5, -0.25, 1.5]


@pytest.fixture(scope="module")
def oracles():
    from oracle.bind import Oracle, Reference
    return Oracle(), Reference()


@pytest.mark.parametrize("n", [1, 2, 3, 16, 33, 64])
@pytest.mark.parametrize("beta", BETAS)
def test_rect_vs_reference(oracles, n, beta):
    O, R = oracles
    from oracle.bind import fill
    A = fill("rect", n, 11)
    P, Po = R.plan("rect", n, beta=beta), O.plan("rect", n, beta=beta)
    Pr, Pir = R.connection(P, n)
    Pc, Pic = O.connection(Po)
    for a, b in zip(Pr + Pir, Pc + Pic):
        assert np.array_equal(a, b)
    O.set_fused(True)
    for fwd in (True, False):
        for tr in "NT":
            a, b = A.copy(order="F"), A.copy(order="F")
            R.execute("rect", P, fwd, tr, a)
            O.execute(Po, fwd, tr, b)
            assert rel2(b, a) <= 1e-14, (fwd, tr, rel2(b, a))
    R.destroy(P)
    O.destroy(Po)
    Pro = O.plan("rect", n, beta=beta, rotations_only=True)
    for fused in (False, True):
        O.set_fused(fused)
        for hi2lo in (True, False):
            a, b = A.copy(order="F"), A.copy(order="F")
            R.rect_rotations(n, beta, hi2lo, a)
            (O.hi2lo if hi2lo else O.lo2hi)(Pro, b)
            if fused:
                assert np.abs(b - a).max() <= 1e-15 * max(1.0, np.abs(a).max()) * max(1, n)
            else:
                assert np.array_equal(a, b), (hi2lo, np.abs(b - a).max())
    O.set_fused(True)
    O.destroy(Pro)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_rect_oracle_vs_golden(oracles, path):
    O, R = oracles
    O.set_fused(False)
    z = np.load(path)
    A = np.asfortranarray(z["A"])
    n = A.shape[0]
    beta = float(z["beta"])
    Po = O.plan("rect", n, beta=beta)
    Pc, Pic = O.connection(Po)
    for i in range(3):
        assert np.array_equal(Pc[i], z[f"P{i}"]) and np.array_equal(Pic[i], z[f"Pinv{i}"])
    for fwd in (True, False):
        for tr in "NT":
            b = A.copy(order="F")
            O.execute(Po, fwd, tr, b)
            assert rel2(b, z[("fwd" if fwd else "bwd") + "_" + tr]) <= 1e-14
    for d in ("hi2lo", "lo2hi"):
        b = A.copy(order="F")
        (O.hi2lo if d == "hi2lo" else O.lo2hi)(Po, b)
        assert np.array_equal(b, z["rot_" + d])
    O.destroy(Po)
    O.set_fused(True)


@pytest.mark.parametrize("n", [64, 128])
def test_rect_reference_round_trips(oracles, n):
    """test/test_drivers.c:1179-1200 (rotations) and 1230-1252 (transforms), on the oracle:
    with the reference test's beta = 0 within 4 sqrt(N) eps and 2N eps; with beta = 1/2,
    where the reference's own round trip exceeds those bounds (2.1x at n = 64, 6.8x at
    n = 128), within twice the reference's own error."""
    O, R = oracles
    from oracle.bind import fill
    A = fill("rect", n, 5)
    for beta in (0.0, 0.5):
        Po = O.plan("rect", n, beta=beta)
        B = A.copy(order="F")
        O.hi2lo(Po, B)
        O.lo2hi(Po, B)
        assert rel2(B, A) <= 4 * np.sqrt(n) * EPS
        B = A.copy(order="F")
        for tr in "NT":
            O.execute(Po, True, tr, B)
            O.execute(Po, False, tr, B)
        O.destroy(Po)
        e2, einf = rel2(B, A), np.abs(B - A).max() / np.abs(A).max()
        if beta == 0.0:
            assert e2 <= 4 * np.sqrt(n) * EPS and einf <= 2 * n * EPS
        else:
            P = R.plan("rect", n, beta=beta)
            C = A.copy(order="F")
            for tr in "NT":
                R.execute("rect", P, True, tr, C)
                R.execute("rect", P, False, tr, C)
            R.destroy(P)
            assert e2 <= 2 * rel2(C, A) and einf <= 2 * np.abs(C - A).max() / np.abs(A).max()
