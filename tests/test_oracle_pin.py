"""Pin the oracle restatement (oracle/ft_oracle.c) to the reference.

Against the golden fixtures (outputs of the reference library compiled from
its own sources, tests/golden/make_golden.py) and, where the reference library
is built, against live reference runs at larger sizes.  CPU only.
"""
import glob
import os

import numpy as np
import pytest

from conftest import EPS, rel2, relinf
from oracle.bind import Oracle, Reference, fill

# the sph / tri / disk fixtures (the spin and Dunkl-Xu fixtures have their own tests)
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if os.path.basename(p).split("_")[0] in ("sph", "tri", "disk"))


@pytest.fixture(scope="module")
def O():
    o = Oracle()
    o.set_fused(True)
    return o


def _case(path):
    z = np.load(path)
    kind = os.path.basename(path).split("_")[0]
    return kind, z


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_connection_matrices_bitwise(O, path):
    kind, z = _case(path)
    n = z["A"].shape[0]
    P = O.plan(kind, n, *z["params"])
    Ps, Pinvs = O.connection(P)
    O.destroy(P)
    for mine, name in zip(Ps + Pinvs, ("P0", "P1", "Pinv0", "Pinv1")):
        assert np.array_equal(np.triu(mine), np.triu(z[name])), name


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_transforms_match_reference(O, path):
    kind, z = _case(path)
    n = z["A"].shape[0]
    P = O.plan(kind, n, *z["params"])
    for fwd in (True, False):
        for tr in "NT":
            B = z["A"].copy(order="F")
            O.execute(P, fwd, tr, B)
            ref = z[("fwd" if fwd else "bwd") + "_" + tr]
            assert rel2(B, ref) <= 1e-14, (fwd, tr, rel2(B, ref))
    O.destroy(P)


SPH_GOLDEN = [p for p in GOLDEN if os.path.basename(p).startswith("sph_")]


@pytest.mark.parametrize("path", SPH_GOLDEN, ids=[os.path.basename(p)[:-4] for p in SPH_GOLDEN])
def test_vector_field_transforms_match_reference(O, path):
    """sphv2fourier / fourier2sphv (src/drivers.c:867-899) on the sph plan."""
    _, z = _case(path)
    n = z["A"].shape[0]
    P = O.plan("sph", n)
    for fwd in (True, False):
        for tr in "NT":
            B = z["A"].copy(order="F")
            O.execute_sphv(P, fwd, tr, B)
            ref = z["v_" + ("fwd" if fwd else "bwd") + "_" + tr]
            assert rel2(B, ref) <= 1e-14, (fwd, tr, rel2(B, ref))
    O.destroy(P)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_rotation_stage_matches_reference(O, path):
    kind, z = _case(path)
    n = z["A"].shape[0]
    P = O.plan(kind, n, *z["params"], rotations_only=True)
    for d in ("hi2lo", "lo2hi"):
        B = z["A"].copy(order="F")
        (O.hi2lo if d == "hi2lo" else O.lo2hi)(P, B)
        assert rel2(B, z["rot_" + d]) <= 1e-15, d
    O.destroy(P)


def test_fill_matches_numpy(O):
    import fasttransforms_b200.utilities as U
    for kind in ("sph", "tri", "disk"):
        for n in (1, 2, 7, 16):
            a = O.fill(kind, n, 99)
            b = fill(kind, n, 99)
            c = U.rand_layout(kind, n, 99)
            assert np.array_equal(a, b) and np.array_equal(b, c)


# the reference's own round-trip checks (test/test_drivers.c:232-248, 704-721, 941-958)
TOL = {"sph": (4, 2), "tri": (32, 8), "disk": (8, 4)}


@pytest.mark.parametrize("kind,params", [("sph", ()), ("tri", (0.0, 0.0, 0.0)), ("tri", (-0.5, -0.5, -0.5)),
                                         ("disk", (0.0, 0.0))])
@pytest.mark.parametrize("n", [64, 127])
def test_oracle_round_trip(O, kind, params, n):
    A = fill(kind, n, 7)
    B = A.copy(order="F")
    P = O.plan(kind, n, *params)
    O.execute(P, True, "N", B)
    O.execute(P, False, "N", B)
    O.execute(P, True, "T", B)
    O.execute(P, False, "T", B)
    O.destroy(P)
    c2, ci = TOL[kind]
    assert rel2(B, A) < c2 * np.sqrt(n) * EPS
    assert relinf(B, A) < ci * n * EPS


def test_invalid_trans_is_noop(O):
    A = fill("sph", 16, 3)
    B = A.copy(order="F")
    P = O.plan("sph", 16)
    O.execute(P, True, "X", B)
    O.destroy(P)
    assert np.array_equal(A, B)


needs_ref = pytest.mark.skipif(not Reference.available(), reason="reference library not built")


@needs_ref
@pytest.mark.parametrize("kind,params,n", [("sph", (), 256), ("sph", (), 255), ("tri", (0.0, 0.0, 0.0), 200),
                                           ("tri", (-0.5, -0.5, -0.5), 128), ("disk", (0.0, 0.0), 128)])
def test_oracle_vs_live_reference(O, kind, params, n):
    R = Reference()
    A = fill(kind, n, 11)
    PO, PR = O.plan(kind, n, *params), R.plan(kind, n, *params)
    Po, Pio = O.connection(PO)
    Pr, Pir = R.connection(PR, n)
    for a, b in zip(Po + Pio, Pr + Pir):
        assert np.array_equal(np.triu(a), np.triu(b))
    for fwd in (True, False):
        for tr in "NT":
            B1 = A.copy(order="F"); B2 = A.copy(order="F")
            O.execute(PO, fwd, tr, B1)
            R.execute(kind, PR, fwd, tr, B2)
            assert rel2(B1, B2) <= 1e-14
    O.destroy(PO)
    R.destroy(PR)
