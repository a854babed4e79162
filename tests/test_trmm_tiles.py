"""CPU restatement of the tensor-core connection multiply's tile list (fasttransforms_b200/csrc/
trmm_mixed.cu: class_cols, order_tiles): Out = op(U) In over the column classes, one 128-row x
TBN-column output tile per entry with the 64-row K-tiles k0 .. k1 it sums.  Checked for the
shapes the library uses (sph and disk: four stride-4 classes; tri: one class; TBN 96 for the
integer form, 128 and 96 for the BF16 form), 'N' (upper-triangular U) and 'T' (its transpose):
  * every (field, class, row tile, column tile) with columns in its class appears exactly once;
  * each entry's K-tiles cover every nonzero of op(U) in its rows and stop where the triangle
    does (no K-tile wholly of zeros for 'N' at the start, none past the diagonal for 'T');
  * entries are grouped by blocks of 8 row tiles (longest K first) and 18 column tiles."""
import pytest

TB, KT = 128, 64
ROW_GROUP, COL_GROUP = 8, 18


def class_cols(M, r, ncls):
    return (M - r + ncls - 1) // ncls


def order_tiles(nf, ncls, nit, nkt, njt, tbn, M, tr):
    v = []
    for f in range(nf):
        for r in range(ncls):
            for it in range(nit):
                jt = 0
                while jt * tbn < class_cols(M, r, ncls):
                    k0 = 0 if tr else 2 * it
                    k1 = min(nkt - 1, 2 * it + 1) if tr else nkt - 1
                    rank = nit - 1 - it if tr else it
                    col = (f * ncls + r) * njt + jt
                    v.append(((rank // ROW_GROUP, col // COL_GROUP, -(k1 - k0 + 1)), (f, r, it, jt, k0, k1)))
                    jt += 1
    v.sort(key=lambda x: x[0])          # stable, as std::stable_sort with the same keys
    return [t for _, t in v]


@pytest.mark.parametrize("family,n", [("sph", 64), ("sph", 1000), ("sph", 4096), ("disk", 300), ("tri", 513), ("tri", 2048)])
@pytest.mark.parametrize("tbn", [96, 128])
@pytest.mark.parametrize("tr", [0, 1])
def test_tiles_cover_the_triangle_once(family, n, tbn, tr):
    M = {"sph": 2 * n - 1, "disk": 4 * n - 3, "tri": n}[family]
    ncls = 1 if family == "tri" else 4
    nf = 2
    nkt, nit = -(-n // KT), -(-n // TB)
    njt = -(-class_cols(M, 0, ncls) // tbn)
    tl = order_tiles(nf, ncls, nit, nkt, njt, tbn, M, tr)
    seen = [(f, r, it, jt) for f, r, it, jt, _, _ in tl]
    want = [(f, r, it, jt) for f in range(nf) for r in range(ncls) for it in range(nit)
            for jt in range(-(-class_cols(M, r, ncls) // tbn))]
    assert sorted(seen) == sorted(want) and len(seen) == len(set(seen))
    for f, r, it, jt, k0, k1 in tl:
        rows = range(TB * it, min(n, TB * it + TB))
        # op(U)[i][k] != 0 only for k >= i ('N', upper triangular) or k <= i ('T')
        need_lo = min(rows) if not tr else 0
        need_hi = n - 1 if not tr else max(rows)
        assert k0 == need_lo // KT and k1 == need_hi // KT, (it, k0, k1)
    keys = []
    for f, r, it, jt, k0, k1 in tl:
        rank = nit - 1 - it if tr else it
        keys.append((rank // ROW_GROUP, ((f * ncls + r) * njt + jt) // COL_GROUP, -(k1 - k0 + 1)))
    assert keys == sorted(keys)
