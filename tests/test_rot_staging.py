"""CPU check of the rotation kernel's (sin, cos) staging (fasttransforms_b200/csrc/rotations.cu,
prefetch_sc, and the padded table of Geo::padded_col in ft_internal.h), restated here with the
kernel's own index formulas.

For every family, direction, launch shape (W stages x B sweeps x chunk E), task, pass, active
stage, chunk and sweep, the kernel bulk-copies the E * CH consecutive entries of the sweep's
padded column that start at chain position ibase.  Checked: (a) the copy lies inside that column's
padded segment when it overlaps the sweep's entries (it then reaches at most E positions past
them, into the padding), and reads the identity row when it does not, so it never reads another
column; (b) entry jj of the copy is the packed table's entry (j, l) exactly where the
sweep has a rotation at that step (the kernel's former per-entry rule: step t within the sweep's
valid steps tlo .. thi, chain position i = ref + 2s - t in hi2lo, t - 2s in lo2hi), and the
identity (sin 0, cos 1) everywhere else."""
import pytest

SPH, TRI, DISK, SPIN, RECT = 0, 1, 2, 3, 4
PADPOS, IDLEN = 16, 64            # Geo::kPadPos, Geo::kIdLen
SHAPES = [(8, 8, 16), (16, 4, 8), (8, 4, 8), (8, 4, 16), (4, 4, 16), (4, 8, 16)]


def fdiv2(x):
    return x // 2   # Python's floor division is Geo::floordiv2


def sphlike(k):
    return k in (SPH, SPIN, RECT)


def ch(k):
    return 2 if sphlike(k) else 1


def step(k):
    return 1 if k == TRI else 2


def top(k, N, j, c):
    if sphlike(k):
        return fdiv2(N - 3 - j - c)
    if k == TRI:
        return N - 2 - j
    return N - 2 - (j + 1) // 2 if j + 1 >= 0 else N - 2 - (-((-(j + 1)) // 2))


def table_base(k, N, j):
    if k == DISK:
        return j * N - (j // 2) * ((j + 1) // 2)
    return j * (2 * N + 1 - j) // 2


def table_cols(k, N):
    return 2 * N - 1 if k == DISK else N


def pad_side(k):
    return PADPOS * ch(k)


def padded_col(k, N, j):
    return IDLEN + table_base(k, N, j) + (2 * j + 1) * pad_side(k)


def task_orders(k):
    return 16 if sphlike(k) else 32


def last_order(k, M):
    return M - 1 if k in (TRI, RECT) else M // 2


def task_sweeps(k, M, mbase, blk, spin=0):
    st, ordn, mlast = step(k), task_orders(k), last_order(k, M)
    omax = mbase + st * (ordn - 1)
    if omax > mlast:
        omax = mbase + st * ((mlast - mbase) // st)
    if k == SPIN:
        emax = 0
        for m in range(mbase, omax + 1, st):
            emax = max(emax, m - spin, spin - m)
        jlo, jhi = (mbase + spin) & 1, emax - st
        return (0 if jhi < jlo else (jhi - jlo) // st + 1), jlo, jhi
    jpar = 0 if k == TRI else (mbase & 1)
    jlo = jpar
    if blk > 0:
        jlo = mbase - st * (((mbase - jpar) // st) % blk)
        for o in range(1, ordn):
            m = mbase + st * o
            if m > mlast:
                break
            jlo = min(jlo, m - st * (((m - jpar) // st) % blk))
    jhi = omax - st
    return (0 if jhi < jlo else (jhi - jlo) // st + 1), jlo, jhi


def tasks(k, M, spin=0):
    mlast = last_order(k, M)
    span = step(k) * task_orders(k)
    if k == TRI:
        return list(range(1, mlast + 1, span))
    if k == SPIN:
        return [mb for p in (0, 1) for mb in range(p, mlast + 1, span)]
    return [mb for p in (0, 1) for mb in range(2 + p, mlast + 1, span)]


def check(k, N, M, hi, shape, blk=0, spin=0, inplace=False):
    W, B, E = shape
    C, ST, WB = ch(k), step(k), shape[0] * shape[1]
    assert E <= PADPOS and E * C <= IDLEN
    L0 = (N + 1) // 2 if sphlike(k) else N
    copies = 0
    for mbase in tasks(k, M, spin):
        nsw, jlo, jhi = task_sweeps(k, M, mbase, blk, spin)
        if nsw == 0:
            continue
        npass = (nsw + WB - 1) // WB
        rem = nsw - (npass - 1) * WB
        for r in range(npass):
            copy_all = r == 0 and not inplace   # a first pass out of place copies the whole column
            s0 = (0 if r == 0 else rem + (r - 1) * WB) if hi else r * WB
            S = (rem if r == 0 else WB) if hi else min(WB, nsw - s0)
            WA = (S + B - 1) // B
            WAB = WA * B
            jfirst = jhi - ST * s0 if hi else jlo + ST * s0
            topc = [top(k, N, jfirst, c) for c in range(C)]
            ref = topc[0] if hi else 0
            emax = ref + S if hi else topc[0] + 1
            if copy_all or emax > L0 - 1:
                emax = L0 - 1
            emax = max(emax, 0)
            tstart = ref - emax if hi else -1
            tend = ref + 2 * WAB if hi else emax + 2 * WAB - 1
            K = (tend - tstart + 1 + E - 1) // E
            for q in range(WA):
                for b in range(B):
                    s = q * B + b
                    j = jfirst - ST * s if hi else jfirst + ST * s
                    lmax = -1
                    if s < S and 0 <= j < table_cols(k, N):
                        for c in range(C):
                            if top(k, N, j, c) >= 0:
                                lmax = max(lmax, C * top(k, N, j, c) + c)
                    # the former rule's valid steps, per chain
                    tlo, thi = [1, 1], [0, 0]
                    for c in range(2):
                        cc = c if c < C else 0
                        ts = top(k, N, jfirst, cc) + s if hi else top(k, N, jfirst, cc) - s
                        if hi:
                            tlo[c], thi[c] = ref + 2 * s - ts, ref + 2 * s
                        else:
                            tlo[c], thi[c] = 2 * s, 2 * s + ts
                        if not (s < S) or ts < 0:
                            tlo[c], thi[c] = 1, 0
                    for kp in range(K):
                        t0p = tstart + kp * E
                        ibase = ref + 2 * s - t0p - E + 1 if hi else t0p - 2 * s
                        copies += 1
                        lo, hi_l = C * ibase, C * ibase + C * E
                        if not (lmax >= 0 and lo <= lmax and hi_l > 0):
                            for c in range(2):   # the identity row: no entry of the chunk has a rotation
                                assert tlo[c] > thi[c] or all(not (tlo[c] <= t0p + u <= thi[c]) for u in range(E))
                            continue
                        length = table_base(k, N, j + 1) - table_base(k, N, j)
                        assert -pad_side(k) <= lo and hi_l <= length + pad_side(k), (k, N, hi, shape, mbase, r, s, kp, lo, hi_l)
                        for jj in range(E * C):
                            c = (jj & 1) if C == 2 else 0
                            u = (E - 1 - (jj >> 1 if C == 2 else jj)) if hi else (jj >> 1 if C == 2 else jj)
                            t = t0p + u
                            l = lo + jj
                            pad_valid = 0 <= l < length and (l // C) <= top(k, N, j, l % C)
                            old_valid = tlo[c] <= t <= thi[c]
                            assert pad_valid == old_valid, (k, N, hi, shape, mbase, r, s, kp, jj)
                            if old_valid:
                                i = ref + 2 * s - t if hi else t - 2 * s
                                assert l == (2 * i + c if C == 2 else i)
    return copies


CASES = [(SPH, n) for n in (2, 3, 5, 17, 64, 129, 300)] + [(TRI, n) for n in (2, 5, 33, 130, 257)] + \
        [(DISK, n) for n in (2, 3, 16, 65, 200)] + [(RECT, n) for n in (3, 40, 131)]


def default_M(k, n):
    return {SPH: 2 * n - 1, TRI: n, DISK: 4 * n - 3, RECT: n}[k]


@pytest.mark.parametrize("k,n", CASES)
def test_staging_copies_match_the_former_rule(k, n):
    shapes = [sh for sh in SHAPES if not (k in (TRI, RECT) and sh == (16, 4, 8))]
    for hi in (True, False):
        for sh in shapes:
            assert check(k, n, default_M(k, n), hi, sh) >= 0
            check(k, n, default_M(k, n), hi, sh, inplace=True)
            if k in (SPH, DISK, TRI) and n >= 64:
                check(k, n, default_M(k, n), hi, sh, blk=32)   # the blocked paths' heads


@pytest.mark.parametrize("n,M", [(17, 9), (64, 31), (64, 200), (33, 141)])
def test_staging_other_M(n, M):
    for hi in (True, False):
        check(SPH, n, M if M % 2 else M + 1, hi, (8, 8, 16))
        check(DISK, n, M if M % 2 else M + 1, hi, (8, 4, 16))


@pytest.mark.parametrize("n,s", [(5, 2), (40, -3), (64, 4), (130, 1)])
def test_staging_spin(n, s):
    for hi in (True, False):
        check(SPIN, n, 2 * n - 1, hi, (8, 4, 8), spin=abs(s))
