/* High-precision oracle -- TEST INFRASTRUCTURE ONLY (tests, __graft_entry__.smoke and bench.py's
 * CPU leg use it as a checker; nothing in the product links it).
 *
 * A __float128 (libquadmath, 113-bit significand) restatement of the reference's rotation
 * tables and default sweep kernels, so that the error of a double-precision result can be
 * measured against (nearly) exact arithmetic on the same operator:
 *   - the tables of ft_plan_rotsphere / ft_plan_rottriangle / ft_plan_rotdisk
 *     (src/rotations.c:116-133, 143-160, 173-190): s = sqrt(nums / den), c = sqrt(numc / den)
 *     with the integer (or parameter) products formed exactly in quad precision;
 *   - the default kernels kernel_{sph,tri,disk}_{hi2lo,lo2hi}_default
 *     (src/rotations/rotations_default.c:31-71): x' = c x + s y, y' = c y - s x (hi2lo), the
 *     transpose for lo2hi, sweeps in the reference's order;
 *   - for sph and disk, the forward transform 'N' (src/drivers.c:833-840, 989-994): the hi2lo
 *     sweeps, then the upper-triangular connection multiply of the column's stride-4 class
 *     (classes 0 and 3 with P[0], 1 and 2 with P[1]), with the plan's double-precision
 *     connection matrices given by the caller (the same numbers both sides use, so that only
 *     the arithmetic of the sweeps and of the multiply is measured).
 * The sweeps of a column involve only that column, and so does the class multiply, so any
 * subset of columns can be computed alone: each selected column's result is returned rounded
 * to double (hi) with its remainder (lo).  Columns run in parallel (OpenMP).
 *
 * The reference has no quad-precision sweeps (its FT_QUADMATH build, Make.inc:174-177, covers
 * the 1-D connection matrices); this file is checked against the double-precision oracle, the
 * compiled reference and an mpmath evaluation in tests/test_oracle_quad.py. */
#include <quadmath.h>
#include <stdlib.h>

typedef __float128 quad;

enum { Q_SPH = 0, Q_TRI = 1, Q_DISK = 2 };

/* (sin, cos) of entry l of sweep (table column) j */
static void table_entry(int kind, int n, double alpha, double beta, double gamma, int l, int j, quad * s, quad * c) {
    (void) n;
    quad nums, numc, den;
    if (kind == Q_SPH) {
        nums = (quad) ((long long) (l + 1) * (l + 2));
        numc = (quad) ((long long) (2 * j + 2) * (2 * l + 2 * j + 5));
        den = (quad) ((long long) (l + 2 * j + 3) * (l + 2 * j + 4));
        *s = sqrtq(nums / den);
        *c = sqrtq(numc / den);
    } else if (kind == Q_TRI) {
        const quad a = alpha, b = beta, g = gamma;
        nums = ((quad) l + 1) * ((quad) l + a + 1);
        numc = (2 * (quad) j + b + g + 2) * (2 * (quad) l + 2 * (quad) j + a + b + g + 4);
        den = ((quad) l + 2 * (quad) j + b + g + 3) * ((quad) l + 2 * (quad) j + a + b + g + 3);
        *s = sqrtq(nums / den);
        *c = sqrtq(numc / den);
    } else {
        const quad a = alpha, b = beta;
        nums = ((quad) l + 1) * ((quad) l + b + 1);
        numc = ((quad) j + a + 1) * (2 * (quad) l + (quad) j + a + b + 3);
        den = ((quad) l + (quad) j + a + 2) * ((quad) l + (quad) j + a + b + 2);
        *s = -sqrtq(nums / den);
        *c = sqrtq(numc / den);
    }
}

/* One column x (n entries) through the sweeps of order m, hi2lo or lo2hi. */
static void column_sweeps(int kind, int n, double alpha, double beta, double gamma, int m, int hi2lo, quad * x) {
    const int d = kind == Q_SPH ? 2 : 1;          /* rotated rows k and k + d */
    const int st = kind == Q_TRI ? 1 : 2;         /* order step between sweeps */
    const int jlo = kind == Q_TRI ? 0 : m % 2, jhi = m - st;
    if (jhi < jlo) return;
    const int nsw = (jhi - jlo) / st + 1;
    for (int t = 0; t < nsw; t++) {
        const int j = hi2lo ? jhi - st * t : jlo + st * t;
        const int K = kind == Q_SPH ? n - 3 - j : (kind == Q_TRI ? n - 2 - j : n - 2 - (j + 1) / 2);
        for (int u = 0; u <= K; u++) {
            const int k = hi2lo ? K - u : u;
            quad s, c;
            table_entry(kind, n, alpha, beta, gamma, k, j, &s, &c);
            const quad X = x[k], Y = x[k + d];
            if (hi2lo) { x[k] = c * X + s * Y; x[k + d] = c * Y - s * X; }
            else       { x[k] = c * X - s * Y; x[k + d] = c * Y + s * X; }
        }
    }
}

/* order of column col: sph and disk, columns 2m - 1 and 2m; tri, column m */
static int column_order(int kind, int col) { return kind == Q_TRI ? col : (col + 1) / 2; }

/* Selected columns cols[0 .. ncols-1] of the N x M column-major matrix A (leading dimension
 * lda): the rotation stage (P0 == NULL) or, for sph and disk, the forward transform 'N' with
 * the connection matrices P0, P1 (n x n column-major, upper triangles used).  hi2lo selects the
 * direction of the rotation stage (the transform always uses hi2lo).  Results rounded to double
 * in out_hi (N x ncols), the remainders in out_lo (may be NULL). */
int quad_columns(int kind, int n, double alpha, double beta, double gamma, const double * A, long long lda,
                 const int * cols, int ncols, int hi2lo, const double * P0, const double * P1, double * out_hi,
                 double * out_lo) {
    if (n < 1 || ncols < 0 || (P0 && kind == Q_TRI)) return -1;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int i = 0; i < ncols; i++) {
        quad * x = malloc(sizeof(quad) * (size_t) n);
        quad * y = malloc(sizeof(quad) * (size_t) n);
        if (!x || !y) { free(x); free(y); bad |= 1; continue; }
        const int col = cols[i];
        for (int k = 0; k < n; k++) x[k] = A[k + (long long) col * lda];
        column_sweeps(kind, n, alpha, beta, gamma, column_order(kind, col), P0 ? 1 : hi2lo, x);
        if (P0) {
            const int r = col % 4;
            const double * U = (r == 0 || r == 3) ? P0 : P1;
            for (int row = 0; row < n; row++) {
                quad acc = 0;
                for (int k = row; k < n; k++) acc += (quad) U[row + (long long) k * n] * x[k];
                y[row] = acc;
            }
        } else {
            for (int k = 0; k < n; k++) y[k] = x[k];
        }
        for (int k = 0; k < n; k++) {
            const double h = (double) y[k];
            out_hi[k + (long long) i * n] = h;
            if (out_lo) out_lo[k + (long long) i * n] = (double) (y[k] - (quad) h);
        }
        free(x);
        free(y);
    }
    return bad ? -2 : 0;
}

/* The tables' entries (j, l) for l = 0 .. len-1, rounded to double (hi) with remainders (lo). */
void quad_table_column(int kind, int n, double alpha, double beta, double gamma, int j, int len, double * s_hi,
                       double * s_lo, double * c_hi, double * c_lo) {
    for (int l = 0; l < len; l++) {
        quad s, c;
        table_entry(kind, n, alpha, beta, gamma, l, j, &s, &c);
        s_hi[l] = (double) s;
        s_lo[l] = (double) (s - (quad) s_hi[l]);
        c_hi[l] = (double) c;
        c_lo[l] = (double) (c - (quad) c_hi[l]);
    }
}
