/*
 * ft_oracle.c -- TEST INFRASTRUCTURE ONLY (see ft_oracle.h).
 *
 * CPU restatement of FastTransforms' harmonic-conversion path.  Every function
 * names the reference file:line it restates (paths relative to the reference
 * project root).  Where bit-for-bit agreement with the reference's plans is
 * wanted (the connection matrices are built in long double and rounded), the
 * arithmetic expressions keep the reference's association order.
 *
 * Build: make -C oracle  ->  oracle/_build/libft_oracle.so
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "ft_oracle.h"

#define MIN(a, b) ((a) < (b) ? (a) : (b))
#define MAX(a, b) ((a) > (b) ? (a) : (b))

static int g_fused = 1;
void oracle_set_fused(int fused) { g_fused = fused ? 1 : 0; }

/* ---------------------------------------------------------------------------
 * Rotation tables.
 * ------------------------------------------------------------------------- */

/* packed triangle index for sph / tri: src/rotations/rotations.h:6-7 */
static inline size_t tri_idx(int n, int l, int m) { return (size_t) l + (size_t) m * (2 * n + 1 - m) / 2; }
/* disk packing: src/rotations/rotations.h:9-10 */
static inline size_t disk_idx(int n, int l, int m) { return (size_t) l + (size_t) m * n - (size_t) (m / 2) * ((m + 1) / 2); }

/* src/rotations.c:116-133 (ft_plan_rotsphere) */
static void plan_rotsphere(int n, double * s, double * c) {
    for (int m = 0; m < n; m++)
        for (int l = 0; l < n - m; l++) {
            double nums = (l + 1) * (l + 2);
            double numc = (2 * m + 2) * (2 * l + 2 * m + 5);
            double den = (l + 2 * m + 3) * (l + 2 * m + 4);
            s[tri_idx(n, l, m)] = sqrt(nums / den);
            c[tri_idx(n, l, m)] = sqrt(numc / den);
        }
}

/* src/rotations.c:143-160 (ft_plan_rottriangle) */
static void plan_rottriangle(int n, double alpha, double beta, double gamma, double * s, double * c) {
    for (int m = 0; m < n; m++)
        for (int l = 0; l < n - m; l++) {
            double nums = (l + 1) * (l + alpha + 1);
            double numc = (2 * m + beta + gamma + 2) * (2 * l + 2 * m + alpha + beta + gamma + 4);
            double den = (l + 2 * m + beta + gamma + 3) * (l + 2 * m + alpha + beta + gamma + 3);
            s[tri_idx(n, l, m)] = sqrt(nums / den);
            c[tri_idx(n, l, m)] = sqrt(numc / den);
        }
}

/* src/rotations.c:173-190 (ft_plan_rotdisk); note the negated sine */
static void plan_rotdisk(int n, double alpha, double beta, double * s, double * c) {
    for (int m = 0; m < 2 * n - 1; m++)
        for (int l = 0; l < n - (m + 1) / 2; l++) {
            double nums = (l + 1) * (l + beta + 1);
            double numc = (m + alpha + 1) * (2 * l + m + alpha + beta + 3);
            double den = (l + m + alpha + 2) * (l + m + alpha + beta + 2);
            s[disk_idx(n, l, m)] = -sqrt(nums / den);
            c[disk_idx(n, l, m)] = sqrt(numc / den);
        }
}

/* src/rotations.c:270-287 (ft_plan_rotrectdisk): the sph packing, beta-dependent entries */
static void plan_rotrectdisk(int n, double beta, double * s, double * c) {
    for (int m = 0; m < n; m++)
        for (int l = 0; l < n - m; l++) {
            double nums = (l + 1) * (l + 2);
            double numc = (2 * m + 2 * beta + 3) * (2 * l + 2 * m + 2 * beta + 6);
            double den = (l + 2 * m + 2 * beta + 4) * (l + 2 * m + 2 * beta + 5);
            s[tri_idx(n, l, m)] = sqrt(nums / den);
            c[tri_idx(n, l, m)] = sqrt(numc / den);
        }
}

/* ---------------------------------------------------------------------------
 * Givens rotations: src/rotations/rotations_default.c:3-15 (scalar form) and
 * src/rotations/rotations_AVX512F.c:4-15 (fused form).
 * ------------------------------------------------------------------------- */

static inline void givens(double S, double C, double * X, double * Y) {
    double x0 = *X, y0 = *Y;
    if (g_fused) {
        double sy = S * y0, sx = S * x0;
        *X = fma(C, x0, sy);
        *Y = fma(C, y0, -sx);
    } else {
        double cx = C * x0, sy = S * y0, cy = C * y0, sx = S * x0;
        *X = cx + sy;
        *Y = cy - sx;
    }
}

static inline void givens_t(double S, double C, double * X, double * Y) {
    double x0 = *X, y0 = *Y;
    if (g_fused) {
        double sy = S * y0, sx = S * x0;
        *X = fma(C, x0, -sy);
        *Y = fma(C, y0, sx);
    } else {
        double cx = C * x0, sy = S * y0, cy = C * y0, sx = S * x0;
        *X = cx - sy;
        *Y = cy + sx;
    }
}

/* src/rotations/rotations_default.c:31-36 (sph), :45-50 (tri), :59-64 (disk), :73-78 (rect) */
void oracle_kernel_hi2lo(const oracle_plan * P, int m1, int m2, double * A, int S) {
    int n = P->n;
    const double * s = P->s, * c = P->c;
    if (P->kind == ORACLE_SPH || P->kind == ORACLE_RECT) {
        for (int j = m2 - 2; j >= m1; j -= 2)
            for (int k = n - 3 - j; k >= 0; k--)
                givens(s[tri_idx(n, k, j)], c[tri_idx(n, k, j)], A + k * S, A + (k + 2) * S);
    } else if (P->kind == ORACLE_TRI) {
        for (int j = m2 - 1; j >= m1; j--)
            for (int k = n - 2 - j; k >= 0; k--)
                givens(s[tri_idx(n, k, j)], c[tri_idx(n, k, j)], A + k * S, A + (k + 1) * S);
    } else {
        for (int j = m2 - 2; j >= m1; j -= 2)
            for (int k = n - 2 - (j + 1) / 2; k >= 0; k--)
                givens(s[disk_idx(n, k, j)], c[disk_idx(n, k, j)], A + k * S, A + (k + 1) * S);
    }
}

/* src/rotations/rotations_default.c:38-43 (sph), :52-57 (tri), :66-71 (disk), :80-85 (rect) */
void oracle_kernel_lo2hi(const oracle_plan * P, int m1, int m2, double * A, int S) {
    int n = P->n;
    const double * s = P->s, * c = P->c;
    if (P->kind == ORACLE_SPH || P->kind == ORACLE_RECT) {
        for (int j = m1; j < m2; j += 2)
            for (int k = 0; k <= n - 3 - j; k++)
                givens_t(s[tri_idx(n, k, j)], c[tri_idx(n, k, j)], A + k * S, A + (k + 2) * S);
    } else if (P->kind == ORACLE_TRI) {
        for (int j = m1; j < m2; j++)
            for (int k = 0; k <= n - 2 - j; k++)
                givens_t(s[tri_idx(n, k, j)], c[tri_idx(n, k, j)], A + k * S, A + (k + 1) * S);
    } else {
        for (int j = m1; j < m2; j += 2)
            for (int k = 0; k <= n - 2 - (j + 1) / 2; k++)
                givens_t(s[disk_idx(n, k, j)], c[disk_idx(n, k, j)], A + k * S, A + (k + 1) * S);
    }
}

/* Execute loops over orders: src/drivers.c:94-110 (sph), :314-326 (tri), :414-430 (disk).
 * Column pair (2m-1, 2m) carries order m for sph and disk; column m carries order m for tri. */
static void execute_rot(const oracle_plan * P, double * A, int M, int hi2lo) {
    int N = P->n;
    if (P->kind == ORACLE_RECT) {   /* src/drivers.c:496-508: order m on column m, m = 2 .. M-1 */
        #pragma omp parallel for schedule(dynamic, 1)
        for (int m = 2; m < M; m++) {
            if (hi2lo) oracle_kernel_hi2lo(P, m % 2, m, A + (size_t) N * m, 1);
            else       oracle_kernel_lo2hi(P, m % 2, m, A + (size_t) N * m, 1);
        }
        return;
    }
    if (P->kind == ORACLE_TRI) {
        #pragma omp parallel for schedule(dynamic, 1)
        for (int m = 1; m < M; m++) {
            if (hi2lo) oracle_kernel_hi2lo(P, 0, m, A + (size_t) N * m, 1);
            else       oracle_kernel_lo2hi(P, 0, m, A + (size_t) N * m, 1);
        }
    } else {
        #pragma omp parallel for schedule(dynamic, 1)
        for (int m = 2; m <= M / 2; m++) {
            for (int h = 0; h < 2; h++) {
                double * col = A + (size_t) N * (2 * m - 1 + h);
                if (hi2lo) oracle_kernel_hi2lo(P, m % 2, m, col, 1);
                else       oracle_kernel_lo2hi(P, m % 2, m, col, 1);
            }
        }
    }
}

void oracle_execute_hi2lo(const oracle_plan * P, double * A, int M) { execute_rot(P, A, M, 1); }
void oracle_execute_lo2hi(const oracle_plan * P, double * A, int M) { execute_rot(P, A, M, 0); }

/* ---------------------------------------------------------------------------
 * Triangular multiplies (the reference calls cblas_dtrmm with ColMajor, Upper,
 * NonUnit, alpha = 1; src/drivers.c:836-863, 924-956, 992-1019).
 * ------------------------------------------------------------------------- */
void oracle_trmm(char side, char trans, int n, const double * U, int nb, double * B, int ldb) {
    #define Uij(i, j) U[(size_t) (i) + (size_t) (j) * n]
    if (side == 'L') {
        /* B is n x nb: column by column */
        #pragma omp parallel
        {
            double * t = malloc(sizeof(double) * n);
            #pragma omp for schedule(static)
            for (int col = 0; col < nb; col++) {
                double * b = B + (size_t) col * ldb;
                for (int i = 0; i < n; i++) {
                    double acc = 0.0;
                    if (trans == 'N') for (int k = i; k < n; k++) acc += Uij(i, k) * b[k];
                    else              for (int k = 0; k <= i; k++) acc += Uij(k, i) * b[k];
                    t[i] = acc;
                }
                memcpy(b, t, sizeof(double) * n);
            }
            free(t);
        }
    } else {
        /* B is nb x n: row by row, B <- B op(U) */
        #pragma omp parallel
        {
            double * t = malloc(sizeof(double) * n);
            #pragma omp for schedule(static)
            for (int row = 0; row < nb; row++) {
                for (int j = 0; j < n; j++) {
                    double acc = 0.0;
                    if (trans == 'N') for (int k = 0; k <= j; k++) acc += B[row + (size_t) k * ldb] * Uij(k, j);
                    else              for (int k = j; k < n; k++) acc += B[row + (size_t) k * ldb] * Uij(j, k);
                    t[j] = acc;
                }
                for (int j = 0; j < n; j++) B[row + (size_t) j * ldb] = t[j];
            }
            free(t);
        }
    }
    #undef Uij
}

/* ---------------------------------------------------------------------------
 * Connection matrices in long double, rounded to double.
 * The triangular-banded generalised eigenvector method of the reference:
 * src/banded_source.c:779-800 (eigenvectors), :2024-2170 (diagonals),
 * :2316-2456 (A and B operators), :1774-1903 (Jacobi operators),
 * :288-343 (banded products and sums); planners in src/transforms.c:50-180.
 * A banded matrix here stores entry (i, j) for -l <= j - i <= u.
 * ------------------------------------------------------------------------- */

typedef long double ld;
#define LD_EPS 0x1p-64L   /* src/ftinternal.h:83 (M_EPSl) */

typedef struct { int n, l, u; ld * d; } bnd;

static bnd bnd_new(int n, int l, int u) {
    bnd A = { n, l, u, calloc((size_t) n * (l + u + 1), sizeof(ld)) };
    return A;
}
static inline ld bget(const bnd * A, int i, int j) {
    if (0 <= i && 0 <= j && -A->l <= j - i && j - i <= A->u && i < A->n && j < A->n)
        return A->d[(size_t) (A->u + i - j) + (size_t) j * (A->l + A->u + 1)];
    return 0;
}
static inline void bset(bnd * A, ld v, int i, int j) {
    if (0 <= i && 0 <= j && -A->l <= j - i && j - i <= A->u && i < A->n && j < A->n)
        A->d[(size_t) (A->u + i - j) + (size_t) j * (A->l + A->u + 1)] = v;
}

/* C <- alpha*A*B + beta*C: src/banded_source.c:288-305 */
static void bmm(ld alpha, const bnd * A, const bnd * B, ld beta, bnd * C) {
    int n = A->n;
    for (int j = 0; j < n; j++)
        for (int i = MAX(0, j - C->u); i < MIN(n, j + C->l + 1); i++) {
            ld ab = 0;
            for (int k = MAX(MAX(0, i - A->l), j - B->u); k < MIN(MIN(n, i + A->u + 1), j + B->l + 1); k++)
                ab += bget(A, i, k) * bget(B, k, j);
            ld c = bget(C, i, j);
            bset(C, alpha * ab + beta * c, i, j);
        }
}

/* C <- alpha*A + beta*B: src/banded_source.c:333-343 */
static void badd(ld alpha, const bnd * A, ld beta, const bnd * B, bnd * C) {
    int n = C->n;
    for (int j = 0; j < n; j++)
        for (int i = MAX(0, j - C->u); i < MIN(n, j + C->l + 1); i++)
            bset(C, alpha * bget(A, i, j) + beta * bget(B, i, j), i, j);
}

/* Generalised eigenvectors of upper-triangular banded (A, B), V pre-loaded with its diagonal:
 * src/banded_source.c:779-800 */
static void tb_eigenvectors(const bnd * A, const bnd * B, ld * V, int n) {
    int b = MAX(A->u, B->u);
    for (int j = 1; j < n; j++) {
        ld lam = bget(A, j, j) / bget(B, j, j);
        for (int i = j - 1; i >= 0; i--) {
            ld t = 0, kt = 0;
            for (int k = i + 1; k < MIN(i + b + 1, n); k++) {
                t += (bget(A, i, k) - lam * bget(B, i, k)) * V[k + (size_t) j * n];
                kt += (fabsl(bget(A, i, k)) + fabsl(lam * bget(B, i, k))) * fabsl(V[k + (size_t) j * n]);
            }
            ld d = lam * bget(B, i, i) - bget(A, i, i);
            ld kd = fabsl(lam * bget(B, i, i)) + fabsl(bget(A, i, i));
            if (fabsl(d) < 4 * kd * LD_EPS || fabsl(t) < 4 * kt * LD_EPS)
                V[i + (size_t) j * n] = 0;
            else
                V[i + (size_t) j * n] = t / d;
        }
    }
}

static double * finish_plan(bnd * A, bnd * B, ld * Vl, int n) {
    tb_eigenvectors(A, B, Vl, n);
    double * V = malloc(sizeof(double) * (size_t) n * n);
    for (size_t i = 0; i < (size_t) n * n; i++) V[i] = (double) Vl[i];
    free(A->d); free(B->d); free(Vl);
    return V;
}

#define ONE ((ld) 1)
#define TWO ((ld) 2)

/* src/banded_source.c:2316-2338 and :2024-2061; planner src/transforms.c:50-63 */
double * oracle_plan_legendre_to_chebyshev(int normleg, int normcheb, int n) {
    bnd A = bnd_new(n, 0, 2), B = bnd_new(n, 0, 2);
    if (n > 1) bset(&A, 2, 1, 1);
    for (int i = 2; i < n; i++) {
        bset(&A, -i * (i - ONE), i - 2, i);
        bset(&A, i * (i + ONE), i, i);
    }
    if (n > 0) bset(&B, normcheb ? sqrtl(2) : 2, 0, 0);
    if (n > 1) bset(&B, 1, 1, 1);
    for (int i = 2; i < n; i++) {
        bset(&B, -1, i - 2, i);
        bset(&B, 1, i, i);
    }
    ld * D = calloc((size_t) n * n, sizeof(ld));
    int inc = n + 1;
    if (normleg) {
        if (normcheb) {
            if (n > 0) D[0] = sqrtl(0.5) * tgammal(0.5);
            if (n > 1) D[inc] = sqrtl(1.5) * D[0];
            for (int i = 2; i < n; i++) D[i * inc] = sqrtl((2 * i + 1) * (2 * i - ONE)) * D[(i - 1) * inc] / (2 * i);
        } else {
            if (n > 0) D[0] = sqrtl(0.5);
            if (n > 1) D[inc] = sqrtl(1.5);
            for (int i = 2; i < n; i++) D[i * inc] = sqrtl((2 * i + 1) * (2 * i - ONE)) * D[(i - 1) * inc] / (2 * i);
        }
    } else {
        if (normcheb) {
            if (n > 0) D[0] = tgammal(0.5);
            if (n > 1) D[inc] = D[0] / sqrtl(2);
            for (int i = 2; i < n; i++) D[i * inc] = (2 * i - 1) * D[(i - 1) * inc] / (2 * i);
        } else {
            if (n > 0) D[0] = 1;
            if (n > 1) D[inc] = 1;
            for (int i = 2; i < n; i++) D[i * inc] = (2 * i - 1) * D[(i - 1) * inc] / (2 * i);
        }
    }
    return finish_plan(&A, &B, D, n);
}

/* src/banded_source.c:2340-2384 and :2063-2100; planner src/transforms.c:65-78 */
double * oracle_plan_chebyshev_to_legendre(int normcheb, int normleg, int n) {
    bnd A = bnd_new(n, 0, 2), B = bnd_new(n, 0, 2);
    if (normleg) {
        if (n > 1) bset(&A, sqrtl(TWO / 5), 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&A, -(i + 1) * sqrtl(((i - ONE) * i) / ((2 * i - ONE) * (2 * i + 1))) * (i + 1), i - 2, i);
            bset(&A, i * sqrtl(((i + ONE) * (i + 2)) / ((2 * i + ONE) * (2 * i + 3))) * i, i, i);
        }
        if (n > 0) bset(&B, sqrtl(TWO / 3), 0, 0);
        if (n > 1) bset(&B, sqrtl(TWO / 5), 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&B, -sqrtl(((i - ONE) * i) / ((2 * i - ONE) * (2 * i + 1))), i - 2, i);
            bset(&B, sqrtl(((i + ONE) * (i + 2)) / ((2 * i + ONE) * (2 * i + 3))), i, i);
        }
    } else {
        if (n > 1) bset(&A, ONE / 3, 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&A, -(i + 1) / (2 * i + ONE) * (i + 1), i - 2, i);
            bset(&A, i / (2 * i + ONE) * i, i, i);
        }
        if (n > 0) bset(&B, 1, 0, 0);
        if (n > 1) bset(&B, ONE / 3, 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&B, -1 / (2 * i + ONE), i - 2, i);
            bset(&B, 1 / (2 * i + ONE), i, i);
        }
    }
    ld * D = calloc((size_t) n * n, sizeof(ld));
    int inc = n + 1;
    if (normcheb) {
        if (normleg) {
            if (n > 0) D[0] = sqrtl(2) / tgammal(0.5);
            if (n > 1) D[inc] = D[0] / sqrtl(1.5);
            for (int i = 2; i < n; i++) D[i * inc] = (2 * i) / sqrtl((2 * i + 1) * (2 * i - ONE)) * D[(i - 1) * inc];
        } else {
            if (n > 0) D[0] = 1 / tgammal(0.5);
            if (n > 1) D[inc] = sqrtl(2) * D[0];
            for (int i = 2; i < n; i++) D[i * inc] = (2 * i) * D[(i - 1) * inc] / (2 * i - 1);
        }
    } else {
        if (normleg) {
            if (n > 0) D[0] = sqrtl(2);
            if (n > 1) D[inc] = 1 / sqrtl(1.5);
            for (int i = 2; i < n; i++) D[i * inc] = (2 * i) / sqrtl((2 * i + 1) * (2 * i - ONE)) * D[(i - 1) * inc];
        } else {
            if (n > 0) D[0] = 1;
            if (n > 1) D[inc] = 1;
            for (int i = 2; i < n; i++) D[i * inc] = (2 * i) * D[(i - 1) * inc] / (2 * i - 1);
        }
    }
    return finish_plan(&A, &B, D, n);
}

/* src/banded_source.c:2386-2430 and :2102-2131; planner src/transforms.c:80-93 */
double * oracle_plan_ultraspherical_to_ultraspherical(int norm1, int norm2, int n, double lambda_d, double mu_d) {
    ld lambda = lambda_d, mu = mu_d;
    bnd A = bnd_new(n, 0, 2), B = bnd_new(n, 0, 2);
    if (norm2) {
        if (n > 1) bset(&A, (1 + 2 * lambda) * copysignl(sqrtl((2 * mu + 1) / (2 * mu + 4)), mu), 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&A, -(i + 2 * mu) * (i + 2 * (mu - lambda)) * copysignl(sqrtl((i * (i - ONE)) / (4 * (i + mu) * (i + mu - 1))), mu), i - 2, i);
            bset(&A, i * (i + 2 * lambda) * copysignl(sqrtl(((i + 2 * mu) * (i + 2 * mu + 1)) / (4 * (i + mu) * (i + mu + 1))), mu), i, i);
        }
        if (n > 0) bset(&B, sqrtl((2 * mu + 1) / (2 * mu + 2)), 0, 0);
        if (n > 1) bset(&B, copysignl(sqrtl((2 * mu + 1) / (2 * mu + 4)), mu), 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&B, -copysignl(sqrtl((i * (i - ONE)) / (4 * (i + mu) * (i + mu - 1))), mu), i - 2, i);
            bset(&B, copysignl(sqrtl(((i + 2 * mu) * (i + 2 * mu + 1)) / (4 * (i + mu) * (i + mu + 1))), mu), i, i);
        }
    } else {
        if (n > 1) bset(&A, (1 + 2 * lambda) * mu / (1 + mu), 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&A, -(i + 2 * mu) * (i + 2 * (mu - lambda)) * mu / (i + mu), i - 2, i);
            bset(&A, i * (i + 2 * lambda) * mu / (i + mu), i, i);
        }
        if (n > 0) bset(&B, 1, 0, 0);
        if (n > 1) bset(&B, mu / (1 + mu), 1, 1);
        for (int i = 2; i < n; i++) {
            bset(&B, -mu / (i + mu), i - 2, i);
            bset(&B, mu / (i + mu), i, i);
        }
    }
    ld * D = calloc((size_t) n * n, sizeof(ld));
    int inc = n + 1;
    if (norm1) {
        if (norm2) {
            if (n > 0) D[0] = sqrtl(tgammal(lambda + 1) / (tgammal(0.5) * tgammal(lambda + 0.5))) * sqrtl(tgammal(0.5) * tgammal(mu + 0.5) / tgammal(mu + 1));
            for (int i = 1; i < n; i++)
                D[i * inc] = sqrtl((i - 1 + mu) / i * (i - 1 + 2 * mu) / (i + mu)) * sqrtl(i / (i - 1 + lambda) * (i + lambda) / (i - 1 + 2 * lambda)) * (i - 1 + lambda) / (i - 1 + mu) * D[(i - 1) * inc];
        } else {
            if (n > 0) D[0] = sqrtl(tgammal(lambda + 1) / (tgammal(0.5) * tgammal(lambda + 0.5)));
            for (int i = 1; i < n; i++)
                D[i * inc] = sqrtl(i / (i - 1 + lambda) * (i + lambda) / (i - 1 + 2 * lambda)) * (i - 1 + lambda) / (i - 1 + mu) * D[(i - 1) * inc];
        }
    } else {
        if (norm2) {
            if (n > 0) D[0] = sqrtl(tgammal(0.5) * tgammal(mu + 0.5) / tgammal(mu + 1));
            for (int i = 1; i < n; i++)
                D[i * inc] = sqrtl((i - 1 + mu) / i * (i - 1 + 2 * mu) / (i + mu)) * (i - 1 + lambda) / (i - 1 + mu) * D[(i - 1) * inc];
        } else {
            if (n > 0) D[0] = 1;
            for (int i = 1; i < n; i++) D[i * inc] = (i - 1 + lambda) / (i - 1 + mu) * D[(i - 1) * inc];
        }
    }
    return finish_plan(&A, &B, D, n);
}

/* Jacobi operators (normalized forms used by the harmonic planners: norm = 1).
 * derivative: src/banded_source.c:1774-1795 */
static bnd jacobi_derivative(int norm, int n, int order, ld alpha, ld beta) {
    bnd A = bnd_new(n, -order, order);
    for (int j = order; j < n; j++) {
        ld v = 1;
        if (norm) {
            for (int k = 0; k < order; k++) v *= (j - k) * (j + alpha + beta + k + 1);
            v = sqrtl(v);
        } else {
            for (int k = 0; k < order; k++) v *= (j + alpha + beta + k + 1) / 2;
        }
        bset(&A, v, j - order, j);
    }
    return A;
}

/* multiplication by x: src/banded_source.c:1797-1841 (norm = 1 branch) */
static bnd jacobi_multiplication(int n, ld alpha, ld beta) {
    bnd A = bnd_new(n, 1, 1);
    for (int j = 0; j < n; j++) {
        ld v;
        if (j == 1)
            v = 2 * sqrtl(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 2) * (alpha + beta + 3)));
        else
            v = 2 * sqrtl((j * (j + alpha) * (j + beta) * (j + alpha + beta)) / ((2 * j + alpha + beta - 1) * (2 * j + alpha + beta) * (2 * j + alpha + beta) * (2 * j + alpha + beta + 1)));
        bset(&A, v, j - 1, j);
        if (j == 0) {
            v = (beta - alpha) / (alpha + beta + 2);
            bset(&A, v, 0, 0);
            v = 2 * sqrtl(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 2) * (alpha + beta + 3)));
            bset(&A, v, 1, 0);
        } else {
            v = ((beta - alpha) * (alpha + beta)) / ((2 * j + alpha + beta) * (2 * j + alpha + beta + 2));
            bset(&A, v, j, j);
            v = 2 * sqrtl(((j + 1) * (j + alpha + 1) * (j + beta + 1) * (j + alpha + beta + 1)) / ((2 * j + alpha + beta + 1) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 3)));
            bset(&A, v, j + 1, j);
        }
    }
    return A;
}

/* raising: src/banded_source.c:1843-1873 (norm = 1 branch) */
static bnd jacobi_raising(int n, ld alpha, ld beta) {
    bnd A = bnd_new(n, 0, 2);
    for (int j = 0; j < n; j++) {
        ld v = -2 * sqrtl(((j - 1) * j * (j + alpha) * (j + beta)) / ((2 * j + alpha + beta - 1) * (2 * j + alpha + beta) * (2 * j + alpha + beta) * (2 * j + alpha + beta + 1)));
        bset(&A, v, j - 2, j);
        v = 2 * (alpha - beta) * sqrtl(j * (j + alpha + beta + 1)) / ((2 * j + alpha + beta) * (2 * j + alpha + beta + 2));
        bset(&A, v, j - 1, j);
        if (j == 0)
            v = 2 * sqrtl(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 3)));
        else
            v = 2 * sqrtl(((j + alpha + 1) * (j + beta + 1) * (j + alpha + beta + 1) * (j + alpha + beta + 2)) / ((2 * j + alpha + beta + 1) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 3)));
        bset(&A, v, j, j);
    }
    return A;
}

/* lowering: src/banded_source.c:1875-1903 (norm = 1 branch) */
static bnd jacobi_lowering(int n, ld alpha, ld beta) {
    bnd A = bnd_new(n, 2, 0);
    for (int j = 0; j < n; j++) {
        ld v;
        if (j == 0)
            v = 2 * sqrtl(((alpha + 1) * (beta + 1)) / ((alpha + beta + 2) * (alpha + beta + 3)));
        else
            v = 2 * sqrtl(((j + alpha + 1) * (j + beta + 1) * (j + alpha + beta + 1) * (j + alpha + beta + 2)) / ((2 * j + alpha + beta + 1) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 3)));
        bset(&A, v, j, j);
        v = 2 * (alpha - beta) * sqrtl((j + 1) * (j + alpha + beta + 2)) / ((2 * j + alpha + beta + 2) * (2 * j + alpha + beta + 4));
        bset(&A, v, j + 1, j);
        v = -2 * sqrtl(((j + 1) * (j + 2) * (j + alpha + 2) * (j + beta + 2)) / ((2 * j + alpha + beta + 3) * (2 * j + alpha + beta + 4) * (2 * j + alpha + beta + 4) * (2 * j + alpha + beta + 5)));
        bset(&A, v, j + 2, j);
    }
    return A;
}

/* A = sigma D^2 + tau D for the Jacobi-Jacobi problem: src/banded_source.c:2432-2451;
 * B = raising: :2453-2456; diagonal: :2133-2142 (norm1 = norm2 = 1);
 * planner src/transforms.c:95-108.  Only the normalized-to-normalized form is
 * used by the tri and disk planners (src/drivers.c:905-910, 963-968). */
double * oracle_plan_jacobi_to_jacobi(int norm1, int norm2, int n, double alpha_d, double beta_d, double gamma_d, double delta_d) {
    (void) norm1; (void) norm2;  /* harmonic planners pass norm1 = norm2 = 1 */
    ld alpha = alpha_d, beta = beta_d, gamma = gamma_d, delta = delta_d;
    bnd A = bnd_new(n, 0, 2);
    bnd D1 = jacobi_derivative(1, n, 1, gamma, delta);
    bnd D2 = jacobi_derivative(1, n, 2, gamma, delta);
    bnd L1 = jacobi_lowering(n, gamma + 1, delta + 1);
    bnd M1 = jacobi_multiplication(n, gamma + 1, delta + 1);
    bmm(-1, &L1, &D2, 0, &A);
    badd(1, &A, alpha - beta, &D1, &A);
    bmm(alpha + beta + 2, &M1, &D1, 1, &A);
    free(D1.d); free(D2.d); free(L1.d); free(M1.d);
    bnd B = jacobi_raising(n, gamma, delta);
    ld * D = calloc((size_t) n * n, sizeof(ld));
    int inc = n + 1;
    if (n > 0)
        D[0] = sqrtl(tgammal(alpha + beta + 2) / (powl(2, alpha + beta + 1) * tgammal(alpha + 1) * tgammal(beta + 1)) * (powl(2, gamma + delta + 1) * tgammal(gamma + 1) * tgammal(delta + 1)) / tgammal(gamma + delta + 2));
    if (n > 1)
        D[inc] = (alpha + beta + 2) / (gamma + delta + 2) * sqrtl((alpha + beta + 3) / ((alpha + 1) * (beta + 1)) * ((gamma + 1) * (delta + 1)) / (gamma + delta + 3)) * D[0];
    for (int i = 2; i < n; i++)
        D[i * inc] = (2 * i + alpha + beta) / (2 * i + gamma + delta) * sqrtl(((2 * i + alpha + beta - 1) * (2 * i + alpha + beta + 1)) / ((i + alpha) * (i + beta) * (i + alpha + beta)) * ((i + gamma) * (i + delta) * (i + gamma + delta)) / ((2 * i + gamma + delta - 1) * (2 * i + gamma + delta + 1))) * D[(i - 1) * inc];
    return finish_plan(&A, &B, D, n);
}

/* ---------------------------------------------------------------------------
 * Plans and full transforms.
 * ------------------------------------------------------------------------- */

oracle_plan * oracle_plan_rotations(int kind, int n, double alpha, double beta, double gamma) {
    oracle_plan * P = calloc(1, sizeof(oracle_plan));
    P->kind = kind; P->n = n;
    P->alpha = alpha; P->beta = beta; P->gamma = gamma;
    size_t len = kind == ORACLE_DISK ? (size_t) n * n : (size_t) n * (n + 1) / 2;
    P->s = calloc(len ? len : 1, sizeof(double));
    P->c = calloc(len ? len : 1, sizeof(double));
    if (kind == ORACLE_SPH) plan_rotsphere(n, P->s, P->c);
    else if (kind == ORACLE_TRI) plan_rottriangle(n, alpha, beta, gamma, P->s, P->c);
    else if (kind == ORACLE_RECT) plan_rotrectdisk(n, beta, P->s, P->c);
    else plan_rotdisk(n, alpha, beta, P->s, P->c);
    return P;
}

/* src/drivers.c:816-831 */
oracle_plan * oracle_plan_sph2fourier(int n) {
    oracle_plan * P = oracle_plan_rotations(ORACLE_SPH, n, 0, 0, 0);
    P->P[0] = oracle_plan_legendre_to_chebyshev(1, 0, n);
    P->P[1] = oracle_plan_ultraspherical_to_ultraspherical(1, 0, n, 1.5, 1.0);
    P->Pinv[0] = oracle_plan_chebyshev_to_legendre(0, 1, n);
    P->Pinv[1] = oracle_plan_ultraspherical_to_ultraspherical(0, 1, n, 1.0, 1.5);
    return P;
}

/* src/drivers.c:901-919 */
oracle_plan * oracle_plan_tri2cheb(int n, double alpha, double beta, double gamma) {
    oracle_plan * P = oracle_plan_rotations(ORACLE_TRI, n, alpha, beta, gamma);
    P->P[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, beta + gamma + 1.0, alpha, -0.5, -0.5);
    P->P[1] = oracle_plan_jacobi_to_jacobi(1, 1, n, gamma, beta, -0.5, -0.5);
    P->Pinv[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, beta + gamma + 1.0, alpha);
    P->Pinv[1] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, gamma, beta);
    return P;
}

/* src/drivers.c:959-987, with plan_jacobi_to_chebyshev / plan_chebyshev_to_jacobi
 * (src/transforms.c:157-180) inlined: row / column scalings by sqrt(2/pi), sqrt(1/pi) etc. */
oracle_plan * oracle_plan_disk2cxf(int n, double alpha, double beta) {
    oracle_plan * P = oracle_plan_rotations(ORACLE_DISK, n, alpha, beta, 0);
    P->P[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, beta, alpha, -0.5, -0.5);
    P->P[1] = oracle_plan_jacobi_to_jacobi(1, 1, n, beta, alpha + 1.0, -0.5, 0.5);
    P->Pinv[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, beta, alpha);
    P->Pinv[1] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, 0.5, beta, alpha + 1.0);
    double * sclrow = malloc(sizeof(double) * (n ? n : 1));
    double * sclcol = malloc(sizeof(double) * (n ? n : 1));
    for (int i = 0; i < n; i++) {
        sclrow[i] = i ? sqrtl(M_2_PIl) : sqrtl(M_1_PIl);
        sclcol[i] = i ? sqrtl(M_PI_2l) : sqrtl(M_PIl);
    }
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) {
            P->P[0][i + (size_t) j * n] *= sclrow[i];
            P->Pinv[0][i + (size_t) j * n] *= sclcol[j];
        }
    free(sclrow); free(sclcol);
    double cst0 = pow(2.0, 0.5 * (alpha + beta + 2.0));
    double cst1 = cst0 * 0.797884560802865355;      /* sqrt(2/pi), src/ftinternal.h:66 */
    double cst0inv = pow(2.0, -0.5 * (alpha + beta + 2.0));
    double cst1inv = cst0inv * 1.253314137315500251; /* sqrt(pi/2), src/ftinternal.h:65 */
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) {
            P->P[0][i + (size_t) j * n] *= cst0;
            P->P[1][i + (size_t) j * n] *= cst1;
            P->Pinv[0][i + (size_t) j * n] *= cst0inv;
            P->Pinv[1][i + (size_t) j * n] *= cst1inv;
        }
    return P;
}

/* plan_ultraspherical_to_chebyshev(1, 0, n, lambda) (src/transforms.c:185-197): the normalised
 * Jacobi connection (lambda - 1/2, lambda - 1/2) -> (-1/2, -1/2), entries i = j, j - 2, .. of
 * row i scaled to the unnormalised Chebyshev basis */
static double * ultraspherical_to_chebyshev(int n, double lambda) {
    double * V = oracle_plan_jacobi_to_jacobi(1, 1, n, lambda - 0.5, lambda - 0.5, -0.5, -0.5);
    for (int j = 0; j < n; j++)
        for (int i = j; i >= 0; i -= 2) {
            double r = i ? sqrtl(M_2_PIl) : sqrtl(M_1_PIl);
            V[i + (size_t) j * n] *= r;
        }
    return V;
}

/* plan_chebyshev_to_ultraspherical(0, 1, n, lambda) (src/transforms.c:199-211) */
static double * chebyshev_to_ultraspherical(int n, double lambda) {
    double * V = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, lambda - 0.5, lambda - 0.5);
    for (int j = 0; j < n; j++) {
        double r = j ? sqrtl(M_PI_2l) : sqrtl(M_PIl);
        for (int i = j; i >= 0; i -= 2) V[i + (size_t) j * n] *= r;
    }
    return V;
}

/* src/drivers.c:1123-1141 */
oracle_plan * oracle_plan_rectdisk2cheb(int n, double beta) {
    oracle_plan * P = oracle_plan_rotations(ORACLE_RECT, n, 0, beta, 0);
    P->P[0] = ultraspherical_to_chebyshev(n, beta + 1.0);
    P->P[1] = oracle_plan_ultraspherical_to_ultraspherical(1, 0, n, beta + 2.0, 1.0);
    P->P[2] = ultraspherical_to_chebyshev(n, beta + 0.5);
    P->Pinv[0] = chebyshev_to_ultraspherical(n, beta + 1.0);
    P->Pinv[1] = oracle_plan_ultraspherical_to_ultraspherical(0, 1, n, 1.0, beta + 2.0);
    P->Pinv[2] = chebyshev_to_ultraspherical(n, beta + 0.5);
    return P;
}

void oracle_destroy_plan(oracle_plan * P) {
    if (!P) return;
    free(P->s); free(P->c);
    for (int i = 0; i < 3; i++) { free(P->P[i]); free(P->Pinv[i]); }
    free(P);
}

/* src/drivers.c:6-24 */
static void cheb_normalize(double * A, int N, int M, int transposed) {
    double r = transposed ? M_SQRT2 : M_SQRT1_2;
    double g = transposed ? M_PI_2 : M_2_PI;
    for (int i = 0; i < N; i++) A[i] *= r;
    for (int j = 0; j < M; j++) {
        A[(size_t) j * N] *= r;
        for (int i = 0; i < N; i++) A[i + (size_t) j * N] *= g;
    }
}

/* Four stride-4N column classes: j = 0,3 (mod 4) use U0; j = 1,2 (mod 4) use U1.
 * src/drivers.c:836-839 */
static void trmm4(char trans, int N, int M, const double * U0, const double * U1, double * A) {
    oracle_trmm('L', trans, N, U0, (M + 3) / 4, A, 4 * N);
    oracle_trmm('L', trans, N, U1, (M + 2) / 4, A + N, 4 * N);
    oracle_trmm('L', trans, N, U1, (M + 1) / 4, A + 2 * N, 4 * N);
    oracle_trmm('L', trans, N, U0, M / 4, A + 3 * N, 4 * N);
}

/* src/drivers.c:833-865 (sph), :921-957 (tri), :989-1021 (disk) */
void oracle_execute(const oracle_plan * P, int forward, char TRANS, double * A, int N, int M) {
    if (TRANS != 'N' && TRANS != 'T') return;
    int tN = TRANS == 'N';
    if (P->kind == ORACLE_RECT) {   /* src/drivers.c:1143-1171; M == N (the right multiply is n x n) */
        double * const * U = forward ? P->P : P->Pinv;
        if ((forward && tN) || (!forward && !tN)) {
            char t = forward ? 'N' : 'T';
            oracle_execute_hi2lo(P, A, M);
            oracle_trmm('L', t, N, U[0], (M + 1) / 2, A, 2 * N);
            oracle_trmm('L', t, N, U[1], M / 2, A + N, 2 * N);
            oracle_trmm('R', forward ? 'T' : 'N', N, U[2], N, A, N);
        } else {
            char t = forward ? 'T' : 'N';
            oracle_trmm('R', forward ? 'N' : 'T', N, U[2], N, A, N);
            oracle_trmm('L', t, N, U[0], (M + 1) / 2, A, 2 * N);
            oracle_trmm('L', t, N, U[1], M / 2, A + N, 2 * N);
            oracle_execute_lo2hi(P, A, M);
        }
        return;
    }
    if (P->kind == ORACLE_TRI) {
        double a = P->alpha, b = P->beta, g = P->gamma;
        int left = (b + g != -1.5) || (a != -0.5);
        int right = (g != -0.5) || (b != -0.5);
        if (forward && tN) {
            oracle_execute_hi2lo(P, A, M);
            if (left) oracle_trmm('L', 'N', N, P->P[0], M, A, N);
            if (right) oracle_trmm('R', 'T', N, P->P[1], N, A, N);
            cheb_normalize(A, N, M, 0);
        } else if (forward) {
            cheb_normalize(A, N, M, 0);
            if (right) oracle_trmm('R', 'N', N, P->P[1], N, A, N);
            if (left) oracle_trmm('L', 'T', N, P->P[0], M, A, N);
            oracle_execute_lo2hi(P, A, M);
        } else if (tN) {
            cheb_normalize(A, N, M, 1);
            if (right) oracle_trmm('R', 'T', N, P->Pinv[1], N, A, N);
            if (left) oracle_trmm('L', 'N', N, P->Pinv[0], M, A, N);
            oracle_execute_lo2hi(P, A, M);
        } else {
            oracle_execute_hi2lo(P, A, M);
            if (left) oracle_trmm('L', 'T', N, P->Pinv[0], M, A, N);
            if (right) oracle_trmm('R', 'N', N, P->Pinv[1], N, A, N);
            cheb_normalize(A, N, M, 1);
        }
        return;
    }
    /* sph and disk share the execute structure */
    if (forward && tN) {
        oracle_execute_hi2lo(P, A, M);
        trmm4('N', N, M, P->P[0], P->P[1], A);
    } else if (forward) {
        trmm4('T', N, M, P->P[0], P->P[1], A);
        oracle_execute_lo2hi(P, A, M);
    } else if (tN) {
        trmm4('N', N, M, P->Pinv[0], P->Pinv[1], A);
        oracle_execute_lo2hi(P, A, M);
    } else {
        oracle_execute_hi2lo(P, A, M);
        trmm4('T', N, M, P->Pinv[0], P->Pinv[1], A);
    }
}

/* sph vector fields (src/drivers.c:198-214, 867-899): order m's sweeps on the column pair
 * (2m+1, 2m+2) for m = 2 .. M/2-1, and P[0] / P[1] swapped in the four column classes. */
static void execute_rot_sphv(const oracle_plan * P, double * A, int M, int hi2lo) {
    int N = P->n;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int m = 2; m <= M / 2 - 1; m++) {
        for (int h = 0; h < 2; h++) {
            double * col = A + (size_t) N * (2 * m + 1 + h);
            if (hi2lo) oracle_kernel_hi2lo(P, m % 2, m, col, 1);
            else       oracle_kernel_lo2hi(P, m % 2, m, col, 1);
        }
    }
}

void oracle_execute_sphv(const oracle_plan * P, int forward, char TRANS, double * A, int N, int M) {
    if (TRANS != 'N' && TRANS != 'T') return;
    int tN = TRANS == 'N';
    if (forward && tN) {
        execute_rot_sphv(P, A, M, 1);
        trmm4('N', N, M, P->P[1], P->P[0], A);
    } else if (forward) {
        trmm4('T', N, M, P->P[1], P->P[0], A);
        execute_rot_sphv(P, A, M, 0);
    } else if (tN) {
        trmm4('N', N, M, P->Pinv[1], P->Pinv[0], A);
        execute_rot_sphv(P, A, M, 0);
    } else {
        execute_rot_sphv(P, A, M, 1);
        trmm4('T', N, M, P->Pinv[1], P->Pinv[0], A);
    }
}

/* ---------------------------------------------------------------------------
 * Seeded fills.  Counter-based splitmix64: value(idx) for the entry at linear
 * column-major index idx = i + j*N is 2*u - 1 with u the top 53 bits of
 * mix(seed + (idx + 1) * 0x9E3779B97F4A7C15) / 2^53.  Entries outside the
 * layout's triangle are zero (src/ftutilities.c:75-113).
 * ------------------------------------------------------------------------- */
static inline double u_pm1(unsigned long long seed, unsigned long long idx) {
    unsigned long long z = seed + (idx + 1ULL) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return 2.0 * ((double) (z >> 11) * 0x1p-53) - 1.0;
}

void oracle_fill(int kind, int N, int M, unsigned long long seed, double * A) {
    for (int j = 0; j < M; j++)
        for (int i = 0; i < N; i++) {
            int on = kind == ORACLE_SPH ? (j < M - 2 * i) : (kind == ORACLE_TRI || kind == ORACLE_RECT) ? (j < M - i) : (j < M - 4 * i);
            size_t idx = (size_t) i + (size_t) j * N;
            A[idx] = on ? u_pm1(seed, idx) : 0.0;
        }
}

/* ---------------------------------------------------------------------------
 * Spin-weighted spherical harmonics.  Complex matrices are interleaved (re, im)
 * doubles, column-major N x M (ft_complex, src/fasttransforms.h:11).
 * ------------------------------------------------------------------------- */

/* src/rotations.c:445-478 (ft_plan_rotspinsphere): s1, c1 are the sph table (same
 * expression); s2, c2 indexed (l, j, m) at l + j n + m |s| n. */
oracle_spin_plan * oracle_plan_spinsph2fourier(int n, int s, int connections) {
    oracle_spin_plan * P = calloc(1, sizeof(oracle_spin_plan));
    P->n = n;
    P->s = s;
    P->sph = connections ? oracle_plan_sph2fourier(n) : oracle_plan_rotations(ORACLE_SPH, n, 0, 0, 0);
    int as = abs(s);
    P->s2 = calloc((size_t) as * n * n + 1, sizeof(double));
    P->c2 = calloc((size_t) as * n * n + 1, sizeof(double));
    for (int m = 0; m < n; m++)
        for (int j = 0; j < as; j++)
            for (int l = 0; l < n - m - j; l++) {
                double nums = (l + 1) * (l + m + 1);
                double numc = (2 * j + m + 1) * (2 * l + 2 * j + 2 * m + 3);
                double den = (l + 2 * j + m + 2) * (l + 2 * j + 2 * m + 2);
                size_t idx = (size_t) l + (size_t) j * n + (size_t) m * as * n;
                P->s2[idx] = sqrt(nums / den);
                P->c2[idx] = sqrt(numc / den);
            }
    return P;
}

void oracle_destroy_spin_plan(oracle_spin_plan * P) {
    if (!P) return;
    oracle_destroy_plan(P->sph);
    free(P->s2);
    free(P->c2);
    free(P);
}

/* src/rotations/rotations_default.c:17-29: the real rotation on both parts */
static inline void cgivens(double S, double C, double * X, double * Y) { givens(S, C, X, Y); givens(S, C, X + 1, Y + 1); }
static inline void cgivens_t(double S, double C, double * X, double * Y) { givens_t(S, C, X, Y); givens_t(S, C, X + 1, Y + 1); }

#define SPIN_S2(P, l, j, m) (P)->s2[(size_t) (l) + (size_t) (j) * (P)->n + (size_t) (m) * abs((P)->s) * (P)->n]
#define SPIN_C2(P, l, j, m) (P)->c2[(size_t) (l) + (size_t) (j) * (P)->n + (size_t) (m) * abs((P)->s) * (P)->n]

/* src/rotations/rotations_default.c:87-101 (kernel_spinsph_hi2lo_default); A: one complex column */
void oracle_kernel_spinsph_hi2lo(const oracle_spin_plan * P, int m, double * A) {
    int n = P->n, s = P->s, as = abs(s), am = abs(m), d = abs(am - as);
    const double * s1 = P->sph->s, * c1 = P->sph->c;
    for (int j = MIN(am, as) - 1; j >= 0; j--)
        for (int k = n - 2 - d - j; k >= 0; k--) {
            if (m * s >= 0) cgivens(SPIN_S2(P, k, j, d), SPIN_C2(P, k, j, d), A + 2 * k, A + 2 * (k + 1));
            else            cgivens_t(SPIN_S2(P, k, j, d), SPIN_C2(P, k, j, d), A + 2 * k, A + 2 * (k + 1));
        }
    for (int j = d - 2; j >= (am + as) % 2; j -= 2)
        for (int k = n - 3 - j; k >= 0; k--)
            cgivens(s1[tri_idx(n, k, j)], c1[tri_idx(n, k, j)], A + 2 * k, A + 2 * (k + 2));
}

/* src/rotations/rotations_default.c:103-117 (kernel_spinsph_lo2hi_default) */
void oracle_kernel_spinsph_lo2hi(const oracle_spin_plan * P, int m, double * A) {
    int n = P->n, s = P->s, as = abs(s), am = abs(m), d = abs(am - as);
    const double * s1 = P->sph->s, * c1 = P->sph->c;
    for (int j = (am + as) % 2; j <= d - 2; j += 2)
        for (int k = 0; k <= n - 3 - j; k++)
            cgivens_t(s1[tri_idx(n, k, j)], c1[tri_idx(n, k, j)], A + 2 * k, A + 2 * (k + 2));
    for (int j = 0; j < MIN(am, as); j++)
        for (int k = 0; k <= n - 2 - d - j; k++) {
            if (m * s >= 0) cgivens_t(SPIN_S2(P, k, j, d), SPIN_C2(P, k, j, d), A + 2 * k, A + 2 * (k + 1));
            else            cgivens(SPIN_S2(P, k, j, d), SPIN_C2(P, k, j, d), A + 2 * k, A + 2 * (k + 1));
        }
}

/* src/drivers.c:677-695: column 0 is order 0, columns 2m - 1 and 2m orders -m and m */
static void execute_spin_rot(const oracle_spin_plan * P, double * A, int M, int hi2lo) {
    int N = P->n;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < M; c++) {
        int m = c == 0 ? 0 : (c % 2 ? -(c + 1) / 2 : c / 2);
        double * col = A + (size_t) 2 * N * c;
        if (hi2lo) oracle_kernel_spinsph_hi2lo(P, m, col);
        else       oracle_kernel_spinsph_lo2hi(P, m, col);
    }
}

void oracle_execute_spinsph_hi2lo(const oracle_spin_plan * P, double * A, int M) { execute_spin_rot(P, A, M, 1); }
void oracle_execute_spinsph_lo2hi(const oracle_spin_plan * P, double * A, int M) { execute_spin_rot(P, A, M, 0); }

/* cblas_ztrmm with a real matrix stored as complex (src/drivers.c:1295-1361): the real
 * triangular multiply on the real and the imaginary parts */
static void ztrmm4(char trans, int N, int M, const double * U0, const double * U1, double * A) {
    size_t nm = (size_t) N * M;
    double * re = malloc(sizeof(double) * nm), * im = malloc(sizeof(double) * nm);
    for (size_t i = 0; i < nm; i++) { re[i] = A[2 * i]; im[i] = A[2 * i + 1]; }
    trmm4(trans, N, M, U0, U1, re);
    trmm4(trans, N, M, U0, U1, im);
    for (size_t i = 0; i < nm; i++) { A[2 * i] = re[i]; A[2 * i + 1] = im[i]; }
    free(re);
    free(im);
}

/* src/drivers.c:1295-1361 (ft_execute_spinsph2fourier / ft_execute_fourier2spinsph):
 * classes 0, 3 take P1 and 1, 2 take P2 for even s, the other way round for odd s */
void oracle_execute_spin(const oracle_spin_plan * P, int forward, char TRANS, double * A, int N, int M) {
    if (TRANS != 'N' && TRANS != 'T') return;
    int even = P->s % 2 == 0;
    const double * U0 = even ? P->sph->P[0] : P->sph->P[1], * U1 = even ? P->sph->P[1] : P->sph->P[0];
    const double * V0 = even ? P->sph->Pinv[0] : P->sph->Pinv[1], * V1 = even ? P->sph->Pinv[1] : P->sph->Pinv[0];
    int tN = TRANS == 'N';
    if (forward && tN) {
        oracle_execute_spinsph_hi2lo(P, A, M);
        ztrmm4('N', N, M, U0, U1, A);
    } else if (forward) {
        ztrmm4('T', N, M, U0, U1, A);
        oracle_execute_spinsph_lo2hi(P, A, M);
    } else if (tN) {
        ztrmm4('N', N, M, V0, V1, A);
        oracle_execute_spinsph_lo2hi(P, A, M);
    } else {
        oracle_execute_spinsph_hi2lo(P, A, M);
        ztrmm4('T', N, M, V0, V1, A);
    }
}

/* spinsphrand's layout (src/ftutilities.c:159-167): rows i < N - |s|, columns j < M - 2i,
 * both parts U(-1,1) from the counter at the double index */
void oracle_fill_spin(int N, int M, int s, unsigned long long seed, double * A) {
    for (int j = 0; j < M; j++)
        for (int i = 0; i < N; i++) {
            size_t e = (size_t) i + (size_t) j * N;
            int on = i < N - abs(s) && j < M - 2 * i;
            A[2 * e] = on ? u_pm1(seed, 2 * e) : 0.0;
            A[2 * e + 1] = on ? u_pm1(seed, 2 * e + 1) : 0.0;
        }
}

/* ---------------------------------------------------------------------------
 * Tetrahedral harmonics.
 * ------------------------------------------------------------------------- */

/* src/drivers.c:1173-1195 */
oracle_tet_plan * oracle_plan_tet2cheb(int n, double alpha, double beta, double gamma, double delta, int connections) {
    oracle_tet_plan * P = calloc(1, sizeof(oracle_tet_plan));
    P->n = n;
    P->alpha = alpha; P->beta = beta; P->gamma = gamma; P->delta = delta;
    P->rp1 = oracle_plan_rotations(ORACLE_TRI, n, alpha, beta, gamma + delta + 1.0);
    P->rp2 = oracle_plan_rotations(ORACLE_TRI, n, beta, gamma, delta);
    if (connections) {
        P->P[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, beta + gamma + delta + 2.0, alpha, -0.5, -0.5);
        P->P[1] = oracle_plan_jacobi_to_jacobi(1, 1, n, gamma + delta + 1.0, beta, -0.5, -0.5);
        P->P[2] = oracle_plan_jacobi_to_jacobi(1, 1, n, delta, gamma, -0.5, -0.5);
        P->Pinv[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, beta + gamma + delta + 2.0, alpha);
        P->Pinv[1] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, gamma + delta + 1.0, beta);
        P->Pinv[2] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, delta, gamma);
    }
    return P;
}

void oracle_destroy_tet_plan(oracle_tet_plan * P) {
    if (!P) return;
    oracle_destroy_plan(P->rp1);
    oracle_destroy_plan(P->rp2);
    for (int i = 0; i < 3; i++) { free(P->P[i]); free(P->Pinv[i]); }
    free(P);
}

/* src/rotations.c:297-321 (ft_kernel_tet_hi2lo / lo2hi): sweeps across the columns of the
 * N x L slab of order m, every row rotated alike */
static void kernel_tet(const oracle_plan * RP, int L, int m, double * A, int hi2lo) {
    int n = RP->n;
    const double * s = RP->s, * c = RP->c;
    if (hi2lo) {
        for (int j = m - 1; j >= 0; j--)
            for (int l = L - 2 - j; l >= 0; l--) {
                double S = s[tri_idx(n, l, j)], C = c[tri_idx(n, l, j)];
                for (int k = 0; k < n; k++) givens(S, C, A + k + (size_t) n * l, A + k + (size_t) n * (l + 1));
            }
    } else {
        for (int j = 0; j < m; j++)
            for (int l = 0; l <= L - 2 - j; l++) {
                double S = s[tri_idx(n, l, j)], C = c[tri_idx(n, l, j)];
                for (int k = 0; k < n; k++) givens_t(S, C, A + k + (size_t) n * l, A + k + (size_t) n * (l + 1));
            }
    }
}
void oracle_kernel_tet(const oracle_plan * RP, int L, int m, double * A, int hi2lo) { kernel_tet(RP, L, m, A, hi2lo); }

/* src/drivers.c:510-528: slab m: the tri sweeps of order l + m down column l (l < L - m),
 * then the sweeps across the slab (lo2hi: the reverse) */
static void execute_tet_rot(const oracle_tet_plan * P, double * A, int L, int M, int hi2lo) {
    int N = P->n;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int m = 0; m < M; m++) {
        double * slab = A + (size_t) N * L * m;
        if (hi2lo) {
            for (int l = 0; l < L - m; l++) oracle_kernel_hi2lo(P->rp1, 0, l + m, slab + (size_t) N * l, 1);
            kernel_tet(P->rp2, L, m, slab, 1);
        } else {
            kernel_tet(P->rp2, L, m, slab, 0);
            for (int l = 0; l < L - m; l++) oracle_kernel_lo2hi(P->rp1, 0, l + m, slab + (size_t) N * l, 1);
        }
    }
}

void oracle_execute_tet_hi2lo(const oracle_tet_plan * P, double * A, int L, int M) { execute_tet_rot(P, A, L, M, 1); }
void oracle_execute_tet_lo2hi(const oracle_tet_plan * P, double * A, int L, int M) { execute_tet_rot(P, A, L, M, 0); }

/* src/drivers.c:26-54: entry (i, l, m) times r if m == 0, r if l == 0, r if i == 0, then g,
 * in that order */
static void cheb_normalize_3d(double * A, int N, int L, int M, int transposed) {
    const double r = transposed ? M_SQRT2 : M_SQRT1_2;
    const double g = transposed ? 1.968701243215302468 : 0.507949087473927758;   /* (pi/2)^1.5, (2/pi)^1.5: src/ftinternal.h:59-60 */
    for (int l = 0; l < L; l++)
        for (int i = 0; i < N; i++) A[i + (size_t) l * N] *= r;
    for (int m = 0; m < M; m++) {
        for (int i = 0; i < N; i++) A[i + (size_t) m * L * N] *= r;
        for (int l = 0; l < L; l++) {
            A[(l + (size_t) m * L) * N] *= r;
            for (int i = 0; i < N; i++) A[i + (l + (size_t) m * L) * N] *= g;
        }
    }
}

/* x <- op(U) x along the m axis of every (i, l) fibre (stride N L): cblas_dtrmv on the fibres */
static void trmv_fibres(char trans, int N, int L, int M, const double * U, double * A) {
    #pragma omp parallel
    {
        double * x = malloc(sizeof(double) * M), * y = malloc(sizeof(double) * M);
        #pragma omp for schedule(static)
        for (int f = 0; f < N * L; f++) {
            for (int m = 0; m < M; m++) x[m] = A[f + (size_t) N * L * m];
            for (int i = 0; i < M; i++) {
                double acc = 0.0;
                if (trans == 'N') for (int k = i; k < M; k++) acc += U[i + (size_t) k * N] * x[k];
                else              for (int k = 0; k <= i; k++) acc += U[k + (size_t) i * N] * x[k];
                y[i] = acc;
            }
            for (int m = 0; m < M; m++) A[f + (size_t) N * L * m] = y[m];
        }
        free(x); free(y);
    }
}

/* src/drivers.c:1197-1257 (N = L = M, as in the reference's tests); each multiply is skipped
 * where the reference skips it (its parameters make it the identity) */
void oracle_execute_tet(const oracle_tet_plan * P, int forward, char TRANS, double * A, int N, int L, int M) {
    if (TRANS != 'N' && TRANS != 'T') return;
    const double a = P->alpha, b = P->beta, g = P->gamma, d = P->delta;
    const int u0 = (b + g + d != -2.5) || (a != -0.5);
    const int u1 = (g + d != -1.5) || (b != -0.5);
    const int u2 = (d != -0.5) || (g != -0.5);
    double * const * U = forward ? P->P : P->Pinv;
    if ((forward && TRANS == 'N') || (!forward && TRANS == 'T')) {
        char t = forward ? 'N' : 'T';
        oracle_execute_tet_hi2lo(P, A, L, M);
        if (u0) oracle_trmm('L', t, N, U[0], L * M, A, N);
        if (u1) for (int m = 0; m < M; m++) oracle_trmm('R', forward ? 'T' : 'N', L, U[1], N, A + (size_t) N * L * m, N);
        if (u2) trmv_fibres(forward ? 'T' : 'N', N, L, M, U[2], A);
        cheb_normalize_3d(A, N, L, M, !forward);
    } else {
        cheb_normalize_3d(A, N, L, M, !forward);
        if (u2) trmv_fibres(forward ? 'N' : 'T', N, L, M, U[2], A);
        if (u1) for (int m = 0; m < M; m++) oracle_trmm('R', forward ? 'N' : 'T', L, U[1], N, A + (size_t) N * L * m, N);
        if (u0) oracle_trmm('L', forward ? 'T' : 'N', N, U[0], L * M, A, N);
        oracle_execute_tet_lo2hi(P, A, L, M);
    }
}

void oracle_fill_tet(int N, int L, int M, unsigned long long seed, double * A) {
    for (int m = 0; m < M; m++)
        for (int l = 0; l < L; l++)
            for (int i = 0; i < N; i++) {
                size_t e = (size_t) i + (size_t) N * l + (size_t) N * L * m;
                A[e] = (l < L - m && i < N - l - m) ? u_pm1(seed, e) : 0.0;
            }
}

/* ---------------------------------------------------------------------------
 * Annulus harmonics (gamma = 0).
 * ------------------------------------------------------------------------- */

/* src/banded_source.c:1797-1830 (create_jacobi_multiplication, norm = 1) as the three diagonals
 * of an m x m matrix: d[j] = X(j, j), lo[j] = X(j + 1, j), up[j] = X(j, j + 1); each entry with the
 * reference's own expression (the lower and upper entries are computed separately) */
static void jacobi_tridiagonal(int m, double a, double b, double * d, double * lo, double * up) {
    for (int j = 0; j < m; j++) {
        double v;
        if (j == 1) v = 2 * sqrt(((a + 1) * (b + 1)) / ((a + b + 2) * (a + b + 2) * (a + b + 3)));
        else v = 2 * sqrt((j * (j + a) * (j + b) * (j + a + b)) / ((2 * j + a + b - 1) * (2 * j + a + b) * (2 * j + a + b) * (2 * j + a + b + 1)));
        if (j >= 1) up[j - 1] = v;
        if (j == 0) {
            d[0] = (b - a) / (a + b + 2);
            if (m > 1) lo[0] = 2 * sqrt(((a + 1) * (b + 1)) / ((a + b + 2) * (a + b + 2) * (a + b + 3)));
        } else {
            d[j] = ((b - a) * (a + b)) / ((2 * j + a + b) * (2 * j + a + b + 2));
            if (j + 1 < m)
                lo[j] = 2 * sqrt(((j + 1) * (j + a + 1) * (j + b + 1) * (j + a + b + 1)) / ((2 * j + a + b + 1) * (2 * j + a + b + 2) * (2 * j + a + b + 2) * (2 * j + a + b + 3)));
        }
    }
}

/* src/banded_source.c:1415-1425 */
static void compute_givens(double x, double y, double * c, double * s, double * r) {
    *r = hypot(x, y);
    if (*r <= DBL_MIN / DBL_EPSILON) { *c = 1; *s = 0; }
    else { *c = x / *r; *s = y / *r; }
}

/* src/banded_source.c:1429-1458: Givens QR of the symmetric tridiagonal (a, b) of size k; R's
 * diagonals r0, r1, r2 */
static void tridiagonal_qr(int k, const double * a, const double * b, double * s, double * c, double * r0, double * r1, double * r2) {
    double r, aip1 = a[0], bip1r = b[0];
    for (int i = 0; i < k - 2; i++) {
        compute_givens(aip1, -b[i], c + i, s + i, &r);
        r0[i] = r;
        r1[i] = c[i] * bip1r - s[i] * a[i + 1];
        r2[i] = -s[i] * b[i + 1];
        aip1 = c[i] * a[i + 1] + s[i] * bip1r;
        bip1r = c[i] * b[i + 1];
    }
    compute_givens(aip1, -b[k - 2], c + k - 2, s + k - 2, &r);
    r0[k - 2] = r;
    r1[k - 2] = c[k - 2] * bip1r - s[k - 2] * a[k - 1];
    r0[k - 1] = c[k - 2] * a[k - 1] + s[k - 2] * bip1r;
}

/* src/banded_source.c:1609-1619 (R-based branch): (aq, bq) of size k - 1 from (ap, bp) of size k */
static void jacobi_similarity(int k, const double * r0, const double * r1, const double * ap, const double * bp, double * aq, double * bq) {
    for (int i = 0; i < k - 2; i++) bq[i] = r0[i + 1] / r0[i] * bp[i];
    aq[0] = ap[0] + r1[0] / r0[0] * bp[0];
    for (int i = 1; i < k - 1; i++) aq[i] = (r0[i] * ap[i] + r1[i] * bp[i] - r1[i - 1] * bq[i - 1]) / r0[i];
}

/* src/banded_source.c:471-498 on the tridiagonal (d, lo, up) of size k: R's diagonal rd and
 * superdiagonal ru (upper Cholesky factor, R^T R = the matrix) */
static void tridiagonal_cholesky(int k, double * d, const double * lo, const double * up, double * rd, double * ru) {
    for (int j = 0; j < k; j++) {
        double v0 = d[j];
        double v1 = j + 1 < k ? lo[j] / v0 : 0.0;
        rd[j] = sqrt(v0);
        if (j + 1 < k) {
            d[j + 1] -= v1 * up[j];
            ru[j] = up[j] / rd[j];
        }
    }
}

/* src/rotations.c:192-262 (ft_plan_rotannulus, gamma = 0): the even orders' sines and cosines
 * from the QR factorisations of the shifted Jacobi matrix and its successive similarity
 * transforms; the odd orders' the same after one Cholesky-based similarity */
static void plan_rotannulus(int n, double alpha, double beta, double rho, double * s, double * c) {
    const double t = 1.0 + 2.0 * rho * rho / (1.0 - rho * rho);
    int k = n + 1;
    double * d = malloc(sizeof(double) * (k + 1)), * lo = malloc(sizeof(double) * (k + 1)), * up = malloc(sizeof(double) * (k + 1));
    double * a = malloc(sizeof(double) * (k + 1)), * b = malloc(sizeof(double) * (k + 1));
    double * a2 = malloc(sizeof(double) * (k + 1)), * b2 = malloc(sizeof(double) * (k + 1));
    double * qs = malloc(sizeof(double) * (k + 1)), * qc = malloc(sizeof(double) * (k + 1));
    double * r0 = malloc(sizeof(double) * (k + 1)), * r1 = malloc(sizeof(double) * (k + 1)), * r2 = malloc(sizeof(double) * (k + 1));
    for (int parity = 0; parity < 2; parity++) {
        jacobi_tridiagonal(n + 1, beta, alpha, d, lo, up);
        for (int i = 0; i < n + 1; i++) a[i] = d[i] + t;
        for (int i = 0; i < n; i++) b[i] = up[i];
        k = n + 1;
        if (parity == 1) {
            /* one similarity by the Cholesky factor of (X + t I) */
            for (int i = 0; i < n + 1; i++) d[i] = t + d[i];
            tridiagonal_cholesky(n + 1, d, lo, up, r0, r1);
            jacobi_similarity(k, r0, r1, a, b, a2, b2);
            k--;
            memcpy(a, a2, sizeof(double) * k);
            if (k > 1) memcpy(b, b2, sizeof(double) * (k - 1));
        }
        for (int m = parity; m < 2 * n - 1; m += 2) {
            tridiagonal_qr(k, a, b, qs, qc, r0, r1, r2);
            for (int l = 0; l < n - (m + 1) / 2; l++) {
                s[disk_idx(n, l, m)] = qs[l];
                c[disk_idx(n, l, m)] = qc[l];
            }
            jacobi_similarity(k, r0, r1, a, b, a2, b2);
            k--;
            memcpy(a, a2, sizeof(double) * k);
            if (k > 1) memcpy(b, b2, sizeof(double) * (k - 1));
        }
    }
    free(d); free(lo); free(up); free(a); free(b); free(a2); free(b2); free(qs); free(qc); free(r0); free(r1); free(r2);
}

/* src/drivers.c:1023-1071 (gamma = 0) */
oracle_ann_plan * oracle_plan_ann2cxf(int n, double alpha, double beta, double rho, int connections) {
    oracle_ann_plan * P = calloc(1, sizeof(oracle_ann_plan));
    P->rho = rho;
    oracle_plan * D = P->disk = calloc(1, sizeof(oracle_plan));
    D->kind = ORACLE_DISK; D->n = n; D->alpha = alpha; D->beta = beta;
    D->s = calloc((size_t) n * n + 1, sizeof(double));
    D->c = calloc((size_t) n * n + 1, sizeof(double));
    plan_rotannulus(n, alpha, beta, rho, D->s, D->c);
    /* MP[1]: the Cholesky factor of (t I + X) of size n (src/drivers.c:1036-1046) */
    const double t = 1.0 + 2.0 * rho * rho / (1.0 - rho * rho);
    double * d = malloc(sizeof(double) * (n + 1)), * lo = malloc(sizeof(double) * (n + 1)), * up = malloc(sizeof(double) * (n + 1));
    jacobi_tridiagonal(n, beta, alpha, d, lo, up);
    for (int i = 0; i < n; i++) d[i] = t + d[i];
    P->rd = calloc(n + 1, sizeof(double));
    P->ru = calloc(n + 1, sizeof(double));
    tridiagonal_cholesky(n, d, lo, up, P->rd, P->ru);
    free(d); free(lo); free(up);
    if (connections) {
        D->P[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, beta, alpha, -0.5, -0.5);
        D->Pinv[0] = oracle_plan_jacobi_to_jacobi(1, 1, n, -0.5, -0.5, beta, alpha);
        for (int j = 0; j < n; j++)
            for (int i = 0; i <= j; i++) {
                double r = i ? sqrtl(M_2_PIl) : sqrtl(M_1_PIl), q = j ? sqrtl(M_PI_2l) : sqrtl(M_PIl);
                D->P[0][i + (size_t) j * n] *= r;
                D->Pinv[0][i + (size_t) j * n] *= q;
            }
        double cst = sqrt(2.0) * pow(2.0 / (1.0 - rho * rho), 0.5 * (alpha + beta + 1.0));
        double cstinv = 1.0 / cst;
        for (int j = 0; j < n; j++)
            for (int i = 0; i <= j; i++) {
                D->P[0][i + (size_t) j * n] *= cst;
                D->Pinv[0][i + (size_t) j * n] *= cstinv;
            }
    }
    return P;
}

void oracle_destroy_ann_plan(oracle_ann_plan * P) {
    if (!P) return;
    oracle_destroy_plan(P->disk);
    free(P->rd); free(P->ru);
    free(P);
}

/* src/banded_source.c:381-422 with b = 1: x <- R^{-1} x, R^{-T} x (solve) or R x, R^T x */
static void bidiagonal(const double * rd, const double * ru, int n, char trans, int solve, double * x) {
    if (solve) {
        if (trans == 'N') for (int i = n - 1; i >= 0; i--) { double t = 0; if (i + 1 < n) t += ru[i] * x[i + 1]; x[i] = (x[i] - t) / rd[i]; }
        else for (int i = 0; i < n; i++) { double t = 0; if (i > 0) t += ru[i - 1] * x[i - 1]; x[i] = (x[i] - t) / rd[i]; }
    } else {
        if (trans == 'N') for (int i = 0; i < n; i++) { double t = 0; t += rd[i] * x[i]; if (i + 1 < n) t += ru[i] * x[i + 1]; x[i] = t; }
        else for (int i = n - 1; i >= 0; i--) { double t = 0; if (i > 0) t += ru[i - 1] * x[i - 1]; t += rd[i] * x[i]; x[i] = t; }
    }
}

/* classes 1 and 2 of the columns (j mod 4 = 1, 2): src/drivers.c:1073-1121 (mpmm: solve; mpsm: multiply;
 * classes 0 and 3 take the identity) */
static void ann_modified(const oracle_ann_plan * P, int N, int M, char trans, int solve, double * A) {
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < M; j++)
        if (j % 4 == 1 || j % 4 == 2) bidiagonal(P->rd, P->ru, N, trans, solve, A + (size_t) j * N);
}

void oracle_execute_ann(const oracle_ann_plan * P, int forward, char TRANS, double * A, int N, int M) {
    if (TRANS != 'N' && TRANS != 'T') return;
    const oracle_plan * D = P->disk;
    if (forward && TRANS == 'N') {
        oracle_execute_hi2lo(D, A, M);
        ann_modified(P, N, M, 'N', 1, A);
        oracle_trmm('L', 'N', N, D->P[0], M, A, N);
    } else if (forward) {
        oracle_trmm('L', 'T', N, D->P[0], M, A, N);
        ann_modified(P, N, M, 'T', 1, A);
        oracle_execute_lo2hi(D, A, M);
    } else if (TRANS == 'N') {
        oracle_trmm('L', 'N', N, D->Pinv[0], M, A, N);
        ann_modified(P, N, M, 'N', 0, A);
        oracle_execute_lo2hi(D, A, M);
    } else {
        oracle_execute_hi2lo(D, A, M);
        ann_modified(P, N, M, 'T', 0, A);
        oracle_trmm('L', 'T', N, D->Pinv[0], M, A, N);
    }
}
