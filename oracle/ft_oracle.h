/*
 * ft_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-source restatement of FastTransforms' harmonic-conversion
 * path (sph2fourier / fourier2sph, tri2cheb / cheb2tri, disk2cxf / cxf2disk, and
 * the spin-weighted, Dunkl-Xu, annulus and tetrahedral transforms): rotation
 * tables, scalar Givens sweeps, the execute loops over orders, the dense
 * connection matrices and the triangular multiplies.  It is the checker
 * for the CUDA library: only tests, the smoke check and bench.py's CPU
 * baseline may load it.  The product never calls into it.
 *
 * Pinned against the reference library compiled from its own sources
 * (oracle/_ref, built by oracle/ref_build/Makefile): see tests/test_oracle_pin.py.
 */
#ifndef FT_ORACLE_H
#define FT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_SPH = 0, ORACLE_TRI = 1, ORACLE_DISK = 2, ORACLE_RECT = 3 };

typedef struct {
    int kind;          /* ORACLE_SPH / ORACLE_TRI / ORACLE_DISK / ORACLE_RECT (Dunkl-Xu rectangularised disk) */
    int n;             /* degree + 1 (rows of the coefficient matrix) */
    double * s;        /* rotation sines, packed triangle (sph, tri) or disk packing */
    double * c;        /* rotation cosines, same packing */
    double * P[3];     /* dense n x n upper-triangular connection matrices, column-major (rect: 3) */
    double * Pinv[3];  /* their inverses */
    double alpha, beta, gamma;
} oracle_plan;

/* Rotation arithmetic.  fused = 1: x' = fma(c, x, s*y), y' = fma(c, y, -(s*x)), the form of
 * the reference's FMA SIMD kernels (src/rotations/rotations_AVX512F.c:4-15).  fused = 0:
 * x' = c*x + s*y with every product rounded, the form of the scalar kernels
 * (src/rotations/rotations_default.c:3-15) when compiled without FMA contraction. */
void oracle_set_fused(int fused);

oracle_plan * oracle_plan_sph2fourier(int n);
oracle_plan * oracle_plan_tri2cheb(int n, double alpha, double beta, double gamma);
oracle_plan * oracle_plan_disk2cxf(int n, double alpha, double beta);
/* src/drivers.c:1123-1141 (ft_plan_rectdisk2cheb) */
oracle_plan * oracle_plan_rectdisk2cheb(int n, double beta);
/* Rotation tables only (no connection matrices): cheap, for rotation-stage checks. */
oracle_plan * oracle_plan_rotations(int kind, int n, double alpha, double beta, double gamma);
void oracle_destroy_plan(oracle_plan * P);

/* Rotation stage over all orders of an N x M matrix (in place). */
void oracle_execute_hi2lo(const oracle_plan * P, double * A, int M);
void oracle_execute_lo2hi(const oracle_plan * P, double * A, int M);

/* Single-column kernels (reference ft_kernel_*_{hi2lo,lo2hi}): orders m1 <- m2 on column A with stride S. */
void oracle_kernel_hi2lo(const oracle_plan * P, int m1, int m2, double * A, int S);
void oracle_kernel_lo2hi(const oracle_plan * P, int m1, int m2, double * A, int S);

/* B <- op(U) B (side 'L') or B <- B op(U) (side 'R'); U upper triangular n x n (ld n);
 * B has n rows (side 'L') or n columns (side 'R'), leading dimension ldb. */
void oracle_trmm(char side, char trans, int n, const double * U, int nb, double * B, int ldb);

/* Full transforms, in place on the N x M column-major matrix A.
 * forward = 1: sph2fourier / tri2cheb / disk2cxf; forward = 0: fourier2sph / cheb2tri / cxf2disk.
 * TRANS 'N' or 'T'; any other character leaves A untouched (as the reference does). */
void oracle_execute(const oracle_plan * P, int forward, char TRANS, double * A, int N, int M);
/* sph vector-field transforms on a sph plan: sphv2fourier (forward = 1) / fourier2sphv. */
void oracle_execute_sphv(const oracle_plan * P, int forward, char TRANS, double * A, int N, int M);

/* Connection-matrix planners (n x n, column-major, caller frees with free()). */
double * oracle_plan_legendre_to_chebyshev(int normleg, int normcheb, int n);
double * oracle_plan_chebyshev_to_legendre(int normcheb, int normleg, int n);
double * oracle_plan_ultraspherical_to_ultraspherical(int norm1, int norm2, int n, double lambda, double mu);
double * oracle_plan_jacobi_to_jacobi(int norm1, int norm2, int n, double alpha, double beta, double gamma, double delta);

/* Spin-weighted spherical harmonics (src/rotations.c:445-485, src/drivers.c:645-791,
 * 1259-1361).  Complex matrices: interleaved (re, im) doubles, column-major N x M. */
typedef struct {
    int n, s;
    double * s2, * c2;   /* the spin sweeps' table, (l, j, m) at l + j n + m |s| n */
    oracle_plan * sph;   /* the sph table (the spin plan's s1, c1) and connection matrices */
} oracle_spin_plan;
/* connections = 0: rotation tables only */
oracle_spin_plan * oracle_plan_spinsph2fourier(int n, int s, int connections);
void oracle_destroy_spin_plan(oracle_spin_plan * P);
void oracle_kernel_spinsph_hi2lo(const oracle_spin_plan * P, int m, double * A);
void oracle_kernel_spinsph_lo2hi(const oracle_spin_plan * P, int m, double * A);
/* src/rotations.c:297-321: the n x L slab (n the triangle plan's) of order m */
void oracle_kernel_tet(const oracle_plan * RP, int L, int m, double * A, int hi2lo);
void oracle_execute_spinsph_hi2lo(const oracle_spin_plan * P, double * A, int M);
void oracle_execute_spinsph_lo2hi(const oracle_spin_plan * P, double * A, int M);
/* forward = 1: spinsph2fourier; 0: fourier2spinsph */
void oracle_execute_spin(const oracle_spin_plan * P, int forward, char TRANS, double * A, int N, int M);
void oracle_fill_spin(int N, int M, int s, unsigned long long seed, double * A);

/* Annulus harmonics, gamma = 0 (src/rotations.c:192-268, src/drivers.c:1023-1121,
 * src/banded_source.c): a disk-shaped plan whose sweep table comes from the QR factorisations
 * of shifted Jacobi matrices; classes 1 and 2 of the columns also go through the bidiagonal
 * Cholesky factor R of (t I + X), t = 1 + 2 rho^2 / (1 - rho^2). */
typedef struct {
    oracle_plan * disk;  /* kind ORACLE_DISK: the annulus table in the disk packing; P[0], Pinv[0] */
    double * rd, * ru;   /* R: diagonal (n) and superdiagonal (n - 1) */
    double rho;
} oracle_ann_plan;
/* connections = 0: rotation table only */
oracle_ann_plan * oracle_plan_ann2cxf(int n, double alpha, double beta, double rho, int connections);
void oracle_destroy_ann_plan(oracle_ann_plan * P);
/* forward = 1: ann2cxf; 0: cxf2ann */
void oracle_execute_ann(const oracle_ann_plan * P, int forward, char TRANS, double * A, int N, int M);

/* Tetrahedral harmonics (src/rotations.c:297-321, src/drivers.c:510-528, 1173-1257).  Tensors
 * are N x L x M column-major (entry (i, l, m) at i + N l + N L m). */
typedef struct {
    int n;
    oracle_plan * rp1;   /* tri table (alpha, beta, gamma + delta + 1): the sweeps down each (l, m) column */
    oracle_plan * rp2;   /* tri table (beta, gamma, delta): the sweeps across the columns of a slab */
    double * P[3], * Pinv[3];
    double alpha, beta, gamma, delta;
} oracle_tet_plan;
/* connections = 0: rotation tables only */
oracle_tet_plan * oracle_plan_tet2cheb(int n, double alpha, double beta, double gamma, double delta, int connections);
void oracle_destroy_tet_plan(oracle_tet_plan * P);
void oracle_execute_tet_hi2lo(const oracle_tet_plan * P, double * A, int L, int M);
void oracle_execute_tet_lo2hi(const oracle_tet_plan * P, double * A, int L, int M);
/* forward = 1: tet2cheb; 0: cheb2tet */
void oracle_execute_tet(const oracle_tet_plan * P, int forward, char TRANS, double * A, int N, int L, int M);
/* tetrand's layout (src/ftutilities.c:140-147): (i, l, m) with l < L - m, i < N - l - m */
void oracle_fill_tet(int N, int L, int M, unsigned long long seed, double * A);

/* Seeded fills in the reference layouts (src/ftutilities.c:75-129), U(-1,1) from splitmix64
 * (rect: rows i, columns j < M - i, like tri). */
void oracle_fill(int kind, int N, int M, unsigned long long seed, double * A);

#ifdef __cplusplus
}
#endif

#endif
