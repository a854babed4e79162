/* Every family's entry points as a C caller of the reference's API would use them (spin-weighted
 * with ft_complex data and its grid, Dunkl-Xu, annulus, tetrahedral, and the grids), built against
 * include/ft_b200.h with -lft_b200.  Without a usable device the first plan reports
 * FT_B200_ENODEV and the program prints "ENODEV"; with one, each family's forward then backward
 * transform must return its input to 1e-10, and the program prints "ok". */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "ft_b200.h"

static double rt(const double * a, const double * b, size_t n) {
    double num = 0, den = 0;
    for (size_t k = 0; k < n; k++) { num += (a[k] - b[k]) * (a[k] - b[k]); den += b[k] * b[k]; }
    return sqrt(num / (den > 0 ? den : 1));
}

static void fill(double * A, size_t n, unsigned long long seed) {
    for (size_t k = 0; k < n; k++) {
        seed = seed * 6364136223846793005ULL + 1442695040888963407ULL;
        A[k] = (double) (seed >> 11) * 0x1p-53 * 2.0 - 1.0;
    }
}

int main(void) {
    const int N = 12, M = 2 * N - 1, MD = 4 * N - 3;
    ft_spin_harmonic_plan * SP = ft_plan_spinsph2fourier(N, 2);
    if (!SP) {
        if (ft_b200_last_status() == FT_B200_ENODEV) { puts("ENODEV"); return 0; }
        fprintf(stderr, "%s\n", ft_b200_last_error());
        return 1;
    }
    int bad = 0;
    /* spin-weighted: the triangular layout, rows i < N - |s| */
    ft_complex * Z = calloc((size_t) N * M, sizeof(ft_complex));
    ft_complex * Z0 = calloc((size_t) N * M, sizeof(ft_complex));
    for (int j = 0; j < M; j++)
        for (int i = 0; i < N - 2; i++)
            if (j < M - 2 * i) { Z[i + j * N][0] = Z0[i + j * N][0] = 0.5 / (1 + i + j); Z[i + j * N][1] = Z0[i + j * N][1] = -0.25 / (1 + i); }
    ft_spinsphere_fftw_plan * ZS = ft_plan_spinsph_synthesis(N, M, 2, FT_FFTW_FLAGS), * ZA = ft_plan_spinsph_analysis(N, M, 2, FT_FFTW_FLAGS);
    bad |= ft_get_spin_spinsphere_fftw_plan(ZA) != 2;
    ft_execute_spinsph2fourier('N', SP, Z, N, M);
    ft_execute_spinsph_synthesis('N', ZS, Z, N, M);
    ft_execute_spinsph_analysis('N', ZA, Z, N, M);
    ft_execute_fourier2spinsph('N', SP, Z, N, M);
    bad |= rt((double *) Z, (double *) Z0, 2 * (size_t) N * M) > 1e-10;
    ft_destroy_spinsphere_fftw_plan(ZS);
    ft_destroy_spinsphere_fftw_plan(ZA);
    ft_destroy_spin_harmonic_plan(SP);
    /* one column's sweeps (the low-level kernels), stride 2, there and back */
    ft_rotation_plan * RS1 = ft_plan_rotsphere(N);
    double col[2 * 12], col0[2 * 12];
    fill(col, 2 * (size_t) N, 4);
    for (int k = 0; k < 2 * N; k++) col0[k] = col[k];
    ft_kernel_sph_hi2lo(RS1, 1, 9, col, 2);
    ft_kernel_sph_lo2hi(RS1, 1, 9, col, 2);
    bad |= rt(col, col0, 2 * (size_t) N) > 1e-13;
    ft_destroy_rotation_plan(RS1);
    /* Dunkl-Xu, annulus, with their grids */
    double * A = malloc(sizeof(double) * (size_t) N * MD), * B = malloc(sizeof(double) * (size_t) N * MD);
    fill(A, (size_t) N * N, 1);
    for (size_t k = 0; k < (size_t) N * N; k++) B[k] = A[k];
    ft_harmonic_plan * R = ft_plan_rectdisk2cheb(N, 0.0);
    ft_rectdisk_fftw_plan * RS = ft_plan_rectdisk_synthesis(N, N, FT_FFTW_FLAGS), * RA = ft_plan_rectdisk_analysis(N, N, FT_FFTW_FLAGS);
    ft_execute_rectdisk2cheb('N', R, A, N, N);
    ft_execute_rectdisk_synthesis('N', RS, A, N, N);
    ft_execute_rectdisk_analysis('N', RA, A, N, N);
    ft_execute_cheb2rectdisk('N', R, A, N, N);
    bad |= rt(A, B, (size_t) N * N) > 1e-10;
    ft_destroy_rectdisk_fftw_plan(RS);
    ft_destroy_rectdisk_fftw_plan(RA);
    ft_destroy_harmonic_plan(R);
    fill(A, (size_t) N * MD, 2);
    for (size_t k = 0; k < (size_t) N * MD; k++) B[k] = A[k];
    ft_harmonic_plan * AN = ft_plan_ann2cxf(N, 0.0, 0.0, 0.0, 0.5);
    ft_annulus_fftw_plan * AS = ft_plan_annulus_synthesis(N, MD, 0.5, FT_FFTW_FLAGS), * AA = ft_plan_annulus_analysis(N, MD, 0.5, FT_FFTW_FLAGS);
    bad |= ft_get_rho_annulus_fftw_plan(AS) != 0.5;
    ft_execute_ann2cxf('N', AN, A, N, MD);
    ft_execute_annulus_synthesis('N', AS, A, N, MD);
    ft_execute_annulus_analysis('N', AA, A, N, MD);
    ft_execute_cxf2ann('N', AN, A, N, MD);
    bad |= rt(A, B, (size_t) N * MD) > 1e-10;
    ft_destroy_annulus_fftw_plan(AS);
    ft_destroy_annulus_fftw_plan(AA);
    ft_destroy_harmonic_plan(AN);
    /* tetrahedral, with its grid */
    double * T = malloc(sizeof(double) * (size_t) N * N * N), * T0 = malloc(sizeof(double) * (size_t) N * N * N);
    fill(T, (size_t) N * N * N, 3);
    for (size_t k = 0; k < (size_t) N * N * N; k++) T0[k] = T[k];
    ft_harmonic_plan * TP = ft_plan_tet2cheb(N, 0.0, 0.0, 0.0, 0.0);
    ft_tetrahedron_fftw_plan * TS = ft_plan_tet_synthesis(N, N, N, FT_FFTW_FLAGS), * TA = ft_plan_tet_analysis(N, N, N, FT_FFTW_FLAGS);
    ft_execute_tet2cheb('N', TP, T, N, N, N);
    ft_execute_tet_synthesis('N', TS, T, N, N, N);
    ft_execute_tet_analysis('N', TA, T, N, N, N);
    ft_execute_cheb2tet('N', TP, T, N, N, N);
    bad |= rt(T, T0, (size_t) N * N * N) > 1e-10;
    ft_destroy_tetrahedron_fftw_plan(TS);
    ft_destroy_tetrahedron_fftw_plan(TA);
    ft_destroy_harmonic_plan(TP);
    /* disk and triangle grids */
    ft_disk_fftw_plan * DS = ft_plan_disk_synthesis(N, MD, FT_FFTW_FLAGS);
    ft_triangle_fftw_plan * QS = ft_plan_tri_synthesis(N, N, FT_FFTW_FLAGS);
    bad |= !DS || !QS;
    ft_destroy_disk_fftw_plan(DS);
    ft_destroy_triangle_fftw_plan(QS);
    free(Z); free(Z0); free(A); free(B); free(T); free(T0);
    if (bad || ft_b200_last_status()) { fprintf(stderr, "failed: %s\n", ft_b200_last_error()); return 1; }
    puts("ok");
    return 0;
}
