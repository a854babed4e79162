/* A C caller of ft_b200_execute_shared_host: five fields of degree 63 sharing one sph plan go
 * forward then backward in one call from host memory (the reference would call
 * ft_execute_sph2fourier / ft_execute_fourier2sph per field, src/drivers.c:833-865).  Prints
 * "ENODEV" and exits 0 without a usable device; else prints the largest round-trip error and
 * exits 0 when it is below 1e-13, in FP64 and in the split-BF16 form (below 1e-5). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "ft_b200.h"

#define NF 5

int main(void) {
    const int N = 64, M = 2 * N - 1;
    double * A[NF];
    double * B[NF];
    unsigned long long z = 20261203ULL;
    for (int f = 0; f < NF; f++) {
        A[f] = calloc((size_t) N * M, sizeof(double));
        B[f] = calloc((size_t) N * M, sizeof(double));
        for (int j = 0; j < M; j++)
            for (int i = 0; i < N; i++)
                if (j < M - 2 * i) {   /* the sph layout (src/ftutilities.c:75-84) */
                    z = z * 6364136223846793005ULL + 1442695040888963407ULL;
                    A[f][i + j * N] = B[f][i + j * N] = (double) (z >> 11) * 0x1p-53 * 2.0 - 1.0;
                }
    }
    ft_harmonic_plan * P = ft_plan_sph2fourier(N);
    if (!P) {
        if (ft_b200_last_status() == FT_B200_ENODEV) { puts("ENODEV"); return 0; }
        fprintf(stderr, "plan failed: %s\n", ft_b200_last_error());
        return 1;
    }
    const int forward[2] = {1, 0};
    const char trans[2] = {'N', 'N'};
    double worst[2] = {0.0, 0.0};
    const int precision[2] = {FT_B200_FP64, FT_B200_MIXED_BF16};
    for (int p = 0; p < 2; p++) {
        if (ft_b200_execute_shared_host(P, 2, forward, trans, A, NF, precision[p]) != FT_B200_OK) {
            fprintf(stderr, "%s\n", ft_b200_last_error());
            return 1;
        }
        for (int f = 0; f < NF; f++) {
            double num = 0, den = 0;
            for (int k = 0; k < N * M; k++) { num += (A[f][k] - B[f][k]) * (A[f][k] - B[f][k]); den += B[f][k] * B[f][k]; }
            if (sqrt(num / den) > worst[p]) worst[p] = sqrt(num / den);
            for (int k = 0; k < N * M; k++) A[f][k] = B[f][k];
        }
    }
    ft_destroy_harmonic_plan(P);
    printf("%.3e\n", worst[0]);
    for (int f = 0; f < NF; f++) { free(A[f]); free(B[f]); }
    return (worst[0] < 1e-13 && worst[1] < 1e-5) ? 0 : 1;
}
