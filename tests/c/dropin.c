/* A caller written against the reference's C API (src/fasttransforms.h): plan, forward and
 * backward sph2fourier on a small seeded matrix, destroy.  Built against include/ft_b200.h and
 * linked with -lft_b200 in place of -lfasttransforms; the only addition is the status check the
 * reference does not have.  Prints "ENODEV" and exits 0 when there is no usable device, else
 * prints the round-trip error and exits 0 when it is below 1e-13. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "ft_b200.h"

int main(void) {
    const int N = 33, M = 2 * N - 1;
    double * A = calloc((size_t) N * M, sizeof(double));
    double * B = calloc((size_t) N * M, sizeof(double));
    unsigned long long z = 20261203ULL;
    for (int j = 0; j < M; j++)
        for (int i = 0; i < N; i++)
            if (j < M - 2 * i) {   /* the sph layout (src/ftutilities.c:75-84) */
                z = z * 6364136223846793005ULL + 1442695040888963407ULL;
                A[i + j * N] = B[i + j * N] = (double) (z >> 11) * 0x1p-53 * 2.0 - 1.0;
            }
    ft_harmonic_plan * P = ft_plan_sph2fourier(N);
    if (!P) {
        if (ft_b200_last_status() == FT_B200_ENODEV) { puts("ENODEV"); return 0; }
        fprintf(stderr, "plan failed: %s\n", ft_b200_last_error());
        return 1;
    }
    ft_execute_sph2fourier('N', P, A, N, M);
    ft_execute_fourier2sph('N', P, A, N, M);
    ft_destroy_harmonic_plan(P);
    if (ft_b200_last_status()) { fprintf(stderr, "%s\n", ft_b200_last_error()); return 1; }
    double num = 0, den = 0;
    for (int k = 0; k < N * M; k++) { num += (A[k] - B[k]) * (A[k] - B[k]); den += B[k] * B[k]; }
    const double err = sqrt(num / den);
    printf("%.3e\n", err);
    free(A);
    free(B);
    return err < 1e-13 ? 0 : 1;
}
