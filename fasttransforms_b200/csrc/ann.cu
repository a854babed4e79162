// Annulus harmonics (gamma = 0): the reference's ft_plan_rotannulus, ft_plan_ann2cxf,
// ft_execute_ann2cxf / ft_execute_cxf2ann (src/rotations.c:192-268, src/drivers.c:1023-1121,
// src/banded_source.c:381-498, 1415-1458, 1609-1619, 1797-1830) on device memory.
//
// The coefficients have the disk layout (N x M, M = 4N - 3, order m on the column pair
// 2m - 1, 2m), and the rotation stage is the disk sweep (the rotation kernel's DISK kind) with
// another table: the sines and cosines of the QR factorisations of the shifted Jacobi matrix
// t I + X (t = 1 + 2 rho^2 / (1 - rho^2)) and of its successive similarity transforms, even
// orders from t I + X itself, odd orders after one similarity by its Cholesky factor (built
// on the host in FP64 by this file's restatement of those recurrences).  Between the sweeps
// and the connection multiply, the columns of classes 1 and 2 (j mod 4 = 1, 2) go through the
// bidiagonal Cholesky factor R of t I + X of size n: x <- R^{-1} x (ann2cxf) or R x (cxf2ann),
// or their transposes (bidiag_kernel, one thread per column); classes 0 and 3 take the
// identity.  The connection multiply is one matrix, P0, on every column.
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "ft_internal.h"

namespace ftb {
namespace {

constexpr int kAnnMagic = 0x4654414e;   // "FTAN"

struct AnnPlan {
    ft_harmonic_plan pub;           // must stay the first member
    int magic = kAnnMagic;
    int n = 0, device = 0;
    ft_rotation_plan * rp_arr[1] = {nullptr};
    double * hostP[1] = {nullptr};
    double * hostPinv[1] = {nullptr};
    double * dP = nullptr, * dPinv = nullptr;
    double * d_rd = nullptr, * d_ru = nullptr;   // R's diagonal (n) and superdiagonal (n - 1)
    double * d_scratch = nullptr;
    size_t scratch_elems = 0;
    double * d_stage = nullptr;
    size_t stage_elems = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
};

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

AnnPlan * as_ann(const ft_harmonic_plan * P) {
    AnnPlan * A = reinterpret_cast<AnnPlan *>(const_cast<ft_harmonic_plan *>(P));
    return (A && A->magic == kAnnMagic) ? A : nullptr;
}

// ---------------------------------------------------------------------------
// Host: the annulus table and the Cholesky factor (FP64, the reference's expressions).
// ---------------------------------------------------------------------------

// The normalised Jacobi multiplication matrix (create_jacobi_multiplication, norm = 1) of size m
// as three diagonals: d[j] = X(j, j), lo[j] = X(j + 1, j), up[j] = X(j, j + 1); the lower and upper
// entries with their own expressions, as the reference computes them
void jacobi_tridiagonal(int m, double a, double b, double * d, double * lo, double * up) {
    for (int j = 0; j < m; j++) {
        double v;
        if (j == 1) v = 2 * std::sqrt(((a + 1) * (b + 1)) / ((a + b + 2) * (a + b + 2) * (a + b + 3)));
        else v = 2 * std::sqrt((j * (j + a) * (j + b) * (j + a + b)) / ((2 * j + a + b - 1) * (2 * j + a + b) * (2 * j + a + b) * (2 * j + a + b + 1)));
        if (j >= 1) up[j - 1] = v;
        if (j == 0) {
            d[0] = (b - a) / (a + b + 2);
            if (m > 1) lo[0] = 2 * std::sqrt(((a + 1) * (b + 1)) / ((a + b + 2) * (a + b + 2) * (a + b + 3)));
        } else {
            d[j] = ((b - a) * (a + b)) / ((2 * j + a + b) * (2 * j + a + b + 2));
            if (j + 1 < m)
                lo[j] = 2 * std::sqrt(((j + 1) * (j + a + 1) * (j + b + 1) * (j + a + b + 1)) /
                                      ((2 * j + a + b + 1) * (2 * j + a + b + 2) * (2 * j + a + b + 2) * (2 * j + a + b + 3)));
        }
    }
}

// the rotation taking (x, y) to (r, 0): r = hypot(x, y), (cos, sin) = (x, y) / r; the identity for r
// at or below the smallest normal over the unit roundoff
void givens_pair(double x, double y, double * cs, double * sn, double * r) {
    *r = std::hypot(x, y);
    if (*r <= DBL_MIN / DBL_EPSILON) { *cs = 1; *sn = 0; }
    else { *cs = x / *r; *sn = y / *r; }
}

// Givens QR of the symmetric tridiagonal T of size k (diagonal dg[0 .. k-1], off-diagonal
// off[0 .. k-2]).  Step i rotates rows i and i + 1 so that the subdiagonal entry vanishes:
// `pivot` is the running (i, i) entry of the partly reduced matrix and `above` its (i, i + 1)
// entry; the step writes R's diagonal rd[i] and superdiagonal ru[i] and the rotation (cs, sn).
// The expressions keep the reference's operation order (src/banded_source.c:1430-1455), so the
// table built from them is bit-identical to the reference's.
void tridiagonal_qr(int k, const double * dg, const double * off, double * sn, double * cs, double * rd, double * ru) {
    double pivot = dg[0], above = off[0];
    for (int i = 0; i + 1 < k; i++) {
        double r;
        givens_pair(pivot, -off[i], cs + i, sn + i, &r);
        rd[i] = r;
        ru[i] = cs[i] * above - sn[i] * dg[i + 1];
        pivot = cs[i] * dg[i + 1] + sn[i] * above;
        if (i + 2 < k) above = cs[i] * off[i + 1];
    }
    rd[k - 1] = pivot;
}

// R X R^{-1} restricted to size k - 1, from the upper-triangular R's first two diagonals
void jacobi_similarity(int k, const double * r0, const double * r1, const double * ap, const double * bp, double * aq, double * bq) {
    for (int i = 0; i < k - 2; i++) bq[i] = r0[i + 1] / r0[i] * bp[i];
    aq[0] = ap[0] + r1[0] / r0[0] * bp[0];
    for (int i = 1; i < k - 1; i++) aq[i] = (r0[i] * ap[i] + r1[i] * bp[i] - r1[i - 1] * bq[i - 1]) / r0[i];
}

// upper Cholesky factor (diagonal rd, superdiagonal ru) of the tridiagonal (d, lo, up) of size k
void tridiagonal_cholesky(int k, double * d, const double * lo, const double * up, double * rd, double * ru) {
    for (int j = 0; j < k; j++) {
        const double v0 = d[j];
        const double v1 = j + 1 < k ? lo[j] / v0 : 0.0;
        rd[j] = std::sqrt(v0);
        if (j + 1 < k) {
            d[j + 1] -= v1 * up[j];
            ru[j] = up[j] / rd[j];
        }
    }
}

// the annulus table in the disk packing (s, c of n^2 entries)
void annulus_table(int n, double alpha, double beta, double rho, double * s, double * c) {
    const double t = 1.0 + 2.0 * rho * rho / (1.0 - rho * rho);
    const size_t len = (size_t) n + 2;
    std::vector<double> d(len), lo(len), up(len), a(len), b(len), a2(len), b2(len), qs(len), qc(len), r0(len), r1(len);
    for (int parity = 0; parity < 2; parity++) {
        jacobi_tridiagonal(n + 1, beta, alpha, d.data(), lo.data(), up.data());
        for (int i = 0; i < n + 1; i++) a[i] = d[i] + t;
        for (int i = 0; i < n; i++) b[i] = up[i];
        int k = n + 1;
        if (parity == 1) {   // one similarity by the Cholesky factor of t I + X
            for (int i = 0; i < n + 1; i++) d[i] = t + d[i];
            tridiagonal_cholesky(n + 1, d.data(), lo.data(), up.data(), r0.data(), r1.data());
            jacobi_similarity(k, r0.data(), r1.data(), a.data(), b.data(), a2.data(), b2.data());
            k--;
            std::copy(a2.begin(), a2.begin() + k, a.begin());
            if (k > 1) std::copy(b2.begin(), b2.begin() + (k - 1), b.begin());
        }
        for (int m = parity; m < 2 * n - 1; m += 2) {
            tridiagonal_qr(k, a.data(), b.data(), qs.data(), qc.data(), r0.data(), r1.data());
            for (int l = 0; l < n - (m + 1) / 2; l++) {
                const long long o = Geo::table_base(DISK, n, m) + l;
                s[o] = qs[l];
                c[o] = qc[l];
            }
            jacobi_similarity(k, r0.data(), r1.data(), a.data(), b.data(), a2.data(), b2.data());
            k--;
            std::copy(a2.begin(), a2.begin() + k, a.begin());
            if (k > 1) std::copy(b2.begin(), b2.begin() + (k - 1), b.begin());
        }
    }
}

// A DISK rotation plan carrying the annulus table
ft_rotation_plan * annulus_rotation_plan(int n, double alpha, double beta, double rho) {
    ft_rotation_plan * RP = rotation_plan_new(DISK, n, alpha, beta, 0.0);
    if (!RP) return nullptr;
    const size_t len = (size_t) n * n;
    annulus_table(n, alpha, beta, rho, RP->s, RP->c);
    std::vector<double2> sc(len);
    for (size_t i = 0; i < len; i++) sc[i] = make_double2(RP->s[i], RP->c[i]);
    if (!ok(cudaMemcpy(RP->d_sc, sc.data(), sizeof(double2) * len, cudaMemcpyHostToDevice), "cudaMemcpy(table)") ||
        !rotation_plan_pad(RP)) {   // the padded copy the rotation kernel reads, from this table
        ft_destroy_rotation_plan(RP);
        return nullptr;
    }
    return RP;
}

// ---------------------------------------------------------------------------
// Device: the bidiagonal stage on column classes 1 and 2.
// ---------------------------------------------------------------------------

// Thread t takes column 4 (t / 2) + 1 + t % 2.  solve: x <- R^{-1} x ('N', rows n-1 .. 0) or
// R^{-T} x ('T', rows 0 .. n-1); else x <- R x or R^T x.  The reference's summation order
// (a running sum from 0; src/banded_source.c:381-422).  The next LA rows are loaded before any
// of them is updated (each update only reads rows already updated or still unread).
constexpr int LA = 8;
__global__ void __launch_bounds__(64) bidiag_kernel(double * A, const double * __restrict__ rd, const double * __restrict__ ru,
                                                    int N, int M, bool trans, bool solve) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = 4 * (t / 2) + 1 + (t & 1);
    if (col >= M) return;
    double * x = A + (long long) col * N;
    double v[LA];
    if (solve && !trans) {          // backward: x_i = (x_i - ru_i x_{i+1}) / rd_i
        double next = 0.0;          // x_{i+1}, already final
        for (int i0 = N - 1; i0 >= 0; i0 -= LA) {
#pragma unroll
            for (int q = 0; q < LA; ++q) if (i0 - q >= 0) v[q] = x[i0 - q];
#pragma unroll
            for (int q = 0; q < LA; ++q) {
                const int i = i0 - q;
                if (i < 0) break;
                double tt = 0.0;
                if (i + 1 < N) tt += ru[i] * next;
                next = (v[q] - tt) / rd[i];
                x[i] = next;
            }
        }
    } else if (solve) {             // forward: x_i = (x_i - ru_{i-1} x_{i-1}) / rd_i
        double prev = 0.0;
        for (int i0 = 0; i0 < N; i0 += LA) {
#pragma unroll
            for (int q = 0; q < LA; ++q) if (i0 + q < N) v[q] = x[i0 + q];
#pragma unroll
            for (int q = 0; q < LA; ++q) {
                const int i = i0 + q;
                if (i >= N) break;
                double tt = 0.0;
                if (i > 0) tt += ru[i - 1] * prev;
                prev = (v[q] - tt) / rd[i];
                x[i] = prev;
            }
        }
    } else if (!trans) {            // x_i = rd_i x_i + ru_i x_{i+1} (old values), rows 0 .. n-1
        for (int i0 = 0; i0 < N; i0 += LA) {
#pragma unroll
            for (int q = 0; q <= LA; ++q) if (i0 + q < N && q < LA + 1) { if (q < LA) v[q] = x[i0 + q]; }
            const double after = i0 + LA < N ? x[i0 + LA] : 0.0;   // row i0 + LA, not yet updated
#pragma unroll
            for (int q = 0; q < LA; ++q) {
                const int i = i0 + q;
                if (i >= N) break;
                const double xn = q + 1 < LA ? v[q + 1] : after;
                double tt = 0.0;
                tt += rd[i] * v[q];
                if (i + 1 < N) tt += ru[i] * xn;
                x[i] = tt;
            }
        }
    } else {                        // x_i = ru_{i-1} x_{i-1} + rd_i x_i (old values), rows n-1 .. 0
        for (int i0 = N - 1; i0 >= 0; i0 -= LA) {
#pragma unroll
            for (int q = 0; q < LA; ++q) if (i0 - q >= 0) v[q] = x[i0 - q];
            const double before = i0 - LA >= 0 ? x[i0 - LA] : 0.0;   // row i0 - LA, not yet updated
#pragma unroll
            for (int q = 0; q < LA; ++q) {
                const int i = i0 - q;
                if (i < 0) break;
                const double xp = q + 1 < LA ? v[q + 1] : before;
                double tt = 0.0;
                if (i > 0) tt += ru[i - 1] * xp;
                tt += rd[i] * v[q];
                x[i] = tt;
            }
        }
    }
}

bool bidiagonal(AnnPlan * P, bool trans, bool solve, double * A, int M, cudaStream_t st) {
    const int nt = 2 * ((M + 2) / 4);   // threads: two per group of four columns (some past M)
    if (nt <= 0) return true;
    prof_begin(FAM_OTHER, st);
    bidiag_kernel<<<(nt + 63) / 64, 64, 0, st>>>(A, P->d_rd, P->d_ru, P->n, M, trans, solve);
    count_launch();
    prof_end(st);
    return ok(cudaGetLastError(), "bidiagonal kernel");
}

bool left(AnnPlan * P, const double * U, bool trans, const double * in, double * out, int M, cudaStream_t st) {
    TrmmLaunch L{};
    L.n = P->n;
    L.ld_in = L.ld_out = P->n;
    L.trans = trans;
    L.nclasses = 1;
    L.cls[0] = TrmmClass{U, in, out, M};
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm(L, st);
    prof_end(st);
    return ok(e, "trmm kernel");
}

// src/drivers.c:1073-1121: the sweeps out of place into the scratch, the bidiagonal stage there,
// the multiply back into A (or the reverse)
bool transform(AnnPlan * P, bool forward, char T, double * A, int M, cudaStream_t st) {
    const int N = P->n;
    if (P->scratch_elems < (size_t) N * M) {
        cudaFree(P->d_scratch);
        P->d_scratch = nullptr;
        P->scratch_elems = 0;
        if (!ok(cudaMalloc(&P->d_scratch, sizeof(double) * (size_t) N * M), "cudaMalloc(scratch)")) return false;
        P->scratch_elems = (size_t) N * M;
        P->pub.B = P->d_scratch;
    }
    double * S = P->d_scratch;
    const double * U = forward ? P->dP : P->dPinv;
    ft_rotation_plan * RP = P->rp_arr[0];
    const bool tN = T == 'N';
    if (forward == tN)   // ann2cxf 'N' (solve) / cxf2ann 'T' (multiply): hi2lo, bidiagonal, P0 or Pinv0^T
        return rotation_sweeps(RP, true, A, S, M, N, st) && bidiagonal(P, !forward, forward, S, M, st) &&
               left(P, U, !forward, S, A, M, st);
    // ann2cxf 'T' / cxf2ann 'N': P0^T or Pinv0, bidiagonal, lo2hi
    return left(P, U, forward, A, S, M, st) && bidiagonal(P, forward, forward, S, M, st) &&
           rotation_sweeps(RP, false, S, A, M, N, st);
}

int check(const AnnPlan * P, char T, const double * A, int N, int M) {
    if (T != 'N' && T != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return FT_B200_EINVAL; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL matrix"); return FT_B200_EINVAL; }
    if (N != P->n) { set_error(FT_B200_EINVAL, "N does not match the plan's n"); return FT_B200_EINVAL; }
    if (M < 1 || (M >= 4 && M % 2 == 0)) {
        set_error(FT_B200_EINVAL, "annulus matrices need an odd number of columns M (orders on column pairs)");
        return FT_B200_EINVAL;
    }
    return FT_B200_OK;
}

void destroy(AnnPlan * P) {
    if (P->stream) { cudaStreamSynchronize(P->stream); cudaStreamDestroy(P->stream); }
    if (P->rp_arr[0]) ft_destroy_rotation_plan(P->rp_arr[0]);
    std::free(P->hostP[0]);
    std::free(P->hostPinv[0]);
    cudaFree(P->dP);
    cudaFree(P->dPinv);
    cudaFree(P->d_rd);
    cudaFree(P->d_ru);
    cudaFree(P->d_scratch);
    cudaFree(P->d_stage);
    P->magic = 0;
    delete P;
}

void execute_host(const ft_harmonic_plan * Pp, bool forward, char T, double * A, int N, int M) {
    clear_error();
    AnnPlan * P = as_ann(Pp);
    if (!P) { set_error(FT_B200_EINVAL, "not an annulus plan of this library"); return; }
    if (check(P, T, A, N, M) != FT_B200_OK) return;
    std::lock_guard<std::mutex> lk(P->mu);
    cudaSetDevice(P->device);
    const size_t elems = (size_t) N * M;
    if (P->stage_elems < elems) {
        cudaFree(P->d_stage);
        P->d_stage = nullptr;
        P->stage_elems = 0;
        if (!ok(cudaMalloc(&P->d_stage, sizeof(double) * elems), "cudaMalloc(stage)")) return;
        P->stage_elems = elems;
    }
    cudaStream_t st = P->stream;
    if (!ok(cudaMemcpyAsync(P->d_stage, A, sizeof(double) * elems, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(H2D)")) return;
    if (!transform(P, forward, T, P->d_stage, M, st)) return;
    if (!ok(cudaMemcpyAsync(A, P->d_stage, sizeof(double) * elems, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(D2H)")) return;
    ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

}  // namespace

bool ann_plan_destroy(ft_harmonic_plan * P) {
    AnnPlan * A = as_ann(P);
    if (!A) return false;
    destroy(A);
    return true;
}

int ann_execute_dev(const ft_harmonic_plan * Pp, bool forward, char TRANS, double * dA, int N, int M, cudaStream_t st) {
    AnnPlan * P = as_ann(Pp);
    if (!P) return -1;
    const int c = check(P, TRANS, dA, N, M);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(P->mu);
    return transform(P, forward, TRANS, dA, M, st) ? FT_B200_OK : ft_b200_last_status();
}

}  // namespace ftb

using namespace ftb;

extern "C" {

ft_rotation_plan * ft_plan_rotannulus(const int n, const double alpha, const double beta, const double gamma, const double rho) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    if (gamma != 0.0) { set_error(FT_B200_EUNSUPPORTED, "annulus plans with gamma != 0 are not implemented (as in the reference)"); return nullptr; }
    return annulus_rotation_plan(n, alpha, beta, rho);
}

ft_harmonic_plan * ft_plan_ann2cxf(const int n, const double alpha, const double beta, const double gamma, const double rho) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    if (gamma != 0.0) { set_error(FT_B200_EUNSUPPORTED, "annulus plans with gamma != 0 are not implemented (as in the reference)"); return nullptr; }
    AnnPlan * P = new AnnPlan();
    std::memset(&P->pub, 0, sizeof(P->pub));
    P->n = n;
    P->rp_arr[0] = annulus_rotation_plan(n, alpha, beta, rho);
    if (!P->rp_arr[0]) { delete P; return nullptr; }
    P->device = P->rp_arr[0]->device;
    // the second modified plan: Cholesky factor of t I + X of size n (src/drivers.c:1034-1046)
    const double t = 1.0 + 2.0 * rho * rho / (1.0 - rho * rho);
    std::vector<double> d(n + 1), lo(n + 1), up(n + 1), rd(n + 1), ru(n + 1);
    jacobi_tridiagonal(n, beta, alpha, d.data(), lo.data(), up.data());
    for (int i = 0; i < n; i++) d[i] = t + d[i];
    tridiagonal_cholesky(n, d.data(), lo.data(), up.data(), rd.data(), ru.data());
    // P0 = plan_jacobi_to_chebyshev(1, 0, n, beta, alpha) times cst, its inverse (src/drivers.c:1050-1061)
    P->hostP[0] = connection_jacobi(n, beta, alpha, -0.5, -0.5);
    P->hostPinv[0] = connection_jacobi(n, -0.5, -0.5, beta, alpha);
    if (!P->hostP[0] || !P->hostPinv[0]) { set_error(FT_B200_ENOMEM, "host allocation (connection matrices)"); destroy(P); return nullptr; }
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) {
            const double r = i ? std::sqrt((long double) M_2_PIl) : std::sqrt((long double) M_1_PIl);
            const double q = j ? std::sqrt((long double) M_PI_2l) : std::sqrt((long double) M_PIl);
            P->hostP[0][i + (size_t) j * n] *= r;
            P->hostPinv[0][i + (size_t) j * n] *= q;
        }
    const double cst = std::sqrt(2.0) * std::pow(2.0 / (1.0 - rho * rho), 0.5 * (alpha + beta + gamma + 1.0));
    const double cstinv = 1.0 / cst;
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) {
            P->hostP[0][i + (size_t) j * n] *= cst;
            P->hostPinv[0][i + (size_t) j * n] *= cstinv;
        }
    const size_t nn = sizeof(double) * (size_t) n * n;
    if (!ok(cudaMalloc(&P->dP, nn), "cudaMalloc(P)") || !ok(cudaMemcpy(P->dP, P->hostP[0], nn, cudaMemcpyHostToDevice), "cudaMemcpy(P)") ||
        !ok(cudaMalloc(&P->dPinv, nn), "cudaMalloc(Pinv)") ||
        !ok(cudaMemcpy(P->dPinv, P->hostPinv[0], nn, cudaMemcpyHostToDevice), "cudaMemcpy(Pinv)") ||
        !ok(cudaMalloc(&P->d_rd, sizeof(double) * (n + 1)), "cudaMalloc(R)") ||
        !ok(cudaMemcpy(P->d_rd, rd.data(), sizeof(double) * (n + 1), cudaMemcpyHostToDevice), "cudaMemcpy(R)") ||
        !ok(cudaMalloc(&P->d_ru, sizeof(double) * (n + 1)), "cudaMalloc(R)") ||
        !ok(cudaMemcpy(P->d_ru, ru.data(), sizeof(double) * (n + 1), cudaMemcpyHostToDevice), "cudaMemcpy(R)") ||
        !ok(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking), "cudaStreamCreate")) {
        destroy(P);
        return nullptr;
    }
    // src/drivers.c:1023-1071: one rotation plan, one connection pair; the modified plans are
    // held on the device (MP is NULL here)
    P->pub.RP = P->rp_arr;
    P->pub.MP = nullptr;
    P->pub.B = nullptr;
    P->pub.P = P->hostP;
    P->pub.Pinv = P->hostPinv;
    P->pub.alpha = alpha;
    P->pub.beta = beta;
    P->pub.gamma = gamma;
    P->pub.rho = rho;
    P->pub.NRP = 1;
    P->pub.NMP = 2;
    P->pub.NP = 1;
    return &P->pub;
}

void ft_execute_ann2cxf(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) {
    execute_host(P, true, TRANS, A, N, M);
}
void ft_execute_cxf2ann(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) {
    execute_host(P, false, TRANS, A, N, M);
}

}  // extern "C"
