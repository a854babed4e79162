// Dunkl-Xu (rectangularised disk) transforms: the reference's ft_plan_rectdisk2cheb,
// ft_execute_rectdisk2cheb / ft_execute_cheb2rectdisk (src/drivers.c:1123-1171) on device
// memory.
//
// Data: an N x M column-major matrix, M = N; order m on column m.  A transform is
//   rectdisk2cheb 'N': the rotation stage hi2lo (the rotation kernel's RECT kind: the sph
//     sweep shape on one column per order, orders 2 .. M - 1), then P0 on the even columns and
//     P1 on the odd columns (left upper-triangular multiplies, column stride 2N), then the
//     right multiply A <- A P2^T;
//   'T' and the inverse transforms the transposes / inverses in the reverse order.
// The connection matrices (src/drivers.c:1127-1136, src/transforms.c:80-93, 185-211):
//   P0 = ultraspherical(beta + 1) -> Chebyshev, P1 = ultraspherical(beta + 2) -> (1),
//   P2 = ultraspherical(beta + 1/2) -> Chebyshev, and the three inverse maps, normalised
//   on the ultraspherical side and unnormalised on the other.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "ft_internal.h"

namespace ftb {
namespace {

constexpr int kRectMagic = 0x46545244;   // "FTRD"

struct RectPlan {
    ft_harmonic_plan pub;           // must stay the first member
    int magic = kRectMagic;
    int n = 0, device = 0;
    ft_rotation_plan * rp_arr[1] = {nullptr};
    double * hostP[3] = {nullptr, nullptr, nullptr};
    double * hostPinv[3] = {nullptr, nullptr, nullptr};
    double * dP[3] = {nullptr, nullptr, nullptr};
    double * dPinv[3] = {nullptr, nullptr, nullptr};
    double * d_scratch = nullptr;   // one N x M matrix
    size_t scratch_elems = 0;
    double * d_stage = nullptr;     // host-pointer calls
    size_t stage_elems = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
};

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

RectPlan * as_rect(const ft_harmonic_plan * P) {
    RectPlan * R = reinterpret_cast<RectPlan *>(const_cast<ft_harmonic_plan *>(P));
    return (R && R->magic == kRectMagic) ? R : nullptr;
}

// plan_ultraspherical_to_chebyshev(1, 0, n, lambda) (src/transforms.c:185-197): the normalised
// Jacobi connection (lambda - 1/2, lambda - 1/2) -> (-1/2, -1/2) with entries i = j, j - 2, ..
// of row i scaled to the unnormalised Chebyshev basis
double * ultraspherical_to_chebyshev(int n, double lambda) {
    double * V = connection_jacobi(n, lambda - 0.5, lambda - 0.5, -0.5, -0.5);
    if (!V) return nullptr;
    const double r0 = std::sqrt((long double) M_1_PIl), r1 = std::sqrt((long double) M_2_PIl);
    for (int j = 0; j < n; j++)
        for (int i = j; i >= 0; i -= 2) V[i + (size_t) j * n] *= i ? r1 : r0;
    return V;
}

// plan_chebyshev_to_ultraspherical(0, 1, n, lambda) (src/transforms.c:199-211)
double * chebyshev_to_ultraspherical(int n, double lambda) {
    double * V = connection_jacobi(n, -0.5, -0.5, lambda - 0.5, lambda - 0.5);
    if (!V) return nullptr;
    const double c0 = std::sqrt((long double) M_PIl), c1 = std::sqrt((long double) M_PI_2l);
    for (int j = 0; j < n; j++)
        for (int i = j; i >= 0; i -= 2) V[i + (size_t) j * n] *= j ? c1 : c0;
    return V;
}

void destroy(RectPlan * R) {
    if (R->stream) { cudaStreamSynchronize(R->stream); cudaStreamDestroy(R->stream); }
    if (R->rp_arr[0]) ft_destroy_rotation_plan(R->rp_arr[0]);
    for (int i = 0; i < 3; i++) {
        std::free(R->hostP[i]);
        std::free(R->hostPinv[i]);
        cudaFree(R->dP[i]);
        cudaFree(R->dPinv[i]);
    }
    cudaFree(R->d_scratch);
    cudaFree(R->d_stage);
    R->magic = 0;
    delete R;
}

// Out = op(U_even) In on the even columns and op(U_odd) In on the odd columns
bool left2(const RectPlan * R, const double * Ue, const double * Uo, bool trans, const double * in, double * out, int M,
           cudaStream_t st) {
    const int N = R->n;
    TrmmLaunch L{};
    L.n = N;
    L.ld_in = L.ld_out = 2LL * N;
    L.trans = trans;
    L.nclasses = 0;
    if ((M + 1) / 2 > 0) L.cls[L.nclasses++] = TrmmClass{Ue, in, out, (M + 1) / 2};
    if (M / 2 > 0) L.cls[L.nclasses++] = TrmmClass{Uo, in + N, out + N, M / 2};
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm(L, st);
    prof_end(st);
    return ok(e, "trmm kernel");
}

bool right(const RectPlan * R, const double * U, bool trans, const double * in, double * out, cudaStream_t st) {
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm_right(U, in, out, R->n, R->n, R->n, trans, st);
    prof_end(st);
    return ok(e, "trmm kernel");
}

// src/drivers.c:1143-1171; the rotation stage runs in place, the multiplies through the scratch
bool transform(RectPlan * R, bool forward, char T, double * A, int M, cudaStream_t st) {
    const int N = R->n;
    if (R->scratch_elems < (size_t) N * M) {
        cudaFree(R->d_scratch);
        R->d_scratch = nullptr;
        R->scratch_elems = 0;
        if (!ok(cudaMalloc(&R->d_scratch, sizeof(double) * (size_t) N * M), "cudaMalloc(scratch)")) return false;
        R->scratch_elems = (size_t) N * M;
        R->pub.B = R->d_scratch;
    }
    double * S = R->d_scratch;
    double * const * U = forward ? R->dP : R->dPinv;
    ft_rotation_plan * RP = R->rp_arr[0];
    const bool tN = T == 'N';
    if (forward == tN) {   // rectdisk2cheb 'N' / cheb2rectdisk 'T': hi2lo, left, right
        return rotation_sweeps(RP, true, A, A, M, N, st) && left2(R, U[0], U[1], !forward, A, S, M, st) &&
               right(R, U[2], forward, S, A, st);
    }
    // rectdisk2cheb 'T' / cheb2rectdisk 'N': right, left, lo2hi
    return right(R, U[2], !forward, A, S, st) && left2(R, U[0], U[1], forward, S, A, M, st) &&
           rotation_sweeps(RP, false, A, A, M, N, st);
}

int check(const RectPlan * R, char T, const double * A, int N, int M) {
    if (T != 'N' && T != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return FT_B200_EINVAL; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL matrix"); return FT_B200_EINVAL; }
    if (N != R->n) { set_error(FT_B200_EINVAL, "N does not match the plan's n"); return FT_B200_EINVAL; }
    if (M != N) { set_error(FT_B200_EINVAL, "Dunkl-Xu transforms need M == N (the right multiply is n x n)"); return FT_B200_EINVAL; }
    return FT_B200_OK;
}

void execute_host(const ft_harmonic_plan * P, bool forward, char T, double * A, int N, int M) {
    clear_error();
    RectPlan * R = as_rect(P);
    if (!R) { set_error(FT_B200_EINVAL, "not a Dunkl-Xu plan of this library"); return; }
    if (check(R, T, A, N, M) != FT_B200_OK) return;
    std::lock_guard<std::mutex> lk(R->mu);
    cudaSetDevice(R->device);
    const size_t elems = (size_t) N * M;
    if (R->stage_elems < elems) {
        cudaFree(R->d_stage);
        R->d_stage = nullptr;
        R->stage_elems = 0;
        if (!ok(cudaMalloc(&R->d_stage, sizeof(double) * elems), "cudaMalloc(stage)")) return;
        R->stage_elems = elems;
    }
    cudaStream_t st = R->stream;
    if (!ok(cudaMemcpyAsync(R->d_stage, A, sizeof(double) * elems, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(H2D)")) return;
    if (!transform(R, forward, T, R->d_stage, M, st)) return;
    if (!ok(cudaMemcpyAsync(A, R->d_stage, sizeof(double) * elems, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(D2H)")) return;
    ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

}  // namespace

bool rect_plan_destroy(ft_harmonic_plan * P) {
    RectPlan * R = as_rect(P);
    if (!R) return false;
    destroy(R);
    return true;
}

int rect_execute_dev(const ft_harmonic_plan * P, bool forward, char TRANS, double * dA, int N, int M, cudaStream_t st) {
    RectPlan * R = as_rect(P);
    if (!R) return -1;
    const int c = check(R, TRANS, dA, N, M);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(R->mu);
    return transform(R, forward, TRANS, dA, M, st) ? FT_B200_OK : ft_b200_last_status();
}

}  // namespace ftb

using namespace ftb;

extern "C" {

ft_harmonic_plan * ft_plan_rectdisk2cheb(const int n, const double beta) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    RectPlan * R = new RectPlan();
    std::memset(&R->pub, 0, sizeof(R->pub));
    R->n = n;
    R->rp_arr[0] = rotation_plan_new(RECT, n, 0.0, beta, 0.0);
    if (!R->rp_arr[0]) { delete R; return nullptr; }
    R->device = R->rp_arr[0]->device;
    R->hostP[0] = ultraspherical_to_chebyshev(n, beta + 1.0);
    R->hostP[1] = connection_ultraspherical(1, 0, n, beta + 2.0, 1.0);
    R->hostP[2] = ultraspherical_to_chebyshev(n, beta + 0.5);
    R->hostPinv[0] = chebyshev_to_ultraspherical(n, beta + 1.0);
    R->hostPinv[1] = connection_ultraspherical(0, 1, n, 1.0, beta + 2.0);
    R->hostPinv[2] = chebyshev_to_ultraspherical(n, beta + 0.5);
    const size_t nn = sizeof(double) * (size_t) n * n;
    for (int i = 0; i < 3; i++) {
        if (!R->hostP[i] || !R->hostPinv[i]) {
            set_error(FT_B200_ENOMEM, "host allocation (connection matrices)");
            destroy(R);
            return nullptr;
        }
        if (!ok(cudaMalloc(&R->dP[i], nn), "cudaMalloc(P)") ||
            !ok(cudaMemcpy(R->dP[i], R->hostP[i], nn, cudaMemcpyHostToDevice), "cudaMemcpy(P)") ||
            !ok(cudaMalloc(&R->dPinv[i], nn), "cudaMalloc(Pinv)") ||
            !ok(cudaMemcpy(R->dPinv[i], R->hostPinv[i], nn, cudaMemcpyHostToDevice), "cudaMemcpy(Pinv)")) {
            destroy(R);
            return nullptr;
        }
    }
    if (!ok(cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking), "cudaStreamCreate")) { destroy(R); return nullptr; }
    // src/drivers.c:1123-1141: one rotation plan, three connection pairs
    R->pub.RP = R->rp_arr;
    R->pub.MP = nullptr;
    R->pub.B = nullptr;
    R->pub.P = R->hostP;
    R->pub.Pinv = R->hostPinv;
    R->pub.beta = beta;
    R->pub.NRP = 1;
    R->pub.NMP = 0;
    R->pub.NP = 3;
    return &R->pub;
}

void ft_execute_rectdisk2cheb(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) {
    execute_host(P, true, TRANS, A, N, M);
}
void ft_execute_cheb2rectdisk(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) {
    execute_host(P, false, TRANS, A, N, M);
}

}  // extern "C"
