// Tetrahedral harmonics: the reference's ft_plan_tet2cheb, ft_execute_tet2cheb /
// ft_execute_cheb2tet and ft_execute_tet_hi2lo / lo2hi (src/drivers.c:26-54, 510-528,
// 1173-1257, src/rotations.c:297-321) on device memory.
//
// Data: an N x L x M column-major tensor (entry (i, l, m) at i + N l + N L m); slab m is the
// N x L matrix of index m.  The rotation stage (hi2lo) of slab m is
//   1. the triangle sweeps of order l + m down each column l < L - m (table RP1), run by the
//      rotation kernel's TRI kind with one field per slab: the field's base is moved back by m
//      columns so that column index = order, and its tasks start at order max(m, 1);
//   2. the sweeps across the slab: j = m - 1 .. 0, rotations of the column pairs (l, l + 1),
//      l = L - 2 - j .. 0 (table RP2), every row alike: tet_sweep_kernel, one thread per row
//      (coalesced across the warp), slabs with the most sweeps first.
// lo2hi runs 2 then 1, transposed.  The connection multiplies: P0 from the left on every
// column (one multiply over all L M columns), P1^T from the right on every slab, P2 along the
// m axis of every (i, l) fibre (a right multiply of the N L x M matrix), then the 3-D
// Chebyshev normalisation; each multiply is skipped where the reference skips it.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "ft_internal.h"

namespace ftb {
namespace {

constexpr int kTetMagic = 0x46545454;   // "FTTT"

struct TriStage {   // device task lists of the triangle sweeps, one launch per group of slabs
    struct Group { int m0, nslabs; RotTask * d_tasks; int ntasks; };
    std::vector<Group> groups;
};

struct TetPlan {
    ft_harmonic_plan pub;           // must stay the first member
    int magic = kTetMagic;
    int n = 0, device = 0;
    ft_rotation_plan * rp_arr[2] = {nullptr, nullptr};
    double * hostP[3] = {nullptr, nullptr, nullptr};
    double * hostPinv[3] = {nullptr, nullptr, nullptr};
    double * dP[3] = {nullptr, nullptr, nullptr};
    double * dPinv[3] = {nullptr, nullptr, nullptr};
    double * d_scratch = nullptr;   // one N x L x M tensor
    size_t scratch_elems = 0;
    double * d_stage = nullptr;     // host-pointer calls
    size_t stage_elems = 0;
    std::map<std::pair<int, int>, TriStage> tri;   // (L, M) -> task lists
    cudaStream_t stream = nullptr;
    std::mutex mu;
};

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

TetPlan * as_tet(const ft_harmonic_plan * P) {
    TetPlan * T = reinterpret_cast<TetPlan *>(const_cast<ft_harmonic_plan *>(P));
    return (T && T->magic == kTetMagic) ? T : nullptr;
}

// Sweeps across the columns of each slab: one thread per row of the slab; the pairs (s, c) are
// the same for every row of a slab (warp-uniform loads).  The elements and pairs of the next
// LA positions are loaded before any of them is rotated (none is written before it is loaded).
constexpr int LA = 8;
__global__ void __launch_bounds__(128) tet_sweep_kernel(double * A, const double2 * __restrict__ tab, int N, int L,
                                                        int M, int n, bool hi2lo) {
    const int m = M - 1 - (int) blockIdx.y;   // the slabs with the most sweeps first
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (m <= 0 || k >= N) return;
    double * a = A + (long long) N * L * m + k;   // element l of this row at a[l N]
    double xs[LA];
    double2 sc[LA];
    if (hi2lo) {
        for (int j = m - 1; j >= 0; --j) {
            const int top = L - 2 - j;   // rotations (l, l + 1), l = top .. 0
            if (top < 0) continue;
            const double2 * tj = tab + Geo::table_base(TRI, n, j);
            double y = a[(long long) (top + 1) * N];
            for (int l0 = top; l0 >= 0; l0 -= LA) {
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (l0 - i >= 0) { xs[i] = a[(long long) (l0 - i) * N]; sc[i] = tj[l0 - i]; }
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (l0 - i >= 0) {
                        const double s = sc[i].x, c = sc[i].y, x = xs[i];
                        const double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
                        a[(long long) (l0 - i + 1) * N] = __fma_rn(c, y, -sx);
                        y = __fma_rn(c, x, sy);
                    }
            }
            a[0] = y;
        }
    } else {
        for (int j = 0; j < m; ++j) {
            const int top = L - 2 - j;   // rotations (l, l + 1), l = 0 .. top
            if (top < 0) continue;
            const double2 * tj = tab + Geo::table_base(TRI, n, j);
            double x = a[0];
            for (int l0 = 0; l0 <= top; l0 += LA) {
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (l0 + i <= top) { xs[i] = a[(long long) (l0 + i + 1) * N]; sc[i] = tj[l0 + i]; }
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (l0 + i <= top) {
                        const double s = sc[i].x, c = sc[i].y, y = xs[i];
                        const double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
                        a[(long long) (l0 + i) * N] = __fma_rn(c, x, -sy);
                        x = __fma_rn(c, y, sx);
                    }
            }
            a[(long long) (top + 1) * N] = x;
        }
    }
}

// src/drivers.c:26-54: entry (i, l, m) times r if m == 0, r if l == 0, r if i == 0, then g, in
// that order (as the reference's loops apply them); out may equal in
__global__ void norm3d_kernel(const double * in, double * out, int N, int L, int M, double r, double g) {
    const long long total = (long long) N * L * M;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
        const int i = (int) (e % N);
        const long long q = e / N;
        const int l = (int) (q % L), m = (int) (q / L);
        double v = in[e];
        if (m == 0) v *= r;
        if (l == 0) v *= r;
        if (i == 0) v *= r;
        out[e] = v * g;
    }
}

// The triangle sweeps' task lists for an L x M tensor: tasks of 32 consecutive orders from
// max(m, 1) up to L - 1 for each slab m, grouped by at most kMaxFields slabs per launch,
// longest first within a launch.
bool build_tri_stage(int N, int L, int M, TriStage * T) {
    for (int m0 = 0; m0 < M; m0 += kMaxFields) {
        const int ns = std::min(kMaxFields, M - m0);
        std::vector<std::pair<long long, RotTask>> v;
        for (int f = 0; f < ns; f++) {
            const int m = m0 + f;
            for (int mb = std::max(m, 1); mb <= L - 1; mb += 32) {
                const int omax = std::min(mb + 31, L - 1);
                v.push_back({(long long) omax * N, RotTask{f, mb}});
            }
        }
        std::stable_sort(v.begin(), v.end(), [](const auto & a, const auto & b) { return a.first > b.first; });
        std::vector<RotTask> t;
        for (auto & x : v) t.push_back(x.second);
        RotTask * d = nullptr;
        if (!t.empty() && (!ok(cudaMalloc(&d, sizeof(RotTask) * t.size()), "cudaMalloc(tasks)") ||
                           !ok(cudaMemcpy(d, t.data(), sizeof(RotTask) * t.size(), cudaMemcpyHostToDevice), "cudaMemcpy(tasks)")))
            return false;
        T->groups.push_back({m0, ns, d, (int) t.size()});
    }
    return true;
}

void free_tri_stage(TriStage * T) {
    for (auto & g : T->groups) cudaFree(g.d_tasks);
    T->groups.clear();
}

bool tri_sweeps(const ft_rotation_plan * RP1, const TriStage & T, bool hi2lo, double * A, int N, int L, cudaStream_t st) {
    static thread_local RotLaunch Lr;   // large parameter block; kept off the stack
    for (const auto & g : T.groups) {
        if (g.ntasks == 0) continue;
        Lr.nfields = g.nslabs;
        for (int f = 0; f < g.nslabs; f++) {
            const int m = g.m0 + f;
            // column index = order: column l of slab m (order l + m) at base + (l + m) N
            double * base = A + (long long) N * L * m - (long long) N * m;
            Lr.fields[f] = RotField{base, base, RP1->d_scp, N, L, TRI, (long long) N, 0, 0};
        }
        Lr.tasks = g.d_tasks;
        Lr.ntasks = g.ntasks;
        Lr.counter = RP1->d_counter;
        Lr.chains = nullptr;
        Lr.nchains = 0;
        Lr.prog = nullptr;
        prof_begin(FAM_ROT, st);
        const cudaError_t e = launch_rotations(TRI, hi2lo, Lr, 0, st);
        prof_end(st);
        if (!ok(e, "rotation kernel")) return false;
    }
    return true;
}

bool tet_sweeps(const ft_rotation_plan * RP2, bool hi2lo, double * A, int N, int L, int M, cudaStream_t st) {
    if (M <= 1 || L < 2) return true;
    const dim3 grid((unsigned) ((N + 127) / 128), (unsigned) M);
    tet_sweep_kernel<<<grid, 128, 0, st>>>(A, RP2->d_sc, N, L, M, RP2->n, hi2lo);
    count_launch();
    return ok(cudaGetLastError(), "tet sweep kernel");
}

bool rotations(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, const TriStage & T, bool hi2lo, double * A,
               int L, int M, cudaStream_t st) {
    const int N = RP1->n;
    if (hi2lo) return tri_sweeps(RP1, T, true, A, N, L, st) && tet_sweeps(RP2, true, A, N, L, M, st);
    return tet_sweeps(RP2, false, A, N, L, M, st) && tri_sweeps(RP1, T, false, A, N, L, st);
}

bool valid_rot(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, int L, int M) {
    if (!RP1 || !RP2 || RP1->kind != TRI || RP2->kind != TRI) {
        set_error(FT_B200_EINVAL, "tetrahedral sweeps take two triangle rotation plans");
        return false;
    }
    if (RP1->n != RP2->n) { set_error(FT_B200_EINVAL, "the two rotation plans differ in n"); return false; }
    if (L < 1 || M < 1 || L > RP1->n) { set_error(FT_B200_EINVAL, "need 1 <= L <= n and M >= 1"); return false; }
    return true;
}

// rotations through the plan's cached task lists
bool plan_rotations(TetPlan * T, bool hi2lo, double * A, int L, int M, cudaStream_t st) {
    auto key = std::make_pair(L, M);
    auto it = T->tri.find(key);
    if (it == T->tri.end()) {
        TriStage S;
        if (!build_tri_stage(T->n, L, M, &S)) { free_tri_stage(&S); return false; }
        it = T->tri.emplace(key, std::move(S)).first;
    }
    return rotations(T->rp_arr[0], T->rp_arr[1], it->second, hi2lo, A, L, M, st);
}

bool left_all(const double * U, bool trans, const double * in, double * out, int N, long long ncols, cudaStream_t st) {
    TrmmLaunch Lt{};
    Lt.n = N;
    Lt.ld_in = Lt.ld_out = N;
    Lt.trans = trans;
    Lt.nclasses = 1;
    Lt.cls[0] = TrmmClass{U, in, out, (int) ncols};
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm(Lt, st);
    prof_end(st);
    return ok(e, "trmm kernel");
}

bool right_slabs(const double * U, bool trans, const double * in, double * out, int N, int L, int M, cudaStream_t st) {
    prof_begin(FAM_TRMM, st);
    cudaError_t e = cudaSuccess;
    for (int m = 0; m < M && e == cudaSuccess; m++)
        e = launch_trmm_right(U, in + (long long) N * L * m, out + (long long) N * L * m, L, N, N, trans, st);
    prof_end(st);
    return ok(e, "trmm kernel");
}

bool right_fibres(const double * U, bool trans, const double * in, double * out, int N, int L, int M, cudaStream_t st) {
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm_right(U, in, out, M, N * L, (long long) N * L, trans, st);
    prof_end(st);
    return ok(e, "trmm kernel");
}

bool normalize(const double * in, double * out, int N, int L, int M, bool transposed, cudaStream_t st) {
    const double r = transposed ? 1.41421356237309504880 : 0.70710678118654752440;   // M_SQRT2, M_SQRT1_2
    const double g = transposed ? 1.968701243215302468 : 0.507949087473927758;      // (pi/2)^1.5, (2/pi)^1.5 (src/ftinternal.h:59-60)
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    prof_begin(FAM_OTHER, st);
    norm3d_kernel<<<sms * 4, 256, 0, st>>>(in, out, N, L, M, r, g);
    count_launch();
    prof_end(st);
    return ok(cudaGetLastError(), "normalize");
}

// src/drivers.c:1197-1257 with N = L = M
bool transform(TetPlan * T, bool forward, char TR, double * A, int N, cudaStream_t st) {
    const int L = N, M = N;
    const size_t elems = (size_t) N * L * M;
    if (T->scratch_elems < elems) {
        cudaFree(T->d_scratch);
        T->d_scratch = nullptr;
        T->scratch_elems = 0;
        if (!ok(cudaMalloc(&T->d_scratch, sizeof(double) * elems), "cudaMalloc(scratch)")) return false;
        T->scratch_elems = elems;
        T->pub.B = T->d_scratch;
    }
    const double a = T->pub.alpha, b = T->pub.beta, g = T->pub.gamma, d = T->pub.delta;
    const bool u0 = (b + g + d != -2.5) || (a != -0.5);
    const bool u1 = (g + d != -1.5) || (b != -0.5);
    const bool u2 = (d != -0.5) || (g != -0.5);
    double * const * U = forward ? T->dP : T->dPinv;
    double * cur = A, * oth = T->d_scratch;
    auto flip = [&]() { std::swap(cur, oth); };
    if ((forward && TR == 'N') || (!forward && TR == 'T')) {
        // hi2lo, left, right on the slabs, along the fibres, normalisation back into A
        if (!plan_rotations(T, true, A, L, M, st)) return false;
        if (u0) { if (!left_all(U[0], !forward, cur, oth, N, (long long) L * M, st)) return false; flip(); }
        if (u1) { if (!right_slabs(U[1], forward, cur, oth, N, L, M, st)) return false; flip(); }
        if (u2) { if (!right_fibres(U[2], !forward, cur, oth, N, L, M, st)) return false; flip(); }
        return normalize(cur, A, N, L, M, !forward, st);
    }
    // normalisation, along the fibres, right on the slabs, left, then lo2hi in A; the
    // normalisation goes out of place when an odd number of multiplies follows, so that the
    // last multiply writes A
    const int k = (u0 ? 1 : 0) + (u1 ? 1 : 0) + (u2 ? 1 : 0);
    if (k % 2) { if (!normalize(A, oth, N, L, M, !forward, st)) return false; flip(); }
    else if (!normalize(A, A, N, L, M, !forward, st)) return false;
    if (u2) { if (!right_fibres(U[2], forward, cur, oth, N, L, M, st)) return false; flip(); }
    if (u1) { if (!right_slabs(U[1], !forward, cur, oth, N, L, M, st)) return false; flip(); }
    if (u0) { if (!left_all(U[0], forward, cur, oth, N, (long long) L * M, st)) return false; flip(); }
    return plan_rotations(T, false, A, L, M, st);
}

int check(const TetPlan * T, char TR, const double * A, int N, int L, int M) {
    if (TR != 'N' && TR != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return FT_B200_EINVAL; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL tensor"); return FT_B200_EINVAL; }
    if (N != T->n) { set_error(FT_B200_EINVAL, "N does not match the plan's n"); return FT_B200_EINVAL; }
    if (L != N || M != N) {
        set_error(FT_B200_EINVAL, "tetrahedral transforms need L == M == N (the multiplies along l and m are n x n)");
        return FT_B200_EINVAL;
    }
    return FT_B200_OK;
}

// host-pointer calls: stage the tensor on the device, run, copy back
template <typename F>
void on_host(double * A, size_t elems, int device, cudaStream_t st, double ** stage, size_t * stage_elems, F run) {
    cudaSetDevice(device);
    if (*stage_elems < elems) {
        cudaFree(*stage);
        *stage = nullptr;
        *stage_elems = 0;
        if (!ok(cudaMalloc(stage, sizeof(double) * elems), "cudaMalloc(stage)")) return;
        *stage_elems = elems;
    }
    if (!ok(cudaMemcpyAsync(*stage, A, sizeof(double) * elems, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(H2D)")) return;
    if (!run(*stage)) return;
    if (!ok(cudaMemcpyAsync(A, *stage, sizeof(double) * elems, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(D2H)")) return;
    ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

void destroy(TetPlan * T) {
    if (T->stream) { cudaStreamSynchronize(T->stream); cudaStreamDestroy(T->stream); }
    for (auto & kv : T->tri) free_tri_stage(&kv.second);
    for (int i = 0; i < 2; i++)
        if (T->rp_arr[i]) ft_destroy_rotation_plan(T->rp_arr[i]);
    for (int i = 0; i < 3; i++) {
        std::free(T->hostP[i]);
        std::free(T->hostPinv[i]);
        cudaFree(T->dP[i]);
        cudaFree(T->dPinv[i]);
    }
    cudaFree(T->d_scratch);
    cudaFree(T->d_stage);
    T->magic = 0;
    delete T;
}

void execute_host(const ft_harmonic_plan * P, bool forward, char TR, double * A, int N, int L, int M) {
    clear_error();
    TetPlan * T = as_tet(P);
    if (!T) { set_error(FT_B200_EINVAL, "not a tetrahedral plan of this library"); return; }
    if (check(T, TR, A, N, L, M) != FT_B200_OK) return;
    std::lock_guard<std::mutex> lk(T->mu);
    on_host(A, (size_t) N * L * M, T->device, T->stream, &T->d_stage, &T->stage_elems,
            [&](double * d) { return transform(T, forward, TR, d, N, T->stream); });
}

void rot_host(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, bool hi2lo, double * A, int L, int M) {
    clear_error();
    if (!A) { set_error(FT_B200_EINVAL, "NULL tensor"); return; }
    if (!valid_rot(RP1, RP2, L, M)) return;
    const int N = RP1->n;
    TriStage S;
    if (!build_tri_stage(N, L, M, &S)) { free_tri_stage(&S); return; }
    double * d = nullptr;
    size_t cap = 0;
    on_host(A, (size_t) N * L * M, RP1->device, 0, &d, &cap,
            [&](double * dA) { return rotations(RP1, RP2, S, hi2lo, dA, L, M, 0); });
    cudaFree(d);
    free_tri_stage(&S);
}

}  // namespace

bool tet_plan_destroy(ft_harmonic_plan * P) {
    TetPlan * T = as_tet(P);
    if (!T) return false;
    destroy(T);
    return true;
}

}  // namespace ftb

using namespace ftb;

extern "C" {

ft_harmonic_plan * ft_plan_tet2cheb(const int n, const double alpha, const double beta, const double gamma,
                                    const double delta) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    TetPlan * T = new TetPlan();
    std::memset(&T->pub, 0, sizeof(T->pub));
    T->n = n;
    T->rp_arr[0] = rotation_plan_new(TRI, n, alpha, beta, gamma + delta + 1.0);
    T->rp_arr[1] = T->rp_arr[0] ? rotation_plan_new(TRI, n, beta, gamma, delta) : nullptr;
    if (!T->rp_arr[0] || !T->rp_arr[1]) { destroy(T); return nullptr; }
    T->device = T->rp_arr[0]->device;
    // src/drivers.c:1179-1186
    T->hostP[0] = connection_jacobi(n, beta + gamma + delta + 2.0, alpha, -0.5, -0.5);
    T->hostP[1] = connection_jacobi(n, gamma + delta + 1.0, beta, -0.5, -0.5);
    T->hostP[2] = connection_jacobi(n, delta, gamma, -0.5, -0.5);
    T->hostPinv[0] = connection_jacobi(n, -0.5, -0.5, beta + gamma + delta + 2.0, alpha);
    T->hostPinv[1] = connection_jacobi(n, -0.5, -0.5, gamma + delta + 1.0, beta);
    T->hostPinv[2] = connection_jacobi(n, -0.5, -0.5, delta, gamma);
    const size_t nn = sizeof(double) * (size_t) n * n;
    for (int i = 0; i < 3; i++) {
        if (!T->hostP[i] || !T->hostPinv[i]) {
            set_error(FT_B200_ENOMEM, "host allocation (connection matrices)");
            destroy(T);
            return nullptr;
        }
        if (!ok(cudaMalloc(&T->dP[i], nn), "cudaMalloc(P)") ||
            !ok(cudaMemcpy(T->dP[i], T->hostP[i], nn, cudaMemcpyHostToDevice), "cudaMemcpy(P)") ||
            !ok(cudaMalloc(&T->dPinv[i], nn), "cudaMalloc(Pinv)") ||
            !ok(cudaMemcpy(T->dPinv[i], T->hostPinv[i], nn, cudaMemcpyHostToDevice), "cudaMemcpy(Pinv)")) {
            destroy(T);
            return nullptr;
        }
    }
    if (!ok(cudaStreamCreateWithFlags(&T->stream, cudaStreamNonBlocking), "cudaStreamCreate")) { destroy(T); return nullptr; }
    T->pub.RP = T->rp_arr;
    T->pub.MP = nullptr;
    T->pub.B = nullptr;
    T->pub.P = T->hostP;
    T->pub.Pinv = T->hostPinv;
    T->pub.alpha = alpha;
    T->pub.beta = beta;
    T->pub.gamma = gamma;
    T->pub.delta = delta;
    T->pub.NRP = 2;
    T->pub.NMP = 0;
    T->pub.NP = 3;
    return &T->pub;
}

void ft_execute_tet2cheb(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int L, const int M) {
    execute_host(P, true, TRANS, A, N, L, M);
}
void ft_execute_cheb2tet(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int L, const int M) {
    execute_host(P, false, TRANS, A, N, L, M);
}

void ft_execute_tet_hi2lo(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, double * A, const int L, const int M) {
    rot_host(RP1, RP2, true, A, L, M);
}
void ft_execute_tet_lo2hi(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, double * A, const int L, const int M) {
    rot_host(RP1, RP2, false, A, L, M);
}

int ft_b200_execute_tet_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int L, int M,
                            void * stream) {
    clear_error();
    TetPlan * T = as_tet(P);
    if (!T) { set_error(FT_B200_EINVAL, "not a tetrahedral plan of this library"); return FT_B200_EINVAL; }
    const int c = check(T, TRANS, dA, N, L, M);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(T->mu);
    return transform(T, forward != 0, TRANS, dA, N, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

int ft_b200_tet_rotations_dev(const ft_harmonic_plan * P, int hi2lo, double * dA, int L, int M, void * stream) {
    clear_error();
    TetPlan * T = as_tet(P);
    if (!T) { set_error(FT_B200_EINVAL, "not a tetrahedral plan of this library"); return FT_B200_EINVAL; }
    if (!dA) { set_error(FT_B200_EINVAL, "NULL tensor"); return FT_B200_EINVAL; }
    if (!valid_rot(T->rp_arr[0], T->rp_arr[1], L, M)) return FT_B200_EINVAL;
    std::lock_guard<std::mutex> lk(T->mu);
    return plan_rotations(T, hi2lo != 0, dA, L, M, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

}  // extern "C"
