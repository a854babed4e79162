// Spin-weighted spherical harmonics (the reference's ft_plan_rotspinsphere,
// ft_execute_spinsph_hi2lo / lo2hi, ft_plan_spinsph2fourier, ft_execute_spinsph2fourier /
// ft_execute_fourier2spinsph: src/rotations.c:431-478, src/rotations/rotations_default.c:
// 17-29, 87-117, src/drivers.c:645-695, 1259-1361) on device memory.
//
// Data: an N x M complex matrix, column-major, interleaved (re, im) doubles.  Column 0
// holds order 0, columns 2m - 1 and 2m orders -m and m.  The sweeps of order m act on
// both parts with the same real rotations, in two stages (hi2lo order):
//   stage 1: min(|m|, |s|) sweeps of adjacent-row rotations (k, k + 1) from the spin
//            table (s2, c2)(k, j, d), d = ||m| - |s||, forward for m s >= 0 and
//            transposed otherwise;
//   stage 2: the sph sweeps of order d (rotations (k, k + 2), j = d - 2, d - 4, ..
//            down to (|m| + |s|) mod 2) with the sph table (the reference's s1, c1 hold
//            the sph table's values).
// lo2hi runs stage 2 then stage 1, each transposed.  Stage 2 is the rotation kernel's
// SPIN kind (rotations.cu: one lane carries the real and imaginary parts of both
// columns of an order through the sph wavefront); stage 1, at most |s| sweeps per
// column, is spin_stage1_kernel below, one thread per column.  The connection multiply
// (cblas_ztrmm with the real sph connection matrices stored as complex) is the real
// class-structured multiply on the real and the imaginary parts, with the matrices of
// the classes swapped for odd s.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "ft_internal.h"

namespace {
constexpr int kSpinRotMagic = 0x46545352;   // "FTSR"
constexpr int kSpinPlanMagic = 0x46545350;  // "FTSP"
}  // namespace

// Opaque in the public header, as in the reference's (src/fasttransforms.h:336).
struct ft_spin_rotation_plan_s {
    int magic = kSpinRotMagic;
    int n = 0, s = 0, device = 0;
    ft_rotation_plan * sph = nullptr;   // the sph table (device copy used by stage 2)
    double2 * d_sc2 = nullptr;      // (s2, c2) pairs, (l, j, m) at l + j n + m |s| n (src/rotations.c:458-468)
    int * d_counter = nullptr;
    std::map<int, std::pair<ftb::RotTask *, int>> tasks;   // M -> stage-2 tasks, longest first
    double * d_stage = nullptr;     // host-pointer calls
    size_t stage_elems = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;                  // host-pointer calls (staging buffer and stream)
    std::mutex task_mu;             // the task lists (taken inside calls that hold mu)
};

namespace ftb {

using SpinRotPlan = ft_spin_rotation_plan_s;

struct SpinHarmonicPlan {
    ft_spin_harmonic_plan pub;      // must stay the first member
    int magic = kSpinPlanMagic;
    int n = 0;
    ft_harmonic_plan * sph = nullptr;   // the sph connection matrices
    double * d_work = nullptr;      // 4 N M: real and imaginary parts in, real and imaginary parts out
    size_t work_elems = 0;
    double * d_stage = nullptr;
    size_t stage_elems = 0;
    std::mutex mu;
};

namespace {

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// The reference's rotation on both parts (fused form): x' = fma(c, x, s y), y' = fma(c, y, -(s x));
// the transposed rotation is the rotation by -s.
__device__ __forceinline__ void rot(double2 & x, double2 & y, double s, double c, bool transposed) {
    const double sg = transposed ? -s : s;
    const double syr = __dmul_rn(sg, y.x), sxr = __dmul_rn(sg, x.x);
    const double syi = __dmul_rn(sg, y.y), sxi = __dmul_rn(sg, x.y);
    const double2 xn = make_double2(__fma_rn(c, x.x, syr), __fma_rn(c, x.y, syi));
    const double2 yn = make_double2(__fma_rn(c, y.x, -sxr), __fma_rn(c, y.y, -sxi));
    x = xn;
    y = yn;
}

// Stage 1, one thread per complex column.  A sweep carries one element down (hi2lo) or up
// (lo2hi) the column; the elements and table pairs of the next LA positions are loaded
// together before any of them is rotated (none of them is written before it is loaded), so
// LA loads are in flight per thread instead of one.
constexpr int LA = 8;
__global__ void __launch_bounds__(64) spin_stage1_kernel(double2 * A, const double2 * __restrict__ tab, int N, int M,
                                                         int s, bool hi2lo) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= M) return;
    const int m = col == 0 ? 0 : ((col & 1) ? -((col + 1) / 2) : col / 2);
    const int as = abs(s), am = abs(m), d = abs(am - as), nsw = min(am, as);
    if (nsw == 0) return;
    // hi2lo: forward for m s >= 0; lo2hi: the transposes of those
    const bool transposed = (m * s >= 0) != hi2lo;
    double2 * a = A + (long long) col * N;
    const double2 * t = tab + (long long) d * as * N;
    double2 xs[LA], sc[LA];
    if (hi2lo) {
        for (int j = nsw - 1; j >= 0; --j) {
            const int top = N - 2 - d - j;   // rotations (k, k + 1), k = top .. 0
            if (top < 0) continue;
            const double2 * tj = t + (long long) j * N;
            double2 y = a[top + 1];
            for (int k0 = top; k0 >= 0; k0 -= LA) {
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (k0 - i >= 0) { xs[i] = a[k0 - i]; sc[i] = tj[k0 - i]; }
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (k0 - i >= 0) {
                        rot(xs[i], y, sc[i].x, sc[i].y, transposed);
                        a[k0 - i + 1] = y;
                        y = xs[i];
                    }
            }
            a[0] = y;
        }
    } else {
        for (int j = 0; j < nsw; ++j) {
            const int top = N - 2 - d - j;   // rotations (k, k + 1), k = 0 .. top
            if (top < 0) continue;
            const double2 * tj = t + (long long) j * N;
            double2 x = a[0];
            for (int k0 = 0; k0 <= top; k0 += LA) {
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (k0 + i <= top) { xs[i] = a[k0 + i + 1]; sc[i] = tj[k0 + i]; }
#pragma unroll
                for (int i = 0; i < LA; ++i)
                    if (k0 + i <= top) {
                        rot(x, xs[i], sc[i].x, sc[i].y, transposed);
                        a[k0 + i] = x;
                        x = xs[i];
                    }
            }
            a[top + 1] = x;
        }
    }
}

// complex N x M (interleaved) <-> real parts and imaginary parts, two N x M matrices
__global__ void split_kernel(const double2 * __restrict__ A, double * __restrict__ re, double * __restrict__ im, long long nm) {
    const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    const double2 v = A[i];
    re[i] = v.x;
    im[i] = v.y;
}
__global__ void merge_kernel(const double * __restrict__ re, const double * __restrict__ im, double2 * __restrict__ A, long long nm) {
    const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    A[i] = make_double2(re[i], im[i]);
}

unsigned blocks(long long n) { return (unsigned) ((n + 255) / 256); }

SpinRotPlan * as_srp(const ft_spin_rotation_plan * P) {
    SpinRotPlan * S = const_cast<SpinRotPlan *>(P);
    return (S && S->magic == kSpinRotMagic) ? S : nullptr;
}
SpinHarmonicPlan * as_sp(const ft_spin_harmonic_plan * P) {
    SpinHarmonicPlan * S = reinterpret_cast<SpinHarmonicPlan *>(const_cast<ft_spin_harmonic_plan *>(P));
    return (S && S->magic == kSpinPlanMagic) ? S : nullptr;
}

void destroy_srp(SpinRotPlan * P) {
    if (!P) return;
    for (auto & kv : P->tasks) cudaFree(kv.second.first);
    cudaFree(P->d_sc2);
    cudaFree(P->d_counter);
    cudaFree(P->d_stage);
    if (P->stream) cudaStreamDestroy(P->stream);
    if (P->sph) ft_destroy_rotation_plan(P->sph);
    P->magic = 0;
    delete P;
}

SpinRotPlan * make_srp(int n, int s) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    SpinRotPlan * P = new SpinRotPlan();
    P->n = n;
    P->s = s;
    P->sph = ft_plan_rotsphere(n);
    if (!P->sph) { delete P; return nullptr; }
    P->device = P->sph->device;
    const int as = std::abs(s);
    // the reference's expressions: integer products, one double division, the square root
    std::vector<double2> sc((size_t) as * n * n + 1, make_double2(0.0, 1.0));
    for (int m = 0; m < n; m++)
        for (int j = 0; j < as; j++)
            for (int l = 0; l < n - m - j; l++) {
                const double nums = (double) ((long long) (l + 1) * (l + m + 1));   // exact integers (no int overflow)
                const double numc = (double) ((long long) (2 * j + m + 1) * (2 * l + 2 * j + 2 * m + 3));
                const double den = (double) ((long long) (l + 2 * j + m + 2) * (l + 2 * j + 2 * m + 2));
                sc[(size_t) l + (size_t) j * n + (size_t) m * as * n] = make_double2(std::sqrt(nums / den), std::sqrt(numc / den));
            }
    if (!ok(cudaMalloc(&P->d_sc2, sizeof(double2) * sc.size()), "cudaMalloc(spin table)") ||
        !ok(cudaMemcpy(P->d_sc2, sc.data(), sizeof(double2) * sc.size(), cudaMemcpyHostToDevice), "cudaMemcpy(spin table)") ||
        !ok(cudaMalloc(&P->d_counter, sizeof(int)), "cudaMalloc(counter)") ||
        !ok(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking), "cudaStreamCreate")) {
        destroy_srp(P);
        return nullptr;
    }
    return P;
}

// stage-2 tasks for M columns: 16 orders of one parity each, longest first
bool spin_tasks(SpinRotPlan * P, int M, RotTask ** d, int * nt) {
    std::lock_guard<std::mutex> lk(P->task_mu);
    auto it = P->tasks.find(M);
    if (it != P->tasks.end()) { *d = it->second.first; *nt = it->second.second; return true; }
    const int mlast = Geo::last_order(SPIN, M), as = std::abs(P->s);
    std::vector<std::pair<long long, RotTask>> v;
    for (int p = 0; p < 2; p++)
        for (int mb = p; mb <= mlast; mb += 2 * Geo::task_orders(SPIN)) {
            int jlo, jhi;
            const int nsw = Geo::task_sweeps(SPIN, M, mb, 0, &jlo, &jhi, as);
            if (nsw > 0) v.push_back({(long long) nsw * (P->n - jlo), RotTask{0, mb}});
        }
    std::stable_sort(v.begin(), v.end(), [](const auto & a, const auto & b) { return a.first > b.first; });
    std::vector<RotTask> t;
    for (auto & x : v) t.push_back(x.second);
    RotTask * dt = nullptr;
    if (!t.empty() && (!ok(cudaMalloc(&dt, sizeof(RotTask) * t.size()), "cudaMalloc(tasks)") ||
                       !ok(cudaMemcpy(dt, t.data(), sizeof(RotTask) * t.size(), cudaMemcpyHostToDevice), "cudaMemcpy(tasks)")))
        return false;
    P->tasks[M] = {dt, (int) t.size()};
    *d = dt;
    *nt = (int) t.size();
    return true;
}

bool stage1(SpinRotPlan * P, bool hi2lo, double * A, int M, cudaStream_t st) {
    if (P->s == 0 || M < 1) return true;
    spin_stage1_kernel<<<(M + 63) / 64, 64, 0, st>>>(reinterpret_cast<double2 *>(A), P->d_sc2, P->n, M, P->s, hi2lo);
    count_launch();
    return ok(cudaGetLastError(), "spin stage 1");
}

bool stage2(SpinRotPlan * P, bool hi2lo, double * A, int M, cudaStream_t st) {
    RotTask * dt = nullptr;
    int nt = 0;
    if (!spin_tasks(P, M, &dt, &nt)) return false;
    if (nt == 0) return true;
    static thread_local RotLaunch L;   // large parameter block; kept off the stack
    L.nfields = 1;
    L.fields[0] = RotField{A, A, P->sph->d_scp, P->n, M, SPIN, (long long) P->n, 0, std::abs(P->s)};
    L.tasks = dt;
    L.ntasks = nt;
    L.counter = P->d_counter;
    L.chains = nullptr;   // no pass pipeline
    L.nchains = 0;
    L.prog = nullptr;
    prof_begin(FAM_ROT, st);
    const cudaError_t e = launch_rotations(SPIN, hi2lo, L, 0, st);
    prof_end(st);
    return ok(e, "spin rotation kernel");
}

bool rotations(SpinRotPlan * P, bool hi2lo, double * A, int M, cudaStream_t st) {
    return hi2lo ? (stage1(P, true, A, M, st) && stage2(P, true, A, M, st))
                 : (stage2(P, false, A, M, st) && stage1(P, false, A, M, st));
}

bool valid_cols(int M) {
    // the reference's loops visit columns 2m - 1 and 2m for m = 1 .. M/2 (src/drivers.c:677-695)
    if (M < 1 || M % 2 == 0) {
        set_error(FT_B200_EINVAL, "spin matrices need an odd number of columns M (orders -m, m in columns 2m - 1, 2m)");
        return false;
    }
    return true;
}

// the connection multiply on both parts: A <- op(U) A over the column classes
bool connection(SpinHarmonicPlan * S, bool inverse, bool trans, double * A, int M, cudaStream_t st) {
    HarmonicPlan * H = as_plan(S->sph);
    const long long nm = (long long) S->n * M;
    if (S->work_elems < 4 * (size_t) nm) {
        cudaFree(S->d_work);
        S->d_work = nullptr;
        S->work_elems = 0;
        if (!ok(cudaMalloc(&S->d_work, sizeof(double) * 4 * (size_t) nm), "cudaMalloc(spin work)")) return false;
        S->work_elems = 4 * (size_t) nm;
    }
    double * re = S->d_work, * im = re + nm, * re2 = im + nm, * im2 = re2 + nm;
    split_kernel<<<blocks(nm), 256, 0, st>>>(reinterpret_cast<const double2 *>(A), re, im, nm);
    count_launch();
    if (!ok(cudaGetLastError(), "split")) return false;
    const bool swap = S->pub.s % 2 != 0;   // odd s: classes 0, 3 take P2 and 1, 2 take P1
    if (!connection_multiply(H, inverse, trans, re, re2, M, st, swap) ||
        !connection_multiply(H, inverse, trans, im, im2, M, st, swap)) return false;
    merge_kernel<<<blocks(nm), 256, 0, st>>>(re2, im2, reinterpret_cast<double2 *>(A), nm);
    count_launch();
    return ok(cudaGetLastError(), "merge");
}

// src/drivers.c:1295-1361
bool transform(SpinHarmonicPlan * S, bool forward, char T, double * A, int M, cudaStream_t st) {
    SpinRotPlan * R = as_srp(S->pub.SRP);
    const bool tN = T == 'N';
    if (forward && tN) return rotations(R, true, A, M, st) && connection(S, false, false, A, M, st);
    if (forward) return connection(S, false, true, A, M, st) && rotations(R, false, A, M, st);
    if (tN) return connection(S, true, false, A, M, st) && rotations(R, false, A, M, st);
    return rotations(R, true, A, M, st) && connection(S, true, true, A, M, st);
}

// host-pointer calls: stage the 2 N M doubles on the device, run, copy back
template <typename F>
void on_host(double * A, int N, int M, int device, cudaStream_t st, double ** stage, size_t * stage_elems, F run) {
    cudaSetDevice(device);
    const size_t elems = 2 * (size_t) N * M;
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

int spin_check(SpinHarmonicPlan * P, char T, const void * A, int N, int M) {
    if (!P) { set_error(FT_B200_EINVAL, "not a spin plan of this library"); return FT_B200_EINVAL; }
    if (T != 'N' && T != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return FT_B200_EINVAL; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL matrix"); return FT_B200_EINVAL; }
    if (N != P->n) { set_error(FT_B200_EINVAL, "N does not match the plan's n"); return FT_B200_EINVAL; }
    if (!valid_cols(M)) return FT_B200_EINVAL;
    return FT_B200_OK;
}

void spin_rot_host(const ft_spin_rotation_plan * Pp, bool hi2lo, ft_complex * A, int M) {
    clear_error();
    SpinRotPlan * P = as_srp(Pp);
    if (!P || !A) { set_error(FT_B200_EINVAL, "NULL or foreign argument"); return; }
    if (!valid_cols(M)) return;
    std::lock_guard<std::mutex> lk(P->mu);
    on_host(reinterpret_cast<double *>(A), P->n, M, P->device, P->stream, &P->d_stage, &P->stage_elems,
            [&](double * d) { return rotations(P, hi2lo, d, M, P->stream); });
}

void spin_host(const ft_spin_harmonic_plan * Pp, bool forward, char T, ft_complex * A, int N, int M) {
    clear_error();
    SpinHarmonicPlan * P = as_sp(Pp);
    if (spin_check(P, T, A, N, M) != FT_B200_OK) return;
    std::lock_guard<std::mutex> lk(P->mu);
    SpinRotPlan * R = as_srp(P->pub.SRP);
    on_host(reinterpret_cast<double *>(A), N, M, R->device, R->stream, &P->d_stage, &P->stage_elems,
            [&](double * d) { return transform(P, forward, T, d, M, R->stream); });
}

// One spin column (the reference's ft_kernel_spinsph_hi2lo / lo2hi, src/rotations.c:479-485, whose
// bodies are src/rotations/rotations_default.c:87-117): the host column A (stride S complex
// entries) of order m; hi2lo runs the first stage (min(|m|, |s|) adjacent sweeps of the spin table,
// forward for m s >= 0, transposed otherwise) and then the sph sweeps of order d = ||m| - |s||;
// lo2hi runs the sph sweeps transposed and then the first stage with the other form.  Both
// stages are column.cu's wavefront on the complex column.
void spin_column_host(const ft_spin_rotation_plan * Pp, bool hi2lo, int m, ft_complex * A, int S) {
    clear_error();
    SpinRotPlan * P = as_srp(Pp);
    if (!P || !A) { set_error(FT_B200_EINVAL, "NULL or foreign argument"); return; }
    if (S < 1) { set_error(FT_B200_EINVAL, "S must be >= 1"); return; }
    if (m < -(1 << 30) || m > (1 << 30)) { set_error(FT_B200_EINVAL, "order m out of range"); return; }
    const int n = P->n, as = std::abs(P->s), am = std::abs(m);
    const int d = std::abs(am - as), mn = std::min(am, as), par = (am + as) % 2;
    const bool fwd1 = hi2lo == ((long long) m * P->s >= 0);
    const int len = std::max(column_touched(SPIN, n, hi2lo, 0, mn, d), column_touched(SPH, n, hi2lo, par, d, 0));
    if (len == 0) return;   // no rotation
    std::vector<double2> h(len);
    for (int k = 0; k < len; k++) h[k] = make_double2(A[(long long) k * S][0], A[(long long) k * S][1]);
    int prev = 0;
    if (!ok(cudaGetDevice(&prev), "cudaGetDevice") || !ok(cudaSetDevice(P->device), "cudaSetDevice")) return;
    double2 * dcol = nullptr;
    const size_t bytes = sizeof(double2) * (size_t) len;
    auto stage1 = [&] { return column_sweeps_dev(dcol, true, P->d_sc2, SPIN, n, 0, mn, hi2lo, fwd1, d, as, len); };
    auto stage2 = [&] { return column_sweeps_dev(dcol, true, P->sph->d_sc, SPH, n, par, d, hi2lo, hi2lo, 0, 0, len); };
    bool good = ok(cudaMalloc(&dcol, bytes), "cudaMalloc") && ok(cudaMemcpy(dcol, h.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(H2D)") &&
                (hi2lo ? (stage1() && stage2()) : (stage2() && stage1())) &&
                ok(cudaMemcpy(h.data(), dcol, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy(D2H)");
    cudaFree(dcol);
    cudaSetDevice(prev);
    if (good)
        for (int k = 0; k < len; k++) { A[(long long) k * S][0] = h[k].x; A[(long long) k * S][1] = h[k].y; }
}

}  // namespace
}  // namespace ftb

using namespace ftb;

extern "C" {

ft_spin_rotation_plan * ft_plan_rotspinsphere(const int n, const int s) { return make_srp(n, s); }

void ft_destroy_spin_rotation_plan(ft_spin_rotation_plan * SRP) { destroy_srp(as_srp(SRP)); }

void ft_execute_spinsph_hi2lo(const ft_spin_rotation_plan * SRP, ft_complex * A, ft_complex *, const int M) {
    spin_rot_host(SRP, true, A, M);
}
void ft_execute_spinsph_lo2hi(const ft_spin_rotation_plan * SRP, ft_complex * A, ft_complex *, const int M) {
    spin_rot_host(SRP, false, A, M);
}
void ft_kernel_spinsph_hi2lo(const ft_spin_rotation_plan * SRP, const int m, ft_complex * A, const int S) {
    spin_column_host(SRP, true, m, A, S);
}
void ft_kernel_spinsph_lo2hi(const ft_spin_rotation_plan * SRP, const int m, ft_complex * A, const int S) {
    spin_column_host(SRP, false, m, A, S);
}

int ft_b200_spin_rotations_dev(const ft_spin_rotation_plan * SRP, int hi2lo, double * dA, int M, void * stream) {
    clear_error();
    SpinRotPlan * P = as_srp(SRP);
    if (!P || !dA) { set_error(FT_B200_EINVAL, "NULL or foreign argument"); return FT_B200_EINVAL; }
    if (!valid_cols(M)) return FT_B200_EINVAL;
    return rotations(P, hi2lo != 0, dA, M, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

ft_spin_harmonic_plan * ft_plan_spinsph2fourier(const int n, const int s) {
    clear_error();
    SpinRotPlan * R = make_srp(n, s);
    if (!R) return nullptr;
    ft_harmonic_plan * H = ft_plan_sph2fourier(n);
    if (!H) { destroy_srp(R); return nullptr; }
    SpinHarmonicPlan * P = new SpinHarmonicPlan();
    P->n = n;
    P->sph = H;
    P->pub.SRP = R;
    P->pub.B = nullptr;
    P->pub.s = s;
    // the connection matrices as the reference keeps them: the real sph matrices stored as
    // complex (src/drivers.c:1273-1286)
    HarmonicPlan * HP = as_plan(H);
    ft_complex ** dst[4] = {&P->pub.P1, &P->pub.P2, &P->pub.P1inv, &P->pub.P2inv};
    const double * src[4] = {HP->hostP[0], HP->hostP[1], HP->hostPinv[0], HP->hostPinv[1]};
    for (int q = 0; q < 4; q++) {
        *dst[q] = static_cast<ft_complex *>(std::calloc((size_t) n * n, sizeof(ft_complex)));
        if (!*dst[q]) { set_error(FT_B200_ENOMEM, "host allocation"); ft_destroy_spin_harmonic_plan(&P->pub); return nullptr; }
        for (size_t i = 0; i < (size_t) n * n; i++) (*dst[q])[i][0] = src[q][i];
    }
    return &P->pub;
}

void ft_destroy_spin_harmonic_plan(ft_spin_harmonic_plan * Pp) {
    SpinHarmonicPlan * P = as_sp(Pp);
    if (!P) return;
    destroy_srp(as_srp(P->pub.SRP));
    if (P->sph) ft_destroy_harmonic_plan(P->sph);
    std::free(P->pub.P1);
    std::free(P->pub.P2);
    std::free(P->pub.P1inv);
    std::free(P->pub.P2inv);
    cudaFree(P->d_work);
    cudaFree(P->d_stage);
    P->magic = 0;
    delete P;
}

void ft_execute_spinsph2fourier(const char TRANS, const ft_spin_harmonic_plan * P, ft_complex * A, const int N, const int M) {
    spin_host(P, true, TRANS, A, N, M);
}
void ft_execute_fourier2spinsph(const char TRANS, const ft_spin_harmonic_plan * P, ft_complex * A, const int N, const int M) {
    spin_host(P, false, TRANS, A, N, M);
}

int ft_b200_execute_spin_dev(const ft_spin_harmonic_plan * Pp, int forward, char TRANS, double * dA, int N, int M, void * stream) {
    clear_error();
    SpinHarmonicPlan * P = as_sp(Pp);
    const int c = spin_check(P, TRANS, dA, N, M);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(P->mu);
    return transform(P, forward != 0, TRANS, dA, M, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

}  // extern "C"
