// C ABI: plans, device residency, execute sequences, error reporting.
//
// Every transform is the reference's sequence (src/drivers.c:833-1021): a
// rotation stage and one or two triangular multiplies (plus the Chebyshev
// normalisation for tri).  The triangular multiplies run out of place between
// the caller's matrix and the plan's device scratch; the rotation stage is
// placed so that the result always lands back in the caller's matrix.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ft_internal.h"

namespace ftb {

namespace {
thread_local int t_status = FT_B200_OK;
thread_local std::string t_message;
std::atomic<unsigned long long> g_launches{0};
}  // namespace

namespace {
struct ProfRec { int family; cudaEvent_t a, b; };
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
std::vector<cudaEvent_t> g_prof_pool;
thread_local int t_prof_family = -1;
thread_local cudaEvent_t t_prof_a = nullptr;
cudaEvent_t prof_event() {
    if (!g_prof_pool.empty()) { cudaEvent_t e = g_prof_pool.back(); g_prof_pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

void prof_begin(int family, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_on) { t_prof_family = -1; return; }
    t_prof_family = family;
    t_prof_a = prof_event();
    cudaEventRecord(t_prof_a, st);
}

void prof_end(cudaStream_t st) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_on || t_prof_family < 0) return;
    cudaEvent_t b = prof_event();
    cudaEventRecord(b, st);
    g_prof.push_back({t_prof_family, t_prof_a, b});
    t_prof_family = -1;
}

std::atomic<int> g_host_threads{0};
int host_threads() { return g_host_threads.load(std::memory_order_relaxed); }

void set_error(int status, const std::string & msg) { t_status = status; t_message = msg; }
void clear_error() { t_status = FT_B200_OK; t_message.clear(); }
void count_launch(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

bool cuda_ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

bool check_device(int * dev_out) {
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) { t_status = FT_B200_ENODEV; return false; }
    int major = 0;
    if (!cuda_ok(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "cudaDeviceGetAttribute")) return false;
    if (major != 10) {
        set_error(FT_B200_ENODEV, "device " + std::to_string(dev) + " is not an sm_100 (B200) device");
        return false;
    }
    *dev_out = dev;
    return true;
}

}  // namespace

HarmonicPlan * as_plan(const ft_harmonic_plan * P) {
    if (!P) return nullptr;
    HarmonicPlan * H = reinterpret_cast<HarmonicPlan *>(const_cast<ft_harmonic_plan *>(P));
    return H->magic == kPlanMagic ? H : nullptr;
}

bool find_tasks(ft_rotation_plan * RP, int M, const RotTask ** d_tasks, int * ntasks) {
    std::lock_guard<std::mutex> lk(*RP->mu);
    auto it = RP->tasks->find(M);
    if (it == RP->tasks->end()) return false;
    *d_tasks = it->second.first;
    *ntasks = it->second.second;
    return true;
}

namespace {

int default_cols(int kind, int n) { return kind == SPH ? 2 * n - 1 : kind == TRI ? n : 4 * n - 3; }

// ---------------------------------------------------------------------------
// rotation plans
// ---------------------------------------------------------------------------
ft_rotation_plan * make_rotation_plan(int kind, int n, double alpha, double beta, double gamma) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    int dev = 0;
    if (!check_device(&dev)) return nullptr;
    const long long len = Geo::table_len(kind, n);
    ft_rotation_plan * RP = new (std::nothrow) ft_rotation_plan_s();
    if (!RP) { set_error(FT_B200_ENOMEM, "host allocation"); return nullptr; }
    RP->n = n; RP->kind = kind; RP->alpha = alpha; RP->beta = beta; RP->gamma = gamma; RP->device = dev;
    RP->s = static_cast<double *>(std::calloc(len, sizeof(double)));
    RP->c = static_cast<double *>(std::calloc(len, sizeof(double)));
    RP->mu = new std::mutex();
    RP->tasks = new std::map<int, std::pair<RotTask *, int>>();
    RP->sched = new std::map<int, RotSchedule *>();
    if (!RP->s || !RP->c) { set_error(FT_B200_ENOMEM, "host allocation"); ft_destroy_rotation_plan(RP); return nullptr; }
    rotation_tables(kind, n, alpha, beta, gamma, RP->s, RP->c);
    std::vector<double2> sc(len);
    for (long long i = 0; i < len; i++) sc[i] = make_double2(RP->s[i], RP->c[i]);
    if (!cuda_ok(cudaMalloc(&RP->d_sc, sizeof(double2) * len), "cudaMalloc(table)") ||
        !cuda_ok(cudaMemcpy(RP->d_sc, sc.data(), sizeof(double2) * len, cudaMemcpyHostToDevice), "cudaMemcpy(table)") ||
        !cuda_ok(cudaMalloc(&RP->d_counter, sizeof(int)), "cudaMalloc(counter)") || !rotation_plan_pad(RP)) {
        ft_destroy_rotation_plan(RP);
        return nullptr;
    }
    return RP;
}

// Device task list for an N x M matrix, longest first (cached per M).
bool get_tasks(ft_rotation_plan * RP, int M, RotTask ** d_tasks, int * ntasks) {
    std::lock_guard<std::mutex> lk(*RP->mu);
    auto it = RP->tasks->find(M);
    if (it != RP->tasks->end()) { *d_tasks = it->second.first; *ntasks = it->second.second; return true; }
    std::vector<RotTask> t = build_tasks(RP->kind, RP->n, M, 0);
    std::stable_sort(t.begin(), t.end(), [&](const RotTask & a, const RotTask & b) {
        return task_cost(RP->kind, RP->n, M, a.mbase) > task_cost(RP->kind, RP->n, M, b.mbase);
    });
    RotTask * d = nullptr;
    if (!t.empty()) {
        if (!cuda_ok(cudaMalloc(&d, sizeof(RotTask) * t.size()), "cudaMalloc(tasks)")) return false;
        if (!cuda_ok(cudaMemcpy(d, t.data(), sizeof(RotTask) * t.size(), cudaMemcpyHostToDevice), "cudaMemcpy(tasks)")) return false;
    }
    (*RP->tasks)[M] = {d, (int) t.size()};
    (*RP->sched)[M] = rot_schedule_new(t);
    *d_tasks = d; *ntasks = (int) t.size();
    return true;
}

// Columns the rotation stage leaves alone (orders 0 and 1): copied when the
// stage runs out of place.
int untouched_cols(int kind, int M) { return std::min(M, kind == TRI ? 1 : (kind == RECT ? 2 : 3)); }

// Device memory of one execute call (call_scratch): the out-of-place matrix S, the rotation
// kernel's work counter and the pass pipeline's progress words, so that calls on one plan share
// none of them.
struct CallScratch {
    void * base = nullptr;     // the one pool allocation holding the rest
    double * S = nullptr;
    int * counter = nullptr;
    int * prog = nullptr;
    int prog_cap = 0;
};

bool rotations(ft_rotation_plan * RP, bool hi2lo, const double * in, double * out, int M, long long lda, cudaStream_t st,
               const CallScratch * cs = nullptr) {
    RotTask * d_tasks = nullptr;
    int ntasks = 0;
    if (!get_tasks(RP, M, &d_tasks, &ntasks)) return false;
    if (in != out) {
        const int nc = untouched_cols(RP->kind, M);
        if (!cuda_ok(cudaMemcpy2DAsync(out, lda * sizeof(double), in, lda * sizeof(double), RP->n * sizeof(double), nc,
                                       cudaMemcpyDeviceToDevice, st), "cudaMemcpy2DAsync")) return false;
    }
    if (ntasks == 0) return true;
    static thread_local RotLaunch L;   // large parameter block; kept off the stack
    L.nfields = 1;
    L.fields[0] = RotField{in, out, RP->d_scp, RP->n, M, RP->kind, lda, 0};
    L.tasks = d_tasks;
    L.ntasks = ntasks;
    L.counter = cs ? cs->counter : RP->d_counter;
    // out of place, the destination holds nothing live yet: the autotuner may time there
    double * const dead[1] = {out};
    prof_begin(FAM_ROT, st);
    RotSchedule * sched = nullptr;
    {
        std::lock_guard<std::mutex> lk(*RP->mu);
        auto it = RP->sched->find(M);
        if (it != RP->sched->end()) sched = it->second;
    }
    const cudaError_t e = launch_rotations(RP->kind, hi2lo, L, 0, st, in != out ? dead : nullptr, sched,
                                           cs ? cs->prog : nullptr, cs ? cs->prog_cap : 0);
    prof_end(st);
    return cuda_ok(e, "rotation kernel");
}

// Vector-field sweeps (src/drivers.c:168-276): order m's rotations on columns 2m + 1 and
// 2m + 2 for m = 2 .. M/2 - 1, i.e. the sph sweeps of the matrix that starts two columns
// later and has M - 2 columns; columns 0 and 1 are left alone.
bool rotations_sphv(ft_rotation_plan * RP, bool hi2lo, const double * in, double * out, int M, long long lda,
                    cudaStream_t st, const CallScratch * cs = nullptr) {
    const int lead = std::min(M, 2);
    if (in != out && !cuda_ok(cudaMemcpy2DAsync(out, lda * sizeof(double), in, lda * sizeof(double), RP->n * sizeof(double),
                                                lead, cudaMemcpyDeviceToDevice, st), "cudaMemcpy2DAsync")) return false;
    if (M <= 2) return true;
    return rotations(RP, hi2lo, in + 2 * lda, out + 2 * lda, M - 2, lda, st, cs);
}

// sph and disk: order m occupies the column pair (2m - 1, 2m) for m = 2 .. M/2
// (src/drivers.c:94-110, 414-430), so an even M >= 4 would put the last order's
// second column at index M, past the matrix; such M are rejected.
bool valid_pairs(int kind, int M) {
    if (kind != TRI && kind != RECT && M >= 4 && M % 2 == 0) {
        set_error(FT_B200_EINVAL, "sph and disk matrices need an odd number of columns M");
        return false;
    }
    return true;
}

bool valid_MN(int kind, int n, int N, int M) {
    if (N != n) { set_error(FT_B200_EINVAL, "N does not match the plan's n"); return false; }
    if (M < 1) { set_error(FT_B200_EINVAL, "M must be positive"); return false; }
    if (!valid_pairs(kind, M)) return false;
    if (kind == TRI && M != N) { set_error(FT_B200_EINVAL, "tri transforms need M == N"); return false; }
    return true;
}

// sph / disk: four stride-4N column classes, P[0] on classes 0 and 3, P[1] on 1 and 2
// (swapped for the sph vector-field transforms, src/drivers.c:867-899)
bool trmm4(HarmonicPlan * H, bool inverse, bool trans, const double * in, double * out, int M, cudaStream_t st,
           bool swap = false) {
    const int N = H->n;
    TrmmLaunch L{};
    L.n = N;
    L.ld_in = L.ld_out = 4LL * N;
    L.trans = trans;
    const int ncols[4] = {(M + 3) / 4, (M + 2) / 4, (M + 1) / 4, M / 4};
    double * const * U = inverse ? H->dPinv : H->dP;
    int c = 0;
    for (int r = 0; r < 4; r++) {
        if (ncols[r] <= 0) continue;
        L.cls[c].U = ((r == 0 || r == 3) != swap) ? U[0] : U[1];
        L.cls[c].in = in + (long long) r * N;
        L.cls[c].out = out + (long long) r * N;
        L.cls[c].ncols = ncols[r];
        c++;
    }
    L.nclasses = c;
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm(L, st);
    prof_end(st);
    return cuda_ok(e, "trmm kernel");
}

bool trmm_left1(HarmonicPlan * H, const double * U, bool trans, const double * in, double * out, int M, cudaStream_t st) {
    TrmmLaunch L{};
    L.n = H->n;
    L.ld_in = L.ld_out = H->n;
    L.trans = trans;
    L.nclasses = 1;
    L.cls[0] = TrmmClass{U, in, out, M};
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm(L, st);
    prof_end(st);
    return cuda_ok(e, "trmm kernel");
}

bool trmm_right(const double * U, const double * in, double * out, int N, long long lda, bool trans, cudaStream_t st) {
    prof_begin(FAM_TRMM, st);
    const cudaError_t e = launch_trmm_right(U, in, out, N, N, lda, trans, st);
    prof_end(st);
    return cuda_ok(e, "trmm kernel");
}

bool normalize(double * A, int N, int M, long long lda, bool transposed, cudaStream_t st) {
    prof_begin(FAM_OTHER, st);
    const cudaError_t e = launch_cheb_normalize(A, N, M, lda, transposed, st);
    prof_end(st);
    return cuda_ok(e, "normalize");
}

// The library's stream-ordered memory pool on device dev (created on first use, kept until the
// process exits).  Its release threshold is unlimited: memory a call frees goes back to the
// pool once the call's stream reaches the free and serves the next call, without returning to
// the driver in between.
cudaMemPool_t call_pool(int dev) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (!cuda_ok(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate")) return nullptr;
    uint64_t keep = UINT64_MAX;
    if (!cuda_ok(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute")) {
        cudaMemPoolDestroy(pool);
        return nullptr;
    }
    pools[dev] = pool;
    return pool;
}

// Scratch of one execute call, allocated on its stream from the pool: elems doubles, the work
// counter and prog_cap progress words.  call_scratch_free returns it on the same stream, after
// the work enqueued before it.
bool call_scratch(int dev, size_t elems, int prog_cap, cudaStream_t st, CallScratch * cs) {
    cudaMemPool_t pool = call_pool(dev);
    if (!pool) return false;
    const size_t s_bytes = (elems * sizeof(double) + 255) & ~(size_t) 255;
    const size_t bytes = s_bytes + 256 + sizeof(int) * (size_t) std::max(prog_cap, 1);
    void * p = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
    if (e != cudaSuccess) {
        set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA,
                  std::string("cudaMallocFromPoolAsync(call scratch): ") + cudaGetErrorString(e));
        return false;
    }
    char * b = static_cast<char *>(p);
    cs->base = p;
    cs->S = reinterpret_cast<double *>(b);
    cs->counter = reinterpret_cast<int *>(b + s_bytes);
    cs->prog = reinterpret_cast<int *>(b + s_bytes + 256);
    cs->prog_cap = prog_cap;
    return true;
}

void call_scratch_free(CallScratch & cs, cudaStream_t st) {
    if (cs.base) cudaFreeAsync(cs.base, st);
    cs = CallScratch{};
}

int execute_dev_impl(HarmonicPlan * H, bool forward, char TRANS, double * A, int N, int M, cudaStream_t st,
                     bool vector = false) {
    if (TRANS != 'N' && TRANS != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return t_status; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL matrix"); return t_status; }
    if (vector && H->kind != SPH) { set_error(FT_B200_EINVAL, "vector-field transforms take a sph plan"); return t_status; }
    if (!valid_MN(H->kind, H->n, N, M)) return t_status;
    ft_rotation_plan * RP = H->rp_arr[0];
    // Everything this call writes besides A comes from the pool, on st: two calls on one plan
    // (from two threads, on two streams) share no device memory.  The pass pipeline needs a
    // progress word per pass of every task, at most ceil(sweeps / 16) <= n / 16 + 1 per task.
    RotTask * d_tasks = nullptr;
    int ntasks = 0;
    if (!get_tasks(RP, vector ? std::max(M - 2, 1) : M, &d_tasks, &ntasks)) return t_status;
    struct Guard {
        CallScratch cs;
        cudaStream_t st;
        ~Guard() { call_scratch_free(cs, st); }
    } guard{CallScratch{}, st};
    if (!call_scratch(H->device, (size_t) N * M, ntasks * (N / 16 + 2), st, &guard.cs)) return t_status;
    const CallScratch * const cs = &guard.cs;
    double * S = guard.cs.S;
    const bool tN = TRANS == 'N';
    const long long lda = N;
    if (H->kind != TRI) {
        // rotations (out of place) then trmm back, or trmm out then rotations back
        // (sph vector fields: the shifted sweeps and the swapped matrices, src/drivers.c:867-899)
        auto rot = [&](bool hi2lo, const double * in, double * out) {
            return vector ? rotations_sphv(RP, hi2lo, in, out, M, lda, st, cs) : rotations(RP, hi2lo, in, out, M, lda, st, cs);
        };
        if (forward && tN) {            // hi2lo, P
            if (!rot(true, A, S)) return t_status;
            if (!trmm4(H, false, false, S, A, M, st, vector)) return t_status;
        } else if (forward) {           // P^T, lo2hi
            if (!trmm4(H, false, true, A, S, M, st, vector)) return t_status;
            if (!rot(false, S, A)) return t_status;
        } else if (tN) {                // Pinv, lo2hi
            if (!trmm4(H, true, false, A, S, M, st, vector)) return t_status;
            if (!rot(false, S, A)) return t_status;
        } else {                        // hi2lo, Pinv^T
            if (!rot(true, A, S)) return t_status;
            if (!trmm4(H, true, true, S, A, M, st, vector)) return t_status;
        }
        return FT_B200_OK;
    }
    // tri: src/drivers.c:921-957
    const double a = H->pub.alpha, b = H->pub.beta, g = H->pub.gamma;
    const bool left = (b + g != -1.5) || (a != -0.5);
    const bool right = (g != -0.5) || (b != -0.5);
    const int k = (left ? 1 : 0) + (right ? 1 : 0);
    double * U0 = forward ? H->dP[0] : H->dPinv[0];
    double * U1 = forward ? H->dP[1] : H->dPinv[1];
    double * cur = A;
    double * oth = S;
    auto flip = [&]() { std::swap(cur, oth); };
    const bool rot_hi2lo_first = (forward && tN) || (!forward && !tN);
    if (rot_hi2lo_first) {
        // rotation, then left / right, then normalisation; the rotation goes out of place iff k is odd
        double * rot_out = (k % 2) ? S : A;
        if (!rotations(RP, true, A, rot_out, M, lda, st, cs)) return t_status;
        cur = rot_out; oth = (rot_out == A) ? S : A;
        if (forward) {   // tri2cheb 'N': left N P0, right T P1
            if (left) { if (!trmm_left1(H, U0, false, cur, oth, M, st)) return t_status; flip(); }
            if (right) { if (!trmm_right(U1, cur, oth, N, lda, true, st)) return t_status; flip(); }
            if (!normalize(cur, N, M, lda, false, st)) return t_status;
        } else {         // cheb2tri 'T': left T Pinv0, right N Pinv1
            if (left) { if (!trmm_left1(H, U0, true, cur, oth, M, st)) return t_status; flip(); }
            if (right) { if (!trmm_right(U1, cur, oth, N, lda, false, st)) return t_status; flip(); }
            if (!normalize(cur, N, M, lda, true, st)) return t_status;
        }
    } else {
        // normalisation, right / left, then the rotation back into A
        if (!normalize(A, N, M, lda, !forward, st)) return t_status;
        if (forward) {   // tri2cheb 'T': right N P1, left T P0
            if (right) { if (!trmm_right(U1, cur, oth, N, lda, false, st)) return t_status; flip(); }
            if (left) { if (!trmm_left1(H, U0, true, cur, oth, M, st)) return t_status; flip(); }
        } else {         // cheb2tri 'N': right T Pinv1, left N Pinv0
            if (right) { if (!trmm_right(U1, cur, oth, N, lda, true, st)) return t_status; flip(); }
            if (left) { if (!trmm_left1(H, U0, false, cur, oth, M, st)) return t_status; flip(); }
        }
        if (!rotations(RP, false, cur, A, M, lda, st, cs)) return t_status;
    }
    return FT_B200_OK;
}

HarmonicPlan * make_harmonic_plan(int kind, int n, double alpha, double beta, double gamma) {
    clear_error();
    if (n < 1) { set_error(FT_B200_EINVAL, "n must be positive"); return nullptr; }
    int dev = 0;
    if (!check_device(&dev)) return nullptr;
    HarmonicPlan * H = new (std::nothrow) HarmonicPlan();
    if (!H) { set_error(FT_B200_ENOMEM, "host allocation"); return nullptr; }
    std::memset(&H->pub, 0, sizeof(H->pub));
    H->magic = kPlanMagic;
    H->kind = kind; H->n = n; H->Mdef = default_cols(kind, n); H->device = dev;
    H->pub.alpha = alpha; H->pub.beta = beta; H->pub.gamma = gamma;
    H->pub.RP = H->rp_arr;
    H->pub.P = H->hostP;
    H->pub.Pinv = H->hostPinv;
    H->pub.NRP = 1; H->pub.NMP = 0; H->pub.NP = 2;
    auto fail = [&]() { ft_destroy_harmonic_plan(&H->pub); return (HarmonicPlan *) nullptr; };
    H->rp_arr[0] = make_rotation_plan(kind, n, alpha, beta, gamma);
    if (!H->rp_arr[0]) return fail();
    if (kind == SPH) {   // src/drivers.c:816-831
        H->hostP[0] = connection_legendre_to_chebyshev(1, 0, n);
        H->hostP[1] = connection_ultraspherical(1, 0, n, 1.5, 1.0);
        H->hostPinv[0] = connection_chebyshev_to_legendre(0, 1, n);
        H->hostPinv[1] = connection_ultraspherical(0, 1, n, 1.0, 1.5);
    } else if (kind == TRI) {   // src/drivers.c:901-919
        H->hostP[0] = connection_jacobi(n, beta + gamma + 1.0, alpha, -0.5, -0.5);
        H->hostP[1] = connection_jacobi(n, gamma, beta, -0.5, -0.5);
        H->hostPinv[0] = connection_jacobi(n, -0.5, -0.5, beta + gamma + 1.0, alpha);
        H->hostPinv[1] = connection_jacobi(n, -0.5, -0.5, gamma, beta);
    } else {   // src/drivers.c:959-987 with src/transforms.c:157-180 inlined
        H->hostP[0] = connection_jacobi(n, beta, alpha, -0.5, -0.5);
        H->hostP[1] = connection_jacobi(n, beta, alpha + 1.0, -0.5, 0.5);
        H->hostPinv[0] = connection_jacobi(n, -0.5, -0.5, beta, alpha);
        H->hostPinv[1] = connection_jacobi(n, -0.5, 0.5, beta, alpha + 1.0);
        if (H->hostP[0] && H->hostPinv[0]) {
            std::vector<double> sclrow(n), sclcol(n);
            for (int i = 0; i < n; i++) {
                sclrow[i] = i ? std::sqrt((long double) M_2_PIl) : std::sqrt((long double) M_1_PIl);
                sclcol[i] = i ? std::sqrt((long double) M_PI_2l) : std::sqrt((long double) M_PIl);
            }
            for (int j = 0; j < n; j++)
                for (int i = 0; i <= j; i++) {
                    H->hostP[0][i + (size_t) j * n] *= sclrow[i];
                    H->hostPinv[0][i + (size_t) j * n] *= sclcol[j];
                }
            const double cst0 = std::pow(2.0, 0.5 * (alpha + beta + 2.0));
            const double cst1 = cst0 * 0.797884560802865355;       // sqrt(2/pi), src/ftinternal.h:66
            const double cst0inv = std::pow(2.0, -0.5 * (alpha + beta + 2.0));
            const double cst1inv = cst0inv * 1.253314137315500251; // sqrt(pi/2), src/ftinternal.h:65
            for (int j = 0; j < n; j++)
                for (int i = 0; i <= j; i++) {
                    H->hostP[0][i + (size_t) j * n] *= cst0;
                    H->hostP[1][i + (size_t) j * n] *= cst1;
                    H->hostPinv[0][i + (size_t) j * n] *= cst0inv;
                    H->hostPinv[1][i + (size_t) j * n] *= cst1inv;
                }
        }
    }
    for (int i = 0; i < 2; i++)
        if (!H->hostP[i] || !H->hostPinv[i]) { set_error(FT_B200_ENOMEM, "host allocation (connection matrices)"); return fail(); }
    const size_t nn = (size_t) n * n * sizeof(double);
    for (int i = 0; i < 2; i++) {
        if (!cuda_ok(cudaMalloc(&H->dP[i], nn), "cudaMalloc(P)") ||
            !cuda_ok(cudaMemcpy(H->dP[i], H->hostP[i], nn, cudaMemcpyHostToDevice), "cudaMemcpy(P)") ||
            !cuda_ok(cudaMalloc(&H->dPinv[i], nn), "cudaMalloc(Pinv)") ||
            !cuda_ok(cudaMemcpy(H->dPinv[i], H->hostPinv[i], nn, cudaMemcpyHostToDevice), "cudaMemcpy(Pinv)"))
            return fail();
    }
    if (!cuda_ok(cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking), "cudaStreamCreate")) return fail();
    // build the default task list now, outside any later stream capture
    RotTask * dt; int nt;
    if (!get_tasks(H->rp_arr[0], H->Mdef, &dt, &nt)) return fail();
    // the pool keeps what one call at the default size takes, ready for the first call
    CallScratch warm;
    if (!call_scratch(dev, (size_t) n * H->Mdef, nt * (n / 16 + 2), H->stream, &warm)) return fail();
    call_scratch_free(warm, H->stream);
    if (!cuda_ok(cudaStreamSynchronize(H->stream), "cudaStreamSynchronize")) return fail();
    return H;
}

// host-pointer execution: stage A on the device, run, copy back, wait (one call per plan at a
// time: concurrent calls from other threads wait for the plan's staging buffer and stream)
void execute_host(const ft_harmonic_plan * P, bool forward, char TRANS, double * A, int N, int M, bool vector = false) {
    clear_error();
    HarmonicPlan * H = as_plan(P);
    if (!H) { set_error(FT_B200_EINVAL, "not a plan created by this library"); return; }
    std::lock_guard<std::mutex> lk(H->host_mu);
    if (TRANS != 'N' && TRANS != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL matrix"); return; }
    if (!valid_MN(H->kind, H->n, N, M)) return;
    const size_t elems = (size_t) N * M;
    if (elems > H->stage_elems) {
        if (H->d_stage) cudaFree(H->d_stage);
        H->d_stage = nullptr; H->stage_elems = 0;
        if (!cuda_ok(cudaMalloc(&H->d_stage, elems * sizeof(double)), "cudaMalloc(stage)")) return;
        H->stage_elems = elems;
    }
    if (!cuda_ok(cudaMemcpyAsync(H->d_stage, A, elems * sizeof(double), cudaMemcpyHostToDevice, H->stream), "cudaMemcpyAsync(H2D)")) return;
    if (execute_dev_impl(H, forward, TRANS, H->d_stage, N, M, H->stream, vector) != FT_B200_OK) { cudaStreamSynchronize(H->stream); return; }
    if (!cuda_ok(cudaMemcpyAsync(A, H->d_stage, elems * sizeof(double), cudaMemcpyDeviceToHost, H->stream), "cudaMemcpyAsync(D2H)")) return;
    cuda_ok(cudaStreamSynchronize(H->stream), "cudaStreamSynchronize");
}

void rotations_host(const ft_rotation_plan * RPc, bool hi2lo, double * A, int M, int kind) {
    clear_error();
    ft_rotation_plan * RP = const_cast<ft_rotation_plan *>(RPc);
    if (!RP || !A) { set_error(FT_B200_EINVAL, "NULL argument"); return; }
    if (RP->kind != kind) { set_error(FT_B200_EINVAL, "rotation plan of another family"); return; }
    if (M < 1) { set_error(FT_B200_EINVAL, "M must be positive"); return; }
    if (!valid_pairs(kind, M)) return;
    const size_t elems = (size_t) RP->n * M;
    double * d = nullptr;
    if (!cuda_ok(cudaMalloc(&d, elems * sizeof(double)), "cudaMalloc")) return;
    if (cuda_ok(cudaMemcpy(d, A, elems * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(H2D)") &&
        rotations(RP, hi2lo, d, d, M, RP->n, 0) &&
        cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize"))
        cuda_ok(cudaMemcpy(A, d, elems * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy(D2H)");
    cudaFree(d);
}

// sphv (src/drivers.c:168-276): order m on the column pair (2m + 1, 2m + 2), m = 2 .. M/2 - 1, the
// sph sweeps on the matrix two columns in; orders exist for M >= 7
void rotations_sphv_host(const ft_rotation_plan * RPc, bool hi2lo, double * A, int M) {
    clear_error();
    ft_rotation_plan * RP = const_cast<ft_rotation_plan *>(RPc);
    if (!RP || !A) { set_error(FT_B200_EINVAL, "NULL argument"); return; }
    if (RP->kind != SPH) { set_error(FT_B200_EINVAL, "sphv sweeps take a sph rotation plan"); return; }
    if (M < 1) { set_error(FT_B200_EINVAL, "M must be positive"); return; }
    if (!valid_pairs(SPH, M) || M < 7) return;
    const size_t elems = (size_t) RP->n * M;
    double * d = nullptr;
    if (!cuda_ok(cudaMalloc(&d, elems * sizeof(double)), "cudaMalloc")) return;
    if (cuda_ok(cudaMemcpy(d, A, elems * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(H2D)") &&
        rotations_sphv(RP, hi2lo, d, d, M, RP->n, 0) &&
        cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize"))
        cuda_ok(cudaMemcpy(A, d, elems * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy(D2H)");
    cudaFree(d);
}

// ---------------------------------------------------------------------------
// batches: many fields in one launch per stage
// ---------------------------------------------------------------------------
struct TrmmSet {
    TrmmBatchClass * d_classes = nullptr;
    TrmmTile * d_tiles[4] = {nullptr, nullptr, nullptr, nullptr};   // tile order per multiply mode
    int ntiles = 0;
};
struct BatchCtx {
    RotTask * d_tasks = nullptr;
    int ntasks = 0;
    TrmmSet left, right;                           // right: tri only
    double * d_work = nullptr;                     // one scratch matrix per field
    std::vector<size_t> work_off;
    int * d_counter = nullptr;
    std::vector<void *> allocs;
    BlkTaskList blk_tasks;                         // blocked-sweep tasks (built on first blocked call)
    bool blk_ready = false;
    BlkTaskList mx_tasks;                          // the same for the split-BF16 products (pairs of fields)
    bool mx_ready = false;
    float * d_T = nullptr;                         // their task-major copy of the columns
    void * mx_trmm = nullptr;                      // sliced inputs and tile lists of the tensor-core multiply
    RotSchedule * sched = nullptr;                 // pass pipeline of the rotation tasks
};
std::mutex g_batch_mu;
std::map<std::string, BatchCtx *> g_batches;

std::string batch_key(HarmonicPlan * const * H, const int * N, const int * M, int nf) {
    std::string k;
    int dev = 0;
    cudaGetDevice(&dev);
    k += std::to_string(dev) + ":";
    for (int f = 0; f < nf; f++) k += std::to_string((uintptr_t) H[f]) + "," + std::to_string(N[f]) + "," + std::to_string(M[f]) + ";";
    return k;
}

template <class T>
bool upload(BatchCtx * B, const std::vector<T> & v, T ** d) {
    if (!cuda_ok(cudaMalloc(d, sizeof(T) * std::max<size_t>(1, v.size())), "cudaMalloc(batch table)")) return false;
    B->allocs.push_back(*d);
    return v.empty() || cuda_ok(cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "cudaMemcpy(batch table)");
}

// tiles of every class, ordered longest K first for each multiply mode
bool build_trmm_set(BatchCtx * B, const std::vector<TrmmBatchClass> & cls, TrmmSet * T) {
    const int bm = trmm_tile_rows(), bn = trmm_tile_cols();
    std::vector<std::pair<long long, TrmmTile>> t[4];
    for (int c = 0; c < (int) cls.size(); c++) {
        const TrmmBatchClass & k = cls[c];
        for (int tm = 0; tm * bm < k.mrows; tm++)
            for (int tn = 0; tn * bn < k.ncols; tn++) {
                const TrmmTile x{c, tm, tn};
                t[0].push_back({(long long) (k.n - tm * bm), x});
                t[1].push_back({(long long) std::min(k.n, (tm + 1) * bm), x});
                t[2].push_back({(long long) std::min(k.n, (tn + 1) * bn), x});
                t[3].push_back({(long long) (k.n - tn * bn), x});
            }
    }
    if (!upload(B, cls, &T->d_classes)) return false;
    for (int m = 0; m < 4; m++) {
        std::stable_sort(t[m].begin(), t[m].end(), [](const auto & a, const auto & b) { return a.first > b.first; });
        std::vector<TrmmTile> o;
        for (auto & x : t[m]) o.push_back(x.second);
        if (!upload(B, o, &T->d_tiles[m])) return false;
        T->ntiles = (int) o.size();
    }
    return true;
}

// Frees every batch context that names plan H (called when H is destroyed).
void release_batches(HarmonicPlan * H) {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    const std::string tag = std::to_string((uintptr_t) H) + ",";
    for (auto it = g_batches.begin(); it != g_batches.end();) {
        const std::string & k = it->first;
        bool hit = false;
        for (size_t pos = k.find(tag); pos != std::string::npos; pos = k.find(tag, pos + 1))
            if (pos > 0 && (k[pos - 1] == ':' || k[pos - 1] == ';')) { hit = true; break; }
        if (!hit) { ++it; continue; }
        BatchCtx * B = it->second;
        for (void * p : B->allocs) cudaFree(p);
        mixed_trmm_work_free(B->mx_trmm);
        rot_schedule_free(B->sched);
        delete B;
        it = g_batches.erase(it);
    }
}

// lane: a second context of the same fields (its own scratch and queue), for work that may run
// concurrently with lane 0's on another stream
BatchCtx * get_batch(HarmonicPlan * const * H, const int * N, const int * M, int nf, int lane = 0) {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    const std::string key = batch_key(H, N, M, nf) + (lane ? "#" + std::to_string(lane) : std::string());
    auto it = g_batches.find(key);
    if (it != g_batches.end()) return it->second;
    BatchCtx * B = new BatchCtx();
    const int kind = H[0]->kind;
    // rotation tasks of every field, longest first
    std::vector<std::pair<double, RotTask>> tv;
    for (int f = 0; f < nf; f++)
        for (const RotTask & t : build_tasks(kind, N[f], M[f], f))
            tv.push_back({task_cost(kind, N[f], M[f], t.mbase), t});
    std::stable_sort(tv.begin(), tv.end(), [](const auto & a, const auto & b) { return a.first > b.first; });
    std::vector<RotTask> tasks;
    for (auto & p : tv) tasks.push_back(p.second);
    std::vector<TrmmBatchClass> left, right;
    for (int f = 0; f < nf; f++) {
        const int n = N[f];
        if (kind == TRI) {   // one class per field: left with U0, right with U1 (src/drivers.c:921-957)
            left.push_back(TrmmBatchClass{f, 0, 0, n, n, M[f], (long long) n});
            right.push_back(TrmmBatchClass{f, 1, 0, n, n, M[f], (long long) n});
        } else {             // four stride-4N classes per field (src/drivers.c:836-839)
            const int nc[4] = {(M[f] + 3) / 4, (M[f] + 2) / 4, (M[f] + 1) / 4, M[f] / 4};
            for (int r = 0; r < 4; r++)
                if (nc[r] > 0) left.push_back(TrmmBatchClass{f, (r == 0 || r == 3) ? 0 : 1, r, n, n, nc[r], 4LL * n});
        }
    }
    size_t work = 0;
    for (int f = 0; f < nf; f++) { B->work_off.push_back(work); work += (size_t) N[f] * M[f]; work = (work + 1) & ~(size_t) 1; }
    bool ok = upload(B, tasks, &B->d_tasks) && build_trmm_set(B, left, &B->left) &&
              (kind != TRI || build_trmm_set(B, right, &B->right)) &&
              cuda_ok(cudaMalloc(&B->d_work, sizeof(double) * std::max<size_t>(1, work)), "cudaMalloc(batch workspace)") &&
              cuda_ok(cudaMalloc(&B->d_counter, sizeof(int)), "cudaMalloc(batch counter)");
    if (B->d_work) B->allocs.push_back(B->d_work);
    if (B->d_counter) B->allocs.push_back(B->d_counter);
    if (!ok) {
        for (void * p : B->allocs) cudaFree(p);
        delete B;
        return nullptr;
    }
    B->ntasks = (int) tasks.size();
    B->sched = rot_schedule_new(tasks);
    g_batches[key] = B;
    return B;
}

// one launch per stage over up to kMaxFields fields of one family
int execute_batch_chunk(HarmonicPlan * const * H, bool forward, char TRANS, double * const * A, const int * N,
                        const int * M, int nf, cudaStream_t st, int precision = FT_B200_FP64, int lane = 0) {
    BatchCtx * B = get_batch(H, N, M, nf, lane);
    if (!B) return t_status;
    const bool mixed = precision == FT_B200_MIXED_BF16 || precision == FT_B200_MIXED_BF16X4;
    // tri's split-BF16 forms keep the sweeps in FP64 (the direct kernel) and put only its two
    // connection multiplies on the tensor cores: the triangle's multiplies amplify a sweep
    // error by a large factor (the sliced sweeps leave 3e-6 .. 9e-6 at degree 2047 with
    // (0, 0, 0)), while sliced multiplies alone stay near 1e-7
    const bool blocked = precision == FT_B200_FP64_BLOCKED || (mixed && H[0]->kind != TRI);
    const int ns = precision == FT_B200_MIXED_BF16X4 ? 4 : 3;
    const int blk = blocked ? blocked_block_size() : 0;
    if (blocked && !mixed && !B->blk_ready) {
        if (!blocked_tasks(H[0]->blocked, nf, N[0], M[0], &B->blk_tasks)) return t_status;
        if (B->blk_tasks.d_tasks) B->allocs.push_back(B->blk_tasks.d_tasks);
        B->blk_ready = true;
    }
    if (mixed && blocked && !B->mx_ready) {
        if (!blocked_tasks_mixed(H[0]->blocked, nf, N[0], M[0], &B->mx_tasks)) return t_status;
        if (B->mx_tasks.d_tasks) B->allocs.push_back(B->mx_tasks.d_tasks);
        const size_t te = blocked_mixed_T_elems(H[0]->blocked, B->mx_tasks.ntasks, N[0]);
        if (!cuda_ok(cudaMalloc(&B->d_T, te * sizeof(float)), "cudaMalloc(blocked task copy)")) return t_status;
        B->allocs.push_back(B->d_T);
        B->mx_ready = true;
    }
    const int kind = H[0]->kind;
    const bool tN = TRANS == 'N';
    std::vector<double *> S(nf);
    for (int f = 0; f < nf; f++) S[f] = B->d_work + B->work_off[f];
    // cur_is_A: which buffer holds the current data (all fields move together)
    auto rot = [&](bool hi2lo, bool from_A, bool to_A) -> bool {
        static thread_local RotLaunch L;
        L.nfields = nf;
        for (int f = 0; f < nf; f++) {
            const double * in = from_A ? A[f] : S[f];
            double * out = to_A ? A[f] : S[f];
            L.fields[f] = RotField{in, out, H[f]->rp_arr[0]->d_scp, N[f], M[f], H[f]->kind, (long long) N[f], blk};
            if (in != out) {
                const int nc = untouched_cols(H[f]->kind, M[f]);
                if (!cuda_ok(cudaMemcpy2DAsync(out, N[f] * sizeof(double), in, N[f] * sizeof(double), N[f] * sizeof(double), nc,
                                               cudaMemcpyDeviceToDevice, st), "cudaMemcpy2DAsync")) return false;
            }
        }
        L.tasks = B->d_tasks;
        L.ntasks = B->ntasks;
        L.counter = B->d_counter;
        // out of place, the destinations hold nothing live yet: the autotuner may time there
        std::vector<double *> dead(nf);
        for (int f = 0; f < nf; f++) dead[f] = to_A ? A[f] : S[f];
        prof_begin(FAM_ROT, st);
        const cudaError_t e = launch_rotations(kind, hi2lo, L, 0, st, from_A != to_A ? dead.data() : nullptr, B->sched);
        prof_end(st);
        return cuda_ok(e, "rotation kernel");
    };
    auto trmm = [&](const TrmmSet & T, int mode, bool inverse, bool from_A) -> bool {
        if (mixed) {
            std::vector<double *> in(nf), out(nf);
            for (int f = 0; f < nf; f++) { in[f] = from_A ? A[f] : S[f]; out[f] = from_A ? S[f] : A[f]; }
            // four slices of the connection matrix for both block precisions: its K runs over all
            // n rows, where three slices would cost about 2e-6 at n = 4096.  Four slices of the
            // input for MIXED_BF16X4 and for tri, whose multiplies cancel more: three leave
            // about 3e-6 there (2e-7 for sph, 1e-6 for disk with generic parameters)
            const int nx = (ns == 4 || kind == TRI) ? 4 : 3;
            cudaError_t e;
            prof_begin(FAM_TRMM, st);
            if (kind != TRI) {          // the four column classes of sph and disk: mode 0 (U In) or 1 (U^T In)
                e = launch_trmm_mixed(H[0], &H[0]->mixed_trmm, &B->mx_trmm, 4, nx, inverse, mode == 1, in.data(),
                                      out.data(), nf, M[0], st);
            } else if (mode < 2) {      // tri, left: U[0] In or U[0]^T In over all columns
                e = launch_trmm_mixed(H[0], &H[0]->mixed_trmm, &B->mx_trmm, 4, nx, inverse, mode == 1, in.data(),
                                      out.data(), nf, M[0], st, 1, 0);
            } else {                    // tri, right: In op(U[1]) = (op(U[1])^T In^T)^T through two transposes
                e = launch_transpose_square(in.data(), out.data(), nf, N[0], st);
                if (e == cudaSuccess)
                    e = launch_trmm_mixed(H[0], &H[0]->mixed_trmm, &B->mx_trmm, 4, nx, inverse, mode == 2, out.data(),
                                          in.data(), nf, M[0], st, 1, 1);
                if (e == cudaSuccess) e = launch_transpose_square(in.data(), out.data(), nf, N[0], st);
            }
            prof_end(st);
            return cuda_ok(e, "tensor-core trmm");
        }
        static thread_local TrmmBatch P;
        bool vec = true;
        for (int f = 0; f < nf; f++) {
            double * const * U = inverse ? H[f]->dPinv : H[f]->dP;
            P.U[f][0] = U[0];
            P.U[f][1] = U[1];
            P.in[f] = from_A ? A[f] : S[f];
            P.out[f] = from_A ? S[f] : A[f];
            vec = vec && (N[f] % 2 == 0) && ((reinterpret_cast<uintptr_t>(A[f]) & 15) == 0) && ((reinterpret_cast<uintptr_t>(S[f]) & 15) == 0);
        }
        P.classes = T.d_classes;
        P.tiles = T.d_tiles[mode];
        prof_begin(FAM_TRMM, st);
        const cudaError_t e = launch_trmm_batched(P, T.ntiles, vec, mode, st);
        prof_end(st);
        return cuda_ok(e, "trmm kernel");
    };
    auto norm = [&](bool on_A, bool transposed) -> bool {
        for (int f = 0; f < nf; f++) {
            prof_begin(FAM_OTHER, st);
            const cudaError_t e = launch_cheb_normalize(on_A ? A[f] : S[f], N[f], M[f], N[f], transposed, st);
            prof_end(st);
            if (!cuda_ok(e, "normalize")) return false;
        }
        return true;
    };
    // blocked products of the whole blocks, in place on the scratch matrices (on_A: on A)
    auto blocks = [&](bool hi2lo, bool on_A = false) -> bool {
        if (!blocked) return true;
        double * const * X = on_A ? A : S.data();
        if (!mixed) {
            prof_begin(FAM_BLOCK, st);
            const cudaError_t e = launch_blocked(H[0]->blocked, hi2lo, X, nf, N[0], M[0], B->blk_tasks, B->d_counter, st);
            prof_end(st);
            return cuda_ok(e, "blocked kernel");
        }
        prof_begin(FAM_OTHER, st);
        cudaError_t e = launch_blocked_transpose(H[0]->blocked, true, X, nf, N[0], M[0], B->d_T, B->mx_tasks, st);
        prof_end(st);
        prof_begin(FAM_BLOCK, st);
        if (e == cudaSuccess) e = launch_blocked_mixed(H[0]->blocked, ns, hi2lo, B->d_T, N[0], M[0], B->mx_tasks, B->d_counter, st);
        prof_end(st);
        prof_begin(FAM_OTHER, st);
        if (e == cudaSuccess) e = launch_blocked_transpose(H[0]->blocked, false, X, nf, N[0], M[0], B->d_T, B->mx_tasks, st);
        prof_end(st);
        return cuda_ok(e, "blocked kernels");
    };
    if (kind != TRI) {   // src/drivers.c:833-865, 989-1021
        bool good;
        if (forward && tN)  good = rot(true, true, false) && blocks(true) && trmm(B->left, 0, false, false);
        else if (forward)   good = trmm(B->left, 1, false, true) && blocks(false) && rot(false, false, true);
        else if (tN)        good = trmm(B->left, 0, true, true) && blocks(false) && rot(false, false, true);
        else                good = rot(true, true, false) && blocks(true) && trmm(B->left, 1, true, false);
        return good ? FT_B200_OK : t_status;
    }
    // tri (src/drivers.c:921-957); all plans share the left / right flags
    const double a = H[0]->pub.alpha, b = H[0]->pub.beta, g = H[0]->pub.gamma;
    const bool left = (b + g != -1.5) || (a != -0.5);
    const bool right = (g != -0.5) || (b != -0.5);
    const int k = (left ? 1 : 0) + (right ? 1 : 0);
    bool cur_A = true;
    if ((forward && tN) || (!forward && !tN)) {
        const bool rot_to_A = (k % 2) == 0;
        if (!rot(true, true, rot_to_A) || !blocks(true, rot_to_A)) return t_status;
        cur_A = rot_to_A;
        const int lm = forward ? 0 : 1, rm = forward ? 3 : 2;
        if (left) { if (!trmm(B->left, lm, !forward, cur_A)) return t_status; cur_A = !cur_A; }
        if (right) { if (!trmm(B->right, rm, !forward, cur_A)) return t_status; cur_A = !cur_A; }
        if (!norm(cur_A, !forward)) return t_status;
    } else {
        if (!norm(true, !forward)) return t_status;
        const int rm = forward ? 2 : 3, lm = forward ? 1 : 0;
        if (right) { if (!trmm(B->right, rm, !forward, cur_A)) return t_status; cur_A = !cur_A; }
        if (left) { if (!trmm(B->left, lm, !forward, cur_A)) return t_status; cur_A = !cur_A; }
        if (!blocks(false, cur_A) || !rot(false, cur_A, true)) return t_status;
    }
    return FT_B200_OK;
}

bool same_tri_flags(HarmonicPlan * const * H, int nf) {
    auto flags = [](HarmonicPlan * h) {
        const double a = h->pub.alpha, b = h->pub.beta, g = h->pub.gamma;
        return ((b + g != -1.5) || (a != -0.5) ? 1 : 0) + ((g != -0.5) || (b != -0.5) ? 2 : 0);
    };
    for (int f = 1; f < nf; f++)
        if (flags(H[f]) != flags(H[0])) return false;
    return true;
}

}  // namespace

// The four stride-4 column classes of sph and disk, exported for the spin-weighted
// transforms (spin.cu), which apply them to the real and the imaginary parts.
bool connection_multiply(HarmonicPlan * H, bool inverse, bool trans, const double * in, double * out, int M,
                         cudaStream_t st, bool swap) {
    return trmm4(H, inverse, trans, in, out, M, st, swap);
}

// Rotation plans and sweeps for the plans of other files (the Dunkl-Xu plans, rectdisk.cu).
ft_rotation_plan * rotation_plan_new(int kind, int n, double alpha, double beta, double gamma) {
    return make_rotation_plan(kind, n, alpha, beta, gamma);
}
bool rotation_sweeps(ft_rotation_plan * RP, bool hi2lo, const double * in, double * out, int M, long long lda,
                     cudaStream_t st) {
    return rotations(RP, hi2lo, in, out, M, lda, st);
}

// ---------------------------------------------------------------------------
// host-pointer fields sharing a plan: the transfers of one group of fields
// overlap the transforms of the previous group and the read-back of the one
// before it (three device buffers in rotation, three streams, events between
// them).  Groups: the first and the last hold half as many fields as the
// others, so that the transfers not hidden behind compute (the first group's
// copy in, the last group's copy out) are short.
// ---------------------------------------------------------------------------
struct HostPipe {
    static constexpr int NBUF = 3;
    static constexpr int LANES = 2;   // compute streams: consecutive groups alternate between them
    cudaStream_t s_in = nullptr, s_comp[LANES] = {}, s_out = nullptr;
    cudaEvent_t ev_in[NBUF] = {}, ev_comp[NBUF] = {}, ev_out[NBUF] = {};
    double * buf[NBUF] = {};   // cap matrices of elems doubles each
    int cap = 0;
    size_t elems = 0;
    std::mutex mu;             // one call at a time per plan
};
std::mutex g_pipe_mu;
std::map<HarmonicPlan *, HostPipe *> g_pipes;

void host_pipe_free(HostPipe * Q) {
    if (!Q) return;
    for (cudaStream_t s : {Q->s_in, Q->s_comp[0], Q->s_comp[1], Q->s_out})
        if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    for (int b = 0; b < HostPipe::NBUF; b++) {
        if (Q->ev_in[b]) cudaEventDestroy(Q->ev_in[b]);
        if (Q->ev_comp[b]) cudaEventDestroy(Q->ev_comp[b]);
        if (Q->ev_out[b]) cudaEventDestroy(Q->ev_out[b]);
        if (Q->buf[b]) cudaFree(Q->buf[b]);
    }
    delete Q;
}

void release_host_pipe(HarmonicPlan * H) {
    std::lock_guard<std::mutex> lk(g_pipe_mu);
    auto it = g_pipes.find(H);
    if (it == g_pipes.end()) return;
    host_pipe_free(it->second);
    g_pipes.erase(it);
}

// The plan's pipeline with buffers for at least cap fields of elems doubles (grown on demand).
HostPipe * host_pipe(HarmonicPlan * H, int cap, size_t elems) {
    std::lock_guard<std::mutex> lk(g_pipe_mu);
    HostPipe *& Q = g_pipes[H];
    if (Q && (Q->cap < cap || Q->elems < elems)) { host_pipe_free(Q); Q = nullptr; }
    if (Q) return Q;
    Q = new HostPipe();
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&Q->s_in, cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_ok(cudaStreamCreateWithFlags(&Q->s_comp[0], cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_ok(cudaStreamCreateWithFlags(&Q->s_comp[1], cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_ok(cudaStreamCreateWithFlags(&Q->s_out, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int b = 0; ok && b < HostPipe::NBUF; b++)
        ok = cuda_ok(cudaEventCreateWithFlags(&Q->ev_in[b], cudaEventDisableTiming), "cudaEventCreate") &&
             cuda_ok(cudaEventCreateWithFlags(&Q->ev_comp[b], cudaEventDisableTiming), "cudaEventCreate") &&
             cuda_ok(cudaEventCreateWithFlags(&Q->ev_out[b], cudaEventDisableTiming), "cudaEventCreate") &&
             cuda_ok(cudaMalloc(&Q->buf[b], sizeof(double) * elems * (size_t) cap), "cudaMalloc(host pipeline buffer)");
    Q->cap = cap;
    Q->elems = elems;
    if (!ok) { host_pipe_free(Q); Q = nullptr; g_pipes.erase(H); }
    return Q;
}

// Group sizes for nfields fields with groups of up to g: halves at both ends.
std::vector<int> host_groups(int nfields, int g) {
    std::vector<int> sizes;
    const int half = std::max(1, g / 2);
    const int first = std::min(nfields, half);
    sizes.push_back(first);
    int rem = nfields - first;
    const int last = std::min(rem, half);
    rem -= last;
    while (rem > 0) { const int s = std::min(rem, g); sizes.push_back(s); rem -= s; }
    if (last > 0) sizes.push_back(last);
    return sizes;
}

int host_group_size() {
    static const int g = [] {
        const char * e = std::getenv("FT_B200_HOST_GROUP");
        const int v = e ? std::atoi(e) : 0;
        return (v >= 1 && v <= kMaxFields) ? v : 4;
    }();
    return g;
}

int shared_prepare(HarmonicPlan * H, int precision) {
    if (precision != FT_B200_FP64 && precision != FT_B200_FP64_BLOCKED && precision != FT_B200_MIXED_BF16 &&
        precision != FT_B200_MIXED_BF16X4) {
        set_error(FT_B200_EINVAL, "unknown precision");
        return FT_B200_EINVAL;
    }
    const bool mixed = precision == FT_B200_MIXED_BF16 || precision == FT_B200_MIXED_BF16X4;
    if (precision == FT_B200_FP64 || (mixed && H->kind == TRI)) return FT_B200_OK;   // no tile products
    if (!H->blocked) {
        H->blocked = blocked_plan_build(H);
        if (!H->blocked) return t_status;
    }
    if (mixed && !blocked_mixed_prepare(H->blocked, precision == FT_B200_MIXED_BF16X4 ? 4 : 3)) return t_status;
    return FT_B200_OK;
}

int shared_run(HarmonicPlan * H, bool forward, char TRANS, double * const * dA, int nfields, int precision, cudaStream_t st,
               int lane = 0) {
    const int M = H->Mdef;
    for (int f0 = 0; f0 < nfields; f0 += kMaxFields) {
        const int nf = std::min(kMaxFields, nfields - f0);
        std::vector<HarmonicPlan *> Hs(nf, H);
        std::vector<int> Ns(nf, H->n), Ms(nf, M);
        if (execute_batch_chunk(Hs.data(), forward, TRANS, dA + f0, Ns.data(), Ms.data(), nf, st, precision, lane) != FT_B200_OK)
            return t_status;
    }
    return FT_B200_OK;
}

int shared_host(HarmonicPlan * H, int nops, const int * forward, const char * TRANS, double * const * A, int nfields,
                int precision) {
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return t_status;
    if (dev != H->device) { set_error(FT_B200_EINVAL, "the plan lives on another device (make it current)"); return t_status; }
    if (shared_prepare(H, precision) != FT_B200_OK) return t_status;
    const std::vector<int> groups = host_groups(nfields, host_group_size());
    const int cap = *std::max_element(groups.begin(), groups.end());
    const size_t elems = (size_t) H->n * H->Mdef, bytes = elems * sizeof(double);
    HostPipe * Q = host_pipe(H, cap, elems);
    if (!Q) return t_status;
    std::lock_guard<std::mutex> lk(Q->mu);
    bool ok = true;
    int f0 = 0;
    for (size_t g = 0; ok && g < groups.size(); g++) {
        // group g computes on lane g mod 2 (its own stream and scratch), so that a group's kernels
        // start on the SMs the previous group's last kernels leave idle
        const int b = (int) (g % HostPipe::NBUF), nf = groups[g], lane = (int) (g % HostPipe::LANES);
        cudaStream_t const sc = Q->s_comp[lane];
        std::vector<double *> d(nf);
        for (int i = 0; i < nf; i++) d[i] = Q->buf[b] + elems * (size_t) i;
        // the buffer is free once the read-back of the group that used it before has finished
        if (g >= (size_t) HostPipe::NBUF) ok = cuda_ok(cudaStreamWaitEvent(Q->s_in, Q->ev_out[b], 0), "cudaStreamWaitEvent");
        for (int i = 0; ok && i < nf; i++)
            ok = cuda_ok(cudaMemcpyAsync(d[i], A[f0 + i], bytes, cudaMemcpyHostToDevice, Q->s_in), "cudaMemcpyAsync(H2D)");
        ok = ok && cuda_ok(cudaEventRecord(Q->ev_in[b], Q->s_in), "cudaEventRecord") &&
             cuda_ok(cudaStreamWaitEvent(sc, Q->ev_in[b], 0), "cudaStreamWaitEvent");
        for (int o = 0; ok && o < nops; o++)
            ok = shared_run(H, forward[o] != 0, TRANS[o], d.data(), nf, precision, sc, lane) == FT_B200_OK;
        ok = ok && cuda_ok(cudaEventRecord(Q->ev_comp[b], sc), "cudaEventRecord") &&
             cuda_ok(cudaStreamWaitEvent(Q->s_out, Q->ev_comp[b], 0), "cudaStreamWaitEvent");
        for (int i = 0; ok && i < nf; i++)
            ok = cuda_ok(cudaMemcpyAsync(A[f0 + i], d[i], bytes, cudaMemcpyDeviceToHost, Q->s_out), "cudaMemcpyAsync(D2H)");
        ok = ok && cuda_ok(cudaEventRecord(Q->ev_out[b], Q->s_out), "cudaEventRecord");
        f0 += nf;
    }
    // the call returns with every result in host memory (or after everything enqueued has ended)
    const bool done = cuda_ok(cudaStreamSynchronize(Q->s_in), "cudaStreamSynchronize") &
                      cuda_ok(cudaStreamSynchronize(Q->s_comp[0]), "cudaStreamSynchronize") &
                      cuda_ok(cudaStreamSynchronize(Q->s_comp[1]), "cudaStreamSynchronize") &
                      cuda_ok(cudaStreamSynchronize(Q->s_out), "cudaStreamSynchronize");
    return (ok && done) ? FT_B200_OK : t_status;
}

}  // namespace ftb

using namespace ftb;

extern "C" {

int ft_b200_last_status(void) { return t_status; }
const char * ft_b200_last_error(void) { return t_message.c_str(); }
unsigned long long ft_b200_kernel_launches(void) { return g_launches.load(); }

void ft_b200_set_rotation_config(int cfg) { set_rotation_config(cfg); }

int ft_b200_profile(int enable) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto & r : g_prof) { g_prof_pool.push_back(r.a); g_prof_pool.push_back(r.b); }
    g_prof.clear();
    g_prof_on = enable != 0;
    return FT_B200_OK;
}

int ft_b200_profile_read(int family, double * ms, int * launches) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_prof_mu);
    double tot = 0;
    int cnt = 0;
    for (auto & r : g_prof) {
        if (r.family != family) continue;
        if (!cuda_ok(cudaEventSynchronize(r.b), "cudaEventSynchronize")) return t_status;
        float t = 0;
        if (!cuda_ok(cudaEventElapsedTime(&t, r.a, r.b), "cudaEventElapsedTime")) return t_status;
        tot += t;
        cnt++;
    }
    if (ms) *ms = tot;
    if (launches) *launches = cnt;
    return FT_B200_OK;
}

ft_harmonic_plan * ft_plan_sph2fourier(const int n) {
    HarmonicPlan * H = make_harmonic_plan(SPH, n, 0, 0, 0);
    return H ? &H->pub : nullptr;
}
ft_harmonic_plan * ft_plan_tri2cheb(const int n, const double alpha, const double beta, const double gamma) {
    HarmonicPlan * H = make_harmonic_plan(TRI, n, alpha, beta, gamma);
    return H ? &H->pub : nullptr;
}
ft_harmonic_plan * ft_plan_disk2cxf(const int n, const double alpha, const double beta) {
    HarmonicPlan * H = make_harmonic_plan(DISK, n, alpha, beta, 0);
    return H ? &H->pub : nullptr;
}

void ft_destroy_harmonic_plan(ft_harmonic_plan * P) {
    HarmonicPlan * H = as_plan(P);
    if (!H) {
        // a Dunkl-Xu plan (rectdisk.cu), a tetrahedral plan (tet.cu), or nothing of this library
        if (!rect_plan_destroy(P) && !tet_plan_destroy(P)) ann_plan_destroy(P);
        return;
    }
    if (H->stream) { cudaStreamSynchronize(H->stream); cudaStreamDestroy(H->stream); }
    if (H->rp_arr[0]) ft_destroy_rotation_plan(H->rp_arr[0]);
    for (int i = 0; i < 2; i++) {
        std::free(H->hostP[i]); std::free(H->hostPinv[i]);
        if (H->dP[i]) cudaFree(H->dP[i]);
        if (H->dPinv[i]) cudaFree(H->dPinv[i]);
    }
    if (H->d_stage) cudaFree(H->d_stage);
    if (H->blocked) blocked_plan_free(H->blocked);
    if (H->mixed_trmm) mixed_trmm_plan_free(H->mixed_trmm);
    release_batches(H);
    release_host_pipe(H);
    H->magic = 0;
    delete H;
}

void ft_execute_sph2fourier(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, true, TRANS, A, N, M); }
void ft_execute_fourier2sph(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, false, TRANS, A, N, M); }
void ft_execute_sphv2fourier(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, true, TRANS, A, N, M, true); }
void ft_execute_fourier2sphv(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, false, TRANS, A, N, M, true); }
void ft_execute_tri2cheb(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, true, TRANS, A, N, M); }
void ft_execute_cheb2tri(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, false, TRANS, A, N, M); }
void ft_execute_disk2cxf(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, true, TRANS, A, N, M); }
void ft_execute_cxf2disk(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M) { execute_host(P, false, TRANS, A, N, M); }

ft_rotation_plan * ft_plan_rotsphere(const int n) { return make_rotation_plan(SPH, n, 0, 0, 0); }
ft_rotation_plan * ft_plan_rottriangle(const int n, const double alpha, const double beta, const double gamma) { return make_rotation_plan(TRI, n, alpha, beta, gamma); }
ft_rotation_plan * ft_plan_rotdisk(const int n, const double alpha, const double beta) { return make_rotation_plan(DISK, n, alpha, beta, 0); }
ft_rotation_plan * ft_plan_rotrectdisk(const int n, const double beta) { return make_rotation_plan(RECT, n, 0, beta, 0); }

void ft_destroy_rotation_plan(ft_rotation_plan * RP) {
    if (!RP) return;
    if (RP->tasks) {
        for (auto & kv : *RP->tasks) if (kv.second.first) cudaFree(kv.second.first);
        delete RP->tasks;
    }
    if (RP->sched) {
        for (auto & kv : *RP->sched) rot_schedule_free(kv.second);
        delete RP->sched;
    }
    delete RP->mu;
    if (RP->d_sc) cudaFree(RP->d_sc);
    if (RP->d_scp) cudaFree(RP->d_scp);
    if (RP->d_counter) cudaFree(RP->d_counter);
    std::free(RP->s);
    std::free(RP->c);
    delete RP;
}

void ft_execute_sph_hi2lo(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, true, A, M, SPH); }
void ft_execute_sph_lo2hi(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, false, A, M, SPH); }
void ft_execute_tri_hi2lo(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, true, A, M, TRI); }
void ft_execute_tri_lo2hi(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, false, A, M, TRI); }
void ft_execute_disk_hi2lo(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, true, A, M, DISK); }
void ft_execute_disk_lo2hi(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, false, A, M, DISK); }
void ft_execute_rectdisk_hi2lo(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, true, A, M, RECT); }
void ft_execute_rectdisk_lo2hi(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_host(RP, false, A, M, RECT); }
// src/drivers.c:56: the reference's OpenMP thread count; here the threads that build plans (the
// transforms run on the GPU).  n < 1 restores the default.
void ft_set_num_threads(const int n) { g_host_threads.store(n > 0 ? std::min(n, 256) : 0, std::memory_order_relaxed); }
// src/fftw.c:62-64: FFTW's threading set-up; the grids here use cuFFT, so these only succeed.
int ft_fftw_init_threads(void) { return 1; }
void ft_fftw_plan_with_nthreads(const int) {}
void ft_execute_sphv_hi2lo(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_sphv_host(RP, true, A, M); }
void ft_execute_sphv_lo2hi(const ft_rotation_plan * RP, double * A, double *, const int M) { rotations_sphv_host(RP, false, A, M); }

int ft_b200_execute_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M, void * stream) {
    clear_error();
    HarmonicPlan * H = as_plan(P);
    if (!H) {
        int r = rect_execute_dev(P, forward != 0, TRANS, dA, N, M, static_cast<cudaStream_t>(stream));
        if (r >= 0) return r;   // a Dunkl-Xu plan (rectdisk.cu)
        r = ann_execute_dev(P, forward != 0, TRANS, dA, N, M, static_cast<cudaStream_t>(stream));
        if (r >= 0) return r;   // an annulus plan (ann.cu)
        set_error(FT_B200_EINVAL, "not a plan created by this library");
        return t_status;
    }
    return execute_dev_impl(H, forward != 0, TRANS, dA, N, M, static_cast<cudaStream_t>(stream));
}

int ft_b200_execute_sphv_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M, void * stream) {
    clear_error();
    HarmonicPlan * H = as_plan(P);
    if (!H) { set_error(FT_B200_EINVAL, "not a plan created by this library"); return t_status; }
    return execute_dev_impl(H, forward != 0, TRANS, dA, N, M, static_cast<cudaStream_t>(stream), true);
}

int ft_b200_rotations_dev(const ft_rotation_plan * RP, int hi2lo, double * dA, int M, void * stream) {
    clear_error();
    if (!RP || !dA || M < 1) { set_error(FT_B200_EINVAL, "bad argument"); return t_status; }
    if (!valid_pairs(RP->kind, M)) return t_status;
    rotations(const_cast<ft_rotation_plan *>(RP), hi2lo != 0, dA, dA, M, RP->n, static_cast<cudaStream_t>(stream));
    return t_status;
}

int ft_b200_execute_shared_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * const * dA, int nfields,
                               int precision, void * stream) {
    clear_error();
    HarmonicPlan * H = as_plan(P);
    if (!H) { set_error(FT_B200_EINVAL, "not a plan created by this library"); return t_status; }
    if (!dA || nfields < 0) { set_error(FT_B200_EINVAL, "bad argument"); return t_status; }
    if (TRANS != 'N' && TRANS != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return t_status; }
    if (precision != FT_B200_FP64 && precision != FT_B200_FP64_BLOCKED && precision != FT_B200_MIXED_BF16 &&
        precision != FT_B200_MIXED_BF16X4) {
        set_error(FT_B200_EINVAL, "unknown precision");
        return t_status;
    }
    for (int f = 0; f < nfields; f++)
        if (!dA[f]) { set_error(FT_B200_EINVAL, "NULL matrix"); return t_status; }
    if (nfields == 0) return FT_B200_OK;
    if (shared_prepare(H, precision) != FT_B200_OK) return t_status;
    return shared_run(H, forward != 0, TRANS, dA, nfields, precision, static_cast<cudaStream_t>(stream));
}

int ft_b200_execute_shared_host(const ft_harmonic_plan * P, int nops, const int * forward, const char * TRANS,
                                double * const * A, int nfields, int precision) {
    clear_error();
    HarmonicPlan * H = as_plan(P);
    if (!H) { set_error(FT_B200_EINVAL, "not a plan created by this library"); return t_status; }
    if (nops < 0 || nfields < 0 || (nops > 0 && (!forward || !TRANS)) || (nfields > 0 && !A)) {
        set_error(FT_B200_EINVAL, "bad argument");
        return t_status;
    }
    for (int o = 0; o < nops; o++)
        if (TRANS[o] != 'N' && TRANS[o] != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return t_status; }
    for (int f = 0; f < nfields; f++)
        if (!A[f]) { set_error(FT_B200_EINVAL, "NULL matrix"); return t_status; }
    if (nfields == 0 || nops == 0) return FT_B200_OK;
    return shared_host(H, nops, forward, TRANS, A, nfields, precision);
}

int ft_b200_device_status(const ft_harmonic_plan * P) {
    clear_error();
    HarmonicPlan * H = as_plan(P);
    if (!H) { set_error(FT_B200_EINVAL, "not a plan created by this library"); return -1; }
    const int a = H->blocked ? blocked_device_error(H->blocked) : 0;
    const int b = H->mixed_trmm ? mixed_trmm_device_error(H->mixed_trmm) : 0;
    const int c = rotation_device_error();   // the rotation kernel's pass-pipeline waits (library-wide)
    return a ? a : (b ? b : c);
}

int ft_b200_plan_kind(const ft_harmonic_plan * P) {
    HarmonicPlan * H = as_plan(P);
    return H ? H->kind : -1;
}
int ft_b200_plan_device(const ft_harmonic_plan * P) {
    HarmonicPlan * H = as_plan(P);
    return H ? H->device : -1;
}

int ft_b200_execute_batched_dev(const ft_harmonic_plan * const * plans, int forward, char TRANS,
                                double * const * dA, const int * N, const int * M, int nfields, void * stream) {
    clear_error();
    if (!plans || !dA || !N || !M || nfields < 0) { set_error(FT_B200_EINVAL, "bad argument"); return t_status; }
    if (TRANS != 'N' && TRANS != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return t_status; }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<HarmonicPlan *> H(nfields);
    for (int f = 0; f < nfields; f++) {
        H[f] = as_plan(plans[f]);
        if (!H[f]) { set_error(FT_B200_EINVAL, "field " + std::to_string(f) + ": not a plan created by this library"); return t_status; }
        if (!dA[f]) { set_error(FT_B200_EINVAL, "field " + std::to_string(f) + ": NULL matrix"); return t_status; }
        if (!valid_MN(H[f]->kind, H[f]->n, N[f], M[f])) return t_status;
        if (H[f]->kind != H[0]->kind) { set_error(FT_B200_EINVAL, "all fields of a batch must be of one family"); return t_status; }
    }
    if (nfields == 0) return FT_B200_OK;
    if (H[0]->kind == TRI && !same_tri_flags(H.data(), nfields)) {
        // tri plans whose parameters call for different multiplies run one after another
        for (int f = 0; f < nfields; f++)
            if (execute_dev_impl(H[f], forward != 0, TRANS, dA[f], N[f], M[f], st) != FT_B200_OK) return t_status;
        return FT_B200_OK;
    }
    for (int f0 = 0; f0 < nfields; f0 += kMaxFields) {
        const int nf = std::min(kMaxFields, nfields - f0);
        if (execute_batch_chunk(H.data() + f0, forward != 0, TRANS, dA + f0, N + f0, M + f0, nf, st) != FT_B200_OK)
            return t_status;
    }
    return FT_B200_OK;
}

}  // extern "C"
