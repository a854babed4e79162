// An execute entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: frameworks that own all
// device memory through their own pool and hand a library only the arrays it
// works on, and long-running services that reserve their memory at start-up
// and must not allocate afterwards, because cudaMalloc / cudaFree can block or
// synchronise the device and can fail under memory pressure in the middle of a
// job.  ft_b200_execute_noalloc_dev serves them: it runs the same transform as
// ft_b200_execute_dev, but its intermediate matrix and the rotation kernel's
// work counter live in a fixed array compiled into this library instead of in
// memory allocated per plan or per call.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (kNoallocBytes + kNoallocHeader) until the process exits.
// Host code cannot use the array's name as a device address: the address is
// obtained once per device with cudaGetSymbolAddress, on the first call made
// with that device current, and passed to the kernels; it is kept for the life
// of the process (a cudaDeviceReset, which invalidates every plan, would also
// invalidate it).
#include <mutex>

#include "ft_internal.h"

namespace ftb {
namespace {

constexpr size_t kNoallocHeader = 256;   // bytes before the matrix: the work counter
constexpr size_t kNoallocBytes = (size_t) FT_B200_NOALLOC_MAX_ELEMS * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocHeader + kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void * g_noalloc_ptr[kMaxDevices] = {};

// Device address of the array on the current device (set up on first use).
bool noalloc_scratch(int dev, unsigned char ** out) {
    if (dev < 0 || dev >= kMaxDevices) { set_error(FT_B200_ENODEV, "device id out of range"); return false; }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void * p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error(FT_B200_ECUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
            return false;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[dev]);
    return true;
}

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// Rotation stage with the caller's work counter; only a task list the plan
// already holds is used (plans build the one for their default M when created).
bool rot(HarmonicPlan * H, bool hi2lo, const double * in, double * out, int M, int * counter, cudaStream_t st) {
    ft_rotation_plan * RP = H->rp_arr[0];
    const RotTask * tasks = nullptr;
    int ntasks = 0;
    if (!find_tasks(RP, M, &tasks, &ntasks)) {
        set_error(FT_B200_EUNSUPPORTED, "no task list for this M on the plan (the allocation-free path only runs the plan's default M)");
        return false;
    }
    const long long lda = H->n;
    if (in != out) {
        const int nc = std::min(M, H->kind == TRI ? 1 : 3);   // orders 0 and 1 have no sweeps
        if (!ok(cudaMemcpy2DAsync(out, lda * sizeof(double), in, lda * sizeof(double), H->n * sizeof(double), nc,
                                  cudaMemcpyDeviceToDevice, st), "cudaMemcpy2DAsync")) return false;
    }
    if (ntasks == 0) return true;
    static thread_local RotLaunch L;
    L.nfields = 1;
    L.fields[0] = RotField{in, out, RP->d_scp, H->n, M, H->kind, lda, 0};
    L.tasks = tasks;
    L.ntasks = ntasks;
    L.counter = counter;   // reset to zero by the launcher before the kernel runs
    return ok(launch_rotations(H->kind, hi2lo, L, 0, st), "rotation kernel");
}

bool trmm4(HarmonicPlan * H, bool inverse, bool trans, const double * in, double * out, int M, cudaStream_t st) {
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
        L.cls[c] = TrmmClass{(r == 0 || r == 3) ? U[0] : U[1], in + (long long) r * N, out + (long long) r * N, ncols[r]};
        c++;
    }
    L.nclasses = c;
    return ok(launch_trmm(L, st), "trmm kernel");
}

bool trmm1(HarmonicPlan * H, const double * U, bool trans, const double * in, double * out, int M, cudaStream_t st) {
    TrmmLaunch L{};
    L.n = H->n;
    L.ld_in = L.ld_out = H->n;
    L.trans = trans;
    L.nclasses = 1;
    L.cls[0] = TrmmClass{U, in, out, M};
    return ok(launch_trmm(L, st), "trmm kernel");
}

int run(HarmonicPlan * H, bool forward, char TRANS, double * A, int N, int M, cudaStream_t st) {
    if (TRANS != 'N' && TRANS != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return FT_B200_EINVAL; }
    if (!A) { set_error(FT_B200_EINVAL, "NULL matrix"); return FT_B200_EINVAL; }
    if (N != H->n || M < 1 || (H->kind == TRI && M != N)) { set_error(FT_B200_EINVAL, "N, M do not match the plan"); return FT_B200_EINVAL; }
    if (H->kind != TRI && M >= 4 && M % 2 == 0) {   // order M/2 would reach column M
        set_error(FT_B200_EINVAL, "sph and disk matrices need an odd number of columns M");
        return FT_B200_EINVAL;
    }
    if ((size_t) N * (size_t) M > (size_t) FT_B200_NOALLOC_MAX_ELEMS) {
        set_error(FT_B200_EINVAL, "N*M = " + std::to_string((long long) N * M) + " exceeds the allocation-free limit of " +
                                  std::to_string((long long) FT_B200_NOALLOC_MAX_ELEMS) + " elements");
        return FT_B200_EINVAL;
    }
    int dev = 0;
    if (!ok(cudaGetDevice(&dev), "cudaGetDevice")) return FT_B200_ECUDA;
    if (dev != H->device) { set_error(FT_B200_EINVAL, "the plan lives on another device"); return FT_B200_EINVAL; }
    unsigned char * base = nullptr;
    if (!noalloc_scratch(dev, &base)) return ft_b200_last_status();
    int * counter = reinterpret_cast<int *>(base);
    double * S = reinterpret_cast<double *>(base + kNoallocHeader);
    const bool tN = TRANS == 'N';
    if (H->kind != TRI) {   // src/drivers.c:833-865, 989-1021
        bool good;
        if (forward && tN)  good = rot(H, true, A, S, M, counter, st) && trmm4(H, false, false, S, A, M, st);
        else if (forward)   good = trmm4(H, false, true, A, S, M, st) && rot(H, false, S, A, M, counter, st);
        else if (tN)        good = trmm4(H, true, false, A, S, M, st) && rot(H, false, S, A, M, counter, st);
        else                good = rot(H, true, A, S, M, counter, st) && trmm4(H, true, true, S, A, M, st);
        return good ? FT_B200_OK : ft_b200_last_status();
    }
    // tri: src/drivers.c:921-957
    const double a = H->pub.alpha, b = H->pub.beta, g = H->pub.gamma;
    const bool left = (b + g != -1.5) || (a != -0.5);
    const bool right = (g != -0.5) || (b != -0.5);
    const int k = (left ? 1 : 0) + (right ? 1 : 0);
    const double * U0 = forward ? H->dP[0] : H->dPinv[0];
    const double * U1 = forward ? H->dP[1] : H->dPinv[1];
    const long long lda = N;
    double * cur = A;
    double * oth = S;
    auto flip = [&]() { std::swap(cur, oth); };
    if ((forward && tN) || (!forward && !tN)) {
        double * rot_out = (k % 2) ? S : A;
        if (!rot(H, true, A, rot_out, M, counter, st)) return ft_b200_last_status();
        cur = rot_out; oth = rot_out == A ? S : A;
        if (left) { if (!trmm1(H, U0, !forward, cur, oth, M, st)) return ft_b200_last_status(); flip(); }
        if (right) {
            if (!ok(launch_trmm_right(U1, cur, oth, N, N, lda, forward, st), "trmm kernel")) return ft_b200_last_status();
            flip();
        }
        if (!ok(launch_cheb_normalize(cur, N, M, lda, !forward, st), "normalize")) return ft_b200_last_status();
    } else {
        if (!ok(launch_cheb_normalize(A, N, M, lda, !forward, st), "normalize")) return ft_b200_last_status();
        if (right) {
            if (!ok(launch_trmm_right(U1, cur, oth, N, N, lda, !forward, st), "trmm kernel")) return ft_b200_last_status();
            flip();
        }
        if (left) { if (!trmm1(H, U0, forward, cur, oth, M, st)) return ft_b200_last_status(); flip(); }
        if (!rot(H, false, cur, A, M, counter, st)) return ft_b200_last_status();
    }
    return FT_B200_OK;
}

}  // namespace
}  // namespace ftb

extern "C" int ft_b200_execute_noalloc_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M,
                                           void * stream) {
    ftb::clear_error();
    ftb::HarmonicPlan * H = ftb::as_plan(P);
    if (!H) { ftb::set_error(FT_B200_EINVAL, "not a plan created by this library"); return FT_B200_EINVAL; }
    return ftb::run(H, forward != 0, TRANS, dA, N, M, static_cast<cudaStream_t>(stream));
}
