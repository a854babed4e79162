// One column's sweeps between two orders (the reference's ft_kernel_{sph,tri,disk,rectdisk}_
// {hi2lo,lo2hi}, src/rotations.c:135-141, 162-168, 262-268, 289-295, whose bodies are
// src/rotations/rotations_default.c:31-85): host column A with stride S, sweeps j of the plan's
// table between orders m1 and m2,
//   hi2lo: j = m2 - st, m2 - 2 st, .. >= m1, each sweep k = K(j) down to 0, G(k, k + p);
//   lo2hi: j = m1, m1 + st, .. < m2, each sweep k = 0 up to K(j), G(k, k + p) transposed;
// with p = 2, st = 2, K(j) = n - 3 - j (sph, rectdisk), p = 1, st = 1, K(j) = n - 2 - j (tri),
// p = 1, st = 2, K(j) = n - 2 - floor((j + 1) / 2) (disk).
//
// One CTA runs the sweeps as a wavefront over the column, held in shared memory when it fits
// (up to 25600 entries; longer columns stay in global memory): thread u of a
// chunk of consecutive sweeps applies its sweep's rotation number s - D u at step s (position
// K(j) - (s - D u) for hi2lo, s - D u for lo2hi), with a barrier between steps.  The lag D (1 for
// hi2lo, p + 1 for lo2hi) makes every entry see its rotations in the sequential order: sweep
// t + 1 reaches an entry only after sweep t has left it for good, and the positions active in one
// step are at least p + 1 apart, so no two rotations of a step share an entry.  The rotations use
// the rotation kernel's form (two products, two FMAs), so each entry's result is bit-identical to
// that of the sequential loops in the same form (the oracle's fused mode).  Chunks of blockDim.x
// sweeps run one after another.
#include <algorithm>
#include <string>
#include <vector>

#include "ft_internal.h"

namespace ftb {
namespace {

struct ColumnGeo {
    int p, st;                       // pair distance, order step
    __device__ __host__ int top(int kind, int n, int j) const {
        if (kind == TRI) return n - 2 - j;
        if (kind == DISK) return n - 2 - (j + 1) / 2;
        return n - 3 - j;
    }
};

__device__ __host__ inline ColumnGeo column_geo(int kind) {
    ColumnGeo g;
    g.p = (kind == TRI || kind == DISK) ? 1 : 2;
    g.st = kind == TRI ? 1 : 2;
    return g;
}

// first sweep's order and the number of sweeps
__device__ __host__ inline int column_sweeps(int kind, bool hi2lo, int m1, int m2, int * j0) {
    const ColumnGeo g = column_geo(kind);
    if (hi2lo) {
        *j0 = m2 - g.st;
        return *j0 >= m1 ? (*j0 - m1) / g.st + 1 : 0;
    }
    *j0 = m1;
    return m2 > m1 ? (m2 - 1 - m1) / g.st + 1 : 0;
}

// a: the column's first `len` entries (every entry the sweeps touch), sc: the plan's table;
// staged: work on a copy in shared memory (else on a itself: the barriers order global memory
// within the block as well)
template <bool HI2LO>
__global__ void __launch_bounds__(1024) column_kernel(double * a, const double2 * __restrict__ sc, int kind, int n, int m1, int m2,
                                                      int len, bool staged) {
    extern __shared__ double smem_col[];
    double * col = staged ? smem_col : a;
    if (staged)
        for (int i = threadIdx.x; i < len; i += blockDim.x) smem_col[i] = a[i];
    __syncthreads();
    const ColumnGeo g = column_geo(kind);
    const int D = HI2LO ? 1 : g.p + 1;
    const int sgn = HI2LO ? -1 : 1;   // direction of the sweep order
    int j0 = 0;
    const int T = column_sweeps(kind, HI2LO, m1, m2, &j0);
    const int B = blockDim.x, u = threadIdx.x;
    for (int t0 = 0; t0 < T; t0 += B) {
        const int nb = min(B, T - t0);
        const int kmax = max(g.top(kind, n, j0 + sgn * g.st * t0), g.top(kind, n, j0 + sgn * g.st * (t0 + nb - 1)));
        const int steps = D * (nb - 1) + kmax + 1;   // the same for every thread of the block
        const int j = j0 + sgn * g.st * (t0 + u);
        const int K = u < nb ? g.top(kind, n, j) : -1;
        const long long base = K >= 0 ? Geo::table_base(kind, n, j) : 0;
        for (int s = 0; s < steps; s++) {
            const int r = s - D * u;
            if (r >= 0 && r <= K) {
                const int k = HI2LO ? K - r : r;
                const double2 t = sc[base + k];
                const double x = col[k], y = col[k + g.p];
                const double sy = __dmul_rn(t.x, y), sx = __dmul_rn(t.x, x);
                if (HI2LO) {
                    col[k] = __fma_rn(t.y, x, sy);
                    col[k + g.p] = __fma_rn(t.y, y, -sx);
                } else {
                    col[k] = __fma_rn(t.y, x, -sy);
                    col[k + g.p] = __fma_rn(t.y, y, sx);
                }
            }
            __syncthreads();
        }
    }
    if (staged)
        for (int i = threadIdx.x; i < len; i += blockDim.x) a[i] = smem_col[i];
}

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// the column's entries 0 .. len - 1 cover every entry the sweeps touch (0 when they touch none)
int touched_len(int kind, int n, bool hi2lo, int m1, int m2) {
    const ColumnGeo g = column_geo(kind);
    int j0 = 0;
    const int T = column_sweeps(kind, hi2lo, m1, m2, &j0);
    int len = 0;
    for (int t = 0; t < T; t += std::max(T - 1, 1)) {   // K(j) is monotone in j: its largest value is at an end
        const int j = hi2lo ? j0 - g.st * t : j0 + g.st * t;
        const int K = g.top(kind, n, j);
        if (K >= 0) len = std::max(len, K + g.p + 1);
    }
    return len;
}

constexpr size_t kColumnSmemMax = 200 * 1024;

void column_host(const ft_rotation_plan * RP, int kind, bool hi2lo, int m1, int m2, double * A, int S) {
    clear_error();
    if (!RP || !A) { set_error(FT_B200_EINVAL, "NULL argument"); return; }
    if (RP->kind != kind) { set_error(FT_B200_EINVAL, "rotation plan of another family"); return; }
    if (m1 < 0 || S < 1) { set_error(FT_B200_EINVAL, "m1 must be >= 0 and S >= 1"); return; }
    const int n = RP->n;
    const int len = touched_len(kind, n, hi2lo, m1, m2);
    if (len == 0) return;   // no sweep has a rotation
    std::vector<double> h(len);
    for (int k = 0; k < len; k++) h[k] = A[(long long) k * S];
    int j0 = 0;
    const int T = column_sweeps(kind, hi2lo, m1, m2, &j0);
    const int threads = std::min(1024, (T + 31) / 32 * 32);
    const size_t bytes = sizeof(double) * len;
    const bool staged = bytes <= kColumnSmemMax;
    const size_t smem = staged ? bytes : 0;
    int prev = 0;
    if (!ok(cudaGetDevice(&prev), "cudaGetDevice") || !ok(cudaSetDevice(RP->device), "cudaSetDevice")) return;
    double * d = nullptr;
    bool good = ok(cudaMalloc(&d, bytes), "cudaMalloc") && ok(cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(H2D)");
    if (good) {
        if (hi2lo) {
            good = ok(cudaFuncSetAttribute(column_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem), "cudaFuncSetAttribute");
            if (good) column_kernel<true><<<1, threads, smem>>>(d, RP->d_sc, kind, n, m1, m2, len, staged);
        } else {
            good = ok(cudaFuncSetAttribute(column_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem), "cudaFuncSetAttribute");
            if (good) column_kernel<false><<<1, threads, smem>>>(d, RP->d_sc, kind, n, m1, m2, len, staged);
        }
        if (good) {
            count_launch();
            good = ok(cudaGetLastError(), "column_kernel") &&
                   ok(cudaMemcpy(h.data(), d, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy(D2H)");
        }
    }
    cudaFree(d);
    cudaSetDevice(prev);
    if (good)
        for (int k = 0; k < len; k++) A[(long long) k * S] = h[k];
}

}  // namespace
}  // namespace ftb

using namespace ftb;

extern "C" {

void ft_kernel_sph_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, SPH, true, m1, m2, A, S);
}
void ft_kernel_sph_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, SPH, false, m1, m2, A, S);
}
void ft_kernel_tri_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, TRI, true, m1, m2, A, S);
}
void ft_kernel_tri_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, TRI, false, m1, m2, A, S);
}
void ft_kernel_disk_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, DISK, true, m1, m2, A, S);
}
void ft_kernel_disk_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, DISK, false, m1, m2, A, S);
}
void ft_kernel_rectdisk_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, RECT, true, m1, m2, A, S);
}
void ft_kernel_rectdisk_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S) {
    column_host(RP, RECT, false, m1, m2, A, S);
}

}  // extern "C"
