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

// geometry of kind's sweeps (SPIN: the first stage of a spin column, adjacent rotations of the
// spin table (s2, c2)(k, j, d) at k + j n + d |s| n, K(j) = n - 2 - d - j)
struct ColumnGeo {
    int p, st;                       // pair distance, order step
    __device__ __host__ int top(int kind, int n, int j, int d) const {
        if (kind == TRI) return n - 2 - j;
        if (kind == DISK) return n - 2 - (j + 1) / 2;
        if (kind == SPIN) return n - 2 - d - j;
        return n - 3 - j;
    }
    __device__ __host__ long long base(int kind, int n, int j, int d, int as) const {
        if (kind == SPIN) return (long long) j * n + (long long) d * as * n;
        return Geo::table_base(kind, n, j);
    }
};

__device__ __host__ inline ColumnGeo column_geo(int kind) {
    ColumnGeo g;
    g.p = (kind == TRI || kind == DISK || kind == SPIN) ? 1 : 2;
    g.st = (kind == TRI || kind == SPIN) ? 1 : 2;
    return g;
}

// first sweep's order and the number of sweeps.  Sweeps of order j >= 2n + 2 have no rotation
// in any kind, so m2 is first brought below 2n + 4 + st with its residue mod st kept (the sweeps
// dropped are empty ones, the others keep their orders).
__device__ __host__ inline int column_sweeps(int kind, bool hi2lo, int m1, int m2, int n, int * j0) {
    const ColumnGeo g = column_geo(kind);
    const long long cap = 2LL * n + 4;
    if (m2 > cap) m2 = (int) (m2 - (((long long) m2 - cap) / g.st) * g.st);
    if (hi2lo) {
        *j0 = m2 - g.st;
        return *j0 >= m1 ? (*j0 - m1) / g.st + 1 : 0;
    }
    *j0 = m1;
    return m2 > m1 ? (m2 - 1 - m1) / g.st + 1 : 0;
}

// the rotation kernel's form: forward x' = c x + s y, y' = c y - s x (the products s y, s x
// rounded, then one FMA each); transposed with the signs of s flipped
__device__ __forceinline__ void rotate(double & x, double & y, double s, double c, bool fwd) {
    const double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
    const double xn = fwd ? __fma_rn(c, x, sy) : __fma_rn(c, x, -sy);
    y = fwd ? __fma_rn(c, y, -sx) : __fma_rn(c, y, sx);
    x = xn;
}
__device__ __forceinline__ void rotate(double2 & x, double2 & y, double s, double c, bool fwd) {
    rotate(x.x, y.x, s, c, fwd);   // the real parts, then the imaginary parts, with the same pair
    rotate(x.y, y.y, s, c, fwd);
}

// a: the column's first `len` entries (every entry the sweeps touch; E = double, or double2 for a
// complex column), sc: the table; staged: work on a copy in shared memory (else on a itself: the
// barriers order global memory within the block as well); fwd: the rotation form; d, as: SPIN only
template <bool HI2LO, typename E>
__global__ void __launch_bounds__(1024) column_kernel(E * a, const double2 * __restrict__ sc, int kind, int n, int m1, int m2,
                                                      int len, bool staged, bool fwd, int d, int as) {
    extern __shared__ double2 smem_raw[];
    E * smem_col = reinterpret_cast<E *>(smem_raw);
    E * col = staged ? smem_col : a;
    if (staged)
        for (int i = threadIdx.x; i < len; i += blockDim.x) smem_col[i] = a[i];
    __syncthreads();
    const ColumnGeo g = column_geo(kind);
    const int D = HI2LO ? 1 : g.p + 1;
    const int sgn = HI2LO ? -1 : 1;   // direction of the sweep order
    int j0 = 0;
    const int T = column_sweeps(kind, HI2LO, m1, m2, n, &j0);
    const int B = blockDim.x, u = threadIdx.x;
    for (int t0 = 0; t0 < T; t0 += B) {
        const int nb = min(B, T - t0);
        const int kmax = max(g.top(kind, n, j0 + sgn * g.st * t0, d), g.top(kind, n, j0 + sgn * g.st * (t0 + nb - 1), d));
        const int steps = D * (nb - 1) + kmax + 1;   // the same for every thread of the block
        const int j = j0 + sgn * g.st * (t0 + u);
        const int K = u < nb ? g.top(kind, n, j, d) : -1;
        const long long base = K >= 0 ? g.base(kind, n, j, d, as) : 0;
        for (int s = 0; s < steps; s++) {
            const int r = s - D * u;
            if (r >= 0 && r <= K) {
                const int k = HI2LO ? K - r : r;
                const double2 t = sc[base + k];
                E x = col[k], y = col[k + g.p];
                rotate(x, y, t.x, t.y, fwd);
                col[k] = x;
                col[k + g.p] = y;
            }
            __syncthreads();
        }
    }
    if (staged)
        for (int i = threadIdx.x; i < len; i += blockDim.x) a[i] = smem_col[i];
}

// The tetrahedral slab (the reference's ft_kernel_tet_hi2lo / lo2hi, src/rotations.c:297-321):
// the n x L matrix A, sweeps j = m - 1 .. 0 of rotations of the column pairs (l, l + 1),
// l = L - 2 - j .. 0, with the triangle table; one thread per row, in the reference's order.
__global__ void tet_slab_kernel(double * A, const double2 * __restrict__ sc, int n, int L, int m, bool hi2lo) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double * a = A + k;   // entry l of this row at a[l n]
    if (hi2lo) {
        for (int j = m - 1; j >= 0; --j) {
            const long long b = Geo::table_base(TRI, n, j);
            for (int l = L - 2 - j; l >= 0; --l) {
                const double2 t = sc[b + l];
                double x = a[(long long) l * n], y = a[(long long) (l + 1) * n];
                rotate(x, y, t.x, t.y, true);
                a[(long long) l * n] = x;
                a[(long long) (l + 1) * n] = y;
            }
        }
    } else {
        for (int j = 0; j < m; ++j) {
            const long long b = Geo::table_base(TRI, n, j);
            for (int l = 0; l <= L - 2 - j; ++l) {
                const double2 t = sc[b + l];
                double x = a[(long long) l * n], y = a[(long long) (l + 1) * n];
                rotate(x, y, t.x, t.y, false);
                a[(long long) l * n] = x;
                a[(long long) (l + 1) * n] = y;
            }
        }
    }
}

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

constexpr size_t kColumnSmemMax = 200 * 1024;

}  // namespace

// the column's entries 0 .. len - 1 cover every entry the sweeps touch (0 when they touch none)
int column_touched(int kind, int n, bool hi2lo, int m1, int m2, int d) {
    const ColumnGeo g = column_geo(kind);
    int j0 = 0;
    const int T = column_sweeps(kind, hi2lo, m1, m2, n, &j0);
    int len = 0;
    for (int t = 0; t < T; t += std::max(T - 1, 1)) {   // K(j) is monotone in j: its largest value is at an end
        const int j = hi2lo ? j0 - g.st * t : j0 + g.st * t;
        const int K = g.top(kind, n, j, d);
        if (K >= 0) len = std::max(len, K + g.p + 1);
    }
    return len;
}

// one launch on the current device's legacy stream; dcol holds len entries (double, or double2
// when cplx), at least column_touched(..) of them
bool column_sweeps_dev(void * dcol, bool cplx, const double2 * tab, int kind, int n, int m1, int m2, bool hi2lo, bool fwd, int d,
                       int as, int len) {
    int j0 = 0;
    const int T = column_sweeps(kind, hi2lo, m1, m2, n, &j0);
    if (T == 0 || len == 0) return true;
    const int threads = std::min(1024, (T + 31) / 32 * 32);
    const size_t bytes = (cplx ? sizeof(double2) : sizeof(double)) * (size_t) len;
    const bool staged = bytes <= kColumnSmemMax;
    const int smem = staged ? (int) bytes : 0;
    cudaError_t e = cudaSuccess;
    if (cplx) {
        auto * a = static_cast<double2 *>(dcol);
        if (hi2lo) {
            e = cudaFuncSetAttribute(column_kernel<true, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e == cudaSuccess) column_kernel<true, double2><<<1, threads, smem>>>(a, tab, kind, n, m1, m2, len, staged, fwd, d, as);
        } else {
            e = cudaFuncSetAttribute(column_kernel<false, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e == cudaSuccess) column_kernel<false, double2><<<1, threads, smem>>>(a, tab, kind, n, m1, m2, len, staged, fwd, d, as);
        }
    } else {
        auto * a = static_cast<double *>(dcol);
        if (hi2lo) {
            e = cudaFuncSetAttribute(column_kernel<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e == cudaSuccess) column_kernel<true, double><<<1, threads, smem>>>(a, tab, kind, n, m1, m2, len, staged, fwd, d, as);
        } else {
            e = cudaFuncSetAttribute(column_kernel<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e == cudaSuccess) column_kernel<false, double><<<1, threads, smem>>>(a, tab, kind, n, m1, m2, len, staged, fwd, d, as);
        }
    }
    if (!ok(e, "cudaFuncSetAttribute")) return false;
    count_launch();
    return ok(cudaGetLastError(), "column_kernel");
}

namespace {

// the first len entries of a host column (stride S entries) through a device copy: run(d) on it
template <typename E, typename F>
void through_device(int device, E * A, int S, int len, F && run) {
    std::vector<E> h(len);
    for (int k = 0; k < len; k++) h[k] = A[(long long) k * S];
    int prev = 0;
    if (!ok(cudaGetDevice(&prev), "cudaGetDevice") || !ok(cudaSetDevice(device), "cudaSetDevice")) return;
    E * d = nullptr;
    const size_t bytes = sizeof(E) * (size_t) len;
    bool good = ok(cudaMalloc(&d, bytes), "cudaMalloc") && ok(cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(H2D)") &&
                run(d) && ok(cudaMemcpy(h.data(), d, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy(D2H)");
    cudaFree(d);
    cudaSetDevice(prev);
    if (good)
        for (int k = 0; k < len; k++) A[(long long) k * S] = h[k];
}

void column_host(const ft_rotation_plan * RP, int kind, bool hi2lo, int m1, int m2, double * A, int S) {
    clear_error();
    if (!RP || !A) { set_error(FT_B200_EINVAL, "NULL argument"); return; }
    if (RP->kind != kind) { set_error(FT_B200_EINVAL, "rotation plan of another family"); return; }
    if (m1 < 0 || S < 1) { set_error(FT_B200_EINVAL, "m1 must be >= 0 and S >= 1"); return; }
    const int n = RP->n;
    const int len = column_touched(kind, n, hi2lo, m1, m2, 0);
    if (len == 0) return;   // no sweep has a rotation
    through_device(RP->device, A, S, len, [&](double * d) {
        return column_sweeps_dev(d, false, RP->d_sc, kind, n, m1, m2, hi2lo, hi2lo, 0, 0, len);
    });
}

void tet_slab_host(const ft_rotation_plan * RP, int L, int m, double * A, bool hi2lo) {
    clear_error();
    if (!RP || !A) { set_error(FT_B200_EINVAL, "NULL argument"); return; }
    if (RP->kind != TRI) { set_error(FT_B200_EINVAL, "tetrahedral slabs take a triangle rotation plan"); return; }
    const int n = RP->n;
    if (L < 0 || L > n || m < 0 || m > n) { set_error(FT_B200_EINVAL, "L and m must lie in 0 .. n"); return; }
    if (L < 2 || m == 0) return;   // no rotation
    const int len = n * L;         // the whole slab, contiguous (S = 1)
    through_device(RP->device, A, 1, len, [&](double * d) {
        tet_slab_kernel<<<(n + 127) / 128, 128>>>(d, RP->d_sc, n, L, m, hi2lo);
        count_launch();
        return ok(cudaGetLastError(), "tet_slab_kernel");
    });
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
void ft_kernel_tet_hi2lo(const ft_rotation_plan * RP, const int L, const int m, double * A) { tet_slab_host(RP, L, m, A, true); }
void ft_kernel_tet_lo2hi(const ft_rotation_plan * RP, const int L, const int m, double * A) { tet_slab_host(RP, L, m, A, false); }

}  // extern "C"
