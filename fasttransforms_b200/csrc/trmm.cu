// Triangular multiplies of the connection stage, FP64 on the tensor pipe.
//
// The reference applies its dense upper-triangular connection matrices with
// cblas_dtrmm, in place (src/drivers.c:836-863, 924-956, 992-1019).  Here the
// product is computed out of place, Out = op(U) * In (left) or Out = In * op(U)
// (right), as a tiled GEMM with mma.sync.m8n8k4.f64 (DMMA) whose K loop only
// visits the nonzero triangle.  Up to four column classes (the stride-4N
// classes of sph / disk, each with its own U) share one launch.
//
// Tile: 128 x 64 outputs per CTA, 8 warps of 32 x 32, K slabs of 16 staged in
// shared memory by a 3-deep cp.async pipeline.  Shared layouts are padded so
// every fragment load is conflict-free.
//
// Summation: the accumulators sum one chunk of 256 consecutive k at a time;
// at the end of each chunk a thread adds them into its outputs in C (which it
// alone writes) and starts the next chunk from zero.  A single accumulation
// over all n terms lets the rounding error grow with n; chunked sums, like a
// BLAS's K panels, keep it near that of 256 terms plus n / 256 additions (the
// reference's round trips, which amplify this error in the ill-conditioned
// triangle transforms, then match its BLAS build).  C must not alias the
// inputs (every caller multiplies out of place).

#include "ft_internal.h"

namespace ftb {
namespace {

constexpr int BM = 128, BN = 64, BK = 16, NSTAGE = 3, NTHREADS = 256;
constexpr int KCHUNK_SLABS = 16;   // slabs of BK summed before a partial sum is added into C

__device__ __forceinline__ void cp_async16(void * smem, const void * gmem, bool valid) {
    unsigned sa = (unsigned) __cvta_generic_to_shared(smem);
    int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async8(void * smem, const void * gmem, bool valid) {
    unsigned sa = (unsigned) __cvta_generic_to_shared(smem);
    int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N)); }

__device__ __forceinline__ void dmma(double & d0, double & d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Operand descriptions.  A(m, k) = a[m * a_sm + k * a_sk]; B(k, n) = b[k * b_sk + n * b_sn].
// A_MC: A contiguous in m (a_sm == 1), else in k.  B_KC: B contiguous in k, else in n.
// Triangle: TRI_SIDE 0 = A is the triangular operand, 1 = B is.
struct GemmClass {
    const double * a; const double * b; double * c;
    long long a_ld, b_ld, c_ld;   // leading dims (the non-unit stride of each operand / of C)
    int mrows, ncols;
};
struct GemmParams {
    GemmClass cls[4];
    int nclasses;
    int n;              // order of the triangular matrix (also the K extent)
    int tiles_m, tiles_n;
    int mode;           // 0: left N (k >= i), 1: left T (k <= i), 2: right N (k <= j), 3: right T (k >= j)
};

// A thread's 32 accumulators (rows m0 + 8a, columns n0 + 8b + {0, 1}) into C:
// C = acc (first chunk) or C + acc, then acc = 0 when more chunks follow.  All
// loads are issued before any store, so they are in flight together.
__device__ __forceinline__ void flush_partial(const GemmClass & C, const int m0, const int n0, double (&acc)[4][4][2],
                                              const bool add, const bool restart) {
    if (add) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int m = m0 + a * 8;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int nn = n0 + b * 8;
                if (m < C.mrows && nn < C.ncols) acc[a][b][0] += C.c[(long long) nn * C.c_ld + m];
                if (m < C.mrows && nn + 1 < C.ncols) acc[a][b][1] += C.c[(long long) (nn + 1) * C.c_ld + m];
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int m = m0 + a * 8;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int nn = n0 + b * 8;
            if (m < C.mrows && nn < C.ncols) C.c[(long long) nn * C.c_ld + m] = acc[a][b][0];
            if (m < C.mrows && nn + 1 < C.ncols) C.c[(long long) (nn + 1) * C.c_ld + m] = acc[a][b][1];
            if (restart) acc[a][b][0] = acc[a][b][1] = 0.0;
        }
    }
}

// One 128 x 64 output tile of class C: rows [tm*BM, ...), columns [tn*BN, ...).
template <bool A_MC, bool B_KC, bool VEC16>
__device__ __forceinline__ void tri_tile(const GemmClass & C, const int n, const int mode, const int tm, const int tn) {
    constexpr int LDA = A_MC ? BM + 4 : BK + 4;   // [k][m] or [m][k]
    constexpr int LDB = B_KC ? BK + 4 : BN + 4;   // [n][k] or [k][n]
    constexpr int ASZ = A_MC ? BK * LDA : BM * LDA;
    constexpr int BSZ = B_KC ? BN * LDB : BK * LDB;
    extern __shared__ double sm[];
    double * As = sm;
    double * Bs = sm + NSTAGE * ASZ;
    const int i0 = tm * BM, j0 = tn * BN;
    if (i0 >= C.mrows || j0 >= C.ncols) return;
    int klo, khi;
    if (mode == 0)      { klo = i0; khi = n; }
    else if (mode == 1) { klo = 0; khi = min(i0 + BM, n); }
    else if (mode == 2) { klo = 0; khi = min(j0 + BN, n); }
    else                { klo = j0; khi = n; }
    klo = (klo / BK) * BK;
    const int nslab = (khi - klo + BK - 1) / BK;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

    auto load_slab = [&](int slab, int stage) {
        const int k0 = klo + slab * BK;
        double * as = As + stage * ASZ;
        double * bs = Bs + stage * BSZ;
        if (VEC16) {
            // A: BM*BK doubles = 1024 pairs
#pragma unroll
            for (int r = 0; r < (BM * BK / 2) / NTHREADS; ++r) {
                const int p = r * NTHREADS + tid;
                int m, k;
                if (A_MC) { k = p / (BM / 2); m = (p % (BM / 2)) * 2; }
                else      { m = p / (BK / 2); k = (p % (BK / 2)) * 2; }
                const int gm = i0 + m, gk = k0 + k;
                const bool ok = gm < C.mrows && gk < n;
                const double * g = A_MC ? C.a + (long long) gk * C.a_ld + gm : C.a + (long long) gm * C.a_ld + gk;
                double * s = A_MC ? as + k * LDA + m : as + m * LDA + k;
                cp_async16(s, ok ? g : C.a, ok);
            }
#pragma unroll
            for (int r = 0; r < (BK * BN / 2) / NTHREADS; ++r) {
                const int p = r * NTHREADS + tid;
                int k, nn;
                if (B_KC) { nn = p / (BK / 2); k = (p % (BK / 2)) * 2; }
                else      { k = p / (BN / 2); nn = (p % (BN / 2)) * 2; }
                const int gk = k0 + k, gn = j0 + nn;
                const bool ok = gk < n && gn < C.ncols;
                const double * g = B_KC ? C.b + (long long) gn * C.b_ld + gk : C.b + (long long) gk * C.b_ld + gn;
                double * s = B_KC ? bs + nn * LDB + k : bs + k * LDB + nn;
                cp_async16(s, ok ? g : C.b, ok);
            }
        } else {
#pragma unroll
            for (int r = 0; r < (BM * BK) / NTHREADS; ++r) {
                const int p = r * NTHREADS + tid;
                int m, k;
                if (A_MC) { k = p / BM; m = p % BM; }
                else      { m = p / BK; k = p % BK; }
                const int gm = i0 + m, gk = k0 + k;
                const bool ok = gm < C.mrows && gk < n;
                const double * g = A_MC ? C.a + (long long) gk * C.a_ld + gm : C.a + (long long) gm * C.a_ld + gk;
                double * s = A_MC ? as + k * LDA + m : as + m * LDA + k;
                cp_async8(s, ok ? g : C.a, ok);
            }
#pragma unroll
            for (int r = 0; r < (BK * BN) / NTHREADS; ++r) {
                const int p = r * NTHREADS + tid;
                int k, nn;
                if (B_KC) { nn = p / BK; k = p % BK; }
                else      { k = p / BN; nn = p % BN; }
                const int gk = k0 + k, gn = j0 + nn;
                const bool ok = gk < n && gn < C.ncols;
                const double * g = B_KC ? C.b + (long long) gn * C.b_ld + gk : C.b + (long long) gk * C.b_ld + gn;
                double * s = B_KC ? bs + nn * LDB + k : bs + k * LDB + nn;
                cp_async8(s, ok ? g : C.b, ok);
            }
        }
    };

    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    bool flushed = false;   // C holds the sum of the chunks before the current one

#pragma unroll
    for (int s = 0; s < NSTAGE - 1; ++s) {
        if (s < nslab) load_slab(s, s);
        cp_commit();
    }
    const int fr = lane >> 2, fc = lane & 3;   // fragment row (m or n) and k index
    for (int slab = 0; slab < nslab; ++slab) {
        cp_wait<NSTAGE - 2>();
        __syncthreads();
        {
            const int nxt = slab + NSTAGE - 1;
            if (nxt < nslab) load_slab(nxt, nxt % NSTAGE);
            cp_commit();
        }
        const double * as = As + (slab % NSTAGE) * ASZ;
        const double * bs = Bs + (slab % NSTAGE) * BSZ;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int m = wm + a * 8 + fr, k = kk + fc;
                af[a] = A_MC ? as[k * LDA + m] : as[m * LDA + k];
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int nn = wn + b * 8 + fr, k = kk + fc;
                bf[b] = B_KC ? bs[nn * LDB + k] : bs[k * LDB + nn];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
        if ((slab + 1) % KCHUNK_SLABS == 0 && slab + 1 < nslab) {   // end of a chunk: into C, restart from zero
            flush_partial(C, i0 + wm + fr, j0 + wn + fc * 2, acc, flushed, true);
            flushed = true;
        }
    }
    cp_wait<0>();

    // epilogue: C(m, n) at c[n * c_ld + m] (plus the earlier chunks' sum)
    flush_partial(C, i0 + wm + fr, j0 + wn + fc * 2, acc, flushed, false);
}

template <bool A_MC, bool B_KC, bool VEC16>
__global__ void __launch_bounds__(NTHREADS, 2)
gemm_tri_kernel(const __grid_constant__ GemmParams P) {
    // block -> (class, tile m, tile n); tiles with the most K work first
    int bid = blockIdx.x;
    const int per_class = P.tiles_m * P.tiles_n;
    const int cl = bid / per_class;
    bid -= cl * per_class;
    int tm, tn;
    if (P.mode == 0)      { tm = bid / P.tiles_n; tn = bid % P.tiles_n; }                 // small i: long K
    else if (P.mode == 1) { tm = P.tiles_m - 1 - bid / P.tiles_n; tn = bid % P.tiles_n; } // large i: long K
    else if (P.mode == 2) { tn = P.tiles_n - 1 - bid / P.tiles_m; tm = bid % P.tiles_m; } // large j
    else                  { tn = bid / P.tiles_m; tm = bid % P.tiles_m; }                 // small j
    tri_tile<A_MC, B_KC, VEC16>(P.cls[cl], P.n, P.mode, tm, tn);
}

// Batched multiplies over many fields: the tile list (longest K first) and the
// pointer-free class table live in device memory; pointers come by value.
// MODE 0/1: left, op(U) = U / U^T; MODE 2/3: right, op(U) = U / U^T.
template <int MODE, bool VEC16>
__global__ void __launch_bounds__(NTHREADS, 2)
gemm_tri_batched_kernel(const __grid_constant__ TrmmBatch P) {
    const TrmmTile t = P.tiles[blockIdx.x];
    const TrmmBatchClass c = P.classes[t.cls];
    GemmClass C;
    const double * X = P.in[c.field] + (long long) c.r * c.n;
    const double * U = P.U[c.field][c.u];
    C.c = P.out[c.field] + (long long) c.r * c.n;
    C.c_ld = c.ld;
    C.mrows = c.mrows;
    C.ncols = c.ncols;
    if (MODE < 2) { C.a = U; C.a_ld = c.n; C.b = X; C.b_ld = c.ld; }
    else          { C.a = X; C.a_ld = c.ld; C.b = U; C.b_ld = c.n; }
    constexpr bool A_MC = MODE != 1;
    constexpr bool B_KC = MODE != 3;
    tri_tile<A_MC, B_KC, VEC16>(C, c.n, MODE, t.tm, t.tn);
}

template <int MODE>
cudaError_t run_batched(const TrmmBatch & P, int ntiles, bool vec16, cudaStream_t st) {
    constexpr bool A_MC = MODE != 1;
    constexpr bool B_KC = MODE != 3;
    constexpr int LDA = A_MC ? BM + 4 : BK + 4;
    constexpr int LDB = B_KC ? BK + 4 : BN + 4;
    constexpr int ASZ = A_MC ? BK * LDA : BM * LDA;
    constexpr int BSZ = B_KC ? BN * LDB : BK * LDB;
    const size_t shm = sizeof(double) * NSTAGE * (ASZ + BSZ);
    cudaError_t e;
    if (vec16) {
        auto k = gemm_tri_batched_kernel<MODE, true>;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
        if (e != cudaSuccess) return e;
        k<<<ntiles, NTHREADS, shm, st>>>(P);
    } else {
        auto k = gemm_tri_batched_kernel<MODE, false>;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
        if (e != cudaSuccess) return e;
        k<<<ntiles, NTHREADS, shm, st>>>(P);
    }
    count_launch();
    return cudaGetLastError();
}

template <bool A_MC, bool B_KC>
cudaError_t run_gemm(const GemmParams & P, bool vec16, cudaStream_t st) {
    constexpr int LDA = A_MC ? BM + 4 : BK + 4;
    constexpr int LDB = B_KC ? BK + 4 : BN + 4;
    constexpr int ASZ = A_MC ? BK * LDA : BM * LDA;
    constexpr int BSZ = B_KC ? BN * LDB : BK * LDB;
    const size_t shm = sizeof(double) * NSTAGE * (ASZ + BSZ);
    const int blocks = P.nclasses * P.tiles_m * P.tiles_n;
    if (blocks == 0) return cudaSuccess;
    cudaError_t e;
    if (vec16) {
        auto k = gemm_tri_kernel<A_MC, B_KC, true>;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
        if (e != cudaSuccess) return e;
        k<<<blocks, NTHREADS, shm, st>>>(P);
    } else {
        auto k = gemm_tri_kernel<A_MC, B_KC, false>;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
        if (e != cudaSuccess) return e;
        k<<<blocks, NTHREADS, shm, st>>>(P);
    }
    count_launch();
    return cudaGetLastError();
}

inline bool aligned16(const void * p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

__global__ void cheb_norm_kernel(double * A, int N, int M, long long lda, double r, double g) {
    // src/drivers.c:6-24: first column and first row scaled by r (entry (0,0) twice), all by g
    const long long total = (long long) N * M;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
        const int i = (int) (e % N), j = (int) (e / N);
        double v = A[(long long) j * lda + i];
        if (j == 0) v *= r;
        if (i == 0) v *= r;
        A[(long long) j * lda + i] = v * g;
    }
}

}  // namespace

cudaError_t launch_trmm(const TrmmLaunch & L, cudaStream_t st) {
    GemmParams P{};
    P.nclasses = L.nclasses;
    P.n = L.n;
    int maxcols = 0;
    bool vec = (L.n % 2 == 0) && (L.ld_in % 2 == 0);
    for (int c = 0; c < L.nclasses; ++c) {
        GemmClass & g = P.cls[c];
        g.a = L.cls[c].U; g.b = L.cls[c].in; g.c = L.cls[c].out;
        g.a_ld = L.n; g.b_ld = L.ld_in; g.c_ld = L.ld_out;
        g.mrows = L.n; g.ncols = L.cls[c].ncols;
        maxcols = std::max(maxcols, g.ncols);
        vec = vec && aligned16(g.a) && aligned16(g.b);
    }
    P.tiles_m = (L.n + BM - 1) / BM;
    P.tiles_n = (maxcols + BN - 1) / BN;
    P.mode = L.trans ? 1 : 0;
    return L.trans ? run_gemm<false, true>(P, vec, st) : run_gemm<true, true>(P, vec, st);
}

cudaError_t launch_trmm_batched(const TrmmBatch & P, int ntiles, bool vec16, int mode, cudaStream_t st) {
    if (ntiles == 0) return cudaSuccess;
    switch (mode) {
        case 0: return run_batched<0>(P, ntiles, vec16, st);
        case 1: return run_batched<1>(P, ntiles, vec16, st);
        case 2: return run_batched<2>(P, ntiles, vec16, st);
        case 3: return run_batched<3>(P, ntiles, vec16, st);
    }
    return cudaErrorInvalidValue;
}

int trmm_tile_rows() { return BM; }
int trmm_tile_cols() { return BN; }

cudaError_t launch_trmm_right(const double * U, const double * in, double * out, int n, int nrows,
                              long long ld, bool trans, cudaStream_t st) {
    // Out(row, j) = sum_k In(row, k) op(U)(k, j): A = In (contiguous in rows), B = op(U)
    GemmParams P{};
    P.nclasses = 1;
    P.n = n;
    GemmClass & g = P.cls[0];
    g.a = in; g.b = U; g.c = out;
    g.a_ld = ld; g.b_ld = n; g.c_ld = ld;
    g.mrows = nrows; g.ncols = n;
    P.tiles_m = (nrows + BM - 1) / BM;
    P.tiles_n = (n + BN - 1) / BN;
    P.mode = trans ? 3 : 2;
    const bool vec = (n % 2 == 0) && (ld % 2 == 0) && aligned16(in) && aligned16(U);
    // op(U) = U: B(k, j) = U[k + j n] contiguous in k; op(U) = U^T: B(k, j) = U[j + k n] contiguous in j
    return trans ? run_gemm<true, false>(P, vec, st) : run_gemm<true, true>(P, vec, st);
}

cudaError_t launch_cheb_normalize(double * A, int N, int M, long long lda, bool transposed, cudaStream_t st) {
    const double r = transposed ? 1.41421356237309504880 : 0.70710678118654752440;   // M_SQRT2, M_SQRT1_2
    const double g = transposed ? 1.57079632679489661923 : 0.63661977236758134308;   // M_PI_2, M_2_PI
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cheb_norm_kernel<<<sms * 4, 256, 0, st>>>(A, N, M, lda, r, g);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ftb
