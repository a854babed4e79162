// The sph and disk connection multiply (src/drivers.c:833-865, 989-1021: four column classes j = 0,1,2,3 mod 4,
// class j multiplied by U[0] for j = 0, 3 and U[1] for j = 1, 2, U upper triangular)
// on the tcgen05 tensor cores, from fixed-point BF16 slices.
//
// Slicing (the Ozaki splitting).  A row i of op(U) is scaled by a power of two
// sU_i with |sU_i U| < 2^7 and cut into NU slices of integers |j_b| <= 2^7:
// sU_i U = j_0 + j_1 2^-8 + ...; a column x of the input is cut the same way
// in chunks of 256 rows, each chunk with its own scale sX (NX slices).  The
// products j_b i_a of one order level L = a + b <= NL - 1 are integers below
// 2^14 and a level sums at most 3 x 256 of them per chunk, below 2^24, so the
// level accumulators in tensor memory are exact whatever rounding the tensor
// core applies.  After each chunk the epilogue folds
//   (A_0 + 2^-8 A_1 + ...) / sX
// into an FP32 running sum per output element; at the end it scales by
// 1 / sU_i and writes FP64.  Configurations: NU = 3 slices of U (levels <= 2,
// six products) and NU = 4 (levels <= 3, nine products), both with NX = 3.
//
// Work: output tiles of 128 rows x TBN columns of one class of one field,
// longest K first, strided over persistent CTAs.  The operands come as
// pre-sliced images in the tensor cores' K-major 128-byte swizzled layout:
// U's once per plan, the input's by a slicing pass before each multiply.
// Warp 8 issues the MMAs (one thread) and owns the TMEM allocation, warp 9
// streams the K-tiles into a two-stage buffer with bulk copies, warps 0-7
// fold the chunks (two warps per TMEM lane quarter, TBN / 2 columns each).
// Configurations (NU, NX, TBN): (4, 3, 128), nine products, and (4, 4, 96), ten
// products, whose fourth input slice takes the input's slicing residual from
// 2^-24 to 2^-32 of a chunk's largest entry (the residual is what the
// cancellation in the multiply amplifies; four input slices at 128 columns
// would not fit two stages into shared memory).
#include <algorithm>
#include <cstdio>
#include <vector>

#include <cuda_bf16.h>

#include "ft_internal.h"
#include "tc05.h"

namespace ftb {
namespace {

constexpr int TB = 128;                     // output tile rows (rows of op(U))
constexpr int KT = 64;                      // K per tile of the images
constexpr int CHUNK_KT = 4;                 // K-tiles per exact chunk (256 rows)
constexpr int PIECE = TB * KT * 2;          // bytes of one slice of one K-tile of op(U) (16 KB)
constexpr int THREADS = 320;

// NU slices of op(U), NX of the input, TBN input columns per output tile
template <int NU, int NX, int TBN> struct Cfg {
    static constexpr int NL = NU;                           // levels kept: 0 .. NU - 1
    static constexpr int XPIECE = TBN * KT * 2;             // bytes of one input slice of one K-tile
    static constexpr int STAGE = NU * PIECE + NX * XPIECE;
    static constexpr size_t SMEM = 2 * (size_t) STAGE + 1024;
    static constexpr uint32_t IDESC = tc::idesc_bf16(TB, TBN);
    static_assert(TBN % 16 == 0 && TBN <= 128, "tile width");
    static_assert(NL * TBN <= 512, "accumulators exceed tensor memory");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

struct MixTile { int field, cls, it, jt, k0, k1; };   // K-tiles k0 .. k1 inclusive

// Order of the tiles (launch_trmm_mixed): blocks of row tiles x column tiles, 0 for one block
constexpr int kRowGroup = 8, kColGroup = 18;

struct MixLaunch {
    double * out[kMaxFields];
    const unsigned char * Uimg[2];      // per class matrix: [it][kt][NU slices]
    const float * Uinv[2];              // 1 / sU per row
    const unsigned char * Ximg;         // [field][cls][jt][kt][NX slices]
    const float * Xinv;                 // [field][cls][jt][chunk][128]: 1 / sX
    const MixTile * tiles;
    int ntiles;
    int n, M, nkt, njt;                 // njt: column tiles per class (max over classes)
    int ncls;                           // column classes: 4 (stride 4, sph and disk) or 1 (all columns)
    int * err;
};

// Column classes: with four, class r holds the columns r + 4 j and takes U[0] for r = 0, 3 and
// U[1] for r = 1, 2; with one, every column, and the single matrix the caller picked.
__host__ __device__ __forceinline__ int class_cols(int M, int r, int ncls) { return (M - r + ncls - 1) / ncls; }
__host__ __device__ __forceinline__ int class_matrix(int r, int ncls) { return (ncls == 4 && (r == 1 || r == 2)) ? 1 : 0; }

// ---------------------------------------------------------------------------
// slicing passes
// ---------------------------------------------------------------------------
__device__ __forceinline__ float pow2_scale(float amax) {
    int E = (int) ((__float_as_uint(amax) >> 23) & 0xFF);   // amax < 2^(E - 126)
    if (E < 8) E = 8;
    return __uint_as_float((uint32_t) (260 - E) << 23);       // 2^(7 - (E - 126))
}

// 8 consecutive K values (already scaled, |t| < 2^7, FP64) -> NS 16-byte chunks of integer
// slices.  The first slice is cut in FP64; its residual times 2^8 (|r| <= 128) then rounds to
// FP32 within 2^-17, which is 2^-32 of the scale 2^7, and the FP32 cuts that follow are exact.
// (Rounding the input itself to FP32 first would leave 2^-24 of every entry, which the fourth
// slice cannot recover and the multiplies of tri amplify.)
template <int NS>
__device__ __forceinline__ void slice8(const double * t_in, uint4 * out) {
    uint32_t w[NS][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double d0 = t_in[2 * q], d1 = t_in[2 * q + 1];
        const double j0 = rint(d0), j1 = rint(d1);
        w[0][q] = tc::pack_bf16_ints((float) j0, (float) j1);
        float t0 = (float) ((d0 - j0) * 256.0), t1 = (float) ((d1 - j1) * 256.0);   // d - j exact
#pragma unroll
        for (int a = 1; a < NS; ++a) {
            const float i0 = tc::round_small(t0), i1 = tc::round_small(t1);
            w[a][q] = tc::pack_bf16_ints(i0, i1);
            t0 = __fmul_rn(__fsub_rn(t0, i0), 256.0f);   // exact: |t - i| <= 1/2, times a power of two
            t1 = __fmul_rn(__fsub_rn(t1, i1), 256.0f);
        }
    }
#pragma unroll
    for (int a = 0; a < NS; ++a) out[a] = make_uint4(w[a][0], w[a][1], w[a][2], w[a][3]);
}

// One warp per row of op(U): scale over the whole row, then every K-tile's slices.
// The FP64 row is sliced in double precision (exact residuals).
template <int NS>
__global__ void slice_matrix_kernel(const double * __restrict__ U, int n, bool trans, int nkt,
                                    unsigned char * __restrict__ img, float * __restrict__ inv) {
    const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= TB * ((n + TB - 1) / TB)) return;
    auto at = [&](int k) -> double {
        if (row >= n || k >= n) return 0.0;
        return trans ? U[(long long) row * n + k] : U[row + (long long) k * n];
    };
    double amax = 0.0;
    for (int k = lane; k < n; k += 32) amax = fmax(amax, fabs(at(k)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    // power of two s with |s U| < 2^7
    int ex = 0;
    if (amax > 0) (void) frexp(amax, &ex);                      // amax < 2^ex
    const double s = amax > 0 ? ldexp(1.0, 7 - ex) : 1.0;
    if (lane == 0) inv[row] = (float) (1.0 / s);
    const int it = row / TB, rr = row % TB;
    for (int kt = 0; kt < nkt; ++kt) {
        if (lane >= 8) continue;                                // 8 lanes x 8 values = one K-tile row
        const int k0 = kt * KT + 8 * lane;
        uint32_t w[NS][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double t0 = at(k0 + 2 * q) * s, t1 = at(k0 + 2 * q + 1) * s;
#pragma unroll
            for (int a = 0; a < NS; ++a) {
                const double i0 = rint(t0), i1 = rint(t1);
                const __nv_bfloat162 b = __floats2bfloat162_rn((float) i0, (float) i1);
                w[a][q] = *reinterpret_cast<const uint32_t *>(&b);
                t0 = (t0 - i0) * 256.0;
                t1 = (t1 - i1) * 256.0;
            }
        }
        unsigned char * base = img + ((long long) it * nkt + kt) * NS * PIECE;
        const uint32_t off = tc::sw128_offset(rr, 8 * lane);
#pragma unroll
        for (int a = 0; a < NS; ++a) *reinterpret_cast<uint4 *>(base + a * PIECE + off) = make_uint4(w[a][0], w[a][1], w[a][2], w[a][3]);
    }
}

struct SliceXLaunch {
    const double * in[kMaxFields];
    int n, M, nkt, njt, ncls;
    unsigned char * img;
    float * inv;
};

// One CTA per (field, class, column tile of TBN, chunk), one warp per column at a
// time: the chunk's 256 rows are read coalesced into shared memory, then each
// lane slices 8 consecutive rows.
template <int NS, int TBN>
__global__ void __launch_bounds__(256) slice_input_kernel(const __grid_constant__ SliceXLaunch L) {
    constexpr int XPIECE = TBN * KT * 2;
    __shared__ double buf[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nch = (L.nkt + CHUNK_KT - 1) / CHUNK_KT;
    int b = blockIdx.x;
    const int q = b % nch; b /= nch;
    const int jt = b % L.njt; b /= L.njt;
    const int r = b % L.ncls;
    const int f = b / L.ncls;
    const int ncols = class_cols(L.M, r, L.ncls);
    const long long tile_base = ((long long) (f * L.ncls + r) * L.njt + jt);
    for (int ci = warp; ci < TBN; ci += 8) {
        const int j = jt * TBN + ci;
        const bool cok = j < ncols;
        const double * col = L.in[f] + (long long) (r + (long long) L.ncls * j) * L.n;
        double amax = 0.0;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int row = q * (KT * CHUNK_KT) + 32 * e + lane;
            const double v = (cok && row < L.n) ? __ldcg(col + row) : 0.0;
            buf[warp][32 * e + lane] = v;
            amax = fmax(amax, fabs(v));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        // the FP32 image of amax keeps its binade or rounds up to the next power of two: either
        // way |s v| < 2^7 for every v of the chunk
        const float s = pow2_scale((float) amax);
        __syncwarp();
        double t[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) t[e] = buf[warp][8 * lane + e] * (double) s;
        __syncwarp();
        const int kt = q * CHUNK_KT + lane / 8;
        if (kt < L.nkt) {
            uint4 ch[NS];
            slice8<NS>(t, ch);
            unsigned char * base = L.img + (tile_base * L.nkt + kt) * NS * XPIECE;
            const uint32_t off = tc::sw128_offset(ci, 8 * (lane % 8));
#pragma unroll
            for (int a = 0; a < NS; ++a) *reinterpret_cast<uint4 *>(base + a * XPIECE + off) = ch[a];
        }
        if (lane == 0) L.inv[(tile_base * nch + q) * TBN + ci] = 1.0f / s;
    }
}

// ---------------------------------------------------------------------------
// the multiply
// ---------------------------------------------------------------------------
// F64: each chunk's level sums (exact integers in FP32) are recombined and scaled in FP64 (exactly:
// the combined value spans about 48 bits, the scales are powers of two) and added into the
// output, which the owning thread reads and writes once per chunk; else they are recombined in
// FP32 into FP32 running sums and written once.  The FP64 form leaves only the slicing residuals,
// for transforms whose multiplies cancel strongly (tri).
template <int NU, int NX, int TBN, bool F64 = false>
__global__ void __launch_bounds__(THREADS, 1) trmm_mixed_kernel(const __grid_constant__ MixLaunch L) {
    using C = Cfg<NU, NX, TBN>;
    constexpr int NL = C::NL;
    constexpr int XPIECE = C::XPIECE;
    constexpr int HALF = TBN / 2;                     // columns per epilogue thread
    extern __shared__ unsigned char smem_raw[];
    unsigned char * const sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    __shared__ __align__(8) uint64_t bar_full[2], bar_empty[2], bar_accf, bar_acce, bar_done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nch = (L.nkt + CHUNK_KT - 1) / CHUNK_KT;

    if (tid == 0) {
        for (int i = 0; i < 2; ++i) { tc::mbar_init(&bar_full[i], 1); tc::mbar_init(&bar_empty[i], 1); }
        tc::mbar_init(&bar_accf, 1);
        tc::mbar_init(&bar_acce, 256);
        tc::mbar_init(&bar_done, 1);
        s_abort = 0;
    }
    if (warp == 8) tc::tmem_alloc(&s_tmem, 512);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;
    auto fail = [&]() { s_abort = 1; atomicExch(L.err, 1); };
    // chunk index of a K-tile, and whether kt starts / ends a chunk of tile range [k0, k1]
    auto chunk_start = [&](int kt, int k0) { return kt == k0 || kt % CHUNK_KT == 0; };
    auto chunk_end = [&](int kt, int k1) { return kt == k1 || kt % CHUNK_KT == CHUNK_KT - 1; };

    __shared__ unsigned s_issued;   // K-tile copies the loader issued
    if (warp == 9) {
        if (lane == 0) {
            unsigned q = 0, issued = 0;
            for (int t = blockIdx.x; t < L.ntiles && !s_abort; t += gridDim.x) {
                const MixTile T = L.tiles[t];
                const unsigned char * ua = L.Uimg[class_matrix(T.cls, L.ncls)] + (long long) T.it * L.nkt * NU * PIECE;
                const unsigned char * xb = L.Ximg + (((long long) (T.field * L.ncls + T.cls) * L.njt + T.jt) * L.nkt) * NX * XPIECE;
                for (int kt = T.k0; kt <= T.k1; ++kt, ++q) {
                    const int st = q & 1, u = q >> 1;
                    if (!tc::mbar_wait(&bar_empty[st], (u & 1) ^ 1, &s_abort)) { fail(); break; }
                    tc::mbar_arrive_expect_tx(&bar_full[st], C::STAGE);
                    tc::bulk_g2s(sm + st * C::STAGE, ua + (long long) kt * NU * PIECE, NU * PIECE, &bar_full[st]);
                    tc::bulk_g2s(sm + st * C::STAGE + NU * PIECE, xb + (long long) kt * NX * XPIECE, NX * XPIECE, &bar_full[st]);
                    issued = q + 1;
                }
            }
            s_issued = issued;
        }
        __syncwarp();
    } else if (warp == 8) {
        if (lane == 0) {
            unsigned q = 0, nacc = 0;
            const uint32_t s0 = tc::smem_addr(sm);
            for (int t = blockIdx.x; t < L.ntiles && !s_abort; t += gridDim.x) {
                const MixTile T = L.tiles[t];
                for (int kt = T.k0; kt <= T.k1 && !s_abort; ++kt, ++q) {
                    const int st = q & 1, u = q >> 1;
                    const bool cs = chunk_start(kt, T.k0);
                    if (cs) {   // the epilogue has read the previous chunk
                        if (!tc::mbar_wait(&bar_acce, (nacc & 1) ^ 1, &s_abort)) { fail(); break; }
                        nacc++;
                    }
                    if (!tc::mbar_wait(&bar_full[st], u & 1, &s_abort)) { fail(); break; }
                    tc::fence_after_sync();
                    const uint32_t ua = s0 + st * C::STAGE, xb = ua + NU * PIECE;
#pragma unroll
                    for (int kk = 0; kk < KT / 16; ++kk)
#pragma unroll
                        for (int lv = 0; lv < NL; ++lv) {
                            const int bmin = lv - (NX - 1) > 0 ? lv - (NX - 1) : 0;
                            const int bmax = lv < NU - 1 ? lv : NU - 1;
#pragma unroll
                            for (int b = bmin; b <= bmax; ++b) {
                                const int a = lv - b;
                                // level lv starts afresh with its first product of the chunk
                                const bool fresh = cs && kk == 0 && b == bmin;
                                tc::mma_bf16(tmem + lv * TBN, tc::desc_sw128(ua + b * PIECE + kk * 32),
                                             tc::desc_sw128(xb + a * XPIECE + kk * 32), C::IDESC, !fresh);
                            }
                        }
                    tc::commit(&bar_empty[st]);
                    if (chunk_end(kt, T.k1)) tc::commit(&bar_accf);
                }
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: lane quarter q4, columns HALF h .. HALF h + HALF - 1 of the tile ----
        const int q4 = warp & 3, h = warp >> 2;
        const int row_in = 32 * q4 + lane;
        const uint32_t tbase = tmem + ((uint32_t) (32 * q4) << 16) + HALF * h;
        unsigned nacc = 0;
        for (int t = blockIdx.x; t < L.ntiles && !s_abort; t += gridDim.x) {
            const MixTile T = L.tiles[t];
            float acc[HALF];
#pragma unroll
            for (int j = 0; j < HALF; ++j) acc[j] = 0.0f;
            const float * xinv = L.Xinv + ((long long) (T.field * L.ncls + T.cls) * L.njt + T.jt) * nch * TBN + HALF * h;
            bool first = true;
            for (int kt = T.k0; kt <= T.k1; ++kt) {
                if (!chunk_end(kt, T.k1)) continue;
                if (!tc::mbar_wait(&bar_accf, nacc & 1, &s_abort)) { fail(); break; }
                nacc++;
                __syncwarp();
                tc::fence_after_sync();
                const float * xi = xinv + (long long) (kt / CHUNK_KT) * TBN;
#pragma unroll
                for (int g = 0; g < HALF / 8; ++g) {
                    uint32_t a[NL][8];
#pragma unroll
                    for (int lv = 0; lv < NL; ++lv) tc::tmem_ld8_async(tbase + lv * TBN + 8 * g, a[lv]);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        if constexpr (F64) {
                            const int row = T.it * TB + row_in;
                            const int jj = T.jt * TBN + HALF * h + 8 * g + e;
                            if (row < L.n && jj < class_cols(L.M, T.cls, L.ncls)) {
                                double y = (double) __uint_as_float(a[NL - 1][e]);
#pragma unroll
                                for (int lv = NL - 2; lv >= 0; --lv) y = fma(y, 0.00390625, (double) __uint_as_float(a[lv][e]));
                                // 1 / (sX sU): powers of two
                                y *= (double) __ldg(xi + 8 * g + e) * (double) __ldg(L.Uinv[class_matrix(T.cls, L.ncls)] + row);
                                double * const p = L.out[T.field] + (long long) (T.cls + (long long) L.ncls * jj) * L.n + row;
                                *p = first ? y : *p + y;
                            }
                        } else {
                            float y = __uint_as_float(a[NL - 1][e]);
#pragma unroll
                            for (int lv = NL - 2; lv >= 0; --lv) y = fmaf(y, 0.00390625f, __uint_as_float(a[lv][e]));
                            acc[8 * g + e] = fmaf(y, __ldg(xi + 8 * g + e), acc[8 * g + e]);
                        }
                    }
                }
                first = false;
                tc::fence_before_sync();
                tc::mbar_arrive(&bar_acce);
            }
            if (s_abort) break;
            if (F64) continue;
            // out = acc / sU_i (acc holds the chunks' sums divided by their sX)
            const int row = T.it * TB + row_in;
            if (row < L.n) {
                const double sc = (double) __ldg(L.Uinv[class_matrix(T.cls, L.ncls)] + row);
                double * const o = L.out[T.field];
                const int ncols = class_cols(L.M, T.cls, L.ncls);
#pragma unroll
                for (int j = 0; j < HALF; ++j) {
                    const int jj = T.jt * TBN + HALF * h + j;
                    if (jj < ncols) __stcg(o + (long long) (T.cls + (long long) L.ncls * jj) * L.n + row, (double) acc[j] * sc);
                }
            }
        }
    }

    __syncthreads();
    __shared__ volatile int s_never;
    if (tid == 0) s_never = 0;
    __syncthreads();
    if (warp == 9 && lane == 0 && s_abort) {
        // after a wait ran out, copies may still be landing: the last one issued into each stage
        // (bounded waits) before the CTA's shared memory goes
        const unsigned issued = s_issued;
        for (unsigned j = issued >= 2 ? issued - 2 : 0; j < issued; ++j)
            (void) tc::mbar_wait(&bar_full[j & 1], (j >> 1) & 1, &s_never);
    }
    if (warp == 8) {
        if (lane == 0) {
            tc::commit(&bar_done);
            if (!tc::mbar_wait(&bar_done, 0, &s_never)) atomicExch(L.err, 2);
        }
        __syncwarp();
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 512);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct MixedTrmmPlan {
    // [slices of U - 3][inverse][trans][matrix]
    unsigned char * img[2][2][2][2] = {};
    float * inv[2][2][2][2] = {};
    int * d_err = nullptr;
};

// Work buffers of one batch, per input configuration (0: three input slices, 128
// columns per tile; 1: four slices, 96 columns), built on first use.
struct MixedTrmmWork {
    int nf = 0, n = 0, M = 0, nkt = 0, nch = 0, ncls = 0;
    struct Sub {
        int njt = 0;
        unsigned char * ximg = nullptr;          // sliced input
        float * xinv = nullptr;
        MixTile * tiles[2] = {nullptr, nullptr}; // [trans], longest K first
        int ntiles = 0;
    } sub[2];
};

// B = A^T for square n x n FP64 matrices of every field (32 x 32 tiles through shared memory).
struct TransposeLaunch {
    const double * in[kMaxFields];
    double * out[kMaxFields];
    int n;
};

__global__ void __launch_bounds__(256) transpose_square_kernel(const __grid_constant__ TransposeLaunch L) {
    __shared__ double tile[32][33];
    const int f = blockIdx.z;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;   // rows, columns of the input tile
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    const double * A = L.in[f];
    double * B = L.out[f];
    for (int y = ty; y < 32; y += 8) {
        const int i = i0 + tx, j = j0 + y;                   // tile[y][tx] = A(i0 + tx, j0 + y)
        tile[y][tx] = (i < L.n && j < L.n) ? __ldcg(A + (long long) j * L.n + i) : 0.0;
    }
    __syncthreads();
    for (int y = ty; y < 32; y += 8) {
        const int i = j0 + tx, j = i0 + y;                   // B(i, j) = A(j, i) = tile[tx][y]
        if (i < L.n && j < L.n) __stcg(B + (long long) j * L.n + i, tile[tx][y]);
    }
}

}  // namespace

cudaError_t launch_transpose_square(double * const * in, double * const * out, int nf, int n, cudaStream_t st) {
    if (nf <= 0 || n <= 0) return cudaSuccess;
    static thread_local TransposeLaunch L;
    for (int f = 0; f < nf; ++f) { L.in[f] = in[f]; L.out[f] = out[f]; }
    L.n = n;
    const dim3 grid((n + 31) / 32, (n + 31) / 32, nf);
    transpose_square_kernel<<<grid, 256, 0, st>>>(L);
    count_launch();
    return cudaGetLastError();
}

namespace {
}  // namespace

void mixed_trmm_plan_free(void * p) {
    MixedTrmmPlan * T = static_cast<MixedTrmmPlan *>(p);
    if (!T) return;
    for (auto & a : T->img) for (auto & b : a) for (auto & c : b) for (auto & d : c) cudaFree(d);
    for (auto & a : T->inv) for (auto & b : a) for (auto & c : b) for (auto & d : c) cudaFree(d);
    cudaFree(T->d_err);
    delete T;
}

void mixed_trmm_work_free(void * p) {
    MixedTrmmWork * W = static_cast<MixedTrmmWork *>(p);
    if (!W) return;
    for (auto & x : W->sub) { cudaFree(x.ximg); cudaFree(x.xinv); cudaFree(x.tiles[0]); cudaFree(x.tiles[1]); }
    delete W;
}

int mixed_trmm_device_error(void * p) {
    MixedTrmmPlan * T = static_cast<MixedTrmmPlan *>(p);
    if (!T || !T->d_err) return 0;
    int v = 0;
    if (cudaMemcpy(&v, T->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (v) cudaMemset(T->d_err, 0, sizeof(int));
    return v;
}

// Out = op(U) In for the column classes of every field, U = P or Pinv of the plan, with nu
// slices of U (4) and nx (3 or 4) of the input.  ncls = 4: the four stride-4 classes of
// sph and disk, U[0] on classes 0 and 3 and U[1] on 1 and 2; ncls = 1: every column,
// U[which].  In and Out may be the same matrices: the input is sliced into the work
// buffers before the multiply writes.  Builds the plan's slice images of op(U) on first
// use (into *plan_slot) and the batch's work buffers (*work_slot).
cudaError_t launch_trmm_mixed(HarmonicPlan * H, void ** plan_slot, void ** work_slot, int nu, int nx, bool inverse,
                              bool trans, double * const * in, double * const * out, int nf, int M, cudaStream_t st,
                              int ncls, int which) {
    const int n = H->n;
    const int nkt = (n + KT - 1) / KT, nit = (n + TB - 1) / TB;
    if (ncls != 4 && ncls != 1) return cudaErrorInvalidValue;
    if (nu != 4 || (nx != 3 && nx != 4)) return cudaErrorInvalidValue;   // the configurations built
    const int cfg = nx == 4 ? 1 : 0;
    const int tbn = cfg ? 96 : 128;
    if (!*plan_slot) *plan_slot = new MixedTrmmPlan();
    MixedTrmmPlan * T = static_cast<MixedTrmmPlan *>(*plan_slot);
    if (!T->d_err) {
        cudaError_t e = cudaMalloc(&T->d_err, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(T->d_err, 0, sizeof(int));
        if (e != cudaSuccess) return e;
    }
    const int ui = nu - 3, ii = inverse ? 1 : 0, ti = trans ? 1 : 0;
    for (int u = 0; u < 2; ++u) {
        if (T->img[ui][ii][ti][u] || (ncls == 1 && u != which)) continue;
        const size_t bytes = (size_t) nit * nkt * nu * PIECE;
        cudaError_t e = cudaMalloc(&T->img[ui][ii][ti][u], bytes);
        if (e == cudaSuccess) e = cudaMalloc(&T->inv[ui][ii][ti][u], sizeof(float) * (size_t) nit * TB);
        if (e != cudaSuccess) return e;
        const double * U = inverse ? H->dPinv[u] : H->dP[u];
        const int rows = nit * TB;
        slice_matrix_kernel<4><<<(rows + 7) / 8, 256, 0, st>>>(U, n, trans, nkt, T->img[ui][ii][ti][u], T->inv[ui][ii][ti][u]);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    MixedTrmmWork * W = static_cast<MixedTrmmWork *>(*work_slot);
    if (!W) {
        W = new MixedTrmmWork();
        *work_slot = W;
        W->nf = nf; W->n = n; W->M = M; W->nkt = nkt; W->ncls = ncls;
        W->nch = (nkt + CHUNK_KT - 1) / CHUNK_KT;
    }
    if (W->nf != nf || W->n != n || W->M != M || W->ncls != ncls) return cudaErrorInvalidValue;
    MixedTrmmWork::Sub & X = W->sub[cfg];
    if (!X.ximg) {
        X.njt = (class_cols(M, 0, ncls) + tbn - 1) / tbn;
        const size_t xbytes = (size_t) nf * ncls * X.njt * nkt * nx * tbn * KT * 2;
        cudaError_t e = cudaMalloc(&X.ximg, xbytes);
        if (e == cudaSuccess) e = cudaMalloc(&X.xinv, sizeof(float) * (size_t) nf * ncls * X.njt * W->nch * tbn);
        if (e != cudaSuccess) return e;
        for (int tr = 0; tr < 2; ++tr) {
            // Tiles in blocks of kRowGroup row tiles (longest K first) x kColGroup column tiles:
            // the persistent CTAs take consecutive tiles, so the tiles in flight share a few row
            // tiles' slices of op(U) and a few column tiles' slices of the input, which stay in
            // L2 (longest first, the input's slices are re-read from DRAM once per row tile).
            // Within a block, longest K first.
            struct Key { int rg, cg, klen, col, it; };
            std::vector<std::pair<Key, MixTile>> v;
            for (int f = 0; f < nf; ++f)
                for (int r = 0; r < ncls; ++r)
                    for (int it = 0; it < nit; ++it)
                        for (int jt = 0; jt * tbn < class_cols(M, r, ncls); ++jt) {
                            const int k0 = tr ? 0 : 2 * it, k1 = tr ? std::min(nkt - 1, 2 * it + 1) : nkt - 1;
                            const int rank = tr ? nit - 1 - it : it;            // row tiles by K length, longest first
                            const int col = (f * ncls + r) * X.njt + jt;
                            const Key k{kRowGroup > 0 ? rank / kRowGroup : 0, kColGroup > 0 ? col / kColGroup : 0, k1 - k0 + 1, col, it};
                            v.push_back({k, MixTile{f, r, it, jt, k0, k1}});
                        }
            std::stable_sort(v.begin(), v.end(), [](const auto & a, const auto & b) {
                if (a.first.rg != b.first.rg) return a.first.rg < b.first.rg;
                if (a.first.cg != b.first.cg) return a.first.cg < b.first.cg;
                return a.first.klen > b.first.klen;
            });
            std::vector<MixTile> tl;
            for (auto & x : v) tl.push_back(x.second);
            X.ntiles = (int) tl.size();
            e = cudaMalloc(&X.tiles[tr], sizeof(MixTile) * std::max<size_t>(1, tl.size()));
            if (e == cudaSuccess && !tl.empty()) e = cudaMemcpy(X.tiles[tr], tl.data(), sizeof(MixTile) * tl.size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return e;
        }
    }
    // slice the input
    static thread_local SliceXLaunch SX;
    for (int f = 0; f < nf; ++f) SX.in[f] = in[f];
    SX.n = n; SX.M = M; SX.nkt = nkt; SX.njt = X.njt; SX.ncls = ncls;
    SX.img = X.ximg; SX.inv = X.xinv;
    const int sgrid = nf * ncls * X.njt * W->nch;
    if (cfg) slice_input_kernel<4, 96><<<sgrid, 256, 0, st>>>(SX);
    else     slice_input_kernel<3, 128><<<sgrid, 256, 0, st>>>(SX);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // multiply
    static thread_local MixLaunch L;
    for (int f = 0; f < nf; ++f) L.out[f] = out[f];
    for (int u = 0; u < 2; ++u) {
        const int us = ncls == 1 ? which : u;   // one class: the chosen matrix in slot 0
        L.Uimg[u] = T->img[ui][ii][ti][us];
        L.Uinv[u] = T->inv[ui][ii][ti][us];
    }
    L.Ximg = X.ximg; L.Xinv = X.xinv;
    L.tiles = X.tiles[ti]; L.ntiles = X.ntiles;
    L.n = n; L.M = M; L.nkt = nkt; L.njt = X.njt; L.ncls = ncls;
    L.err = T->d_err;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ctas = std::min(sms, X.ntiles);
    if (ctas <= 0) return cudaSuccess;
    if (cfg && ncls == 1) {   // one class (tri): chunks folded into the output in FP64
        auto kern = trmm_mixed_kernel<4, 4, 96, true>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Cfg<4, 4, 96>::SMEM);
        if (e == cudaSuccess) { kern<<<ctas, THREADS, Cfg<4, 4, 96>::SMEM, st>>>(L); e = cudaGetLastError(); }
    } else if (cfg) {
        auto kern = trmm_mixed_kernel<4, 4, 96>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Cfg<4, 4, 96>::SMEM);
        if (e == cudaSuccess) { kern<<<ctas, THREADS, Cfg<4, 4, 96>::SMEM, st>>>(L); e = cudaGetLastError(); }
    } else {
        auto kern = trmm_mixed_kernel<4, 3, 128>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Cfg<4, 3, 128>::SMEM);
        if (e == cudaSuccess) { kern<<<ctas, THREADS, Cfg<4, 3, 128>::SMEM, st>>>(L); e = cudaGetLastError(); }
    }
    count_launch();
    return e;
}

}  // namespace ftb
