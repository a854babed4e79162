// The sph and disk connection multiply (src/drivers.c:833-865, 989-1021: four column classes j = 0,1,2,3 mod 4,
// class j multiplied by U[0] for j = 0, 3 and U[1] for j = 1, 2, U upper triangular)
// on the tcgen05 tensor cores, in two forms: from 8-bit integer digits with exact 32-bit
// accumulation over whole columns (the "8-bit integer form" below, the one the library uses),
// and from fixed-point BF16 slices with exact FP32 sums of 256-row chunks (this header; kept for
// comparison, FT_B200_MULTIPLY=bf16).
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
#include <cstdlib>
#include <cstring>
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
// 8-bit integer form
// ---------------------------------------------------------------------------
// The same multiply from 8-bit integer digits: a row of op(U) scaled by a power of two
// sU_i with |sU_i U| < 64, a column of the input by one power of two sX_j over all its rows
// (|sX_j x| < 64), both cut into balanced digits of base 2^7,
//   t = d_0 + d_1 2^-7 + d_2 2^-14 + ...,  d_k = nearest integer of the remaining value,
// every digit in [-64, 64] (each remainder is at most 1/2 before the factor 2^7; the cuts are
// exact in FP64).  Products d_b e_a of one level L = a + b <= LMAX are at most 2^12 and a level
// sums at most 5 of them per row of K, so its 32-bit integer accumulator (tcgen05.mma kind::i8) is
// exact for any K below 2^31 / (5 2^12) = 104857: one accumulator set per output tile, no folds
// along K.  The epilogue recombines the levels in FP64 (exact: integers below 2^31, powers of two)
// and scales by 1 / (sU_i sX_j).  Digits: NU = 5 of op(U) (34 bits), NX = 4 (27 bits) or 5 (34)
// of the input, at twice the BF16 rate.  K-tiles of 64 rows are 64-byte rows of one-byte digits
// (the 64-byte swizzle), three stages in flight.
constexpr int KT8 = 64;                      // K per tile (a 64-byte row of one-byte digits)
constexpr int PIECE8 = TB * KT8;             // bytes of one digit of one K-tile of op(U) (8 KB)
constexpr int NSTAGE8 = 3;
// configurations (NU, NX, TBN, levels kept 0 .. LMAX): four input digits -> (5, 4, 96, 4),
// fourteen products; five input digits (tri, MIXED_BF16X4) -> (5, 5, 96, 4), fifteen products.
// (Levels 0 .. 3 only would let 128-column tiles fill tensor memory with ten products, 30 % less
// time in the multiply, but the dropped level doubles the mixed forms' error.)
constexpr int TBN8_4 = 96, LMAX8_4 = 4;
constexpr int TBN8_5 = 96, LMAX8_5 = 4;

template <int NU, int NX, int TBN, int LMAX> struct Cfg8 {
    static constexpr int NL = LMAX + 1;                     // accumulators per tile
    static constexpr int XPIECE = TBN * KT8;                // bytes of one input digit of one K-tile
    static constexpr int STAGE = NU * PIECE8 + NX * XPIECE;
    static constexpr size_t SMEM = NSTAGE8 * (size_t) STAGE + 1024;
    static constexpr uint32_t IDESC = tc::idesc_s8(TB, TBN);
    static_assert(TBN % 16 == 0 && TBN <= 128, "tile width");
    static_assert(NL * TBN <= 512, "accumulators exceed tensor memory");
    static_assert(XPIECE % 512 == 0 && STAGE % 512 == 0, "swizzle atoms must stay aligned");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

// 16 consecutive K values (scaled, |t| < 64) -> ND 16-byte chunks of digits
template <int ND>
__device__ __forceinline__ void digits16(const double * t_in, uint4 * out) {
    uint32_t w[ND][4];
#pragma unroll
    for (int a = 0; a < ND; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) w[a][q] = 0u;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        double t = t_in[e];
#pragma unroll
        for (int a = 0; a < ND; ++a) {
            const double i = rint(t);
            w[a][e >> 2] |= ((uint32_t) (int) i & 0xFFu) << (8 * (e & 3));
            t = (t - i) * 128.0;                         // exact
        }
    }
#pragma unroll
    for (int a = 0; a < ND; ++a) out[a] = make_uint4(w[a][0], w[a][1], w[a][2], w[a][3]);
}

// One warp per row of op(U): its power-of-two scale, then NU digits of every K-tile
// (image [row tile][K-tile][digit], pieces of TB rows x 64 bytes).
template <int NU>
__global__ void slice_matrix_s8_kernel(const double * __restrict__ U, int n, bool trans, int nkt,
                                       unsigned char * __restrict__ img, double * __restrict__ inv) {
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
    int ex = 0;
    if (amax > 0) (void) frexp(amax, &ex);                      // amax < 2^ex
    const double s = amax > 0 ? ldexp(1.0, 6 - ex) : 1.0;       // |s U| < 64
    if (lane == 0) inv[row] = 1.0 / s;
    const int it = row / TB, rr = row % TB;
    for (int kt = 0; kt < nkt; ++kt) {
        if (lane >= KT8 / 16) continue;                         // 4 lanes x 16 values = one K-tile row
        double t[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) t[e] = at(kt * KT8 + 16 * lane + e) * s;
        uint4 ch[NU];
        digits16<NU>(t, ch);
        unsigned char * base = img + ((long long) it * nkt + kt) * NU * PIECE8;
        const uint32_t off = tc::sw64_byte(rr, 16 * lane);
#pragma unroll
        for (int a = 0; a < NU; ++a) *reinterpret_cast<uint4 *>(base + a * PIECE8 + off) = ch[a];
    }
}

struct SliceX8Launch {
    const double * in[kMaxFields];
    int nf, n, M, nkt, njt, ncls;
    unsigned char * img;                // [field][cls][jt][kt][NX digits], pieces of TBN x 64 bytes
    double * inv;                       // [field][cls][jt][TBN]: 1 / sX per column
};

// One warp per input column: its power-of-two scale over all n rows.
__global__ void column_scale_kernel(const __grid_constant__ SliceX8Launch L, int TBN) {
    const int lane = threadIdx.x & 31;
    const long long w = (long long) blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const long long per_f = (long long) L.ncls * L.njt * TBN;
    if (w >= per_f * L.nf) return;                     // the whole warp: w is uniform
    const int f = (int) (w / per_f);
    const long long rem = w % per_f;
    const int r = (int) (rem / ((long long) L.njt * TBN)), j = (int) (rem % ((long long) L.njt * TBN));
    double amax = 0.0;
    if (j < class_cols(L.M, r, L.ncls)) {
        const double * col = L.in[f] + (long long) (r + (long long) L.ncls * j) * L.n;
        for (int k = lane; k < L.n; k += 32) amax = fmax(amax, fabs(__ldcg(col + k)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    int ex = 0;
    if (amax > 0) (void) frexp(amax, &ex);
    if (lane == 0) L.inv[w] = amax > 0 ? ldexp(1.0, ex - 6) : 1.0;   // 1 / s, |s x| < 64
}

// One CTA per (field, class, column tile, 256 rows), one warp per column at a time, each lane
// 8 consecutive rows: NX digits into the column's row of the K-tile pieces.
template <int NX, int TBN>
__global__ void __launch_bounds__(256) slice_input_s8_kernel(const __grid_constant__ SliceX8Launch L) {
    constexpr int XPIECE = TBN * KT8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nch = (L.nkt + 3) / 4;                    // 256-row chunks: four K-tiles of 64
    int b = blockIdx.x;
    const int q = b % nch; b /= nch;
    const int jt = b % L.njt; b /= L.njt;
    const int r = b % L.ncls;
    const int f = b / L.ncls;
    const int ncols = class_cols(L.M, r, L.ncls);
    const long long tile_base = ((long long) (f * L.ncls + r) * L.njt + jt);
    const int kt = q * 4 + lane / 8;                    // K-tile of this lane's 8 rows
    const int kb = 8 * (lane % 8);                      // their first byte in the 64-byte row
    if (kt >= L.nkt) return;
    for (int ci = warp; ci < TBN; ci += 8) {
        const int j = jt * TBN + ci;
        const bool cok = j < ncols;
        const double s = 1.0 / L.inv[tile_base * TBN + ci];
        const double * col = L.in[f] + (long long) (r + (long long) L.ncls * j) * L.n;
        uint32_t w[NX][2];
#pragma unroll
        for (int a = 0; a < NX; ++a) { w[a][0] = 0u; w[a][1] = 0u; }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int row = kt * KT8 + kb + e;
            double t = (cok && row < L.n) ? __ldcg(col + row) * s : 0.0;
#pragma unroll
            for (int a = 0; a < NX; ++a) {
                const double i = rint(t);
                w[a][e >> 2] |= ((uint32_t) (int) i & 0xFFu) << (8 * (e & 3));
                t = (t - i) * 128.0;
            }
        }
        unsigned char * base = L.img + (tile_base * L.nkt + kt) * NX * XPIECE;
        const uint32_t off = tc::sw64_byte(ci, kb);
#pragma unroll
        for (int a = 0; a < NX; ++a) *reinterpret_cast<uint2 *>(base + a * XPIECE + off) = make_uint2(w[a][0], w[a][1]);
    }
}

struct Mix8Launch {
    double * out[kMaxFields];
    const unsigned char * Uimg[2];      // per class matrix: [it][kt][NU digits]
    const double * Uinv[2];             // 1 / sU per row
    const unsigned char * Ximg;         // [field][cls][jt][kt][NX digits]
    const double * Xinv;                // [field][cls][jt][TBN]: 1 / sX per column
    const MixTile * tiles;
    int ntiles;
    int n, M, nkt, njt, ncls;
    int * err;
};

template <int NU, int NX, int TBN, int LMAX>
__global__ void __launch_bounds__(THREADS, 1) trmm_s8_kernel(const __grid_constant__ Mix8Launch L) {
    using C = Cfg8<NU, NX, TBN, LMAX>;
    constexpr int NL = C::NL;
    constexpr int XPIECE = C::XPIECE;
    constexpr int HALF = TBN / 2;                     // columns per epilogue thread
    extern __shared__ unsigned char smem_raw[];
    unsigned char * const sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    __shared__ __align__(8) uint64_t bar_full[NSTAGE8], bar_empty[NSTAGE8], bar_accf, bar_acce, bar_done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ unsigned s_issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int i = 0; i < NSTAGE8; ++i) { tc::mbar_init(&bar_full[i], 1); tc::mbar_init(&bar_empty[i], 1); }
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

    if (warp == 9) {
        if (lane == 0) {
            unsigned q = 0, issued = 0;
            for (int t = blockIdx.x; t < L.ntiles && !s_abort; t += gridDim.x) {
                const MixTile T = L.tiles[t];
                const unsigned char * ua = L.Uimg[class_matrix(T.cls, L.ncls)] + (long long) T.it * L.nkt * NU * PIECE8;
                const unsigned char * xb = L.Ximg + (((long long) (T.field * L.ncls + T.cls) * L.njt + T.jt) * L.nkt) * NX * XPIECE;
                for (int kt = T.k0; kt <= T.k1; ++kt, ++q) {
                    const int st = (int) (q % NSTAGE8), u = (int) (q / NSTAGE8);
                    if (!tc::mbar_wait(&bar_empty[st], (u & 1) ^ 1, &s_abort)) { fail(); break; }
                    tc::mbar_arrive_expect_tx(&bar_full[st], C::STAGE);
                    tc::bulk_g2s(sm + st * C::STAGE, ua + (long long) kt * NU * PIECE8, NU * PIECE8, &bar_full[st]);
                    tc::bulk_g2s(sm + st * C::STAGE + NU * PIECE8, xb + (long long) kt * NX * XPIECE, NX * XPIECE, &bar_full[st]);
                    issued = q + 1;
                }
            }
            s_issued = issued;
        }
        __syncwarp();
    } else if (warp == 8) {
        if (lane == 0) {
            unsigned q = 0, ntile = 0;
            const uint32_t s0 = tc::smem_addr(sm);
            for (int t = blockIdx.x; t < L.ntiles && !s_abort; t += gridDim.x, ++ntile) {
                const MixTile T = L.tiles[t];
                // the epilogue has read the previous tile's accumulators
                if (!tc::mbar_wait(&bar_acce, (ntile & 1) ^ 1, &s_abort)) { fail(); break; }
                for (int kt = T.k0; kt <= T.k1 && !s_abort; ++kt, ++q) {
                    const int st = (int) (q % NSTAGE8), u = (int) (q / NSTAGE8);
                    if (!tc::mbar_wait(&bar_full[st], u & 1, &s_abort)) { fail(); break; }
                    tc::fence_after_sync();
                    const uint32_t ua = s0 + st * C::STAGE, xb = ua + NU * PIECE8;
#pragma unroll
                    for (int kk = 0; kk < KT8 / 32; ++kk)
#pragma unroll
                        for (int lv = 0; lv < NL; ++lv) {
                            const int bmin = lv - (NX - 1) > 0 ? lv - (NX - 1) : 0;
                            const int bmax = lv < NU - 1 ? lv : NU - 1;
#pragma unroll
                            for (int b = bmin; b <= bmax; ++b) {
                                const int a = lv - b;
                                // level lv starts afresh with its first product of the tile
                                const bool fresh = kt == T.k0 && kk == 0 && b == bmin;
                                tc::mma_s8(tmem + lv * TBN, tc::desc_sw64(ua + b * PIECE8 + kk * 32),
                                           tc::desc_sw64(xb + a * XPIECE + kk * 32), C::IDESC, !fresh);
                            }
                        }
                    tc::commit(&bar_empty[st]);
                }
                tc::commit(&bar_accf);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: lane quarter q4, columns HALF h .. HALF h + HALF - 1 of the tile ----
        const int q4 = warp & 3, h = warp >> 2;
        const int row_in = 32 * q4 + lane;
        const uint32_t tbase = tmem + ((uint32_t) (32 * q4) << 16) + HALF * h;
        unsigned ntile = 0;
        for (int t = blockIdx.x; t < L.ntiles && !s_abort; t += gridDim.x, ++ntile) {
            const MixTile T = L.tiles[t];
            if (!tc::mbar_wait(&bar_accf, ntile & 1, &s_abort)) { fail(); break; }
            __syncwarp();
            tc::fence_after_sync();
            const int row = T.it * TB + row_in;
            const int ncols = class_cols(L.M, T.cls, L.ncls);
            const double su = row < L.n ? __ldg(L.Uinv[class_matrix(T.cls, L.ncls)] + row) : 0.0;
            const double * xinv = L.Xinv + ((long long) (T.field * L.ncls + T.cls) * L.njt + T.jt) * TBN + HALF * h;
            double * const o = L.out[T.field];
#pragma unroll
            for (int g = 0; g < HALF / 8; ++g) {
                uint32_t a[NL][8];
#pragma unroll
                for (int lv = 0; lv < NL; ++lv) tc::tmem_ld8_async(tbase + lv * TBN + 8 * g, a[lv]);
                tc::tmem_wait_ld();
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const int jj = T.jt * TBN + HALF * h + 8 * g + e;
                    // a 32-bit integer as FP64 without the conversion unit: 2^52 + 2^31 + A in the
                    // bits, then subtract 2^52 + 2^31 (exact)
                    auto as_f64 = [](uint32_t v) { return __hiloint2double(0x43300000, (int) (v ^ 0x80000000u)) - 4503601774854144.0; };
                    double y = as_f64(a[NL - 1][e]);
#pragma unroll
                    for (int lv = NL - 2; lv >= 0; --lv) y = fma(y, 0.0078125, as_f64(a[lv][e]));   // 2^-7
                    if (row < L.n && jj < ncols)
                        __stcg(o + (long long) (T.cls + (long long) L.ncls * jj) * L.n + row, y * su * __ldg(xinv + 8 * g + e));
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&bar_acce);
        }
    }

    __syncthreads();
    __shared__ volatile int s_never;
    if (tid == 0) s_never = 0;
    __syncthreads();
    if (warp == 9 && lane == 0 && s_abort) {
        // after a wait ran out, copies may still be landing: the last one issued into each stage
        const unsigned issued = s_issued;
        for (unsigned j = issued >= NSTAGE8 ? issued - NSTAGE8 : 0; j < issued; ++j)
            (void) tc::mbar_wait(&bar_full[j % NSTAGE8], (j / NSTAGE8) & 1, &s_never);
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
    // the 8-bit integer form: [inverse][trans][matrix]
    unsigned char * img8[2][2][2] = {};
    double * inv8[2][2][2] = {};
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
    struct Sub8 {                                // the 8-bit integer form: four or five input digits
        int njt = 0;
        unsigned char * ximg = nullptr;
        double * xinv = nullptr;                 // 1 / sX per column
        MixTile * tiles[2] = {nullptr, nullptr};
        int ntiles = 0;
    } sub8[2];
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

// Output tiles of every field and class in blocks of kRowGroup row tiles (longest K first) x
// kColGroup column tiles: the persistent CTAs take consecutive tiles, so the tiles in flight
// share a few row tiles' slices of op(U) and a few column tiles' slices of the input, which stay
// in L2 (longest first, the input's slices are re-read from DRAM once per row tile).  Within a
// block, longest K first.  K-tiles of 64 rows; tr: op(U) = U^T (K-tiles 0 .. the tile's last).
std::vector<MixTile> order_tiles(int nf, int ncls, int nit, int nkt, int njt, int tbn, int M, int tr) {
    struct Key { int rg, cg, klen; };
    std::vector<std::pair<Key, MixTile>> v;
    for (int f = 0; f < nf; ++f)
        for (int r = 0; r < ncls; ++r)
            for (int it = 0; it < nit; ++it)
                for (int jt = 0; jt * tbn < class_cols(M, r, ncls); ++jt) {
                    const int k0 = tr ? 0 : 2 * it, k1 = tr ? std::min(nkt - 1, 2 * it + 1) : nkt - 1;
                    const int rank = tr ? nit - 1 - it : it;            // row tiles by K length, longest first
                    const int col = (f * ncls + r) * njt + jt;
                    const Key k{kRowGroup > 0 ? rank / kRowGroup : 0, kColGroup > 0 ? col / kColGroup : 0, k1 - k0 + 1};
                    v.push_back({k, MixTile{f, r, it, jt, k0, k1}});
                }
    std::stable_sort(v.begin(), v.end(), [](const auto & a, const auto & b) {
        if (a.first.rg != b.first.rg) return a.first.rg < b.first.rg;
        if (a.first.cg != b.first.cg) return a.first.cg < b.first.cg;
        return a.first.klen > b.first.klen;
    });
    std::vector<MixTile> tl;
    for (auto & x : v) tl.push_back(x.second);
    return tl;
}

cudaError_t upload_tiles(const std::vector<MixTile> & tl, MixTile ** d, int * ntiles) {
    *ntiles = (int) tl.size();
    cudaError_t e = cudaMalloc(d, sizeof(MixTile) * std::max<size_t>(1, tl.size()));
    if (e == cudaSuccess && !tl.empty()) e = cudaMemcpy(*d, tl.data(), sizeof(MixTile) * tl.size(), cudaMemcpyHostToDevice);
    return e;
}

}  // namespace

void mixed_trmm_plan_free(void * p) {
    MixedTrmmPlan * T = static_cast<MixedTrmmPlan *>(p);
    if (!T) return;
    for (auto & a : T->img) for (auto & b : a) for (auto & c : b) for (auto & d : c) cudaFree(d);
    for (auto & a : T->inv) for (auto & b : a) for (auto & c : b) for (auto & d : c) cudaFree(d);
    for (auto & a : T->img8) for (auto & b : a) for (auto & c : b) cudaFree(c);
    for (auto & a : T->inv8) for (auto & b : a) for (auto & c : b) cudaFree(c);
    cudaFree(T->d_err);
    delete T;
}

void mixed_trmm_work_free(void * p) {
    MixedTrmmWork * W = static_cast<MixedTrmmWork *>(p);
    if (!W) return;
    for (auto & x : W->sub) { cudaFree(x.ximg); cudaFree(x.xinv); cudaFree(x.tiles[0]); cudaFree(x.tiles[1]); }
    for (auto & x : W->sub8) { cudaFree(x.ximg); cudaFree(x.xinv); cudaFree(x.tiles[0]); cudaFree(x.tiles[1]); }
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

namespace {

// The integer form of the multiply serves the call (NX = 4 input digits where the BF16 form
// would cut three slices, 5 where it would cut four: tri, MIXED_BF16X4) unless FT_B200_MULTIPLY
// is "bf16", which selects the BF16 form (kept for comparison).
bool multiply_s8() {
    static const bool on = [] {
        const char * e = std::getenv("FT_B200_MULTIPLY");
        return !(e && std::strcmp(e, "bf16") == 0);
    }();
    return on;
}

cudaError_t launch_trmm_s8(HarmonicPlan * H, MixedTrmmPlan * T, MixedTrmmWork * W, int nx8, bool inverse, bool trans,
                           double * const * in, double * const * out, int nf, int M, cudaStream_t st, int ncls, int which) {
    const int n = H->n;
    const int nkt = (n + KT8 - 1) / KT8, nit = (n + TB - 1) / TB;
    const int cfg = nx8 == 5 ? 1 : 0, tbn = cfg ? TBN8_5 : TBN8_4;
    const int ii = inverse ? 1 : 0, ti = trans ? 1 : 0;
    for (int u = 0; u < 2; ++u) {
        if (T->img8[ii][ti][u] || (ncls == 1 && u != which)) continue;
        const size_t bytes = (size_t) nit * nkt * 5 * PIECE8;
        cudaError_t e = cudaMalloc(&T->img8[ii][ti][u], bytes);
        if (e == cudaSuccess) e = cudaMalloc(&T->inv8[ii][ti][u], sizeof(double) * (size_t) nit * TB);
        if (e != cudaSuccess) return e;
        const double * U = inverse ? H->dPinv[u] : H->dP[u];
        const int rows = nit * TB;
        slice_matrix_s8_kernel<5><<<(rows + 7) / 8, 256, 0, st>>>(U, n, trans, nkt, T->img8[ii][ti][u], T->inv8[ii][ti][u]);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    MixedTrmmWork::Sub8 & X = W->sub8[cfg];
    if (!X.ximg) {
        X.njt = (class_cols(M, 0, ncls) + tbn - 1) / tbn;
        const size_t xbytes = (size_t) nf * ncls * X.njt * nkt * nx8 * tbn * KT8;
        cudaError_t e = cudaMalloc(&X.ximg, xbytes);
        if (e == cudaSuccess) e = cudaMalloc(&X.xinv, sizeof(double) * (size_t) nf * ncls * X.njt * tbn);
        if (e != cudaSuccess) return e;
        for (int tr = 0; tr < 2; ++tr) {
            e = upload_tiles(order_tiles(nf, ncls, nit, nkt, X.njt, tbn, M, tr), &X.tiles[tr], &X.ntiles);
            if (e != cudaSuccess) return e;
        }
    }
    // the input's column scales, then its digits
    static thread_local SliceX8Launch SX;
    for (int f = 0; f < nf; ++f) SX.in[f] = in[f];
    SX.nf = nf; SX.n = n; SX.M = M; SX.nkt = nkt; SX.njt = X.njt; SX.ncls = ncls;
    SX.img = X.ximg; SX.inv = X.xinv;
    const long long ncolw = (long long) nf * ncls * X.njt * tbn;        // one warp per column
    column_scale_kernel<<<(unsigned) ((ncolw + 7) / 8), 256, 0, st>>>(SX, tbn);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int sgrid = nf * ncls * X.njt * ((nkt + 3) / 4);
    if (cfg) slice_input_s8_kernel<5, TBN8_5><<<sgrid, 256, 0, st>>>(SX);
    else     slice_input_s8_kernel<4, TBN8_4><<<sgrid, 256, 0, st>>>(SX);
    count_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    static thread_local Mix8Launch L;
    for (int f = 0; f < nf; ++f) L.out[f] = out[f];
    for (int u = 0; u < 2; ++u) {
        const int us = ncls == 1 ? which : u;   // one class: the chosen matrix in slot 0
        L.Uimg[u] = T->img8[ii][ti][us];
        L.Uinv[u] = T->inv8[ii][ti][us];
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
    if (cfg) {
        using C = Cfg8<5, 5, TBN8_5, LMAX8_5>;
        auto kern = trmm_s8_kernel<5, 5, TBN8_5, LMAX8_5>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) C::SMEM);
        if (e == cudaSuccess) { kern<<<ctas, THREADS, C::SMEM, st>>>(L); e = cudaGetLastError(); }
    } else {
        using C = Cfg8<5, 4, TBN8_4, LMAX8_4>;
        auto kern = trmm_s8_kernel<5, 4, TBN8_4, LMAX8_4>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) C::SMEM);
        if (e == cudaSuccess) { kern<<<ctas, THREADS, C::SMEM, st>>>(L); e = cudaGetLastError(); }
    }
    count_launch();
    return e;
}

}  // namespace

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
    MixedTrmmWork * W = static_cast<MixedTrmmWork *>(*work_slot);
    if (!W) {
        W = new MixedTrmmWork();
        *work_slot = W;
        W->nf = nf; W->n = n; W->M = M; W->nkt = nkt; W->ncls = ncls;
        W->nch = (nkt + CHUNK_KT - 1) / CHUNK_KT;
    }
    if (W->nf != nf || W->n != n || W->M != M || W->ncls != ncls) return cudaErrorInvalidValue;
    if (multiply_s8()) return launch_trmm_s8(H, T, W, nx == 4 ? 5 : 4, inverse, trans, in, out, nf, M, st, ncls, which);
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
    MixedTrmmWork::Sub & X = W->sub[cfg];
    if (!X.ximg) {
        X.njt = (class_cols(M, 0, ncls) + tbn - 1) / tbn;
        const size_t xbytes = (size_t) nf * ncls * X.njt * nkt * nx * tbn * KT * 2;
        cudaError_t e = cudaMalloc(&X.ximg, xbytes);
        if (e == cudaSuccess) e = cudaMalloc(&X.xinv, sizeof(float) * (size_t) nf * ncls * X.njt * W->nch * tbn);
        if (e != cudaSuccess) return e;
        for (int tr = 0; tr < 2; ++tr) {
            e = upload_tiles(order_tiles(nf, ncls, nit, nkt, X.njt, tbn, M, tr), &X.tiles[tr], &X.ntiles);
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
