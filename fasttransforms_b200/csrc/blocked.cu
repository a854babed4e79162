// Blocked rotation sweeps for fields that share one plan (sph, disk or tri).
//
// The sweeps of a parity are cut into blocks of BLK consecutive sweeps on a
// fixed grid (block beta holds sweeps j = p + STEP*BLK*(beta + 1) - STEP - STEP*s,
// s = 0 .. BLK-1, with STEP = 2 for sph and disk and 1 for tri, whose sweeps
// have no parity), and each block into parallelogram tiles: tile k holds the
// rotations of sweep s at chain positions [k*TL + s, k*TL + s + TL), which
// touch the TL + BLK = WIN positions [k*TL, k*TL + WIN).  (Every family's
// sweep j rotates the chain positions 0 .. top(j), and the top rises by one
// from one sweep of a block to the next.)  The rotations of a tile multiply
// into one dense orthogonal WIN x WIN matrix Q (built in FP64 at plan time), so
// a block is a chain of tile products X <- Q X running down the column (hi2lo;
// Q^T running up for lo2hi), consecutive tiles overlapping in BLK positions.
// The X of a product is every column that needs the whole block, across all
// fields: that is what turns the sweeps into tensor-core work.  A column's
// sweeps above its last whole block (its "head", fewer than BLK sweeps) run in
// the direct rotation kernel, before the blocks in hi2lo and after them in
// lo2hi.
//
// Chains: a sph column is two chains (even and odd rows, rotations between
// rows k and k + 2); a disk or tri column is one chain (rows k and k + 1).  A
// task has two chain slots: the two chains of the same columns for sph, the
// same band of two groups of fields for disk and tri (whose tiles are the same
// for both slots and stored once).
//
// FP64 kernel: persistent CTAs over tasks (fields, parity, band), a band being
// the columns of BLK consecutive orders of one parity that need the same
// blocks; 8 warps, warps 0-3 do slot 0 and 4-7 slot 1 of each tile product as
// 32 x 32 DMMA (mma.m8n8k4.f64) tiles.  The WIN-position window of both slots
// stays in shared memory as a circular buffer (slot = position mod WIN), so
// the overlap rows never move.
#include <algorithm>
#include <cstdio>

#include <cuda_bf16.h>

#include "ft_internal.h"
#include "tc05.h"

namespace ftb {
namespace {

constexpr int BLK = 32;            // sweeps per block
constexpr int TL = 32;             // tile height (positions)
constexpr int WIN = BLK + TL;      // window (positions)
constexpr int FT = 2 * BLK;        // columns per task (BLK orders x cos, sin)
constexpr int LDQ = WIN + 4;       // padded rows of Q in shared memory
constexpr int LDX = FT + 1;        // padded rows of the window
constexpr int NT = 256;

// A task: fields field .. field + fields per task - 1, parity p, band >= 1 (orders of the
// band need blocks 0 .. band - 1; nb = min(band, blocks of the plan), the blocks above
// those hold no rotations), and its index in the task-major copy of the split-BF16 path.
struct BlkTask { int field, p, band, nb, slot; };

// Family-dependent shape of the blocked stage.
//   sph:  two chains (even / odd rows) of (N + 1) / 2 positions; sweeps j = p, p + 2, ...
//   disk: one chain (the column) of N positions; sweeps j = p, p + 2, ...
//   tri:  one chain (the column) of N positions; sweeps j = 0, 1, ...
// A band of a field: BLK orders of one parity, two columns each (cos, sin) for sph and
// disk, one for tri (src/drivers.c:94-110, 314-326, 414-430 for the column of an order).
struct Shape {
    int kind;
    __host__ __device__ bool two_chains() const { return kind == SPH; }
    __host__ __device__ int step() const { return kind == TRI ? 1 : 2; }
    __host__ __device__ int band_cols() const { return kind == TRI ? BLK : 2 * BLK; }
    __host__ __device__ int positions(int N) const { return kind == SPH ? (N + 1) / 2 : N; }
    // matrix row of chain position pos of chain c (also the sweep's table entry)
    __host__ __device__ int row(int pos, int c) const { return kind == SPH ? 2 * pos + c : pos; }
    // highest sweep of block beta of parity p
    __host__ __device__ int block_top(int p, int beta) const { return p + step() * BLK * (beta + 1) - step(); }
    // fields of one chain slot of a task `width` columns wide, and of the whole task
    __host__ __device__ int slot_fields(int width) const { return width / band_cols(); }
    __host__ __device__ int task_fields(int width) const { return slot_fields(width) * (two_chains() ? 1 : 2); }
    // column i of chain slot c of task t: its field f and matrix column, -1 past the last order
    __host__ __device__ long long column(const BlkTask & t, int width, int c, int i, int mlast, int & f) const {
        const int bc = band_cols();
        f = t.field + (two_chains() ? 0 : c * slot_fields(width)) + i / bc;
        const int n = i % bc;
        if (kind == TRI) {
            const int m = BLK * t.band + n;
            return m <= mlast ? m : -1;
        }
        const int m = t.p + 2 * BLK * t.band + 2 * (n >> 1);
        return m <= mlast ? 2LL * m - 1 + (n & 1) : -1;
    }
};

struct BlockedLaunch {
    double * A[kMaxFields];        // in place
    int nf;
    Shape sh;
    const double * Q;              // all tiles, row-major WIN x WIN each
    const long long * qbase;       // [2 parities][nbeta]: index of tile (c = 0, k = -1)
    const int * kmax;              // [2][nbeta]
    int nbeta;                     // blocks per parity slot
    int cq;                        // 1: one tile chain per slot (sph), 0: both slots share chain 0
    const BlkTask * tasks;
    int ntasks;
    int * counter;
    int N, M;
};

__device__ __forceinline__ void dmma(double & d0, double & d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// plan time: Q of every tile.  One CTA per (parity, block, chain, tile); the
// WIN columns of Q evolve independently under the rotations' row operations,
// one thread per column.  Rotation (s, c) on positions (i, i + 1) of the chain
// is the reference's Givens step (src/rotations/rotations_default.c:31-36, 45-50,
// 59-64), entry Geo::table_base(j) + row(i) of the packed tables.
// ---------------------------------------------------------------------------
__global__ void build_q_kernel(const double2 * __restrict__ sc, Shape sh, int N, int p, int beta, int c, double * Qout) {
    __shared__ double Q[WIN][WIN + 1];
    const int k = (int) blockIdx.x - 1;   // tiles k = -1 .. kmax
    const int col = threadIdx.x;
    for (int r = 0; r < WIN; ++r) Q[r][col] = r == col ? 1.0 : 0.0;
    const int j0 = sh.block_top(p, beta);
    const int T0 = Geo::top(sh.kind, N, j0, c);
    const int lo = k * TL;
    for (int s = 0; s < BLK; ++s) {
        const int j = j0 - sh.step() * s;
        const long long base = Geo::table_base(sh.kind, N, j);
        const int Ts = T0 + s;
        const int ihi = min(lo + s + TL - 1, Ts), ilo = max(lo + s, 0);
        for (int i = ihi; i >= ilo; --i) {
            const double2 v = sc[base + sh.row(i, c)];
            const int a = i - lo;
            const double x = Q[a][col], y = Q[a + 1][col];
            Q[a][col] = __fma_rn(v.y, x, __dmul_rn(v.x, y));
            Q[a + 1][col] = __fma_rn(v.y, y, -__dmul_rn(v.x, x));
        }
    }
    __syncthreads();
    double * out = Qout + (long long) blockIdx.x * WIN * WIN;
    for (int r = 0; r < WIN; ++r) out[(long long) r * WIN + col] = Q[r][col];
}

// ---------------------------------------------------------------------------
// the blocked products
// ---------------------------------------------------------------------------
template <bool HI2LO>
__global__ void __launch_bounds__(NT, 1) blocked_kernel(const __grid_constant__ BlockedLaunch L) {
    extern __shared__ double smem[];
    double * Qs = smem;                              // [2][WIN][LDQ]
    double * Xw = smem + 2 * WIN * LDQ;              // [WIN slots][2 chains][LDX]
    __shared__ int s_task;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c_w = warp >> 2;                       // chain of this warp
    const int wm = ((warp & 3) >> 1) * 32, wn = (warp & 1) * 32;
    const int fr = lane >> 2, fc = lane & 3;
    const int N = L.N, mlast = Geo::last_order(L.sh.kind, L.M);
    const Shape sh = L.sh;
    const bool two = sh.two_chains();

    for (;;) {
        if (tid == 0) s_task = atomicAdd(L.counter, 1);
        __syncthreads();
        const int t_id = s_task;
        __syncthreads();
        if (t_id >= L.ntasks) break;
        const BlkTask T = L.tasks[t_id];
        const int p = T.p;
        // column n of slot c: its matrix (null past the fields or the last order) and column
        auto col_of = [&](int c, int n, double *& A) -> long long {
            int f;
            const long long col = sh.column(T, FT, c, n, mlast, f);
            A = (col >= 0 && f < L.nf) ? L.A[f] : nullptr;
            return col;
        };
        for (int bi = 0; bi < T.nb; ++bi) {
            const int beta = HI2LO ? T.nb - 1 - bi : bi;
            const int kmax = L.kmax[p * L.nbeta + beta];
            const long long qb = L.qbase[p * L.nbeta + beta];
            const int nk = kmax + 2;
            for (int ki = 0; ki < nk; ++ki) {
                const int k = HI2LO ? kmax - ki : ki - 1;
                const int lo = k * TL;
                const bool first = ki == 0, last = ki == nk - 1;
                // positions entering the window: all of it for the first tile, else TL of them
                const int plo = first ? lo : (HI2LO ? lo : lo + BLK);
                const int pcnt = first ? WIN : TL;
                // load positions [plo, plo + pcnt) of both slots' FT columns
                for (int f = tid; f < FT * 2 * pcnt; f += NT) {
                    const int n = f / (2 * pcnt), r = f % (2 * pcnt);
                    const int c = two ? (r & 1) : r / pcnt;
                    const int pos = plo + (two ? (r >> 1) : r % pcnt);
                    const int row = sh.row(pos, c);
                    double * A;
                    const long long col = col_of(c, n, A);
                    double v = 0.0;
                    if (A && pos >= 0 && row < N) v = __ldcg(A + col * N + row);
                    Xw[((pos & (WIN - 1)) * 2 + c) * LDX + n] = v;
                }
                // both slots' Q for this tile (the same tile for one-chain families)
                for (int f = tid; f < 2 * WIN * WIN; f += NT) {
                    const int c = f / (WIN * WIN), e = f % (WIN * WIN);
                    const double * q = L.Q + (qb + (long long) c * L.cq * nk + (k + 1)) * WIN * WIN;
                    Qs[(c * WIN + e / WIN) * LDQ + e % WIN] = __ldg(q + e);
                }
                __syncthreads();
                // Y_c = op(Q_c) X_c on this warp's 32 x 32 block
                double acc[4][4][2];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
                const double * Qc = Qs + c_w * WIN * LDQ;
#pragma unroll 4
                for (int kk = 0; kk < WIN; kk += 4) {
                    double af[4], bf[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const int m = wm + a * 8 + fr, kq = kk + fc;
                        af[a] = HI2LO ? Qc[m * LDQ + kq] : Qc[kq * LDQ + m];
                    }
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int n = wn + b * 8 + fr, kq = kk + fc;
                        bf[b] = Xw[(((lo + kq) & (WIN - 1)) * 2 + c_w) * LDX + n];
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
                }
                __syncthreads();
                // outputs: final positions to global, the overlap back into the window
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int m = wm + a * 8 + fr;
                    const int pos = lo + m;
                    const bool fin = last || (HI2LO ? m >= BLK : m < TL);
                    const int row = sh.row(pos, c_w);
#pragma unroll
                    for (int b = 0; b < 4; ++b)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int n = wn + b * 8 + 2 * fc + h;
                            if (fin) {
                                double * A;
                                const long long col = col_of(c_w, n, A);
                                if (A && pos >= 0 && row < N) __stcg(A + col * N + row, acc[a][b][h]);
                            } else {
                                Xw[((pos & (WIN - 1)) * 2 + c_w) * LDX + n] = acc[a][b][h];
                            }
                        }
                }
                __syncthreads();
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Split-BF16 products on the tensor cores (tcgen05)
//
// The same block / tile decomposition, with every product computed from NS
// BF16 pieces per operand on the tensor cores with FP32 accumulation.  The
// pieces are fixed-point slices (the Ozaki splitting), not floating ones: a
// window column x (64 positions) is scaled by a power of two s so that
// |s x| < 2^8, and
//   s x = i_0 + i_1 2^-9 + ... + i_{NS-1} 2^-9(NS-1),   integers |i_a| <= 2^8,
// each rounded to nearest; a tile matrix entry (|q| <= 1) likewise with the
// fixed scale 2^8 (slices j_b).  Integers up to 2^8 are exact in BF16 (eight
// significant bits), every product i_a j_b is an integer of magnitude at most
// 2^16, and the products of one order level L = a + b go to their own FP32
// accumulator in tensor memory.  Levels L <= 3 are kept (NS = 3: eight
// products, NS = 4: ten); a level sums at most 4 x 64 such products, at most
// 2^24 in magnitude, so the accumulation is exact whatever rounding the tensor
// core applies.  The epilogue recombines
//   y = (A_0 + 2^-9 A_1 + ... ) 2^-8 / s
// in FP32 with round-to-nearest.  The errors are the slicing and the dropped
// levels (relative order 2^-9 NS of the window's largest entry and of the
// tile matrix entries, summed over the 64 products of a row) and the FP32
// rounding of y, all unbiased; a window position is carried between tiles as
// FP32, in global memory the matrix stays FP64.
//
// A task is two chain slots of 128 columns each: one band of two fields (sph,
// both chains), four fields (disk) or eight (tri).  The product is
// D^T = X^T op(Q)^T with M = 128 (columns), N = WIN (output positions),
// K = WIN (input positions), so each thread of the epilogue owns one column
// (its TMEM lane) and half of the window.  Warps 0-7 carry slot 0, warps 8-15
// slot 1, warp 16 issues the MMAs (one thread) and owns the TMEM allocation,
// warp 17 streams the tile images into shared memory, one buffer per slot.
// The slots alternate on the tensor cores, so one slot's epilogue runs while
// the other slot's products are in flight.
// ---------------------------------------------------------------------------
constexpr int MX_COLS = 128;                          // columns per task
constexpr int MX_PIECE = MX_COLS * WIN * 2;           // bytes of one BF16 piece of one chain's window
constexpr int MX_QPIECE = WIN * WIN * 2;              // bytes of one BF16 piece of one tile matrix
constexpr int MX_THREADS = 576;                       // 16 epilogue warps, MMA warp, loader warp
constexpr uint32_t MX_IDESC = tc::idesc_bf16(MX_COLS, WIN);
constexpr int MX_TMEM_COLS = 512;                     // 2 chains x 4 levels x WIN accumulator columns

template <int NS> struct MxCfg {
    static constexpr int QCHAIN = NS * MX_QPIECE;     // one chain's tile image
    // the positions entering the next window, per chain and buffer: 8 quads x MX_COLS columns
    // (FP32), bulk-copied one tile ahead where shared memory allows (three slices)
    static constexpr bool ROWS = NS == 3;
    static constexpr int ROWBUF = 8 * MX_COLS * 16;
    static constexpr size_t SMEM = 2 * NS * (size_t) MX_PIECE + 2 * (size_t) QCHAIN + (ROWS ? 4 * (size_t) ROWBUF : 0) + 1024;
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

// The blocked stage works on its own copy of the columns, task-major, in FP32:
// task (fields, parity, band) -> 2 slots x 128 columns, and element (slot c,
// position pos, column i) at ((c * Lq + pos / 4) * 128 + i) * 4 + pos % 4 of the
// task's part, with Lq position quads per slot.  A thread moves four
// consecutive positions of its column as one 16-byte access, and a warp (32
// adjacent columns) 512 contiguous bytes.  Positions past a chain's end hold
// zeros: the tile products never rotate them, so they stay zero.
struct MixedLaunch {
    float * T;                     // task-major copy of the columns (in place)
    int Lq;                        // position quads per slot in T
    const __nv_bfloat16 * img;     // tile images of the direction: [tile][slot chain][piece][WIN x WIN swizzled]
    const long long * qbase;       // [2][nbeta], as for the FP64 tiles
    const int * kmax;
    int nbeta;
    int cq;                        // 1: one tile chain per slot (sph), 0: both slots share chain 0
    const BlkTask * tasks;         // field: first field of the task
    int ntasks;
    int * counter;
    int * err;
    int N, M;
};

// Q of one (parity, block): every tile and chain into its NS-slice BF16 image
// (B[o][w] = Q[o][w] for hi2lo, Q[w][o] for lo2hi; rows o K-major, swizzled);
// tile k + 1 of chain c of the block is image qb + (k + 1) * nch + c.
template <int NS>
__global__ void build_img_kernel(const double * __restrict__ Q, long long qb, int nk, int nch, bool transpose,
                                 __nv_bfloat16 * __restrict__ img) {
    const int k1 = blockIdx.x, c = blockIdx.y;    // tile k = k1 - 1
    const double * q = Q + (qb + (long long) c * nk + k1) * WIN * WIN;
    unsigned char * out = reinterpret_cast<unsigned char *>(img) + (qb + (long long) k1 * nch + c) * (long long) MxCfg<NS>::QCHAIN;
    for (int e = threadIdx.x; e < WIN * WIN; e += blockDim.x) {
        const int o = e / WIN, w = e % WIN;
        // 256 q = j_0 + j_1 2^-9 + ..., integers |j| <= 2^8, stored negated (-j_b; a zero as +0)
        // because the window's slices are -i_a: the products (-i_a)(-j_b) are those of the slices
        double t = (transpose ? q[(long long) w * WIN + o] : q[e]) * 256.0;
        const uint32_t off = tc::sw128_offset(o, w);
        for (int b = 0; b < NS; ++b) {
            const double j = rint(t);
            *reinterpret_cast<__nv_bfloat16 *>(out + b * MX_QPIECE + off) = __float2bfloat16_rn(j == 0.0 ? 0.0f : (float) -j);
            t = (t - j) * 512.0;
        }
    }
}

// Power-of-two scale s with |s x| < 2^8 for every |x| <= amax (s = 1 for amax = 0).
__device__ __forceinline__ float slice_scale(float amax) {
    int E = (int) ((__float_as_uint(amax) >> 23) & 0xFF);   // amax < 2^(E - 126)
    if (E < 8) E = 8;                                         // tiny or zero windows
    return __uint_as_float((uint32_t) (261 - E) << 23);       // 2^(8 - (E - 126))
}

// Pairs of FP32 values in one 64-bit register, with sm_100's packed `.f32x2` arithmetic: each
// half is rounded exactly as the scalar instruction rounds it (round to nearest, subnormals kept),
// so a pair costs one instruction where two scalar ones gave the same bits.
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
    uint64_t d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ void f2_unpack(uint64_t d, float & lo, float & hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(d));
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// eight consecutive window positions, scaled by s (a power of two), -> NS 16-byte chunks of
// integer-valued BF16 slices, negated: s x = i_0 + i_1 2^-9 + ..., stored -i_a (the tile images
// hold -j_b, so every product keeps its sign).  Each cut is one FMA that scales and adds
// 1.5 * 2^23 (rounding to the nearest integer, |s x| < 2^8) and one subtraction from 1.5 * 2^23,
// which gives -i_a exactly; the residual is one FMA with that same -i_a (s x - i_0, 2^9 t - i_a:
// exact, |residual| <= 1/2 and a multiple of the operand's last place), the values those of
// rounding s x, subtracting and scaling in turn.  Two positions go through each instruction.
template <int NS>
__device__ __forceinline__ void slice8(const float * v, float s, uint4 * out) {
    constexpr float kMagic = 12582912.0f;         // 1.5 * 2^23
    const uint64_t magic = f2_pack(kMagic, kMagic), c512 = f2_pack(512.0f, 512.0f);
    uint32_t w[NS][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint64_t t = f2_pack(v[2 * q], v[2 * q + 1]), m = f2_pack(s, s);
#pragma unroll
        for (int a = 0; a < NS; ++a) {
            const uint64_t u = f2_fma(t, m, magic);
            const uint64_t ni = f2_sub(magic, u);
            float i0, i1;
            f2_unpack(ni, i0, i1);
            w[a][q] = tc::pack_bf16_ints(i0, i1);
            if (a + 1 < NS) {
                t = f2_fma(t, m, ni);
                m = c512;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < NS; ++a) out[a] = make_uint4(w[a][0], w[a][1], w[a][2], w[a][3]);
}

// NS slices per operand; products of levels 0 .. LV, one accumulator per level
template <bool HI2LO, int NS, int LV>
__global__ void __launch_bounds__(MX_THREADS, 1) blocked_mixed_kernel(const __grid_constant__ MixedLaunch L) {
    constexpr int QCHAIN = MxCfg<NS>::QCHAIN;
    constexpr int NL = LV + 1;                            // accumulators per chain
    static_assert(2 * NL * WIN <= MX_TMEM_COLS, "accumulators exceed tensor memory");
    extern __shared__ unsigned char smem_raw[];
    unsigned char * const sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    unsigned char * const Xs = sm;                        // [chain][piece]: MX_COLS rows x WIN slots
    unsigned char * const Qs = sm + 2 * NS * MX_PIECE;    // [chain]: the chain's tile image
    float4 * const Rs = reinterpret_cast<float4 *>(Qs + 2 * QCHAIN);   // [chain][buffer][quad][column]: entering positions
    constexpr bool ROWS = MxCfg<NS>::ROWS;
    __shared__ __align__(8) uint64_t bar_qfull[2], bar_qempty[2], bar_xready[2], bar_acc[2], bar_pmax[2], bar_block[2], bar_done;
    __shared__ __align__(8) uint64_t bar_rows[2][2];   // [chain][buffer]: entering positions landed
    __shared__ uint32_t s_tmem;
    __shared__ int s_task;
    __shared__ volatile int s_abort;
    __shared__ float s_pmax[2][2][MX_COLS];             // [chain][half][column]: largest window entry
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&bar_qfull[i], 1);
            tc::mbar_init(&bar_qempty[i], 1);
            tc::mbar_init(&bar_xready[i], 256);
            tc::mbar_init(&bar_pmax[i], 256);
            tc::mbar_init(&bar_block[i], 256);
            tc::mbar_init(&bar_acc[i], 1);
        }
        tc::mbar_init(&bar_done, 1);
        for (int i = 0; i < 4; ++i) tc::mbar_init(&bar_rows[i >> 1][i & 1], 1);
        s_abort = 0;
    }
    if (warp == 16) tc::tmem_alloc(&s_tmem, MX_TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;

    auto fail = [&]() {
        s_abort = 1;
        atomicExch(L.err, 1);
    };
    // per-role pipeline counters (identical traversal in every role)
    unsigned qt = 0;                 // tiles issued (loader) / consumed (MMA)
    unsigned xr[2] = {0, 0};         // x-ready phases consumed (MMA)
    unsigned ac = 0;                 // accumulator phases consumed (epilogue, own chain)
    unsigned pp = 0;                 // window-maximum exchanges (epilogue, own chain)
    unsigned bs = 0;                 // block boundaries passed (epilogue, own chain)
    int last_u = -1;                 // loader: last use of the chain buffers
    unsigned rk = 0;                 // entering-position copies of the own chain so far (epilogue, finishing half)
    unsigned rk_issued = 0;          // the same, issued (the chain's issuing thread)

    for (;;) {
        if (tid == 0) s_task = atomicAdd(L.counter, 1);
        __syncthreads();
        const int t_id = s_task;
        __syncthreads();
        if (t_id >= L.ntasks || s_abort) break;
        const BlkTask T = L.tasks[t_id];
        const int p = T.p, nb = T.nb;

        if (warp == 17) {
            // ---- tile images into shared memory, one buffer per chain ----
            if (lane == 0) {
                const int nch = 1 + L.cq;                 // tile chains stored per tile
                for (int bi = 0; bi < nb && !s_abort; ++bi) {
                    const int beta = HI2LO ? nb - 1 - bi : bi;
                    const int kmax = L.kmax[p * L.nbeta + beta];
                    const long long tb = L.qbase[p * L.nbeta + beta];
                    const unsigned char * const img0 = reinterpret_cast<const unsigned char *>(L.img) + tb * QCHAIN;
                    // the block's first tiles into L2 ahead of their copies
                    for (int ki = 0; ki < 2 && ki < kmax + 2; ++ki)
                        tc::prefetch_l2(img0 + (HI2LO ? kmax - ki + 1 : ki) * (long long) nch * QCHAIN, nch * QCHAIN);
                    for (int ki = 0; ki < kmax + 2 && !s_abort; ++ki, ++qt) {
                        const int k = HI2LO ? kmax - ki : ki - 1;
                        const int u = (int) qt;
                        const unsigned char * src = img0 + (k + 1) * (long long) nch * QCHAIN;
                        if (ki + 2 < kmax + 2)   // two tiles ahead
                            tc::prefetch_l2(img0 + (HI2LO ? k - 2 + 1 : k + 2 + 1) * (long long) nch * QCHAIN, nch * QCHAIN);
                        for (int c = 0; c < 2; ++c) {
                            if (!tc::mbar_wait(&bar_qempty[c], (u & 1) ^ 1, &s_abort)) { fail(); break; }
                            tc::mbar_arrive_expect_tx(&bar_qfull[c], QCHAIN);
                            tc::bulk_g2s(Qs + c * QCHAIN, src + c * L.cq * QCHAIN, QCHAIN, &bar_qfull[c]);
                        }
                        last_u = u;
                    }
                }
            }
            __syncwarp();
        } else if (warp == 16) {
            // ---- MMA issue ----
            if (lane == 0) {
                const uint32_t xs0 = tc::smem_addr(Xs), qs0 = tc::smem_addr(Qs);
                for (int bi = 0; bi < nb && !s_abort; ++bi) {
                    const int beta = HI2LO ? nb - 1 - bi : bi;
                    const int kmax = L.kmax[p * L.nbeta + beta];
                    for (int ki = 0; ki < kmax + 2 && !s_abort; ++ki, ++qt) {
                        const int k = HI2LO ? kmax - ki : ki - 1;
                        const int lo = k * TL;
                        const unsigned u = qt;
                        for (int c = 0; c < 2; ++c) {
                            if (!tc::mbar_wait(&bar_qfull[c], u & 1, &s_abort)) { fail(); break; }
                            if (!tc::mbar_wait(&bar_xready[c], xr[c] & 1, &s_abort)) { fail(); break; }
                            xr[c]++;
                            tc::fence_after_sync();
                            for (int kk = 0; kk < WIN / 16; ++kk) {
                                const uint32_t sc = (uint32_t) (((lo + 16 * kk) & (WIN - 1)) >> 4);
#pragma unroll
                                for (int lv = 0; lv <= LV; ++lv) {
                                    const int bmin = lv - (NS - 1) > 0 ? lv - (NS - 1) : 0;
                                    const int bmax = lv < NS - 1 ? lv : NS - 1;
#pragma unroll
                                    for (int b = bmin; b <= bmax; ++b) {
                                        const int a = lv - b;
                                        const uint64_t ad = tc::desc_sw128(xs0 + (c * NS + a) * MX_PIECE + sc * 32);
                                        const uint64_t bd = tc::desc_sw128(qs0 + c * QCHAIN + b * MX_QPIECE + kk * 32);
                                        // the level's first product of the tile starts its accumulator
                                        tc::mma_bf16(tmem + (c * NL + lv) * WIN, ad, bd, MX_IDESC, !(kk == 0 && b == bmin));
                                    }
                                }
                            }
                            tc::commit(&bar_acc[c]);
                            tc::commit(&bar_qempty[c]);
                        }
                    }
                }
            }
            __syncwarp();
        } else {
            // ---- epilogue: one column (TMEM lane) and half a window per thread ----
            // warps 8c .. 8c + 7 carry chain c; warp 8c + 4 hf + q owns TMEM lanes 32 q ..
            // and window offsets 32 hf .. 32 hf + 31
            const int c = warp >> 3;
            const int quarter = warp & 3, hf = (warp >> 2) & 1;
            const int r = 32 * quarter + lane;
            const int fh = HI2LO ? 1 : 0;                 // the half whose outputs leave the window
            // this column's quads: quad Q of the chain at Tq[Q * MX_COLS]
            float4 * const Tq = reinterpret_cast<float4 *>(L.T + T.slot * (8LL * L.Lq * MX_COLS)) +
                                (long long) c * L.Lq * MX_COLS + r;
            const int Pend = 4 * L.Lq;                    // positions held in the copy
            unsigned char * const xrow = Xs + c * NS * MX_PIECE;
            const uint32_t tacc = tmem + ((uint32_t) (quarter * 32) << 16) + c * NL * WIN + 32 * hf;
            float scale = 1.0f;   // slicing scale of the window the products in flight were computed from
            // 32 positions from pos0 (a multiple of 32): 8 quads, zero outside the copy
            // entering positions: one thread of the finishing half bulk-copies the 32 positions
            // from pos0 (a multiple of 32) for all MX_COLS columns, 8 quads x MX_COLS float4,
            // contiguous in the task-major copy, into buffer rk & 1 of the chain (fewer quads at the
            // end of the copy, none before its start); the half's threads read them back from there
            const bool issuer = ROWS && hf == fh && quarter == 0 && lane == 0;
            float4 * const Tq0 = Tq - r;                  // column 0 of this chain's quads
            auto issue_rows = [&](int pos0, unsigned idx) {
                const int q0 = pos0 >> 2;
                const int nq = pos0 < 0 ? 0 : max(0, min(8, L.Lq - q0));
                uint64_t * const bar = &bar_rows[c][idx & 1];
                asm volatile("fence.proxy.async.global;\n" ::: "memory");   // the positions were written through the generic proxy
                tc::mbar_arrive_expect_tx(bar, (uint32_t) (nq * MX_COLS * 16));
                if (nq > 0) tc::bulk_g2s(Rs + ((c * 2 + (idx & 1)) * 8) * MX_COLS, Tq0 + (long long) q0 * MX_COLS,
                                         (uint32_t) (nq * MX_COLS * 16), bar);
                rk_issued = idx + 1;
            };
            auto read_rows = [&](int pos0, unsigned idx, float * v) -> bool {
                if (!tc::mbar_wait(&bar_rows[c][idx & 1], (idx >> 1) & 1, &s_abort)) { fail(); return false; }
                const float4 * const buf = Rs + ((c * 2 + (idx & 1)) * 8) * MX_COLS + r;
#pragma unroll
                for (int qd = 0; qd < TL / 4; ++qd) {
                    const int P = pos0 + 4 * qd;
                    const float4 x = (P >= 0 && P < Pend) ? buf[qd * MX_COLS] : make_float4(0.f, 0.f, 0.f, 0.f);
                    v[4 * qd] = x.x; v[4 * qd + 1] = x.y; v[4 * qd + 2] = x.z; v[4 * qd + 3] = x.w;
                }
                return true;
            };
            auto load32 = [&](int pos0, float * v) {
#pragma unroll
                for (int qd = 0; qd < TL / 4; ++qd) {
                    const int P = pos0 + 4 * qd;
                    const float4 x = (P >= 0 && P < Pend) ? __ldcg(Tq + (long long) (P >> 2) * MX_COLS) : make_float4(0.f, 0.f, 0.f, 0.f);
                    v[4 * qd] = x.x; v[4 * qd + 1] = x.y; v[4 * qd + 2] = x.z; v[4 * qd + 3] = x.w;
                }
            };
            // 32 positions from pos0 (a multiple of 32), the values v times vs (a power of two),
            // into their window slots, with one scale for the whole window: the two halves
            // exchange their largest entries
            auto put32 = [&](int pos0, const float * v, float vs) -> bool {
                float m0 = 0.0f, m1 = 0.0f, m2 = 0.0f, m3 = 0.0f;
#pragma unroll
                for (int e = 0; e < TL; e += 4) {
                    m0 = fmaxf(m0, fabsf(v[e]));
                    m1 = fmaxf(m1, fabsf(v[e + 1]));
                    m2 = fmaxf(m2, fabsf(v[e + 2]));
                    m3 = fmaxf(m3, fabsf(v[e + 3]));
                }
                const float pm = fmaxf(fmaxf(m0, m1), fmaxf(m2, m3)) * vs;
                s_pmax[c][hf][r] = pm;
                tc::mbar_arrive(&bar_pmax[c]);
                if (!tc::mbar_wait(&bar_pmax[c], pp & 1, &s_abort)) { fail(); return false; }
                pp++;
                const float sc = slice_scale(fmaxf(pm, s_pmax[c][hf ^ 1][r]));
                scale = sc;
#pragma unroll
                for (int g = 0; g < TL / 8; ++g) {
                    uint4 ch[NS];
                    slice8<NS>(v + 8 * g, sc * vs, ch);
                    const uint32_t off = tc::sw128_offset(r, (pos0 + 8 * g) & (WIN - 1));
#pragma unroll
                    for (int a = 0; a < NS; ++a) *reinterpret_cast<uint4 *>(xrow + a * MX_PIECE + off) = ch[a];
                }
                tc::fence_async_smem();
                tc::fence_before_sync();
                tc::mbar_arrive(&bar_xready[c]);
                return true;
            };
            for (int bi = 0; bi < nb && !s_abort; ++bi) {
                const int beta = HI2LO ? nb - 1 - bi : bi;
                const int kmax = L.kmax[p * L.nbeta + beta];
                const int nk = kmax + 2;
                float src[TL];
                // the positions entering the second window (tile 0's), ahead of the first window
                auto enter_pos = [&](int kk) { const int lk = kk * TL; return HI2LO ? lk - TL : lk + WIN; };
                if (issuer && nk > 1) issue_rows(enter_pos(HI2LO ? kmax : -1), rk);
                {   // first tile: the whole window
                    const int pos0 = (HI2LO ? kmax : -1) * TL + TL * hf;
                    load32(pos0, src);
                    if (!put32(pos0, src, 1.0f)) break;
                }
                for (int ki = 0; ki < nk; ++ki) {
                    const int k = HI2LO ? kmax - ki : ki - 1;
                    const int lo = k * TL;
                    const bool last = ki == nk - 1;
                    const bool fin = last || hf == fh;    // this half's outputs leave the window
                    const int npos = HI2LO ? lo - TL : lo + WIN;
                    // the rows entering the tile after next into L2 (32 positions x 128 columns,
                    // contiguous in the task-major copy)
                    if (hf == fh && quarter == 0 && lane == 0 && ki + 2 < nk) {
                        const int ppos = HI2LO ? npos - TL : npos + TL;
                        const int qlo = ppos < 0 ? 0 : ppos >> 2;
                        const int qhi = min((ppos + TL) >> 2, L.Lq);
                        if (qhi > qlo) tc::prefetch_l2(Tq - r + (long long) qlo * MX_COLS, (uint32_t) (qhi - qlo) * MX_COLS * 16);
                    }
                    // the finishing half brings the positions entering the next tile (with ROWS,
                    // one tile ahead into shared memory, read back before the next window is cut)
                    if (ROWS) {
                        if (issuer && ki + 2 < nk) issue_rows(enter_pos(HI2LO ? k - 1 : k + 1), rk + 1);
                    } else if (!last && hf == fh) {
                        load32(npos, src);
                    }
                    if (!tc::mbar_wait(&bar_acc[c], ac & 1, &s_abort)) { fail(); break; }
                    ac++;
                    __syncwarp();
                    tc::fence_after_sync();
                    const float unscale = 0.00390625f / scale;    // 2^-8 / s, a power of two
                    const uint64_t c2m9 = f2_pack(0.001953125f, 0.001953125f), unscale2 = f2_pack(unscale, unscale);
#pragma unroll
                    for (int g = 0; g < TL / 8; ++g) {             // 8 window positions at a time
                        uint32_t a[NL][8];
#pragma unroll
                        for (int lv = 0; lv < NL; ++lv) tc::tmem_ld8_async(tacc + lv * WIN + 8 * g, a[lv]);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int hq = 0; hq < 2; ++hq) {           // one quad of positions at a time
                            // levels recombined highest first, y = 2^-9 y + A_lv, two positions a step
                            uint64_t y[2];
#pragma unroll
                            for (int e2 = 0; e2 < 2; ++e2) {
                                const int e = 4 * hq + 2 * e2;
                                y[e2] = f2_pack(__uint_as_float(a[NL - 1][e]), __uint_as_float(a[NL - 1][e + 1]));
#pragma unroll
                                for (int lv = NL - 2; lv >= 0; --lv)
                                    y[e2] = f2_fma(y[e2], c2m9, f2_pack(__uint_as_float(a[lv][e]), __uint_as_float(a[lv][e + 1])));
                            }
                            const int P = lo + TL * hf + 8 * g + 4 * hq;
                            if (fin) {
                                float4 o;
                                f2_unpack(f2_mul(y[0], unscale2), o.x, o.y);
                                f2_unpack(f2_mul(y[1], unscale2), o.z, o.w);
                                if (P >= 0 && P < Pend) __stcg(Tq + (long long) (P >> 2) * MX_COLS, o);
                            } else {   // kept unscaled: the window cut below applies unscale
                                float v[4];
                                f2_unpack(y[0], v[0], v[1]);
                                f2_unpack(y[1], v[2], v[3]);
#pragma unroll
                                for (int e = 0; e < 4; ++e) src[8 * g + 4 * hq + e] = v[e];
                            }
                        }
                    }
                    // next window: the overlap stays in its slots, the entering positions take
                    // the finished ones' slots
                    if (ROWS && !last && hf == fh) {
                        if (!read_rows(npos, rk, src)) break;
                        rk++;
                    }
                    if (!last && !put32(hf == fh ? npos : lo + TL * hf, src, hf == fh ? 1.0f : unscale)) break;
                }
                // block boundary: the next block's first window reads rows of global memory that
                // the other half of this chain's threads wrote
                asm volatile("fence.proxy.async.global;\n" ::: "memory");   // stores visible to the next block's bulk copies
                tc::mbar_arrive(&bar_block[c]);
                if (!tc::mbar_wait(&bar_block[c], bs & 1, &s_abort)) { fail(); break; }
                bs++;
            }
        }
    }

    // ---- teardown: nothing of this CTA may be in flight when TMEM is freed ----
    __syncthreads();
    __shared__ volatile int s_never;
    if (tid == 0) s_never = 0;
    __syncthreads();
    if (warp == 17 && lane == 0 && s_abort && last_u >= 0) {
        for (int c = 0; c < 2; ++c) (void) tc::mbar_wait(&bar_qfull[c], last_u & 1, &s_never);
    }
    if (ROWS && s_abort && lane == 0 && warp < 16 && (warp & 7) == 4 * (HI2LO ? 1 : 0)) {
        // a chain's issuing thread: its last two entering-position copies (one per buffer)
        for (unsigned i = rk_issued >= 2 ? rk_issued - 2 : 0; i < rk_issued; ++i)
            (void) tc::mbar_wait(&bar_rows[warp >> 3][i & 1], (i >> 1) & 1, &s_never);
    }
    if (warp == 16) {
        if (lane == 0) {
            tc::commit(&bar_done);
            if (!tc::mbar_wait(&bar_done, 0, &s_never)) atomicExch(L.err, 2);
        }
        __syncwarp();
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, MX_TMEM_COLS);
    }
}

struct BlockedPlan {
    int n = 0;
    Shape sh{SPH};
    int nch = 2;                // tile chains per block: 2 (sph), 1 (disk, tri)
    int npar = 2;               // parity slots: 2 (sph, disk), 1 (tri)
    int nbeta = 0;
    double * d_Q = nullptr;
    long long * d_qbase = nullptr;
    int * d_kmax = nullptr;
    std::vector<int> kmax;      // [npar][nbeta]
    std::vector<long long> qbase;
    long long ntiles = 0;       // tiles over all blocks and chains
    size_t bytes = 0;
    __nv_bfloat16 * d_img[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // tile images [3 or 4 slices][hi2lo, lo2hi]
    int * d_err = nullptr;      // set by a tensor-core kernel whose wait ran out
};

// last tile of block beta of parity p (chain 0, the longer one): tiles k = -1 .. kmax
int kmax_of(const Shape & sh, int N, int p, int beta) {
    const int T0 = Geo::top(sh.kind, N, sh.block_top(p, beta), 0);
    return T0 >= 0 ? T0 / TL : -1;
}

// blocks holding any rotation: block beta of parity p rotates something iff its lowest
// sweep does (the tops fall as j rises)
int blocks_of(const Shape & sh, int N, int npar) {
    int nb = 0;
    for (int p = 0; p < npar; p++) {
        int b = 0;
        while (Geo::top(sh.kind, N, sh.block_top(p, b) - sh.step() * (BLK - 1), 0) >= 0) b++;
        nb = std::max(nb, b);
    }
    return nb;
}

bool cuda_fine(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

int quads(const BlockedPlan * B, int N) { return (B->sh.positions(N) + 3) / 4; }

// Tasks (fields, parity, band >= 1) `width` columns per chain slot, longest first.
bool make_tasks(const BlockedPlan * B, int width, int nf, int M, BlkTaskList * out) {
    const Shape & sh = B->sh;
    const int mlast = Geo::last_order(sh.kind, M);
    const int fpt = sh.task_fields(width);
    std::vector<std::pair<long long, BlkTask>> v;
    for (int f = 0; f < nf; f += fpt)
        for (int p = 0; p < B->npar; p++)
            // band b holds the orders p + STEP BLK b + STEP o, o < BLK, which need blocks 0 .. b - 1
            for (int band = 1; p + sh.step() * BLK * band <= mlast; band++) {
                const int nb = std::min(band, B->nbeta);
                if (nb == 0) break;
                long long cost = 0;
                for (int beta = 0; beta < nb; beta++) cost += B->kmax[p * B->nbeta + beta] + 2;
                v.push_back({cost, BlkTask{f, p, band, nb, 0}});
            }
    std::stable_sort(v.begin(), v.end(), [](const auto & a, const auto & b) { return a.first > b.first; });
    std::vector<BlkTask> t;
    for (auto & x : v) {
        t.push_back(x.second);
        t.back().slot = (int) t.size() - 1;
    }
    out->ntasks = (int) t.size();
    if (t.empty()) return true;
    if (!cuda_fine(cudaMalloc(&out->d_tasks, sizeof(BlkTask) * t.size()), "cudaMalloc(blocked tasks)")) return false;
    return cuda_fine(cudaMemcpy(out->d_tasks, t.data(), sizeof(BlkTask) * t.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
}

int sm_count() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace

// Build (once) the tile matrices of a plan.
void * blocked_plan_build(HarmonicPlan * H) {
    const int N = H->n;
    BlockedPlan * B = new BlockedPlan();
    B->n = N;
    B->sh = Shape{H->kind};
    B->nch = B->sh.two_chains() ? 2 : 1;
    B->npar = B->sh.step();
    B->nbeta = blocks_of(B->sh, N, B->npar);
    const int slots = B->npar * std::max(1, B->nbeta);
    std::vector<long long> qbase(slots);
    B->kmax.assign(slots, -1);
    long long tiles = 0;
    for (int p = 0; p < B->npar; p++)
        for (int beta = 0; beta < B->nbeta; beta++) {
            const int km = kmax_of(B->sh, N, p, beta);
            B->kmax[p * B->nbeta + beta] = km;
            qbase[p * B->nbeta + beta] = tiles;
            tiles += (long long) B->nch * (km + 2);
        }
    B->bytes = (size_t) std::max(1LL, tiles) * WIN * WIN * sizeof(double);
    B->qbase = qbase;
    B->ntiles = tiles;
    const double2 * sc = H->rp_arr[0]->d_sc;
    bool ok = cuda_fine(cudaMalloc(&B->d_Q, B->bytes), "cudaMalloc(blocked Q)") &&
              cuda_fine(cudaMalloc(&B->d_qbase, sizeof(long long) * qbase.size()), "cudaMalloc") &&
              cuda_fine(cudaMalloc(&B->d_kmax, sizeof(int) * B->kmax.size()), "cudaMalloc") &&
              cuda_fine(cudaMemcpy(B->d_qbase, qbase.data(), sizeof(long long) * qbase.size(), cudaMemcpyHostToDevice), "cudaMemcpy") &&
              cuda_fine(cudaMemcpy(B->d_kmax, B->kmax.data(), sizeof(int) * B->kmax.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    for (int p = 0; ok && p < B->npar; p++)
        for (int beta = 0; ok && beta < B->nbeta; beta++) {
            const int km = B->kmax[p * B->nbeta + beta];
            for (int c = 0; c < B->nch; c++) {
                double * out = B->d_Q + (qbase[p * B->nbeta + beta] + (long long) c * (km + 2)) * WIN * WIN;
                build_q_kernel<<<km + 2, WIN>>>(sc, B->sh, N, p, beta, c, out);
                count_launch();
            }
            ok = cuda_fine(cudaGetLastError(), "build_q_kernel");
        }
    ok = ok && cuda_fine(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    if (!ok) {
        cudaFree(B->d_Q); cudaFree(B->d_qbase); cudaFree(B->d_kmax);
        delete B;
        return nullptr;
    }
    return B;
}

void blocked_plan_free(void * p) {
    BlockedPlan * B = static_cast<BlockedPlan *>(p);
    if (!B) return;
    cudaFree(B->d_Q); cudaFree(B->d_qbase); cudaFree(B->d_kmax);
    for (auto & im : B->d_img) { cudaFree(im[0]); cudaFree(im[1]); }
    cudaFree(B->d_err);
    delete B;
}

int blocked_block_size() { return BLK; }

// Blocked products over nf fields (in place) for one sweep direction.
cudaError_t launch_blocked(void * plan, bool hi2lo, double * const * A, int nf, int N, int M, const BlkTaskList & tl,
                           int * counter, cudaStream_t st) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    if (tl.ntasks == 0) return cudaSuccess;
    static thread_local BlockedLaunch L;
    for (int f = 0; f < nf; f++) L.A[f] = A[f];
    L.nf = nf;
    L.sh = B->sh;
    L.Q = B->d_Q;
    L.qbase = B->d_qbase;
    L.kmax = B->d_kmax;
    L.nbeta = B->nbeta;
    L.cq = B->nch - 1;
    L.tasks = reinterpret_cast<const BlkTask *>(tl.d_tasks);
    L.ntasks = tl.ntasks;
    L.counter = counter;
    L.N = N;
    L.M = M;
    const size_t shm = sizeof(double) * (2 * WIN * LDQ + WIN * 2 * LDX);
    auto kern = hi2lo ? blocked_kernel<true> : blocked_kernel<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    kern<<<std::min(sm_count(), tl.ntasks), NT, shm, st>>>(L);
    count_launch();
    return cudaGetLastError();
}

// FP64 tasks: FT columns per chain slot (one sph field, two disk fields, four tri fields per task).
bool blocked_tasks(void * plan, int nf, int N, int M, BlkTaskList * out) {
    (void) N;
    return make_tasks(static_cast<BlockedPlan *>(plan), FT, nf, M, out);
}

// Split-BF16 tile images with ns (3 or 4) slices, both directions (built once
// per plan and slice count, from the FP64 tiles).
bool blocked_mixed_prepare(void * plan, int ns) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    if (ns != 3 && ns != 4) { set_error(FT_B200_EINVAL, "slice count must be 3 or 4"); return false; }
    __nv_bfloat16 ** img = B->d_img[ns - 3];
    if (!B->d_err) {
        if (!cuda_fine(cudaMalloc(&B->d_err, sizeof(int)), "cudaMalloc")) return false;
        if (!cuda_fine(cudaMemset(B->d_err, 0, sizeof(int)), "cudaMemset")) return false;
    }
    if (img[0] && img[1]) return true;
    const size_t bytes = (size_t) std::max(1LL, B->ntiles) * (size_t) ns * MX_QPIECE;
    for (int d = 0; d < 2; d++) {
        if (img[d]) continue;
        void * p = nullptr;
        if (!cuda_fine(cudaMalloc(&p, bytes), "cudaMalloc(split tile images)")) return false;
        img[d] = static_cast<__nv_bfloat16 *>(p);
        for (int par = 0; par < B->npar; par++)
            for (int beta = 0; beta < B->nbeta; beta++) {
                const int nk = B->kmax[par * B->nbeta + beta] + 2;
                const long long qb = B->qbase[par * B->nbeta + beta];
                if (ns == 3) build_img_kernel<3><<<dim3(nk, B->nch), 256>>>(B->d_Q, qb, nk, B->nch, d == 1, img[d]);
                else         build_img_kernel<4><<<dim3(nk, B->nch), 256>>>(B->d_Q, qb, nk, B->nch, d == 1, img[d]);
                count_launch();
            }
        if (!cuda_fine(cudaGetLastError(), "build_img_kernel")) return false;
    }
    return cuda_fine(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
}

// Split-BF16 tasks: MX_COLS columns per chain slot (two sph, four disk, eight tri fields per task).
bool blocked_tasks_mixed(void * plan, int nf, int N, int M, BlkTaskList * out) {
    (void) N;
    return make_tasks(static_cast<BlockedPlan *>(plan), MX_COLS, nf, M, out);
}

cudaError_t launch_blocked_mixed(void * plan, int ns, bool hi2lo, float * T, int N, int M, const BlkTaskList & tl,
                                 int * counter, cudaStream_t st) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    if (tl.ntasks == 0) return cudaSuccess;
    static thread_local MixedLaunch L;
    L.T = T;
    L.Lq = quads(B, N);
    L.img = B->d_img[ns - 3][hi2lo ? 0 : 1];
    L.qbase = B->d_qbase;
    L.kmax = B->d_kmax;
    L.nbeta = B->nbeta;
    L.cq = B->nch - 1;
    L.tasks = reinterpret_cast<const BlkTask *>(tl.d_tasks);
    L.ntasks = tl.ntasks;
    L.counter = counter;
    L.err = B->d_err;
    L.N = N;
    L.M = M;
    // three slices: levels 0 .. 3 (eight products); four slices: levels 0 .. 3 (ten products)
    auto kern = ns == 3 ? (hi2lo ? blocked_mixed_kernel<true, 3, 3> : blocked_mixed_kernel<false, 3, 3>)
                        : (hi2lo ? blocked_mixed_kernel<true, 4, 3> : blocked_mixed_kernel<false, 4, 3>);
    const size_t smem = ns == 3 ? MxCfg<3>::SMEM : MxCfg<4>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    kern<<<std::min(sm_count(), tl.ntasks), MX_THREADS, smem, st>>>(L);
    count_launch();
    return cudaGetLastError();
}

// Elements of the task-major copy used by the split-BF16 products (ntasks from blocked_tasks_mixed).
size_t blocked_mixed_T_elems(void * plan, int ntasks, int N) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    return (size_t) std::max(1, ntasks) * 2 * (size_t) quads(B, N) * 4 * MX_COLS;
}

// S (the fields' FP64 matrices) <-> T (task-major FP32 copy of the columns the
// blocks apply to); one CTA per (task, 32 positions of both slots).
struct TransLaunch {
    double * A[kMaxFields];
    int nf, N, M, Lq;
    Shape sh;
    float * T;
    const BlkTask * tasks;
};

template <bool TO_T>
__global__ void __launch_bounds__(256) transpose_kernel(const __grid_constant__ TransLaunch L) {
    // [row of the chunk][column]; chunk row rr holds position pl = 0 .. 31 of the chunk in
    // slot c: rr = 2 pl + c (sph: the rows of the matrix in order) or 32 c + pl
    __shared__ float tile[64][MX_COLS + 1];
    const BlkTask t = L.tasks[blockIdx.x];
    const int q = blockIdx.y;                           // positions 32q .. 32q + 31
    const int tid = threadIdx.x;
    const int N = L.N, mlast = Geo::last_order(L.sh.kind, L.M);
    const bool two = L.sh.two_chains();
    float * const Tt = L.T + t.slot * (8LL * L.Lq * MX_COLS);
    // element (slot c, position pos, column i) of the task's copy
    auto at = [&](int c, int pos, int i) -> long long { return (((long long) c * L.Lq + (pos >> 2)) * MX_COLS + i) * 4 + (pos & 3); };
    auto chunk_row = [&](int c, int pl) -> int { return two ? 2 * pl + c : 32 * c + pl; };
    const int rr = tid & 63;
    const int c_r = two ? (rr & 1) : (rr >> 5), pl_r = two ? (rr >> 1) : (rr & 31);
    const int row = L.sh.row(32 * q + pl_r, c_r);        // matrix row of chunk row rr
    if (TO_T) {
        for (int i = tid >> 6; i < MX_COLS; i += 4) {
            int f;
            const long long col = L.sh.column(t, MX_COLS, c_r, i, mlast, f);
            tile[rr][i] = (col >= 0 && f < L.nf && row < N) ? (float) __ldcg(L.A[f] + col * N + row) : 0.0f;
        }
        __syncthreads();
        const int i = tid & (MX_COLS - 1);
        for (int e = tid >> 7; e < 16; e += 2) {       // e = 2 * (quad - 8q) + c
            const int c = e & 1, qd = e >> 1, Q = 8 * q + qd;
            if (Q < L.Lq) {
                const float4 v = make_float4(tile[chunk_row(c, 4 * qd)][i], tile[chunk_row(c, 4 * qd + 1)][i],
                                             tile[chunk_row(c, 4 * qd + 2)][i], tile[chunk_row(c, 4 * qd + 3)][i]);
                __stcg(reinterpret_cast<float4 *>(Tt + at(c, 4 * Q, i)), v);
            }
        }
    } else {
        const int i = tid & (MX_COLS - 1);
        for (int e = tid >> 7; e < 16; e += 2) {       // e = 2 * (quad - 8q) + c
            const int c = e & 1, qd = e >> 1, Q = 8 * q + qd;
            const float4 v = Q < L.Lq ? __ldcg(reinterpret_cast<const float4 *>(Tt + at(c, 4 * Q, i))) : make_float4(0.f, 0.f, 0.f, 0.f);
            tile[chunk_row(c, 4 * qd)][i] = v.x; tile[chunk_row(c, 4 * qd + 1)][i] = v.y;
            tile[chunk_row(c, 4 * qd + 2)][i] = v.z; tile[chunk_row(c, 4 * qd + 3)][i] = v.w;
        }
        __syncthreads();
        for (int i2 = tid >> 6; i2 < MX_COLS; i2 += 4) {
            int f;
            const long long col = L.sh.column(t, MX_COLS, c_r, i2, mlast, f);
            if (col >= 0 && f < L.nf && row < N) __stcg(L.A[f] + col * N + row, (double) tile[rr][i2]);
        }
    }
}

cudaError_t launch_blocked_transpose(void * plan, bool to_T, double * const * A, int nf, int N, int M, float * T,
                                     const BlkTaskList & tl, cudaStream_t st) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    if (tl.ntasks == 0) return cudaSuccess;
    static thread_local TransLaunch L;
    for (int f = 0; f < nf; f++) L.A[f] = A[f];
    L.nf = nf;
    L.N = N;
    L.M = M;
    L.sh = B->sh;
    L.Lq = quads(B, N);
    L.T = T;
    L.tasks = reinterpret_cast<const BlkTask *>(tl.d_tasks);
    const dim3 grid(tl.ntasks, (4 * L.Lq + 31) / 32);
    if (to_T) transpose_kernel<true><<<grid, 256, 0, st>>>(L);
    else      transpose_kernel<false><<<grid, 256, 0, st>>>(L);
    count_launch();
    return cudaGetLastError();
}

// Reads and clears the flag a tensor-core kernel sets when one of its waits ran out.
int blocked_device_error(void * plan) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    if (!B || !B->d_err) return 0;
    int v = 0;
    if (cudaMemcpy(&v, B->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (v) cudaMemset(B->d_err, 0, sizeof(int));
    return v;
}

}  // namespace ftb
