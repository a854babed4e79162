// Givens-rotation sweeps (hi2lo / lo2hi) for the sph, tri and disk families on
// sm_100a, in FP64 with the reference's FMA arithmetic:
//   hi2lo: x' = fma(c, x, s*y),  y' = fma(c, y, -(s*x))
//   lo2hi: x' = fma(c, x, -(s*y)), y' = fma(c, y, s*x)
// (src/rotations/rotations_AVX512F.c:4-15; x is row k, y is row k+d).
//
// Work decomposition
// ------------------
// A task is a group of columns that receive the same sweeps (sph: 16 orders
// of one parity, cos and sin column each; disk: 32 orders of one parity, cos
// and sin each; tri: 32 consecutive orders).  Orders in a group differ, so a sweep j is applied to the columns
// whose order m satisfies j <= m - STEP and is an exact no-op (sin 0, cos 1)
// for the others.  Tasks are pulled from a longest-first queue by persistent
// CTAs (one per SM), which balances the triangular cost over orders.
//
// Inside a CTA the sweeps of a task run as a wavefront.  Warp q (a "stage")
// owns B consecutive sweeps.  Each lane owns one chain of the columns of one
// order and keeps, per column, a window of 2B consecutive chain positions in
// registers.  At every step the
// window slides by one position: one element enters, B independent rotations
// are applied (sweep b at window slots 2b, 2b+1), one element leaves.  The
// element leaving stage q is the element entering stage q+1 at the same step,
// passed through a shared-memory ring buffer.  All W warps share the global
// traffic: during each iteration every warp loads its share of the next
// chunk's column segments into registers (latency hidden behind the sweeps)
// and writes its share of the last stage's finished chunk back, so one pass of
// W*B sweeps reads and writes each column once.  The lanes of a warp that carry
// the same chain use the same (sin, cos) pair at each rotation, read as a
// broadcast 16-byte shared-memory load (two pairs per warp for two-chain kinds);
// each sweep's pairs of a chunk arrive in shared memory by one bulk copy from a
// padded table (identity pairs outside the sweep), issued one chunk ahead.
// With W = 8 warps every SM sub-partition holds two warps and the register
// budget per thread is the full 255.  In the pipelined configurations each pass
// of a task is a work unit of its own that streams behind the previous pass.
//
// Within a CTA no thread waits on another except through __syncthreads.  The
// one spin loop is the pass pipeline's wait on another CTA's progress word
// (pipelined configurations only), bounded, after which the launch records a
// device status and every later wait gives up.  Every global access is
// bounds-checked against the field's N, M.

#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include <map>
#include <mutex>
#include <tuple>
#include <string>

#include "ft_internal.h"
#include "tc05.h"

namespace ftb {
namespace {

template <int KIND>
struct KT {
    static constexpr int CH = (KIND == SPH || KIND == SPIN || KIND == RECT) ? 2 : 1;   // chains per column
    static constexpr int STEP = KIND == TRI ? 1 : 2;      // order step between sweeps
    // sequences per order sharing the rotations: cos, sin columns (sph, disk), the column
    // (tri, rect), or the real and imaginary parts of the columns of -m and m (spin)
    static constexpr int NCOL = (KIND == TRI || KIND == RECT) ? 1 : (KIND == SPIN ? 4 : 2);
    static constexpr int ES = KIND == SPIN ? 2 : 1;       // doubles per element (interleaved complex)
    static constexpr int ORD = 32 / CH;                   // orders per task (one lane per order and chain)
    static constexpr int COLS = ORD * NCOL;               // columns per task
    static constexpr int CPAD = COLS + 1;                 // padded column dimension of the stage buffers
};

// Builds the padded table (Geo::padded_col): block j fills column j's padded segment, blocks
// >= cols the identity rows at both ends.
__global__ void pad_table_kernel(const double2 * __restrict__ sc, double2 * __restrict__ out, int kind, int N) {
    const int cols = Geo::table_cols(kind, N), ch = Geo::chains(kind);
    const long long side = Geo::pad_side(kind);
    const double2 id = make_double2(0.0, 1.0);
    const int j = blockIdx.x;
    if (j >= cols) {   // the identity row before column 0, and the one after the last column
        double2 * row = j == cols ? out : out + Geo::padded_col(kind, N, cols - 1) + (Geo::table_base(kind, N, cols) -
                                                                                     Geo::table_base(kind, N, cols - 1)) + side;
        for (int e = threadIdx.x; e < Geo::kIdLen; e += blockDim.x) row[e] = id;
        return;
    }
    const long long len = Geo::table_base(kind, N, j + 1) - Geo::table_base(kind, N, j);
    const long long base = Geo::table_base(kind, N, j);
    double2 * col = out + Geo::padded_col(kind, N, j);
    for (long long l = -side + threadIdx.x; l < len + side; l += blockDim.x) {
        const bool valid = l >= 0 && l < len && (int) (l / ch) <= Geo::top(kind, N, j, (int) (l % ch));
        col[l] = valid ? sc[base + l] : id;
    }
}

__device__ __forceinline__ void rot_hi2lo(double & x, double & y, double s, double c) {
    const double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
    const double xn = __fma_rn(c, x, sy);
    const double yn = __fma_rn(c, y, -sx);
    x = xn; y = yn;
}
__device__ __forceinline__ void rot_lo2hi(double & x, double & y, double s, double c) {
    const double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
    const double xn = __fma_rn(c, x, -sy);
    const double yn = __fma_rn(c, y, sx);
    x = xn; y = yn;
}

// Status word of the rotation kernel: nonzero once a wait of the pass pipeline ran out
// (its output is then not valid).  Read and cleared by rotation_device_error().
__device__ int g_rot_status;

// Progress word of a pipeline unit: hi2lo, -X where every position >= X of its columns is
// final for the pass; lo2hi, X where every position <= X is final.  The launcher clears the
// words to a value below any position; a finished unit publishes INT_MAX.  Thread 0 publishes
// after a CTA barrier: the barrier orders every thread's stores of the chunk before its release,
// and a release is cumulative, so one thread's release covers the whole CTA's stores (the
// consumer's thread 0 acquires, then a barrier orders its CTA's loads after that).  A release
// reduction (max: the words only rise) does not hold the thread the way a fence does.
__device__ __forceinline__ void publish_progress(int * p, int v) {
    asm volatile("red.release.gpu.global.max.s32 [%0], %1;\n" :: "l"(p), "r"(v) : "memory");
}
// Waits until *p >= need and returns the value read; gives up after about 2^32 SM cycles,
// setting the status word, and at once when the word is already set (so one failed wait costs
// a launch about that long, not that long per unit).
__device__ __forceinline__ int wait_progress(const int * p, int need) {
    const long long t0 = clock64();
    for (;;) {
        int v;
        asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
        if (v >= need) return v;
        if (*(volatile int *) &g_rot_status != 0) return v;
        if (clock64() - t0 > (1LL << 32)) { atomicExch(&g_rot_status, 3); return v; }
        __nanosleep(128);
    }
}

// Lane layout: lane = o * CH + c owns chain c of the NCOL columns of order
// mbase + STEP * o (sph: cos and sin columns 2m-1, 2m; disk: the same pair;
// tri: column m; spin: the real and imaginary parts of the complex columns of
// orders -m and m, which share the sph sweeps of order |m - s|).  The NCOL columns
// of a lane share every (sin, cos) pair, so one shared-memory load feeds NCOL
// rotations.
template <int KIND, bool HI2LO, int W, int B, int E>
__global__ void __launch_bounds__(W * 32, W <= 4 ? 2 : 1)
rot_kernel(const __grid_constant__ RotLaunch L) {
    using T = KT<KIND>;
    constexpr int CH = T::CH, STEP = T::STEP, NCOL = T::NCOL, ORD = T::ORD, COLS = T::COLS, CPAD = T::CPAD, ES = T::ES;
    constexpr int WB = W * B;
    static_assert(E % (2 * B) == 0, "chunk must be a multiple of the window");
    static_assert((B * E * CH) % 32 == 0, "a chunk's (sin, cos) entries must split evenly over the lanes");
    extern __shared__ double smem[];
    // buffer q (0..W): input of stage q (q = W: output of the last stage), 2 slots,
    // element (step u, chain c, task column cl)
    auto buf = [&](int q, int slot, int u, int c) -> double * {
        return smem + ((((q * 2 + slot) * E + u) * CH + c) * CPAD);
    };
    // (sin, cos) pairs of the chunk a stage works on, staged one iteration ahead
    double2 * const sc_stage_base = reinterpret_cast<double2 *>(smem + (W + 1) * 2 * E * CH * CPAD);
    auto sc_stage = [&](int q, int slot) -> double2 * { return sc_stage_base + ((q * 2 + slot) * B) * (E * CH); };
    static_assert(E <= Geo::kPadPos, "the padded table must cover a chunk's overhang");
    static_assert(E * CH <= Geo::kIdLen, "the identity row must cover a chunk");
    __shared__ int s_task;
    __shared__ __align__(8) uint64_t s_mbar[W * 2];   // per stage and slot: its (sin, cos) staged

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp;                       // stage index
    const int o_lane = lane / CH, c_lane = lane % CH;
    if (threadIdx.x == 0) {
        for (int i = 0; i < W * 2; ++i) tc::mbar_init(&s_mbar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    uint32_t sc_phase = 0u;                   // bit s: parity of the next phase of this stage's mbarrier s
    uint32_t sc_live = 0u;                    // bit s: the chunk staged for slot s has a rotation (warp-uniform)

    const bool pipe = L.chains != nullptr;
    for (;;) {
        if (threadIdx.x == 0) s_task = atomicAdd(L.counter, 1);
        __syncthreads();
        const int tid = s_task;
        __syncthreads();
        if (tid >= (pipe ? L.nchains : L.ntasks)) break;
        // passes first, first + stride, .. of a task (pipeline), or all of its passes
        const RotChain chain = pipe ? L.chains[tid] : RotChain{tid, 0, 0, 1};
        const RotTask task = L.tasks[chain.task];
        const RotField & F = L.fields[task.field];
        const int N = F.N;
        const long long lda = F.lda;
        const int mlast = Geo::last_order(KIND, F.M);
        const int mbase = task.mbase;
        // lowest sweep of every column (spin: the parity of the effective orders |m - s|)
        const int jpar = KIND == TRI ? 0 : (KIND == SPIN ? ((mbase + F.spin) & 1) : (mbase & 1));
        // With F.blk > 0 a column of order m runs only its sweeps j >= jcut(m): the
        // (m - jpar)/STEP mod blk sweeps above its last whole block of blk sweeps.
        auto jcut = [&](int m) -> int {
            return F.blk > 0 ? m - STEP * (((m - jpar) / STEP) % F.blk) : jpar;
        };
        int jlo, jhi;
        const int nsw = Geo::task_sweeps(KIND, F.M, mbase, F.blk, &jlo, &jhi, F.spin);
        if (nsw == 0) continue;   // nothing to do for this task (uniform)
        const int npass = (nsw + WB - 1) / WB;
        if (chain.first >= npass || chain.stride < 1) {   // a schedule that does not match this launch shape
            if (threadIdx.x == 0) atomicExch(&g_rot_status, 4);
            continue;
        }
        const int m_lane = mbase + STEP * o_lane;
        const int jcut_lane = jcut(m_lane);
        // the order whose sweeps a lane runs: its own, or |m - s| for spin; emin: the least
        // over the task's orders (every sweep below emin - STEP applies to all lanes)
        const int me_lane = KIND == SPIN ? abs(m_lane - F.spin) : m_lane;
        int emin = mbase;
        if (KIND == SPIN) {
            emin = abs(mbase - F.spin);
            for (int o = 1; o < ORD; ++o) {
                const int m = mbase + STEP * o;
                if (m <= mlast) emin = min(emin, abs(m - F.spin));
            }
        }
        int jlo_all_max = jpar;   // highest first sweep over the task's columns
        if (F.blk > 0)
            for (int o = 0; o < ORD; ++o) {
                const int m = mbase + STEP * o;
                if (m <= mlast) jlo_all_max = max(jlo_all_max, jcut(m));
            }
        const int L0 = Geo::chain_len(KIND, N, 0);

        for (int r = chain.first; r < npass; r += chain.stride) {
            const double * src = r == 0 ? F.in : F.out;
            double * dst = F.out;
            const bool copy_all = r == 0 && F.in != F.out;
            // Passes of W*B sweeps; the one partial pass is the one with the shortest
            // sweeps (the first in hi2lo order, the last in lo2hi order), and only its
            // first WA stages run, so its cost scales with its sweeps.
            const int rem = nsw - (npass - 1) * WB;   // sweeps of the partial pass (1..WB)
            const int s0 = HI2LO ? (r == 0 ? 0 : rem + (r - 1) * WB) : r * WB;
            const int S = HI2LO ? (r == 0 ? rem : WB) : min(WB, nsw - s0);
            const int WA = (S + B - 1) / B;            // active stages
            const int WAB = WA * B;
            const int jfirst = HI2LO ? jhi - STEP * s0 : jlo + STEP * s0;
            int topc[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) topc[c] = Geo::top(KIND, N, jfirst, c);
            const int ref = HI2LO ? topc[0] : 0;
            int emax = HI2LO ? ref + S : topc[0] + 1;
            if (copy_all || emax > L0 - 1) emax = L0 - 1;
            if (emax < 0) emax = 0;
            const int tstart = HI2LO ? ref - emax : -1;
            const int tend = HI2LO ? ref + 2 * WAB : emax + 2 * WAB - 1;
            const int K = (tend - tstart + 1 + E - 1) / E;
            // pass pipeline: the previous pass's progress word and this pass's own
            const int * const prev_prog = (pipe && r > 0) ? L.prog + chain.prog0 + r - 1 : nullptr;
            int * const my_prog = pipe ? L.prog + chain.prog0 + r : nullptr;
            int seen = -0x7fffffff - 1;   // (thread 0) the predecessor's progress as last read

            // ---- stage state: per column a window of 2B chain positions ----
            double win[NCOL][2 * B];
#pragma unroll
            for (int h = 0; h < NCOL; ++h)
#pragma unroll
                for (int x = 0; x < 2 * B; ++x) win[h][x] = 0.0;
            // lane b < B: the padded-table column of sweep q*B + b and its last entry with a
            // rotation, or -1 where the sweep has none (beyond the pass, or a column with no
            // positions): the identity row
            long long my_col = -1;
            int my_lmax = -1;
            if (lane < B) {
                const int s = q * B + lane;
                const int j = HI2LO ? jfirst - STEP * s : jfirst + STEP * s;
                if (s < S && j >= 0 && j < Geo::table_cols(KIND, N)) {
#pragma unroll
                    for (int c = 0; c < CH; ++c) {
                        const int tc = Geo::top(KIND, N, j, c);
                        if (tc >= 0) my_lmax = max(my_lmax, CH * tc + c);
                    }
                    if (my_lmax >= 0) my_col = Geo::padded_col(KIND, N, j);
                }
            }
            const int jmax = HI2LO ? jfirst - STEP * (q * B) : jfirst + STEP * (q * B + B - 1);
            const int jmin = HI2LO ? jfirst - STEP * (q * B + B - 1) : jfirst + STEP * (q * B);
            // every sweep of this stage applies to every order of the task
            const bool full_lanes = jmax <= emin - STEP && (F.blk == 0 || jmin >= jlo_all_max);
            unsigned lane_mask = 0;                          // sweeps that apply to this lane's order
#pragma unroll
            for (int b = 0; b < B; ++b) {
                const int sg = q * B + b;
                const int j = HI2LO ? jfirst - STEP * sg : jfirst + STEP * sg;
                if (j <= me_lane - STEP && j >= jcut_lane) lane_mask |= 1u << b;
            }

            // Stage the (sin, cos) pairs of a chunk: entry (b, jj) is the pair sweep b uses at step
            // u of the chunk on chain c (jj = CH u + c, u reversed in hi2lo), i.e. the CH E
            // consecutive entries of its padded column starting at chain position ibase, where the
            // padding holds the identity (sin 0, cos 1) wherever the sweep has no rotation at that
            // step: every chunk runs the same straight-line code and those rotations are exact
            // no-ops.  One bulk copy per sweep (lanes 0 .. B-1) completes on the stage's mbarrier
            // for the slot.  A chunk in which none of the stage's sweeps has a rotation is not
            // staged at all: the stage passes its elements through unrotated (sc_live).
            auto prefetch_sc = [&](int kp) {
                const int t0p = tstart + kp * E;
                const int slot = kp & 1;
                double2 * const d = sc_stage(q, slot);
                uint64_t * const bar = &s_mbar[q * 2 + slot];
                int lo = 0;
                bool overlaps = false;
                if (lane < B) {
                    const int sg = q * B + lane;
                    lo = CH * (HI2LO ? ref + 2 * sg - t0p - E + 1 : t0p - 2 * sg);   // first entry
                    // a chunk overlapping the sweep's entries reaches at most E positions past
                    // them, into the padding; one outside them reads the identity row
                    overlaps = my_col >= 0 && lo <= my_lmax && lo + CH * E > 0;
                }
                const bool live = __ballot_sync(0xffffffffu, overlaps) != 0u;
                sc_live = live ? (sc_live | (1u << slot)) : (sc_live & ~(1u << slot));
                if (!live) return;
                if (lane == 0) tc::mbar_arrive_expect_tx(bar, (uint32_t) (B * E * CH * sizeof(double2)));
                __syncwarp();
                if (lane < B) {
                    const double2 * src = overlaps ? F.sc + my_col + lo : F.sc;
                    tc::bulk_g2s(d + lane * (E * CH), src, (uint32_t) (E * CH * sizeof(double2)), bar);
                }
            };
            // wait until the stage's (sin, cos) of chunk k have landed (bounded: a wait that runs out
            // sets the status word, and every later wait of the launch gives up at once)
            auto wait_sc = [&](int k) {
                const int slot = k & 1;
                if (!tc::mbar_wait(&s_mbar[q * 2 + slot], (sc_phase >> slot) & 1u, (volatile int *) &g_rot_status)) {
                    if (lane == 0) atomicCAS(&g_rot_status, 0, 5);
                }
                sc_phase ^= 1u << slot;
            };

            // ---- global traffic, shared by all warps: warp w moves elements
            //      v in [w*PER_W, (w+1)*PER_W) of each chunk (f = v*32 + lane) ----
            constexpr int RPC = E * CH;                // rows of one column segment per chunk
            constexpr int PER = COLS * RPC / 32;       // elements per lane per chunk (all warps)
            constexpr int PER_W = PER / W;             // this warp's share
            static_assert(PER % W == 0, "chunk must split evenly over the warps");
            double pre[PER_W];
            // Element v of this lane's share: task column cl and row offset rr inside
            // the chunk's contiguous row range (row = CH * pmin + rr).  Everything but
            // pmin is fixed for the pass, so it is computed once here.
            const double * gsrc[PER_W];
            double * gdst[PER_W];
            int ioff[PER_W];     // rr >> (CH - 1): position offset from pmin
            int rro[PER_W];      // rr: row offset from CH * pmin
            int soff[PER_W];     // shared-memory offset inside a slot
            bool colok[PER_W];
#pragma unroll
            for (int v = 0; v < PER_W; ++v) {
                const int f = (q * PER_W + v) * 32 + lane;
                const int cl = f / RPC, rr = f % RPC;
                const int o = cl / NCOL, h = cl % NCOL;
                const int mcl = mbase + STEP * o;
                long long coff;
                if constexpr (KIND == SPIN) {
                    // h: real / imaginary part (h & 1) of the column of -m (h < 2: 2m - 1, or 0
                    // for m = 0) or of m (2m)
                    const long long colc = h < 2 ? (mcl == 0 ? 0 : 2 * mcl - 1) : 2 * mcl;
                    colok[v] = mcl <= mlast && !(mcl == 0 && h >= 2) && colc < F.M;
                    coff = colok[v] ? ES * (colc * lda + rr) + (h & 1) : 0;
                } else {
                    const long long colc = (KIND == TRI || KIND == RECT) ? mcl : 2 * mcl - 1 + h;
                    colok[v] = mcl <= mlast;
                    coff = colok[v] ? colc * lda + rr : 0;
                }
                gsrc[v] = src + coff;
                gdst[v] = dst + coff;
                ioff[v] = CH == 2 ? (rr >> 1) : rr;
                rro[v] = rr;
                const int c = CH == 2 ? (rr & 1) : 0;
                const int u = HI2LO ? E - 1 - ioff[v] : ioff[v];
                soff[v] = (u * CH + c) * CPAD + cl;
            }
            // lowest chain position of chunk k entering stage 0 (storer: leaving stage W-1)
            auto pmin_of = [&](int k, bool storer) -> int {
                const int t0 = tstart + k * E;
                return HI2LO ? ref - t0 - E + 1 + (storer ? 2 * WAB : 0) : t0 + 1 - (storer ? 2 * WAB : 0);
            };
            auto row_ok = [&](int pmin, int v) -> bool {
                const int p = pmin + ioff[v];
                const int row = CH * pmin + rro[v];
                return colok[v] && p >= 0 && p <= emax && row < N;
            };
            // (thread 0) wait until the predecessor has finished the positions chunk k loads
            auto wait_chunk = [&](int k) {
                if (!prev_prog || k >= K) return;
                const int pmin = pmin_of(k, false), pmax = pmin + E - 1;
                if (pmax < 0 || pmin > emax) return;                 // nothing of the chunk is loaded
                // the predecessor publishes every few chunks and runs ahead: one acquire covers the
                // chunks up to the progress it read, which the words only ever raise
                const int need = HI2LO ? -max(pmin, 0) : min(pmax, emax);
                if (seen < need) seen = wait_progress(prev_prog, need);
            };
            auto load_chunk = [&](int k) {
                const int pmin = pmin_of(k, false);
#pragma unroll
                for (int v = 0; v < PER_W; ++v)
                    pre[v] = (k < K && row_ok(pmin, v)) ? __ldcg(gsrc[v] + (long long) ES * CH * pmin) : 0.0;
            };
            auto stash_chunk = [&](int k) {
                double * const b0 = buf(0, k & 1, 0, 0);
#pragma unroll
                for (int v = 0; v < PER_W; ++v) b0[soff[v]] = pre[v];
            };
            // the pass pipeline publishes progress every stored chunk for short columns, every
            // fourth for long ones (and after the last): a successor trailing by a few chunks more
            // loses little of a long pass, while a publish costs its CTA a fence and a release
            auto publishes = [&](int k) {
                const int m = F.N >= 2048 ? 3 : 0;
                return (k & m) == m || k == K - 1;
            };
            auto store_chunk = [&](int k) {
                const int pmin = pmin_of(k, true);
                const double * const bw = buf(WA, k & 1, 0, 0);
#pragma unroll
                for (int v = 0; v < PER_W; ++v)
                    if (row_ok(pmin, v)) __stcg(gdst[v] + (long long) ES * CH * pmin, bw[soff[v]]);
            };
            if (pipe) {
                if (threadIdx.x == 0) {
                    wait_chunk(0);
                    wait_chunk(1);
                    // hi2lo: positions above this pass's range are final once the predecessor
                    // has finished the first chunk's (they belong to earlier passes only)
                    publish_progress(my_prog, HI2LO ? -(emax + 1) : -1);
                }
                __syncthreads();
            }
            load_chunk(0);
            stash_chunk(0);
            if (q == 0) prefetch_sc(0);
            __syncthreads();

            for (int it = 0; it < K + WA; ++it) {
                // chunk it+1: loads in flight while the stages work on their chunks
                if (it + 1 < K) load_chunk(it + 1);
                // the last active stage finished chunk it-WA in the previous iteration
                if (it - WA >= 0 && it - WA < K) store_chunk(it - WA);
                // (sin, cos) of the chunk this stage works on next iteration
                if (q < WA && it + 1 - q >= 0 && it + 1 - q < K) prefetch_sc(it + 1 - q);
                const int k = it - q;
                if (q < WA && k >= 0 && k < K && !((sc_live >> (k & 1)) & 1u)) {
                    // no rotation of this stage in the chunk: the window only shifts, every element
                    // leaves the stage as it entered (the sequential loops do not touch them either)
                    const int slot = k & 1;
#pragma unroll
                    for (int u = 0; u < E; ++u) {
                        const int pn = u % (2 * B);
                        const double * bin = buf(q, slot, u, c_lane) + o_lane * NCOL;
                        double * bout = buf(q + 1, slot, u, c_lane) + o_lane * NCOL;
#pragma unroll
                        for (int h = 0; h < NCOL; ++h) {
                            const double in = bin[h];
                            bout[h] = win[h][pn];
                            win[h][pn] = in;
                        }
                    }
                } else if (q < WA && k >= 0 && k < K) {
                    const int slot = k & 1;
                    wait_sc(k);
                    const double2 * const scb = sc_stage(q, slot);
                    const bool masked = !full_lanes;
                    // two copies of the step loop: all sweeps apply to all lanes, or per-lane masks
                    auto run = [&](auto masked_tag) {
                        constexpr bool MASKED = decltype(masked_tag)::value;
#pragma unroll
                        for (int u = 0; u < E; ++u) {
                            // The window is circular: at step u, window position x lives in
                            // register slot (u - x) mod 2B.  The element leaving (position
                            // 2B-1 of the previous step) sits in slot u mod 2B, which the
                            // entering element (position 0) takes over.  E is a multiple of
                            // 2B, so the mapping is the same at every chunk boundary.
                            constexpr int W2 = 2 * B;
                            const int pn = u % W2;
                            const double * bin = buf(q, slot, u, c_lane) + o_lane * NCOL;
                            double * bout = buf(q + 1, slot, u, c_lane) + o_lane * NCOL;
#pragma unroll
                            for (int h = 0; h < NCOL; ++h) {
                                const double in = bin[h];
                                bout[h] = win[h][pn];
                                win[h][pn] = in;
                            }
                            const int obase = HI2LO ? (CH == 2 ? 2 * (E - 1 - u) : E - 1 - u) : (CH == 2 ? 2 * u : u);
#pragma unroll
                            for (int b = 0; b < B; ++b) {
                                const double2 sc = scb[b * (E * CH) + obase + (CH == 2 ? c_lane : 0)];
                                double sn = sc.x, cs = sc.y;
                                if (MASKED) {
                                    const bool on = (lane_mask >> b) & 1u;
                                    sn = on ? sn : 0.0;
                                    cs = on ? cs : 1.0;
                                }
                                const int xl = (u - 2 * b + 2 * W2) % W2;       // window position 2b
                                const int xu = (u - 2 * b - 1 + 2 * W2) % W2;   // window position 2b+1
#pragma unroll
                                for (int h = 0; h < NCOL; ++h) {
                                    if (HI2LO) rot_hi2lo(win[h][xl], win[h][xu], sn, cs);
                                    else       rot_lo2hi(win[h][xu], win[h][xl], sn, cs);
                                }
                            }
                        }
                    };
                    if (masked) run(std::true_type{});
                    else        run(std::false_type{});
                }
                if (it + 1 < K) stash_chunk(it + 1);
                if (pipe && threadIdx.x == 0) wait_chunk(it + 2);   // loaded next iteration
                __syncthreads();
                // the chunks stored up to this iteration are final: publish them
                if (pipe && threadIdx.x == 0 && it - WA >= 0 && it - WA < K && publishes(it - WA)) {
                    const int pmin = pmin_of(it - WA, true);
                    publish_progress(my_prog, HI2LO ? -pmin : pmin + E - 1);
                }
            }
            if (pipe && threadIdx.x == 0) publish_progress(my_prog, 0x7fffffff);
        }
    }
}

template <int KIND, bool HI2LO, int W, int B, int E>
cudaError_t launch_cfg(const RotLaunch & L, int max_ctas, cudaStream_t st) {
    constexpr int CH = KT<KIND>::CH, CPAD = KT<KIND>::CPAD;
    const size_t shm = sizeof(double) * (size_t) (W + 1) * 2 * E * CH * CPAD + sizeof(double2) * (size_t) W * 2 * B * E * CH;
    auto kern = rot_kernel<KIND, HI2LO, W, B, E>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 1;   // resident CTAs per SM (two for the four-warp shapes)
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, shm) != cudaSuccess || per_sm < 1) per_sm = 1;
    int ctas = sms * per_sm;
    if (max_ctas > 0 && ctas > max_ctas) ctas = max_ctas;
    const int work = L.chains ? L.nchains : L.ntasks;   // queue entries: pipeline entries or tasks
    if (ctas > work) ctas = work;
    if (ctas <= 0) return cudaSuccess;
    e = cudaMemsetAsync(L.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    kern<<<ctas, W * 32, shm, st>>>(L);
    count_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, kern);
        std::fprintf(stderr, "rot_kernel launch failed (%s): regs %d, static smem %zu, dyn smem %zu, max threads %d, params %zu B\n",
                     cudaGetErrorString(e), fa.numRegs, fa.sharedSizeBytes, shm, fa.maxThreadsPerBlock, sizeof(RotLaunch));
    }
    return e;
}

}  // namespace

// Configurations: W stage warps x B sweeps per warp, chunk E.
//   0: W = 8,  B = 8, E = 16 (255 registers, two warps per sub-partition)
//   1: W = 16, B = 4, E = 8  (128 registers, four warps per sub-partition)
//   2: W = 8,  B = 4, E = 8  (fewer sweeps per warp: lighter register pressure)
//   3: W = 8,  B = 4, E = 16
//   4: W = 4,  B = 4, E = 16 (two CTAs per SM)
//   5: W = 4,  B = 8, E = 16 (two CTAs per SM where shared memory allows: tri, disk)
template <int KIND, bool HI2LO>
cudaError_t launch_kind(int cfg, const RotLaunch & L, int max_ctas, cudaStream_t st) {
    if constexpr (KIND == SPIN) {
        (void) cfg;   // four sequences per lane: only 8 x 4 x 8 fits the stage buffers
        return launch_cfg<KIND, HI2LO, 8, 4, 8>(L, max_ctas, st);
    } else {
        if constexpr (KIND != TRI && KIND != RECT) {   // one sequence per lane: too few rows per warp
            if (cfg == 1) return launch_cfg<KIND, HI2LO, 16, 4, 8>(L, max_ctas, st);
        }
        if (cfg == 2) return launch_cfg<KIND, HI2LO, 8, 4, 8>(L, max_ctas, st);
        if (cfg == 3) return launch_cfg<KIND, HI2LO, 8, 4, 16>(L, max_ctas, st);
        if (cfg == 4) return launch_cfg<KIND, HI2LO, 4, 4, 16>(L, max_ctas, st);
        if (cfg == 5) return launch_cfg<KIND, HI2LO, 4, 8, 16>(L, max_ctas, st);
        return launch_cfg<KIND, HI2LO, 8, 8, 16>(L, max_ctas, st);
    }
}

int g_rot_cfg = -2;

// A configuration is a launch shape 0 .. 5 plus 8 x a pass-pipeline mode 0 .. 2
// (schedule_passes).  FT_B200_ROT_CFG forces one (as does ft_b200_set_rotation_config);
// otherwise -1 (chosen per launch shape).
constexpr int kPipeModes = 3;
bool valid_config(int cfg) { return cfg >= 0 && (cfg & 7) <= 5 && cfg < 8 * kPipeModes; }

int rotation_config() {
    if (g_rot_cfg == -2) {
        const char * e = std::getenv("FT_B200_ROT_CFG");
        const int v = e ? std::atoi(e) : -1;
        g_rot_cfg = (e && e[0] >= '0' && e[0] <= '9' && valid_config(v)) ? v : -1;
    }
    return g_rot_cfg;
}

void set_rotation_config(int cfg) { g_rot_cfg = valid_config(cfg) ? cfg : -1; }

struct RotSchedule {
    std::vector<RotTask> tasks;                          // host copy of the device list (same order)
    struct Units { RotChain * d_chains = nullptr; int * d_prog = nullptr; int n = 0, nprog = 0; };
    std::map<std::tuple<int, int, int>, Units> lists;    // (sweeps per pass, heads only, mode) -> queue
    std::mutex mu;
};

RotSchedule * rot_schedule_new(const std::vector<RotTask> & tasks) {
    RotSchedule * s = new RotSchedule();
    s->tasks = tasks;
    return s;
}

void rot_schedule_free(RotSchedule * s) {
    if (!s) return;
    for (auto & kv : s->lists) { cudaFree(kv.second.d_chains); cudaFree(kv.second.d_prog); }
    delete s;
}

bool rotation_plan_pad(ft_rotation_plan * RP) {
    if (RP->d_scp) { cudaFree(RP->d_scp); RP->d_scp = nullptr; }
    const long long len = Geo::padded_len(RP->kind, RP->n);
    cudaError_t e = cudaMalloc(&RP->d_scp, sizeof(double2) * len);
    if (e != cudaSuccess) {
        RP->d_scp = nullptr;
        set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string("cudaMalloc(padded table): ") + cudaGetErrorString(e));
        return false;
    }
    pad_table_kernel<<<Geo::table_cols(RP->kind, RP->n) + 2, 256>>>(RP->d_sc, RP->d_scp, RP->kind, RP->n);
    count_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        set_error(FT_B200_ECUDA, std::string("pad_table_kernel: ") + cudaGetErrorString(e));
        return false;
    }
    return true;
}

int rotation_device_error() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_rot_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_rot_status, &z, sizeof(int)) != cudaSuccess) return -1;
    }
    return v;
}

namespace {

// Sweeps per pass (W x B) of each launch shape.
int shape_pass(int cfg) {
    static const int wb[6] = {64, 64, 32, 32, 16, 32};
    return (cfg >= 0 && cfg < 6) ? wb[cfg] : 64;
}

// The queue of the pass pipeline for L's tasks with passes of wb sweeps, built on first use;
// null when the stream is capturing then (the upload synchronises) or on an allocation
// failure.  One entry per pass, pass-major (every task's pass r before any task's pass r + 1,
// tasks in list order, longest first), so a pass's predecessor is always pulled first: a
// pass rarely waits long for it, but consecutive passes of a task run far apart in time, so
// its columns leave L2 between them when the matrix is large.  (Splitting each task into a
// few entries that take every D-th pass side by side, which keeps the columns in L2, measured
// slower at every size: a CTA whose entry waits for its task's previous pass cannot take
// other work meanwhile.)
// mode 2 (bounded): pass-major over only the longest tasks whose columns fit in half the L2
// (so consecutive passes of a task still find them there), then every other task as one
// entry running all its passes, longest first: the long tasks no longer end the launch alone,
// and the short ones fill in at the end.
const RotSchedule::Units * schedule_passes(RotSchedule * S, int kind, const RotLaunch & L, int wb, int mode, cudaStream_t st) {
    const int blk = L.fields[0].blk;
    std::lock_guard<std::mutex> lk(S->mu);
    const auto key = std::make_tuple(wb, blk > 0 ? 1 : 0, mode);
    auto it = S->lists.find(key);
    if (it != S->lists.end()) return it->second.d_chains ? &it->second : nullptr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    const int nt = (int) S->tasks.size();
    std::vector<int> npass(nt, 0), prog0(nt, 0);
    int nprog = 0, maxp = 0;
    for (int t = 0; t < nt; ++t) {
        const RotTask & T = S->tasks[t];
        const RotField & F = L.fields[T.field];
        int jlo, jhi;
        const int nsw = Geo::task_sweeps(kind, F.M, T.mbase, F.blk, &jlo, &jhi, F.spin);
        npass[t] = (nsw + wb - 1) / wb;
        prog0[t] = nprog;
        nprog += npass[t];
        maxp = std::max(maxp, npass[t]);
    }
    // tasks pipelined pass by pass: all (mode 1), or the longest ones (the list is longest first)
    // whose columns fit in half the L2 (mode 2)
    int npipe = nt;
    if (mode == 2) {
        int dev = 0, l2 = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
        const int seqs = (kind == TRI || kind == RECT) ? 1 : (kind == SPIN ? 4 : 2);   // doubles per order and row
        const long long cols = (long long) Geo::task_orders(kind) * seqs;
        const long long foot = cols * (long long) L.fields[0].N * (long long) sizeof(double);
        npipe = (int) std::min<long long>(nt, std::max<long long>(1, (l2 / 2) / std::max<long long>(foot, 1)));
    }
    std::vector<RotChain> q;   // entry: pass r of task t alone (stride npass), or all of its passes
    for (int r = 0; r < maxp; ++r)
        for (int t = 0; t < npipe; ++t)
            if (r < npass[t]) q.push_back(RotChain{t, prog0[t], r, npass[t]});
    for (int t = npipe; t < nt; ++t)
        if (npass[t] > 0) q.push_back(RotChain{t, prog0[t], 0, 1});
    RotSchedule::Units U;
    U.n = (int) q.size();
    U.nprog = nprog;
    if (U.n > 0) {
        if (cudaMalloc(&U.d_chains, sizeof(RotChain) * q.size()) != cudaSuccess ||
            cudaMalloc(&U.d_prog, sizeof(int) * std::max(nprog, 1)) != cudaSuccess ||
            cudaMemcpy(U.d_chains, q.data(), sizeof(RotChain) * q.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(U.d_chains); cudaFree(U.d_prog);
            U = RotSchedule::Units{};
        }
    }
    S->lists[key] = U;
    return U.d_chains ? &S->lists[key] : nullptr;
}

cudaError_t launch_with(int kind, bool hi2lo, int cfg, const RotLaunch & L, int max_ctas, cudaStream_t st) {
    switch (kind) {
        case SPH:  return hi2lo ? launch_kind<SPH, true>(cfg, L, max_ctas, st) : launch_kind<SPH, false>(cfg, L, max_ctas, st);
        case TRI:  return hi2lo ? launch_kind<TRI, true>(cfg, L, max_ctas, st) : launch_kind<TRI, false>(cfg, L, max_ctas, st);
        case DISK: return hi2lo ? launch_kind<DISK, true>(cfg, L, max_ctas, st) : launch_kind<DISK, false>(cfg, L, max_ctas, st);
        case SPIN: return hi2lo ? launch_kind<SPIN, true>(cfg, L, max_ctas, st) : launch_kind<SPIN, false>(cfg, L, max_ctas, st);
        case RECT: return hi2lo ? launch_kind<RECT, true>(cfg, L, max_ctas, st) : launch_kind<RECT, false>(cfg, L, max_ctas, st);
    }
    return cudaErrorInvalidValue;
}

// One launch in configuration cfg: shape cfg & 7, through the pass pipeline in mode cfg >> 3
// (schedule_passes) when the task list has a schedule (else, and in mode 0, each CTA runs
// every pass of its tasks).  The progress words are the call's own (prog_call) when it has
// them, else the schedule's.
cudaError_t launch_shape(int kind, bool hi2lo, int cfg, const RotLaunch & L, int max_ctas, cudaStream_t st,
                         RotSchedule * sched, int * prog_call = nullptr, int prog_cap = 0) {
    const int shape = cfg & 7, mode = cfg >> 3;
    const RotSchedule::Units * U = (mode > 0 && sched) ? schedule_passes(sched, kind, L, shape_pass(shape), mode, st) : nullptr;
    // a call with words of its own too few for this queue runs whole tasks per CTA instead
    if (!U || (prog_call && U->nprog > prog_cap)) return launch_with(kind, hi2lo, shape, L, max_ctas, st);
    int * const prog = prog_call ? prog_call : U->d_prog;
    static thread_local RotLaunch P;
    P = L;
    P.chains = U->d_chains;
    P.nchains = U->n;
    P.prog = prog;
    const cudaError_t e = cudaMemsetAsync(prog, 0x80, sizeof(int) * U->nprog, st);   // below any position
    if (e != cudaSuccess) return e;
    return launch_with(kind, hi2lo, shape, P, max_ctas, st);
}

// Configuration without measurements: launches that run only the heads above whole
// blocks (blk > 0: fewer than blk sweeps per column, 2 blk - 2 per task at most) keep more
// stages busy with 4 sweeps per warp; full sweeps use 8 per warp.
int default_config(const RotLaunch & L) { return (L.nfields > 0 && L.fields[0].blk > 0) ? 3 : 0; }

// The autotuner's choices, by launch shape: family, direction, heads only or all sweeps,
// fields, tasks, and the first field's N and M (the tasks of a shape are the same).
std::mutex g_tune_mu;
std::map<std::string, int> g_tuned;

std::string shape_key(int kind, bool hi2lo, const RotLaunch & L) {
    char k[160];
    std::snprintf(k, sizeof k, "%d/%d/%d/%d/%d/%d/%d", kind, hi2lo ? 1 : 0, L.fields[0].blk > 0 ? 1 : 0, L.nfields,
                  L.ntasks, L.fields[0].N, L.fields[0].M);
    return k;
}

bool autotune_enabled() {
    static const bool on = [] {
        const char * e = std::getenv("FT_B200_AUTOTUNE");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Times every configuration once (after one untimed launch) with CUDA events on the
// launch stream, on a copy of L whose fields read and write only dead[f] (memory whose
// contents the caller no longer needs, at least the field's N x M at its leading
// dimension); returns the fastest, or -1 if a launch or an event failed.  The rotation
// kernel's cost does not depend on the values, and every configuration computes the same
// results bit for bit (each element meets its rotations in the same order).
int tune(int kind, bool hi2lo, const RotLaunch & L, double * const * dead, int max_ctas, cudaStream_t st,
         RotSchedule * sched, int * prog_call, int prog_cap) {
    static thread_local RotLaunch S;
    S = L;
    for (int f = 0; f < L.nfields; ++f) { S.fields[f].in = dead[f]; S.fields[f].out = dead[f]; }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return -1;
    }
    int best = -1;
    float best_ms = 0.0f;
    // every shape, each also through the pass pipeline when the list has a schedule (it
    // spreads a task's passes over SMs: worth it when there are few tasks, not when the
    // columns would leave L2 between passes)
    for (int cfg = 0; cfg < 8 * kPipeModes; ++cfg) {
        if ((cfg & 7) > 5 || ((kind == TRI || kind == RECT) && (cfg & 7) == 1)) continue;   // tri, rect: shape 1 not built
        if ((cfg >> 3) && !sched) continue;
        if (launch_shape(kind, hi2lo, cfg, S, max_ctas, st, sched, prog_call, prog_cap) != cudaSuccess) { best = -1; break; }
        if (cudaEventRecord(e0, st) != cudaSuccess) { best = -1; break; }
        if (launch_shape(kind, hi2lo, cfg, S, max_ctas, st, sched, prog_call, prog_cap) != cudaSuccess) { best = -1; break; }
        float ms = 0.0f;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) { best = -1; break; }
        if (best < 0 || ms < best_ms) { best = cfg; best_ms = ms; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace

cudaError_t launch_rotations(int kind, bool hi2lo, const RotLaunch & L, int max_ctas, cudaStream_t st,
                             double * const * dead, RotSchedule * sched, int * prog_call, int prog_cap) {
    if (L.ntasks <= 0) return cudaSuccess;
    int cfg = rotation_config();
    if (cfg < 0) {
        cfg = default_config(L);
        if (autotune_enabled() && L.nfields > 0) {
            const std::string key = shape_key(kind, hi2lo, L);
            int known = -1;
            {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                auto it = g_tuned.find(key);
                if (it != g_tuned.end()) known = it->second;
            }
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (known >= 0) {
                cfg = known;
            } else if (dead && cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
                const int t = tune(kind, hi2lo, L, dead, max_ctas, st, sched, prog_call, prog_cap);
                if (t >= 0) {
                    std::lock_guard<std::mutex> lk(g_tune_mu);
                    g_tuned[key] = t;
                    cfg = t;
                }
            }
        }
    }
    return launch_shape(kind, hi2lo, cfg, L, max_ctas, st, sched, prog_call, prog_cap);
}


}  // namespace ftb
