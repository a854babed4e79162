// Givens-rotation sweeps (hi2lo / lo2hi) for the sph, tri and disk families on
// sm_100a, in FP64 with the reference's FMA arithmetic:
//   hi2lo: x' = fma(c, x, s*y),  y' = fma(c, y, -(s*x))
//   lo2hi: x' = fma(c, x, -(s*y)), y' = fma(c, y, s*x)
// (src/rotations/rotations_AVX512F.c:4-15; x is row k, y is row k+d).
//
// Work decomposition
// ------------------
// A task is a group of 32 columns that receive the same sweeps (sph / disk:
// 16 orders of one parity, cos and sin column each; tri: 32 consecutive
// orders).  Orders in a group differ, so a sweep j is applied to the columns
// whose order m satisfies j <= m - STEP and is an exact no-op (sin 0, cos 1)
// for the others.  Tasks are pulled from a longest-first queue by persistent
// CTAs (one per SM), which balances the triangular cost over orders.
//
// Inside a CTA the sweeps of a task run as a wavefront.  Warp q (a "stage")
// owns B consecutive sweeps.  Each lane owns one column; per chain it keeps a
// window of 2B consecutive chain positions in registers.  At every step the
// window slides by one position: one element enters, B independent rotations
// are applied (sweep b at window slots 2b, 2b+1), one element leaves.  The
// element leaving stage q is the element entering stage q+1 at the same step,
// passed through a shared-memory ring buffer.  A loader warp streams the
// column segments of the next chunk from global memory into the first buffer
// and a storer warp writes the last buffer back, so one pass of W*B sweeps
// reads and writes each column once.  All lanes of a warp use the same
// (sin, cos) pair at each rotation, read as a warp-broadcast 16-byte load.
//
// No thread waits on another except through __syncthreads; there are no spin
// loops.  Every global access is bounds-checked against the field's N, M.

#include "ft_internal.h"

namespace ftb {
namespace {

template <int KIND>
struct KT {
    static constexpr int CH = KIND == SPH ? 2 : 1;        // chains per column
    static constexpr int STEP = KIND == TRI ? 1 : 2;      // order step between sweeps
    static constexpr int ORDERS = KIND == TRI ? 32 : 16;  // orders per task
};

constexpr int PAD = 33;   // padded lane dimension of the stage buffers (bank spread)

struct SweepInfo {
    long long tbase;   // packed-table offset of the sweep's column
    int j;             // order of the sweep
    int tlo[2], thi[2];   // steps at which the sweep has a valid position, per chain
};

__device__ __forceinline__ void rot_hi2lo(double & x, double & y, double s, double c) {
    double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
    double xn = __fma_rn(c, x, sy);
    double yn = __fma_rn(c, y, -sx);
    x = xn; y = yn;
}
__device__ __forceinline__ void rot_lo2hi(double & x, double & y, double s, double c) {
    double sy = __dmul_rn(s, y), sx = __dmul_rn(s, x);
    double xn = __fma_rn(c, x, -sy);
    double yn = __fma_rn(c, y, sx);
    x = xn; y = yn;
}

template <int KIND, bool HI2LO, int W, int B, int E>
__global__ void __maxnreg__(200)
rot_kernel(const __grid_constant__ RotLaunch L) {
    constexpr int CH = KT<KIND>::CH, STEP = KT<KIND>::STEP, ORD = KT<KIND>::ORDERS;
    constexpr int WB = W * B;
    static_assert(E % (2 * B) == 0, "chunk must be a multiple of the window");
    extern __shared__ double smem[];
    // buffer q (0..W): input of stage q (q = W: output of the last stage), 2 slots
    auto buf = [&](int q, int slot, int u, int c) -> double * {
        return smem + ((((q * 2 + slot) * E + u) * CH + c) * PAD);
    };
    __shared__ int s_task;
    __shared__ SweepInfo sweep_info[W * B];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool is_loader = warp == 0, is_storer = warp == W + 1;
    const int q = warp - 1;   // stage index for stage warps

    for (;;) {
        if (threadIdx.x == 0) s_task = atomicAdd(L.counter, 1);
        __syncthreads();
        const int tid = s_task;
        __syncthreads();
        if (tid >= L.ntasks) break;
        const RotTask task = L.tasks[tid];
        const RotField & F = L.fields[task.field];
        const int N = F.N;
        const long long lda = F.lda;
        const int mlast = Geo::last_order(KIND, F.M);
        const int mbase = task.mbase;
        int omax = mbase + STEP * (ORD - 1);
        if (omax > mlast) omax = mbase + STEP * ((mlast - mbase) / STEP);
        const int jlo = KIND == TRI ? 0 : (mbase & 1);
        const int jhi = omax - STEP;
        const int nsw = (jhi - jlo) / STEP + 1;
        const int npass = (nsw + WB - 1) / WB;

        // this lane's column (for the loader and storer, the lane index is a column too)
        const int m_lane = KIND == TRI ? mbase + lane : mbase + 2 * (lane >> 1);
        const int col_lane = KIND == TRI ? m_lane : 2 * m_lane - 1 + (lane & 1);
        const bool lane_ok = m_lane <= mlast;
        const int L0 = Geo::chain_len(KIND, N, 0);

        for (int r = 0; r < npass; ++r) {
            const double * src = r == 0 ? F.in : F.out;
            double * dst = F.out;
            const bool copy_all = r == 0 && F.in != F.out;
            const int s0 = r * WB;
            const int S = min(WB, nsw - s0);
            const int jfirst = HI2LO ? jhi - STEP * s0 : jlo + STEP * s0;
            int topc[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) topc[c] = Geo::top(KIND, N, jfirst, c);
            const int ref = HI2LO ? topc[0] : 0;
            int emax = HI2LO ? ref + S : topc[0] + 1;
            if (copy_all || emax > L0 - 1) emax = L0 - 1;
            if (emax < 0) emax = 0;
            const int tstart = HI2LO ? ref - emax : -1;
            const int tend = HI2LO ? ref + 2 * WB : emax + 2 * WB - 1;
            const int K = (tend - tstart + 1 + E - 1) / E;

            // ---- stage state ----
            double win[CH][2 * B];
#pragma unroll
            for (int c = 0; c < CH; ++c)
#pragma unroll
                for (int x = 0; x < 2 * B; ++x) win[c][x] = 0.0;
            // per sweep of this stage (lane b < B computes sweep q*B + b): order j,
            // table column base and valid step range per chain, kept in shared memory
            SweepInfo * const my = sweep_info + (is_loader || is_storer ? 0 : q * B);
            bool full_lanes = false;
            if (!is_loader && !is_storer) {
                if (lane < B) {
                    const int s = q * B + lane;
                    SweepInfo si;
                    si.j = HI2LO ? jfirst - STEP * s : jfirst + STEP * s;
                    const bool sv = s < S;
                    si.tbase = sv ? Geo::table_base(KIND, N, si.j) : 0;
#pragma unroll
                    for (int c = 0; c < CH; ++c) {
                        const int ts = HI2LO ? topc[c] + s : topc[c] - s;
                        if (HI2LO) { si.tlo[c] = ref + 2 * s - ts; si.thi[c] = ref + 2 * s; }
                        else       { si.tlo[c] = 2 * s;            si.thi[c] = 2 * s + ts; }
                        if (!sv || ts < 0) { si.tlo[c] = 1; si.thi[c] = 0; }   // empty
                    }
                    my[lane] = si;
                }
                __syncwarp();
                const int jmax = HI2LO ? jfirst - STEP * (q * B) : jfirst + STEP * (q * B + B - 1);
                full_lanes = jmax <= mbase - STEP;
            }

            // ---- loader: chunk k goes to slot k & 1 one iteration before stage 0 reads it ----
            constexpr int PER = (E * CH * 32) / 32;   // elements per lane per chunk
            double pre[PER];
            auto chunk_row = [&](int k, int rr, int & row, int & u, int & c, bool storer) -> bool {
                // rr: row offset within the chunk's contiguous row range; returns validity
                const int t0 = tstart + k * E;
                int pmin;
                if (HI2LO) pmin = ref - t0 - E + 1 + (storer ? 2 * WB : 0);
                else       pmin = t0 + 1 - (storer ? 2 * WB : 0);
                int p;
                if (CH == 2) { p = pmin + (rr >> 1); c = rr & 1; row = 2 * p + c; }
                else         { p = pmin + rr; c = 0; row = p; }
                u = HI2LO ? (pmin + E - 1 - p) : (p - pmin);
                return p >= 0 && p <= emax && row < N;
            };
            auto load_chunk = [&](int k, double * dstv) {
#pragma unroll
                for (int v = 0; v < PER; ++v) {
                    const int f = v * 32 + lane;
                    const int cl = f / (E * CH), rr = f % (E * CH);
                    int row, u, c;
                    const bool ok = chunk_row(k, rr, row, u, c, false);
                    const int mcl = KIND == TRI ? mbase + cl : mbase + 2 * (cl >> 1);
                    const int colc = KIND == TRI ? mcl : 2 * mcl - 1 + (cl & 1);
                    double val = 0.0;
                    if (ok && k < K && mcl <= mlast) val = __ldcg(src + (long long) colc * lda + row);
                    dstv[v] = val;
                }
            };
            auto store_pre = [&](int k, const double * v_) {
#pragma unroll
                for (int v = 0; v < PER; ++v) {
                    const int f = v * 32 + lane;
                    const int cl = f / (E * CH), rr = f % (E * CH);
                    int row, u, c;
                    chunk_row(k, rr, row, u, c, false);
                    buf(0, k & 1, u, c)[cl] = v_[v];
                }
            };
            if (is_loader) {
                load_chunk(0, pre);
                store_pre(0, pre);
            }
            __syncthreads();

            for (int it = 0; it < K + W; ++it) {
                if (is_loader) {
                    // chunk it+1: its loads are in flight while the stages work on chunk it
                    if (it + 1 < K) {
                        load_chunk(it + 1, pre);
                        store_pre(it + 1, pre);
                    }
                } else if (is_storer) {
                    const int k = it - W;
                    if (k >= 0 && k < K) {
#pragma unroll
                        for (int v = 0; v < PER; ++v) {
                            const int f = v * 32 + lane;
                            const int cl = f / (E * CH), rr = f % (E * CH);
                            int row, u, c;
                            const bool ok = chunk_row(k, rr, row, u, c, true);
                            const int mcl = KIND == TRI ? mbase + cl : mbase + 2 * (cl >> 1);
                            const int colc = KIND == TRI ? mcl : 2 * mcl - 1 + (cl & 1);
                            const double val = buf(W, k & 1, u, c)[cl];
                            if (ok && mcl <= mlast) __stcg(dst + (long long) colc * lda + row, val);
                        }
                    }
                } else {
                    const int k = it - q;
                    if (k >= 0 && k < K) {
                        const int t0 = tstart + k * E;
                        const int slot = k & 1;
                        bool mine = true;
                        const double2 * tpl = F.sc;
                        if (lane < B) {
                            const SweepInfo si = my[lane];
#pragma unroll
                            for (int c = 0; c < CH; ++c) mine = mine && t0 >= si.tlo[c] && t0 + E - 1 <= si.thi[c];
                            const int s = q * B + lane;
                            long long off;
                            if (HI2LO) off = (CH == 2) ? 2LL * (ref + 2 * s - t0) : (long long) (ref + 2 * s - t0);
                            else       off = (CH == 2) ? 2LL * (t0 - 2 * s) : (long long) (t0 - 2 * s);
                            tpl = F.sc + si.tbase + off;
                        }
                        const bool interior = full_lanes && __all_sync(0xffffffffu, mine);
                        if (interior) {
                            // table pointers at step t0 for every sweep of the stage
                            const double2 * tp[B];
#pragma unroll
                            for (int b = 0; b < B; ++b)
                                tp[b] = reinterpret_cast<const double2 *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(tpl), b));
#pragma unroll
                            for (int u = 0; u < E; ++u) {
#pragma unroll
                                for (int c = 0; c < CH; ++c) {
                                    const double in = buf(q, slot, u, c)[lane];
                                    const double out = win[c][2 * B - 1];
#pragma unroll
                                    for (int x = 2 * B - 1; x > 0; --x) win[c][x] = win[c][x - 1];
                                    win[c][0] = in;
                                    buf(q + 1, slot, u, c)[lane] = out;
                                }
#pragma unroll
                                for (int b = 0; b < B; ++b) {
#pragma unroll
                                    for (int c = 0; c < CH; ++c) {
                                        const int o = HI2LO ? (CH == 2 ? -2 * u + c : -u) : (CH == 2 ? 2 * u + c : u);
                                        const double2 sc = __ldg(tp[b] + o);
                                        if (HI2LO) rot_hi2lo(win[c][2 * b], win[c][2 * b + 1], sc.x, sc.y);
                                        else       rot_lo2hi(win[c][2 * b + 1], win[c][2 * b], sc.x, sc.y);
                                    }
                                }
                            }
                        } else {
#pragma unroll
                            for (int u = 0; u < E; ++u) {
                                const int t = t0 + u;
#pragma unroll
                                for (int c = 0; c < CH; ++c) {
                                    const double in = buf(q, slot, u, c)[lane];
                                    const double out = win[c][2 * B - 1];
#pragma unroll
                                    for (int x = 2 * B - 1; x > 0; --x) win[c][x] = win[c][x - 1];
                                    win[c][0] = in;
                                    buf(q + 1, slot, u, c)[lane] = out;
                                }
#pragma unroll
                                for (int b = 0; b < B; ++b) {
                                    const int s = q * B + b;
                                    const SweepInfo si = my[b];
                                    const bool lane_on = si.j <= m_lane - STEP;
#pragma unroll
                                    for (int c = 0; c < CH; ++c) {
                                        if (t >= si.tlo[c] && t <= si.thi[c]) {
                                            const int i = HI2LO ? ref + 2 * s - t : t - 2 * s;
                                            const int krow = CH == 2 ? 2 * i + c : i;
                                            const double2 sc = __ldg(F.sc + si.tbase + krow);
                                            const double sn = lane_on ? sc.x : 0.0;
                                            const double cs = lane_on ? sc.y : 1.0;
                                            if (HI2LO) rot_hi2lo(win[c][2 * b], win[c][2 * b + 1], sn, cs);
                                            else       rot_lo2hi(win[c][2 * b + 1], win[c][2 * b], sn, cs);
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
                __syncthreads();
            }
        }
        (void) lane_ok; (void) col_lane;
    }
}

template <int KIND, bool HI2LO, int W, int B, int E>
cudaError_t launch_cfg(const RotLaunch & L, int max_ctas, cudaStream_t st) {
    constexpr int CH = KT<KIND>::CH;
    const size_t shm = sizeof(double) * (size_t) (W + 1) * 2 * E * CH * PAD;
    auto kern = rot_kernel<KIND, HI2LO, W, B, E>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) shm);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int ctas = sms;
    if (max_ctas > 0 && ctas > max_ctas) ctas = max_ctas;
    if (ctas > L.ntasks) ctas = L.ntasks;
    if (ctas <= 0) return cudaSuccess;
    e = cudaMemsetAsync(L.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    kern<<<ctas, (W + 2) * 32, shm, st>>>(L);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

// Tuned configuration per family: W stage warps x B sweeps per warp, chunk E.
cudaError_t launch_rotations(int kind, bool hi2lo, const RotLaunch & L, int max_ctas, cudaStream_t st) {
    if (L.ntasks <= 0) return cudaSuccess;
    switch (kind) {
        case SPH:  return hi2lo ? launch_cfg<SPH, true, 8, 8, 16>(L, max_ctas, st) : launch_cfg<SPH, false, 8, 8, 16>(L, max_ctas, st);
        case TRI:  return hi2lo ? launch_cfg<TRI, true, 8, 8, 16>(L, max_ctas, st) : launch_cfg<TRI, false, 8, 8, 16>(L, max_ctas, st);
        case DISK: return hi2lo ? launch_cfg<DISK, true, 8, 8, 16>(L, max_ctas, st) : launch_cfg<DISK, false, 8, 8, 16>(L, max_ctas, st);
    }
    return cudaErrorInvalidValue;
}

int rotation_ctas_per_sm(int) { return 1; }

}  // namespace ftb
