// Blocked rotation sweeps for fields that share one sph plan.
//
// The sweeps of a parity are cut into blocks of BLK consecutive sweeps on a
// fixed grid (block beta holds sweeps j = p + 2*BLK*beta + 2*BLK - 2 - 2s,
// s = 0 .. BLK-1), and each block into parallelogram tiles: tile k holds the
// rotations of sweep s at chain positions [k*TL + s, k*TL + s + TL), which
// touch the TL + BLK = WIN positions [k*TL, k*TL + WIN).  The rotations of a
// tile multiply into one dense orthogonal WIN x WIN matrix Q (built in FP64 at
// plan time), so a block is a chain of tile products X <- Q X running down the
// column (hi2lo; Q^T running up for lo2hi), consecutive tiles overlapping in
// BLK positions.  The X of a product is every column that needs the whole
// block, across all fields: that is what turns the sweeps into tensor-core
// work.  A column's sweeps above its last whole block (its "head", fewer than
// BLK sweeps) run in the direct rotation kernel, before the blocks in hi2lo
// and after them in lo2hi.
//
// Kernel: persistent CTAs over tasks (field, parity, band), a band being the
// 2*BLK columns of BLK consecutive orders that need the same blocks; 8 warps,
// warps 0-3 do chain 0 (even rows) and 4-7 chain 1 (odd rows) of each tile
// product as 32 x 32 DMMA (mma.m8n8k4.f64) tiles.  The WIN-position window of
// both chains stays in shared memory as a circular buffer (slot = position mod
// WIN), so the overlap rows never move.
#include <algorithm>
#include <cstdio>

#include "ft_internal.h"

namespace ftb {
namespace {

constexpr int BLK = 32;            // sweeps per block
constexpr int TL = 32;             // tile height (positions)
constexpr int WIN = BLK + TL;      // window (positions)
constexpr int FT = 2 * BLK;        // columns per task (BLK orders x cos, sin)
constexpr int LDQ = WIN + 4;       // padded rows of Q in shared memory
constexpr int LDX = FT + 1;        // padded rows of the window
constexpr int NT = 256;

struct BlkTask { int field, p, band; };

struct BlockedLaunch {
    double * A[kMaxFields];        // in place
    const double * Q;              // all tiles, row-major WIN x WIN each
    const long long * qbase;       // [2 parities][nbeta]: index of tile (c = 0, k = -1)
    const int * kmax;              // [2][nbeta]
    int nbeta;                     // blocks per parity slot
    const BlkTask * tasks;
    int ntasks;
    int * counter;
    int N, M;
};

__device__ __forceinline__ void dmma(double & d0, double & d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

__device__ __forceinline__ int top_sph(int N, int j, int c) {
    const int x = N - 3 - j - c;
    return x >= 0 ? x / 2 : -((1 - x) / 2);
}

// ---------------------------------------------------------------------------
// plan time: Q of every tile.  One CTA per (parity, block, chain, tile); the
// WIN columns of Q evolve independently under the rotations' row operations,
// one thread per column.
// ---------------------------------------------------------------------------
__global__ void build_q_kernel(const double2 * __restrict__ sc, int N, int p, int beta, int c, int kmax, double * Qout) {
    __shared__ double Q[WIN][WIN + 1];
    const int k = (int) blockIdx.x - 1;   // tiles k = -1 .. kmax
    const int col = threadIdx.x;
    for (int r = 0; r < WIN; ++r) Q[r][col] = r == col ? 1.0 : 0.0;
    const int j0 = p + 2 * BLK * beta + 2 * BLK - 2;
    const int T0 = top_sph(N, j0, c);
    const int lo = k * TL;
    for (int s = 0; s < BLK; ++s) {
        const int j = j0 - 2 * s;
        const long long base = (long long) j * (2 * N + 1 - j) / 2;
        const int Ts = T0 + s;
        const int ihi = min(lo + s + TL - 1, Ts), ilo = max(lo + s, 0);
        for (int i = ihi; i >= ilo; --i) {
            const double2 v = sc[base + 2 * i + c];
            const int a = i - lo;
            const double x = Q[a][col], y = Q[a + 1][col];
            Q[a][col] = __fma_rn(v.y, x, __dmul_rn(v.x, y));
            Q[a + 1][col] = __fma_rn(v.y, y, -__dmul_rn(v.x, x));
        }
    }
    __syncthreads();
    (void) kmax;
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
    const int N = L.N, mlast = L.M / 2;

    for (;;) {
        if (tid == 0) s_task = atomicAdd(L.counter, 1);
        __syncthreads();
        const int t_id = s_task;
        __syncthreads();
        if (t_id >= L.ntasks) break;
        const BlkTask T = L.tasks[t_id];
        double * const A = L.A[T.field];
        const int p = T.p, band = T.band;
        // task column n: order m = p + 2*BLK*band + 2*(n/2), column 2m - 1 + (n & 1)
        auto col_of = [&](int n, bool & ok) -> long long {
            const int m = p + 2 * BLK * band + 2 * (n >> 1);
            ok = m <= mlast;
            return 2LL * m - 1 + (n & 1);
        };
        for (int bi = 0; bi < band; ++bi) {
            const int beta = HI2LO ? band - 1 - bi : bi;
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
                // load rows [2*plo, 2*(plo + pcnt)) of the FT columns
                for (int f = tid; f < FT * 2 * pcnt; f += NT) {
                    const int n = f / (2 * pcnt), r = f % (2 * pcnt);
                    const int pos = plo + (r >> 1), c = r & 1;
                    const int row = 2 * pos + c;
                    bool ok;
                    const long long col = col_of(n, ok);
                    double v = 0.0;
                    if (ok && pos >= 0 && row < N) v = __ldcg(A + col * N + row);
                    Xw[((pos & (WIN - 1)) * 2 + c) * LDX + n] = v;
                }
                // both chains' Q for this tile
                for (int f = tid; f < 2 * WIN * WIN; f += NT) {
                    const int c = f / (WIN * WIN), e = f % (WIN * WIN);
                    const double * q = L.Q + (qb + (long long) c * nk + (k + 1)) * WIN * WIN;
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
                    const int row = 2 * pos + c_w;
#pragma unroll
                    for (int b = 0; b < 4; ++b)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int n = wn + b * 8 + 2 * fc + h;
                            if (fin) {
                                bool ok;
                                const long long col = col_of(n, ok);
                                if (ok && pos >= 0 && row < N) __stcg(A + col * N + row, acc[a][b][h]);
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

struct BlockedPlan {
    int n = 0;
    int nbeta = 0;
    double * d_Q = nullptr;
    long long * d_qbase = nullptr;
    int * d_kmax = nullptr;
    std::vector<int> kmax;      // [2][nbeta]
    size_t bytes = 0;
};

int kmax_of(int N, int p, int beta) {
    const int j0 = p + 2 * BLK * beta + 2 * BLK - 2;
    const int x = N - 3 - j0;
    const int T0 = x >= 0 ? x / 2 : -((1 - x) / 2);
    return T0 >= 0 ? T0 / TL : -1;
}

bool cuda_fine(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

}  // namespace

// Build (once) the tile matrices of a sph plan.
void * blocked_plan_build(HarmonicPlan * H) {
    const int N = H->n;
    BlockedPlan * B = new BlockedPlan();
    B->n = N;
    // blocks exist for sweeps j <= N - 3: beta with p + 2*BLK*beta + 2*BLK - 2 <= N - 3
    B->nbeta = std::max(0, (N - 1) / (2 * BLK));
    std::vector<long long> qbase(2 * std::max(1, B->nbeta));
    B->kmax.assign(2 * std::max(1, B->nbeta), -1);
    long long tiles = 0;
    for (int p = 0; p < 2; p++)
        for (int beta = 0; beta < B->nbeta; beta++) {
            const int km = kmax_of(N, p, beta);
            B->kmax[p * B->nbeta + beta] = km;
            qbase[p * B->nbeta + beta] = tiles;
            tiles += 2LL * (km + 2);
        }
    B->bytes = (size_t) std::max(1LL, tiles) * WIN * WIN * sizeof(double);
    const double2 * sc = H->rp_arr[0]->d_sc;
    bool ok = cuda_fine(cudaMalloc(&B->d_Q, B->bytes), "cudaMalloc(blocked Q)") &&
              cuda_fine(cudaMalloc(&B->d_qbase, sizeof(long long) * qbase.size()), "cudaMalloc") &&
              cuda_fine(cudaMalloc(&B->d_kmax, sizeof(int) * B->kmax.size()), "cudaMalloc") &&
              cuda_fine(cudaMemcpy(B->d_qbase, qbase.data(), sizeof(long long) * qbase.size(), cudaMemcpyHostToDevice), "cudaMemcpy") &&
              cuda_fine(cudaMemcpy(B->d_kmax, B->kmax.data(), sizeof(int) * B->kmax.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    for (int p = 0; ok && p < 2; p++)
        for (int beta = 0; ok && beta < B->nbeta; beta++) {
            const int km = B->kmax[p * B->nbeta + beta];
            for (int c = 0; c < 2; c++) {
                double * out = B->d_Q + (qbase[p * B->nbeta + beta] + (long long) c * (km + 2)) * WIN * WIN;
                build_q_kernel<<<km + 2, WIN>>>(sc, N, p, beta, c, km, out);
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
    L.Q = B->d_Q;
    L.qbase = B->d_qbase;
    L.kmax = B->d_kmax;
    L.nbeta = B->nbeta;
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
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ctas = std::min(sms, tl.ntasks);
    kern<<<ctas, NT, shm, st>>>(L);
    count_launch();
    return cudaGetLastError();
}

// Tasks (field, parity, band >= 1), longest first.
bool blocked_tasks(void * plan, int nf, int N, int M, BlkTaskList * out) {
    BlockedPlan * B = static_cast<BlockedPlan *>(plan);
    const int mlast = M / 2;
    std::vector<std::pair<long long, BlkTask>> v;
    for (int f = 0; f < nf; f++)
        for (int p = 0; p < 2; p++) {
            const int m0 = p == 0 ? 2 : 3;
            for (int band = 1; p + 2 * BLK * band <= mlast; band++) {
                if (p + 2 * BLK * band < m0) continue;
                if (band > B->nbeta) {   // cannot happen for M = 2N - 1; guards the tile tables
                    set_error(FT_B200_EINVAL, "column band beyond the plan's blocks");
                    return false;
                }
                long long cost = 0;
                for (int beta = 0; beta < band; beta++) cost += B->kmax[p * B->nbeta + beta] + 2;
                v.push_back({cost, BlkTask{f, p, band}});
            }
        }
    std::stable_sort(v.begin(), v.end(), [](const auto & a, const auto & b) { return a.first > b.first; });
    std::vector<BlkTask> t;
    for (auto & x : v) t.push_back(x.second);
    out->ntasks = (int) t.size();
    if (t.empty()) return true;
    if (!cuda_fine(cudaMalloc(&out->d_tasks, sizeof(BlkTask) * t.size()), "cudaMalloc(blocked tasks)")) return false;
    return cuda_fine(cudaMemcpy(out->d_tasks, t.data(), sizeof(BlkTask) * t.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
}

}  // namespace ftb
