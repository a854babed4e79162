// Internal declarations shared by the host plan code and the CUDA kernels.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ft_b200.h"

namespace ftb {

// SPIN: stage two of the spin-weighted sweeps (sph sweeps of order |m - |s|| on interleaved
// complex columns, both columns of an order in one lane; spin.cu).
// RECT: the Dunkl-Xu (rectangularised disk) sweeps: the sph sweep shape (rotations (k, k + 2),
// j = m - 2 .. m mod 2) on one column per order, column m for m = 2 .. M - 1.
enum Kind { SPH = 0, TRI = 1, DISK = 2, SPIN = 3, RECT = 4 };

// ---------------------------------------------------------------------------
// Rotation geometry.
//
// A column of the coefficient matrix is swept by Givens rotations G(k, k+d)
// (d = 2 for sph: rows of equal parity; d = 1 for tri and disk).  Splitting a
// sph column into its even and odd rows gives two independent "chains" in
// which every rotation couples neighbouring chain positions (i, i+1); tri and
// disk columns are a single chain.  Chain position i of chain c is row
// 2i + c (sph) or row i (tri, disk).
//
// Sweep j rotates positions (i, i+1) for i = 0 .. top(j, c).  Consecutive
// sweeps of one column differ by STEP in j (2 for sph and disk: orders keep
// their parity; 1 for tri) and their tops by exactly one position, the fact
// the wavefront schedule in rotations.cu is built on.
//   sph  (src/rotations/rotations_default.c:31-43):  top = floor((N-3-j-c)/2)
//   tri  (src/rotations/rotations_default.c:45-57):  top = N-2-j
//   disk (src/rotations/rotations_default.c:59-71):  top = N-2-floor((j+1)/2)
// Sine/cosine tables use the reference packings (src/rotations/rotations.h:6-10).
// ---------------------------------------------------------------------------
struct Geo {
    __host__ __device__ static inline int floordiv2(int x) { return x >= 0 ? x / 2 : -((1 - x) / 2); }
    __host__ __device__ static inline bool sphlike(int kind) { return kind == SPH || kind == SPIN || kind == RECT; }
    __host__ __device__ static inline int chains(int kind) { return sphlike(kind) ? 2 : 1; }
    __host__ __device__ static inline int step(int kind) { return kind == TRI ? 1 : 2; }
    __host__ __device__ static inline int top(int kind, int N, int j, int c) {
        if (sphlike(kind)) return floordiv2(N - 3 - j - c);
        if (kind == TRI) return N - 2 - j;
        return N - 2 - (j + 1) / 2;
    }
    // number of positions of chain c in a column of N rows
    __host__ __device__ static inline int chain_len(int kind, int N, int c) {
        return sphlike(kind) ? (N - c + 1) / 2 : N;
    }
    // packed table offset of column j (entry l of sweep j is at offset + l)
    __host__ __device__ static inline long long table_base(int kind, int N, int j) {
        if (kind == DISK) return (long long) j * N - (long long) (j / 2) * ((j + 1) / 2);
        return (long long) j * (2 * N + 1 - j) / 2;
    }
    __host__ __device__ static inline long long table_len(int kind, int N) {
        return kind == DISK ? (long long) N * N : (long long) N * (N + 1) / 2;
    }
    // Padded copy of the table, read by the rotation kernel's bulk copies: an identity row of
    // kIdLen pairs (sin 0, cos 1), then every column j of the packed table with kPadPos chain
    // positions of identity pairs on each side, then another identity row.  Inside a column,
    // entry l is the packed entry where the sweep has a rotation (0 <= l / CH <= top(j, l % CH)),
    // the identity elsewhere, so a chunk of consecutive positions that overlaps the sweep's
    // entries can be copied without a range check (kPadPos >= the chunk length E); a chunk
    // entirely outside them is copied from an identity row.
    static constexpr int kPadPos = 16;
    static constexpr int kIdLen = 64;
    __host__ __device__ static inline int table_cols(int kind, int N) { return kind == DISK ? 2 * N - 1 : N; }
    __host__ __device__ static inline long long pad_side(int kind) { return (long long) kPadPos * chains(kind); }
    // offset of entry l = 0 of column j in the padded table
    __host__ __device__ static inline long long padded_col(int kind, int N, int j) {
        return kIdLen + table_base(kind, N, j) + (2LL * j + 1) * pad_side(kind);
    }
    __host__ __device__ static inline long long padded_len(int kind, int N) {
        return 2LL * kIdLen + table_len(kind, N) + 2LL * table_cols(kind, N) * pad_side(kind);
    }
    // number of order columns the rotation stage visits for an N x M matrix
    // sph / disk: pairs (2m-1, 2m), m = 2 .. M/2; tri: column m, m = 1 .. M-1
    __host__ __device__ static inline int first_order(int kind) { return kind == TRI ? 1 : (kind == SPIN ? 0 : 2); }
    // orders per rotation task: one lane per (order, chain) of a 32-lane warp
    __host__ __device__ static inline int task_orders(int kind) { return sphlike(kind) ? 16 : 32; }
    __host__ __device__ static inline int last_order(int kind, int M) { return (kind == TRI || kind == RECT) ? M - 1 : M / 2; }
    // Sweeps of the rotation task of lowest order mbase: every sweep j = jlo, jlo + step, ..,
    // jhi applies to at least one of its columns (order m runs j = jpar .. m - step; with
    // blk > 0 only its sweeps above its last whole block of blk sweeps).  Returns their number
    // (0: nothing to do).  The kernel and the host's pass schedule both use this.
    // SPIN: order m runs the sph sweeps of order |m - spin|, j = (m + spin) mod 2 .. |m - spin| - 2.
    __host__ __device__ static inline int task_sweeps(int kind, int M, int mbase, int blk, int * jlo_out, int * jhi_out,
                                                      int spin = 0) {
        const int st = step(kind), ord = task_orders(kind), mlast = last_order(kind, M);
        int omax = mbase + st * (ord - 1);
        if (omax > mlast) omax = mbase + st * ((mlast - mbase) / st);
        if (kind == SPIN) {
            int emax = 0;   // largest effective order of the task
            for (int m = mbase; m <= omax; m += st) emax = (m - spin > emax) ? m - spin : (spin - m > emax ? spin - m : emax);
            const int jlo = (mbase + spin) & 1, jhi = emax - st;
            *jlo_out = jlo;
            *jhi_out = jhi;
            return jhi < jlo ? 0 : (jhi - jlo) / st + 1;
        }
        const int jpar = kind == TRI ? 0 : (mbase & 1);
        int jlo = jpar;
        if (blk > 0) {
            jlo = mbase - st * (((mbase - jpar) / st) % blk);
            for (int o = 1; o < ord; ++o) {
                const int m = mbase + st * o;
                if (m > mlast) break;
                const int c = m - st * (((m - jpar) / st) % blk);
                if (c < jlo) jlo = c;
            }
        }
        const int jhi = omax - st;
        *jlo_out = jlo;
        *jhi_out = jhi;
        return jhi < jlo ? 0 : (jhi - jlo) / st + 1;
    }
};

// A unit of work of the rotation kernel: the columns of task_orders(kind)
// orders that share their sweeps.  sph: 16 orders of one parity, m = mbase + 2*o,
// two columns each; disk: 32 orders of one parity, two columns each; tri: 32
// consecutive orders m = mbase + o.
struct RotTask {
    int field;   // index into the field table of the launch
    int mbase;   // lowest order of the group
};

// One coefficient matrix of a launch.
struct RotField {
    const double * in;      // first pass reads here
    double * out;           // every pass writes here (in == out allowed)
    const double2 * sc;     // the padded (sin, cos) table of the field's rotation plan (Geo::padded_col)
    int N, M, kind;
    long long lda;
    int blk;                // 0: all sweeps; > 0: only each column's sweeps above the last
                            // whole block of blk sweeps (the rest run as blocked products)
    int spin;               // SPIN: |s|
};

// Kernel launchers (rotations.cu).  The field table travels by value in the
// kernel parameters (kept under the classic 4 KB parameter limit).
constexpr int kMaxFields = 64;
struct RotLaunch {
    RotField fields[kMaxFields];
    int nfields;
    const RotTask * tasks;     // device, longest first
    int ntasks;
    int * counter;             // device work counter (reset by the launcher)
    // Pass pipeline (null chains: each CTA runs every pass of a task itself).  Queue entry c
    // runs passes first, first + stride, ... of task chains[c].task (the launcher queues one
    // pass per entry); pass r streams down the columns behind pass r - 1 of the same task,
    // pulled earlier from the queue, waiting on that pass's progress word prog[prog0 + r - 1]
    // and publishing its own, prog[prog0 + r] (cleared by the launcher).
    const struct RotChain * chains;
    int nchains;
    int * prog;
};
struct RotChain { int task, prog0, first, stride; };
// Host side of the pass pipeline of one task list: the host copy of the device list (same
// order) and the unit lists built from it per pass length and head mode (rotations.cu).
struct RotSchedule;
RotSchedule * rot_schedule_new(const std::vector<RotTask> & tasks);
void rot_schedule_free(RotSchedule * s);
int rotation_device_error();   // reads and clears the rotation kernel's status word (-1: read failed)
// dead: per field, memory the caller has no live data in (N x M at the field's leading
// dimension), or null.  With it, the first launch of a shape times every configuration
// there and keeps the fastest for the shape (the autotuner; FT_B200_AUTOTUNE=0 turns it off).
// sched: the task list's schedule (null: no pass pipeline).  prog_call: progress words of the
// calling execute (prog_cap of them) for the pass pipeline instead of the schedule's own, so
// that concurrent calls on one plan do not share them; a queue needing more runs without the
// pipeline.
cudaError_t launch_rotations(int kind, bool hi2lo, const RotLaunch & L, int max_ctas, cudaStream_t st,
                             double * const * dead = nullptr, RotSchedule * sched = nullptr,
                             int * prog_call = nullptr, int prog_cap = 0);
void set_rotation_config(int cfg);   // 0 .. 3 forces a configuration, -1 chooses per shape
// (Re)builds RP->d_scp from RP->d_sc (call after every change of d_sc; synchronous)
bool rotation_plan_pad(ft_rotation_plan * RP);

// Triangular multiplies (trmm.cu).  Out = op(U) * In on column classes.
struct TrmmClass {
    const double * U;     // n x n upper triangular, column-major, ld = n
    const double * in;    // first column of the class
    double * out;
    int ncols;            // columns in the class
};
struct TrmmLaunch {
    TrmmClass cls[4];
    int nclasses;
    int n;
    long long ld_in, ld_out;   // column stride within a class (4N for sph/disk, N for tri)
    bool trans;                // op(U) = U^T
};
cudaError_t launch_trmm(const TrmmLaunch & L, cudaStream_t st);
// Batched left multiplies (many fields, one launch).  A class is one column
// class of one field: columns r, r + cstride, ... of that field's matrix.
struct TrmmBatchClass {
    int field;       // index into the pointer tables
    int u;           // which of the field's two matrices
    int r;           // first column of the class (column offset r * n)
    int n;           // order of the triangular matrix
    int mrows;       // rows of the product
    int ncols;       // columns of the product
    long long ld;    // column stride inside the class (4n for sph / disk, n for tri)
};
struct TrmmTile { int cls, tm, tn; };
struct TrmmBatch {
    const double * U[kMaxFields][2];
    const double * in[kMaxFields];
    double * out[kMaxFields];
    const TrmmBatchClass * classes;   // device
    const TrmmTile * tiles;           // device, longest K first
};
// mode 0 / 1: Out = U In / U^T In; mode 2 / 3: Out = In U / In U^T
cudaError_t launch_trmm_batched(const TrmmBatch & P, int ntiles, bool vec16, int mode, cudaStream_t st);
int trmm_tile_rows();
int trmm_tile_cols();
// Right multiply for tri: Out = In * op(U) (rows of In are independent).
cudaError_t launch_trmm_right(const double * U, const double * in, double * out, int n, int nrows,
                              long long ld, bool trans, cudaStream_t st);
// tri normalisation (src/drivers.c:6-24), in place
cudaError_t launch_cheb_normalize(double * A, int N, int M, long long lda, bool transposed, cudaStream_t st);

// Host plan generation (plan.cpp).
void rotation_tables(int kind, int n, double alpha, double beta, double gamma, double * s, double * c);
double * connection_legendre_to_chebyshev(int normleg, int normcheb, int n);
double * connection_chebyshev_to_legendre(int normcheb, int normleg, int n);
double * connection_ultraspherical(int norm1, int norm2, int n, double lambda, double mu);
double * connection_jacobi(int n, double alpha, double beta, double gamma, double delta);
std::vector<RotTask> build_tasks(int kind, int N, int M, int field);
double task_cost(int kind, int N, int M, int mbase);

// The harmonic plan behind ft_harmonic_plan * (the public struct is its first member).
constexpr int kPlanMagic = 0x46544232;   // "FTB2"
struct HarmonicPlan {
    ft_harmonic_plan pub;       // must stay the first member
    int magic;
    int kind, n, Mdef;
    ft_rotation_plan * rp_arr[1];
    double * hostP[2];
    double * hostPinv[2];
    double * dP[2];
    double * dPinv[2];
    std::mutex host_mu;         // one host-pointer call at a time (they share d_stage and stream)
    double * d_stage;           // device copy of A for host-pointer calls
    size_t stage_elems;
    cudaStream_t stream;
    int device;
    void * blocked;             // tile matrices of the blocked sweeps (built on first use)
    void * mixed_trmm;          // sliced images of the connection matrices (built on first use)
};
// Out = op(U) In over the four stride-4 column classes (U[0] on 0 and 3, U[1] on 1 and 2; swapped
// with swap), U = the plan's P or Pinv (api.cu)
bool connection_multiply(HarmonicPlan * H, bool inverse, bool trans, const double * in, double * out, int M,
                         cudaStream_t st, bool swap);
// NULL unless P is a live plan of this library (api.cu)
HarmonicPlan * as_plan(const ft_harmonic_plan * P);
// A rotation plan of any kind, and its sweeps on device memory (in == out allowed) (api.cu)
ft_rotation_plan * rotation_plan_new(int kind, int n, double alpha, double beta, double gamma);
bool rotation_sweeps(ft_rotation_plan * RP, bool hi2lo, const double * in, double * out, int M, long long lda,
                     cudaStream_t st);
// Dunkl-Xu plans (rectdisk.cu): false / -1 when P is not one
bool rect_plan_destroy(ft_harmonic_plan * P);
// Tetrahedral plans (tet.cu): false when P is not one
bool tet_plan_destroy(ft_harmonic_plan * P);
// Annulus plans (ann.cu): false / -1 when P is not one
bool ann_plan_destroy(ft_harmonic_plan * P);
int ann_execute_dev(const ft_harmonic_plan * P, bool forward, char TRANS, double * dA, int N, int M, cudaStream_t st);
int rect_execute_dev(const ft_harmonic_plan * P, bool forward, char TRANS, double * dA, int N, int M, cudaStream_t st);
// device task list already built for (RP, M), without building one (api.cu)
bool find_tasks(ft_rotation_plan * RP, int M, const RotTask ** d_tasks, int * ntasks);

// Blocked sweeps for fields sharing one plan (blocked.cu).
struct BlkTaskList { void * d_tasks = nullptr; int ntasks = 0; };
void * blocked_plan_build(HarmonicPlan * H);
void blocked_plan_free(void * p);
int blocked_block_size();
bool blocked_tasks(void * plan, int nf, int N, int M, BlkTaskList * out);
cudaError_t launch_blocked(void * plan, bool hi2lo, double * const * A, int nf, int N, int M, const BlkTaskList & tl,
                           int * counter, cudaStream_t st);
// split-BF16 tensor-core products of the same blocks
bool blocked_mixed_prepare(void * plan, int ns);
bool blocked_tasks_mixed(void * plan, int nf, int N, int M, BlkTaskList * out);
cudaError_t launch_blocked_mixed(void * plan, int ns, bool hi2lo, float * T, int N, int M, const BlkTaskList & tl,
                                 int * counter, cudaStream_t st);
size_t blocked_mixed_T_elems(void * plan, int ntasks, int N);   // ntasks of blocked_tasks_mixed
cudaError_t launch_blocked_transpose(void * plan, bool to_T, double * const * A, int nf, int N, int M, float * T,
                                     const BlkTaskList & tl, cudaStream_t st);
int blocked_device_error(void * plan);
// connection multiply on the tensor cores from BF16 slices (trmm_mixed.cu), with nu = 4
// slices of U and nx = 3 (128-column tiles) or 4 (96-column tiles) of the input:
// ncls = 4, the column classes of sph and disk; ncls = 1, every column with U[which] (tri)
cudaError_t launch_trmm_mixed(HarmonicPlan * H, void ** plan_slot, void ** work_slot, int nu, int nx, bool inverse,
                              bool trans, double * const * in, double * const * out, int nf, int M, cudaStream_t st,
                              int ncls = 4, int which = 0);
// out = in^T for square n x n matrices of nf fields
cudaError_t launch_transpose_square(double * const * in, double * const * out, int nf, int n, cudaStream_t st);
void mixed_trmm_plan_free(void * p);
void mixed_trmm_work_free(void * p);
int mixed_trmm_device_error(void * p);

// Error state (api.cu).
void set_error(int status, const std::string & msg);
void clear_error();
void count_launch(unsigned long long n = 1);
// host threads for plan construction: the value of ft_set_num_threads, 0 when it was not called
int host_threads();
// column.cu: one column's sweeps (kinds SPH, TRI, DISK, RECT, and SPIN for a spin column's first
// stage with its table at k + j n + d |s| n) on device memory of len entries (double2 if cplx)
int column_touched(int kind, int n, bool hi2lo, int m1, int m2, int d);
bool column_sweeps_dev(void * dcol, bool cplx, const double2 * tab, int kind, int n, int m1, int m2, bool hi2lo, bool fwd, int d,
                       int as, int len);
// measurement hook: bracket a launch with events on its stream when profiling is on
enum { FAM_ROT = 0, FAM_TRMM = 1, FAM_OTHER = 2, FAM_BLOCK = 3 };
void prof_begin(int family, cudaStream_t st);
void prof_end(cudaStream_t st);

}  // namespace ftb

// The rotation plan behind the public opaque type.  The first three members
// mirror the reference's struct so code that reads RP->s / RP->c / RP->n works.
struct ft_rotation_plan_s {
    double * s;
    double * c;
    int n;
    // ---- B200 state ----
    int kind;
    double alpha, beta, gamma;
    int device;
    double2 * d_sc;            // interleaved table
    double2 * d_scp;           // the same, padded for the rotation kernel's bulk copies (Geo::padded_col)
    int * d_counter;           // work counter for the persistent kernel
    std::mutex * mu;
    std::map<int, std::pair<ftb::RotTask *, int>> * tasks;   // M -> device task list (longest first)
    std::map<int, ftb::RotSchedule *> * sched;               // M -> pass schedule of that list
};
