// Synthesis and analysis on the sphere's tensor-product grid (the reference's
// ft_plan_sph_synthesis / ft_execute_sph_synthesis and friends, src/fftw.c:63-277):
// the Fourier coefficients that sph2fourier produces become values at the N x M
// points theta_i = (i + 1/2) pi / N, phi_k = 2 pi k / M, and back.
//
// Two one-dimensional stages:
//   theta (down each column, length N): the four stride-4 column classes take the
//     plan's two kinds (classes 0 and 3 the first, 1 and 2 the second), each a
//     cosine or sine transform of type II (analysis) or III (synthesis) in FFTW's
//     unnormalised definitions (REDFT10 / RODFT10 / REDFT01 / RODFT01);
//   phi (along each row, length M): a real DFT, complex-to-real for synthesis and
//     real-to-complex for analysis, unnormalised, on the half spectrum laid out as
//     the reference's: column 2j is the real part of frequency j, column 2j - 1 the
//     negated imaginary part.
// with the reference's scalings and end-entry factors in between.
//
// The cosine transforms go through complex FFTs of length N (Makhoul's reordering):
//   DCT-II:  v = (x_0, x_2, x_4, .., x_5, x_3, x_1), V = DFT(v),
//            y_k = 2 Re(exp(-i pi k / 2N) V_k);
//   DCT-III: V_k = (y_k - i y_{N-k}) exp(i pi k / 2N) (y_N = 0), a Hermitian
//            spectrum, v = unnormalised inverse DFT(V), x = v un-permuted;
// and the sine transforms through them: DST-II(x)_k = DCT-II((-1)^n x_n)_{N-1-k},
// DST-III(x)_k = (-1)^k DCT-III(x reversed)_k.  The DFTs are cuFFT's (library
// FFTs, batched over all M columns at once); the reorderings, twiddles, scalings and
// the half-spectrum packing are this file's kernels.
//
// The spin-weighted sphere's grid (a complex N x M matrix, src/fftw.c:755-960) runs the same
// theta stage on the 2M real columns of its split parts, and a complex DFT along the rows around
// the reference's column permutation (columns 2j and 2j - 1 to j and M - j).
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include <cufft.h>

#include "ft_internal.h"

namespace ftb {
namespace {

// FFTW r2r kinds used by the plans (the values of fftw3.h's enum)
enum { K_REDFT01 = 4, K_REDFT10 = 5, K_REDFT11 = 6, K_RODFT01 = 8, K_RODFT10 = 9 };
enum Op { SPH_SYN = 0, SPH_ANA = 1, SPHV_SYN = 2, SPHV_ANA = 3, DISK_SYN = 4, DISK_ANA = 5, TRI_SYN = 6, TRI_ANA = 7,
          ANN_SYN = 8, ANN_ANA = 9, RECT_SYN = 10, RECT_ANA = 11, TET_SYN = 12, TET_ANA = 13, SPIN_SYN = 14, SPIN_ANA = 15 };
// plan families: the sphere's (sph, sphv), the disk's, the triangle's, the annulus's, the
// rectangularised disk's, the tetrahedron's (an n x n x n tensor held as the n x n^2 matrix of its
// columns), the spin-weighted sphere's (a complex N x M matrix)
enum Family { F_SPHERE = 0, F_DISK = 1, F_TRI = 2, F_ANN = 3, F_RECT = 4, F_TET = 5, F_SPIN = 6 };

constexpr int kGridMagic = 0x46544753;   // "FTGS"

// The reference's constants (src/ftinternal.h:48-56)
constexpr double C_1_4_SQRT_PI = 0.141047395886939072;   // 1 / (4 sqrt(pi))
constexpr double C_1_2_SQRT_PI = 0.282094791773878143;   // 1 / (2 sqrt(pi))
constexpr double C_4_SQRT_PI = 7.089815403622064109;     // 4 sqrt(pi)
constexpr double C_2_SQRT_PI = 3.544907701811032055;     // 2 sqrt(pi)
constexpr double C_1_2_SQRT_2PI = 0.199471140200716338;  // 1 / (2 sqrt(2 pi))
constexpr double C_2_SQRT_2PI = 5.013256549262001005;    // 2 sqrt(2 pi)
constexpr double C_SQRT2 = 1.41421356237309504880;
constexpr double C_SQRT1_2 = 0.70710678118654752440;

bool is_dst(int kind) { return kind == K_RODFT01 || kind == K_RODFT10; }
bool is_type3(int kind) { return kind == K_REDFT01 || kind == K_RODFT01; }

}  // namespace

struct SphereGridPlan {
    int magic = kGridMagic;
    int family = F_SPHERE;
    int N = 0, M = 0;
    int kind[2] = {0, 0};        // theta kinds of column classes {0, 3} and {1, 2} (tri: both dimensions;
                                 // rect: even and odd columns)
    int kind_rows = 0;           // rect: the kind along the rows
    double rho = 0.0;            // annulus: the radius ratio
    int spin = 0;                // spin: the plan's spin S (its parity picks the kinds and the end entries)
    int zsign = 0;               // spin: the row DFT's sign (+1 backward, -1 forward; 0: by the kinds)
    double * d_w = nullptr;      // annulus: the N radial weights
    int device = 0;
    cufftHandle t_r2c = 0;       // length N, batch M (cosine type II)
    cufftHandle t_c2r = 0;       // length N, batch M (cosine type III)
    cufftHandle p_r2c = 0;       // length M along rows, batch N
    cufftHandle p_c2r = 0;
    cufftHandle p_z2z = 0;       // spin: complex DFT of length M along rows, batch N
    bool have_t_r2c = false, have_t_c2r = false, have_p_r2c = false, have_p_c2r = false, have_p_z2z = false;
    // (spin: the theta stage runs on 2M real columns, so the work buffers below hold 2M columns)
    double * d_work = nullptr;   // N x M real
    double2 * d_cwork = nullptr; // (N/2 + 1) x M complex
    double2 * d_Y = nullptr;     // N x (M/2 + 1) complex, element (i, j) at i + j N (spin: N x M)
    double * d_stage = nullptr;  // N x M, host-pointer calls
    // disk: the DCT-IV of the columns of classes 1 and 2 (nq of them) as a zero-padded complex
    // DFT of length 2N
    cufftHandle t4 = 0;
    bool have_t4 = false;
    int nq = 0;
    double2 * d_u = nullptr;     // 2N x nq
    double * d_work2 = nullptr;  // tri: N x N, the transposed matrix; spin: N x 2M, the parts split
    cudaStream_t stream = nullptr;
    std::mutex mu;
};

namespace {

// ---------------------------------------------------------------------------
// theta stage kernels: one thread per (entry, column); column j uses the kind of
// its class, cls(j) = j mod 4 in {0, 3} -> kind[0], {1, 2} -> kind[1]
// ---------------------------------------------------------------------------
// k1dst bit 1 set: the classes are the even and odd columns instead (the rectangularised disk's);
// bit 2 set: column j is part j & 1 of complex column j >> 1, whose class decides (the spin grid's)
__device__ __forceinline__ bool col_dst(int j, int k0dst, int k1dst) {
    if (k1dst & 4) { j >>= 1; k1dst &= 1; }
    if (k1dst & 2) return (j & 1) ? (k1dst & 1) : k0dst;
    const int r = j & 3;
    return (r == 0 || r == 3) ? k0dst : k1dst;
}

// type II, before the FFT: v = permute(sign-flipped x) into work
__global__ void t2_pre(const double * __restrict__ X, double * __restrict__ V, int N, int M, int k0dst, int k1dst) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * M) return;
    const int j = (int) (idx / N), n = (int) (idx % N);
    const bool dst = col_dst(j, k0dst, k1dst);
    // v[n] = x'[2n] for n < ceil(N/2), v[N-1-n'] = x'[2n'+1]
    const int h = (N + 1) / 2;
    const int src = n < h ? 2 * n : 2 * (N - 1 - n) + 1;
    double x = X[(long long) j * N + src];
    if (dst && (src & 1)) x = -x;            // (-1)^n x_n
    V[(long long) j * N + n] = x;
}

// type II, after the FFT: y_k = 2 Re(exp(-i pi k / 2N) V_k), reversed for sine columns
__global__ void t2_post(const double2 * __restrict__ C, double * __restrict__ X, int N, int M, int k0dst, int k1dst) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * M) return;
    const int j = (int) (idx / N), k = (int) (idx % N);
    const bool dst = col_dst(j, k0dst, k1dst);
    const int H = N / 2 + 1;
    double2 v = k < H ? C[(long long) j * H + k] : C[(long long) j * H + (N - k)];
    if (k >= H) v.y = -v.y;                  // V_k = conj(V_{N-k})
    double s, c;
    sincospi((double) k / (2.0 * N), &s, &c);
    const double y = 2.0 * (c * v.x + s * v.y);   // Re((c - i s)(v.x + i v.y))
    X[(long long) j * N + (dst ? N - 1 - k : k)] = y;
}

// type III, before the inverse FFT: V_k = (y_k - i y_{N-k}) exp(i pi k / 2N), k <= N/2,
// with y reversed for sine columns
__global__ void t3_pre(const double * __restrict__ X, double2 * __restrict__ C, int N, int M, int k0dst, int k1dst) {
    const int H = N / 2 + 1;
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) H * M) return;
    const int j = (int) (idx / H), k = (int) (idx % H);
    const bool dst = col_dst(j, k0dst, k1dst);
    const double * y = X + (long long) j * N;
    auto yy = [&](int t) -> double { return t >= N ? 0.0 : (dst ? y[N - 1 - t] : y[t]); };
    const double a = yy(k), b = k == 0 ? 0.0 : yy(N - k);
    double s, c;
    sincospi((double) k / (2.0 * N), &s, &c);
    double2 v = make_double2(a * c + b * s, a * s - b * c);   // (a - i b)(c + i s)
    if ((N & 1) == 0 && k == N / 2) v.y = 0.0;                // the Nyquist term is real
    C[(long long) j * H + k] = v;
}

// type III, after the inverse FFT: x un-permuted, (-1)^k for sine columns
__global__ void t3_post(const double * __restrict__ V, double * __restrict__ X, int N, int M, int k0dst, int k1dst) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * M) return;
    const int j = (int) (idx / N), k = (int) (idx % N);
    const bool dst = col_dst(j, k0dst, k1dst);
    const int h = (N + 1) / 2;
    const int n = (k & 1) ? N - 1 - (k >> 1) : (k >> 1);     // x[2n] = v[n], x[2n+1] = v[N-1-n]
    double x = V[(long long) j * N + n];
    if (dst && (k & 1)) x = -x;
    (void) h;
    X[(long long) j * N + k] = x;
}

// ---------------------------------------------------------------------------
// DCT-IV (REDFT11) of the columns of classes 1 and 2 (column 4 (q / 2) + 1 + q % 2 for q < nq):
//   y_k = 2 sum_j x_j cos(pi (j + 1/2)(k + 1/2) / N)
//       = 2 Re(exp(-i pi (2k + 1) / 4N) DFT_2N(x_j exp(-i pi j / 2N), zero-padded)_k)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int class12_col(int q) { return 4 * (q / 2) + 1 + (q & 1); }

__global__ void dct4_pre(const double * __restrict__ X, double2 * __restrict__ U, int N, int nq) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2LL * N * nq) return;
    const int q = (int) (idx / (2 * N)), j = (int) (idx % (2 * N));
    double2 u = make_double2(0.0, 0.0);
    if (j < N) {
        const double x = X[(long long) class12_col(q) * N + j];
        double s, c;
        sincospi((double) j / (2.0 * N), &s, &c);
        u = make_double2(x * c, -x * s);
    }
    U[idx] = u;
}

__global__ void dct4_post(const double2 * __restrict__ U, double * __restrict__ X, int N, int nq) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * nq) return;
    const int q = (int) (idx / N), k = (int) (idx % N);
    const double2 v = U[(long long) q * 2 * N + k];
    double s, c;
    sincospi((double) (2 * k + 1) / (4.0 * N), &s, &c);
    X[(long long) class12_col(q) * N + k] = 2.0 * (c * v.x + s * v.y);   // 2 Re((c - i s) v)
}

// entries (row, start + step t) times f
__global__ void scale_row(double * X, int N, int M, int row, int start, int step, double f) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const long long j = start + (long long) step * t;
    if (j < M) X[j * N + row] *= f;
}

// annulus: the columns of classes 1 and 2 (j mod 4 = 1, 2) times w_i (divide: divided by w_i)
__global__ void ann_weights(double * X, const double * __restrict__ w, int N, int M, bool divide) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * M) return;
    const int j = (int) (idx / N), i = (int) (idx % N);
    const int r = j & 3;
    if (r != 1 && r != 2) return;
    X[idx] = divide ? X[idx] / w[i] : X[idx] * w[i];
}

// rect: column 0 times f0 and every entry times s or divided by d (d > 0), in the reference's order
// (f0 first when f0_first, else last)
__global__ void col0_scale(double * X, int N, int M, double f0, double s, double d, bool f0_first) {
    const long long total = (long long) N * M;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
        const bool c0 = e < N;
        double v = X[e];
        if (f0_first && c0) v *= f0;
        v = d > 0.0 ? v / d : v * s;
        if (!f0_first && c0) v *= f0;
        X[e] = v;
    }
}

// tetrahedron: out = in with axes 0 and 1 (swap01) or 0 and 2 swapped, an n x n x n tensor
__global__ void permute3(const double * __restrict__ in, double * __restrict__ out, int n, bool swap01) {
    const long long total = (long long) n * n * n;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
        const long long i = e % n, l = (e / n) % n, m = e / ((long long) n * n);
        const long long o = swap01 ? l + n * i + (long long) n * n * m : m + n * l + (long long) n * n * i;
        out[o] = in[e];
    }
}

// tetrahedron scalings (src/fftw.c:351-402): entry (i, l, m) times ef when m == 0, when i == 0, when
// l == 0 (in the reference's order), then times s or divided by d (d > 0)
__global__ void tet_scale(double * X, int n, double ef, double s, double d) {
    const long long total = (long long) n * n * n;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
        const long long i = e % n, l = (e / n) % n, m = e / ((long long) n * n);
        double v = X[e];
        if (m == 0) v *= ef;
        if (i == 0) v *= ef;
        if (l == 0) v *= ef;
        X[e] = d > 0.0 ? v / d : v * s;
    }
}

// triangle scalings (src/fftw.c:292-330), entry (i, j) of the N x M matrix: times ef when
// j == 0, times ef when i == 0, then times s (mul) or divided by d (d > 0)
__global__ void tri_scale(double * X, int N, int M, double ef, double s, double d) {
    const long long total = (long long) N * M;
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
        const int i = (int) (e % N), j = (int) (e / N);
        double v = X[e];
        if (j == 0) v *= ef;
        if (i == 0) v *= ef;
        X[e] = d > 0.0 ? v / d : v * s;
    }
}

// ---------------------------------------------------------------------------
// phi stage packing and the scalings
// ---------------------------------------------------------------------------
// Y(i, 0) = (s X(i, 0)) f0; Y(i, j) = s (X(i, 2j) - i X(i, 2j - 1)), j = 1 .. M/2
__global__ void pack_r2c(const double * __restrict__ X, double2 * __restrict__ Y, int N, int M, double s, double f0) {
    const int H = M / 2 + 1;
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * H) return;
    const int j = (int) (idx / N), i = (int) (idx % N);
    double2 v;
    if (j == 0) v = make_double2((s * X[i]) * f0, 0.0);
    else        v = make_double2(s * X[i + (long long) (2 * j) * N], -s * X[i + (long long) (2 * j - 1) * N]);
    Y[idx] = v;
}

// X(i, 0) = (s Re Y(i, 0)) f0; X(i, 2j) = s Re Y(i, j); X(i, 2j - 1) = s (-Im Y(i, j))
__global__ void unpack_c2r(const double2 * __restrict__ Y, double * __restrict__ X, int N, int M, double s, double f0) {
    const int H = M / 2 + 1;
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * H) return;
    const int j = (int) (idx / N), i = (int) (idx % N);
    const double2 v = Y[idx];
    if (j == 0) { X[i] = (s * v.x) * f0; return; }
    X[i + (long long) (2 * j) * N] = s * v.x;
    X[i + (long long) (2 * j - 1) * N] = -s * v.y;
}

// Multiplies the first (last = 0) or last (last = 1) entry of the columns
// {c0} (c0 >= 0) and {start + 4t, start + 1 + 4t, t >= 0} by f.
__global__ void scale_ends(double * X, int N, int M, bool last, int c0, int start, double f) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = last ? N - 1 : 0;
    if (t == 0 && c0 >= 0 && c0 < M) X[(long long) c0 * N + row] *= f;
    const int j0 = start + 4 * t;
    if (j0 < M) X[(long long) j0 * N + row] *= f;
    if (j0 + 1 < M) X[(long long) (j0 + 1) * N + row] *= f;
}

// ---------------------------------------------------------------------------
// spin grids (src/fftw.c:6-38, 801-960): the complex N x M matrix X (interleaved parts) and W, the
// real N x 2M matrix whose column 2c + p is part p of column c, on which the theta stage runs.
// Column c of the destination comes from column src(c) of the source:
//   perm 0: src(c) = c;
//   perm 1 (colswap_t): src(0) = 0, src(2j) = j, src(2j - 1) = M - j;
//   perm 2 (colswap):   src(0) = 0, src(k) = 2k for k <= (M - 1) / 2, 2 (M - k) - 1 above (M odd);
// then every entry times s, and the entries of `row` in the column classes {0, 3} (set 0) or
// {1, 2} (set 1) times f as well (row -1: none).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int spin_src(int c, int M, int perm) {
    if (perm == 0 || c == 0) return c;
    if (perm == 1) return (c & 1) ? M - (c + 1) / 2 : c / 2;
    return c <= (M - 1) / 2 ? 2 * c : 2 * (M - c) - 1;
}
__device__ __forceinline__ bool spin_end(int i, int c, int row, int set) {
    const int r = c & 3;
    return i == row && ((r == 1 || r == 2) ? 1 : 0) == set;
}

// X (2 N M doubles) -> W (N x 2M)
__global__ void spin_split(const double * __restrict__ X, double * __restrict__ W, int N, int M, int perm, double s,
                           int row, int set, double f) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * M) return;
    const int c = (int) (idx / N), i = (int) (idx % N);
    const long long from = 2 * ((long long) spin_src(c, M, perm) * N + i);
    double re = X[from] * s, im = X[from + 1] * s;
    if (spin_end(i, c, row, set)) { re *= f; im *= f; }
    W[(long long) (2 * c) * N + i] = re;
    W[(long long) (2 * c + 1) * N + i] = im;
}

// W (N x 2M) -> X (2 N M doubles)
__global__ void spin_merge(const double * __restrict__ W, double * __restrict__ X, int N, int M, int perm, double s,
                           int row, int set, double f) {
    const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long) N * M) return;
    const int c = (int) (idx / N), i = (int) (idx % N);
    const int q = spin_src(c, M, perm);
    double re = W[(long long) (2 * q) * N + i] * s, im = W[(long long) (2 * q + 1) * N + i] * s;
    if (spin_end(i, c, row, set)) { re *= f; im *= f; }
    X[2 * idx] = re;
    X[2 * idx + 1] = im;
}

bool ok(cudaError_t e, const char * what) {
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}
bool fok(cufftResult r, const char * what) {
    if (r == CUFFT_SUCCESS) return true;
    set_error(r == CUFFT_ALLOC_FAILED ? FT_B200_ENOMEM : FT_B200_ECUDA, std::string(what) + ": cuFFT error " + std::to_string((int) r));
    return false;
}

unsigned blocks(long long n) { return (unsigned) ((n + 255) / 256); }

SphereGridPlan * make_plan(int N, int M, int k0, int k1, int family = F_SPHERE, int krows = 0, double rho = 0.0) {
    clear_error();
    const bool square = family == F_TRI || family == F_RECT;   // row transforms through a square transpose
    const bool nophi = square || family == F_TET;
    if (N < 1 || M < 1) { set_error(FT_B200_EINVAL, "N and M must be positive"); return nullptr; }
    if (!nophi && M % 2 == 0) {
        set_error(FT_B200_EINVAL, family == F_SPIN ? "M must be odd (the column permutation pairs columns 2j - 1, 2j)"
                                                   : "M must be odd (the half spectrum holds columns 2j - 1, 2j)");
        return nullptr;
    }
    if (square && M != N) {
        set_error(FT_B200_EINVAL, family == F_TRI ? "triangle grids need M == N (the reference's 2-D plan reads the matrix both ways)"
                                                  : "rectangularised-disk grids need M == N here (the rows go through a square transpose)");
        return nullptr;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error(FT_B200_ENODEV, "no CUDA device"); return nullptr; }
    SphereGridPlan * P = new SphereGridPlan();
    P->family = family;
    P->N = N; P->M = M; P->kind[0] = k0; P->kind[1] = k1; P->kind_rows = krows; P->rho = rho;
    cudaGetDevice(&P->device);
    const bool spin = family == F_SPIN;
    const int TM = spin ? 2 * M : M;   // real columns of the theta stage
    const size_t nm = (size_t) N * TM;
    bool good = ok(cudaMalloc(&P->d_work, sizeof(double) * nm), "cudaMalloc(grid work)") &&
                ok(cudaMalloc(&P->d_cwork, sizeof(double2) * (size_t) (N / 2 + 1) * TM), "cudaMalloc(grid work)") &&
                (nophi || ok(cudaMalloc(&P->d_Y, sizeof(double2) * (size_t) N * (spin ? M : M / 2 + 1)), "cudaMalloc(grid spectrum)")) &&
                (!(nophi || spin) || ok(cudaMalloc(&P->d_work2, sizeof(double) * nm), "cudaMalloc(grid work)")) &&
                ok(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (good && family == F_DISK) {
        P->nq = (M + 2) / 4 + (M + 1) / 4;
        if (P->nq > 0) {
            int n2[1] = {2 * N};
            good = ok(cudaMalloc(&P->d_u, sizeof(double2) * 2 * (size_t) N * P->nq), "cudaMalloc(grid work)") &&
                   fok(cufftPlanMany(&P->t4, 1, n2, nullptr, 1, 2 * N, nullptr, 1, 2 * N, CUFFT_Z2Z, P->nq), "cufftPlanMany");
            P->have_t4 = good;
        }
    }
    if (good) {
        int n[1] = {N};
        if (is_type3(k0)) {
            good = fok(cufftPlanMany(&P->t_c2r, 1, n, nullptr, 1, N / 2 + 1, nullptr, 1, N, CUFFT_Z2D, TM), "cufftPlanMany");
            P->have_t_c2r = good;
        } else {
            good = fok(cufftPlanMany(&P->t_r2c, 1, n, nullptr, 1, N, nullptr, 1, N / 2 + 1, CUFFT_D2Z, TM), "cufftPlanMany");
            P->have_t_r2c = good;
        }
    }
    if (good && family == F_ANN) {   // src/fftw.c:545-551
        std::vector<double> w(N);
        for (int n = 0; n < N; n++) {
            const double t = (N - n - 0.5) * M_PI / (2.0 * N);
            const double ct = std::sin(t), st = std::cos(t);
            w[n] = std::sqrt(2.0 * (ct * ct + rho * rho * st * st) / (1.0 - rho * rho));
        }
        good = ok(cudaMalloc(&P->d_w, sizeof(double) * N), "cudaMalloc(weights)") &&
               ok(cudaMemcpy(P->d_w, w.data(), sizeof(double) * N, cudaMemcpyHostToDevice), "cudaMemcpy(weights)");
    }
    if (good && spin) {
        // phi: complex, along rows, element stride N, rows one apart
        int m[1] = {M};
        good = fok(cufftPlanMany(&P->p_z2z, 1, m, m, N, 1, m, N, 1, CUFFT_Z2Z, N), "cufftPlanMany");
        P->have_p_z2z = good;
    } else if (good && !nophi) {
        // phi: along rows, element stride N, rows one apart
        int m[1] = {M}, hm[1] = {M / 2 + 1};
        good = fok(cufftPlanMany(&P->p_c2r, 1, m, hm, N, 1, m, N, 1, CUFFT_Z2D, N), "cufftPlanMany");
        P->have_p_c2r = good;
        if (good) {
            good = fok(cufftPlanMany(&P->p_r2c, 1, m, m, N, 1, hm, N, 1, CUFFT_D2Z, N), "cufftPlanMany");
            P->have_p_r2c = good;
        }
    }
    if (!good) {
        ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
        return nullptr;
    }
    return P;
}

// theta transforms of all M columns in place (the plan's kinds by column class; disk: kind[0]
// on every column here, the DCT-IV of classes 1 and 2 in theta_disk)
bool theta(SphereGridPlan * P, double * X, cudaStream_t st, bool rows = false) {
    const int N = P->N, M = P->family == F_SPIN ? 2 * P->M : P->M;
    int d0 = is_dst(P->kind[0]), d1 = P->family == F_SPHERE ? is_dst(P->kind[1]) : d0;
    if (P->family == F_SPIN) d1 = is_dst(P->kind[1]) | 4;   // W's columns by their complex column's class
    if (P->family == F_RECT) {
        if (rows) { d0 = is_dst(P->kind_rows); d1 = d0; }   // every column of the transposed matrix
        else d1 = is_dst(P->kind[1]) | 2;                    // even and odd columns
    }
    if (is_type3(P->kind[0])) {
        if (!fok(cufftSetStream(P->t_c2r, st), "cufftSetStream")) return false;
        t3_pre<<<blocks((long long) (N / 2 + 1) * M), 256, 0, st>>>(X, P->d_cwork, N, M, d0, d1);
        count_launch();
        if (!ok(cudaGetLastError(), "t3_pre")) return false;
        if (!fok(cufftExecZ2D(P->t_c2r, reinterpret_cast<cufftDoubleComplex *>(P->d_cwork), P->d_work), "cufftExecZ2D")) return false;
        t3_post<<<blocks((long long) N * M), 256, 0, st>>>(P->d_work, X, N, M, d0, d1);
        count_launch();
        return ok(cudaGetLastError(), "t3_post");
    }
    if (!fok(cufftSetStream(P->t_r2c, st), "cufftSetStream")) return false;
    t2_pre<<<blocks((long long) N * M), 256, 0, st>>>(X, P->d_work, N, M, d0, d1);
    count_launch();
    if (!ok(cudaGetLastError(), "t2_pre")) return false;
    if (!fok(cufftExecD2Z(P->t_r2c, P->d_work, reinterpret_cast<cufftDoubleComplex *>(P->d_cwork)), "cufftExecD2Z")) return false;
    t2_post<<<blocks((long long) N * M), 256, 0, st>>>(P->d_cwork, X, N, M, d0, d1);
    count_launch();
    return ok(cudaGetLastError(), "t2_post");
}

// disk: classes 1 and 2 by the DCT-IV (their inputs read before theta overwrites them)
bool theta_disk(SphereGridPlan * P, double * X, cudaStream_t st) {
    const int N = P->N, nq = P->nq;
    if (nq > 0) {
        dct4_pre<<<blocks(2LL * N * nq), 256, 0, st>>>(X, P->d_u, N, nq);
        count_launch();
        if (!ok(cudaGetLastError(), "dct4_pre") || !fok(cufftSetStream(P->t4, st), "cufftSetStream") ||
            !fok(cufftExecZ2Z(P->t4, reinterpret_cast<cufftDoubleComplex *>(P->d_u), reinterpret_cast<cufftDoubleComplex *>(P->d_u),
                              CUFFT_FORWARD), "cufftExecZ2Z"))
            return false;
    }
    if (!theta(P, X, st)) return false;
    if (nq > 0) {
        dct4_post<<<blocks((long long) N * nq), 256, 0, st>>>(P->d_u, X, N, nq);
        count_launch();
        return ok(cudaGetLastError(), "dct4_post");
    }
    return true;
}

// triangle: the plan's kind along both dimensions of the square matrix
bool theta_tri(SphereGridPlan * P, double * X, cudaStream_t st) {
    double * a[1] = {X}, * b[1] = {P->d_work2};
    return theta(P, X, st) && ok(launch_transpose_square(a, b, 1, P->N, st), "transpose") && theta(P, P->d_work2, st) &&
           ok(launch_transpose_square(b, a, 1, P->N, st), "transpose");
}

// rect: the plan's row kind along the rows of the square matrix (transpose, columns, transpose back)
bool theta_rows(SphereGridPlan * P, double * X, cudaStream_t st) {
    double * a[1] = {X}, * b[1] = {P->d_work2};
    return ok(launch_transpose_square(a, b, 1, P->N, st), "transpose") && theta(P, P->d_work2, st, true) &&
           ok(launch_transpose_square(b, a, 1, P->N, st), "transpose");
}

// tetrahedron: the plan's kind along all three axes (axis 0 as the columns of the n x n^2 matrix,
// the other two after swapping them with axis 0)
bool theta_tet(SphereGridPlan * P, double * X, cudaStream_t st) {
    const int n = P->N;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto perm = [&](const double * a, double * b, bool swap01) {
        permute3<<<sms * 4, 256, 0, st>>>(a, b, n, swap01);
        count_launch();
        return ok(cudaGetLastError(), "permute3");
    };
    return theta(P, X, st) && perm(X, P->d_work2, true) && theta(P, P->d_work2, st) && perm(P->d_work2, X, true) &&
           perm(X, P->d_work2, false) && theta(P, P->d_work2, st) && perm(P->d_work2, X, false);
}

bool tet_scaling(SphereGridPlan * P, double * X, double ef, double s, double d, cudaStream_t st) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    tet_scale<<<sms * 4, 256, 0, st>>>(X, P->N, ef, s, d);
    count_launch();
    return ok(cudaGetLastError(), "tet_scale");
}

bool row_factor(SphereGridPlan * P, double * X, int row, int start, int step, double f, cudaStream_t st) {
    const int t = (P->M - start + step - 1) / step;
    if (t <= 0) return true;
    scale_row<<<blocks(t), 256, 0, st>>>(X, P->N, P->M, row, start, step, f);
    count_launch();
    return ok(cudaGetLastError(), "scale_row");
}

bool weights(SphereGridPlan * P, double * X, bool divide, cudaStream_t st) {
    ann_weights<<<blocks((long long) P->N * P->M), 256, 0, st>>>(X, P->d_w, P->N, P->M, divide);
    count_launch();
    return ok(cudaGetLastError(), "ann_weights");
}

bool col0_scaling(SphereGridPlan * P, double * X, double f0, double s, double d, bool f0_first, cudaStream_t st) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    col0_scale<<<sms * 4, 256, 0, st>>>(X, P->N, P->M, f0, s, d, f0_first);
    count_launch();
    return ok(cudaGetLastError(), "col0_scale");
}

bool tri_scaling(SphereGridPlan * P, double * X, double ef, double s, double d, cudaStream_t st) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    tri_scale<<<sms * 4, 256, 0, st>>>(X, P->N, P->M, ef, s, d);
    count_launch();
    return ok(cudaGetLastError(), "tri_scale");
}

bool phi_c2r(SphereGridPlan * P, const double * X, double s, double f0, cudaStream_t st) {
    const int N = P->N, M = P->M;
    pack_r2c<<<blocks((long long) N * (M / 2 + 1)), 256, 0, st>>>(X, P->d_Y, N, M, s, f0);
    count_launch();
    if (!ok(cudaGetLastError(), "pack_r2c")) return false;
    return fok(cufftSetStream(P->p_c2r, st), "cufftSetStream") &&
           fok(cufftExecZ2D(P->p_c2r, reinterpret_cast<cufftDoubleComplex *>(P->d_Y), const_cast<double *>(X)), "cufftExecZ2D");
}

bool phi_r2c(SphereGridPlan * P, double * X, double s, double f0, cudaStream_t st) {
    const int N = P->N, M = P->M;
    if (!fok(cufftSetStream(P->p_r2c, st), "cufftSetStream") ||
        !fok(cufftExecD2Z(P->p_r2c, X, reinterpret_cast<cufftDoubleComplex *>(P->d_Y)), "cufftExecD2Z")) return false;
    unpack_c2r<<<blocks((long long) N * (M / 2 + 1)), 256, 0, st>>>(P->d_Y, X, N, M, s, f0);
    count_launch();
    return ok(cudaGetLastError(), "unpack_c2r");
}

bool ends(SphereGridPlan * P, double * X, bool last, int c0, int start, double f, cudaStream_t st) {
    const int t = (P->M - start + 3) / 4 + 1;
    scale_ends<<<blocks(t > 0 ? t : 1), 256, 0, st>>>(X, P->N, P->M, last, c0, start, f);
    count_launch();
    return ok(cudaGetLastError(), "scale_ends");
}

// The reference's execute sequences (src/fftw.c:131-277).  End-entry factors: first
// entries of {0, 3, 4, 7, 8, ..} (sph) or {1, 2, 5, 6, ..} (sphv); last entries of
// {1, 2, 5, 6, ..} (sph) or {0, 3, 4, 7, 8, ..} (sphv).
// spin: X <-> the split matrix in d_work2 (see spin_split / spin_merge)
bool split(SphereGridPlan * P, const double * X, int perm, double s, int row, int set, double f, cudaStream_t st) {
    spin_split<<<blocks((long long) P->N * P->M), 256, 0, st>>>(X, P->d_work2, P->N, P->M, perm, s, row, set, f);
    count_launch();
    return ok(cudaGetLastError(), "spin_split");
}
bool merge(SphereGridPlan * P, double * X, int perm, double s, int row, int set, double f, cudaStream_t st) {
    spin_merge<<<blocks((long long) P->N * P->M), 256, 0, st>>>(P->d_work2, X, P->N, P->M, perm, s, row, set, f);
    count_launch();
    return ok(cudaGetLastError(), "spin_merge");
}
// spin: the unnormalised complex DFT along the rows, from `in` to `out` (FFTW_BACKWARD, exp(+i..),
// for the synthesis plans; FFTW_FORWARD for the analysis plans)
bool phi_z2z(SphereGridPlan * P, const double * in, double * out, cudaStream_t st) {
    const int dir = P->zsign ? (P->zsign > 0 ? CUFFT_INVERSE : CUFFT_FORWARD) : (is_type3(P->kind[0]) ? CUFFT_INVERSE : CUFFT_FORWARD);
    return fok(cufftSetStream(P->p_z2z, st), "cufftSetStream") &&
           fok(cufftExecZ2Z(P->p_z2z, reinterpret_cast<cufftDoubleComplex *>(const_cast<double *>(in)),
                            reinterpret_cast<cufftDoubleComplex *>(out), dir), "cufftExecZ2Z");
}

// src/fftw.c:801-960.  The end entries: row 0 of the classes {0, 3} for even S ({1, 2} for odd S)
// before the synthesis / after the analysis; row N - 1 of the other classes in the 'C' forms.
bool run_spin(SphereGridPlan * P, int op, char T, double * X, cudaStream_t st) {
    if (T != 'N' && T != 'C') return true;
    const int N = P->N, M = P->M;
    const int first = P->spin % 2 == 0 ? 0 : 1, last = 1 - first;
    double * Y = reinterpret_cast<double *>(P->d_Y);
    const double sa = C_2_SQRT_2PI / (2.0 * N * M);
    if (op == SPIN_SYN) {
        if (T == 'N') return split(P, X, 0, 1.0, 0, first, 2.0, st) && theta(P, P->d_work2, st) &&
                             merge(P, Y, 2, C_1_2_SQRT_2PI, -1, 0, 1.0, st) && phi_z2z(P, Y, X, st);
        return phi_z2z(P, X, Y, st) && split(P, Y, 1, C_1_2_SQRT_2PI, -1, 0, 1.0, st) && theta(P, P->d_work2, st) &&
               merge(P, X, 0, 1.0, N - 1, last, 0.5, st);
    }
    if (T == 'N') return phi_z2z(P, X, Y, st) && split(P, Y, 1, sa, -1, 0, 1.0, st) && theta(P, P->d_work2, st) &&
                         merge(P, X, 0, 1.0, 0, first, 0.5, st);
    return split(P, X, 0, 1.0, N - 1, last, 2.0, st) && theta(P, P->d_work2, st) && merge(P, Y, 2, sa, -1, 0, 1.0, st) &&
           phi_z2z(P, Y, X, st);
}

bool run(SphereGridPlan * P, int op, char T, double * X, cudaStream_t st) {
    const int N = P->N, M = P->M;
    const double nm2 = 2.0 * N * M;
    if (op == SPIN_SYN || op == SPIN_ANA) return run_spin(P, op, T, X, st);
    if (op == DISK_SYN || op == DISK_ANA) {   // src/fftw.c:460-532: first entries of {0, 3, 4, 7, 8, ..} only
        auto first = [&](double f) { return ends(P, X, false, 0, 3, f, st); };
        if (op == DISK_SYN) {
            if (T == 'N') return first(2.0) && theta_disk(P, X, st) && phi_c2r(P, X, C_1_4_SQRT_PI, C_SQRT2, st);
            return phi_r2c(P, X, C_1_2_SQRT_PI, C_SQRT1_2, st) && theta_disk(P, X, st);
        }
        if (T == 'N') return phi_r2c(P, X, C_4_SQRT_PI / nm2, C_SQRT1_2, st) && theta_disk(P, X, st) && first(0.5);
        return theta_disk(P, X, st) && phi_c2r(P, X, C_2_SQRT_PI / nm2, C_SQRT2, st);
    }
    if (op == ANN_SYN || op == ANN_ANA) {     // src/fftw.c:583-658: every column the plan's kind, classes 1, 2 weighted
        if (op == ANN_SYN) {
            if (T == 'N') return row_factor(P, X, 0, 0, 1, 2.0, st) && theta(P, X, st) && weights(P, X, false, st) &&
                                 phi_c2r(P, X, C_1_4_SQRT_PI, C_SQRT2, st);
            return phi_r2c(P, X, C_1_2_SQRT_PI, C_SQRT1_2, st) && weights(P, X, false, st) && theta(P, X, st);
        }
        if (T == 'N') return phi_r2c(P, X, C_4_SQRT_PI / nm2, C_SQRT1_2, st) && weights(P, X, true, st) && theta(P, X, st) &&
                             row_factor(P, X, 0, 0, 1, 0.5, st);
        return theta(P, X, st) && weights(P, X, true, st) && phi_c2r(P, X, C_2_SQRT_PI / nm2, C_SQRT2, st);
    }
    if (op == RECT_SYN || op == RECT_ANA) {   // src/fftw.c:697-753
        const double nm = (double) N * M;
        if (op == RECT_SYN) {
            if (T == 'N') return row_factor(P, X, 0, 0, 2, 2.0, st) && theta(P, X, st) && col0_scaling(P, X, 2.0, 0.25, 0.0, true, st) &&
                                 theta_rows(P, X, st);
            return theta_rows(P, X, st) && col0_scaling(P, X, 1.0, 0.25, 0.0, true, st) && theta(P, X, st) &&
                   row_factor(P, X, N - 1, 1, 2, 0.5, st);
        }
        if (T == 'N') return theta_rows(P, X, st) && col0_scaling(P, X, 0.5, 1.0, nm, false, st) && theta(P, X, st) &&
                             row_factor(P, X, 0, 0, 2, 0.5, st);
        return row_factor(P, X, N - 1, 1, 2, 2.0, st) && theta(P, X, st) && theta_rows(P, X, st) &&
               col0_scaling(P, X, 1.0, 1.0, nm, false, st);
    }
    if (op == TET_SYN || op == TET_ANA) {     // src/fftw.c:351-402 (n x n x n)
        const int n = N;
        if (n <= 1) return true;
        const double nlm = (double) n * n * n;
        if (op == TET_SYN) {
            if (T == 'N') return tet_scaling(P, X, 2.0, 0.125, 0.0, st) && theta_tet(P, X, st);
            return theta_tet(P, X, st) && tet_scaling(P, X, 1.0, 0.125, 0.0, st);
        }
        if (T == 'N') return theta_tet(P, X, st) && tet_scaling(P, X, 0.5, 1.0, nlm, st);
        return tet_scaling(P, X, 1.0, 1.0, nlm, st) && theta_tet(P, X, st);
    }
    if (op == TRI_SYN || op == TRI_ANA) {     // src/fftw.c:292-330
        if (N <= 1 || M <= 1) return true;
        const double nm = (double) N * M;
        if (op == TRI_SYN) return tri_scaling(P, X, T == 'N' ? 2.0 : 1.0, 0.25, 0.0, st) && theta_tri(P, X, st);
        if (T == 'N') return theta_tri(P, X, st) && tri_scaling(P, X, 0.5, 1.0, nm, st);
        return tri_scaling(P, X, 1.0, 1.0, nm, st) && theta_tri(P, X, st);
    }
    const bool sph = op == SPH_SYN || op == SPH_ANA;
    auto first = [&](double f) { return sph ? ends(P, X, false, 0, 3, f, st) : ends(P, X, false, -1, 1, f, st); };
    auto last = [&](double f) { return sph ? ends(P, X, true, -1, 1, f, st) : ends(P, X, true, 0, 3, f, st); };
    if (op == SPH_SYN || op == SPHV_SYN) {
        if (T == 'N') return first(2.0) && theta(P, X, st) && phi_c2r(P, X, C_1_4_SQRT_PI, C_SQRT2, st);
        return phi_r2c(P, X, C_1_2_SQRT_PI, C_SQRT1_2, st) && theta(P, X, st) && last(0.5);
    }
    if (T == 'N') return phi_r2c(P, X, C_4_SQRT_PI / nm2, C_SQRT1_2, st) && theta(P, X, st) && first(0.5);
    return last(2.0) && theta(P, X, st) && phi_c2r(P, X, C_2_SQRT_PI / nm2, C_SQRT2, st);
}

SphereGridPlan * as_grid(const ft_sphere_fftw_plan * P) {
    SphereGridPlan * G = reinterpret_cast<SphereGridPlan *>(const_cast<ft_sphere_fftw_plan *>(P));
    return (G && G->magic == kGridMagic) ? G : nullptr;
}

int family_of(int op) {
    if (op <= SPHV_ANA) return F_SPHERE;
    if (op <= DISK_ANA) return F_DISK;
    if (op <= TRI_ANA) return F_TRI;
    if (op <= ANN_ANA) return F_ANN;
    if (op <= RECT_ANA) return F_RECT;
    return op <= TET_ANA ? F_TET : F_SPIN;
}

int check_call(SphereGridPlan * G, char T, const double * X, int N, int M, int family = F_SPHERE) {
    if (!G || G->family != family) { set_error(FT_B200_EINVAL, "not a grid plan of this family of this library"); return FT_B200_EINVAL; }
    // spin: 'N' and 'C' run, any other TRANS leaves X untouched, as the reference's (its own
    // round-trip test, test/test_fftw.c:504-505, passes 'T')
    if (family != F_SPIN && T != 'N' && T != 'T') { set_error(FT_B200_EINVAL, "TRANS must be 'N' or 'T'"); return FT_B200_EINVAL; }
    if (!X) { set_error(FT_B200_EINVAL, "NULL matrix"); return FT_B200_EINVAL; }
    if (N != G->N || M != G->M) { set_error(FT_B200_EINVAL, "N, M do not match the plan"); return FT_B200_EINVAL; }
    return FT_B200_OK;
}

void execute_host(int op, char T, const void * P, double * X, int N, int M) {
    clear_error();
    SphereGridPlan * G = as_grid(static_cast<const ft_sphere_fftw_plan *>(P));
    if (check_call(G, T, X, N, M, family_of(op)) != FT_B200_OK) return;
    if (G->family == F_SPIN && T != 'N' && T != 'C') return;
    std::lock_guard<std::mutex> lk(G->mu);
    cudaSetDevice(G->device);
    const size_t bytes = sizeof(double) * (size_t) N * M * (G->family == F_SPIN ? 2 : 1);   // spin: complex
    if (!G->d_stage && !ok(cudaMalloc(&G->d_stage, bytes), "cudaMalloc(grid stage)")) return;
    if (!ok(cudaMemcpyAsync(G->d_stage, X, bytes, cudaMemcpyHostToDevice, G->stream), "cudaMemcpyAsync(H2D)")) return;
    if (!run(G, op, T, G->d_stage, G->stream)) return;
    if (!ok(cudaMemcpyAsync(X, G->d_stage, bytes, cudaMemcpyDeviceToHost, G->stream), "cudaMemcpyAsync(D2H)")) return;
    ok(cudaStreamSynchronize(G->stream), "cudaStreamSynchronize");
}

}  // namespace
}  // namespace ftb

using namespace ftb;

extern "C" {

ft_sphere_fftw_plan * ft_plan_sph_synthesis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_sphere_fftw_plan *>(make_plan(N, M, K_REDFT01, K_RODFT01));
}
ft_sphere_fftw_plan * ft_plan_sph_analysis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_sphere_fftw_plan *>(make_plan(N, M, K_REDFT10, K_RODFT10));
}
ft_sphere_fftw_plan * ft_plan_sphv_synthesis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_sphere_fftw_plan *>(make_plan(N, M, K_RODFT01, K_REDFT01));
}
ft_sphere_fftw_plan * ft_plan_sphv_analysis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_sphere_fftw_plan *>(make_plan(N, M, K_RODFT10, K_REDFT10));
}

void ft_destroy_sphere_fftw_plan(ft_sphere_fftw_plan * Pp) {
    SphereGridPlan * P = as_grid(Pp);
    if (!P) return;
    if (P->have_t_r2c) cufftDestroy(P->t_r2c);
    if (P->have_t_c2r) cufftDestroy(P->t_c2r);
    if (P->have_p_r2c) cufftDestroy(P->p_r2c);
    if (P->have_p_c2r) cufftDestroy(P->p_c2r);
    if (P->have_t4) cufftDestroy(P->t4);
    if (P->have_p_z2z) cufftDestroy(P->p_z2z);
    cudaFree(P->d_work); cudaFree(P->d_cwork); cudaFree(P->d_Y); cudaFree(P->d_stage); cudaFree(P->d_u); cudaFree(P->d_work2);
    cudaFree(P->d_w);
    if (P->stream) cudaStreamDestroy(P->stream);
    P->magic = 0;
    delete P;
}

void ft_execute_sph_synthesis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(SPH_SYN, TRANS, P, X, N, M);
}
void ft_execute_sph_analysis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(SPH_ANA, TRANS, P, X, N, M);
}
void ft_execute_sphv_synthesis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(SPHV_SYN, TRANS, P, X, N, M);
}
void ft_execute_sphv_analysis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(SPHV_ANA, TRANS, P, X, N, M);
}

ft_disk_fftw_plan * ft_plan_disk_synthesis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_disk_fftw_plan *>(make_plan(N, M, K_REDFT01, K_REDFT11, F_DISK));
}
ft_disk_fftw_plan * ft_plan_disk_analysis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_disk_fftw_plan *>(make_plan(N, M, K_REDFT10, K_REDFT11, F_DISK));
}
void ft_destroy_disk_fftw_plan(ft_disk_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    if (G && G->family == F_DISK) ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
}
void ft_execute_disk_synthesis(const char TRANS, const ft_disk_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(DISK_SYN, TRANS, P, X, N, M);
}
void ft_execute_disk_analysis(const char TRANS, const ft_disk_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(DISK_ANA, TRANS, P, X, N, M);
}

ft_triangle_fftw_plan * ft_plan_tri_synthesis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_triangle_fftw_plan *>(make_plan(N, M, K_REDFT01, K_REDFT01, F_TRI));
}
ft_triangle_fftw_plan * ft_plan_tri_analysis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_triangle_fftw_plan *>(make_plan(N, M, K_REDFT10, K_REDFT10, F_TRI));
}
void ft_destroy_triangle_fftw_plan(ft_triangle_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    if (G && G->family == F_TRI) ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
}
void ft_execute_tri_synthesis(const char TRANS, const ft_triangle_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(TRI_SYN, TRANS, P, X, N, M);
}
void ft_execute_tri_analysis(const char TRANS, const ft_triangle_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(TRI_ANA, TRANS, P, X, N, M);
}

ft_annulus_fftw_plan * ft_plan_annulus_synthesis(const int N, const int M, const double rho, const unsigned) {
    return reinterpret_cast<ft_annulus_fftw_plan *>(make_plan(N, M, K_REDFT01, K_REDFT01, F_ANN, 0, rho));
}
ft_annulus_fftw_plan * ft_plan_annulus_analysis(const int N, const int M, const double rho, const unsigned) {
    return reinterpret_cast<ft_annulus_fftw_plan *>(make_plan(N, M, K_REDFT10, K_REDFT10, F_ANN, 0, rho));
}
void ft_destroy_annulus_fftw_plan(ft_annulus_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    if (G && G->family == F_ANN) ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
}
double ft_get_rho_annulus_fftw_plan(ft_annulus_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    return (G && G->family == F_ANN) ? G->rho : 0.0;
}
void ft_execute_annulus_synthesis(const char TRANS, const ft_annulus_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(ANN_SYN, TRANS, P, X, N, M);
}
void ft_execute_annulus_analysis(const char TRANS, const ft_annulus_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(ANN_ANA, TRANS, P, X, N, M);
}

ft_rectdisk_fftw_plan * ft_plan_rectdisk_synthesis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_rectdisk_fftw_plan *>(make_plan(N, M, K_REDFT01, K_RODFT01, F_RECT, K_REDFT01));
}
ft_rectdisk_fftw_plan * ft_plan_rectdisk_analysis(const int N, const int M, const unsigned) {
    return reinterpret_cast<ft_rectdisk_fftw_plan *>(make_plan(N, M, K_REDFT10, K_RODFT10, F_RECT, K_REDFT10));
}
void ft_destroy_rectdisk_fftw_plan(ft_rectdisk_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    if (G && G->family == F_RECT) ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
}
void ft_execute_rectdisk_synthesis(const char TRANS, const ft_rectdisk_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(RECT_SYN, TRANS, P, X, N, M);
}
void ft_execute_rectdisk_analysis(const char TRANS, const ft_rectdisk_fftw_plan * P, double * X, const int N, const int M) {
    execute_host(RECT_ANA, TRANS, P, X, N, M);
}

// the tetrahedron's grids: N = L = M = n, the tensor as the n x n^2 matrix of its columns
static ft_tetrahedron_fftw_plan * tet_grid_plan(int N, int L, int M, int kind) {
    clear_error();
    if (N < 1 || L != N || M != N) {
        set_error(FT_B200_EINVAL, "tetrahedral grids need N = L = M (the reference's 3-D plan reads the tensor in reverse)");
        return nullptr;
    }
    return reinterpret_cast<ft_tetrahedron_fftw_plan *>(make_plan(N, N * N, kind, kind, F_TET));
}
ft_tetrahedron_fftw_plan * ft_plan_tet_synthesis(const int N, const int L, const int M, const unsigned) {
    return tet_grid_plan(N, L, M, K_REDFT01);
}
ft_tetrahedron_fftw_plan * ft_plan_tet_analysis(const int N, const int L, const int M, const unsigned) {
    return tet_grid_plan(N, L, M, K_REDFT10);
}
void ft_destroy_tetrahedron_fftw_plan(ft_tetrahedron_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    if (G && G->family == F_TET) ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
}
static int tet_dims(const void * P, int N, int L, int M, int * cols) {
    const SphereGridPlan * G = as_grid(static_cast<const ft_sphere_fftw_plan *>(P));
    if (!G || G->family != F_TET || L != N || M != N || N != G->N) {
        set_error(FT_B200_EINVAL, "not a tetrahedral grid plan of this size");
        return FT_B200_EINVAL;
    }
    *cols = L * M;
    return FT_B200_OK;
}
void ft_execute_tet_synthesis(const char TRANS, const ft_tetrahedron_fftw_plan * P, double * X, const int N, const int L, const int M) {
    clear_error();
    int cols = 0;
    if (tet_dims(P, N, L, M, &cols) == FT_B200_OK) execute_host(TET_SYN, TRANS, P, X, N, cols);
}
void ft_execute_tet_analysis(const char TRANS, const ft_tetrahedron_fftw_plan * P, double * X, const int N, const int L, const int M) {
    clear_error();
    int cols = 0;
    if (tet_dims(P, N, L, M, &cols) == FT_B200_OK) execute_host(TET_ANA, TRANS, P, X, N, cols);
}
int ft_b200_execute_tet_grid_dev(const ft_tetrahedron_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int L, int M,
                                 void * stream) {
    clear_error();
    int cols = 0;
    if (tet_dims(P, N, L, M, &cols) != FT_B200_OK) return FT_B200_EINVAL;
    SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    const int c = check_call(G, TRANS, dX, N, cols, F_TET);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, analysis ? TET_ANA : TET_SYN, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

int ft_b200_execute_annulus_grid_dev(const ft_annulus_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream) {
    clear_error();
    SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    const int c = check_call(G, TRANS, dX, N, M, F_ANN);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, analysis ? ANN_ANA : ANN_SYN, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

int ft_b200_execute_rectdisk_grid_dev(const ft_rectdisk_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream) {
    clear_error();
    SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    const int c = check_call(G, TRANS, dX, N, M, F_RECT);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, analysis ? RECT_ANA : RECT_SYN, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

int ft_b200_execute_disk_grid_dev(const ft_disk_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream) {
    clear_error();
    SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    const int c = check_call(G, TRANS, dX, N, M, F_DISK);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, analysis ? DISK_ANA : DISK_SYN, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

int ft_b200_execute_tri_grid_dev(const ft_triangle_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream) {
    clear_error();
    SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    const int c = check_call(G, TRANS, dX, N, M, F_TRI);
    if (c != FT_B200_OK) return c;
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, analysis ? TRI_ANA : TRI_SYN, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

// ---------------------------------------------------------------------------
// plans with caller-chosen kinds (src/fftw.c:76-102, 281-288, 340-347, 414-449, 534-571, 660-686,
// 755-787).  The kinds are FFTW's r2r constants.  Accepted: the combinations this file's
// kernels compute -- cosine and sine kinds of type II (REDFT10, RODFT10) or III (REDFT01,
// RODFT01), one type per plan, REDFT11 as the disk's second kind, the phi kind R2HC or HC2R (which
// of the two is not used: every plan here holds both row transforms) -- and FT_B200_EUNSUPPORTED
// otherwise.
// ---------------------------------------------------------------------------
static bool theta_kind(int k) { return k == K_REDFT01 || k == K_REDFT10 || k == K_RODFT01 || k == K_RODFT10; }
static bool kinds_ok(bool good) {
    clear_error();
    if (!good) set_error(FT_B200_EUNSUPPORTED, "transform kinds not supported by these grid plans");
    return good;
}
static bool phi_kind(int k) { return k == 0 || k == 1; }   // FFTW_R2HC, FFTW_HC2R

ft_sphere_fftw_plan * ft_plan_sph_with_kind(const int N, const int M, const int kind[3][1], const unsigned) {
    if (!kind || !kinds_ok(theta_kind(kind[0][0]) && theta_kind(kind[1][0]) && is_type3(kind[0][0]) == is_type3(kind[1][0]) &&
                           phi_kind(kind[2][0]))) return nullptr;
    return reinterpret_cast<ft_sphere_fftw_plan *>(make_plan(N, M, kind[0][0], kind[1][0]));
}
ft_disk_fftw_plan * ft_plan_disk_with_kind(const int N, const int M, const int kind[3][1], const unsigned) {
    if (!kind || !kinds_ok(theta_kind(kind[0][0]) && kind[1][0] == K_REDFT11 && phi_kind(kind[2][0]))) return nullptr;
    return reinterpret_cast<ft_disk_fftw_plan *>(make_plan(N, M, kind[0][0], K_REDFT11, F_DISK));
}
ft_triangle_fftw_plan * ft_plan_tri_with_kind(const int N, const int M, const int kind0, const int kind1, const unsigned) {
    if (!kinds_ok(kind0 == kind1 && (kind0 == K_REDFT01 || kind0 == K_REDFT10))) return nullptr;
    return reinterpret_cast<ft_triangle_fftw_plan *>(make_plan(N, M, kind0, kind0, F_TRI));
}
ft_annulus_fftw_plan * ft_plan_annulus_with_kind(const int N, const int M, const double rho, const int kind[2][1], const unsigned) {
    if (!kind || !kinds_ok((kind[0][0] == K_REDFT01 || kind[0][0] == K_REDFT10) && phi_kind(kind[1][0]))) return nullptr;
    return reinterpret_cast<ft_annulus_fftw_plan *>(make_plan(N, M, kind[0][0], kind[0][0], F_ANN, 0, rho));
}
ft_rectdisk_fftw_plan * ft_plan_rectdisk_with_kind(const int N, const int M, const int kind[3][1], const unsigned) {
    if (!kind || !kinds_ok(theta_kind(kind[0][0]) && theta_kind(kind[1][0]) && theta_kind(kind[2][0]) &&
                           is_type3(kind[0][0]) == is_type3(kind[1][0]) && is_type3(kind[0][0]) == is_type3(kind[2][0])))
        return nullptr;
    return reinterpret_cast<ft_rectdisk_fftw_plan *>(make_plan(N, M, kind[0][0], kind[1][0], F_RECT, kind[2][0]));
}
ft_tetrahedron_fftw_plan * ft_plan_tet_with_kind(const int N, const int L, const int M, const int kind0, const int kind1, const int kind2,
                                                 const unsigned) {
    if (!kinds_ok(kind0 == kind1 && kind1 == kind2 && (kind0 == K_REDFT01 || kind0 == K_REDFT10))) return nullptr;
    return tet_grid_plan(N, L, M, kind0);
}
ft_spinsphere_fftw_plan * ft_plan_spinsph_with_kind(const int N, const int M, const int S, const int kind[2][1], const int sign,
                                                    const unsigned) {
    if (!kind || !kinds_ok(theta_kind(kind[0][0]) && theta_kind(kind[1][0]) && is_type3(kind[0][0]) == is_type3(kind[1][0]) &&
                           (sign == 1 || sign == -1))) return nullptr;
    SphereGridPlan * P = make_plan(N, M, kind[0][0], kind[1][0], F_SPIN);
    if (P) { P->spin = S; P->zsign = sign; }
    return reinterpret_cast<ft_spinsphere_fftw_plan *>(P);
}

// the spin-weighted sphere's grids (src/fftw.c:743-960): kinds by the parity of S
static ft_spinsphere_fftw_plan * spin_grid_plan(int N, int M, int S, bool analysis) {
    const bool even = S % 2 == 0;
    const int k0 = analysis ? (even ? K_REDFT10 : K_RODFT10) : (even ? K_REDFT01 : K_RODFT01);
    const int k1 = analysis ? (even ? K_RODFT10 : K_REDFT10) : (even ? K_RODFT01 : K_REDFT01);
    SphereGridPlan * P = make_plan(N, M, k0, k1, F_SPIN);
    if (P) P->spin = S;
    return reinterpret_cast<ft_spinsphere_fftw_plan *>(P);
}
ft_spinsphere_fftw_plan * ft_plan_spinsph_synthesis(const int N, const int M, const int S, const unsigned) {
    return spin_grid_plan(N, M, S, false);
}
ft_spinsphere_fftw_plan * ft_plan_spinsph_analysis(const int N, const int M, const int S, const unsigned) {
    return spin_grid_plan(N, M, S, true);
}
void ft_destroy_spinsphere_fftw_plan(ft_spinsphere_fftw_plan * P) {
    SphereGridPlan * G = as_grid(reinterpret_cast<ft_sphere_fftw_plan *>(P));
    if (G && G->family == F_SPIN) ft_destroy_sphere_fftw_plan(reinterpret_cast<ft_sphere_fftw_plan *>(P));
}
int ft_get_spin_spinsphere_fftw_plan(const ft_spinsphere_fftw_plan * P) {
    const SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    return (G && G->family == F_SPIN) ? G->spin : 0;
}
void ft_execute_spinsph_synthesis(const char TRANS, const ft_spinsphere_fftw_plan * P, ft_complex * X, const int N, const int M) {
    execute_host(SPIN_SYN, TRANS, P, reinterpret_cast<double *>(X), N, M);
}
void ft_execute_spinsph_analysis(const char TRANS, const ft_spinsphere_fftw_plan * P, ft_complex * X, const int N, const int M) {
    execute_host(SPIN_ANA, TRANS, P, reinterpret_cast<double *>(X), N, M);
}
int ft_b200_execute_spinsph_grid_dev(const ft_spinsphere_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M,
                                     void * stream) {
    clear_error();
    SphereGridPlan * G = as_grid(reinterpret_cast<const ft_sphere_fftw_plan *>(P));
    const int c = check_call(G, TRANS, dX, N, M, F_SPIN);
    if (c != FT_B200_OK) return c;
    if (reinterpret_cast<uintptr_t>(dX) % 16 != 0) {   // cuFFT's complex operands
        set_error(FT_B200_EINVAL, "dX must be 16-byte aligned (complex doubles)");
        return FT_B200_EINVAL;
    }
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, analysis ? SPIN_ANA : SPIN_SYN, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

int ft_b200_execute_sph_grid_dev(const ft_sphere_fftw_plan * P, int op, char TRANS, double * dX, int N, int M, void * stream) {
    clear_error();
    SphereGridPlan * G = as_grid(P);
    const int c = check_call(G, TRANS, dX, N, M);
    if (c != FT_B200_OK) return c;
    if (op < SPH_SYN || op > SPHV_ANA) { set_error(FT_B200_EINVAL, "op must be 0 .. 3"); return FT_B200_EINVAL; }
    std::lock_guard<std::mutex> lk(G->mu);
    return run(G, op, TRANS, dX, static_cast<cudaStream_t>(stream)) ? FT_B200_OK : ft_b200_last_status();
}

}  // extern "C"
