/*
 * ft_b200.h -- C ABI of the B200 (sm_100a) harmonic-conversion library.
 *
 * Drop-in for FastTransforms' harmonic-conversion path: the Givens-rotation
 * sweeps behind sph2fourier / fourier2sph and the same kernel family used by
 * tri2cheb / cheb2tri and disk2cxf / cxf2disk, with the sphere's vector-field and
 * spin-weighted transforms, the Dunkl-Xu, annulus and tetrahedral transforms and
 * the sphere, disk and triangle grids.  Link with -lft_b200 instead of
 * -lfasttransforms; existing callers of the functions below need no change.
 *
 * Conventions (identical to the reference):
 *   - A is column-major with leading dimension N (host memory for the drop-in
 *     entry points, device memory for the *_dev entry points);
 *     M = 2N-1 (sph, spin), N (tri, rectdisk), 4N-3 (disk, annulus);
 *     N x L x M tensors for the tetrahedron.
 *   - Column pair (2m-1, 2m) carries order m for sph and disk; column m for tri.
 *   - TRANS 'N' applies the operator, 'T' its transpose; any other character
 *     is a no-op (the reference silently ignores it; here the status is
 *     FT_B200_EINVAL and A is left untouched).
 *   - In place on A.  ft_b200_execute_dev and ft_b200_execute_sphv_dev on sph,
 *     tri and disk plans are reentrant: each call takes its scratch matrix,
 *     work counter and progress words from the library's stream-ordered memory
 *     pool on its own stream (freed there after its work), so calls on ONE plan
 *     may run concurrently from several threads on several streams.  The pool
 *     keeps what it has handed out (at most the peak of concurrent calls) for
 *     reuse until the process exits.  The
 *     host-pointer calls (ft_execute_*) on one plan share its staging buffer
 *     and stream and run one at a time (a call from another thread waits).
 *     Every other entry point keeps plan-owned scratch, as the reference's plan
 *     owns P->B: concurrent calls on one such plan are not reentrant.  Different
 *     plans may run concurrently on different streams.
 *
 * Everything runs on the current CUDA device.  There is no CPU fallback: if no
 * sm_100 device is present, plan creation fails (NULL) and the status says why.
 */
#ifndef FT_B200_H
#define FT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes and errors (the reference has none: it prints and exits).   */
/* ------------------------------------------------------------------------ */
#define FT_B200_OK          0
#define FT_B200_EINVAL      1   /* bad TRANS, sizes that do not match the plan, NULL pointers */
#define FT_B200_ECUDA       2   /* a CUDA runtime call failed (message has the CUDA error) */
#define FT_B200_ENOMEM      3   /* device or host allocation failed */
#define FT_B200_ENODEV      4   /* no usable sm_100 device */
#define FT_B200_ETIMEOUT    5   /* a bounded device-side wait ran out (queue stalled) */
#define FT_B200_EUNSUPPORTED 6  /* option not supported for this plan kind */

/* Status of the last call made on this host thread (0 = success). */
int ft_b200_last_status(void);
/* Human-readable message for the last failure on this host thread ("" if none). */
const char * ft_b200_last_error(void);

/* ------------------------------------------------------------------------ */
/* Plan structures.                                                         */
/* ------------------------------------------------------------------------ */

/* Rotation plan.  The first three members are layout-compatible with the
 * reference's struct (src/ftinternal.h:370-374): host copies of the sine and
 * cosine tables in the reference's packing, and n.  The rest is device state. */
typedef struct ft_rotation_plan_s ft_rotation_plan;

/* Harmonic plan.  Layout-compatible prefix with the reference's public struct
 * (src/fasttransforms.h:370-385): RP, MP, B, P, Pinv, alpha..rho, NRP, NMP, NP,
 * with host copies of the connection matrices in P / Pinv and NULL MP.  B is a
 * device pointer to the plan's scratch (the reference's host scratch). */
typedef struct {
    ft_rotation_plan ** RP;
    void ** MP;
    double * B;
    double ** P;
    double ** Pinv;
    double alpha;
    double beta;
    double gamma;
    double delta;
    double rho;
    int NRP;
    int NMP;
    int NP;
} ft_harmonic_plan;

/* ------------------------------------------------------------------------ */
/* Drop-in entry points: same names, signatures and meaning as the          */
/* reference (src/fasttransforms.h:297-415).  Host pointers.  Errors are    */
/* reported through ft_b200_last_status() / ft_b200_last_error().           */
/* ------------------------------------------------------------------------ */

/* replaces ft_plan_sph2fourier, src/drivers.c:816-831 */
ft_harmonic_plan * ft_plan_sph2fourier(const int n);
/* replaces ft_execute_sph2fourier, src/drivers.c:833-848 */
void ft_execute_sph2fourier(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);
/* replaces ft_execute_fourier2sph, src/drivers.c:850-865 */
void ft_execute_fourier2sph(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);

/* replaces ft_execute_sphv2fourier, src/drivers.c:867-882: vector fields on a sph plan
 * (order m's sweeps on columns 2m+1, 2m+2; P[0] and P[1] swapped in the column classes) */
void ft_execute_sphv2fourier(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);
/* replaces ft_execute_fourier2sphv, src/drivers.c:884-899 */
void ft_execute_fourier2sphv(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);

/* replaces ft_plan_tri2cheb, src/drivers.c:901-919 */
ft_harmonic_plan * ft_plan_tri2cheb(const int n, const double alpha, const double beta, const double gamma);
/* replaces ft_execute_tri2cheb, src/drivers.c:921-938 */
void ft_execute_tri2cheb(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);
/* replaces ft_execute_cheb2tri, src/drivers.c:940-957 */
void ft_execute_cheb2tri(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);

/* replaces ft_plan_disk2cxf, src/drivers.c:959-987 */
ft_harmonic_plan * ft_plan_disk2cxf(const int n, const double alpha, const double beta);
/* replaces ft_execute_disk2cxf, src/drivers.c:989-1004 */
void ft_execute_disk2cxf(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);
/* replaces ft_execute_cxf2disk, src/drivers.c:1006-1021 */
void ft_execute_cxf2disk(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);

/* replaces ft_plan_rectdisk2cheb, src/drivers.c:1123-1141: Dunkl-Xu (rectangularised disk)
 * transforms; the plan has NP = 3 connection pairs in P / Pinv (host copies) */
ft_harmonic_plan * ft_plan_rectdisk2cheb(const int n, const double beta);
/* replace ft_execute_rectdisk2cheb / ft_execute_cheb2rectdisk, src/drivers.c:1143-1171;
 * M must equal N (the right multiply is n x n), as in the reference's tests */
void ft_execute_rectdisk2cheb(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);
void ft_execute_cheb2rectdisk(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);

/* replaces ft_plan_ann2cxf, src/drivers.c:1023-1071: annulus harmonics (the disk layout,
 * M = 4N - 3); gamma must be 0 (the reference implements no other: it warns), else NULL with
 * FT_B200_EUNSUPPORTED.  NRP = 1, NP = 1; the two modified plans (identity and the Cholesky
 * factor of t I + X) are held on the device: NMP = 2, MP = NULL. */
ft_harmonic_plan * ft_plan_ann2cxf(const int n, const double alpha, const double beta, const double gamma, const double rho);
/* replace ft_execute_ann2cxf / ft_execute_cxf2ann, src/drivers.c:1073-1121 */
void ft_execute_ann2cxf(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);
void ft_execute_cxf2ann(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int M);

/* replaces ft_plan_tet2cheb, src/drivers.c:1173-1195: tetrahedral harmonics; NRP = 2 rotation
 * plans (triangle tables), NP = 3 connection pairs (host copies) */
ft_harmonic_plan * ft_plan_tet2cheb(const int n, const double alpha, const double beta, const double gamma, const double delta);
/* replace ft_execute_tet2cheb / ft_execute_cheb2tet, src/drivers.c:1197-1257: A is N x L x M
 * column-major (entry (i, l, m) at i + N l + N L m); L and M must equal N, as in the
 * reference's tests (its multiplies along l and m are n x n) */
void ft_execute_tet2cheb(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int L, const int M);
void ft_execute_cheb2tet(const char TRANS, const ft_harmonic_plan * P, double * A, const int N, const int L, const int M);

/* replaces ft_destroy_harmonic_plan, src/drivers.c:793-814 (every plan kind above) */
void ft_destroy_harmonic_plan(ft_harmonic_plan * P);

/* Synthesis and analysis on the sphere's grid (theta_i = (i + 1/2) pi / N,
 * phi_k = 2 pi k / M), src/fftw.c.  The plan type is this library's own (the
 * reference's holds FFTW plans); the flags argument is accepted and not used.
 * M must be odd.  Host-pointer calls stage X on the device and synchronise;
 * ft_b200_execute_sph_grid_dev is the device-pointer form. */
typedef struct ft_sphere_fftw_plan_s ft_sphere_fftw_plan;
/* replace ft_plan_sph_synthesis / ft_plan_sph_analysis, src/fftw.c:104-112 */
ft_sphere_fftw_plan * ft_plan_sph_synthesis(const int N, const int M, const unsigned flags);
ft_sphere_fftw_plan * ft_plan_sph_analysis(const int N, const int M, const unsigned flags);
/* replace ft_plan_sphv_synthesis / ft_plan_sphv_analysis, src/fftw.c:114-122 */
ft_sphere_fftw_plan * ft_plan_sphv_synthesis(const int N, const int M, const unsigned flags);
ft_sphere_fftw_plan * ft_plan_sphv_analysis(const int N, const int M, const unsigned flags);
/* replaces ft_destroy_sphere_fftw_plan, src/fftw.c:66-74 */
void ft_destroy_sphere_fftw_plan(ft_sphere_fftw_plan * P);
/* replace ft_execute_sph_synthesis / ft_execute_sph_analysis, src/fftw.c:124-200 */
void ft_execute_sph_synthesis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M);
void ft_execute_sph_analysis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M);
/* replace ft_execute_sphv_synthesis / ft_execute_sphv_analysis, src/fftw.c:202-277 */
void ft_execute_sphv_synthesis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M);
void ft_execute_sphv_analysis(const char TRANS, const ft_sphere_fftw_plan * P, double * X, const int N, const int M);
/* the reference's flags for these planners (src/ftutilities.h:24); not used here */
#define FT_FFTW_FLAGS 0u

/* Synthesis and analysis on the disk's grid (src/fftw.c:404-532) and the triangle's
 * (src/fftw.c:279-330); this library's own plan types, flags not used.  Disk: M odd (the
 * reference's M = 4N - 3).  Triangle: M must equal N (the reference's 2-D plan reads the
 * column-major matrix as row-major, which agrees only when M == N). */
typedef struct ft_disk_fftw_plan_s ft_disk_fftw_plan;
/* replace ft_plan_disk_synthesis / ft_plan_disk_analysis, src/fftw.c:450-458 */
ft_disk_fftw_plan * ft_plan_disk_synthesis(const int N, const int M, const unsigned flags);
ft_disk_fftw_plan * ft_plan_disk_analysis(const int N, const int M, const unsigned flags);
/* replaces ft_destroy_disk_fftw_plan, src/fftw.c:404-412 */
void ft_destroy_disk_fftw_plan(ft_disk_fftw_plan * P);
/* replace ft_execute_disk_synthesis / ft_execute_disk_analysis, src/fftw.c:460-532 */
void ft_execute_disk_synthesis(const char TRANS, const ft_disk_fftw_plan * P, double * X, const int N, const int M);
void ft_execute_disk_analysis(const char TRANS, const ft_disk_fftw_plan * P, double * X, const int N, const int M);
typedef struct ft_triangle_fftw_plan_s ft_triangle_fftw_plan;
/* replace ft_plan_tri_synthesis / ft_plan_tri_analysis, src/fftw.c:289-290 */
ft_triangle_fftw_plan * ft_plan_tri_synthesis(const int N, const int M, const unsigned flags);
ft_triangle_fftw_plan * ft_plan_tri_analysis(const int N, const int M, const unsigned flags);
/* replaces ft_destroy_triangle_fftw_plan, src/fftw.c:276-279 */
void ft_destroy_triangle_fftw_plan(ft_triangle_fftw_plan * P);
/* replace ft_execute_tri_synthesis / ft_execute_tri_analysis, src/fftw.c:292-330 */
void ft_execute_tri_synthesis(const char TRANS, const ft_triangle_fftw_plan * P, double * X, const int N, const int M);
void ft_execute_tri_analysis(const char TRANS, const ft_triangle_fftw_plan * P, double * X, const int N, const int M);

/* Annulus grids (src/fftw.c:534-658): M odd (the reference's M = 4N - 3), rho the radius ratio. */
typedef struct ft_annulus_fftw_plan_s ft_annulus_fftw_plan;
/* replace ft_plan_annulus_synthesis / ft_plan_annulus_analysis, src/fftw.c:573-581 */
ft_annulus_fftw_plan * ft_plan_annulus_synthesis(const int N, const int M, const double rho, const unsigned flags);
ft_annulus_fftw_plan * ft_plan_annulus_analysis(const int N, const int M, const double rho, const unsigned flags);
/* replaces ft_destroy_annulus_fftw_plan, src/fftw.c:524-530 */
void ft_destroy_annulus_fftw_plan(ft_annulus_fftw_plan * P);
/* replaces ft_get_rho_annulus_fftw_plan, src/fftw.c:532 */
double ft_get_rho_annulus_fftw_plan(ft_annulus_fftw_plan * P);
/* replace ft_execute_annulus_synthesis / ft_execute_annulus_analysis, src/fftw.c:583-658 */
void ft_execute_annulus_synthesis(const char TRANS, const ft_annulus_fftw_plan * P, double * X, const int N, const int M);
void ft_execute_annulus_analysis(const char TRANS, const ft_annulus_fftw_plan * P, double * X, const int N, const int M);

/* Tetrahedral grids (src/fftw.c:332-402): N = L = M (the reference's 3-D plan reads the
 * column-major tensor in reverse order, which agrees only for a cube). */
typedef struct ft_tetrahedron_fftw_plan_s ft_tetrahedron_fftw_plan;
/* replace ft_plan_tet_synthesis / ft_plan_tet_analysis, src/fftw.c:348-349 */
ft_tetrahedron_fftw_plan * ft_plan_tet_synthesis(const int N, const int L, const int M, const unsigned flags);
ft_tetrahedron_fftw_plan * ft_plan_tet_analysis(const int N, const int L, const int M, const unsigned flags);
/* replaces ft_destroy_tetrahedron_fftw_plan, src/fftw.c:335-338 */
void ft_destroy_tetrahedron_fftw_plan(ft_tetrahedron_fftw_plan * P);
/* replace ft_execute_tet_synthesis / ft_execute_tet_analysis, src/fftw.c:351-402 */
void ft_execute_tet_synthesis(const char TRANS, const ft_tetrahedron_fftw_plan * P, double * X, const int N, const int L, const int M);
void ft_execute_tet_analysis(const char TRANS, const ft_tetrahedron_fftw_plan * P, double * X, const int N, const int L, const int M);

/* Dunkl-Xu (rectangularised disk) grids (src/fftw.c:653-753): M must equal N here (the rows go
 * through a square transpose; the reference's tests use M = N). */
typedef struct ft_rectdisk_fftw_plan_s ft_rectdisk_fftw_plan;
/* replace ft_plan_rectdisk_synthesis / ft_plan_rectdisk_analysis, src/fftw.c:687-695 */
ft_rectdisk_fftw_plan * ft_plan_rectdisk_synthesis(const int N, const int M, const unsigned flags);
ft_rectdisk_fftw_plan * ft_plan_rectdisk_analysis(const int N, const int M, const unsigned flags);
/* replaces ft_destroy_rectdisk_fftw_plan, src/fftw.c:653-658 */
void ft_destroy_rectdisk_fftw_plan(ft_rectdisk_fftw_plan * P);
/* replace ft_execute_rectdisk_synthesis / ft_execute_rectdisk_analysis, src/fftw.c:697-753 */
void ft_execute_rectdisk_synthesis(const char TRANS, const ft_rectdisk_fftw_plan * P, double * X, const int N, const int M);
void ft_execute_rectdisk_analysis(const char TRANS, const ft_rectdisk_fftw_plan * P, double * X, const int N, const int M);

/* Spin-weighted spherical harmonics.  Complex matrices are interleaved (re, im)
 * doubles, N x M column-major: column 0 holds order 0, columns 2m - 1 and 2m the
 * orders -m and m (src/drivers.c:645-695).  M must be odd. */
typedef double ft_complex[2];   /* src/fasttransforms.h:11 */
/* Opaque, as in the reference's public header (src/fasttransforms.h:336). */
typedef struct ft_spin_rotation_plan_s ft_spin_rotation_plan;
/* replaces ft_plan_rotspinsphere, src/rotations.c:445-478 */
ft_spin_rotation_plan * ft_plan_rotspinsphere(const int n, const int s);
/* replaces ft_destroy_spin_rotation_plan, src/rotations.c:431-437 */
void ft_destroy_spin_rotation_plan(ft_spin_rotation_plan * SRP);
/* replace ft_execute_spinsph_hi2lo / lo2hi, src/drivers.c:645-675; B (the reference's
 * scratch) is accepted and not used */
void ft_execute_spinsph_hi2lo(const ft_spin_rotation_plan * SRP, ft_complex * A, ft_complex * B, const int M);
void ft_execute_spinsph_lo2hi(const ft_spin_rotation_plan * SRP, ft_complex * A, ft_complex * B, const int M);
/* replace ft_kernel_spinsph_hi2lo / lo2hi, src/rotations.c:479-485: one host column A of order m
 * (stride S >= 1 complex entries); only the entries the sweeps touch are read and written. */
void ft_kernel_spinsph_hi2lo(const ft_spin_rotation_plan * SRP, const int m, ft_complex * A, const int S);
void ft_kernel_spinsph_lo2hi(const ft_spin_rotation_plan * SRP, const int m, ft_complex * A, const int S);
/* Same members as the reference's (src/fasttransforms.h:441-450).  P1 .. P2inv are
 * host copies of the connection matrices (the real sph matrices stored as complex);
 * B is NULL. */
typedef struct {
    ft_spin_rotation_plan * SRP;
    ft_complex * B;
    ft_complex * P1;
    ft_complex * P2;
    ft_complex * P1inv;
    ft_complex * P2inv;
    int s;
} ft_spin_harmonic_plan;
/* replaces ft_plan_spinsph2fourier, src/drivers.c:1269-1293 */
ft_spin_harmonic_plan * ft_plan_spinsph2fourier(const int n, const int s);
/* replaces ft_destroy_spin_harmonic_plan, src/drivers.c:1259-1267 */
void ft_destroy_spin_harmonic_plan(ft_spin_harmonic_plan * P);
/* replace ft_execute_spinsph2fourier / ft_execute_fourier2spinsph, src/drivers.c:1295-1361 */
void ft_execute_spinsph2fourier(const char TRANS, const ft_spin_harmonic_plan * P, ft_complex * A, const int N, const int M);
void ft_execute_fourier2spinsph(const char TRANS, const ft_spin_harmonic_plan * P, ft_complex * A, const int N, const int M);

/* Synthesis and analysis on the spin-weighted sphere's grid (N x M complex, M odd).  Opaque
 * (the reference's struct holds FFTW plans).  TRANS 'N' or 'C'; any other character leaves X
 * untouched, as in the reference. */
typedef struct ft_spinsphere_fftw_plan_s ft_spinsphere_fftw_plan;
/* replace ft_plan_spinsph_synthesis / ft_plan_spinsph_analysis, src/fftw.c:789-799 */
ft_spinsphere_fftw_plan * ft_plan_spinsph_synthesis(const int N, const int M, const int S, const unsigned flags);
ft_spinsphere_fftw_plan * ft_plan_spinsph_analysis(const int N, const int M, const int S, const unsigned flags);
/* replaces ft_destroy_spinsphere_fftw_plan, src/fftw.c:743-751 */
void ft_destroy_spinsphere_fftw_plan(ft_spinsphere_fftw_plan * P);
/* replaces ft_get_spin_spinsphere_fftw_plan, src/fftw.c:753 */
int ft_get_spin_spinsphere_fftw_plan(const ft_spinsphere_fftw_plan * P);
/* replace ft_execute_spinsph_synthesis / ft_execute_spinsph_analysis, src/fftw.c:801-960 */
void ft_execute_spinsph_synthesis(const char TRANS, const ft_spinsphere_fftw_plan * P, ft_complex * X, const int N, const int M);
void ft_execute_spinsph_analysis(const char TRANS, const ft_spinsphere_fftw_plan * P, ft_complex * X, const int N, const int M);

/* Grid plans with caller-chosen kinds (replace ft_plan_{sph,disk,tri,annulus,rectdisk,tet,spinsph}_
 * with_kind, src/fftw.c:76-102, 414-449, 281-288, 534-571, 660-686, 340-347, 755-787).  The kinds
 * are FFTW's r2r constants (fftw3.h: R2HC 0, HC2R 1, REDFT01 4, REDFT10 5, REDFT11 6, RODFT01 8,
 * RODFT10 9), passed as int.  Accepted: cosine and sine kinds of one type per plan (II: REDFT10 /
 * RODFT10, III: REDFT01 / RODFT01), REDFT11 as the disk's second kind, a cosine kind for the
 * triangle, annulus and tetrahedron (one kind for all their dimensions), R2HC or HC2R for the sphere's,
 * disk's and annulus's phi kind, sign +1 or -1 for the spin grid's row DFT.  Other combinations
 * return NULL with FT_B200_EUNSUPPORTED. */
ft_sphere_fftw_plan * ft_plan_sph_with_kind(const int N, const int M, const int kind[3][1], const unsigned flags);
ft_disk_fftw_plan * ft_plan_disk_with_kind(const int N, const int M, const int kind[3][1], const unsigned flags);
ft_triangle_fftw_plan * ft_plan_tri_with_kind(const int N, const int M, const int kind0, const int kind1, const unsigned flags);
ft_annulus_fftw_plan * ft_plan_annulus_with_kind(const int N, const int M, const double rho, const int kind[2][1], const unsigned flags);
ft_rectdisk_fftw_plan * ft_plan_rectdisk_with_kind(const int N, const int M, const int kind[3][1], const unsigned flags);
ft_tetrahedron_fftw_plan * ft_plan_tet_with_kind(const int N, const int L, const int M, const int kind0, const int kind1, const int kind2,
                                                 const unsigned flags);
ft_spinsphere_fftw_plan * ft_plan_spinsph_with_kind(const int N, const int M, const int S, const int kind[2][1], const int sign,
                                                    const unsigned flags);

/* Rotation level. */
/* replaces ft_plan_rotsphere, src/rotations.c:116-133 */
ft_rotation_plan * ft_plan_rotsphere(const int n);
/* replaces ft_plan_rottriangle, src/rotations.c:143-160 */
ft_rotation_plan * ft_plan_rottriangle(const int n, const double alpha, const double beta, const double gamma);
/* replaces ft_plan_rotdisk, src/rotations.c:173-190 */
ft_rotation_plan * ft_plan_rotdisk(const int n, const double alpha, const double beta);
/* replaces ft_plan_rotannulus, src/rotations.c:192-268 (gamma = 0): a disk-kind plan (use it with
 * ft_execute_disk_hi2lo / lo2hi, as the reference's ann2cxf does) */
ft_rotation_plan * ft_plan_rotannulus(const int n, const double alpha, const double beta, const double gamma, const double rho);
/* replaces ft_plan_rotrectdisk, src/rotations.c:270-287 */
ft_rotation_plan * ft_plan_rotrectdisk(const int n, const double beta);
/* replaces ft_set_num_threads, src/drivers.c:56: the reference's OpenMP thread count; here the
 * host threads that build plans (n < 1: the default, the hardware threads up to 32). */
void ft_set_num_threads(const int n);
/* replace ft_fftw_init_threads / ft_fftw_plan_with_nthreads, src/fftw.c:62-64: FFTW's threading
 * set-up; the grid plans here run on cuFFT, so the first returns 1 (success) and the second does
 * nothing. */
int ft_fftw_init_threads(void);
void ft_fftw_plan_with_nthreads(const int n);
/* replaces ft_destroy_rotation_plan, src/rotations.c:6-10 */
void ft_destroy_rotation_plan(ft_rotation_plan * RP);
/* replace ft_execute_{sph,tri,disk}_{hi2lo,lo2hi}, src/drivers.c:58-92, 278-312, 378-412.
 * B is the reference's host scratch argument; it is accepted and not used. */
void ft_execute_sph_hi2lo(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_sph_lo2hi(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_tri_hi2lo(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_tri_lo2hi(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_disk_hi2lo(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_disk_lo2hi(const ft_rotation_plan * RP, double * A, double * B, const int M);
/* replace ft_execute_sphv_hi2lo / lo2hi, src/drivers.c:168-276: a sph rotation plan on the sphv
 * layout (order m on columns 2m + 1, 2m + 2, m = 2 .. M/2 - 1; M odd); B is accepted and not used. */
void ft_execute_sphv_hi2lo(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_sphv_lo2hi(const ft_rotation_plan * RP, double * A, double * B, const int M);
/* replace ft_execute_tet_hi2lo / lo2hi, src/drivers.c:510-528: RP1, RP2 triangle plans of one n
 * (ft_plan_rottriangle(n, alpha, beta, gamma + delta + 1) and (n, beta, gamma, delta) for the
 * tetrahedral transform); A is n x L x M with L <= n */
void ft_execute_tet_hi2lo(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, double * A, const int L, const int M);
void ft_execute_tet_lo2hi(const ft_rotation_plan * RP1, const ft_rotation_plan * RP2, double * A, const int L, const int M);
/* replace ft_execute_rectdisk_hi2lo / lo2hi, src/drivers.c:488-508 (order m on column m) */
void ft_execute_rectdisk_hi2lo(const ft_rotation_plan * RP, double * A, double * B, const int M);
void ft_execute_rectdisk_lo2hi(const ft_rotation_plan * RP, double * A, double * B, const int M);
/* replace ft_kernel_{sph,tri,disk,rectdisk}_{hi2lo,lo2hi}, src/rotations.c:135-141, 162-168,
 * 262-268, 289-295: one host column A with stride S >= 1 (its entries k S), the sweeps from order
 * m2 down to order m1 (hi2lo) or from m1 up to m2 (lo2hi), m1 >= 0, with the plan's table.  Only
 * the entries the sweeps touch are read and written. */
void ft_kernel_sph_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_sph_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_tri_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_tri_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_disk_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_disk_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_rectdisk_hi2lo(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
void ft_kernel_rectdisk_lo2hi(const ft_rotation_plan * RP, const int m1, const int m2, double * A, const int S);
/* replace ft_kernel_tet_hi2lo / lo2hi, src/rotations.c:297-321: the contiguous n x L slab A (n the
 * triangle plan's), sweeps j = m - 1 .. 0 of rotations of its column pairs (l, l + 1);
 * 0 <= L <= n, 0 <= m <= n. */
void ft_kernel_tet_hi2lo(const ft_rotation_plan * RP, const int L, const int m, double * A);
void ft_kernel_tet_lo2hi(const ft_rotation_plan * RP, const int L, const int m, double * A);

/* ------------------------------------------------------------------------ */
/* Device-pointer entry points (no host copies).  A is a device pointer     */
/* (N x M, leading dimension N); stream is a cudaStream_t (NULL = legacy    */
/* default stream).  Asynchronous: they return once the work is enqueued.   */
/* Return FT_B200_OK or an error code.                                      */
/* ------------------------------------------------------------------------ */
enum { FT_B200_SPH = 0, FT_B200_TRI = 1, FT_B200_DISK = 2 };

/* Full transform.  forward = 1: sph2fourier / tri2cheb / disk2cxf / rectdisk2cheb / ann2cxf;
 * forward = 0: fourier2sph / cheb2tri / cxf2disk / cheb2rectdisk / cxf2ann.  Reentrant per
 * plan for sph, tri and disk plans (per-call scratch from a stream-ordered pool: N x M doubles
 * and a few hundred KB per call while it runs); rectdisk and annulus plans are not. */
int ft_b200_execute_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M, void * stream);
/* Grid synthesis / analysis on device memory: op 0 sph synthesis, 1 sph analysis,
 * 2 sphv synthesis, 3 sphv analysis (the sequences of the ft_execute_* above, with
 * the plan's transform kinds), asynchronous on stream.  No counterpart in the
 * reference (its calls take host memory). */
int ft_b200_execute_sph_grid_dev(const ft_sphere_fftw_plan * P, int op, char TRANS, double * dX, int N, int M, void * stream);
/* Disk and triangle grids on device memory: analysis = 0 runs the plan through the synthesis
 * sequence, 1 through the analysis sequence (the plan's kinds either way, as the reference's
 * tests cross them), asynchronous on stream.  No counterpart in the reference. */
int ft_b200_execute_disk_grid_dev(const ft_disk_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream);
int ft_b200_execute_tri_grid_dev(const ft_triangle_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream);
int ft_b200_execute_annulus_grid_dev(const ft_annulus_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream);
int ft_b200_execute_rectdisk_grid_dev(const ft_rectdisk_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M, void * stream);
int ft_b200_execute_tet_grid_dev(const ft_tetrahedron_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int L, int M, void * stream);

/* The sph vector-field transforms on device memory (forward = 1: sphv2fourier). */
int ft_b200_execute_sphv_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M, void * stream);
/* Rotation stage alone (hi2lo = 1: ft_execute_*_hi2lo; 0: *_lo2hi). */
int ft_b200_rotations_dev(const ft_rotation_plan * RP, int hi2lo, double * dA, int M, void * stream);
/* Spin-weighted transforms on device memory: dA holds 2 N M doubles (interleaved
 * complex); forward = 1: spinsph2fourier, 0: fourier2spinsph. */
int ft_b200_execute_spin_dev(const ft_spin_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M, void * stream);
/* Tetrahedral transforms on device memory (forward = 1: tet2cheb, 0: cheb2tet), and the
 * plan's rotation stage alone (hi2lo = 1: ft_execute_tet_hi2lo with the plan's two tables). */
int ft_b200_execute_tet_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int L, int M, void * stream);
int ft_b200_tet_rotations_dev(const ft_harmonic_plan * P, int hi2lo, double * dA, int L, int M, void * stream);
/* The spin rotation stage alone (hi2lo = 1: ft_execute_spinsph_hi2lo; 0: _lo2hi). */
int ft_b200_spin_rotations_dev(const ft_spin_rotation_plan * SRP, int hi2lo, double * dA, int M, void * stream);
/* The spin grid's synthesis (analysis = 0) or analysis sequence with the plan's kinds on device
 * memory: dX holds 2 N M doubles (interleaved complex, 16-byte aligned), asynchronous on stream.
 * No counterpart in the reference. */
int ft_b200_execute_spinsph_grid_dev(const ft_spinsphere_fftw_plan * P, int analysis, char TRANS, double * dX, int N, int M,
                                     void * stream);

/* Batched drop-in: nfields fields, each with its own plan (plans may repeat,
 * degrees may differ), all in one persistent launch per stage.  dA[f] is the
 * device pointer of field f, N[f] x M[f].  Same transform and TRANS for all. */
int ft_b200_execute_batched_dev(const ft_harmonic_plan * const * plans, int forward, char TRANS,
                                double * const * dA, const int * N, const int * M, int nfields, void * stream);

/* Allocation-free variant of ft_b200_execute_dev.  No counterpart in the
 * reference (whose plans own host scratch).
 *
 * For callers that cannot let a library allocate device memory: frameworks
 * that own all device memory through their own pool and hand a library only
 * the arrays it works on, and long-running services that reserve memory at
 * start-up and must not allocate afterwards, because cudaMalloc / cudaFree can
 * block or synchronise the device and can fail under memory pressure.
 *
 * Same transform and arguments as ft_b200_execute_dev; A is the caller's
 * device matrix (input and output).  The intermediate matrix and the rotation
 * kernel's work counter live in a fixed device array compiled into the library
 * (FT_B200_NOALLOC_MAX_ELEMS doubles, 8 MiB, plus 256 bytes), which every GPU
 * that loads the library holds until the process exits.  The call makes no
 * cudaMalloc / cudaFree and no allocating library call.
 *   - N*M above FT_B200_NOALLOC_MAX_ELEMS is rejected with FT_B200_EINVAL.
 *   - M must be the plan's default (2N-1, N, 4N-3); other M return
 *     FT_B200_EUNSUPPORTED, since their task list would have to be allocated.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call
 *     before any stream capture.  The address is kept for the life of the
 *     process, so do not use this entry point across a cudaDeviceReset (which
 *     also invalidates every plan made before it).
 *   - All calls share the one array, which keeps the last call's contents; the
 *     work counter is cleared by every call.  Calls that overlap on the GPU
 *     (concurrent streams, or several host threads) race on the array and must
 *     be serialised by the caller. */
#define FT_B200_NOALLOC_MAX_ELEMS (1 << 20)
int ft_b200_execute_noalloc_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * dA, int N, int M, void * stream);

/* Fields sharing one plan (same n, same M, same family), in one call.
 * precision FT_B200_FP64: the direct sweeps, as ft_b200_execute_batched_dev.
 * precision FT_B200_FP64_BLOCKED: blocks of 32 consecutive sweeps
 * are cut into tiles whose rotations are pre-multiplied (in FP64, once per
 * plan) into dense orthogonal 64 x 64 matrices, applied to every field's
 * columns as FP64 tensor-core (DMMA) products; a column's sweeps above its
 * last whole block stay direct.  Not bit-identical to the direct sweeps (the
 * products round differently); the relative 2-norm difference is of the order
 * of 1e-14.  The first call on a plan builds its tile matrices (device memory,
 * about 550 MB for sph at n = 4096; disk and tri keep one chain of tiles per
 * block, twice as long); make it before any stream capture.
 * precision FT_B200_MIXED_BF16: the same blocks, each tile product
 * computed on the tcgen05 tensor cores from three 9-bit fixed-point BF16
 * slices per operand (eight slice products, exact FP32 accumulation per order
 * level); a value is carried between tiles at FP32 accuracy, in global memory
 * the matrices stay FP64.  The connection multiply runs on the tensor cores
 * too, from 8-bit integer digits (five of each row of the matrix, four of
 * each input column, five for tri; exact 32-bit integer accumulation over the
 * whole column, recombined in FP64; tri's right multiply through two
 * transposes, its normalisation in FP64).  Relative 2-norm error against the
 * FP64 transform about 3.5e-7 for sph at n = 4096; the connection multiplies
 * amplify the sweeps' error by a factor that depends on the family and its
 * parameters (disk with generic parameters about 3e-6 at n = 2048).  tri
 * keeps its sweeps in FP64 (direct) in both mixed forms and runs only its two
 * connection multiplies on the tensor cores: its multiplies amplify errors
 * strongly (a sliced sweep's to 3e-6 .. 3e-5 at n = 2048).
 * precision FT_B200_MIXED_BF16X4: four slices in the blocks (ten products)
 * and five digits of the input in the connection multiply: about 1.5e-7 for
 * sph at n = 4096.  The first call of either builds its slice images of the
 * tiles and of the connection matrices (about 1 GB at n = 4096).
 * FT_B200_MULTIPLY=bf16 in the environment selects the earlier connection
 * multiply from BF16 slices (exact FP32 sums of 256-row chunks). */
#define FT_B200_FP64 0
#define FT_B200_FP64_BLOCKED 1
#define FT_B200_MIXED_BF16 2
#define FT_B200_MIXED_BF16X4 3
int ft_b200_execute_shared_dev(const ft_harmonic_plan * P, int forward, char TRANS, double * const * dA, int nfields,
                               int precision, void * stream);

/* Host-pointer form of ft_b200_execute_shared_dev for a sequence of transforms:
 * every field A[f] (a host N x M column-major matrix, the plan's N and default
 * M) goes through transforms o = 0 .. nops-1 (forward[o] nonzero: the
 * forward transform, else the backward one; TRANS[o] 'N' or 'T'), in place,
 * at the given precision.  The reference's counterpart is one
 * ft_execute_sph2fourier / ft_execute_fourier2sph call per field and
 * transform (src/drivers.c:833-865, host pointers, in place).
 * The fields move in groups through three device buffers owned by the plan:
 * the copy of group g + 1 to the device and the copy of group g - 1 back to
 * the host overlap the transforms of group g (streams of the plan's own,
 * events between them); the first and the last group hold half as many
 * fields as the others (FT_B200_HOST_GROUP, default 4), so that the copies
 * that cannot overlap are short.  Returns when every result is back in host
 * memory.  The copies overlap only from page-locked host memory
 * (cudaHostAlloc / cudaHostRegister); pageable memory gives the same results
 * with serial copies.  The first call allocates the buffers (3 groups of the
 * largest group size, about 1 GB per field slot at n = 4096); they are freed
 * with the plan.  Calls on one plan are serialised. */
int ft_b200_execute_shared_host(const ft_harmonic_plan * P, int nops, const int * forward, const char * TRANS,
                                double * const * A, int nfields, int precision);

/* Reads and clears the plan's device status word: 0 normally; nonzero when a
 * wait inside one of its tensor-core kernels gave up (the kernel then stops
 * early and its output is not valid).  Synchronises with the device.  No
 * counterpart in the reference, whose kernels have no device waits. */
int ft_b200_device_status(const ft_harmonic_plan * P);

/* Kind of a plan (FT_B200_SPH / TRI / DISK), or -1. */
int ft_b200_plan_kind(const ft_harmonic_plan * P);
/* Device id the plan lives on. */
int ft_b200_plan_device(const ft_harmonic_plan * P);

/* Number of kernels this library launched since load (all entry points). */
unsigned long long ft_b200_kernel_launches(void);

/* Measurement hook.  While enabled, every kernel launch is bracketed by a pair
 * of CUDA events recorded on its launch stream.  ft_b200_profile(1) resets the
 * record; ft_b200_profile_read waits for the recorded events and returns, for
 * one kernel family (0 = rotation sweeps, 1 = triangular multiplies, 2 = other),
 * the summed device time in ms and the launch count.  Off by default. */
int ft_b200_profile(int enable);
int ft_b200_profile_read(int family, double * ms, int * launches);

/* Launch configuration of the rotation kernel (no counterpart in the reference,
 * whose kernels have no launch shape).  cfg = s + 8 p forces shape s = 0 .. 5
 * (warps x sweeps per warp x chunk: 8 x 8 x 16, 16 x 4 x 8, 8 x 4 x 8, 8 x 4 x 16,
 * 4 x 4 x 16 and 4 x 8 x 16, the last two with as many CTAs per SM as fit; tri has
 * no 16 x 4 x 8 and runs 8 x 8 x 16 for it) and pass-pipeline mode p = 0 .. 2.
 * p = 1: each pass of 16 .. 64 sweeps of a task is its own work unit, queued
 * pass-major, and streams down the columns on another SM right behind the previous
 * pass (for inputs with fewer tasks than SMs; it loses where the columns would
 * leave L2 between passes); p = 2: the same for the longest tasks whose columns
 * fit in half the L2, every other task as one unit, after them.
 * cfg = -1 (the default, or FT_B200_ROT_CFG unset) lets the autotuner choose:
 * the first out-of-place launch of each shape (family, direction, all sweeps or
 * heads only, fields, tasks, N, M) times every configuration once on its
 * destination, whose contents are not needed yet, and keeps the fastest for that
 * shape.  That first launch synchronises with the stream, so make it before any
 * stream capture; a capturing stream or an in-place launch uses the untimed
 * default (8 x 8 x 16, 8 x 4 x 16 for heads, no pipeline).  FT_B200_AUTOTUNE=0
 * turns the timing off.  Results are bit-identical for every configuration.
 * Process-wide. */
void ft_b200_set_rotation_config(int cfg);

#ifdef __cplusplus
}
#endif

#endif
