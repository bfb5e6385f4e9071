/*
 * momwire_b200 — C ABI of the B200 (sm_100a) dense-solve path for momwire's
 * B-spline Galerkin thin-wire solver.
 *
 * Every entry point takes plain pointers and sizes.  Pointers marked
 * "device" must be device memory of the current CUDA device; the caller
 * owns every buffer.  `stream` is a cudaStream_t passed as void* (NULL =
 * the legacy default stream).  All calls are asynchronous on `stream`
 * unless stated otherwise and return an mw_status (0 = success).
 *
 * The reference (momwire 0.37.0) reaches the same work through its
 * pybind11 module `momwire._accelerators` and scipy's LAPACK; each
 * declaration cites the reference interface it replaces
 * (paths relative to the momwire source tree, src/momwire/).
 *
 * Matrix layout: complex values are interleaved (re, im) pairs of the
 * element type.  Dense matrices are column-major with a leading dimension
 * (the layout scipy.linalg.solve factors in place, bspline.py:2432).
 */
#ifndef MOMWIRE_B200_H
#define MOMWIRE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t mw_status;

#define MW_OK             0
#define MW_ERR_INVALID   -1  /* bad argument (size, pointer, degree)        */
#define MW_ERR_CUDA      -2  /* a CUDA runtime call failed                  */
#define MW_ERR_CANCELLED -3  /* the host cancel flag was raised             */
#define MW_ERR_TIMEOUT   -4  /* a bounded device wait gave up               */
#define MW_ERR_SINGULAR  -5  /* exact zero pivot (LAPACK info > 0)          */
#define MW_ERR_WORKSPACE -6  /* workspace smaller than the size query asked */

/* Library version (major*10000 + minor*100 + patch). */
int32_t mw_version(void);

/* Human-readable text for the last error raised on this host thread. */
const char* mw_last_error(void);

/* Number of kernels this library has launched in this process (a running
 * host-side count; the difference across a region counts its launches). */
int64_t mw_launch_count(void);

/* Optional per-kernel-class timing with CUDA events recorded around each
 * launch on its own stream (for roofline figures).  Classes: 0 same-edge
 * table, 1 fill, 2 image fill, 3 LU panel, 4 row swaps, 5 triangular solve
 * block, 6 complex128 GEMM, 7 tensor-core complex GEMM, 8 refinement,
 * 9 other, 10 Sommerfeld grid, 11 Sommerfeld remainder, 14 the rows
 * below a static-pivot panel's diagonal block; 12 and 13 enclose
 * whole factorisations and whole many-right-hand-side triangular solves
 * (their wall time on the calling stream, overlapping classes 3-9).
 * mw_profile_enable(1) clears the counters and starts recording;
 * mw_profile_read synchronises the recorded events and returns the launch
 * count, summed device time and the algorithmic flops / bytes of a class. */
void mw_profile_enable(int32_t on);
int32_t mw_profile_read(int32_t cls, int64_t* launches, double* total_ms,
                        double* flops, double* bytes);

/* Failure-handling self-test (no counterpart in the reference, whose
 * kernels have no device waits): runs one of this library's bounded device
 * waits with a short limit and an event that never comes -- which = 0 the
 * complex128 panel's grid barrier, 1 the tensor-core kernels' mbarrier
 * wait -- and returns the status the wait recorded: MW_ERR_TIMEOUT when it
 * gave up as designed (the context stays usable).  spin_limit in
 * [256, 2^24]; workspace: 16 bytes of device memory; synchronises stream. */
mw_status mw_selftest_wait_timeout(int32_t which, int64_t spin_limit, void* workspace, void* stream);

/* Ground models served by the fill (bspline.py:182-287 ground kwargs). */
#define MW_GROUND_NONE        0  /* free space                              */
#define MW_GROUND_PEC         1  /* perfect image, ground_eps=None          */
#define MW_GROUND_REFL        2  /* ground_model="refl-coef" (Fresnel)      */
#define MW_GROUND_SOMM_IMAGE  3  /* ground_model="sommerfeld": C2 image     */

/* Phi-term image-charge weighting for MW_GROUND_REFL
 * (_ground_refl.py:243-269, ground_phi_mode). */
#define MW_PHI_RHO_V   0
#define MW_PHI_IMAGE   1
#define MW_PHI_NORMAL  2
#define MW_PHI_BLEND   3

/*
 * Segment geometry of one structure, all device pointers.
 * Segments are numbered wire by wire, edge by edge (bspline.py:988-1093).
 */
typedef struct mw_segments {
    int32_t        n_seg;
    const double*  seg_l;        /* (n_seg, 3) segment start points          */
    const double*  seg_r;        /* (n_seg, 3) segment end points            */
    const double*  tangent;      /* (n_seg, 3) unit tangents                 */
    const double*  radius;       /* (n_seg)    wire radius of each segment   */
    const int32_t* edge;         /* (n_seg)    straight edge of each segment */
    const int32_t* pos_in_edge;  /* (n_seg)    index along that edge         */
    const int32_t* ek_group;     /* (n_seg) coaxial labels, or NULL (EK off) */
    const int32_t* ek_group_img; /* (n_seg) labels of the mirrored sources
                                    from the joint real+image scan, or NULL  */
} mw_segments;

/*
 * Uniform straight edges: the unit of the same-edge analytic split.
 * Table entry (edge e, delta = j - i) lives at row table_off[e] + delta +
 * n_in_edge[e] - 1 of a (rows, d+1, d+1) complex128 table.
 */
typedef struct mw_edges {
    int32_t        n_edge;
    const int32_t* n_in_edge;   /* (n_edge) segments per edge (device)      */
    const int64_t* table_off;   /* (n_edge) first table row (device)        */
    const double*  h;           /* (n_edge) segment length (device)         */
    const double*  radius;      /* (n_edge) radius (device)                 */
    int64_t        table_rows;  /* sum over edges of 2*n_in_edge - 1        */
    int32_t        max_n;       /* max n_in_edge                            */
} mw_edges;

/*
 * Basis tables (bspline.py:1216-1414): basis m has d+1 wings; wing a lies
 * on segment supp[m*(d+1)+a] (-1 = padded wing) with monomial coefficients
 * polys[(m*(d+1)+a)*(d+1)+p] of u^p, u the local arc length.
 *
 * Tiles: the fill works on tiles of consecutive bases.  Tile t covers
 * bases [tile_first[t], tile_first[t]+tile_nb[t]) whose wings touch the
 * tile_ns[t] segments listed at tile_seg[t*max_tile_seg ...]; loc[m*(d+1)+a]
 * is the position of wing (m,a)'s segment in its own tile's list (-1 for a
 * padded wing).  Built on the host by momwire_b200._tables.
 */
typedef struct mw_basis {
    int32_t        degree;       /* 1 or 2                                  */
    int32_t        n_basis;
    const int32_t* supp;         /* (n_basis, d+1) device                   */
    const double*  polys;        /* (n_basis, d+1, d+1) device              */
    int32_t        n_tile;
    int32_t        max_tile_basis;  /* <= 16                                */
    int32_t        max_tile_seg;    /* <= MW_MAX_TILE_SEG                   */
    const int32_t* tile_first;   /* (n_tile) device                         */
    const int32_t* tile_nb;      /* (n_tile) device                         */
    const int32_t* tile_ns;      /* (n_tile) device                         */
    const int32_t* tile_seg;     /* (n_tile, max_tile_seg) device           */
    const int32_t* loc;          /* (n_basis, d+1) device                   */
} mw_basis;

#define MW_MAX_TILE_BASIS 16
#define MW_MAX_TILE_SEG   24

/* Physical parameters of one frequency (bspline.py:343-346, 151-152). */
typedef struct mw_freq {
    double k;        /* wavenumber  = omega / c                             */
    double omega;    /* angular frequency                                   */
    double eps0;     /* 8.8541878188e-12 (the solver's own constants)       */
    double mu0;      /* 1.25663706127e-6                                    */
} mw_freq;

/* Ground description for the image fill (_ground_spec.py:90-126). */
typedef struct mw_ground {
    int32_t model;        /* MW_GROUND_*                                    */
    int32_t phi_mode;     /* MW_PHI_* (MW_GROUND_REFL only)                 */
    double  ground_z;
    double  eps_re, eps_im;  /* complex relative permittivity eps~(omega)    */
} mw_ground;

/*
 * Same-edge Toeplitz table: static (closed-kernel 1/R, + EK correction)
 * plus smooth (exp(-jkR)-1)/R moments for every uniform edge and every
 * offset delta.  Replaces seg_seg_static_moments_bspline_uniform[_ek]
 * (_accelerators.cpp:2954/2959, called from _bspline_kernels.py:333) and
 * seg_seg_reg_moments_bspline_swept[_ek] (_accelerators.cpp:330/339,
 * called from _bspline_kernels.py:480).
 * out: (edges->table_rows, d+1, d+1) complex128, device.
 */
mw_status mw_same_edge_table(const mw_edges* edges, int32_t degree,
                             int32_t n_qp, int32_t extended_kernel,
                             double k, double* out, void* stream);

/*
 * Off-edge moment tensor J[p][P][i][j] over two segment sets (real
 * sources, or sources mirrored through z = ground_z when mirror != 0).
 * Replaces seg_seg_full_moments_bspline[_ek] (_accelerators.cpp:2683/2740,
 * called from _bspline_kernels.py:599).  Used by the parity tests; the
 * product fill never materialises J.
 * seg_i / seg_j: segment sets (device); groups_i/groups_j may be NULL.
 * out: (d+1, d+1, n_i, n_j) complex128, device.
 */
mw_status mw_offedge_moments(const mw_segments* seg_i, const mw_segments* seg_j,
                             int32_t degree, int32_t n_qp, double k,
                             int32_t mirror, double ground_z,
                             const int32_t* groups_i, const int32_t* groups_j,
                             double* out, void* stream);

/*
 * Fused Galerkin fill: Z = j w mu sum (t.t) C J C + (1/(j w eps)) sum C' J C'
 * over every basis pair, with same-edge pairs taken from `table` (from
 * mw_same_edge_table at the same k) and every other pair by n_qp x n_qp
 * Gauss-Legendre quadrature of exp(-jkR)/(4 pi R).  Writes all of Z.
 * Replaces _compute_Z_operator's free-space part: _build_J_blocks +
 * assemble_Z_bspline (bspline.py:2222-2348, _accelerators.cpp:1767) and
 * the chunked route _compute_Z_dense_chunked + assemble_Z_bspline_windowed
 * (bspline.py:2386-2550, _accelerators.cpp:1447).
 * Z: complex128 column-major (n_basis x n_basis, leading dim ldz), device.
 * Z32 (optional, may be NULL): complex64 copy written in the same pass
 * (leading dim ldz32), for the mixed-precision factorisation.
 */
mw_status mw_fill_z(const mw_segments* seg, const mw_basis* basis,
                    const double* table, const mw_edges* edges,
                    const mw_freq* freq, int32_t n_qp,
                    double* Z, int64_t ldz, float* Z32, int64_t ldz32,
                    void* stream);

/*
 * Ground image: Z -= weighted Galerkin assembly over mirrored sources
 * (PEC mirror tangent dot; Fresnel w_A/w_Phi per segment pair; or the
 * Sommerfeld C2-scaled exact image).  Replaces _accumulate_Z_image_chunked
 * (bspline.py:2552-2661) with assemble_Z_bspline_weighted_windowed
 * (_accelerators.cpp:1612) and the weight producers of
 * _potential_ground.py:711-810.  Z32 as for mw_fill_z (may be NULL; when
 * given it is overwritten with the updated Z).
 */
mw_status mw_fill_z_image(const mw_segments* seg, const mw_basis* basis,
                          const mw_ground* ground, const mw_freq* freq,
                          int32_t n_qp, double* Z, int64_t ldz,
                          float* Z32, int64_t ldz32, void* stream);

/*
 * One side of an off-edge block: n_basis bases whose d+1 wings index this
 * side's own segment arrays (supp (n_basis, d+1), -1 = no wing; polys
 * (n_basis, d+1, d+1) monomial coefficients in local arc length), the
 * segments' end points and unit tangents (n_seg, 3), and for the extended
 * kernel their coaxial group labels (n_seg; -1 = none) or NULL.  All device
 * pointers.
 */
typedef struct mw_block_side {
    int32_t        n_basis;
    const int32_t* supp;
    const double*  polys;
    int32_t        n_seg;
    const double*  seg_l;
    const double*  seg_r;
    const double*  tangent;
    const int32_t* ek_group;
} mw_block_side;

/* Reflection-coefficient image weights of the block sampler: eps~ and the
 * charge weight w_Phi = c0 + c1 rho_v (_ground_refl.py phi_mode_coeffs). */
typedef struct mw_block_refl {
    double eps_re, eps_im;
    double phi_c0_re, phi_c0_im;
    double phi_c1_re, phi_c1_im;
} mw_block_refl;

/*
 * The off-edge Galerkin block Z[I, J] (row-major, Z[m * ldz + n],
 * complex128) between two basis sets by plain n_qp x n_qp Gauss quadrature
 * of every wing pair, fused with the EFIE combine: the H-matrix / array-
 * block ACA row, column and block sampler.  refl == NULL: free space (or a
 * PEC image with the J side passed mirrored); refl != NULL: the Fresnel
 * image, J side mirrored.  a_ek > 0 applies the extended kernel's coaxial
 * factor (radius a_ek) on pairs with equal non-negative group labels.
 * gl_t / gl_w: n_qp <= 8 host-side nodes and weights on [0, 1].  Replaces
 * bspline_assemble_offedge_block, _refl, _ek and _refl_ek
 * (_accelerators.cpp:1977-2680, bound at :6440-6500) as called by
 * hmatrix.py _offedge_block_evaluators_uniform (hmatrix.py:1157-1290).
 */
mw_status mw_offedge_block(int32_t degree, const mw_block_side* I, const mw_block_side* J, double a_squared,
                           const mw_freq* freq, int32_t n_qp, const double* gl_t, const double* gl_w,
                           const mw_block_refl* refl, double a_ek, double* Z, int64_t ldz, void* stream);

/*
 * Singular basis enrichment (bspline.py:3048-3076 specs): one basis per
 * wire end at a junction of at least enrichment_min_k ends, on the segment
 * beside the junction, shaped u log u - P(u) with u the normalised distance
 * from the junction and P the polynomial proj[0..d] (zeros: the "raw"
 * shape; the "stable" shape subtracts its bubble projection).
 */
typedef struct mw_enrich {
    int32_t        n_enrich;
    const int32_t* seg;      /* (n_enrich) segment of each basis (device)      */
    const int32_t* origin;   /* (n_enrich) 0: junction at the segment's start,
                                1: at its end (device)                         */
    int32_t        n_qp;     /* Gauss nodes per axis (n_qp_sing)               */
    const double*  t01;      /* (n_qp) nodes on [0, 1] (device)                */
    const double*  w01;      /* (n_qp) weights on [0, 1] (device)              */
    double         proj[4];  /* P's monomial coefficients, degree <= 3         */
    double         radius;   /* the structure's (uniform) wire radius          */
} mw_enrich;

/*
 * The enrichment blocks of the augmented system [[Z, Z_pe], [Z_ep, Z_ee]]:
 * Z_pe into rows 0..n_basis-1 / columns n_basis.., Z_ep and Z_ee into rows
 * n_basis.. of the column-major Z (ldz >= n_basis + n_enrich; the
 * polynomial block is mw_fill_z's, written separately), and their complex64
 * copy into Z32 when it is not NULL.  ground (NULL = free space): PEC,
 * reflection-coefficient and Sommerfeld C2 image reactions are subtracted;
 * the Sommerfeld remainder is the caller's (mw_somm_field_proj).  Replaces
 * assemble_Z_enrich (_accelerators.cpp:2997) and
 * _assemble_Z_enrich_image_numpy (bspline.py:3308-3521) as called by
 * _enrichment_Z_assemble (bspline.py:3523-3693).
 */
mw_status mw_enrich_blocks(const mw_segments* seg, const mw_basis* basis, const mw_enrich* en,
                           const mw_freq* freq, const mw_ground* ground, double* Z, int64_t ldz,
                           float* Z32, int64_t ldz32, void* stream);

/*
 * mw_fill_z for callers that cannot allocate device memory -- no
 * counterpart in the reference (its fills run on the host).  Some hosts
 * own every device allocation (a plugin given only its input and output
 * buffers by a process with its own memory pool, or a binding with no
 * route to cudaMalloc); for them the same-edge scratch table that
 * mw_fill_z takes from the caller lives here in a fixed device array that
 * the library holds from load until exit.  This call allocates nothing.
 * Writes the same Z as mw_same_edge_table + mw_fill_z (Z32 not written).
 * Limits: at most mw_fill_z_noalloc_capacity(degree) table rows (32768 at
 * degree 2, 73728 at degree 1; a structure needs the sum over its straight
 * edges of 2*n_segments - 1), otherwise MW_ERR_WORKSPACE.  All calls share
 * the array, so calls that overlap on the GPU race: serialise them.  Each
 * call outside stream capture looks up the array's device address on the
 * current device (so a device reset or a non-primary context is picked
 * up); a call during capture reuses the last address seen on that device,
 * so make one call on each device before any stream capture.
 */
mw_status mw_fill_z_noalloc(const mw_segments* seg, const mw_basis* basis,
                            const mw_edges* edges, const mw_freq* freq,
                            int32_t n_qp, int32_t extended_kernel,
                            double* Z, int64_t ldz, void* stream);

/* Table rows mw_fill_z_noalloc can hold at this degree (0 unless the
 * degree is 1 or 2). */
size_t mw_fill_z_noalloc_capacity(int32_t degree);

/*
 * Tensor-core complex update C -= A B for complex64 column-major matrices
 * (A m x k, B k x n, C m x n), on tcgen05 (kind::tf32) with the 3xTF32
 * split (hi*hi + hi*lo + lo*hi) and fp32 accumulation in TMEM: the
 * trailing update of the mixed-precision factorisation.  The fp64 path of
 * the reference has no counterpart (its LAPACK zgetrf runs in complex128,
 * bspline.py:2979).  `workspace` (device) holds the packed operand planes:
 * mw_cgemm_tc_workspace_size(m, n, k) bytes.  `status` (device int32) is
 * set to MW_ERR_TIMEOUT if a bounded device wait gave up (left untouched
 * otherwise; the caller zeroes it).
 */
size_t mw_cgemm_tc_workspace_size(int64_t m, int64_t n, int64_t k);
mw_status mw_cgemm_tc_sub(int64_t m, int64_t n, int64_t k,
                          const float* A, int64_t lda, const float* B, int64_t ldb,
                          float* C, int64_t ldc, void* workspace,
                          size_t workspace_bytes, int32_t* status, void* stream);

/*
 * Workspace (bytes, device) needed by mw_zgetrf / mw_cgetrf for order n.
 */
size_t mw_getrf_workspace_size(int64_t n);

/*
 * In-place LU with partial pivoting of a complex128 column-major matrix,
 * P A = L U, pivots 1-based as LAPACK zgetrf (ipiv device, length n).
 * Replaces LAPACK zgetrf inside scipy.linalg.solve (bspline.py:2979).
 * `info` (device, 1 int32) receives LAPACK's info (0, or j+1 for an exact
 * zero pivot U(j,j)).  `cancel` (host-mapped or device int32, may be NULL)
 * is polled between panels; a raised flag returns MW_ERR_CANCELLED.
 */
mw_status mw_zgetrf(int64_t n, double* A, int64_t lda, int32_t* ipiv,
                    int32_t* info, void* workspace, size_t workspace_bytes,
                    const volatile int32_t* cancel, void* stream);

/*
 * Solve A X = B with the factors of mw_zgetrf (LAPACK zgetrs, 'N'), B
 * overwritten by X: (n x nrhs, leading dim ldb), complex128, device.
 * Replaces the zgetrs half of scipy.linalg.solve (bspline.py:2979).
 */
mw_status mw_zgetrs(int64_t n, int64_t nrhs, const double* LU, int64_t lda,
                    const int32_t* ipiv, double* B, int64_t ldb, void* stream);

/*
 * complex64 LU with partial pivoting (same conventions as mw_zgetrf),
 * trailing updates on the tensor cores (mw_cgemm_tc_sub), and the matching
 * triangular solve.  The factorisation of the mixed-precision path; its
 * fp64 counterpart in the reference is LAPACK zgetrf/zgetrs
 * (bspline.py:2979).  Workspace: mw_cgetrf_workspace_size(n, nrhs_max)
 * bytes, nrhs_max the widest right-hand side later passed to mw_cgetrs.
 * info[1] receives MW_ERR_TIMEOUT if a bounded device wait gave up.
 */
size_t mw_cgetrf_workspace_size(int64_t n, int64_t nrhs_max);
mw_status mw_cgetrf(int64_t n, float* A, int64_t lda, int32_t* ipiv,
                    int32_t* info, void* workspace, size_t workspace_bytes,
                    int64_t nrhs_max, const volatile int32_t* cancel, void* stream);
mw_status mw_cgetrs(int64_t n, int64_t nrhs, const float* LU, int64_t lda,
                    const int32_t* ipiv, float* B, int64_t ldb, void* workspace,
                    size_t workspace_bytes, void* stream);

/*
 * Mixed-precision drop-in for the complex128 solve of
 * _solve_with_kcl_ports (bspline.py:2971-2989): factor Z32 (a complex64
 * copy of Z, overwritten by its LU) with mw_cgetrf, then refine
 * X <- X + LU32 \ (B - Z X) with the residual in FP64 against Z until, in
 * every column, the correction r = ||dX||_inf / ||X||_inf -- or, once
 * successive corrections contract by q = r / r_prev <= 1/2 (the initial
 * solve from X = 0 counting as a correction of 1), the error
 * estimated to remain after it, r q -- is <= tol, or max_iter corrections.
 * X (n x nrhs, complex128) receives the solution.  *iterations /
 * *last_correction (host pointers, may be NULL) report the refinement
 * (last_correction: the largest controlling value above).  Synchronises `stream` once per refinement step.  Returns
 * MW_ERR_SINGULAR if tol was not reached.  The workspace holds, beside the
 * factorisation's, the solves' block operators and every block column of
 * the factors packed as a tensor-core operand (about 32 n^2 bytes: 3.5 GB
 * at n = 10,496).
 */
size_t mw_zgesv_mixed_workspace_size(int64_t n, int64_t nrhs);
mw_status mw_zgesv_mixed(int64_t n, int64_t nrhs, const double* Z, int64_t ldz,
                         float* Z32, int64_t ldz32, int32_t* ipiv,
                         const double* B, int64_t ldb, double* X, int64_t ldx,
                         double tol, int32_t max_iter, void* workspace,
                         size_t workspace_bytes, int32_t* info,
                         int32_t* iterations, double* last_correction,
                         const volatile int32_t* cancel, void* stream);

/* Pivoting of mw_zgesv_mixed's complex64 factorisation (no counterpart in
 * the reference, whose LAPACK zgesv always pivots over whole columns).
 * mode 0 (default): pivots are chosen within each 128-row diagonal block
 * (static pivoting -- no column-wide search, so no grid-wide exchange per
 * column); the factorisation is rejected when any |L21| (|re| + |im|)
 * exceeds 64 or a block is singular, and when the FP64 refinement does not
 * reach its tolerance, and the solve is then repeated with partial
 * pivoting.  mode 1: partial pivoting over whole columns (LAPACK's rows).
 * Process-wide; returns the previous mode (MW_ERR_INVALID for another
 * value). */
int32_t mw_set_mixed_pivoting(int32_t mode);

/* Pivoting the last mw_zgesv_mixed on this host thread used: 0 static,
 * 1 partial, 2 static rejected then partial; -1 before the first call. */
int32_t mw_last_mixed_pivoting(void);

/* Largest |L21| (|re| + |im|) of the last static-pivot factorisation made
 * by mw_zgesv_mixed on this host thread (partial pivoting keeps it <= 1). */
double mw_last_mixed_growth(void);

/* The controlling relative correction of each refinement step of the last
 * mw_zgesv_mixed on this host thread (the initial solve first): writes at
 * most max_n values to out and returns how many steps there were. */
int32_t mw_last_mixed_history(double* out, int32_t max_n);

/*
 * Frequency-batched fill: Z_b (and Z32_b when Z32 != NULL) for n_k
 * wavenumbers k_dev[b] / omega_dev[b] (device arrays), free space or a PEC
 * ground (pec_ground != 0), in two launches.  `table` (device) holds
 * n_k same-edge tables: n_k * edges->table_rows * (d+1)^2 complex128.
 * Matrices are z_stride (z32_stride) complex elements apart.  Replaces the
 * k-batched reference fill seg_seg_full_moments_bspline_swept +
 * assemble_Z_bspline_swept (_accelerators.cpp:2711, :1922; driven by
 * bspline.py:4283-4439).
 */
mw_status mw_fill_z_batch(const mw_segments* seg, const mw_basis* basis,
                          const mw_edges* edges, int32_t n_k, const double* k_dev,
                          const double* omega_dev, double eps0, double mu0,
                          int32_t n_qp, int32_t extended_kernel, double ground_z,
                          int32_t pec_ground, double* table, double* Z, int64_t ldz,
                          int64_t z_stride, float* Z32, int64_t ldz32,
                          int64_t z32_stride, void* stream);

/*
 * Batched mixed-precision solve of `batch` same-order systems Z_b X_b = B_b
 * (complex128, n x nrhs; B shared when b_stride == 0): complex64 LU of Z32_b
 * (overwritten) with one CTA per matrix panel and the batched tensor-core
 * update, then FP64 refinement of every X_b against Z_b with the stopping
 * rule of mw_zgesv_mixed applied to every matrix of the batch.  X is batch x n x nrhs,
 * contiguous.  The reference's counterpart is the stacked complex128
 * numpy.linalg.solve of _solve_with_kcl_swept_ports (bspline.py:3017).
 * Strides count complex elements.  panel_width: columns per batched panel
 * (8, 16 or 32; 0 = 16) -- the n x panel_width complex64 panel must fit in
 * 200 KB of shared memory (n <= 1600 at 16 columns).
 */
size_t mw_zgesv_mixed_batched_workspace_size(int32_t n, int32_t nrhs, int32_t batch);
mw_status mw_zgesv_mixed_batched(int32_t n, int32_t nrhs, int32_t batch, int32_t panel_width,
                                 const double* Z, int64_t ldz, int64_t z_stride,
                                 float* Z32, int64_t ldz32, int64_t z32_stride,
                                 int32_t* ipiv, int32_t* info, const double* B,
                                 int64_t ldb, int64_t b_stride, double* X, double tol,
                                 int32_t max_iter, void* workspace,
                                 size_t workspace_bytes, int32_t* iterations,
                                 double* last_correction, void* stream);

/*
 * out (ld x ncols complex128, column-major) = 0, then out[rows[q], cols[q]]
 * += vals[q] for the nnz entries (device arrays; vals interleaved re/im).
 * Builds the sparse port right-hand sides [B | kcl_con^T] and the KCL rows
 * on the device (the dense host matrices of bspline.py:3841-3867 are mostly
 * zeros: a few basis functions per feed, a few +-1 per junction).
 */
mw_status mw_scatter_c128(int64_t ld, int64_t ncols, int64_t nnz, const int64_t* rows,
                          const int64_t* cols, const double* vals, double* out, void* stream);

/*
 * Distributed series wire loading (bspline.py:2732-2760, _apply_loading;
 * _wire_loading.py series_impedance_per_wire): for every matrix b of a
 * batch, Z_b[rows[q], cols[q]] += zw[b * n_wires + wire[q]] * vals[q].
 * The nnz entries are the coalesced same-wire basis-overlap Gram (unique
 * (row, col) pairs, vals real, wire the wire both bases lie on); zw holds
 * each matrix's per-wire series impedance Z'_w(omega) (complex128, Ohm/m).
 * Z is column-major complex128 with leading dimension ldz and z_stride
 * complex elements between matrices; Z32 (optional, complex64, ld32,
 * z32_stride) receives the rounded updated values, so a mixed-precision
 * copy written by the fill stays the rounded Z.  All arrays are device
 * memory.  Entries out of range are skipped and counted into *bad
 * (optional device int32).
 */
mw_status mw_add_loading(int64_t n, int32_t batch, int64_t nnz, const int64_t* rows, const int64_t* cols,
                         const double* vals, const int32_t* wire, const double* zw, int32_t n_wires, double* Z,
                         int64_t ldz, int64_t z_stride, float* Z32, int64_t ld32, int64_t z32_stride, int32_t* bad,
                         void* stream);

/*
 * Pad `count` column-major matrices of order nb whose leading n x n block is
 * filled to [[Z, 0], [0, I]] (complex128 Z with leading dimension ldz and
 * z_stride complex elements between matrices; the complex64 mirror Z32 the
 * same when given).  Structures of different orders then share one batched
 * factorisation: partial pivoting never selects a padding row for a column
 * < n, and the padding block of the solution is exactly zero.
 */
mw_status mw_pad_identity(int64_t n, int64_t nb, int32_t count, double* Z, int64_t ldz, int64_t z_stride,
                          float* Z32, int64_t ld32, int64_t z32_stride, void* stream);

/*
 * Host function (no device work): the fill's basis tiles.  Greedy split of
 * the n_b bases (supp: n_b x wings int32, -1 = no segment) into runs of at
 * most max_basis consecutive bases whose wings touch at most max_seg
 * distinct segments.  Outputs (caller-allocated host arrays, n_b entries
 * each at most): first, nb, ns per tile; seg (tile-major, max_seg columns,
 * sorted, -1 padded); loc (n_b x wings: a wing's slot in its tile's list,
 * -1 for no segment); *n_tile.  The tiling itself has no counterpart in the
 * reference (its fill is organised by observer chunks, bspline.py:2386).
 */
mw_status mw_build_tiles(const int32_t* supp, int64_t n_b, int32_t wings, int32_t max_basis, int32_t max_seg,
                         int32_t* first, int32_t* nb, int32_t* ns, int32_t* seg, int32_t* loc, int64_t* n_tile);

/*
 * Host function (no device work): the basis polynomials of
 * _build_basis_polynomials (bspline.py:1318-1414) for m kept bases, basis b
 * being local basis js[b] of wire bw[b].  garc: every wire's knot arc
 * positions back to back (wire w at arc_off[w], wire_n[w] + 1 values);
 * wire_first[w]: global index of its first segment.  Outputs supp (m x
 * (d+1) int32, -1 where a wing has no segment) and poly (m x (d+1) x (d+1):
 * wing a's monomial coefficients in the local arc length).
 */
mw_status mw_basis_polys(const double* garc, const int64_t* arc_off, const int64_t* wire_n, const int64_t* wire_first,
                         int64_t n_wires, int32_t degree, const int64_t* js, const int64_t* bw, int64_t m,
                         int32_t* supp, double* poly);

/*
 * Y (n_out x ncols, complex128 column-major, ld ldy) = S X with S sparse in
 * CSR form (row_ptr[n_out + 1], col_idx, vals interleaved re/im; a row's
 * entries are summed in stored order, so results are deterministic) and X
 * column-major with ld ldx.  The port and KCL matrices of the solve are a
 * few nonzeros per row: Y = B^T X (bspline.py:4179) and the Schur products
 * A Xc, A W (bspline.py:2984-2987) as sparse gathers instead of dense GEMMs
 * whose inner dimension is the number of unknowns.
 */
mw_status mw_csr_mm_c128(int64_t n_out, int64_t ncols, const int64_t* row_ptr, const int64_t* col_idx,
                         const double* vals, const double* X, int64_t ldx, double* Y, int64_t ldy, void* stream);

/*
 * C = alpha * op(A) * op(B) + beta * C for complex128 column-major
 * matrices, op = 'N' or 'T' (transA/transB 0/1).  Used for the KCL Schur
 * step and Y = B^T X (bspline.py:2984-2989, 4179).
 */
mw_status mw_zgemm(int32_t transA, int32_t transB, int64_t m, int64_t n, int64_t k,
                   double alpha_re, double alpha_im, const double* A, int64_t lda,
                   const double* B, int64_t ldb, double beta_re, double beta_im,
                   double* C, int64_t ldc, void* stream);

/* ------------------------------------------------------------------------
 * Sommerfeld ground (ground_model="sommerfeld")
 * ------------------------------------------------------------------------ */

/*
 * One (R1, theta) interpolation grid of the four remainder surfaces
 * (I_rho^V, I_z^V, I_rho^H, I_phi^H), the layout of SommerfeldGrid
 * (_sommerfeld.py:648-813, flattened as grid_cpp_args :917): 4 regions
 * (R1 <= r_break / <= r_near, theta <= / > th_split) or 6 (plus the far
 * zone past r_near).  Region r has n_r[r] x n_th[r] nodes at
 * (r0 + i dr, th0 + j dth), stored node-major from node offset[r]:
 * vals[((offset[r] + i n_th[r] + j) * 4 + s)] complex128, s the surface.
 * value_scale multiplies every interpolated surface (the frequency factor
 * (omega mu)/(omega0 mu0) of a wavelength-normalised master, else 1).
 */
typedef struct mw_somm_grid {
    int32_t       n_region;      /* 4 or 6                                  */
    int32_t       n_r[6], n_th[6];
    int64_t       offset[6];     /* first node of each region               */
    double        r0[6], dr[6], th0[6], dth[6];  /* lengths, radians       */
    double        r1_max, r_break, th_split, r_near;
    double        value_scale;
    const double* vals;          /* device, complex128 (nodes, 4)           */
} mw_somm_grid;

/*
 * The four surfaces at n_nodes grid nodes (device arrays r1, rho = R1 cos,
 * h = R1 sin, theta): eqs 156-159 from the six Sommerfeld integrals
 * (eqs 148-153, fig-13/14 contours), eqs 169-172 where r1 == 0.  out is
 * complex128 (n_nodes, 4).  Replaces iv_surfaces_direct (_sommerfeld.py:535)
 * over somm_six_integrals_batch (_accelerators.cpp:5792).  workspace:
 * mw_somm_surfaces_workspace_size() device bytes.
 */
size_t mw_somm_surfaces_workspace_size(void);
mw_status mw_somm_surfaces(int64_t n_nodes, const double* r1, const double* rho,
                           const double* h, const double* theta, double eps_re,
                           double eps_im, double k2, double omega, double mu,
                           double rtol, double* out, void* workspace, void* stream);

/* As mw_somm_surfaces with a permittivity per node (device arrays). */
mw_status mw_somm_surfaces_eps(int64_t n_nodes, const double* r1, const double* rho,
                               const double* h, const double* theta, const double* eps_re,
                               const double* eps_im, double k2, double omega, double mu,
                               double rtol, double* out, void* workspace, void* stream);

/*
 * out[m * n_src + n] = t_obs[m] . F(obs[m], src[n]) . t_src[n] (complex128)
 * for points (n, 3) and unit tangents (n, 3) on the device: the projected
 * remainder field of a unit current moment (eqs 143-147).  Replaces
 * remainder_field_proj_batch (_accelerators.cpp:5981; _sommerfeld.py:940).
 */
mw_status mw_somm_field_proj(int64_t n_obs, const double* obs, const double* t_obs,
                             int64_t n_src, const double* src, const double* t_src,
                             double ground_z, double k, const mw_somm_grid* grid,
                             double* out, void* stream);

/*
 * Z -= Q (and Z32 = complex64(Z) where Z32 != NULL): the Galerkin block of
 * the remainder field over n_qp Gauss nodes per segment on the fill's basis
 * tiles.  Replaces sommerfeld_remainder_bspline_Q (_accelerators.cpp:6081)
 * as called by _Z_sommerfeld_remainder (bspline.py:1791-1915).
 */
mw_status mw_somm_remainder_q(const mw_segments* seg, const mw_basis* basis,
                              const mw_somm_grid* grid, int32_t n_qp, double ground_z,
                              double k, double* Z, int64_t ldz, float* Z32,
                              int64_t ldz32, void* stream);

/*
 * *out (device double) = the largest distance from a segment endpoint to
 * the ground image of another (unscaled; the grid sizing multiplies by
 * 1.001).  Replaces max_image_distance (_sommerfeld.py:154-205).
 */
mw_status mw_max_image_distance(int32_t n_seg, const double* seg_l, const double* seg_r,
                                double ground_z, double* out, void* stream);

/* ------------------------------------------------------------------------
 * Learned Sommerfeld surrogate (no reference counterpart: the reference
 * tabulates the remainder surfaces by quadrature, _sommerfeld.py:648-813)
 *
 * A 5 -> 128 -> 128 -> 128 -> 128 -> 8 MLP with GELU.  Parameters are one
 * flat FP32 vector of mw_mlp_param_count() entries, layer by layer
 * [W_l (out x in, row-major), b_l]; the forward pass uses a BF16 copy of it
 * (mw_mlp_to_bf16) with FP32 accumulation.  Inputs are 5 normalised
 * features per row, outputs 8 (Re/Im of the four surfaces, scaled).
 * ------------------------------------------------------------------------ */
int32_t mw_mlp_param_count(void);
size_t mw_mlp_train_workspace_size(int32_t batch);
mw_status mw_mlp_to_bf16(const float* params, void* params_bf16, void* stream);
/* FP32 forward of the training numerics: Y (n x 8) from X (n x 5). */
mw_status mw_mlp_forward(int32_t n, const float* X, const void* params_bf16, const float* params,
                         float* Y, void* workspace, size_t workspace_bytes, void* stream);
/* Gradient of the mean squared error against T (n x 8), and the loss. */
mw_status mw_mlp_grad(int32_t n, const float* X, const float* T, const void* params_bf16,
                      const float* params, float* grad, float* loss, void* workspace,
                      size_t workspace_bytes, void* stream);
/* One Adam step (bias-corrected, step >= 1) on a batch; *loss += batch loss.
 * rows != NULL: the batch is rows X[rows[i]], T[rows[i]] of a larger set. */
mw_status mw_mlp_train_step(int32_t n, const float* X, const float* T, const int64_t* rows, float* params,
                            void* params_bf16, float* adam_m, float* adam_v, int32_t step,
                            float lr, float beta1, float beta2, float eps, float* loss,
                            void* workspace, size_t workspace_bytes, void* stream);
/* Tensor-core (tcgen05, BF16 weights, hi/lo BF16 activations) inference;
 * *err (device) is set non-zero if a bounded wait timed out. */
mw_status mw_mlp_infer(int64_t n, const float* X, const void* params_bf16, const float* params,
                       float* Y, int32_t* err, void* stream);

/*
 * Z -= Q with the four surfaces predicted by the surrogate instead of
 * interpolated from a grid (mw_somm_remainder_q's contract otherwise).
 * struct_features: the three per-structure inputs (normalised log|eps~|,
 * arg eps~, log f); value_scale: output scale x (omega mu)/(omega0 mu0).
 * Every node pair must lie in the surrogate's domain (the caller checks).
 */
mw_status mw_somm_remainder_q_mlp(const mw_segments* seg, const mw_basis* basis,
                                  const void* params_bf16, const float* params,
                                  const float* struct_features, double wavelength,
                                  double value_scale, int32_t n_qp, double ground_z, double k,
                                  double* Z, int64_t ldz, float* Z32, int64_t ldz32,
                                  int32_t* err, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MOMWIRE_B200_H */
