/*
 * ceres_b200.h - C ABI of the B200 (sm_100a) Schur bundle-adjustment kernels.
 *
 * Plain C: raw device pointers, sizes and a cudaStream_t (passed as void*).
 * Every entry point returns 0 on success or a negative CERES_B200_E* code and
 * never allocates device memory; the caller owns every buffer named in
 * ceres_b200_ba_t (the Python host allocates them with torch).
 *
 * The reference (ceres-torch) computes this path in Python/PyTorch on a dense
 * Jacobian; each entry point below names the reference code it replaces
 * (paths relative to the ceres-torch project root).
 */
#ifndef CERES_B200_H
#define CERES_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CERES_B200_ABI_VERSION 5

/* status codes */
#define CERES_B200_OK 0
#define CERES_B200_EINVAL (-1)       /* bad argument (null pointer, size, enum) */
#define CERES_B200_ECUDA (-2)        /* a CUDA launch/runtime call failed */
#define CERES_B200_ESMEM (-3)        /* shared memory request above the device limit */
#define CERES_B200_ECOOP (-4)        /* cooperative launch not possible */
#define CERES_B200_ETOOBIG (-5)      /* size above a fixed capacity */

/* device-side error bits, OR-ed into stats[CERES_B200_STAT_ERROR] */
#define CERES_B200_DEVERR_LOSS 1     /* rho'' > 0 but rho' <= 0 (losses.py:177-179) */
#define CERES_B200_DEVERR_BARRIER 2  /* a grid barrier wait hit its iteration limit */
#define CERES_B200_DEVERR_NOT_PD 4   /* the dense reduced camera matrix was not positive definite */

/* loss kinds (losses.py:21-133) */
enum {
  CERES_B200_LOSS_TRIVIAL = 0,
  CERES_B200_LOSS_HUBER = 1,
  CERES_B200_LOSS_SOFTLONE = 2,
  CERES_B200_LOSS_CAUCHY = 3,
  CERES_B200_LOSS_ARCTAN = 4,
  CERES_B200_LOSS_TOLERANT = 5,
  CERES_B200_LOSS_TUKEY = 6
};

/* preconditioners for the reduced camera system (types.py:26-33) */
enum {
  CERES_B200_PRECOND_IDENTITY = 0,
  CERES_B200_PRECOND_JACOBI = 1,
  CERES_B200_PRECOND_SCHUR_JACOBI = 2,
  /* SCHUR_POWER_SERIES_EXPANSION (linear.py:482-497): blocks of the damped Hbb,
   * series in ceres_b200_ba_pcg_spse; single-problem path only */
  CERES_B200_PRECOND_SCHUR_POWER_SERIES = 3,
  /* CLUSTER_JACOBI / CLUSTER_TRIDIAGONAL (linear.py:1032-1085): the inverse of S kept on
   * the visibility cluster pairs, built by ceres_b200_ba_cluster_factor and applied by
   * ceres_b200_ba_pcg_cluster; camera_assemble treats it as IDENTITY */
  CERES_B200_PRECOND_CLUSTER = 4
};
/* or-ed into camera_assemble's preconditioner: also build the Hbb blocks of the
 * SPSE initial point (use_spse_initialization, linear.py:745-756) in the scratch */
#define CERES_B200_PRECOND_FLAG_SPSE_BASE 0x100

/* precision of the Jacobian store, point-block inverses and PCG vectors */
enum { CERES_B200_FP64 = 0, CERES_B200_FP32 = 1 };

/* indices into the float64 stats vector (length CERES_B200_NSTATS) */
enum {
  CERES_B200_STAT_COST = 0,          /* sum_i 0.5 rho(|r_i|^2) at the current parameters */
  CERES_B200_STAT_GMAX_P = 1,        /* max |J^T r| over point columns */
  CERES_B200_STAT_GSQ_P = 2,         /* |J^T r|^2 over point columns */
  CERES_B200_STAT_GMAX_C = 3,        /* max |J^T r| over camera columns */
  CERES_B200_STAT_GSQ_C = 4,         /* |J^T r|^2 over camera columns */
  CERES_B200_STAT_CAND_COST = 5,     /* cost at the candidate parameters */
  CERES_B200_STAT_MODEL = 6,         /* 0.5|r|^2 - 0.5|r + J step|^2 (not clamped) */
  CERES_B200_STAT_STEP_SQ_P = 7,     /* |step|^2 over point columns */
  CERES_B200_STAT_STEP_SQ_C = 8,     /* |step|^2 over camera columns */
  CERES_B200_STAT_NONFINITE = 9,     /* count of non-finite step entries */
  CERES_B200_STAT_PCG_ITERS = 10,    /* PCG iterations of the last solve */
  CERES_B200_STAT_PCG_SUCCESS = 11,  /* 1 if the PCG met its tolerance */
  CERES_B200_STAT_PCG_RNORM = 12,    /* |r| at PCG exit */
  CERES_B200_STAT_ERROR = 13,        /* OR of CERES_B200_DEVERR_* bits */
  CERES_B200_STAT_RHS_NORM = 14,     /* |rhs| of the reduced camera system */
  CERES_B200_STAT_REFINE_RNORM = 15, /* float64 residual |rhs - S x| after refinement */
  CERES_B200_STAT_CAND_STATE_SQ_P = 16, /* |candidate points|^2 (all point blocks) */
  CERES_B200_STAT_CAND_STATE_SQ_C = 17, /* |candidate cameras|^2 (all camera blocks) */
  CERES_B200_NSTATS = 18
};

/*
 * Device-resident state of one bundle-adjustment problem.
 *
 * Observations live in a sliced-ELL "point-major" store: points are sorted by
 * track length (descending, stable in point id) and cut into slices of 32;
 * lane l of slice s owns point q = 32 s + l (q is the "sorted point" index);
 * observation k of that point sits in slot slice_base[s] + 32 k + l.
 * Padding slots carry slot_cam = -1. A camera-major list (cam_offsets /
 * cam_entries) names, for each camera, the (slot, q) pairs of its
 * observations in increasing slot order.
 *
 * Jacobian records are 24 scalars per slot (camera row 0 [9], camera row 1
 * [9], point row 0 [3], point row 1 [3]) of float (FP32) or double (FP64).
 * When cm_jac is set, the evaluation writes each record twice: at its slot
 * (point-major) and at its camera-major position (cm_jac[e], e the entry's index
 * in cam_entries), and the camera-side passes stream the copy; with cm_jac null
 * they gather the records by slot.
 * Camera work items cut every camera's entries into consecutive runs; item i =
 * (camera, first entry) covers its entries up to the next item of the same camera
 * (or the camera's last entry), and cam_items[c] .. cam_items[c + 1] - 1 are camera
 * c's items. The run length is the host's choice (the autotuner picks it);
 * CERES_B200_CAM_ITEM is the default.
 */
#define CERES_B200_CAM_ITEM 256
typedef struct ceres_b200_ba_t {
  int32_t num_cameras;
  int32_t num_observations;  /* real observations (entries of the camera-major list) */
  int32_t num_points;        /* sorted point slots = 32 * num_slices (padded) */
  int32_t num_slices;
  int32_t num_slots;         /* sum over slices of 32 * slice_len */
  int32_t max_slice_len;
  int32_t precision;         /* CERES_B200_FP64 / CERES_B200_FP32 */
  int32_t has_duplicate_cameras; /* 1 if some point sees one camera twice */
  int32_t loss_kind;         /* CERES_B200_LOSS_* */
  double loss_a, loss_b;     /* loss parameters (a; b only for Tolerant) */
  double loss_scale;         /* ScaledLoss factor (1 when unscaled) */
  int32_t inner_loss_kind;   /* ComposedLoss inner kind, -1 when not composed */
  int32_t pad0;
  double inner_a, inner_b;
  double inner_scale;        /* ScaledLoss factor of the inner loss (1 when unscaled) */

  /* structure (read-only) */
  const int32_t* slice_base;   /* [num_slices] first slot of the slice (multiple of 32) */
  const int32_t* slice_len;    /* [num_slices] observations per lane (max over lanes) */
  const int32_t* slot_cam;     /* [num_slots] camera of the slot, -1 padding */
  const double* slot_obs;      /* [num_slots][2] observed pixel */
  const int32_t* cam_offsets;  /* [num_cameras + 1] */
  const int32_t* cam_entries;  /* [num_observations][2] (slot, q) grouped by camera */
  const uint8_t* cam_const;    /* [num_cameras] 1 = constant camera block */
  const uint8_t* pt_const;     /* [num_points] 1 = constant point or padding lane */

  /* parameters (float64 master copies) */
  double* cameras;             /* [num_cameras][9] current */
  double* points;              /* [num_points][3] current (sorted-point order) */
  double* cand_cameras;        /* [num_cameras][9] candidate = current + step */
  double* cand_points;         /* [num_points][3] */

  /* per-slot evaluation */
  void* jac;                   /* [num_slots][24] float or double, 32-byte aligned */
  double* res;                 /* [num_slots][2] corrected residuals, 16-byte aligned */

  /* point-side Schur pieces */
  double* point_raw;           /* [num_points][9] J_p^T J_p (symmetric, 6) and J_p^T r (3), written by evaluate */
  void* winv;                  /* [num_points][6] (W + D_p)^-1, symmetric, float or double, 8-byte aligned */
  double* winv_ga;             /* [num_points][3] W^-1 g_a with g_a = -J_p^T r, 8-byte aligned */
  double* step_points;         /* [num_points][3] */

  /* camera-side Schur pieces */
  double* cam_diag;            /* [num_cameras][9] damping D_c added to the diagonal */
  void* precond;               /* [num_cameras][81] preconditioner inverse blocks, double in both precisions */
  double* rhs;                 /* [num_cameras][9] reduced right-hand side */
  double* step_cameras;        /* [num_cameras][9] */

  /* PCG vectors (float64 in both precisions), [num_cameras][9] each */
  void* pcg_x;
  void* pcg_r;
  void* pcg_z;
  void* pcg_p;                 /* [2][num_cameras][9] double-buffered direction */
  void* pcg_ap;

  /* camera-major copy of the Jacobian store and the camera work items */
  const int32_t* slot_pos;     /* [num_slots] camera-major position of the slot's observation, -1 padding */
  void* cm_jac;                /* [num_observations][24] float or double, 32-byte aligned, or null */
  const int32_t* cam_items;    /* [num_cameras + 1] first item of each camera */
  const int32_t* items;        /* [num_items][2] (camera, first entry) */
  int32_t num_items;
  int32_t max_camera_obs;      /* largest entry count of a camera */

  /* scratch owned by the caller */
  void* scratch;               /* per-CTA partial sums; see ceres_b200_scratch_bytes */
  int64_t scratch_bytes;
  uint32_t* counters;          /* [16] zero-initialised once; kernels leave them zero */
  double* stats;               /* [CERES_B200_NSTATS] */

  /* the explicit reduced camera matrix in a fixed summation order (dense_schur_solve,
   * schur_matrix), listed block by block (cameras a <= b), each block's contributions
   * (slot i of a, slot j of b, point lane q) with the points ascending: -G_i W_q^-1 G_j^T,
   * plus Jc_i^T Jc_i where i == j (a diagonal block lists each observation of the
   * camera with itself and every ordered pair of its observations of one point).
   * Null: the blocks are summed with float64 atomics, in an order that varies from run
   * to run. */
  const int32_t* schur_blocks;       /* [num_schur_blocks][2] cameras a <= b */
  const int64_t* schur_block_start;  /* [num_schur_blocks + 1] first contribution of each block */
  const int32_t* schur_contrib;      /* [contributions][3] (slot i, slot j, point lane q) */
  int64_t num_schur_blocks;
} ceres_b200_ba_t;

/* ABI version of the loaded library (CERES_B200_ABI_VERSION). */
int ceres_b200_abi_version(void);

/* sizeof(ceres_b200_ba_t) as compiled into the library (binding check). */
int ceres_b200_ba_struct_bytes(void);

/* Number of kernels this library has launched since it was loaded. */
uint64_t ceres_b200_launch_count(void);

/* Bytes of scratch the PCG and reductions need for this problem on this device. */
int ceres_b200_scratch_bytes(const ceres_b200_ba_t* ba, int64_t* bytes_out);

/*
 * Residuals, Jacobian and robust correction at ba->cameras / ba->points.
 * Writes ba->res, ba->jac and ba->point_raw (when with_jacobian) and stats[COST].
 * Replaces Problem.evaluate (problem.py:377-413, :486-520), the autodiff
 * Jacobian of the Snavely residual (costs.py:31-44 over
 * examples/simple_bundle_adjuster.py:73-79, rotation.py:104-110, :211-222)
 * and the Ceres corrector (losses.py:158-193).
 */
int ceres_b200_ba_evaluate(const ceres_b200_ba_t* ba, int with_jacobian, void* stream);

/*
 * The same evaluation as ceres_b200_ba_evaluate for callers that cannot allocate
 * device memory - for example a host runtime whose device memory is owned by
 * another allocator, or one that forbids allocation after start-up - and so have
 * no scratch buffer to put in ba->scratch (it is ignored here). The per-CTA cost
 * partials go to a static 256 KB array inside the library (32768 float64 slots,
 * one per evaluation CTA; each loaded GPU keeps it until the process exits). The
 * first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) and remembers the context it was taken in; a later call in
 * a new context of that device (after a device reset) looks it up again. Make the
 * first call in each context before any stream capture. Sizes
 * that need more slots return CERES_B200_ETOOBIG. Calls share the array: two
 * calls that overlap on the GPU race. No memory is allocated or freed.
 * This entry point has no counterpart in the reference.
 */
int ceres_b200_ba_evaluate_noalloc(const ceres_b200_ba_t* ba, int with_jacobian, void* stream);

/*
 * Point side of the Schur system for a trust-region radius, from the point
 * sums of the last evaluation: Jacobi damping D_p (linear.py:539-551),
 * W_p = J_p^T J_p + D_p inverted per point
 * (linear.py:808 on the block-diagonal Haa), W^-1 g_a, and the point
 * gradient stats. Replaces the Haa part of linear.py:794-839.
 */
int ceres_b200_ba_point_assemble(const ceres_b200_ba_t* ba, double radius, double min_diagonal,
                                 double max_diagonal, int jacobi_scaling, void* stream);

/*
 * Camera side: damping D_c, reduced rhs = g_b - H_ba W^-1 g_a, camera
 * gradient stats and the preconditioner blocks of S (SCHUR_JACOBI: inverse
 * of each 9x9 diagonal block of S, Cholesky with an LU fallback as in
 * linear.py:1156-1182; JACOBI: 1/max(diag S, eps), linear.py:530).
 * Replaces the Hbb / rhs part of linear.py:794-839 and linear.py:462-536.
 */
int ceres_b200_ba_camera_assemble(const ceres_b200_ba_t* ba, double radius, double min_diagonal,
                                  double max_diagonal, int jacobi_scaling, int preconditioner,
                                  void* stream);

/*
 * Preconditioned conjugate gradients on S x = rhs with the implicit Schur
 * product S p = (U + D_c) p - H_ba W^-1 H_ab p streamed from the Jacobian
 * store, in one cooperative persistent launch (x0 = 0; stop when
 * |r| <= tolerance * max(|rhs|, eps) after min_iterations).
 * Writes ba->step_cameras and stats[PCG_*]. With FP32 precision and
 * max_refinements > 0, float64 refinement passes recompute rhs - S x with
 * float64 accumulation and solve for a correction.
 * Replaces linear.py:702-776 and the PCG of linear.py:1216-1256.
 */
int ceres_b200_ba_pcg(const ceres_b200_ba_t* ba, int preconditioner, int min_iterations,
                      int max_iterations, double tolerance, int max_refinements, void* stream);

/*
 * ceres_b200_ba_pcg with the power series of SCHUR_POWER_SERIES_EXPANSION
 * (preconditioner CERES_B200_PRECOND_SCHUR_POWER_SERIES; linear.py:59-67):
 * z = sum_i (B E)^i B r, B the inverted damped Hbb blocks, E = H_ba W^-1 H_ab,
 * term i >= 1 added while |term| > spse_tolerance * max(|sum so far|, 1), at
 * most spse_terms terms (max_num_spse_iterations). spse_init != 0: the start
 * point is x0 = that series applied to rhs with the Hbb blocks of
 * camera_assemble's CERES_B200_PRECOND_FLAG_SPSE_BASE (or of the preconditioner
 * itself when it is the power series), and r0 = rhs - S x0 (linear.py:745-756,
 * :1226-1227). spse_terms >= 1 and spse_tolerance >= 0 when either is used.
 */
int ceres_b200_ba_pcg_spse(const ceres_b200_ba_t* ba, int preconditioner, int min_iterations,
                           int max_iterations, double tolerance, int max_refinements, int spse_terms,
                           double spse_tolerance, int spse_init, void* stream);

/*
 * y = S x for a camera vector x (float64 in and out, accumulated in float64
 * from the stored Jacobian). Replaces the S @ p of linear.py:1237.
 */
int ceres_b200_ba_schur_matvec(const ceres_b200_ba_t* ba, const double* x, double* y, void* stream);

/*
 * Back-substitution of the point step (linear.py:766), candidate parameters
 * x + step (problem.py:462-474, manifolds.py:81-82), the model decrease
 * 0.5|r|^2 - 0.5|r + J step|^2 (solver.py:798-802) and the candidate cost
 * (solver.py:216), in one pass over the observations.
 */
int ceres_b200_ba_step(const ceres_b200_ba_t* ba, void* stream);

/*
 * Exact solve of the reduced camera system: assembles the explicit float64
 * S = H_bb - H_ba H_aa^-1 H_ab (+ D_c) into work (ceres_b200_dense_schur_bytes
 * bytes) and solves S x = rhs by Cholesky (one CTA in shared memory up to
 * 17 cameras, a cooperative global-memory factorisation above that). Writes
 * ba->step_cameras. Replaces schur_solve_dense (linear.py:667-699), which the
 * reference reaches for DENSE_SCHUR and, via solver.py:791-792, SPARSE_SCHUR,
 * and the dense block-Schur split of native/cuda/ceres_torch_cuda_kernel.cu:107-132.
 */
int ceres_b200_dense_schur_bytes(const ceres_b200_ba_t* ba, int64_t* bytes_out);
int ceres_b200_ba_dense_schur_solve(const ceres_b200_ba_t* ba, double* work, void* stream);

/*
 * Cholesky solve of a dense symmetric positive definite float64 system
 * H x = rhs (H [n][n] row-major, overwritten by its factor). flags points to
 * four zero-initialised uint32 words (three for the grid barrier, one for
 * CERES_B200_DEVERR_NOT_PD). Used by the dense-A registry backends after
 * H = A^T A + diag(d) is formed; replaces the at::linalg_solve calls of
 * native/cuda/ceres_torch_cuda_kernel.cu:93-105.
 */
int ceres_b200_dense_cholesky_solve(double* H, const double* rhs, double* x, int64_t n, uint32_t* flags,
                                    void* stream);

/*
 * The explicit reduced camera matrix S = H_bb - H_ba H_aa^-1 H_ab + D_c (float64, [n][n]
 * row-major, n = 9 num_cameras) at the last evaluation and assembly; the block of a
 * constant camera is the identity. With point_assemble / camera_assemble called with
 * radius = +inf (no damping), S^-1 is the camera block of (J^T J)^-1: the camera
 * covariance that covariance.py:86-445 computes from the dense Jacobian's SVD.
 */
int ceres_b200_ba_schur_matrix(const ceres_b200_ba_t* ba, double* S, void* stream);

/*
 * inv = A^-1 for a symmetric positive definite float64 A ([n][n], overwritten by its
 * Cholesky factor; n <= 32768): cooperative right-looking Cholesky, then one CTA per
 * column of the inverse. flags: four uint32 (three for the grid barrier, zeroed here;
 * flags[3] gets CERES_B200_DEVERR_NOT_PD when A is not positive definite, which the
 * caller zeroes). Used for the camera covariance (covariance.py:86-445).
 */
int ceres_b200_dense_spd_inverse(double* A, double* inv, int64_t n, uint32_t* flags, void* stream);

/*
 * Visibility-cluster preconditioner of the reduced camera system (CLUSTER_JACOBI and
 * CLUSTER_TRIDIAGONAL, linear.py:498-521 and :1032-1085). The host clusters the cameras
 * (linear.py:842-1028) and passes the kept camera block pairs; the kept matrix is block
 * diagonal over the connected groups of cameras ("components") that the pairs link.
 * All pointers are device memory; the struct itself is read on the host.
 */
typedef struct ceres_b200_clusters {
  int32_t num_components;
  int32_t num_pairs;           /* kept camera block pairs (a, b), a <= b */
  int32_t max_dim;             /* largest component dimension (9 x its cameras) */
  int32_t tridiagonal;         /* 1: CLUSTER_TRIDIAGONAL (halve the blocks between
                                * clusters when the kept matrix is not positive definite) */
  int64_t num_elements;        /* comp_base[num_components]: length of inv */
  const int32_t* pairs;        /* [num_pairs][2] camera ids a <= b */
  const int32_t* entries;      /* [num_observations][2] (slot, point lane) of every camera,
                                * camera-major (offsets cam_offsets), by point lane within a camera */
  const int32_t* cam_comp;     /* [num_cameras] component of the camera, -1 for one outside */
  const int32_t* cam_pos;      /* [num_cameras] position of the camera in its component */
  const int32_t* cam_cluster;  /* [num_cameras] cluster of the camera */
  const int32_t* comp_cams;    /* the cameras of the components, component after component */
  const int32_t* comp_cam_off; /* [num_components + 1] */
  const int64_t* comp_base;    /* [num_components + 1] first element of the component's
                                * matrix in inv (row-major, dim x dim) */
  const int64_t* comp_piv;     /* [num_components + 1] first element of its sweep workspace in piv:
                                * 64 x dim + 32 x 32 doubles (a block's 32 rows, A11^-1 times them,
                                * and the block's inverse) */
  double* inv;                 /* [comp_base[num_components]] the kept matrices, then their inverses */
  double* piv;                 /* [comp_piv[num_components]] sweep workspace */
  uint32_t* flags;             /* [8], zeroed by cluster_factor: [0] the kept matrix was not
                                * positive definite, [1] nor was the halved one, [2] a zero
                                * pivot, [3..5] grid barrier words ([5]: CERES_B200_DEVERR_BARRIER
                                * when a barrier wait gave up) */
} ceres_b200_clusters_t;

/* sizeof(ceres_b200_clusters_t) as compiled into the library (binding check). */
int ceres_b200_clusters_struct_bytes(void);

/*
 * Builds the kept matrices of S at the current assembly (float64 arithmetic on the
 * Jacobian store, deterministic: one warp per block pair, shared points in point order)
 * and inverts them with the symmetric sweep operator in one cooperative launch (all
 * components at once, 32 pivots per block, three grid barriers per block). Non-positive
 * pivots set flags[0]; with
 * tridiagonal set, the matrices are rebuilt with the blocks between different clusters
 * halved and inverted again (flags[1] when that one is not positive definite either,
 * where the reference falls back to a general solve of the same matrix, which the
 * sweep's inverse equals). A zero pivot sets flags[2]. Call after camera_assemble.
 */
int ceres_b200_ba_cluster_factor(const ceres_b200_ba_t* ba, const ceres_b200_clusters_t* cl, void* stream);

/*
 * ceres_b200_ba_pcg with z = M^-1 r from the inverses of ceres_b200_ba_cluster_factor
 * (one grid barrier more per iteration: z of a camera needs r of its whole component).
 */
int ceres_b200_ba_pcg_cluster(const ceres_b200_ba_t* ba, const ceres_b200_clusters_t* cl, int min_iterations,
                              int max_iterations, double tolerance, int max_refinements, void* stream);

/*
 * Check of the bounded waits of the cooperative kernels (failure detection without a
 * GPU fault): two CTAs meet at the grid barrier of ceres_b200_ba_pcg, except that the
 * second never arrives. The first gives up after spin_limit polls (at most the
 * library's own limit of 2^24), ORs CERES_B200_DEVERR_BARRIER into words[2] and
 * returns, so the context stays usable. words: three zero-initialised uint32 (arrival
 * count, generation, error flag). No counterpart in the reference.
 */
int ceres_b200_debug_barrier_timeout(uint32_t* words, uint32_t spin_limit, void* stream);

/* ------------------------------------------------------------------------------------
 * Batched solves: many independent bundle-adjustment problems in one persistent launch.
 *
 * Each thread-block cluster takes whole problems from a work counter (queue[0], zeroed
 * by the caller) and runs the complete Levenberg-Marquardt solve of one problem at a
 * time on the device: evaluation, Schur assembly, implicit-Schur PCG, step and the trust-region
 * decisions of ceres-torch's solver.py:35-357 (monotonic steps, ITERATIVE_SCHUR).
 * No host round trip happens between iterations; a problem's result does not depend
 * on the other problems of the batch. This has no counterpart in the reference, which
 * solves one problem per tc.solve call.
 *
 * Problems are concatenated: problem b owns cameras [cam_off[b], cam_off[b+1]),
 * slices [slice_off[b], slice_off[b+1]) and the sorted points 32 * slice_off[b] ...
 * of the same sliced-ELL layout as ceres_b200_ba_t (slot_cam holds the camera index
 * local to the problem; cam_entries hold (global slot, global sorted point)).
 * ---------------------------------------------------------------------------------- */
#define CERES_B200_BATCH_RESULT 16 /* float64 per problem in result[] */
#define CERES_B200_BATCH_TRACE 10  /* float64 per iteration record in trace[] */

enum { /* result[b * CERES_B200_BATCH_RESULT + i] */
  CERES_B200_BR_INITIAL_COST = 0,
  CERES_B200_BR_FINAL_COST = 1,
  CERES_B200_BR_RECORDS = 2,          /* iteration records written (iteration 0 included) */
  CERES_B200_BR_TERMINATION = 3,      /* CERES_B200_TERM_* */
  CERES_B200_BR_MESSAGE = 4,          /* CERES_B200_MSG_* */
  CERES_B200_BR_SUCCESSFUL = 5,
  CERES_B200_BR_UNSUCCESSFUL = 6,
  CERES_B200_BR_JACOBIAN_EVALS = 7,
  CERES_B200_BR_RESIDUAL_EVALS = 8,
  CERES_B200_BR_LINEAR_SOLVES = 9,
  CERES_B200_BR_ERROR = 10,           /* OR of CERES_B200_DEVERR_* bits */
  CERES_B200_BR_FINAL_GMAX = 11
};
enum { /* trace[(b * max_trace + k) * CERES_B200_BATCH_TRACE + i] */
  CERES_B200_BT_COST = 0,
  CERES_B200_BT_COST_CHANGE = 1,
  CERES_B200_BT_GMAX = 2,
  CERES_B200_BT_GNORM = 3,
  CERES_B200_BT_STEP_NORM = 4,
  CERES_B200_BT_RHO = 5,
  CERES_B200_BT_RADIUS = 6,
  CERES_B200_BT_LINEAR_ITERATIONS = 7,
  CERES_B200_BT_FLAGS = 8             /* bit 0 valid, bit 1 successful, bit 2 nonmonotonic */
};
enum { CERES_B200_TERM_CONVERGENCE = 0, CERES_B200_TERM_NO_CONVERGENCE = 1, CERES_B200_TERM_FAILURE = 2 };
enum {
  CERES_B200_MSG_GRADIENT = 0,        /* "Gradient tolerance reached." */
  CERES_B200_MSG_MAX_ITERATIONS = 1,  /* "Maximum iterations reached." */
  CERES_B200_MSG_INVALID_STEPS = 2,   /* "Too many invalid trust-region steps." */
  CERES_B200_MSG_PARAMETER = 3,       /* "Parameter tolerance reached." */
  CERES_B200_MSG_FUNCTION = 4,        /* "Function tolerance reached." */
  CERES_B200_MSG_MIN_RADIUS = 5       /* "Minimum trust-region radius reached." */
};

typedef struct ceres_b200_batch_t {
  int32_t num_problems;
  int32_t precision;            /* CERES_B200_FP64 or CERES_B200_FP32 (Jacobian store and PCG) */
  int32_t max_cameras;          /* largest camera count of a problem (sizes the shared memory) */
  int32_t has_duplicate_cameras;
  int32_t loss_kind;
  int32_t inner_loss_kind;
  double loss_a, loss_b, loss_scale, inner_a, inner_b, inner_scale;
  /* SolverOptions (types.py) */
  int32_t max_num_iterations;
  int32_t min_linear_solver_iterations;
  int32_t max_linear_solver_iterations;
  int32_t preconditioner;       /* CERES_B200_PRECOND_* */
  int32_t jacobi_scaling;
  int32_t max_consecutive_invalid_steps;
  int32_t max_refinements;      /* float64 refinement passes after a float32 PCG that missed eta */
  int32_t max_trace;            /* iteration records kept per problem */
  double function_tolerance, gradient_tolerance, parameter_tolerance, min_relative_decrease;
  double initial_radius, max_radius, min_radius, min_lm_diagonal, max_lm_diagonal, eta;
  /* per-problem offsets, num_problems + 1 entries each */
  const int32_t* cam_off;
  const int32_t* slice_off;
  /* layout (concatenated; see above) */
  const int32_t* slice_base;
  const int32_t* slice_len;
  const int32_t* slot_cam;
  const double* slot_obs;
  const int32_t* cam_offsets;   /* [total cameras + 1], into cam_entries */
  const int32_t* cam_entries;   /* [entries][2] */
  const uint8_t* cam_const;
  const uint8_t* pt_const;
  /* state (float64 unless noted) */
  double* cameras;              /* [total cameras][9], solved in place */
  double* points;               /* [32 * total slices][3] sorted order, solved in place */
  double* cand_cameras;
  double* cand_points;
  void* jac;                    /* [slots][24] float or double, 32-byte aligned */
  double* res;                  /* [slots][2] */
  double* point_raw;            /* [points][9] */
  void* winv;                   /* [points][6] float or double */
  double* winv_ga;              /* [points][3] */
  double* step_points;          /* [points][3] */
  double* cam_diag;             /* [cameras][9] */
  void* precond;                /* [cameras][81] double in both precisions */
  double* rhs;                  /* [cameras][9] */
  double* step_cameras;         /* [cameras][9] */
  double* cam_acc;              /* [cameras][72] */
  double* frames;               /* [cameras][24] */
  double* pcg;                  /* [8][9 * total cameras]: x, r, z, p (two buffers), Ap, refinement residual, spare */
  double* result;               /* [num_problems][CERES_B200_BATCH_RESULT] */
  double* trace;                /* [num_problems][max_trace][CERES_B200_BATCH_TRACE] */
  uint32_t* queue;              /* [1] work counter, zero before the launch */
} ceres_b200_batch_t;

/* sizeof(ceres_b200_batch_t) as compiled into the library (binding check). */
int ceres_b200_batch_struct_bytes(void);

/*
 * Solves every problem of the batch in one persistent launch. A thread-block cluster
 * of cluster_size CTAs (1, 2, 4, 8 or 16; 0 means 1) solves one problem at a time:
 * larger clusters give a problem more SMs (lower latency per problem), smaller ones
 * more problems in flight. CTA shapes (threads_per_cta, ctas_per_sm): (128, 1|2),
 * (128, 4), (256, 1), (256, 2), (512, 1); ctas_per_sm sets the register cap, 0 picks
 * (256, 1). Asynchronous on stream; results appear in result/trace and the
 * parameters are updated in place.
 */
int ceres_b200_batch_solve(const ceres_b200_batch_t* batch, int threads_per_cta, int ctas_per_sm, int cluster_size,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CERES_B200_H */
