/*
 * airt.h -- C-ABI of libairt, the B200 (sm_100a) engine behind the AIR Tools II
 * solver and operator API.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (AIRT_OK = 0) and leaves a message for airt_last_error() on failure.  Host
 * buffers are caller-owned, MATLAB column-major doubles; the library copies in,
 * keeps FP32 CSR/CSC matrices and FP64 vectors in HBM, and owns device memory
 * until airt_destroy().  Functions ending in _device take device pointers and
 * run on the problem's CUDA stream (airt_problem_stream) without host copies.
 * A handle keeps work buffers between calls, so calls on the same handle must
 * not overlap (one host thread at a time per handle); distinct handles are
 * independent.  airt_last_error() is per host thread.
 *
 * Reference interfaces replaced (AIR Tools II V1.0, paths inside its tree):
 *   airt_problem_from_csc  -> auxil/check_inputs.m:67-71 (matrix wrapped as afun)
 *   airt_problem_parallel  -> testprobs/paralleltomo.m:112-301
 *   airt_problem_fan       -> testprobs/fanlineartomo.m:141-358,
 *                             testprobs/fancurvedtomo.m:140-339
 *   airt_problem_seismic   -> testprobs/seismictomo.m:96-287
 *   airt_problem_spherical -> testprobs/sphericaltomo.m:108-270
 *   airt_apply             -> auxil/afun_matrix.m:44-53 and the isMatrix=0 handles
 *                             testprobs/paralleltomo.m:146-177,280-288
 *   airt_weights           -> auxil/get_mfun_dfun.m:43-250
 *   airt_rho               -> auxil/calc_relaxpar.m:91-103 (eigs of D*A'*M*A)
 *   airt_rho_custom        -> the same, custom weights of get_mfun_dfun.m:252-307
 *   airt_sirt              -> sirt/sirt.m:147-261 with auxil/check_stoprules.m:54-94,153-161
 *   airt_cart              -> cart/cart.m:139-320 (cart/columnaction.m)
 *   airt_fbp               -> auxil/fbp.m:40-79
 *   airt_art               -> art/art.m:138-309
 */
#ifndef AIRT_H
#define AIRT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define AIRT_OK 0
#define AIRT_ERR_ARG 1     /* invalid argument (size, pointer, option)      */
#define AIRT_ERR_OOM 2     /* device allocation failed                       */
#define AIRT_ERR_CUDA 3    /* CUDA runtime error                             */
#define AIRT_ERR_TIMEOUT 4 /* a bounded device wait gave up                  */
#define AIRT_ERR_UNSUPPORTED 5

/* ---- SIRT methods (sirt/sirt.m:17-26) ---------------------------------- */
#define AIRT_LANDWEBER 0
#define AIRT_CIMMINO 1
#define AIRT_CAV 2
#define AIRT_DROP 3
#define AIRT_SART 4
#define AIRT_CUSTOM 5 /* diagonal M and/or D given by the caller */

/* ---- stopping rules (auxil/check_stoprules.m) --------------------------- */
#define AIRT_STOP_NONE 0
#define AIRT_STOP_DP 1
#define AIRT_STOP_ME 2
#define AIRT_STOP_NCP 3 /* normalized cumulative periodogram, check_stoprules.m:97-150 */

/* ---- relaxation strategy (auxil/calc_relaxpar.m: casel) ----------------- */
#define AIRT_RELAX_CONST 1 /* relaxpar constant                     */
#define AIRT_RELAX_LINE 2  /* line search, sirt/sirt.m:219-222      */
#define AIRT_RELAX_TABLE 3 /* per-iteration table (psi1/psi2 rules) */

/* ---- bound kinds --------------------------------------------------------- */
#define AIRT_BOUND_NONE 0
#define AIRT_BOUND_SCALAR 1
#define AIRT_BOUND_VECTOR 2

typedef struct airt_problem airt_problem;

typedef struct {
    int method;               /* AIRT_LANDWEBER..AIRT_CUSTOM                    */
    const double *M;          /* AIRT_CUSTOM: m-vector diagonal of M, or NULL=I  */
    const double *D;          /* AIRT_CUSTOM: n-vector diagonal of D, or NULL=I  */
    int relax_kind;           /* AIRT_RELAX_*                                    */
    double relaxpar;          /* AIRT_RELAX_CONST                                */
    const double *relax_table;/* AIRT_RELAX_TABLE: kmax entries                  */
    int stoprule;             /* AIRT_STOP_*                                     */
    double taudelta;          /* DP / ME threshold                               */
    int lb_kind, ub_kind;     /* AIRT_BOUND_*                                    */
    double lb, ub;            /* scalar bounds                                   */
    const double *lbv, *ubv;  /* vector bounds (n entries)                       */
    int64_t kmax;             /* maximum number of iterations (K(end))           */
    /* NCP only (options.stoprule.res_dims / ncp_smooth, check_inputs.m:171-209):
       the residual is reshaped column-major to ncp_rows x ncp_cols (ncp_cols = 1
       for a 1D res_dims) and ncp_smooth values are compared.                    */
    int ncp_rows, ncp_cols, ncp_smooth;
    /* AIRT_CUSTOM only: M (D) points to a full column-major m x m (n x n)
       matrix instead of a diagonal, the Mflag/Dflag = 2 case of
       auxil/get_mfun_dfun.m:252-307 (M*r and D*g are dense products).      */
    int M_full, D_full;
} airt_sirt_opts;

typedef struct {
    int order_kind;           /* 0 kaczmarz, 1 symkaczmarz, 2 caller row list  */
    const int64_t *rows;      /* order_kind 2: 0-based rows, nrows per sweep;
                                 rows_per_sweep_stride>0 gives a new list per
                                 sweep (randkaczmarz index stream)             */
    int64_t nrows;
    int64_t rows_stride;      /* 0 = same list every sweep                      */
    double relaxpar;          /* constant relaxpar (default 1)                  */
    const double *relax_table;/* optional relaxpar per row step: kmax blocks of
                                 one entry per step of a sweep (the values of
                                 the art.m:273-275 handle), or NULL           */
    double damp;              /* art.m:206                                      */
    int stoprule;             /* AIRT_STOP_NONE, AIRT_STOP_DP or AIRT_STOP_NCP  */
    double taudelta;
    int lb_kind, ub_kind;
    double lb, ub;
    const double *lbv, *ubv;
    int64_t kmax;             /* sweeps (already halved for symkaczmarz)        */
    int ncp_rows, ncp_cols, ncp_smooth; /* NCP, as in airt_sirt_opts           */
} airt_art_opts;

typedef struct {
    int order_kind;           /* 0 columnaction (every nonzero column, in order),
                                 2 caller column list                          */
    const int64_t *cols;      /* order_kind 2: 0-based columns, ncols of them  */
    int64_t ncols;
    double relaxpar;          /* scalar relaxpar (default 0.25, calc_relaxpar.m) */
    double damp;              /* cart.m: normAj + damp*max(normAj)             */
    int stoprule;             /* AIRT_STOP_NONE, AIRT_STOP_DP or AIRT_STOP_NCP  */
    double taudelta;
    int lb_kind, ub_kind;
    double lb, ub;
    const double *lbv, *ubv;
    int64_t kmax;
    int ncp_rows, ncp_cols, ncp_smooth;
    double thr;               /* flagging threshold THR (check_inputs.m, 1e-4)  */
    int64_t kbegin;           /* first sweep that may flag (Kbegin, 10)          */
    int64_t nunflag;          /* unflagging parameter (Nunflag, round(kmax/4))   */
    uint64_t seed;            /* seed of the unflagging draws                    */
} airt_cart_opts;

typedef struct {
    int stoprule;       /* 0 max iterations, 1 NCP, 2 DP, 3 ME (check_stoprules.m:27-31) */
    int64_t finaliter;  /* iterations performed                                 */
    double relaxpar;    /* relaxpar of the final iteration                      */
    int64_t nsaved;     /* columns written to X                                 */
    double gpu_ms;      /* device time of the call (CUDA events)                */
} airt_info;

/* ---- errors and version -------------------------------------------------- */
const char *airt_last_error(void);
int airt_version(void);

/* ---- problem construction ------------------------------------------------- */
/* MATLAB sparse layout (mxGetJc / mxGetIr / mxGetPr): jc n+1 column starts,
 * ir nnz row indices, pr nnz values, in MATLAB's canonical form (row indices
 * strictly increasing within each column: AIRT_ERR_ARG otherwise).  Replaces
 * the matrix branch of auxil/check_inputs.m:67-71 and auxil/afun_matrix.m:44-53. */
int airt_problem_from_csc(int64_t m, int64_t n, const uint64_t *jc, const uint64_t *ir,
                          const double *pr, airt_problem **out);

/* paralleltomo geometry (testprobs/paralleltomo.m:112-301): nA angles given
 * as cosd/sind tables, p ray offsets (linspace(-d/2,d/2,p)).  matrix_free=0
 * builds the system matrix on the GPU (bit-exact sparsity with the FP64 ray
 * trace); matrix_free=1 keeps only the geometry and recomputes rays. */
int airt_problem_parallel(int N, int nA, const double *cos_t, const double *sin_t, int p,
                          const double *offsets, int matrix_free, airt_problem **out);

/* fanlineartomo geometry (testprobs/fanlineartomo.m:141-358): source
 * distance R (absolute), per-angle cosd/sind of theta, per-detector cosd/sind
 * of the ray angle omega. */
int airt_problem_fan(int N, int nA, const double *cos_t, const double *sin_t, int p,
                     const double *cos_w, const double *sin_w, double R, int matrix_free,
                     airt_problem **out);

/* seismictomo geometry (testprobs/seismictomo.m:96-287): s sources at
 * (src_x, src_y), p receivers at (rcv_x, rcv_y); ray (i, j) runs from source i
 * through receiver j and is row i*p + j.  The reference's defaults put the
 * sources on the right edge and the receivers on the left and top edges. */
int airt_problem_seismic(int N, int s, const double *src_x, const double *src_y, int p,
                         const double *rcv_x, const double *rcv_y, int matrix_free,
                         airt_problem **out);

/* sphericaltomo geometry (testprobs/sphericaltomo.m:108-270): nA centre
 * angles as cosd/sind tables; nc circles of radius radius[n] (linspace(0,2,
 * nc+1)(2:end)), each sampled at the nphi[n] + 1 angles k = (0:nphi[n]) *
 * (2*pi/nphi[n]) whose cosines and sines the caller passes in cos_k / sin_k,
 * circle after circle.  Row i*nc + n holds, for every pixel the samples of
 * circle n about angle i hit w times, the value 2*pi*radius[n]/nphi[n] * w. */
int airt_problem_spherical(int N, int nA, const double *cos_t, const double *sin_t, int nc,
                           const double *radius, const int64_t *nphi, const double *cos_k,
                           const double *sin_k, int matrix_free, airt_problem **out);

int airt_problem_size(const airt_problem *h, int64_t *m, int64_t *n, int64_t *nnz);
int airt_problem_stream(const airt_problem *h, void **cuda_stream);

/* Copy the stored matrix back as MATLAB CSC (jc n+1, ir nnz, pr nnz). */
int airt_problem_export_csc(airt_problem *h, uint64_t *jc, uint64_t *ir, double *pr);

int airt_destroy(airt_problem *h);

/* ---- operator (afun) ------------------------------------------------------ */
/* y = A*x (transp=0) or y = A'*x (transp=1); host doubles. */
int airt_apply(airt_problem *h, const double *in, double *out, int transp);
int airt_apply_device(airt_problem *h, const double *d_in, double *d_out, int transp);

/* ---- weights and spectral radius ----------------------------------------- */
/* Diagonals of M (m) and D (n) of a built-in method (get_mfun_dfun.m). */
int airt_weights(airt_problem *h, int method, double *M, double *D);

/* rho = largest eigenvalue of D*A'*M*A (FP64 Lanczos iteration on
 * D^(1/2)*A'*M*A*D^(1/2) from the ones vector, stopped when the largest Ritz
 * value changes by at most the given relative tolerance; maxit bounds the
 * operator applications). */
int airt_rho(airt_problem *h, int method, const double *Mcustom, const double *Dcustom,
             double tol, int maxit, double *rho);
/* rho for a custom method whose M and/or D may be full matrices (M_full /
 * D_full as in airt_sirt_opts; a NULL M or D is the identity): the
 * dominant eigenvalue of D*A'*M*A by a power iteration on that operator
 * (the general operator of calc_relaxpar.m:91-103's eigs; the symmetric
 * Lanczos form of airt_rho needs diagonal weights), stopped when the
 * Rayleigh quotient changes by at most tol (relative) after at least five
 * steps, or after maxit steps. */
int airt_rho_custom(airt_problem *h, const double *M, int M_full, const double *D, int D_full,
                    double tol, int maxit, double *rho);

/* ---- solvers ---------------------------------------------------------------- */
/* SIRT loop.  K: nK strictly increasing 1-based iteration numbers (K(end) =
 * opts->kmax).  X: n x nK column-major output; the first info->nsaved columns
 * are written (sirt.m:246-250,270).  resnorms (optional): kmax+1 entries,
 * ||b - A x_k|| for k = 0..finaliter. */
int airt_sirt(airt_problem *h, const airt_sirt_opts *opts, const double *b, const double *x0,
              const int64_t *K, int64_t nK, double *X, double *resnorms, airt_info *info);
int airt_sirt_device(airt_problem *h, const airt_sirt_opts *opts, const double *d_b,
                     const double *d_x0, const int64_t *K, int64_t nK, double *d_X,
                     double *resnorms, airt_info *info);

/* SIRT on K right-hand sides of the same stored matrix at once (no
 * counterpart in the reference, which takes one b per sirt call): device
 * arrays d_B (m x K, column-major: right-hand side after right-hand side),
 * d_X0 (n x K starting vectors, or NULL for zeros), d_X (n x K final
 * iterates).  opts gives the built-in method, a constant or tabulated
 * relaxpar, scalar bounds and kmax; opts->stoprule AIRT_STOP_DP stops every
 * instance on its own at ||b_k - A x_k|| <= taudelta[k] (check_stoprules.m:
 * 56-72), AIRT_STOP_NONE runs kmax iterations.  The iterates are kept
 * interleaved by instance so that A is read once per iteration for all K.
 * relaxpar (host, K values) gives every instance its own relaxpar, NULL the
 * one of opts.  Ksave (nsave strictly increasing iteration numbers in
 * 1..kmax) saves every instance's iterate after those iterations into
 * d_Xsave (nsave blocks of n x K; an instance that has stopped keeps its
 * final iterate).  finaliter / stoprule: K entries. */
int airt_sirt_multi_device(airt_problem *h, const airt_sirt_opts *opts, int K, const double *d_B,
                           const double *d_X0, const double *taudelta, const double *relaxpar,
                           const int64_t *Ksave, int64_t nsave, double *d_Xsave, double *d_X,
                           int64_t *finaliter, int *stoprule, double *gpu_ms);

/* ART (Kaczmarz) sweeps, art.m:138-309.  Same K / X / info conventions. */
int airt_art(airt_problem *h, const airt_art_opts *opts, const double *b, const double *x0,
             const int64_t *K, int64_t nK, double *X, double *resnorms, airt_info *info);

/* CART column-action sweeps, cart/cart.m:139-320 (cart/columnaction.m).  Same K /
 * X / info conventions as airt_art.  The residual is updated column by column
 * as in the reference.  Each unflagging decision draws randi(nunflag) from a
 * counter-based generator keyed by (seed, sweep, column), because MATLAB's
 * randi stream cannot be reproduced. */
int airt_cart(airt_problem *h, const airt_cart_opts *opts, const double *b, const double *x0,
              const int64_t *K, int64_t nK, double *X, double *resnorms, airt_info *info);

/* Filtered back projection, auxil/fbp.m:40-79: b is the nr x na sinogram
 * (nr = rows/na); every column is circularly convolved with `kernel`
 * (order >= 2*nr - 1 entries: real(ifft) of fbp.m's zero-padded filter,
 * computed by the caller) and cropped to nr samples; x = A'*(that) *
 * pi/(2*na).  The 'none' filter is airt_apply with transp = 1. */
int airt_fbp(airt_problem *h, const double *b, int na, const double *kernel, int order, double *x);

/* ---- batches of independent problems --------------------------------------- */
/* No counterpart in the reference (one problem per sirt/art call, sirt/sirt.m:1).
 * ninst paralleltomo instances (N[k], nA[k] angles, p[k] rays); cos_t/sin_t
 * concatenate the per-instance angle tables, offsets the ray offsets.  The
 * batch is stored as one block-diagonal FP32 CSR + CSC generated on the GPU;
 * vectors are the instances' vectors concatenated in order (row_off/col_off
 * from airt_batch_layout, ninst+1 entries each). */
typedef struct airt_batch airt_batch;
int airt_batch_parallel(int ninst, const int *N, const int *nA, const int *p, const double *cos_t,
                        const double *sin_t, const double *offsets, airt_batch **out);
int airt_batch_layout(const airt_batch *h, int64_t *row_off, int64_t *col_off, int64_t *nnz);
int airt_batch_stream(const airt_batch *h, void **cuda_stream);
/* Per-instance rho of D*A_k'*M*A_k (power iteration, as airt_rho). */
int airt_batch_rho(airt_batch *h, int method, double tol, int maxit, double *rho);
/* SIRT on every instance at once: relaxpar[k], optional taudelta[k] (DP rule
 * per instance; NULL = run kmax iterations), scalar bounds; x receives the
 * final iterates, finaliter/stoprule one entry per instance. */
int airt_batch_sirt(airt_batch *h, int method, const double *relaxpar, const double *b,
                    const double *taudelta, int64_t kmax, int lb_kind, double lb, int ub_kind,
                    double ub, const double *x0, double *x, int64_t *finaliter, int *stoprule,
                    double *gpu_ms);
int airt_batch_sirt_device(airt_batch *h, int method, const double *relaxpar, const double *d_b,
                           const double *taudelta, int64_t kmax, int lb_kind, double lb, int ub_kind,
                           double ub, const double *d_x0, double *d_x, int64_t *finaliter,
                           int *stoprule, double *gpu_ms);
/* airt_batch_sirt with any stopping rule of auxil/check_stoprules.m applied
 * per instance: stoprule AIRT_STOP_NONE, DP (54-72), ME (74-94) or NCP
 * (96-151); taudelta[k] for DP and ME; NCP reshapes instance k's residual to
 * its p_k x nA_k projections and compares ncp_smooth values. */
int airt_batch_sirt_rule(airt_batch *h, int method, const double *relaxpar, const double *b,
                         int stoprule, const double *taudelta, int ncp_smooth, int64_t kmax,
                         int lb_kind, double lb, int ub_kind, double ub, const double *x0, double *x,
                         int64_t *finaliter, int *stoprule_out, double *gpu_ms);
/* Nonzeros of each instance's matrix (ninst entries). */
int airt_batch_nnz(const airt_batch *h, int64_t *nnz);
/* The batch's operator (afun of the block-diagonal system, afun_matrix.m:44-53):
 * y = A*x (transp = 0) or y = A'*x (transp = 1) on device vectors. */
int airt_batch_apply(airt_batch *h, const double *d_in, double *d_out, int transp);
/* x = D .* A'(M .* b) per instance with the weights of `method` (device
 * vectors): the first iterate of sirt (sirt/sirt.m:229) from x0 = 0
 * with relaxpar 1 and no bounds, computed with one transpose pass. */
int airt_batch_backproject(airt_batch *h, int method, const double *d_b, double *d_x, double *gpu_ms);
/* fbp of every instance at once (auxil/fbp.m:40-79): all instances have
 * projections of nr rays; d_b holds rows/nr such columns, col_scale (host,
 * one entry per column) the pi/(2*na_k) of the column's instance. */
int airt_batch_fbp(airt_batch *h, const double *d_b, int nr, const double *kernel, int order,
                   const double *col_scale, double *d_x, double *gpu_ms);
/* Kaczmarz sweeps in the kaczmarz row order, one CTA per instance, x0 = 0. */
int airt_batch_kaczmarz(airt_batch *h, const double *b, int64_t sweeps, double relaxpar,
                        int lb_kind, double lb, int ub_kind, double ub, double *x, double *gpu_ms);
int airt_batch_destroy(airt_batch *h);

/* ---- learned warm start ---------------------------------------------------- */
/* No counterpart in the reference; the network's output enters the solvers
 * only as x0 (sirt/sirt.m:5).  A U-Net of `levels` levels (two 3x3
 * conv+ReLU per level, widths base*2^l, 2x2 max-pool down, nearest 2x up with
 * skip concatenation, 1x1 head) on H x W images, BF16 activations and tensor-
 * core GEMMs with FP32 accumulation, FP32 master weights and Adam.  Images
 * are FP32 device arrays of B images in the solvers' x(:) (column-major)
 * order.  Parameters flatten per convolution (W[cout][9*cin] with K index
 * (kh*3+kw)*cin+ci, then b[cout]) followed by the head (w[base], b). */
typedef struct airt_unet airt_unet;
int airt_unet_create(int H, int W, int base, int levels, int max_batch, uint64_t seed,
                     airt_unet **out);
int airt_unet_destroy(airt_unet *h);
int airt_unet_stream(const airt_unet *h, void **cuda_stream);
int airt_unet_num_params(const airt_unet *h, int64_t *n);
int airt_unet_get_params(airt_unet *h, float *host);
int airt_unet_set_params(airt_unet *h, const float *host);
int airt_unet_get_grads(airt_unet *h, float *host);
int airt_unet_forward(airt_unet *h, const float *d_in, float *d_out, int B);
/* Inference on FP64 solver vectors: B images of d_in (x(:) order) to d_out,
 * any B (processed max_batch at a time), ordered after the work queued on
 * cuda_stream (NULL: the network's own stream) and before later work on it. */
int airt_unet_forward_f64(airt_unet *h, const double *d_in, double *d_out, int B,
                          void *cuda_stream);
/* MSE loss mean((net(in) - target)^2) and its gradient (airt_unet_get_grads). */
int airt_unet_gradients(airt_unet *h, const float *d_in, const float *d_tgt, int B, float *loss);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on the batch; returns the loss. */
int airt_unet_train_step(airt_unet *h, const float *d_in, const float *d_tgt, int B, float lr,
                         float *loss);

/* Random-ellipse phantoms (training data of the warm start): nimg images of
 * N x N, nell ellipses each given as 7 doubles (amplitude, semi-axes a and b,
 * centre x0 and y0, cos and sin of the rotation) on the grid of
 * testprobs/phantomgallery.m:188-190, summed and clipped to [lo, hi], written
 * as FP64 x(:) images to device memory. */
int airt_phantom_ellipses(int N, int nimg, int nell, const double *params, double lo, double hi,
                          double *d_out, void *cuda_stream);

/* ---- allocation-free residual ------------------------------------------------ */
/* No counterpart in the reference.  r = b - A*x and ||r|| (into d_resnorm) for
 * a caller that holds an FP32 CSR (d_rp m+1, d_ci/d_rv nnz), x, b and r on
 * the device and cannot allocate device memory: an application that owns the
 * GPU memory budget through its own pool, or code that must not call
 * cudaMalloc/cudaFree because they synchronise the device.  It allocates
 * nothing; its scratch is a static 4 MiB + 256 B device array, so n is limited
 * to 1,048,576 unknowns (AIRT_ERR_ARG beyond).  The array's address belongs
 * to a CUDA context: the first call in each context (the first call on a
 * device, and again after cudaDeviceReset or in a context the caller made
 * current) looks it up and should come before any stream capture.  Calls that
 * overlap on the GPU race on the shared scratch, so order them.  Every d_ci
 * entry must lie in [0, n) and d_rp must be nondecreasing with d_rp[m] the
 * number of entries; an index outside [0, n) is skipped and the call writes
 * NaN to d_resnorm.  Runs on cuda_stream (NULL = legacy default stream). */
int airt_residual_noalloc(int64_t m, int64_t n, const int64_t *d_rp, const int *d_ci,
                          const float *d_rv, const double *d_x, const double *d_b, double *d_r,
                          double *d_resnorm, void *cuda_stream);

/* ---- test hooks ----------------------------------------------------------- */
/* No counterpart in the reference.  For tests of the bounded device waits:
 * airt_test_set_wait_budget sets the clock64 cycle budget of each wait of the
 * Kaczmarz sweep kernel (default 4e9, about 2 s); airt_test_inject_stall(1)
 * makes the first step of every sweep wait for a completion stamp that no
 * step writes, so the wait runs out, the kernel leaves and airt_art returns
 * AIRT_ERR_TIMEOUT.  Process-wide; not for production use. */
int airt_test_set_wait_budget(long long cycles);
int airt_test_inject_stall(int on);
/* airt_test_fail_alloc(k), k >= 0: the next k device allocations of the
 * library succeed and the one after fails as an out-of-memory error
 * (AIRT_ERR_OOM, message "injected allocation failure"); k < 0 turns it off. */
int airt_test_fail_alloc(int after);
/* airt_test_split_trace: for every ray of a straight-ray geometry problem,
 * compare the entries of the whole trace with those of the two halves the
 * matrix-free kernels trace on two threads (count and an order-independent
 * hash); *mismatched = rays that differ, *split = rays that were split. */
int airt_test_split_trace(airt_problem *h, int64_t *mismatched, int64_t *split);

/* ---- instrumentation ------------------------------------------------------- */
/* When on, each SIRT kernel launch is bracketed by CUDA events on the problem
 * stream; airt_profile_read returns launches and summed device milliseconds
 * of kernel `which` (0 forward residual SpMV, 1 transpose SpMV + update). */
int airt_profile_enable(airt_problem *h, int on);
int airt_profile_read(airt_problem *h, int which, int64_t *launches, double *total_ms);

#ifdef __cplusplus
}
#endif
#endif /* AIRT_H */
