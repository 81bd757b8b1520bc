/* gpumat.h -- C ABI of libgpumat, the B200 (sm_100a) closed-form matting
 * hot path.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the reference's names, arguments and
 *     semantics (void returns, legacy default stream, caller-owned memory):
 *     the BandedMatrix / Vector / Solve API of gpumatting.  Each cites the
 *     reference function it replaces (paths within the gpumatting tree).
 *     Errors are reported through gm_last_status() / gm_last_error().
 *
 *  2. The native gm_* API: status returns, an explicit cudaStream_t
 *     (passed as void*), solver parameters and results, the symmetric
 *     mixed-precision band store, the adjoint and batched solves.
 *
 * Memory layout conventions
 *   - A BandedMatrix holds nbands planes of `rows` floats, band j of row i at
 *     a[i + j*apitch]; bands[j] is the column offset (BandedMatrix.h:23-38).
 *     On the device, apitch is in floats (BandedMatrix.cu:39).
 *   - Reference vectors are zero-padded on both sides and the pointer points
 *     at element 0 (Vector.cu:23-30); the Levin store needs a pad of at least
 *     2W+2 (main.cu:229 uses ((2W+2)/32)*32+32).
 *   - gm_levin_store planes are row-major [H][pitch] with pitch a multiple
 *     of 8 elements >= W.
 * All device pointers must be 16-byte aligned unless stated otherwise.
 */
#ifndef GPUMAT_H
#define GPUMAT_H

#include <stddef.h>
#include <stdint.h>

/* Default arguments of the reference's C++ declarations (Vector.cu:23,37,43),
 * present when the header is compiled as C++ and absent in C. */
#ifdef __cplusplus
#define GM_DEFAULT(v) = v
#else
#define GM_DEFAULT(v)
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status                                                              */
/* ------------------------------------------------------------------ */
enum {
    GM_OK = 0,
    GM_ERR_INVALID = 1,        /* bad argument (sizes, alignment, nulls)      */
    GM_ERR_CUDA = 2,           /* a CUDA runtime call failed                  */
    GM_ERR_UNSUPPORTED = 3,    /* device is not sm_100 class, or shape unsupported */
    GM_ERR_TIMEOUT = 4,        /* a bounded wait inside a kernel gave up      */
    GM_ERR_BREAKDOWN = 5,      /* p^T A p <= 0 or a non-finite scalar         */
    GM_ERR_NOT_CONVERGED = 6,  /* max_iters reached above rtol                */
    GM_ERR_NOMEM = 7           /* device allocation failed                    */
};

int gm_last_status(void);
const char* gm_last_error(void);
const char* gm_version(void);

/* ------------------------------------------------------------------ */
/* Reference-compatible types and drop-in entry points                 */
/* ------------------------------------------------------------------ */

/* BandedMatrix.h:23-38 (same field order and types). */
typedef struct BandedMatrix_s {
    float* a;
    size_t apitch;
    int* bands;
    int nbands;
    int rows;
    int cols;
} BandedMatrix;

/* float4 of the reference's RGBA images (ppm.h:309-333). */
typedef struct gm_float4_s { float x, y, z, w; } gm_float4;

/* BandedMatrix.cu:23-41: allocate a pitched device copy of a host matrix;
 * dA->apitch is returned in floats. */
void bmCopyToDevice(BandedMatrix* dA, const BandedMatrix* hA);
/* BandedMatrix.cu:43-47 */
void bmDeviceFree(BandedMatrix* dA);
/* Vector.cu:23-30: zeroed device vector of length+lpad+rpad floats; *dx
 * points at element 0 (after the left pad). */
void vecDeviceMalloc(float** dx, int length, int leftPadding GM_DEFAULT(0), int rightPadding GM_DEFAULT(0));
/* Vector.cu:37-41 */
void vecCopyToDevice(float** dx, const float* hx, int length, int leftPadding GM_DEFAULT(0),
                     int rightPadding GM_DEFAULT(0));
/* Vector.cu:43-46 */
void vecDeviceFree(float* dx, int leftPadding GM_DEFAULT(0));

/* main.cu:57 / :458-526: `iterations` CG iterations on L alpha = b (device
 * data, alpha padded by `pad`), restarting every restartInterval. */
void cgSolve(float* alpha, BandedMatrix L, float* b, int pad, int iterations, int restartInterval);
/* main.cu:46 / :406-456: steepest descent with exact line search. */
void gradSolve(float* alpha, BandedMatrix L, float* b, int iterations, int pad);
/* main.cu:77-84 / :528-556: damped Jacobi sweeps (result left in x). */
void jacobi(float* x, const BandedMatrix a, const float* b, float omega, int pad, int iterations);

/* Matting.cu:39-219: Levin Laplacian + scribbles into the 25-band store.
 * HOST pointers, as in the reference; the work runs on the GPU with the
 * reference's arithmetic (results bit-identical) and gamma = 1.  Unlike the
 * reference's CPU loop it needs a CUDA device: it allocates device buffers
 * and copies synchronously on each call, and without a usable device it
 * sets GM_ERR_NOMEM or GM_ERR_CUDA and leaves L.a and b untouched. */
void hostLevinLaplacian(BandedMatrix L, float* b, float lambda, gm_float4* im,
                        unsigned char* scribs, int imW, int imH, size_t imPitch);

/* Solve.cpp:3-33 / Solve.h:17.  HOST matrix and vectors, any band pattern
 * (middle band = diagonal, as in the reference); x must be addressable
 * max |offset| elements either side, as the reference reads it.  Runs on the
 * GPU over a level schedule of the sequential sweep (rows whose non-zero
 * couplings to earlier rows are all to earlier levels update together), so
 * every iterate is bit-identical to the reference's sequential sweep for
 * finite data.  Needs a CUDA device; the arithmetic never runs on the host. */
void gaussSeidel_host(float* x, const BandedMatrix* A, const float* b, size_t iterations);
/* Solve.cpp:35-85 / Solve.h:31.  HOST matrix and vectors (x padded by xpad
 * >= max |offset|); the damped Jacobi iteration with the reference's FP32
 * operation order on the GPU, bit-identical iterates.  The last iterate
 * always ends in x (the reference loses it when `iterations` is odd,
 * Solve.cpp:72-83). */
void jacobi_host(float* x, const BandedMatrix* A, const float* b, size_t iterations, int xpad,
                 float omega);
/* Levels of gaussSeidel_host's schedule for a host matrix: the number of
 * dependent steps of one sweep (W + 3H - 3 or fewer for the Levin stencil
 * of a W x H image; `rows` for a pattern whose rows form one chain).  -1 on
 * bad arguments.  No counterpart in the reference. */
int gm_gs_host_levels(const BandedMatrix* A);

/* main.cu:558-577: prints "Ground truth MSE: %.3e" for HOST alpha/gt. */
void computeError(float* alpha, float* gtAlpha, int imW, int imH);

/* ------------------------------------------------------------------ */
/* Native API: kernels of the reference's L2 layer                     */
/* stream arguments are cudaStream_t passed as void* (NULL = legacy).  */
/* ------------------------------------------------------------------ */

/* b = A x (BandedMatrix.cu:107-141, :194-198); x padded so x[i+bands[j]]
 * is addressable for every row; a and b on the device. */
int gm_bm_ax(float* b, BandedMatrix a, const float* x, void* stream);
/* b = A x + y (add != 0) or A x - y (BandedMatrix.cu:152-189, :203-207). */
int gm_bm_axpy(float* b, BandedMatrix a, const float* x, const float* y, int add, void* stream);
/* xx = omega (x + (b - A x) / a_ii) + (1 - omega) x (BandedMatrix.cu:61-98);
 * the diagonal is the band with offset 0. */
int gm_jacobi_step(float* xx, const float* x, BandedMatrix a, const float* b, float omega,
                   void* stream);
/* *result = <x, y> in FP64 with a fixed summation order, rounded to float
 * (Vector.cu:195-265, without its inter-block race). result on the device. */
int gm_inner_prod(float* result, const float* x, const float* y, int len, void* stream);
/* FP64 result, written to a device double. */
int gm_inner_prod_f64(double* result, const float* x, const float* y, int len, void* stream);
/* Same result as gm_inner_prod_f64, bit for bit, with no device allocation:
 * the per-block partial sums go to a fixed 4096-double array inside the
 * library (one per device) instead of a stream-ordered buffer.  For callers
 * that must not allocate while they run (their own allocator owns device
 * memory, or a latency-critical loop cannot afford pool growth).  No
 * counterpart in the reference, whose innerProd allocates nothing but races
 * between blocks (Vector.cu:195-265).  Limits: lengths whose launch would need
 * more than 4096 partials are rejected (GM_ERR_INVALID; never on a 148-SM
 * B200, which uses at most 592); calls that overlap in time on one device
 * share the array and race, so serialise them; make the first call on each
 * device outside stream capture, since it resolves the array's address.  The
 * address is resolved again whenever the device's context changes (after a
 * cudaDeviceReset, say), so the first call after such a change must also
 * come outside stream capture. */
int gm_inner_prod_f64_noalloc(double* result, const float* x, const float* y, int len, void* stream);
/* Vector.cu:124-183 */
int gm_vec_add(float* result, const float* x, const float* y, int len, void* stream);
int gm_vec_sub(float* result, const float* x, const float* y, int len, void* stream);
int gm_vec_scale_const(float* result, const float* x, float s, int len, void* stream);
/* s is a device scalar (vecScale_k). */
int gm_vec_scale(float* result, const float* x, const float* s, int len, void* stream);

/* 25 offsets of the Levin stencil, centre at index 12 (main.cu:164-190). */
void gm_levin_band_offsets(int W, int offs[25]);
/* main.cu:229: ((2W+2)/32)*32+32. */
int gm_levin_pad(int W);

/* Clamped MSE (main.cu:558-577), FP64 accumulation; device inputs. */
int gm_compute_error(double* mse_host, const float* alpha, const float* gt, int W, int H,
                     void* stream);

/* CG building blocks over pitched row blocks (rows runs of W floats, each
 * pitch floats apart; device pointers), used by the row-slab solver that
 * splits one image over several GPUs.  No counterpart in the reference,
 * which solves one image per process.
 * gm_cg_dots4: out4 (device, 4 doubles) = FP64 sums of r.r, p.q, r.q, q.q;
 * the per-block sums are added in block order (deterministic).
 * gm_cg_update: x += alpha p; r -= alpha q; then p = r + beta p when
 * update_p is nonzero (FP32, one pass).  The four blocks must not overlap. */
int gm_cg_dots4(double* out4, const float* r, int r_pitch, const float* p, int p_pitch,
                const float* q, int q_pitch, int W, int rows, void* stream);
int gm_cg_update(float* x, int x_pitch, float* r, int r_pitch, float* p, int p_pitch,
                 const float* q, int q_pitch, int W, int rows, float alpha, float beta,
                 int update_p, void* stream);
/* The same iteration with its scalars kept on the device, so a host loop
 * need not read them back every iteration.  gm_cg_scalars (one thread)
 * turns the summed sums4 = [r.r, p.q, r.q, q.q] into coef = [alpha, beta,
 * mode] for gm_cg_update_dev (mode 0: no change, 1: x and r, 2: x, r and p)
 * and advances state (device, 6 doubles):
 *   [0] in:  threshold on the recurrence's next r.r (rtol^2 b.b; < 0 none)
 *   [1] out: r.r of this iteration      [2] out: the recurrence's next r.r
 *   [3] in/out: iterations taken
 *   [4] in/out: stop code -- 0 running; 1 the next r.r met the threshold or
 *       [3] reached [5] (x and r updated, p kept for a residual
 *       replacement); 2 breakdown (p.q <= 0 or NaN; nothing updated)
 *   [5] in:  iteration count at which to stop
 * With a nonzero stop code on entry nothing changes and mode is 0. */
int gm_cg_scalars(double* coef, double* state, const double* sums4, void* stream);
int gm_cg_update_dev(float* x, int x_pitch, float* r, int r_pitch, float* p, int p_pitch,
                     const float* q, int q_pitch, int W, int rows, const double* coef,
                     void* stream);

/* ------------------------------------------------------------------ */
/* Native API: Levin store, assembly and solvers                       */
/* ------------------------------------------------------------------ */

enum { GM_PREC_FP32 = 0, GM_PREC_FP16 = 1, GM_PREC_BF16 = 2 };
/* GM_SOLVER_PCG: CG preconditioned with the operator's diagonal (Jacobi);
 * symmetric store only (gm_levin_solve*, batches).  No counterpart in the
 * reference, whose cgSolve is unpreconditioned.
 * GM_SOLVER_MG: CG preconditioned with an aggregation multigrid V-cycle
 * (2x2 piecewise-constant aggregates, Galerkin coarse operators, one damped
 * Jacobi step before and after each coarse correction, exact solve of the
 * coarsest level of <= 128 cells); symmetric stores (gm_levin_solve,
 * gm_levin_solve_rhs, gm_levin_adjoint, gm_levin_solve_mg_many) and batches
 * (gm_batch_solve, one graph launch per image).  The outer matrix products
 * read the FP16 planes of an FP16 store when rtol >= 1e-7 (or <= 0), else the
 * FP32 planes; convergence is always judged on the FP32 operator's FP64
 * residual.  The reference
 * sketches aggregation operators over superpixels for this purpose
 * (gridoperators.h:18-138, SLIC.cpp:32, commented out at main.cu:201-218)
 * without finishing them. */
enum { GM_SOLVER_CG = 0, GM_SOLVER_GD = 1, GM_SOLVER_JACOBI = 2, GM_SOLVER_PCG = 3, GM_SOLVER_MG = 4 };
enum { GM_IMAGE_RGB8 = 0, GM_IMAGE_RGBA32F = 1 };
/* Assembly arithmetic: FP64 throughout (rounded once), or the reference's
 * float/double mix (bit-identical to hostLevinLaplacian). */
enum { GM_ASSEMBLY_FP64 = 0, GM_ASSEMBLY_REFERENCE = 1 };

typedef struct gm_image_s {
    const void* data;     /* device pointer                               */
    int format;           /* GM_IMAGE_RGB8 (3 bytes/px) or GM_IMAGE_RGBA32F */
    size_t pitch_bytes;   /* bytes between image rows                     */
} gm_image;

/* Scribbles: either a uint8 map (0 background, 255 foreground, anything
 * else unknown; Matting.cu:205-216) with one weight gamma_value, or per-pixel
 * weights gamma_map and targets s_map ([H][W] floats).  Device pointers. */
typedef struct gm_scribbles_s {
    const uint8_t* map;
    size_t map_pitch;     /* bytes between rows of map                     */
    float gamma_value;
    const float* gamma_map;
    const float* s_map;
} gm_scribbles;

/* Symmetric Levin store: 12 planes of upper affinities
 * w_k(i) = -L(i, i + du_k + W dv_k), k = du + 5 dv in 1..12.  The Laplacian
 * diagonal is not stored as a band: the true operator is
 *   y_i = gamma_i x_i + sum_j w_ij (x_i - x_j)          (rows sum to gamma)
 * and each set of planes carries the diagonal of exactly its own rounded
 * weights, d_i = gamma_i + sum_j w_ij (summed in FP64, stored in FP32), so
 * the low-precision operator y_i = d_i x_i - sum_j w_ij x_j keeps zero row
 * sums too.  All planes are [H][pitch] on the device. */
typedef struct gm_levin_store_s {
    int W, H, pitch;
    int precision;        /* element type of w                            */
    void* w;              /* [12][H][pitch] affinities in `precision`     */
    float* w32;           /* [12][H][pitch] FP32 affinities (true operator) */
    float* gamma;         /* [H][pitch] scribble weight                   */
    float* b;             /* [H][pitch] right-hand side gamma_i * s_i      */
    float* d;             /* [H][pitch] gamma + row sum of w               */
    float* d32;           /* [H][pitch] gamma + row sum of w32             */
    int owns;             /* set by gm_levin_store_alloc                  */
    size_t plane_stride;  /* elements between consecutive planes of w and
                             w32; 0 means H * pitch (a view into a larger
                             canvas, as batched stores use, sets it)       */
} gm_levin_store;

int gm_levin_store_alloc(gm_levin_store* st, int W, int H, int precision);
int gm_levin_store_free(gm_levin_store* st);

/* Assemble the symmetric store (FP64 arithmetic, rounded once) from an
 * image and scribbles (Matting.cu:79-218 math with eps and gamma as
 * parameters).  If bands25 is not NULL it also receives the reference's
 * 25-band FP32 layout: nbands=25, apitch floats, offsets gm_levin_band_offsets,
 * rows = W*H; bands25->a must be device memory of 25*apitch floats. */
int gm_levin_assemble(gm_levin_store* st, const gm_image* im, const gm_scribbles* sc,
                      double eps, BandedMatrix* bands25, float* b25, void* stream);

/* Restrict an assembled store to the unknown pixels (hard constraints): the
 * pixels `sc` marks as known (map 0/255, or gamma_map > 0 with targets s_map)
 * are fixed at their targets and eliminated.  Unknown rows keep their full
 * diagonal, their couplings to known pixels move to the right-hand side
 * (b_i += w_ij s_j) and are removed; known rows become x_i = s_i, decoupled
 * from the rest (an initial guess equal to s there keeps them exact; from any
 * other guess they converge with the solve).  Levin's trimap restriction, left commented out in the
 * reference (matlab/getLevinLap.m:20, :24, :33-35); no C counterpart. */
int gm_levin_restrict(gm_levin_store* st, const gm_scribbles* sc, void* stream);

/* Reference-layout assembly only (25 bands FP32 + b), with either
 * arithmetic.  a, b: device; a has 25 planes of apitch floats. */
int gm_levin_assemble_bands25(float* a, size_t apitch, float* b, const gm_image* im,
                              const gm_scribbles* sc, double eps, int W, int H, int arithmetic,
                              void* stream);

typedef struct gm_solve_params_s {
    int solver;           /* GM_SOLVER_*                                   */
    double rtol;          /* stop at ||b - A x|| <= rtol ||b||; <= 0: run max_iters */
    int max_iters;
    int restart;          /* CG: reset the search direction every `restart` iterations (0 = never) */
    int replace_every;    /* true-residual replacement period (0 = only at exit) */
    float omega;          /* Jacobi damping                                */
    int use_low;          /* mixed store: 1 = iterate with the low-precision planes */
    double timeout_s;     /* limit on any single wait inside the kernel     */
    int ctas_per_sm;      /* fused solver CTAs per SM: 0 = auto (as many as fit);
                             2 selects the deep-ring variant of 192-column
                             strips for FP16/BF16 stores                   */
    int strip_width;      /* fused solver strip width in columns: 0 = auto
                             (192), 192, or 128 (FP16/BF16 stores; up to 4
                             CTAs per SM)                                  */
    int inject;           /* test hook, 0 in normal use: 1 = the first grid barrier
                             waits for one arrival that never comes, so the call
                             must end with GM_ERR_TIMEOUT after timeout_s */
    float mg_omega;       /* GM_SOLVER_MG: smoother damping (0 = 0.8)      */
    float mg_scale;       /* GM_SOLVER_MG: coarse-correction scale (0 = 1.5) */
} gm_solve_params;

typedef struct gm_solve_info_s {
    int status;
    int iters;            /* Krylov (or Jacobi) sweeps applied to x        */
    int replacements;     /* true-residual sweeps run                      */
    double rel_residual;  /* ||b - A x|| / ||b|| of the returned x, FP64, true operator */
    double bnorm;
    float kernel_ms;      /* device time of the solver kernel              */
    int grid;             /* CTAs launched                                  */
    int where;            /* which bounded wait gave up, if any            */
    int solver;           /* GM_SOLVER_* that produced the result: the one
                             asked for, or GM_SOLVER_MG after gm_levin_adjoint
                             fell back to it                               */
} gm_solve_info;

void gm_default_params(gm_solve_params* p);

/* Solve (L + diag(gamma)) alpha = b with the store's operator.  alpha:
 * device [H][W] floats (pitch W), initial guess in, solution out. */
int gm_levin_solve(const gm_levin_store* st, float* alpha, const gm_solve_params* p,
                   gm_solve_info* info, void* stream);

/* y = A x with the store's operator in one streaming pass (the banded SpMV
 * of BandedMatrix.cu:107-141 on the symmetric layout).  which = 0: the
 * iteration operator of the store's precision, y_i = d_i x_i - sum_j w_ij x_j;
 * which = 1: the true operator in FP32 planes, y_i = gamma_i x_i +
 * sum_j w32_ij (x_i - x_j).  FP32 accumulation.  x: device [H][xpitch]
 * floats, 16-byte aligned, xpitch a multiple of 4; y: [H][ypitch], 8-byte
 * aligned, ypitch even. */
int gm_levin_apply(const gm_levin_store* st, const float* x, int xpitch, float* y, int ypitch, int which,
                   void* stream);

/* Solve the store's system for another right-hand side: rhs and x are
 * device [H][W] floats (pitch W); x holds the initial guess on entry. */
int gm_levin_solve_rhs(const gm_levin_store* st, const float* rhs, float* x, const gm_solve_params* p,
                       gm_solve_info* info, void* stream);

/* Adjoint of assemble + solve for a scalar loss of alpha (no counterpart in
 * the reference, which has no gradients).  Given the solved alpha and
 * dalpha = dloss/dalpha (device [H][W] floats), solves the symmetric system
 * (L + diag(gamma)) lambda = dalpha with the store's solver (lambda's input
 * contents are ignored; it receives lambda), then writes
 *   dimage: dloss/dI for the [0,1] RGB values the store was assembled from,
 *           `dimage_channels` (3, or 4 with the fourth set to 0) floats per
 *           pixel, rows dimage_pitch floats apart;
 *   dgamma: dloss/dgamma_i = lambda_i (s_i - alpha_i), [H][W], may be NULL
 *           (s_i is the scribble target, 0 on pixels without one).
 * im, sc and eps must be the ones the store was assembled with.  When the
 * lambda solve with CG, Jacobi PCG, GD or Jacobi ends GM_ERR_NOT_CONVERGED
 * (CG stalls on this right-hand side at small eps and large sizes), lambda is
 * solved again from zero with GM_SOLVER_MG and info->solver says so.  Returns
 * the final lambda solve's status (GM_ERR_NOT_CONVERGED still writes the
 * gradients). */
int gm_levin_adjoint(const gm_levin_store* st, const gm_image* im, const gm_scribbles* sc, double eps,
                     const float* alpha, const float* dalpha, float* lambda, float* dimage,
                     size_t dimage_pitch, int dimage_channels, float* dgamma, const gm_solve_params* p,
                     gm_solve_info* info, void* stream);

/* Solves `count` independent assembled stores with GM_SOLVER_MG (p->solver
 * is ignored), each with its own right-hand side st->b, alpha k in/out
 * ([H_k][W_k] device floats, initial guess in).  The solves run as one graph
 * launch each, spread over up to 8 concurrent streams forked from `stream`
 * and joined back to it, with one host synchronisation for the whole set
 * (small images do not fill the GPU alone).  All stores must have the same
 * precision.  infos: `count` results (kernel_ms is the whole set's time).
 * Returns the largest per-image status.  No counterpart in the reference,
 * which solves one image per process (main.cu:106-316); the batched solver
 * (gm_batch_solve) runs CG / PCG in one persistent launch instead. */
int gm_levin_solve_mg_many(const gm_levin_store* const* stores, float* const* alphas, int count,
                           const gm_solve_params* p, gm_solve_info* infos, void* stream);

/* Level shapes of the GM_SOLVER_MG hierarchy for a W x H image: *nlevels
 * levels, dims[2l], dims[2l+1] = width, height of level l (up to cap). */
int gm_levin_mg_levels(int W, int H, int* nlevels, int* dims, int cap);

/* Builds the GM_SOLVER_MG hierarchy of an assembled store (use_low: on the
 * low-precision planes, as the solver does) and, when r and z are given,
 * applies ONE V-cycle z = M^-1 r (device [H][W] floats).  When level >= 1 and
 * c_host / d_host are given, copies that level's 4 coupling planes (E, SW, S,
 * SE; [4][H_l][W_l]) and diagonal ([H_l][W_l]) to host memory.  For tests and
 * diagnostics of the preconditioner (the aggregation operators of
 * gridoperators.h:18-138, here on 2x2 blocks). */
int gm_levin_mg_inspect(const gm_levin_store* st, int use_low, const float* r, float* z, int level,
                        float* c_host, float* d_host, void* stream);

/* ------------------------------------------------------------------ */
/* Data formats either side of the solve                               */
/* ------------------------------------------------------------------ */

/* A PNM image as read from a file: host bytes, w*h*channels, row-major. */
typedef struct gm_pnm_s {
    int w, h;
    int channels;         /* 1 (P5/P2 graymap) or 3 (P6/P3 pixmap)        */
    int maxval;
    unsigned char* data;  /* host memory owned by the struct: gm_pnm_free */
} gm_pnm;

/* ppm.h:32-127 pgmread and :178-278 ppmread: binary or ASCII, header lines
 * as the reference reads them; pixmaps with maxval outside 0..255 are
 * rejected as the reference rejects them.  Host only. */
int gm_pnm_read(const char* path, gm_pnm* img);
void gm_pnm_free(gm_pnm* img);
/* ppm.h:345-414 pgmwrite: "P5"/"P2", optional "# comment", maxval 255; the
 * same bytes as the reference writes.  data: host w*h bytes. */
int gm_pgm_write(const char* path, int w, int h, const unsigned char* data, const char* comment, int binary);
/* ppm.h:309-333 ppmread_float4's normalisation on the device: RGB bytes to
 * (r, g, b, 1) / maxval.  dst 16-byte aligned. */
int gm_rgb8_to_float4(gm_float4* dst, const unsigned char* src, int n, int maxval, void* stream);
/* ppm.h:430-451 pgmwrite_float's quantisation on the device: 0 below 0, 255
 * above 1, else (unsigned char)(255 * alpha). */
int gm_alpha_to_gray8(unsigned char* dst, const float* alpha, int n, void* stream);
/* main.cu:334-355 dump: the A.bin file, nbands x rows floats, band-major.
 * on_device: L.a is device memory (copied band by band). */
int gm_bands_dump(const char* path, BandedMatrix L, int on_device);

/* ------------------------------------------------------------------ */
/* Batched solves: many images of different sizes in one persistent   */
/* launch (no counterpart in the reference, which solves one image).   */
/* ------------------------------------------------------------------ */
typedef struct gm_batch_s gm_batch;

/* Allocates one canvas store + work vectors for `count` images of the given
 * sizes (stacked, 2 zero rows apart) in `precision`; everything zeroed. */
int gm_batch_create(gm_batch** b, int count, const int* widths, const int* heights, int precision);
int gm_batch_destroy(gm_batch* b);
/* View of image k's planes inside the canvas (plane_stride set; owns = 0):
 * usable with gm_levin_assemble, gm_levin_apply, gm_levin_solve. */
int gm_batch_store(const gm_batch* b, int k, gm_levin_store* view);
/* gm_levin_assemble into image k's view. */
int gm_batch_assemble(gm_batch* b, int k, const gm_image* im, const gm_scribbles* sc, double eps,
                      void* stream);
/* Times the candidate launch shapes (ring configuration x CTAs per SM x
 * rows per unit) for `iters` fixed iterations each and keeps the fastest. */
int gm_batch_tune(gm_batch* b, const gm_solve_params* p, int iters, void* stream);
/* Solves every image in one cooperative launch, replayed from a CUDA graph
 * captured on first use (recaptured when the parameters or the shape
 * change).  alphas: host array of `count` device pointers ([H_k][W_k],
 * initial guess in, solution out); infos: `count` results (kernel_ms and
 * grid are those of the one launch).  p->ctas_per_sm = 0 uses the tuned
 * shape (tuning on first use).  Returns the worst per-image status.
 * GM_SOLVER_MG runs gm_levin_solve_mg_many over the images' store views
 * instead (one graph launch per image on concurrent streams; kernel_ms is
 * the whole set's time). */
int gm_batch_solve(gm_batch* b, float* const* alphas, const gm_solve_params* p, gm_solve_info* infos,
                   void* stream);
/* Tuned shape (0 / -1 before tuning), graph launches so far, last grid. */
int gm_batch_info(const gm_batch* b, int* tuned_ctas_per_sm, int* tuned_ring_cfg, int* tuned_row_mult,
                  int* graph_launches, int* grid);

/* Solve with a 25-band BandedMatrix on the device (reference layout).
 * W > 0 declares the Levin stencil of an image W wide (rows = W*H) and
 * selects the fused stencil kernel; W = 0 (or offsets that are not the Levin
 * pattern) uses the generic band path.  alpha padded as in the reference
 * (pad >= max |offset|), b unpadded, both device. */
int gm_banded_solve(BandedMatrix L, int W, float* alpha, int pad, const float* b,
                    const gm_solve_params* p, gm_solve_info* info, void* stream);

#ifdef __cplusplus
}

/* Solve.h:17 and :31 take the matrix by const reference and default
 * `iterations` and `omega`; these overloads let the reference's C++ callers
 * (main.cu:264, :267) compile unchanged against this header.  They forward
 * to the C entry points above. */
inline void gaussSeidel_host(float* x, const BandedMatrix& A, const float* b, size_t iterations = 1)
{
    gaussSeidel_host(x, &A, b, iterations);
}
inline void jacobi_host(float* x, const BandedMatrix& A, const float* b, size_t iterations, int xpad,
                        float omega = 2.f / 3.f)
{
    jacobi_host(x, &A, b, iterations, xpad, omega);
}
#if defined(__VECTOR_TYPES_H__)
/* Matting.cu:39 takes CUDA's float4 (same layout as gm_float4); available
 * when the caller has included the CUDA runtime headers first. */
inline void hostLevinLaplacian(BandedMatrix L, float* b, float lambda, float4* im, unsigned char* scribs, int imW,
                               int imH, size_t imPitch)
{
    hostLevinLaplacian(L, b, lambda, reinterpret_cast<gm_float4*>(im), scribs, imW, imH, imPitch);
}
#endif
#endif
#endif /* GPUMAT_H */
