/* gm_oracle.h -- CPU oracle for the closed-form matting hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product library (libgpumat.so) never links
 * or calls it.
 *
 * Contents (each function cites the reference code it restates; paths are
 * relative to the gpumatting source tree):
 *   - orc_levin_ref32:   FP32-faithful restatement of hostLevinLaplacian
 *                        (Matting.cu:39-219), bit-exact with the reference
 *                        when both are compiled without FMA contraction.
 *   - orc_levin_sym64:   the same Laplacian computed entirely in FP64
 *                        (Matting.cu:79-189, matlab/getLevinLapRaster.m:22-62),
 *                        returned as the 12 unique upper off-diagonal
 *                        affinities w_k(i) = -L(i, i+off_k).
 *   - orc_apply_*:       operators y = A x for the 25-band store and for the
 *                        symmetric store (implicit Laplacian diagonal).
 *   - orc_cg64 / orc_gd64 / orc_jacobi64: FP64 solvers (main.cu:406-556
 *                        semantics), OpenMP-parallel.
 *   - orc_gs_host / orc_jacobi_host: restatement of Solve.cpp:3-85 (FP32,
 *                        single thread), the reference's CPU solve path.
 *   - orc_compute_error: main.cu:558-577.
 *   - orc_levin_backward64: FP64 adjoint of the Laplacian assembly.
 */
#ifndef GM_ORACLE_H
#define GM_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Band offsets of the 25-band Levin store: band 12+du+5*dv <-> du + W*dv
 * (main.cu:164-190). */
void orc_levin_offsets(int W, int offs[25]);

void orc_levin_ref32(float* a, size_t apitch, float* b, float lambda, float gamma,
                     const float* im4, const unsigned char* scribs,
                     int W, int H, size_t imPitch);

/* w: 12 planes of N doubles, plane k-1 holds w_k(i) = -L(i, i+off_k),
 * k = 1..12 (upper half, offsets 1, 2, W-2, W-1, W, W+1, W+2, 2W-2 .. 2W+2).
 * im3: N*3 doubles (RGB in [0,1], row-major, pitch W). */
void orc_levin_sym64(double* w, const double* im3, double eps, int W, int H);

/* Expand the symmetric store to the 25-band layout (double), diagonal =
 * sum of affinities + gamma_i. */
void orc_sym_to_bands64(double* a, const double* w, const double* gamma, int W, int H);

/* y = A x, 25 (or nb) linear bands, a[i + j*N], x unpadded: out-of-range
 * columns contribute nothing. */
void orc_apply_bands64(double* y, const double* a, const int* offs, int nb,
                       const double* x, int N);
/* y = diag(gamma) x + L x with L given by the symmetric store. */
void orc_apply_sym64(double* y, const double* w, const double* gamma,
                     const double* x, int W, int H);

typedef struct {
    int kind;             /* 0 = symmetric store, 1 = bands */
    int W, H, N;
    const double* w;      /* kind 0 */
    const double* gamma;  /* kind 0 */
    const double* a;      /* kind 1 */
    const int* offs;      /* kind 1 */
    int nb;               /* kind 1 */
} orc_op;

void orc_apply(const orc_op* op, const double* x, double* y);

/* CG on A x = b (standard Hestenes-Stiefel, main.cu:458-526 semantics).
 * restart > 0 recomputes r = b - A x and resets p every `restart`
 * iterations; rtol <= 0 runs exactly maxit iterations.  Returns the number
 * of iterations run; *relres is ||b - A x|| / ||b|| at exit. */
int orc_cg64(const orc_op* op, const double* b, double* x, double rtol, int maxit,
             int restart, double* relres);
/* Steepest descent with exact line search (main.cu:406-456). */
int orc_gd64(const orc_op* op, const double* b, double* x, double rtol, int maxit,
             double* relres);
/* Damped Jacobi x <- x + omega (b - A x) / diag(A) (BandedMatrix.cu:61-98). */
int orc_jacobi64(const orc_op* op, const double* b, double* x, double omega,
                 double rtol, int maxit, double* relres);

/* Solve.cpp restatements; x is padded by xpad zero floats on both sides. */
void orc_gs_host(float* x, const float* a, size_t apitch, const int* bands, int nbands,
                 int rows, const float* b, size_t iterations);
void orc_jacobi_host(float* x, const float* a, size_t apitch, const int* bands, int nbands,
                     int rows, const float* b, size_t iterations, int xpad, float omega);

double orc_compute_error(const float* alpha, const float* gt, int W, int H);

/* Adjoint of the assembly.  Given the upstream gradient of the loss with
 * respect to every affinity, gw[k-1][i] = dloss/dw_k(i) (12 planes), returns
 * dloss/dim3 (N*3, accumulated into dim3). */
void orc_levin_backward64(double* dim3, const double* gw, const double* im3,
                          double eps, int W, int H);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
