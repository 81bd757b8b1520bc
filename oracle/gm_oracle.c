/* gm_oracle.c -- CPU oracle for the closed-form matting hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).  FMA
 * contraction must stay off so orc_levin_ref32 rounds exactly like the
 * reference's host code.
 *
 * Citations are paths within the gpumatting source tree.
 */
#include "gm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* main.cu:164-190: band 12+k holds offset k-th entry of
 * {0,1,2,W-2,W-1,W,W+1,W+2,2W-2,2W-1,2W,2W+1,2W+2}; band 12-k its negation.
 * Equivalently band 12 + du + 5 dv <-> linear offset du + W dv. */
void orc_levin_offsets(int W, int offs[25])
{
    for (int dv = -2; dv <= 2; ++dv)
        for (int du = -2; du <= 2; ++du)
            offs[12 + du + 5 * dv] = du + W * dv;
}

/* Restatement of hostLevinLaplacian (Matting.cu:39-219).  Every operation
 * keeps the reference's precision: float colour sums and means, float
 * products promoted into double covariance sums (:98-120), double
 * determinant and cofactors (:130-137), whitened colour rounded to float
 * (:151-153), float pair similarity (:177), float accumulation into the band
 * store in window raster order (:180), double row sum (:192-203) and the
 * scribble rule (:205-216).  `gamma` replaces the reference's hard-coded
 * gamma = 1 (:48); `lambda` is its regulariser argument. */
void orc_levin_ref32(float* a, size_t ap, float* b, float lambda, float gamma,
                     const float* im, const unsigned char* scribs,
                     int W, int H, size_t pitch)
{
    const float winSize = 9.0f;
    const int iband = 12;
    for (int v = 1; v < H - 1; ++v) {
        for (int u = 1; u < W - 1; ++u) {
            double c11 = 0, c12 = 0, c13 = 0, c22 = 0, c23 = 0, c33 = 0;
            float mx = 0.f, my = 0.f, mz = 0.f;
            int n = 0;
            for (int v1 = v - 1; v1 <= v + 1; ++v1)
                for (int u1 = u - 1; u1 <= u + 1; ++u1) {
                    const float* t = im + 4 * ((size_t)u1 + (size_t)v1 * pitch);
                    mx += t[0]; my += t[1]; mz += t[2];
                    c11 += t[0] * t[0];
                    c12 += t[0] * t[1];
                    c13 += t[0] * t[2];
                    c22 += t[1] * t[1];
                    c23 += t[1] * t[2];
                    c33 += t[2] * t[2];
                    ++n;
                }
            mx /= n; my /= n; mz /= n;
            c11 = c11 / n - mx * mx + lambda / n;
            c12 = c12 / n - mx * my;
            c13 = c13 / n - mx * mz;
            c22 = c22 / n - my * my + lambda / n;
            c23 = c23 / n - my * mz;
            c33 = c33 / n - mz * mz + lambda / n;
            double cdet = c11 * c22 * c33 + c12 * c23 * c13 + c13 * c12 * c23
                        - c13 * c22 * c13 - c12 * c12 * c33 - c11 * c23 * c23;
            double d11 = (c33 * c22 - c23 * c23);
            double d12 = (c13 * c23 - c33 * c12);
            double d13 = (c23 * c12 - c22 * c13);
            double d22 = (c33 * c11 - c13 * c13);
            double d23 = (c12 * c13 - c23 * c11);
            double d33 = (c22 * c11 - c12 * c12);
            for (int v1 = v - 1; v1 <= v + 1; ++v1)
                for (int u1 = u - 1; u1 <= u + 1; ++u1) {
                    int i = u1 + v1 * W;
                    const float* p1 = im + 4 * ((size_t)u1 + (size_t)v1 * pitch);
                    float rx = p1[0] - mx, ry = p1[1] - my, rz = p1[2] - mz;
                    float wx = (float)((d11 * rx + d12 * ry + d13 * rz) / cdet);
                    float wy = (float)((d12 * rx + d22 * ry + d23 * rz) / cdet);
                    float wz = (float)((d13 * rx + d23 * ry + d33 * rz) / cdet);
                    for (int v2 = v - 1; v2 <= v + 1; ++v2)
                        for (int u2 = u - 1; u2 <= u + 1; ++u2) {
                            int off = (u2 - u1) + (v2 - v1) * 5;
                            const float* p2 = im + 4 * ((size_t)u2 + (size_t)v2 * pitch);
                            float sx = p2[0] - mx, sy = p2[1] - my, sz = p2[2] - mz;
                            float negSim = -(1.0f + wx * sx + wy * sy + wz * sz) / winSize;
                            a[(size_t)i + (size_t)(iband + off) * ap] += negSim;
                        }
                }
        }
    }
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            size_t i = (size_t)u + (size_t)v * W;
            double rowSum = 0;
            for (int jb = 0; jb < 25; ++jb)
                rowSum += a[i + (size_t)jb * ap];
            a[i + (size_t)iband * ap] -= rowSum;
            unsigned char s = scribs[(size_t)u + (size_t)v * pitch];
            if (s == 255) {
                a[i + (size_t)iband * ap] += gamma;
                b[i] = gamma;
            } else if (s == 0) {
                a[i + (size_t)iband * ap] += gamma;
                b[i] = 0;
            } else {
                b[i] = 0;
            }
        }
}

/* Per-window statistics in FP64: mean mu, regularised covariance
 * K = sum x x^T / 9 - mu mu^T + eps/9 I (getLevinLapRaster.m:40-41) and its
 * inverse by cofactors (Matting.cu:130-137 with the division applied). */
typedef struct { double mu[3]; double kinv[3][3]; double x[9][3]; } orc_win;

static void win_stats(orc_win* s, const double* im3, double eps, int W, int cu, int cv)
{
    double m[3] = {0, 0, 0}, c[3][3] = {{0}};
    for (int q = 0; q < 9; ++q) {
        int u = cu + (q % 3) - 1, v = cv + (q / 3) - 1;
        const double* p = im3 + 3 * ((size_t)u + (size_t)v * W);
        for (int a = 0; a < 3; ++a) {
            s->x[q][a] = p[a];
            m[a] += p[a];
            for (int b = 0; b < 3; ++b) c[a][b] += p[a] * p[b];
        }
    }
    for (int a = 0; a < 3; ++a) m[a] /= 9.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            c[a][b] = c[a][b] / 9.0 - m[a] * m[b] + (a == b ? eps / 9.0 : 0.0);
    double d00 = c[1][1] * c[2][2] - c[1][2] * c[2][1];
    double d01 = c[0][2] * c[2][1] - c[0][1] * c[2][2];
    double d02 = c[0][1] * c[1][2] - c[0][2] * c[1][1];
    double d11 = c[0][0] * c[2][2] - c[0][2] * c[2][0];
    double d12 = c[0][2] * c[1][0] - c[0][0] * c[1][2];
    double d22 = c[0][0] * c[1][1] - c[0][1] * c[1][0];
    double det = c[0][0] * d00 + c[0][1] * (c[1][2] * c[2][0] - c[1][0] * c[2][2]) + c[0][2] * (c[1][0] * c[2][1] - c[1][1] * c[2][0]);
    s->kinv[0][0] = d00 / det; s->kinv[0][1] = d01 / det; s->kinv[0][2] = d02 / det;
    s->kinv[1][0] = d01 / det; s->kinv[1][1] = d11 / det; s->kinv[1][2] = d12 / det;
    s->kinv[2][0] = d02 / det; s->kinv[2][1] = d12 / det; s->kinv[2][2] = d22 / det;
    for (int q = 0; q < 9; ++q)
        for (int a = 0; a < 3; ++a) s->x[q][a] -= m[a];
    for (int a = 0; a < 3; ++a) s->mu[a] = m[a];
}

/* Upper-band plane index (k-1) for the pair of window slots (qa, qb) with
 * linear index i_a < i_b, or -1 when i_a >= i_b. */
static int pair_plane(int qa, int qb)
{
    int du = (qb % 3) - (qa % 3), dv = (qb / 3) - (qa / 3);
    int k = du + 5 * dv;
    return k > 0 ? k - 1 : -1;
}

/* FP64 Levin affinities, gather form: for pixel i and upper neighbour j the
 * affinity sums (1 + (x_i-mu)^T K^-1 (x_j-mu)) / 9 over every interior 3x3
 * window holding both (Matting.cu:139-186; getLevinLapRaster.m:44). */
void orc_levin_sym64(double* w, const double* im3, double eps, int W, int H)
{
    size_t N = (size_t)W * H;
    memset(w, 0, sizeof(double) * 12 * N);
    /* Window rows cv and cv+3 touch disjoint pixel rows, so three phases of
     * row-parallel accumulation never write the same entry concurrently and
     * the per-entry summation order is fixed. */
    for (int phase = 0; phase < 3; ++phase) {
#pragma omp parallel for schedule(static)
        for (int cv = 1 + phase; cv < H - 1; cv += 3)
            for (int cu = 1; cu < W - 1; ++cu) {
                orc_win s;
                win_stats(&s, im3, eps, W, cu, cv);
                double white[9][3];
                for (int q = 0; q < 9; ++q)
                    for (int a = 0; a < 3; ++a)
                        white[q][a] = s.kinv[a][0] * s.x[q][0] + s.kinv[a][1] * s.x[q][1] + s.kinv[a][2] * s.x[q][2];
                for (int qa = 0; qa < 9; ++qa) {
                    size_t ia = (size_t)(cu + (qa % 3) - 1) + (size_t)(cv + (qa / 3) - 1) * W;
                    for (int qb = 0; qb < 9; ++qb) {
                        int k = pair_plane(qa, qb);
                        if (k < 0) continue;
                        double t = (1.0 + white[qa][0] * s.x[qb][0] + white[qa][1] * s.x[qb][1] + white[qa][2] * s.x[qb][2]) / 9.0;
                        w[(size_t)k * N + ia] += t;
                    }
                }
            }
    }
}

static void sym_offsets(int W, int du[13], int dv[13])
{
    for (int k = 0; k <= 12; ++k) {
        /* k = du + 5 dv with du in [-2,2], dv in [0,2] */
        int d = ((k + 2) / 5);
        dv[k] = d;
        du[k] = k - 5 * d;
    }
    (void)W;
}

void orc_sym_to_bands64(double* a, const double* w, const double* gamma, int W, int H)
{
    size_t N = (size_t)W * H;
    int du[13], dv[13];
    sym_offsets(W, du, dv);
    memset(a, 0, sizeof(double) * 25 * N);
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            size_t i = (size_t)u + (size_t)v * W;
            double diag = gamma ? gamma[i] : 0.0;
            for (int k = 1; k <= 12; ++k) {
                int uj = u + du[k], vj = v + dv[k];
                if (uj >= 0 && uj < W && vj < H) {
                    double x = w[(size_t)(k - 1) * N + i];
                    a[i + (size_t)(12 + k) * N] = -x;
                    diag += x;
                }
                int ul = u - du[k], vl = v - dv[k];
                if (ul >= 0 && ul < W && vl >= 0) {
                    size_t il = (size_t)ul + (size_t)vl * W;
                    double x = w[(size_t)(k - 1) * N + il];
                    a[i + (size_t)(12 - k) * N] = -x;
                    diag += x;
                }
            }
            a[i + 12 * N] = diag;
        }
}

void orc_apply_bands64(double* y, const double* a, const int* offs, int nb,
                       const double* x, int N)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        double s = 0;
        for (int j = 0; j < nb; ++j) {
            long c = (long)i + offs[j];
            if (c >= 0 && c < N) s += a[(size_t)i + (size_t)j * N] * x[c];
        }
        y[i] = s;
    }
}

void orc_apply_sym64(double* y, const double* w, const double* gamma,
                     const double* x, int W, int H)
{
    size_t N = (size_t)W * H;
    int du[13], dv[13];
    sym_offsets(W, du, dv);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            size_t i = (size_t)u + (size_t)v * W;
            double xi = x[i];
            double s = gamma ? gamma[i] * xi : 0.0;
            for (int k = 1; k <= 12; ++k) {
                int uj = u + du[k], vj = v + dv[k];
                if (uj >= 0 && uj < W && vj < H) {
                    size_t j = (size_t)uj + (size_t)vj * W;
                    s += w[(size_t)(k - 1) * N + i] * (xi - x[j]);
                }
                int ul = u - du[k], vl = v - dv[k];
                if (ul >= 0 && ul < W && vl >= 0) {
                    size_t j = (size_t)ul + (size_t)vl * W;
                    s += w[(size_t)(k - 1) * N + j] * (xi - x[j]);
                }
            }
            y[i] = s;
        }
}

void orc_apply(const orc_op* op, const double* x, double* y)
{
    if (op->kind == 0)
        orc_apply_sym64(y, op->w, op->gamma, x, op->W, op->H);
    else
        orc_apply_bands64(y, op->a, op->offs, op->nb, x, op->N);
}

static double dot(const double* x, const double* y, int n)
{
    double s = 0;
#pragma omp parallel for reduction(+:s) schedule(static)
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

static double true_relres(const orc_op* op, const double* b, const double* x, double* tmp, double bn)
{
    orc_apply(op, x, tmp);
    double s = 0;
    for (int i = 0; i < op->N; ++i) { double d = b[i] - tmp[i]; s += d * d; }
    return bn > 0 ? sqrt(s) / bn : sqrt(s);
}

/* cgSolve (main.cu:458-526): r = b - A x, p = r, then per iteration
 * q = A p, alpha = r.r / p.q, x += alpha p, r -= alpha q, beta = r'.r'/r.r,
 * p = r + beta p; a restart every `restart` iterations recomputes r and
 * resets p (main.cu:483-491).  The reference's sign convention (r = A x - b,
 * p = -r) gives the same iterates. */
int orc_cg64(const orc_op* op, const double* b, double* x, double rtol, int maxit,
             int restart, double* relres)
{
    int n = op->N;
    double* r = malloc(sizeof(double) * n);
    double* p = malloc(sizeof(double) * n);
    double* q = malloc(sizeof(double) * n);
    double bn = sqrt(dot(b, b, n));
    double rr = 0;
    int it = 0, inner = 0;
    for (it = 0; it < maxit; ++it) {
        if (inner == 0) {
            orc_apply(op, x, q);
            for (int i = 0; i < n; ++i) { r[i] = b[i] - q[i]; p[i] = r[i]; }
            rr = dot(r, r, n);
            inner = restart > 0 ? restart : -1;
        }
        if (rtol > 0 && sqrt(rr) <= rtol * bn) break;
        orc_apply(op, p, q);
        double pq = dot(p, q, n);
        if (!(pq > 0)) break;
        double al = rr / pq;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) { x[i] += al * p[i]; r[i] -= al * q[i]; }
        double rr2 = dot(r, r, n);
        double be = rr2 / rr;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) p[i] = r[i] + be * p[i];
        rr = rr2;
        if (inner > 0) --inner;
    }
    if (relres) *relres = true_relres(op, b, x, q, bn);
    free(r); free(p); free(q);
    return it;
}

/* gradSolve (main.cu:406-456): d = b - A x, e = A d, k = d.d / d.e (the
 * exact line search the reference writes as (<d,b> - <e,x>) / <e,d> with
 * d = A x - b), x += k d. */
int orc_gd64(const orc_op* op, const double* b, double* x, double rtol, int maxit,
             double* relres)
{
    int n = op->N;
    double* d = malloc(sizeof(double) * n);
    double* e = malloc(sizeof(double) * n);
    double bn = sqrt(dot(b, b, n));
    int it;
    for (it = 0; it < maxit; ++it) {
        orc_apply(op, x, e);
        for (int i = 0; i < n; ++i) d[i] = b[i] - e[i];
        double dd = dot(d, d, n);
        if (rtol > 0 && sqrt(dd) <= rtol * bn) break;
        orc_apply(op, d, e);
        double de = dot(d, e, n);
        if (!(de > 0)) break;
        double k = dd / de;
        for (int i = 0; i < n; ++i) x[i] += k * d[i];
    }
    if (relres) *relres = true_relres(op, b, x, e, bn);
    free(d); free(e);
    return it;
}

static void op_diag(const orc_op* op, double* dg)
{
    int n = op->N;
    if (op->kind == 1) {
        int c = -1;
        for (int j = 0; j < op->nb; ++j) if (op->offs[j] == 0) c = j;
        for (int i = 0; i < n; ++i) dg[i] = c >= 0 ? op->a[(size_t)i + (size_t)c * n] : 0.0;
        return;
    }
    /* diag = gamma + sum of affinities on row i */
    int du[13], dv[13];
    sym_offsets(op->W, du, dv);
    for (int v = 0; v < op->H; ++v)
        for (int u = 0; u < op->W; ++u) {
            size_t i = (size_t)u + (size_t)v * op->W;
            double s = op->gamma ? op->gamma[i] : 0.0;
            for (int k = 1; k <= 12; ++k) {
                int uj = u + du[k], vj = v + dv[k];
                if (uj >= 0 && uj < op->W && vj < op->H) s += op->w[(size_t)(k - 1) * n + i];
                int ul = u - du[k], vl = v - dv[k];
                if (ul >= 0 && ul < op->W && vl >= 0) s += op->w[(size_t)(k - 1) * n + (size_t)ul + (size_t)vl * op->W];
            }
            dg[i] = s;
        }
}

/* jacobi / jacobi_k (main.cu:528-556, BandedMatrix.cu:61-98): the residual
 * form x' = omega (x + (b - A x) / a_ii) + (1 - omega) x. */
int orc_jacobi64(const orc_op* op, const double* b, double* x, double omega,
                 double rtol, int maxit, double* relres)
{
    int n = op->N;
    double* q = malloc(sizeof(double) * n);
    double* dg = malloc(sizeof(double) * n);
    op_diag(op, dg);
    double bn = sqrt(dot(b, b, n));
    int it;
    for (it = 0; it < maxit; ++it) {
        orc_apply(op, x, q);
        double rr = 0;
        for (int i = 0; i < n; ++i) { double r = b[i] - q[i]; rr += r * r; q[i] = r; }
        if (rtol > 0 && sqrt(rr) <= rtol * bn) break;
        for (int i = 0; i < n; ++i) x[i] += omega * q[i] / dg[i];
    }
    if (relres) *relres = true_relres(op, b, x, q, bn);
    free(q); free(dg);
    return it;
}

/* gaussSeidel_host (Solve.cpp:3-33): in-place sweep skipping the middle
 * band, x_i = (b_i - sum_{j != mid} a_ij x_{i+off_j}) / a_i,mid. */
void orc_gs_host(float* x, const float* a, size_t ap, const int* bands, int nbands,
                 int rows, const float* b, size_t iterations)
{
    int mid = nbands / 2;
    for (; iterations > 0; --iterations)
        for (int i = 0; i < rows; ++i) {
            float t = 0.f;
            for (int j = 0; j < nbands; ++j) {
                if (j == mid) continue;
                t += a[(size_t)i + (size_t)j * ap] * x[(long)i + bands[j]];
            }
            t = b[i] - t;
            x[i] = t / a[(size_t)i + (size_t)mid * ap];
        }
}

/* jacobi_host (Solve.cpp:35-85): damped Jacobi with a ping-pong buffer.
 * The reference swaps pointers and frees the scratch buffer at exit, so an
 * odd iteration count leaves the result in a freed buffer (Solve.cpp:72-83);
 * this restatement copies the last iterate back into x instead. */
void orc_jacobi_host(float* x, const float* a, size_t ap, const int* bands, int nbands,
                     int rows, const float* b, size_t iterations, int xpad, float omega)
{
    int mid = nbands / 2;
    float omega1 = 1.f - omega;
    float* base = calloc((size_t)rows + 2 * (size_t)xpad, sizeof(float));
    float* xx = base + xpad;
    float* cur = x;
    float* nxt = xx;
    for (; iterations > 0; --iterations) {
        for (int i = 0; i < rows; ++i) {
            float t = 0.f;
            for (int j = 0; j < nbands; ++j) {
                if (j == mid) continue;
                t += a[(size_t)i + (size_t)j * ap] * cur[(long)i + bands[j]];
            }
            t = b[i] - t;
            nxt[i] = omega * t / a[(size_t)i + (size_t)mid * ap] + omega1 * cur[i];
        }
        float* sw = cur; cur = nxt; nxt = sw;
    }
    if (cur != x) memcpy(x, cur, sizeof(float) * (size_t)rows);
    free(base);
}

/* computeError (main.cu:558-577): MSE against ground truth with alpha
 * clamped to [0,1]. */
double orc_compute_error(const float* alpha, const float* gt, int W, int H)
{
    double ssd = 0.0;
    for (int i = 0; i < H; ++i)
        for (int j = 0; j < W; ++j) {
            float a = alpha[j + i * W], g = gt[j + i * W];
            if (a > 1.0f) ssd += (1.0f - g) * (1.0f - g);
            else if (a < 0.0f) ssd += g * g;
            else ssd += (a - g) * (a - g);
        }
    return ssd / ((double)W * H);
}

/* Adjoint of orc_levin_sym64.  Per window: with X the centred colours
 * (9x3), K^-1 the regularised inverse covariance and G the symmetric 9x9
 * matrix holding dloss/dT_ab / 2 for each upper pair (a,b),
 *   dX  = 2/9 G X K^-1 + 2/9 X GK,  GK = -K^-1 (X^T G X / 9) K^-1,
 *   dI  = (I - 11^T/9) dX           (centring),
 * accumulated over the 9 windows holding each pixel. */
void orc_levin_backward64(double* dim3, const double* gw, const double* im3,
                          double eps, int W, int H)
{
    size_t N = (size_t)W * H;
    for (int phase = 0; phase < 3; ++phase)
#pragma omp parallel for schedule(static)
    for (int cv = 1 + phase; cv < H - 1; cv += 3)
        for (int cu = 1; cu < W - 1; ++cu) {
            orc_win s;
            win_stats(&s, im3, eps, W, cu, cv);
            double G[9][9] = {{0}};
            size_t idx[9];
            for (int q = 0; q < 9; ++q)
                idx[q] = (size_t)(cu + (q % 3) - 1) + (size_t)(cv + (q / 3) - 1) * W;
            for (int qa = 0; qa < 9; ++qa)
                for (int qb = 0; qb < 9; ++qb) {
                    int k = pair_plane(qa, qb);
                    if (k < 0) continue;
                    double g = gw[(size_t)k * N + idx[qa]];
                    G[qa][qb] += 0.5 * g;
                    G[qb][qa] += 0.5 * g;
                }
            double GX[9][3] = {{0}};
            for (int a = 0; a < 9; ++a)
                for (int c = 0; c < 3; ++c)
                    for (int b = 0; b < 9; ++b) GX[a][c] += G[a][b] * s.x[b][c];
            double M[3][3] = {{0}};
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d)
                    for (int a = 0; a < 9; ++a) M[c][d] += s.x[a][c] * GX[a][d] / 9.0;
            double T1[3][3] = {{0}}, GK[3][3] = {{0}};
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) T1[c][d] += s.kinv[c][e] * M[e][d];
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) GK[c][d] -= T1[c][e] * s.kinv[e][d];
            double dX[9][3];
            for (int a = 0; a < 9; ++a)
                for (int c = 0; c < 3; ++c) {
                    double t = 0;
                    for (int e = 0; e < 3; ++e) t += GX[a][e] * s.kinv[e][c] + s.x[a][e] * GK[e][c];
                    dX[a][c] = 2.0 / 9.0 * t;
                }
            double mean[3] = {0, 0, 0};
            for (int a = 0; a < 9; ++a)
                for (int c = 0; c < 3; ++c) mean[c] += dX[a][c] / 9.0;
            for (int a = 0; a < 9; ++a)
                for (int c = 0; c < 3; ++c) dim3[3 * idx[a] + c] += dX[a][c] - mean[c];
        }
}
