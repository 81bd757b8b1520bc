/* test_native.c -- the native Levin-store API from plain C: RGB8 image and
 * scribble map on the device, gm_levin_store_alloc (FP16 planes),
 * gm_levin_assemble, gm_levin_solve with the fused CG, the Jacobi-PCG and the
 * multigrid PCG, gm_levin_solve_mg_many over two stores, a two-image
 * gm_batch solve and gm_levin_adjoint.  Every solution is checked on the host
 * against the store's own FP32 planes (FP64 residual of the true operator
 * y_i = gamma_i x_i + sum_j w_ij (x_i - x_j)).  Prints "Test PASSED" and
 * exits 0 when every check holds. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "gpumat.h"

#define RTOL 1e-6

static int fail(const char* what)
{
    printf("%s failed: status %d (%s)\nTest FAILED\n", what, gm_last_status(), gm_last_error());
    return 1;
}

/* One synthetic problem: a soft edge between two colours with a little
 * deterministic noise, background strokes on the left, foreground strokes on
 * the right. */
typedef struct {
    int W, H;
    unsigned char* d_rgb;
    unsigned char* d_map;
    gm_image im;
    gm_scribbles sc;
} problem;

static int make_problem(problem* pb, int W, int H, int seed)
{
    const int N = W * H;
    unsigned char* rgb = (unsigned char*)malloc((size_t)3 * N);
    unsigned char* map = (unsigned char*)malloc((size_t)N);
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            const int i = u + v * W;
            const double a = 1.0 / (1.0 + exp(-(u - W / 2 + 5.0 * sin(v * 0.17 + seed)) / 2.0));
            const double fg[3] = {230, 60, 30}, bg[3] = {25, 80, 200};
            for (int c = 0; c < 3; ++c) {
                const int n = (int)((i * 7919u + c * 104729u + seed * 31u) % 9u) - 4;
                double val = a * fg[c] + (1 - a) * bg[c] + n;
                rgb[3 * i + c] = (unsigned char)(val < 0 ? 0 : val > 255 ? 255 : val + 0.5);
            }
            map[i] = 128;
            if (u >= W - 6 && u < W - 2 && (v % 3) != 0) map[i] = 255;
            if (u >= 2 && u < 6 && (v % 3) != 1) map[i] = 0;
        }
    pb->W = W;
    pb->H = H;
    if (cudaMalloc((void**)&pb->d_rgb, (size_t)3 * N) != cudaSuccess) return 1;
    if (cudaMalloc((void**)&pb->d_map, (size_t)N) != cudaSuccess) return 1;
    cudaMemcpy(pb->d_rgb, rgb, (size_t)3 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(pb->d_map, map, (size_t)N, cudaMemcpyHostToDevice);
    free(rgb);
    free(map);
    pb->im.data = pb->d_rgb;
    pb->im.format = GM_IMAGE_RGB8;
    pb->im.pitch_bytes = (size_t)3 * W;
    memset(&pb->sc, 0, sizeof(pb->sc));
    pb->sc.map = pb->d_map;
    pb->sc.map_pitch = (size_t)W;
    pb->sc.gamma_value = 100.0f;
    return 0;
}

static void free_problem(problem* pb)
{
    cudaFree(pb->d_rgb);
    cudaFree(pb->d_map);
}

/* Host copy of a store's FP32 planes: w32 [12][H][W], gamma, b. */
typedef struct {
    int W, H;
    float *w, *gamma, *b;
} host_store;

static void fetch(host_store* hs, const gm_levin_store* st)
{
    const int W = st->W, H = st->H;
    const size_t stride = st->plane_stride ? st->plane_stride : (size_t)H * st->pitch;
    hs->W = W;
    hs->H = H;
    hs->w = (float*)malloc(sizeof(float) * 12 * W * H);
    hs->gamma = (float*)malloc(sizeof(float) * W * H);
    hs->b = (float*)malloc(sizeof(float) * W * H);
    for (int k = 0; k < 12; ++k)
        cudaMemcpy2D(hs->w + (size_t)k * W * H, sizeof(float) * W, st->w32 + k * stride,
                     sizeof(float) * st->pitch, sizeof(float) * W, H, cudaMemcpyDeviceToHost);
    cudaMemcpy2D(hs->gamma, sizeof(float) * W, st->gamma, sizeof(float) * st->pitch, sizeof(float) * W, H,
                 cudaMemcpyDeviceToHost);
    cudaMemcpy2D(hs->b, sizeof(float) * W, st->b, sizeof(float) * st->pitch, sizeof(float) * W, H,
                 cudaMemcpyDeviceToHost);
}

static void release(host_store* hs)
{
    free(hs->w);
    free(hs->gamma);
    free(hs->b);
}

/* ||b - A x|| / ||b||, FP64, A the true operator of the FP32 planes; plane
 * k = du + 5 dv couples (u, v) with (u + du, v + dv). */
static double relres(const host_store* hs, const float* x)
{
    const int W = hs->W, H = hs->H, N = W * H;
    double* y = (double*)calloc((size_t)N, sizeof(double));
    for (int i = 0; i < N; ++i) y[i] = (double)hs->gamma[i] * x[i];
    for (int k = 1; k <= 12; ++k) {
        const int du = ((k + 2) % 5) - 2, dv = (k + 2) / 5;
        for (int v = 0; v < H; ++v)
            for (int u = 0; u < W; ++u) {
                const int uj = u + du, vj = v + dv;
                if (uj < 0 || uj >= W || vj >= H) continue;
                const int i = u + v * W, j = uj + vj * W;
                const double w = hs->w[(size_t)(k - 1) * N + i];
                y[i] += w * ((double)x[i] - x[j]);
                y[j] += w * ((double)x[j] - x[i]);
            }
    }
    double rr = 0.0, bb = 0.0;
    for (int i = 0; i < N; ++i) {
        rr += (hs->b[i] - y[i]) * (hs->b[i] - y[i]);
        bb += (double)hs->b[i] * hs->b[i];
    }
    free(y);
    return sqrt(rr / bb);
}

static float* device_half(int n)
{
    float* h = (float*)malloc(sizeof(float) * n);
    for (int i = 0; i < n; ++i) h[i] = 0.5f;
    float* d = NULL;
    if (cudaMalloc((void**)&d, sizeof(float) * n) != cudaSuccess) d = NULL;
    else cudaMemcpy(d, h, sizeof(float) * n, cudaMemcpyHostToDevice);
    free(h);
    return d;
}

static int check_solution(const char* what, const host_store* hs, const float* d_alpha, const gm_solve_info* info,
                          float* out)
{
    const int N = hs->W * hs->H;
    cudaMemcpy(out, d_alpha, sizeof(float) * N, cudaMemcpyDeviceToHost);
    const double rel = relres(hs, out);
    int finite = 1;
    for (int i = 0; i < N; ++i) finite &= isfinite(out[i]) != 0;
    printf("%s: status %d, %d iters, reported rel-res %.3e, host FP64 rel-res %.3e\n", what, info->status,
           info->iters, info->rel_residual, rel);
    if (info->status != GM_OK || !finite || !(info->rel_residual <= RTOL) || !(rel <= 2 * RTOL)) {
        printf("%s: not solved\nTest FAILED\n", what);
        return 1;
    }
    return 0;
}

int main(void)
{
    problem p0, p1;
    if (make_problem(&p0, 96, 64, 0) || make_problem(&p1, 70, 41, 1)) return fail("cudaMalloc");
    const int N0 = p0.W * p0.H, N1 = p1.W * p1.H;
    const double eps = 1e-5;

    gm_levin_store s0, s1;
    if (gm_levin_store_alloc(&s0, p0.W, p0.H, GM_PREC_FP16) != GM_OK) return fail("gm_levin_store_alloc");
    if (gm_levin_store_alloc(&s1, p1.W, p1.H, GM_PREC_FP16) != GM_OK) return fail("gm_levin_store_alloc");
    if (gm_levin_assemble(&s0, &p0.im, &p0.sc, eps, NULL, NULL, NULL) != GM_OK) return fail("gm_levin_assemble");
    if (gm_levin_assemble(&s1, &p1.im, &p1.sc, eps, NULL, NULL, NULL) != GM_OK) return fail("gm_levin_assemble");
    cudaDeviceSynchronize();
    host_store h0, h1;
    fetch(&h0, &s0);
    fetch(&h1, &s1);

    float* out = (float*)malloc(sizeof(float) * N0);
    float* mg0 = (float*)malloc(sizeof(float) * N0);

    /* single solves with the three Krylov solvers */
    const int solvers[3] = {GM_SOLVER_CG, GM_SOLVER_PCG, GM_SOLVER_MG};
    const char* names[3] = {"CG", "PCG", "MG"};
    int iters[3];
    for (int s = 0; s < 3; ++s) {
        float* d_alpha = device_half(N0);
        gm_solve_params prm;
        gm_default_params(&prm);
        prm.solver = solvers[s];
        prm.rtol = RTOL;
        prm.max_iters = 5000;
        gm_solve_info info;
        if (gm_levin_solve(&s0, d_alpha, &prm, &info, NULL) != GM_OK) return fail(names[s]);
        if (check_solution(names[s], &h0, d_alpha, &info, out)) return 1;
        iters[s] = info.iters;
        if (s == 2) memcpy(mg0, out, sizeof(float) * N0);
        cudaFree(d_alpha);
    }
    if (!(iters[2] < iters[1] && iters[1] < iters[0])) {
        printf("iteration counts not ordered MG < PCG < CG\nTest FAILED\n");
        return 1;
    }

    /* two stores through gm_levin_solve_mg_many: store 0 matches its single
     * MG solve bit for bit */
    {
        float* a0 = device_half(N0);
        float* a1 = device_half(N1);
        const gm_levin_store* stores[2] = {&s0, &s1};
        float* alphas[2] = {a0, a1};
        gm_solve_params prm;
        gm_default_params(&prm);
        prm.rtol = RTOL;
        prm.max_iters = 500;
        gm_solve_info infos[2];
        if (gm_levin_solve_mg_many(stores, alphas, 2, &prm, infos, NULL) != GM_OK) return fail("gm_levin_solve_mg_many");
        if (check_solution("mg_many[0]", &h0, a0, &infos[0], out)) return 1;
        if (memcmp(out, mg0, sizeof(float) * N0) != 0) {
            printf("mg_many[0] differs from the single MG solve\nTest FAILED\n");
            return 1;
        }
        if (check_solution("mg_many[1]", &h1, a1, &infos[1], out)) return 1;
        cudaFree(a0);
        cudaFree(a1);
    }

    /* both images in one batched persistent launch */
    {
        gm_batch* bt = NULL;
        const int ws[2] = {p0.W, p1.W}, hs[2] = {p0.H, p1.H};
        if (gm_batch_create(&bt, 2, ws, hs, GM_PREC_FP16) != GM_OK) return fail("gm_batch_create");
        if (gm_batch_assemble(bt, 0, &p0.im, &p0.sc, eps, NULL) != GM_OK) return fail("gm_batch_assemble");
        if (gm_batch_assemble(bt, 1, &p1.im, &p1.sc, eps, NULL) != GM_OK) return fail("gm_batch_assemble");
        float* a0 = device_half(N0);
        float* a1 = device_half(N1);
        float* alphas[2] = {a0, a1};
        gm_solve_params prm;
        gm_default_params(&prm);
        prm.solver = GM_SOLVER_CG;
        prm.rtol = RTOL;
        prm.max_iters = 5000;
        prm.ctas_per_sm = 3;
        gm_solve_info infos[2];
        if (gm_batch_solve(bt, alphas, &prm, infos, NULL) != GM_OK) return fail("gm_batch_solve");
        /* the views' planes are the canvas's: check against them */
        gm_levin_store v0, v1;
        gm_batch_store(bt, 0, &v0);
        gm_batch_store(bt, 1, &v1);
        host_store b0, b1;
        fetch(&b0, &v0);
        fetch(&b1, &v1);
        if (check_solution("batch[0]", &b0, a0, &infos[0], out)) return 1;
        if (check_solution("batch[1]", &b1, a1, &infos[1], out)) return 1;
        release(&b0);
        release(&b1);
        cudaFree(a0);
        cudaFree(a1);
        gm_batch_destroy(bt);
    }

    /* adjoint of assemble + MG solve for loss = sum(alpha): finite image
     * gradients, dgamma_i = lambda_i (s_i - alpha_i) */
    {
        float* d_alpha = NULL;
        float *d_dalpha = NULL, *d_lambda = NULL, *d_dimg = NULL, *d_dgam = NULL;
        cudaMalloc((void**)&d_alpha, sizeof(float) * N0);
        cudaMemcpy(d_alpha, mg0, sizeof(float) * N0, cudaMemcpyHostToDevice);
        d_dalpha = device_half(N0);
        cudaMalloc((void**)&d_lambda, sizeof(float) * N0);
        cudaMalloc((void**)&d_dimg, sizeof(float) * 3 * N0);
        cudaMalloc((void**)&d_dgam, sizeof(float) * N0);
        gm_solve_params prm;
        gm_default_params(&prm);
        prm.solver = GM_SOLVER_MG;
        prm.rtol = RTOL;
        prm.max_iters = 500;
        gm_solve_info info;
        if (gm_levin_adjoint(&s0, &p0.im, &p0.sc, eps, d_alpha, d_dalpha, d_lambda, d_dimg, (size_t)3 * p0.W, 3,
                             d_dgam, &prm, &info, NULL) != GM_OK)
            return fail("gm_levin_adjoint");
        float* dimg = (float*)malloc(sizeof(float) * 3 * N0);
        float* lam = (float*)malloc(sizeof(float) * N0);
        float* dgam = (float*)malloc(sizeof(float) * N0);
        cudaMemcpy(dimg, d_dimg, sizeof(float) * 3 * N0, cudaMemcpyDeviceToHost);
        cudaMemcpy(lam, d_lambda, sizeof(float) * N0, cudaMemcpyDeviceToHost);
        cudaMemcpy(dgam, d_dgam, sizeof(float) * N0, cudaMemcpyDeviceToHost);
        unsigned char* map = (unsigned char*)malloc((size_t)N0);
        cudaMemcpy(map, p0.d_map, (size_t)N0, cudaMemcpyDeviceToHost);
        int ok = 1;
        double gnorm = 0.0, derr = 0.0;
        for (int i = 0; i < 3 * N0; ++i) {
            ok &= isfinite(dimg[i]) != 0;
            gnorm += fabs(dimg[i]);
        }
        for (int i = 0; i < N0; ++i) {
            const double s = map[i] == 255 ? 1.0 : 0.0;
            const double want = (double)lam[i] * (s - mg0[i]);
            derr = fmax(derr, fabs(dgam[i] - want) / (1e-6 + fabs(want)));
        }
        printf("adjoint: lambda solve %d iters, sum |dimage| %.3e, max rel dgamma error %.2e\n", info.iters, gnorm,
               derr);
        if (!ok || !(gnorm > 0.0) || !(derr < 1e-4)) {
            printf("adjoint gradients wrong\nTest FAILED\n");
            return 1;
        }
        free(dimg);
        free(lam);
        free(dgam);
        free(map);
        cudaFree(d_alpha);
        cudaFree(d_dalpha);
        cudaFree(d_lambda);
        cudaFree(d_dimg);
        cudaFree(d_dgam);
    }

    release(&h0);
    release(&h1);
    free(out);
    free(mg0);
    gm_levin_store_free(&s0);
    gm_levin_store_free(&s1);
    free_problem(&p0);
    free_problem(&p1);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail("cudaDeviceSynchronize");
    printf("Test PASSED\n");
    return 0;
}
