/* test_dropin.c -- the reference's own call sequence (main.cu:160-290) in
 * plain C against libgpumat: a host BandedMatrix filled by
 * hostLevinLaplacian, bmCopyToDevice, vecCopyToDevice, cgSolve / gradSolve,
 * copy back, computeError, then the frees.  Prints "Test PASSED" and exits 0
 * when cgSolve solves the system, gradSolve reduces its residual, and both
 * mattes hold the scribbled values (the reference's own test convention,
 * tests/BandedMatrixTest.cu). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "gpumat.h"

#define W 96
#define H 64
#define N (W * H)

static int fail(const char* what)
{
    printf("%s failed: status %d (%s)\nTest FAILED\n", what, gm_last_status(), gm_last_error());
    return 1;
}

/* ||b - A x|| / ||b|| on the host with the 25 reference bands */
static double relres(const BandedMatrix* L, const float* b, const float* x)
{
    double rr = 0.0, bb = 0.0;
    for (int i = 0; i < N; ++i) {
        double y = 0.0;
        for (int j = 0; j < L->nbands; ++j) {
            const int k = i + L->bands[j];
            if (k >= 0 && k < N) y += (double)L->a[i + (size_t)j * L->apitch] * x[k];
        }
        rr += (b[i] - y) * (b[i] - y);
        bb += (double)b[i] * b[i];
    }
    return sqrt(rr / bb);
}

int main(void)
{
    gm_float4* im = (gm_float4*)malloc(sizeof(gm_float4) * N);
    unsigned char* scribs = (unsigned char*)malloc(N);
    float* gt = (float*)malloc(sizeof(float) * N);
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            const int i = u + v * W;
            /* soft vertical edge between a red foreground and a blue background */
            const float a = 1.0f / (1.0f + expf(-(float)(u - W / 2 + 6.0 * sin(v * 0.2)) / 2.5f));
            const float fg[3] = {0.9f, 0.2f, 0.1f}, bg[3] = {0.1f, 0.3f, 0.8f};
            const float n = 0.01f * (float)((i * 7919) % 13 - 6);
            im[i].x = a * fg[0] + (1 - a) * bg[0] + n;
            im[i].y = a * fg[1] + (1 - a) * bg[1] - n;
            im[i].z = a * fg[2] + (1 - a) * bg[2] + n;
            im[i].w = 1.0f;
            gt[i] = a;
            scribs[i] = 128;
            if (u > W - 8 && u < W - 3) scribs[i] = 255;  /* foreground strokes */
            if (u > 2 && u < 7) scribs[i] = 0;            /* background strokes */
        }

    /* main.cu:164-194: 25 bands, centre 12, offset du + W dv */
    BandedMatrix L;
    L.nbands = 25;
    L.rows = L.cols = N;
    L.apitch = N;
    L.bands = (int*)malloc(sizeof(int) * 25);
    for (int dv = -2; dv <= 2; ++dv)
        for (int du = -2; du <= 2; ++du) L.bands[12 + du + 5 * dv] = du + W * dv;
    L.a = (float*)calloc((size_t)25 * N, sizeof(float));
    float* b = (float*)calloc(N, sizeof(float));
    float* alpha = (float*)malloc(sizeof(float) * N);

    hostLevinLaplacian(L, b, 1e-2f, im, scribs, W, H, W);
    if (gm_last_status() != GM_OK) return fail("hostLevinLaplacian");

    const int pad = ((2 * W + 2) / 32) * 32 + 32;  /* main.cu:229 */
    BandedMatrix dL;
    bmCopyToDevice(&dL, &L);
    if (gm_last_status() != GM_OK) return fail("bmCopyToDevice");
    float* dB = NULL;
    if (cudaMalloc((void**)&dB, sizeof(float) * N) != cudaSuccess) return fail("cudaMalloc");
    cudaMemcpy(dB, b, sizeof(float) * N, cudaMemcpyHostToDevice);

    const char* names[2] = {"cgSolve", "gradSolve"};
    for (int which = 0; which < 2; ++which) {
        for (int i = 0; i < N; ++i) alpha[i] = 0.5f;  /* main.cu:198-199 */
        float* dAlpha = NULL;
        vecCopyToDevice(&dAlpha, alpha, N, pad, pad);
        if (gm_last_status() != GM_OK) return fail("vecCopyToDevice");
        if (which == 0) cgSolve(dAlpha, dL, dB, pad, 3000, 101);
        else gradSolve(dAlpha, dL, dB, 200, pad);
        if (gm_last_status() != GM_OK) return fail(names[which]);
        cudaMemcpy(alpha, dAlpha, sizeof(float) * N, cudaMemcpyDeviceToHost);
        vecDeviceFree(dAlpha, pad);

        const double rel = relres(&L, b, alpha);
        /* the strokes hold their values: mean alpha on the foreground and
         * background strokes */
        double fgm = 0.0, bgm = 0.0;
        int nf = 0, nb = 0, finite = 1;
        for (int i = 0; i < N; ++i) {
            finite &= isfinite(alpha[i]) != 0;
            if (scribs[i] == 255) { fgm += alpha[i]; ++nf; }
            if (scribs[i] == 0) { bgm += alpha[i]; ++nb; }
        }
        fgm /= nf;
        bgm /= nb;
        printf("%s: rel-res %.3e, mean alpha on strokes fg %.3f bg %.3f\n", names[which], rel, fgm, bgm);
        computeError(alpha, gt, W, H); /* prints the MSE, as main.cu:303 */
        if (!finite) { printf("%s: non-finite alpha\nTest FAILED\n", names[which]); return 1; }
        if (which == 0 && !(rel < 1e-3)) { printf("cgSolve did not solve the system\nTest FAILED\n"); return 1; }
        if (which == 1 && !(rel < 0.5)) { printf("gradSolve did not reduce the residual\nTest FAILED\n"); return 1; }
        if (!(fgm > 0.8 && bgm < 0.2)) { printf("%s: strokes not held\nTest FAILED\n", names[which]); return 1; }
    }

    cudaFree(dB);
    bmDeviceFree(&dL);
    free(L.a); free(L.bands); free(b); free(alpha); free(im); free(scribs); free(gt);
    printf("Test PASSED\n");
    return 0;
}
