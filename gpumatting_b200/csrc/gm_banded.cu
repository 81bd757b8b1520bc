// gm_banded.cu -- the reference's BandedMatrix API on sm_100a for arbitrary
// band patterns (BandedMatrix.cu): device copies, y = A x (+/- y), the
// damped Jacobi step, and a generic CG / steepest-descent / Jacobi driver
// for patterns that are not the Levin stencil (that one goes to the fused
// persistent kernel in gm_solver.cu).
//
// Conventions kept from the reference: band j of row i is a[i + j*apitch],
// x is zero-padded so x[i + bands[j]] is addressable for every row, and
// band entries that would reach outside the matrix are zero
// (BandedMatrix.cu:128-130).  The band offsets live in device memory (as
// bmCopyToDevice leaves them) and are staged into shared memory per block;
// unlike the reference's fixed __shared__ int sdata[nbands] (sized by a
// template argument smaller than a.nbands), the stage is sized by nbands.
#include <string.h>

#include <algorithm>
#include <vector>

#include "gm_internal.cuh"
#include "gm_solver_api.h"

int gm_note_status(int s);

namespace gm {
int dot_blocks(int n);
int dot_with_scratch(const float* x, const float* y, int n, double* scratch, int nb, float* outf, double* outd,
                     cudaStream_t st);

constexpr int kBandThreads = 256;
constexpr int kMaxBands = 128;

// mode 0: b = A x; 1: b = A x + y; 2: b = A x - y
__global__ void bm_ax_kernel(float* __restrict__ b, const float* __restrict__ a, size_t apitch,
                             const int* __restrict__ bands, int nbands, int rows, const float* __restrict__ x,
                             const float* __restrict__ y, int mode)
{
    __shared__ int off[kMaxBands];
    for (int j = threadIdx.x; j < nbands; j += blockDim.x) off[j] = bands[j];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int j = 0; j < nbands; ++j) s += a[i + (size_t)j * apitch] * __ldg(x + i + off[j]);
        if (mode == 1) s += y[i];
        else if (mode == 2) s -= y[i];
        b[i] = s;
    }
}

// The same product, four consecutive rows per thread: one 128-bit load per
// band for the four rows' coefficients (a 16-byte aligned, apitch a multiple
// of 4), the x values gathered through the read-only path, each row summed
// in band order exactly as bm_ax_kernel does (bit-identical results).  Four
// times the bytes in flight per thread: 0.82 -> 0.94 of HBM for 25 FP32
// bands at 4096^2.
__global__ void bm_ax4_kernel(float* __restrict__ b, const float* __restrict__ a, size_t apitch,
                              const int* __restrict__ bands, int nbands, int rows, const float* __restrict__ x,
                              const float* __restrict__ y, int mode)
{
    __shared__ int off[kMaxBands];
    for (int j = threadIdx.x; j < nbands; j += blockDim.x) off[j] = bands[j];
    __syncthreads();
    const long long nq = rows / 4;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long t = t0; t < nq; t += stride) {
        const long long i = t * 4;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll 5
        for (int j = 0; j < nbands; ++j) {
            const float4 av = __ldg(reinterpret_cast<const float4*>(a + i + (size_t)j * apitch));
            const float* xp = x + i + off[j];
            s0 += av.x * __ldg(xp);
            s1 += av.y * __ldg(xp + 1);
            s2 += av.z * __ldg(xp + 2);
            s3 += av.w * __ldg(xp + 3);
        }
        if (mode == 1) {
            s0 += y[i]; s1 += y[i + 1]; s2 += y[i + 2]; s3 += y[i + 3];
        } else if (mode == 2) {
            s0 -= y[i]; s1 -= y[i + 1]; s2 -= y[i + 2]; s3 -= y[i + 3];
        }
        b[i] = s0; b[i + 1] = s1; b[i + 2] = s2; b[i + 3] = s3;
    }
    // the last rows % 4 rows, one per thread
    for (long long i = nq * 4 + t0; i < rows; i += stride) {
        float s = 0.f;
        for (int j = 0; j < nbands; ++j) s += a[i + (size_t)j * apitch] * __ldg(x + i + off[j]);
        if (mode == 1) s += y[i];
        else if (mode == 2) s -= y[i];
        b[i] = s;
    }
}

// BandedMatrix.cu:61-98 in residual form with the diagonal found by offset.
__global__ void bm_jacobi_kernel(float* __restrict__ xx, const float* __restrict__ x, const float* __restrict__ a,
                                 size_t apitch, const int* __restrict__ bands, int nbands, int rows,
                                 const float* __restrict__ b, float omega, double* part)
{
    __shared__ int off[kMaxBands];
    __shared__ int dband;
    __shared__ double red[32];
    if (threadIdx.x == 0) dband = -1;
    __syncthreads();
    for (int j = threadIdx.x; j < nbands; j += blockDim.x) {
        off[j] = bands[j];
        if (off[j] == 0) atomicMax(&dband, j);
    }
    __syncthreads();
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        float s = b[i];
        for (int j = 0; j < nbands; ++j) s -= a[i + (size_t)j * apitch] * __ldg(x + i + off[j]);
        acc[0] += (double)s * (double)s;
        const float d = dband >= 0 ? a[i + (size_t)dband * apitch] : 1.f;
        const float xi = x[i];
        xx[i] = omega * (xi + s / d) + (1.f - omega) * xi;
    }
    if (part) {
        block_sum<1>(acc, red);
        if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
    }
}

static int band_blocks(int rows)
{
    int nb = (rows + kBandThreads - 1) / kBandThreads;
    return std::max(1, std::min(nb, 148 * 8));
}

static int check_bm(const BandedMatrix& a)
{
    if (!a.a || !a.bands || a.nbands <= 0 || a.nbands > kMaxBands || a.rows < 0 || a.apitch < (size_t)a.rows) {
        gm_set_error_msg("bad BandedMatrix (need device a and bands, 0 < nbands <= %d, apitch >= rows)", kMaxBands);
        return GM_ERR_INVALID;
    }
    return GM_OK;
}

// ---------------------------------------------------------------------------
// Generic solver: a handful of kernels per iteration on the caller's stream.
// ---------------------------------------------------------------------------
__global__ void gen_scalars_kernel(const double* part, int nb, double* sc, int slot)
{
    __shared__ double red[32];
    double t[1];
    grid_total<1>(part, nb, t, red);
    if (threadIdx.x == 0) sc[slot] = t[0];
}

// Scalar slots: 0 rr, 1 pq (or de), 2 rr_new, 3 bb, 4 alpha, 5 flags
__global__ void gen_update_kernel(float* __restrict__ x, float* __restrict__ r, const float* __restrict__ p,
                                  const float* __restrict__ q, int n, const double* sc, double* part)
{
    __shared__ double red[32];
    const double pq = sc[1];
    const float al = pq > 0.0 ? (float)(sc[0] / pq) : 0.f;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += al * p[i];
        const float rn = r[i] - al * q[i];
        r[i] = rn;
        acc[0] += (double)rn * (double)rn;
    }
    block_sum<1>(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

__global__ void gen_pupdate_kernel(float* __restrict__ p, const float* __restrict__ r, int n, double* sc, int zero_beta)
{
    const double rr = sc[0], rn = sc[2];
    const float be = (zero_beta || !(rr > 0.0)) ? 0.f : (float)(rn / rr);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = r[i] + be * p[i];
}

__global__ void gen_rotate_kernel(double* sc) { sc[0] = sc[2]; }

__global__ void gen_residual_kernel(float* __restrict__ r, float* __restrict__ p, const float* __restrict__ a,
                                    size_t apitch, const int* __restrict__ bands, int nbands, int rows,
                                    const float* __restrict__ x, const float* __restrict__ b, double* part)
{
    __shared__ int off[kMaxBands];
    __shared__ double red[32];
    for (int j = threadIdx.x; j < nbands; j += blockDim.x) off[j] = bands[j];
    __syncthreads();
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < nbands; ++j) s += (double)a[i + (size_t)j * apitch] * (double)__ldg(x + i + off[j]);
        const float rv = (float)((double)b[i] - s);
        r[i] = rv;
        if (p) p[i] = rv;
        acc[0] += (double)rv * (double)rv;
        acc[1] += (double)b[i] * (double)b[i];
    }
    block_sum<2>(acc, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = acc[0];
        part[gridDim.x + blockIdx.x] = acc[1];
    }
}

__global__ void gen_scalars2_kernel(const double* part, int nb, double* sc)
{
    __shared__ double red[64];
    double t[2];
    grid_total<2>(part, nb, t, red);
    if (threadIdx.x == 0) { sc[0] = t[0]; sc[3] = t[1]; }
}

int generic_solve(const BandedMatrix& L, float* alpha, int pad, const float* b, const gm_solve_params& p,
                  gm_solve_info* info, cudaStream_t st)
{
    GM_TRY(check_bm(L));
    const int n = L.rows;
    const int nb = band_blocks(n);
    const size_t padded = (size_t)n + 2 * (size_t)pad;
    // r, q unpadded; p padded (operand of the SpMV)
    unsigned char* ws = nullptr;
    const size_t bytes = (size_t)n * 8 + padded * 4 + (size_t)nb * 16 + 64 + 1024;
    GM_CUDA_TRY(cudaMallocAsync((void**)&ws, bytes, st));
    float* r = (float*)ws;
    float* q = r + n;
    float* pp = q + n;
    float* pv = pp + pad;
    double* part = (double*)(((uintptr_t)(pp + padded) + 255) & ~(uintptr_t)255);
    double* sc = part + 2 * nb;
    cudaMemsetAsync(pp, 0, padded * 4, st);
    cudaMemsetAsync(sc, 0, 64, st);
    int it = 0, nrep = 0;
    double rr_host = 0, bb_host = 0, rr_true = 0;
    auto residual = [&](bool reset_p) {
        gen_residual_kernel<<<nb, kBandThreads, 0, st>>>(r, reset_p ? pv : nullptr, L.a, L.apitch, L.bands, L.nbands,
                                                         n, alpha, b, part);
        gen_scalars2_kernel<<<1, 32, 0, st>>>(part, nb, sc);
        ++nrep;
    };
    auto read_scalars = [&]() -> int {
        double h[4];
        GM_CUDA_TRY(cudaMemcpyAsync(h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
        GM_CUDA_TRY(cudaStreamSynchronize(st));
        rr_host = h[0];
        bb_host = h[3];
        return GM_OK;
    };
    int rc = GM_OK;
    if (p.solver == GM_SOLVER_JACOBI) {
        float* x2 = nullptr;
        GM_CUDA_TRY(cudaMallocAsync((void**)&x2, padded * 4, st));
        cudaMemsetAsync(x2, 0, padded * 4, st);
        float* cur = alpha;
        float* nxt = x2 + pad;
        for (it = 0; it < p.max_iters; ++it) {
            bm_jacobi_kernel<<<nb, kBandThreads, 0, st>>>(nxt, cur, L.a, L.apitch, L.bands, L.nbands, n, b, p.omega,
                                                         nullptr);
            std::swap(cur, nxt);
        }
        if (cur != alpha) cudaMemcpyAsync(alpha, cur, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        residual(false);
        rc = read_scalars();
        cudaFreeAsync(x2, st);
    } else {
        residual(true);
        const bool gd = p.solver == GM_SOLVER_GD;
        for (it = 0; it < p.max_iters && rc == GM_OK; ++it) {
            const bool restart = it > 0 && p.restart > 0 && it % p.restart == 0;
            const bool replace = it > 0 && (gd || (p.replace_every > 0 && it % p.replace_every == 0));
            if (restart || (gd && replace)) residual(true);
            else if (replace) residual(false);
            if (p.rtol > 0 && (it % 50 == 0)) {
                rc = read_scalars();
                if (rc != GM_OK) break;
                if (std::sqrt(rr_host / (bb_host > 0 ? bb_host : 1.0)) <= p.rtol) break;
            }
            bm_ax_kernel<<<nb, kBandThreads, 0, st>>>(q, L.a, L.apitch, L.bands, L.nbands, n, pv, nullptr, 0);
            GM_TRY(dot_with_scratch(pv, q, n, part, nb, nullptr, sc + 1, st));
            gen_update_kernel<<<nb, kBandThreads, 0, st>>>(alpha, r, pv, q, n, sc, part);
            gen_scalars_kernel<<<1, 32, 0, st>>>(part, nb, sc, 2);
            gen_pupdate_kernel<<<nb, kBandThreads, 0, st>>>(pv, r, n, sc, gd ? 1 : 0);
            gen_rotate_kernel<<<1, 1, 0, st>>>(sc);
        }
        residual(false);
        if (rc == GM_OK) rc = read_scalars();
    }
    rr_true = rr_host;
    cudaFreeAsync(ws, st);
    if (rc == GM_OK) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { gm_set_error_msg("generic solve: %s", cudaGetErrorString(e)); rc = GM_ERR_CUDA; }
    }
    if (info) {
        memset(info, 0, sizeof(*info));
        info->iters = it;
        info->replacements = nrep;
        info->bnorm = std::sqrt(bb_host);
        info->rel_residual = std::sqrt(rr_true / (bb_host > 0 ? bb_host : 1.0));
        info->status = rc;
        info->solver = p.solver;
        if (rc == GM_OK && p.rtol > 0 && !(info->rel_residual <= p.rtol)) info->status = GM_ERR_NOT_CONVERGED;
    }
    return rc == GM_OK && info ? info->status : rc;
}

}  // namespace gm

using namespace gm;

// b = A x (+/- y): four rows per thread when the band planes allow 128-bit
// loads, else one row per thread; the same sums either way.
static int bm_ax_launch(float* b, const BandedMatrix& a, const float* x, const float* y, int mode, cudaStream_t st)
{
    const bool vec = (reinterpret_cast<uintptr_t>(a.a) & 15) == 0 && a.apitch % 4 == 0 && a.rows >= 4;
    if (vec) {
        const int nq = a.rows / 4;
        bm_ax4_kernel<<<band_blocks(nq), kBandThreads, 0, st>>>(b, a.a, a.apitch, a.bands, a.nbands, a.rows, x, y,
                                                                mode);
    } else {
        bm_ax_kernel<<<band_blocks(a.rows), kBandThreads, 0, st>>>(b, a.a, a.apitch, a.bands, a.nbands, a.rows, x,
                                                                   y, mode);
    }
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_bm_ax(float* b, BandedMatrix a, const float* x, void* stream)
{
    GM_TRY(check_bm(a));
    if (a.rows == 0) return GM_OK;
    return bm_ax_launch(b, a, x, nullptr, 0, (cudaStream_t)stream);
}

extern "C" int gm_bm_axpy(float* b, BandedMatrix a, const float* x, const float* y, int add, void* stream)
{
    GM_TRY(check_bm(a));
    if (a.rows == 0) return GM_OK;
    return bm_ax_launch(b, a, x, y, add ? 1 : 2, (cudaStream_t)stream);
}

extern "C" int gm_jacobi_step(float* xx, const float* x, BandedMatrix a, const float* b, float omega, void* stream)
{
    GM_TRY(check_bm(a));
    if (a.rows == 0) return GM_OK;
    bm_jacobi_kernel<<<band_blocks(a.rows), kBandThreads, 0, (cudaStream_t)stream>>>(xx, x, a.a, a.apitch, a.bands,
                                                                                    a.nbands, a.rows, b, omega, nullptr);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

// BandedMatrix.cu:23-41
extern "C" void bmCopyToDevice(BandedMatrix* dA, const BandedMatrix* hA)
{
    if (!dA || !hA || !hA->a || !hA->bands || hA->nbands <= 0 || hA->rows < 0) {
        gm_set_error_msg("bmCopyToDevice: bad host matrix");
        gm_note_status(GM_ERR_INVALID);
        return;
    }
    *dA = *hA;
    size_t pitch = 0;
    float* a = nullptr;
    int* bands = nullptr;
    const size_t wbytes = (size_t)(hA->rows > 0 ? hA->rows : 1) * sizeof(float);
    if (cudaMallocPitch((void**)&a, &pitch, wbytes, hA->nbands) != cudaSuccess ||
        cudaMalloc((void**)&bands, hA->nbands * sizeof(int)) != cudaSuccess) {
        gm_set_error_msg("bmCopyToDevice: allocation failed");
        gm_note_status(GM_ERR_NOMEM);
        return;
    }
    if (hA->rows > 0 &&
        cudaMemcpy2D(a, pitch, hA->a, hA->apitch * sizeof(float), (size_t)hA->rows * sizeof(float), hA->nbands,
                     cudaMemcpyHostToDevice) != cudaSuccess) {
        gm_set_error_msg("bmCopyToDevice: copy failed");
        gm_note_status(GM_ERR_CUDA);
        return;
    }
    cudaMemcpy(bands, hA->bands, hA->nbands * sizeof(int), cudaMemcpyHostToDevice);
    dA->a = a;
    dA->apitch = pitch / sizeof(float);
    dA->bands = bands;
    gm_note_status(GM_OK);
}

// BandedMatrix.cu:43-47
extern "C" void bmDeviceFree(BandedMatrix* dA)
{
    if (dA) {
        if (dA->bands) cudaFree(dA->bands);
        if (dA->a) cudaFree(dA->a);
        dA->a = nullptr;
        dA->bands = nullptr;
    }
    gm_note_status(GM_OK);
}
