// gm_levin.cu -- Levin matting Laplacian assembly on the GPU.
//
// Gather form (no atomics): a CTA covers a TW x TH pixel tile.  It stages
// the tile's colours plus a 2-pixel halo, computes the statistics of every
// 3x3 window touching the tile once (mean and regularised inverse
// covariance), then each thread sums, for its own pixel i and each of the 24
// neighbours j of the 5x5 stencil, the window terms
//     (1 + (x_i - mu)^T (Sigma + eps/9 I)^-1 (x_j - mu)) / 9
// over the windows holding both, in window raster order (Matting.cu:79-189,
// matlab/getLevinLapRaster.m:22-62).  Rows therefore need no cross-thread
// reduction and every entry is written once.
//
// Two arithmetic modes:
//   levin_sym_kernel   FP64 throughout, rounded once to the store types
//                      (symmetric store + optional 25-band FP32 copy).
//   levin_ref_kernel   the reference's own float/double mix with IEEE
//                      round-to-nearest intrinsics and no FMA contraction,
//                      bit-identical to hostLevinLaplacian (Matting.cu:39-219).
#include <string.h>

#include "gm_internal.cuh"

int gm_note_status(int s);

namespace gm {

constexpr int TW = 32, TH = 8;
constexpr int NWIN = (TW + 2) * (TH + 2);

struct ImgView {
    const unsigned char* data;
    int format;
    size_t pitch;
};

__device__ __forceinline__ void load_rgb_d(const ImgView& im, int u, int v, double& r, double& g, double& b)
{
    if (im.format == GM_IMAGE_RGB8) {
        const unsigned char* p = im.data + (size_t)v * im.pitch + 3 * (size_t)u;
        r = (double)p[0] / 255.0;
        g = (double)p[1] / 255.0;
        b = (double)p[2] / 255.0;
    } else {
        const float4 q = reinterpret_cast<const float4*>(im.data + (size_t)v * im.pitch)[u];
        r = q.x; g = q.y; b = q.z;
    }
}

// ppm.h:325-327: channel / maxval in float (maxval = 255).
__device__ __forceinline__ void load_rgb_f(const ImgView& im, int u, int v, float& r, float& g, float& b)
{
    if (im.format == GM_IMAGE_RGB8) {
        const unsigned char* p = im.data + (size_t)v * im.pitch + 3 * (size_t)u;
        r = __fdiv_rn((float)p[0], 255.0f);
        g = __fdiv_rn((float)p[1], 255.0f);
        b = __fdiv_rn((float)p[2], 255.0f);
    } else {
        const float4 q = reinterpret_cast<const float4*>(im.data + (size_t)v * im.pitch)[u];
        r = q.x; g = q.y; b = q.z;
    }
}

struct ScribView {
    const unsigned char* map;
    size_t map_pitch;
    float gamma_value;
    const float* gamma_map;
    const float* s_map;
    int W;
};

// Matting.cu:205-216: 255 -> (gamma, b = gamma), 0 -> (gamma, b = 0), else
// (0, 0); or per-pixel weights and targets.  Returns whether gamma is added
// to the diagonal (the reference adds nothing on unknown pixels).
__device__ __forceinline__ bool scribble(const ScribView& s, int u, int v, float& gam, float& bv)
{
    if (s.gamma_map) {
        gam = s.gamma_map[(size_t)v * s.W + u];
        bv = s.s_map ? gam * s.s_map[(size_t)v * s.W + u] : 0.f;
        return true;
    }
    if (s.map) {
        const unsigned char c = s.map[(size_t)v * s.map_pitch + u];
        if (c == 255) { gam = s.gamma_value; bv = s.gamma_value; return true; }
        if (c == 0) { gam = s.gamma_value; bv = 0.f; return true; }
    }
    gam = 0.f;
    bv = 0.f;
    return false;
}

template <class T> __device__ __forceinline__ T from_double(double x);
template <> __device__ __forceinline__ float from_double<float>(double x) { return __double2float_rn(x); }
template <> __device__ __forceinline__ __half from_double<__half>(double x) { return __double2half(x); }
template <> __device__ __forceinline__ __nv_bfloat16 from_double<__nv_bfloat16>(double x) { return __double2bfloat16(x); }

struct SymOut {
    void* w;          // [12][H][pitch] in T
    float* w32;       // [12][H][pitch]
    float* gamma;     // [H][pitch]
    float* b;         // [H][pitch]
    int pitch;
    size_t plane;     // elements between planes of w / w32
    float* a25;       // optional [25][apitch]
    size_t apitch;
    float* b25;       // optional [N]
};

template <class T>
__global__ void __launch_bounds__(TW * TH) levin_sym_kernel(ImgView im, ScribView sc, double eps, int W, int H,
                                                            SymOut o)
{
    __shared__ double col[TH + 4][TW + 4][3];
    __shared__ double wmu[NWIN][3];
    __shared__ double wki[NWIN][6];  // inverse covariance: 00 01 02 11 12 22
    const int u0 = blockIdx.x * TW, v0 = blockIdx.y * TH;
    const int tid = threadIdx.x;
    for (int t = tid; t < (TH + 4) * (TW + 4); t += blockDim.x) {
        const int x = t % (TW + 4), y = t / (TW + 4);
        const int u = u0 - 2 + x, v = v0 - 2 + y;
        double r = 0, g = 0, b = 0;
        if (u >= 0 && u < W && v >= 0 && v < H) load_rgb_d(im, u, v, r, g, b);
        col[y][x][0] = r; col[y][x][1] = g; col[y][x][2] = b;
    }
    __syncthreads();
    for (int t = tid; t < NWIN; t += blockDim.x) {
        const int wx = t % (TW + 2), wy = t / (TW + 2);
        const int cu = u0 - 1 + wx, cv = v0 - 1 + wy;
        if (cu < 1 || cu > W - 2 || cv < 1 || cv > H - 2) continue;
        double m[3] = {0, 0, 0}, c[6] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < 9; ++q) {
            const double* p = col[wy + q / 3][wx + q % 3];
            m[0] += p[0]; m[1] += p[1]; m[2] += p[2];
            c[0] += p[0] * p[0]; c[1] += p[0] * p[1]; c[2] += p[0] * p[2];
            c[3] += p[1] * p[1]; c[4] += p[1] * p[2]; c[5] += p[2] * p[2];
        }
        for (int a = 0; a < 3; ++a) m[a] /= 9.0;
        const double e9 = eps / 9.0;
        const double s00 = c[0] / 9.0 - m[0] * m[0] + e9, s01 = c[1] / 9.0 - m[0] * m[1],
                     s02 = c[2] / 9.0 - m[0] * m[2], s11 = c[3] / 9.0 - m[1] * m[1] + e9,
                     s12 = c[4] / 9.0 - m[1] * m[2], s22 = c[5] / 9.0 - m[2] * m[2] + e9;
        const double a00 = s11 * s22 - s12 * s12, a01 = s02 * s12 - s01 * s22, a02 = s01 * s12 - s02 * s11;
        const double a11 = s00 * s22 - s02 * s02, a12 = s02 * s01 - s00 * s12, a22 = s00 * s11 - s01 * s01;
        const double det = s00 * a00 + s01 * a01 + s02 * a02;
        const double id = 1.0 / det;
        wmu[t][0] = m[0]; wmu[t][1] = m[1]; wmu[t][2] = m[2];
        wki[t][0] = a00 * id; wki[t][1] = a01 * id; wki[t][2] = a02 * id;
        wki[t][3] = a11 * id; wki[t][4] = a12 * id; wki[t][5] = a22 * id;
    }
    __syncthreads();
    const int lx = tid % TW, ly = tid / TW;
    const int u = u0 + lx, v = v0 + ly;
    if (u >= W || v >= H) return;
    double acc[25];
#pragma unroll
    for (int k = 0; k < 25; ++k) acc[k] = 0.0;
    const double* xi = col[ly + 2][lx + 2];
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int cu = u + dx, cv = v + dy;
            if (cu < 1 || cu > W - 2 || cv < 1 || cv > H - 2) continue;
            const int t = (ly + 1 + dy) * (TW + 2) + (lx + 1 + dx);
            const double* mu = wmu[t];
            const double* k = wki[t];
            const double x0 = xi[0] - mu[0], x1 = xi[1] - mu[1], x2 = xi[2] - mu[2];
            const double w0 = k[0] * x0 + k[1] * x1 + k[2] * x2;
            const double w1 = k[1] * x0 + k[3] * x1 + k[4] * x2;
            const double w2 = k[2] * x0 + k[4] * x1 + k[5] * x2;
#pragma unroll
            for (int qy = -1; qy <= 1; ++qy) {
#pragma unroll
                for (int qx = -1; qx <= 1; ++qx) {
                    const int ju = dx + qx, jv = dy + qy;  // neighbour offset from i
                    if (ju == 0 && jv == 0) continue;
                    const double* xj = col[ly + 2 + jv][lx + 2 + ju];
                    const double t2 = (1.0 + w0 * (xj[0] - mu[0]) + w1 * (xj[1] - mu[1]) + w2 * (xj[2] - mu[2])) / 9.0;
                    acc[12 + ju + 5 * jv] += t2;
                }
            }
        }
    }
    float gam, bv;
    scribble(sc, u, v, gam, bv);
    const size_t plane = o.plane;
    const size_t gi = (size_t)v * o.pitch + u;
    T* wl = reinterpret_cast<T*>(o.w);
#pragma unroll
    for (int k = 1; k <= 12; ++k) {
        wl[(size_t)(k - 1) * plane + gi] = from_double<T>(acc[12 + k]);
        o.w32[(size_t)(k - 1) * plane + gi] = __double2float_rn(acc[12 + k]);
    }
    o.gamma[gi] = gam;
    o.b[gi] = bv;
    if (o.a25) {
        const size_t i = (size_t)v * W + u;
        double rs = 0.0;
#pragma unroll
        for (int k = 0; k < 25; ++k) {
            if (k == 12) continue;
            const float a = __double2float_rn(-acc[k]);
            o.a25[(size_t)k * o.apitch + i] = a;
            rs -= (double)a;
        }
        o.a25[(size_t)12 * o.apitch + i] = __double2float_rn(rs + (double)gam);
        if (o.b25) o.b25[i] = bv;
    }
}

// ---- reference arithmetic (Matting.cu:79-218), bit-exact ----
struct RefWin {
    float mx, my, mz;
    double d11, d12, d13, d22, d23, d33, cdet;
};

__global__ void __launch_bounds__(TW * TH) levin_ref_kernel(ImgView im, ScribView sc, float lambda, int W, int H,
                                                            float* a, size_t apitch, float* bout)
{
    __shared__ float col[TH + 4][TW + 4][3];
    __shared__ RefWin win[NWIN];
    const int u0 = blockIdx.x * TW, v0 = blockIdx.y * TH;
    const int tid = threadIdx.x;
    for (int t = tid; t < (TH + 4) * (TW + 4); t += blockDim.x) {
        const int x = t % (TW + 4), y = t / (TW + 4);
        const int u = u0 - 2 + x, v = v0 - 2 + y;
        float r = 0, g = 0, b = 0;
        if (u >= 0 && u < W && v >= 0 && v < H) load_rgb_f(im, u, v, r, g, b);
        col[y][x][0] = r; col[y][x][1] = g; col[y][x][2] = b;
    }
    __syncthreads();
    for (int t = tid; t < NWIN; t += blockDim.x) {
        const int wx = t % (TW + 2), wy = t / (TW + 2);
        const int cu = u0 - 1 + wx, cv = v0 - 1 + wy;
        if (cu < 1 || cu > W - 2 || cv < 1 || cv > H - 2) continue;
        float mx = 0.f, my = 0.f, mz = 0.f;
        double c11 = 0, c12 = 0, c13 = 0, c22 = 0, c23 = 0, c33 = 0;
        for (int q = 0; q < 9; ++q) {  // Matting.cu:98-113, raster order
            const float* p = col[wy + q / 3][wx + q % 3];
            mx = __fadd_rn(mx, p[0]); my = __fadd_rn(my, p[1]); mz = __fadd_rn(mz, p[2]);
            c11 = __dadd_rn(c11, (double)__fmul_rn(p[0], p[0]));
            c12 = __dadd_rn(c12, (double)__fmul_rn(p[0], p[1]));
            c13 = __dadd_rn(c13, (double)__fmul_rn(p[0], p[2]));
            c22 = __dadd_rn(c22, (double)__fmul_rn(p[1], p[1]));
            c23 = __dadd_rn(c23, (double)__fmul_rn(p[1], p[2]));
            c33 = __dadd_rn(c33, (double)__fmul_rn(p[2], p[2]));
        }
        mx = __fdiv_rn(mx, 9.0f); my = __fdiv_rn(my, 9.0f); mz = __fdiv_rn(mz, 9.0f);
        const double l9 = (double)__fdiv_rn(lambda, 9.0f);
        c11 = __dadd_rn(__dsub_rn(__ddiv_rn(c11, 9.0), (double)__fmul_rn(mx, mx)), l9);
        c12 = __dsub_rn(__ddiv_rn(c12, 9.0), (double)__fmul_rn(mx, my));
        c13 = __dsub_rn(__ddiv_rn(c13, 9.0), (double)__fmul_rn(mx, mz));
        c22 = __dadd_rn(__dsub_rn(__ddiv_rn(c22, 9.0), (double)__fmul_rn(my, my)), l9);
        c23 = __dsub_rn(__ddiv_rn(c23, 9.0), (double)__fmul_rn(my, mz));
        c33 = __dadd_rn(__dsub_rn(__ddiv_rn(c33, 9.0), (double)__fmul_rn(mz, mz)), l9);
        // Matting.cu:130-137, left to right
        const double t1 = __dmul_rn(__dmul_rn(c11, c22), c33);
        const double t2 = __dmul_rn(__dmul_rn(c12, c23), c13);
        const double t3 = __dmul_rn(__dmul_rn(c13, c12), c23);
        const double t4 = __dmul_rn(__dmul_rn(c13, c22), c13);
        const double t5 = __dmul_rn(__dmul_rn(c12, c12), c33);
        const double t6 = __dmul_rn(__dmul_rn(c11, c23), c23);
        RefWin w;
        w.cdet = __dsub_rn(__dsub_rn(__dsub_rn(__dadd_rn(__dadd_rn(t1, t2), t3), t4), t5), t6);
        w.d11 = __dsub_rn(__dmul_rn(c33, c22), __dmul_rn(c23, c23));
        w.d12 = __dsub_rn(__dmul_rn(c13, c23), __dmul_rn(c33, c12));
        w.d13 = __dsub_rn(__dmul_rn(c23, c12), __dmul_rn(c22, c13));
        w.d22 = __dsub_rn(__dmul_rn(c33, c11), __dmul_rn(c13, c13));
        w.d23 = __dsub_rn(__dmul_rn(c12, c13), __dmul_rn(c23, c11));
        w.d33 = __dsub_rn(__dmul_rn(c22, c11), __dmul_rn(c12, c12));
        w.mx = mx; w.my = my; w.mz = mz;
        win[t] = w;
    }
    __syncthreads();
    const int lx = tid % TW, ly = tid / TW;
    const int u = u0 + lx, v = v0 + ly;
    if (u >= W || v >= H) return;
    float acc[25];
#pragma unroll
    for (int k = 0; k < 25; ++k) acc[k] = 0.f;
    const float* xi = col[ly + 2][lx + 2];
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int cu = u + dx, cv = v + dy;
            if (cu < 1 || cu > W - 2 || cv < 1 || cv > H - 2) continue;
            const RefWin& w = win[(ly + 1 + dy) * (TW + 2) + (lx + 1 + dx)];
            const float rx = __fsub_rn(xi[0], w.mx), ry = __fsub_rn(xi[1], w.my), rz = __fsub_rn(xi[2], w.mz);
            // Matting.cu:151-153
            const float wx = __double2float_rn(__ddiv_rn(
                __dadd_rn(__dadd_rn(__dmul_rn(w.d11, (double)rx), __dmul_rn(w.d12, (double)ry)), __dmul_rn(w.d13, (double)rz)),
                w.cdet));
            const float wy = __double2float_rn(__ddiv_rn(
                __dadd_rn(__dadd_rn(__dmul_rn(w.d12, (double)rx), __dmul_rn(w.d22, (double)ry)), __dmul_rn(w.d23, (double)rz)),
                w.cdet));
            const float wz = __double2float_rn(__ddiv_rn(
                __dadd_rn(__dadd_rn(__dmul_rn(w.d13, (double)rx), __dmul_rn(w.d23, (double)ry)), __dmul_rn(w.d33, (double)rz)),
                w.cdet));
#pragma unroll
            for (int qy = -1; qy <= 1; ++qy) {
#pragma unroll
                for (int qx = -1; qx <= 1; ++qx) {
                    const int ju = dx + qx, jv = dy + qy;
                    const float* xj = col[ly + 2 + jv][lx + 2 + ju];
                    const float sx = __fsub_rn(xj[0], w.mx), sy = __fsub_rn(xj[1], w.my), sz = __fsub_rn(xj[2], w.mz);
                    // Matting.cu:177
                    const float t = __fadd_rn(__fadd_rn(__fadd_rn(1.0f, __fmul_rn(wx, sx)), __fmul_rn(wy, sy)),
                                              __fmul_rn(wz, sz));
                    const float neg = __fdiv_rn(-t, 9.0f);
                    acc[12 + ju + 5 * jv] = __fadd_rn(acc[12 + ju + 5 * jv], neg);
                }
            }
        }
    }
    // Matting.cu:192-216
    double rs = 0.0;
#pragma unroll
    for (int k = 0; k < 25; ++k) rs = __dadd_rn(rs, (double)acc[k]);
    float diag = __double2float_rn(__dsub_rn((double)acc[12], rs));
    float gam, bv;
    if (scribble(sc, u, v, gam, bv)) diag = __fadd_rn(diag, gam);
    acc[12] = diag;
    const size_t i = (size_t)v * W + u;
#pragma unroll
    for (int k = 0; k < 25; ++k) a[(size_t)k * apitch + i] = acc[k];
    if (bout) bout[i] = bv;
}

// d_i = gamma_i + sum of the affinities of row i as stored (upper planes at
// i, lower ones at the neighbour), summed in FP64 and rounded once, for the
// low-precision planes (d) and the FP32 planes (d32).
template <class T>
__global__ void levin_diag_kernel(const T* __restrict__ w, const float* __restrict__ w32,
                                  const float* __restrict__ gamma, float* d, float* d32, int W, int H, int pitch,
                                  size_t plane)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W) return;
    const size_t i = (size_t)v * pitch + u;
    double s = gamma[i], s32 = gamma[i];
#pragma unroll
    for (int k = 1; k <= 12; ++k) {
        const int dv = (k + 2) / 5, du = k - 5 * dv;
        s += (double)Cvt<T>::to_f(w[(k - 1) * plane + i]);
        s32 += (double)w32[(k - 1) * plane + i];
        const int ul = u - du, vl = v - dv;
        if (ul >= 0 && ul < W && vl >= 0) {
            const size_t j = (size_t)vl * pitch + ul;
            s += (double)Cvt<T>::to_f(w[(k - 1) * plane + j]);
            s32 += (double)w32[(k - 1) * plane + j];
        }
    }
    d[i] = __double2float_rn(s);
    d32[i] = __double2float_rn(s32);
}

template <class T>
static void launch_sym(const ImgView& im, const ScribView& sc, double eps, int W, int H, const SymOut& o,
                       float* d, float* d32, cudaStream_t st)
{
    dim3 grid((W + TW - 1) / TW, (H + TH - 1) / TH);
    levin_sym_kernel<T><<<grid, TW * TH, 0, st>>>(im, sc, eps, W, H, o);
    dim3 g2((W + 127) / 128, H);
    levin_diag_kernel<T><<<g2, 128, 0, st>>>(reinterpret_cast<const T*>(o.w), o.w32, o.gamma, d, d32, W, H, o.pitch,
                                             o.plane);
}

// ---------------------------------------------------------------------------
// Adjoint of the assembly
// ---------------------------------------------------------------------------
// For a loss of alpha with lam = A^-1 dloss/dalpha (A is symmetric), every
// pair (i, j) the store couples has dloss/dw_ij = -(lam_i - lam_j)(alpha_i -
// alpha_j), and each window k adds w_ij += (1 + x_i^T K^-1 x_j) / 9 with
// x = I - mu_k and K = Sigma_k + eps/9 I.  Summing the pair gradients of one
// window collapses to two 3-vectors,
//   ka = K^-1 sum_a x_a alpha_a,   kl = K^-1 sum_a x_a lam_a,
// and pixel a of the window receives
//   dI_a += [(lam_a - mean lam) ka + (alpha_a - mean alpha) kl] / 9
//           - [(x_a . kl) ka + (x_a . ka) kl] / 81.
// The window statistics are recomputed from the image (the forward pass
// stores none).  FP64 throughout, one FP32 rounding per output.

// Scribble target s_i: the value b_i / gamma_i the forward pass encodes
// (0 where the pixel carries no scribble).
__device__ __forceinline__ float scribble_target(const ScribView& s, int u, int v)
{
    if (s.gamma_map) return s.s_map ? s.s_map[(size_t)v * s.W + u] : 0.f;
    if (s.map) return s.map[(size_t)v * s.map_pitch + u] == 255 ? 1.f : 0.f;
    return 0.f;
}

struct AdjOut {
    float* dimage;   // [H][dpitch] floats, `channels` per pixel
    size_t dpitch;
    int channels;    // 3 or 4 (the fourth is written as 0)
    float* dgamma;   // [H][W] or NULL
};

__global__ void __launch_bounds__(TW * TH) levin_adjoint_kernel(ImgView im, ScribView sc, double eps, int W, int H,
                                                                const float* __restrict__ lam,
                                                                const float* __restrict__ alpha, AdjOut o)
{
    __shared__ double col[TH + 4][TW + 4][3];
    __shared__ double sl[TH + 4][TW + 4];
    __shared__ double sa[TH + 4][TW + 4];
    __shared__ double wmu[NWIN][3];
    __shared__ double wka[NWIN][3];
    __shared__ double wkl[NWIN][3];
    __shared__ double wbar[NWIN][2];  // mean lam, mean alpha
    const int u0 = blockIdx.x * TW, v0 = blockIdx.y * TH;
    const int tid = threadIdx.x;
    for (int t = tid; t < (TH + 4) * (TW + 4); t += blockDim.x) {
        const int x = t % (TW + 4), y = t / (TW + 4);
        const int u = u0 - 2 + x, v = v0 - 2 + y;
        double r = 0, g = 0, b = 0, l = 0, a = 0;
        if (u >= 0 && u < W && v >= 0 && v < H) {
            load_rgb_d(im, u, v, r, g, b);
            l = lam[(size_t)v * W + u];
            a = alpha[(size_t)v * W + u];
        }
        col[y][x][0] = r; col[y][x][1] = g; col[y][x][2] = b;
        sl[y][x] = l;
        sa[y][x] = a;
    }
    __syncthreads();
    for (int t = tid; t < NWIN; t += blockDim.x) {
        const int wx = t % (TW + 2), wy = t / (TW + 2);
        const int cu = u0 - 1 + wx, cv = v0 - 1 + wy;
        if (cu < 1 || cu > W - 2 || cv < 1 || cv > H - 2) continue;
        double m[3] = {0, 0, 0}, c[6] = {0, 0, 0, 0, 0, 0}, lb = 0, ab = 0;
        for (int q = 0; q < 9; ++q) {
            const double* p = col[wy + q / 3][wx + q % 3];
            m[0] += p[0]; m[1] += p[1]; m[2] += p[2];
            c[0] += p[0] * p[0]; c[1] += p[0] * p[1]; c[2] += p[0] * p[2];
            c[3] += p[1] * p[1]; c[4] += p[1] * p[2]; c[5] += p[2] * p[2];
            lb += sl[wy + q / 3][wx + q % 3];
            ab += sa[wy + q / 3][wx + q % 3];
        }
        for (int a = 0; a < 3; ++a) m[a] /= 9.0;
        const double e9 = eps / 9.0;
        const double s00 = c[0] / 9.0 - m[0] * m[0] + e9, s01 = c[1] / 9.0 - m[0] * m[1],
                     s02 = c[2] / 9.0 - m[0] * m[2], s11 = c[3] / 9.0 - m[1] * m[1] + e9,
                     s12 = c[4] / 9.0 - m[1] * m[2], s22 = c[5] / 9.0 - m[2] * m[2] + e9;
        const double a00 = s11 * s22 - s12 * s12, a01 = s02 * s12 - s01 * s22, a02 = s01 * s12 - s02 * s11;
        const double a11 = s00 * s22 - s02 * s02, a12 = s02 * s01 - s00 * s12, a22 = s00 * s11 - s01 * s01;
        const double id = 1.0 / (s00 * a00 + s01 * a01 + s02 * a02);
        double va[3] = {0, 0, 0}, vl[3] = {0, 0, 0};
        for (int q = 0; q < 9; ++q) {
            const double* p = col[wy + q / 3][wx + q % 3];
            const double l = sl[wy + q / 3][wx + q % 3], a = sa[wy + q / 3][wx + q % 3];
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const double x = p[e] - m[e];
                va[e] += x * a;
                vl[e] += x * l;
            }
        }
        wmu[t][0] = m[0]; wmu[t][1] = m[1]; wmu[t][2] = m[2];
        wka[t][0] = (a00 * va[0] + a01 * va[1] + a02 * va[2]) * id;
        wka[t][1] = (a01 * va[0] + a11 * va[1] + a12 * va[2]) * id;
        wka[t][2] = (a02 * va[0] + a12 * va[1] + a22 * va[2]) * id;
        wkl[t][0] = (a00 * vl[0] + a01 * vl[1] + a02 * vl[2]) * id;
        wkl[t][1] = (a01 * vl[0] + a11 * vl[1] + a12 * vl[2]) * id;
        wkl[t][2] = (a02 * vl[0] + a12 * vl[1] + a22 * vl[2]) * id;
        wbar[t][0] = lb / 9.0;
        wbar[t][1] = ab / 9.0;
    }
    __syncthreads();
    const int lx = tid % TW, ly = tid / TW;
    const int u = u0 + lx, v = v0 + ly;
    if (u >= W || v >= H) return;
    const double* xi = col[ly + 2][lx + 2];
    const double li = sl[ly + 2][lx + 2], ai = sa[ly + 2][lx + 2];
    double g[3] = {0, 0, 0};
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int cu = u + dx, cv = v + dy;
            if (cu < 1 || cu > W - 2 || cv < 1 || cv > H - 2) continue;
            const int t = (ly + 1 + dy) * (TW + 2) + (lx + 1 + dx);
            const double x0 = xi[0] - wmu[t][0], x1 = xi[1] - wmu[t][1], x2 = xi[2] - wmu[t][2];
            const double* ka = wka[t];
            const double* kl = wkl[t];
            const double xkl = x0 * kl[0] + x1 * kl[1] + x2 * kl[2];
            const double xka = x0 * ka[0] + x1 * ka[1] + x2 * ka[2];
            const double dl = (li - wbar[t][0]) / 9.0 - xkl / 81.0;
            const double da = (ai - wbar[t][1]) / 9.0 - xka / 81.0;
#pragma unroll
            for (int e = 0; e < 3; ++e) g[e] += dl * ka[e] + da * kl[e];
        }
    }
    float* out = o.dimage + (size_t)v * o.dpitch + (size_t)o.channels * u;
    out[0] = __double2float_rn(g[0]);
    out[1] = __double2float_rn(g[1]);
    out[2] = __double2float_rn(g[2]);
    if (o.channels == 4) out[3] = 0.f;
    if (o.dgamma) {
        const double s = scribble_target(sc, u, v);
        o.dgamma[(size_t)v * W + u] = __double2float_rn(li * (s - ai));
    }
}

// ---------------------------------------------------------------------------
// Restriction to the unknown pixels (hard constraints)
// ---------------------------------------------------------------------------
// Pixels with a scribble (or a positive gamma_map weight) are known: their
// value is fixed at the target s.  The store becomes the system on the
// unknown pixels with the known ones eliminated: for an unknown pixel i and a
// known neighbour j, w_ij (x_i - s_j) moves to the diagonal (gamma_i += w_ij)
// and the right-hand side (b_i += w_ij s_j); known rows become x_i = s_i;
// every coupling that touches a known pixel is removed.  Pass 1 gathers the
// new gamma and b per pixel (reads planes only), pass 2 zeroes the removed
// couplings, then the diagonal planes are recomputed.

__device__ __forceinline__ bool known_at(const ScribView& s, int u, int v, float& target)
{
    float gam, bv;
    const bool has = scribble(s, u, v, gam, bv);
    target = scribble_target(s, u, v);
    return has && gam > 0.f;
}

__global__ void levin_restrict_gather_kernel(ScribView sc, const float* __restrict__ w32, float* gamma, float* b,
                                             int W, int H, int pitch, size_t plane)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W) return;
    const size_t i = (size_t)v * pitch + u;
    float si;
    if (known_at(sc, u, v, si)) {
        gamma[i] = 1.f;
        b[i] = si;
        return;
    }
    double g = gamma[i], bb = b[i];
#pragma unroll
    for (int k = 1; k <= 12; ++k) {
        const int dv = (k + 2) / 5, du = k - 5 * dv;
        const int uf = u + du, vf = v + dv;  // upper partner: coupling stored at i
        float sj;
        if (uf >= 0 && uf < W && vf < H && known_at(sc, uf, vf, sj)) {
            const double w = w32[(size_t)(k - 1) * plane + i];
            g += w;
            bb += w * (double)sj;
        }
        const int ul = u - du, vl = v - dv;  // lower partner: coupling stored at the partner
        if (ul >= 0 && ul < W && vl >= 0 && known_at(sc, ul, vl, sj)) {
            const double w = w32[(size_t)(k - 1) * plane + (size_t)vl * pitch + ul];
            g += w;
            bb += w * (double)sj;
        }
    }
    gamma[i] = __double2float_rn(g);
    b[i] = __double2float_rn(bb);
}

template <class T>
__global__ void levin_restrict_cut_kernel(ScribView sc, T* w, float* w32, int W, int H, int pitch, size_t plane)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W) return;
    const size_t i = (size_t)v * pitch + u;
    float t;
    const bool ki = known_at(sc, u, v, t);
#pragma unroll
    for (int k = 1; k <= 12; ++k) {
        const int dv = (k + 2) / 5, du = k - 5 * dv;
        const int uf = u + du, vf = v + dv;
        const bool kj = uf >= 0 && uf < W && vf < H && known_at(sc, uf, vf, t);
        if (ki || kj) {
            w[(size_t)(k - 1) * plane + i] = from_double<T>(0.0);
            w32[(size_t)(k - 1) * plane + i] = 0.f;
        }
    }
}

}  // namespace gm

using namespace gm;

static int make_views(const gm_image* im, const gm_scribbles* sc, int W, ImgView& iv, ScribView& sv)
{
    if (!im || !im->data) { gm_set_error_msg("image is NULL"); return GM_ERR_INVALID; }
    if (im->format != GM_IMAGE_RGB8 && im->format != GM_IMAGE_RGBA32F) { gm_set_error_msg("unknown image format"); return GM_ERR_INVALID; }
    iv.data = (const unsigned char*)im->data;
    iv.format = im->format;
    iv.pitch = im->pitch_bytes;
    if (im->format == GM_IMAGE_RGBA32F && (((uintptr_t)im->data & 15) || (im->pitch_bytes & 15))) {
        gm_set_error_msg("RGBA32F image must be 16-byte aligned with a 16-byte multiple pitch");
        return GM_ERR_INVALID;
    }
    memset(&sv, 0, sizeof(sv));
    sv.W = W;
    if (sc) {
        sv.map = sc->map;
        sv.map_pitch = sc->map_pitch ? sc->map_pitch : (size_t)W;
        sv.gamma_value = sc->gamma_value;
        sv.gamma_map = sc->gamma_map;
        sv.s_map = sc->s_map;
    }
    return GM_OK;
}

extern "C" int gm_levin_store_alloc(gm_levin_store* st, int W, int H, int precision)
{
    if (!st || W <= 0 || H <= 0) { gm_set_error_msg("bad store size"); return GM_ERR_INVALID; }
    if (precision < GM_PREC_FP32 || precision > GM_PREC_BF16) { gm_set_error_msg("bad precision"); return GM_ERR_INVALID; }
    memset(st, 0, sizeof(*st));
    st->W = W;
    st->H = H;
    st->pitch = (W + 7) & ~7;
    st->precision = precision;
    const size_t plane = (size_t)H * st->pitch;
    const size_t esz = precision == GM_PREC_FP32 ? 4 : 2;
    const size_t lo_bytes = precision == GM_PREC_FP32 ? 0 : ((12 * plane * esz + 255) & ~(size_t)255);
    const size_t b32 = (12 * plane * 4 + 255) & ~(size_t)255;
    const size_t b1 = (plane * 4 + 255) & ~(size_t)255;
    unsigned char* m = nullptr;
    if (cudaMalloc((void**)&m, lo_bytes + b32 + 4 * b1) != cudaSuccess) {
        gm_set_error_msg("store allocation failed");
        return GM_ERR_NOMEM;
    }
    st->w32 = (float*)m;
    st->w = precision == GM_PREC_FP32 ? (void*)m : (void*)(m + b32);
    st->gamma = (float*)(m + b32 + lo_bytes);
    st->b = (float*)(m + b32 + lo_bytes + b1);
    st->d = (float*)(m + b32 + lo_bytes + 2 * b1);
    st->d32 = (float*)(m + b32 + lo_bytes + 3 * b1);
    st->owns = 1;
    return GM_OK;
}

extern "C" int gm_levin_store_free(gm_levin_store* st)
{
    if (!st) return GM_ERR_INVALID;
    if (st->owns && st->w32) cudaFree(st->w32);
    memset(st, 0, sizeof(*st));
    return GM_OK;
}

extern "C" int gm_levin_assemble(gm_levin_store* st, const gm_image* im, const gm_scribbles* sc, double eps,
                                 BandedMatrix* bands25, float* b25, void* stream)
{
    if (!st || !st->w || !st->w32 || !st->gamma || !st->b || !st->d || !st->d32) {
        gm_set_error_msg("store not allocated");
        return GM_ERR_INVALID;
    }
    if (!(eps >= 0.0)) { gm_set_error_msg("eps must be >= 0"); return GM_ERR_INVALID; }
    GM_TRY(gm_check_device(nullptr));
    ImgView iv;
    ScribView sv;
    GM_TRY(make_views(im, sc, st->W, iv, sv));
    SymOut o;
    memset(&o, 0, sizeof(o));
    o.w = st->w;
    o.w32 = st->w32;
    o.gamma = st->gamma;
    o.b = st->b;
    o.pitch = st->pitch;
    o.plane = st->plane_stride ? st->plane_stride : (size_t)st->H * st->pitch;
    if (bands25) {
        if (!bands25->a || bands25->nbands != 25 || bands25->rows != st->W * st->H ||
            bands25->apitch < (size_t)bands25->rows) {
            gm_set_error_msg("bands25 must be a device BandedMatrix of 25 bands and W*H rows");
            return GM_ERR_INVALID;
        }
        o.a25 = bands25->a;
        o.apitch = bands25->apitch;
        o.b25 = b25;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (st->precision == GM_PREC_FP16) launch_sym<__half>(iv, sv, eps, st->W, st->H, o, st->d, st->d32, s);
    else if (st->precision == GM_PREC_BF16) launch_sym<__nv_bfloat16>(iv, sv, eps, st->W, st->H, o, st->d, st->d32, s);
    else launch_sym<float>(iv, sv, eps, st->W, st->H, o, st->d, st->d32, s);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_levin_assemble_bands25(float* a, size_t apitch, float* b, const gm_image* im,
                                         const gm_scribbles* sc, double eps, int W, int H, int arithmetic,
                                         void* stream)
{
    if (!a || W <= 0 || H <= 0 || apitch < (size_t)W * H) { gm_set_error_msg("bad 25-band output"); return GM_ERR_INVALID; }
    GM_TRY(gm_check_device(nullptr));
    ImgView iv;
    ScribView sv;
    GM_TRY(make_views(im, sc, W, iv, sv));
    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid((W + TW - 1) / TW, (H + TH - 1) / TH);
    if (arithmetic == GM_ASSEMBLY_REFERENCE) {
        levin_ref_kernel<<<grid, TW * TH, 0, s>>>(iv, sv, (float)eps, W, H, a, apitch, b);
    } else {
        // FP64 path through a scratch symmetric store.
        gm_levin_store tmp;
        GM_TRY(gm_levin_store_alloc(&tmp, W, H, GM_PREC_FP32));
        BandedMatrix bm;
        bm.a = a; bm.apitch = apitch; bm.bands = nullptr; bm.nbands = 25; bm.rows = W * H; bm.cols = W * H;
        int rc = gm_levin_assemble(&tmp, im, sc, eps, &bm, b, stream);
        cudaStreamSynchronize(s);
        gm_levin_store_free(&tmp);
        if (rc != GM_OK) return rc;
    }
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

// Image and scribble-weight gradients from lam and alpha (both [H][W] floats
// on the device).  Used by gm_levin_adjoint after its lam solve.
int gm_levin_adjoint_grads(const gm_image* im, const gm_scribbles* sc, double eps, int W, int H,
                           const float* lam, const float* alpha, float* dimage, size_t dimage_pitch,
                           int dimage_channels, float* dgamma, cudaStream_t stream)
{
    if (W <= 0 || H <= 0 || !lam || !alpha || !dimage) { gm_set_error_msg("adjoint: bad arguments"); return GM_ERR_INVALID; }
    if (dimage_channels != 3 && dimage_channels != 4) { gm_set_error_msg("adjoint: dimage_channels must be 3 or 4"); return GM_ERR_INVALID; }
    if (dimage_pitch < (size_t)dimage_channels * W) { gm_set_error_msg("adjoint: dimage_pitch below channels * W"); return GM_ERR_INVALID; }
    if (!(eps >= 0.0)) { gm_set_error_msg("eps must be >= 0"); return GM_ERR_INVALID; }
    ImgView iv;
    ScribView sv;
    GM_TRY(make_views(im, sc, W, iv, sv));
    AdjOut o;
    o.dimage = dimage;
    o.dpitch = dimage_pitch;
    o.channels = dimage_channels;
    o.dgamma = dgamma;
    dim3 grid((W + TW - 1) / TW, (H + TH - 1) / TH);
    levin_adjoint_kernel<<<grid, TW * TH, 0, stream>>>(iv, sv, eps, W, H, lam, alpha, o);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_levin_restrict(gm_levin_store* st, const gm_scribbles* sc, void* stream)
{
    if (!st || !st->w || !st->w32 || !st->gamma || !st->b || !st->d || !st->d32 || !sc) {
        gm_set_error_msg("gm_levin_restrict: bad arguments");
        return GM_ERR_INVALID;
    }
    if (!sc->map && !sc->gamma_map) { gm_set_error_msg("gm_levin_restrict: no known pixels given"); return GM_ERR_INVALID; }
    GM_TRY(gm_check_device(nullptr));
    ScribView sv;
    memset(&sv, 0, sizeof(sv));
    sv.W = st->W;
    sv.map = sc->map;
    sv.map_pitch = sc->map_pitch ? sc->map_pitch : (size_t)st->W;
    sv.gamma_value = 1.f;  // only "known or not" matters here
    sv.gamma_map = sc->gamma_map;
    sv.s_map = sc->s_map;
    const int W = st->W, H = st->H, P = st->pitch;
    const size_t plane = st->plane_stride ? st->plane_stride : (size_t)H * P;
    cudaStream_t s = (cudaStream_t)stream;
    dim3 g((W + 127) / 128, H);
    levin_restrict_gather_kernel<<<g, 128, 0, s>>>(sv, st->w32, st->gamma, st->b, W, H, P, plane);
    if (st->precision == GM_PREC_FP16)
        levin_restrict_cut_kernel<__half><<<g, 128, 0, s>>>(sv, (__half*)st->w, st->w32, W, H, P, plane);
    else if (st->precision == GM_PREC_BF16)
        levin_restrict_cut_kernel<__nv_bfloat16><<<g, 128, 0, s>>>(sv, (__nv_bfloat16*)st->w, st->w32, W, H, P, plane);
    else
        levin_restrict_cut_kernel<float><<<g, 128, 0, s>>>(sv, (float*)st->w, st->w32, W, H, P, plane);
    if (st->precision == GM_PREC_FP16)
        levin_diag_kernel<__half><<<g, 128, 0, s>>>((const __half*)st->w, st->w32, st->gamma, st->d, st->d32, W, H, P, plane);
    else if (st->precision == GM_PREC_BF16)
        levin_diag_kernel<__nv_bfloat16><<<g, 128, 0, s>>>((const __nv_bfloat16*)st->w, st->w32, st->gamma, st->d,
                                                           st->d32, W, H, P, plane);
    else
        levin_diag_kernel<float><<<g, 128, 0, s>>>((const float*)st->w, st->w32, st->gamma, st->d, st->d32, W, H, P, plane);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}
