// gm_mg.cu -- CG preconditioned with an aggregation multigrid V-cycle on the
// symmetric Levin store (GM_SOLVER_MG).
//
// The reference's unfinished direction for faster solves is a hierarchy of
// piecewise-constant aggregation operators (gridoperators.h:18-138: restriction
// matrices with unit entries, pixel -> label) over superpixels (SLIC.cpp:32;
// the call sits commented out at main.cu:201-218).  Here the aggregates are
// fixed 2x2 blocks, so every level keeps a banded stencil that streams like
// the fine one:
//
//   level 0      the store's iteration operator (12 upper planes w + the
//                diagonal d; FP16 / BF16 / FP32 planes);
//   level l+1    Galerkin P^T A_l P with P the 2x2 aggregation: 4 FP32 upper
//                coupling planes (E, SW, S, SE) + diagonal Gamma + sum of the
//                couplings leaving the aggregate;
//   coarsest     the first level with <= kCoarseMax cells, inverted once per
//                solve (FP64 Gauss-Jordan in shared memory).
//
// V-cycle on level l with right-hand side b: x1 = omega b / D,
// b_{l+1} = P^T (b - A x1), recurse, y = x1 + scale P x_{l+1},
// x = y + omega (b - A y) / D.  Each level above the tail costs two streaming
// kernels ("down": smoothing + residual + restriction; "up": prolongation +
// smoothing), both the persistent TMA-ring stencil kernel mg_fine_kernel; x1
// is recomputed from b in "up" instead of stored.  The small levels at the
// bottom (up to 160 KB of operators) run in one CTA (mg_tail_kernel), staged
// in shared memory with block barriers between their phases.
//
// Outer loop: PCG with FP64 solution (plus an FP32 increment folded in after
// each replacement), FP32 vectors and FP64 scalars on the true FP32 operator;
// only the preconditioner reads the low-precision planes (the few MG
// iterations make the outer operator's bytes minor, and a BF16 outer operator
// would stall the recurrence).  The true residual b - A x in FP64 arithmetic
// replaces the recurrence every `replace_every` iterations and decides
// convergence (the same reliable-update rule as the fused CG).
// All scalars stay on the device: every reduction ends in the last CTA to
// finish (fixed summation order, so results are deterministic), and the whole
// solve is ONE CUDA graph launch whose iteration loop is a device-side
// conditional WHILE node -- no host round trip per iteration.  Kernels are
// chained with programmatic dependent launch.  gm_levin_solve_mg_many runs
// many such solves on concurrent streams.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "gm_internal.cuh"

namespace gm {
namespace mg {

constexpr int kCoarseMax = 128;   // cells of the directly solved level
// Smoother damping and coarse-correction scale.  A sweep on the GPU over
// omega in {0.7 .. 1.0} x scale in {1.5 .. 2.4} put (0.8, 1.5) among the
// fastest at 640x480, 1920x1080 and 4096^2 (eps 1e-7); omega = 1.0 stalls.
constexpr float kDefaultOmega = 0.8f;
constexpr float kDefaultScale = 1.5f;
constexpr int kMaxLevels = 24;
constexpr int kThreads = 256;     // 32 x 8
constexpr int kTX = 64;           // tile columns (2 per thread)
constexpr int kTY = 8;            // tile rows of apply / up / replacement tiles
constexpr int kHalo = 2;
constexpr int kPW = kTX + 16;     // plane tile width: tile + 8 columns each side (16-byte aligned loads)
constexpr int kVW = kTX + 2 * kHalo;
constexpr int kMaxParts = 4096;

// Stencils.  Fine: 12 upper planes, plane k couples (x, y) with
// (x + du, y + dv), du = ((k + 3) % 5) - 2, dv = (k + 3) / 5 (k = 0..11 is the
// store's k = 1..12).  Coarse: 4 upper planes E (1,0), SW (-1,1), S (0,1),
// SE (1,1).
struct FineSten {
    static constexpr int NP = 12;
    __host__ __device__ static constexpr int du(int k) { return ((k + 3) % 5) - 2; }
    __host__ __device__ static constexpr int dv(int k) { return (k + 3) / 5; }
};
struct CoarseSten {
    static constexpr int NP = 4;
    __host__ __device__ static constexpr int du(int k) { return k == 0 ? 1 : (k == 1 ? -1 : (k == 2 ? 0 : 1)); }
    __host__ __device__ static constexpr int dv(int k) { return k == 0 ? 0 : 1; }
};

// Device-resident solver state (scalars of the outer PCG).
struct State {
    double rz, pq, alpha, beta, rr, bn2, rr_true;
    int iter, done, status, need_replace, replacements;
    int fold_at;  // iteration whose update folds the FP32 increment into x
    int restart;  // the next search direction is z alone (beta = 0)
    unsigned ticket[8];
};
enum { T_PQ = 0, T_RR = 1, T_TRUE = 2, T_RZ = 3 };

// One level's operator and vectors (l >= 1: FP32 planes of its own; level 0
// points into the store and the fine work vectors).
struct Lev {
    int W, H, P;          // cells, rows, pitch (elements)
    void* c;              // planes [NP][H][P] (level 0: the store's w, type T)
    size_t ps;            // plane stride (elements)
    float* D;             // diagonal [H][P]
    float* Di;            // 1 / D (0 where D = 0): the smoothers multiply
    float* gam;           // summed scribble weight (l >= 1)
    float* b;             // right-hand side of the V-cycle on this level
    float* x;             // V-cycle result on this level
};

struct Args {
    Lev lev[kMaxLevels];
    int L;                // index of the coarsest level
    int lt;               // first level of the single-CTA tail (1 <= lt <= L)
    int W, H, P;          // fine grid (== lev[0])
    const float* w32;     // true operator: FP32 planes, gamma and d32 = gamma + row sum
    size_t ps32;
    const float* gamma;
    const float* d32;
    const float* bvec;    // right-hand side [H][bpitch]
    int bpitch;
    const float* alpha_in;
    float* alpha_out;     // [H][W]
    double* x;            // FP64 solution [H][P]; the solution is x + xinc
    float* xinc;          // FP32 increment since the last replacement [H][P]
    float *r, *q, *p0, *p1;  // fine vectors [H][P]; z is lev[0].x
    double* minv;         // coarsest inverse [n][n]
    double* parts;        // [5][kMaxParts]: pq, rr, true rr + bb, rz
    State* st;
    double rtol;
    int max_iters, replace_every;
    int outer_low;  // the level-0 SpMV streams the FP16 iteration planes, not w32
    int spare;      // keeps the struct free of padding (it is compared bytewise)
    float omega, scale;
    unsigned long long cond;  // conditional-node handle (0 = host-driven loop)
};

// ---------------------------------------------------------------------------
// Tile loaders
// ---------------------------------------------------------------------------

template <class T> __device__ __forceinline__ float tof(T v) { return Cvt<T>::to_f(v); }

// Programmatic dependent launch: every kernel of the solve is launched with
// programmatic stream serialisation, lets its successor start launching at
// once, and waits for its predecessor's completion (and memory) before its
// first access.  This hides the launch gap between the many short kernels of
// a V-cycle.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter()
{
    pdl_wait();
    pdl_trigger();
}

// Plane tile: NP planes x ROWS rows (y0 - 2 .. y0 + ROWS - 3) x kPW columns
// starting at x0 - 8 (16-byte aligned: x0 is a multiple of 64 and P of 8).
// Elements outside the W x H level read as zero.  Every thread issues all of
// its 16-byte loads before the first shared-memory store, so a tile's loads
// are in flight together.
template <class T, int NP, int ROWS>
__device__ __forceinline__ void load_planes(T* sm, const T* g, size_t ps, int P, int W, int H, int x0, int y0)
{
    constexpr int EPV = 16 / sizeof(T);
    constexpr int VPR = kPW / EPV;
    constexpr int TOTAL = NP * ROWS * VPR;
    constexpr int ITER = (TOTAL + kThreads - 1) / kThreads;
    constexpr int CH = 6;  // loads in flight per thread (registers: 4 per load)
#pragma unroll
    for (int j0 = 0; j0 < ITER; j0 += CH) {
        uint4 val[CH];
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const int i = threadIdx.x + (j0 + j) * kThreads;
            const int v = i % VPR, r = (i / VPR) % ROWS, k = i / (VPR * ROWS);
            const int gx = x0 - 8 + v * EPV, gy = y0 - kHalo + r;
            val[j] = make_uint4(0u, 0u, 0u, 0u);
            if (j0 + j < ITER && i < TOTAL && gy >= 0 && gy < H && gx >= 0 && gx < W)
                val[j] = __ldg(reinterpret_cast<const uint4*>(g + (size_t)k * ps + (size_t)gy * P + gx));
        }
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const int i = threadIdx.x + (j0 + j) * kThreads;
            if (j0 + j < ITER && i < TOTAL) {
                const int v = i % VPR;
                const int gx = x0 - 8 + v * EPV;
                T* dst = sm + (size_t)(i / VPR) * kPW + v * EPV;
                *reinterpret_cast<uint4*>(dst) = val[j];
                if (gx + EPV > W && gx < W) {
                    for (int e = W - gx; e < EPV; ++e) dst[e] = T(0.0f);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Deterministic grid reductions: each CTA publishes its partial sums, the
// last CTA to arrive adds all partials in index order.
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ bool last_cta_total(double (&v)[NV], double* parts, unsigned* ticket)
{
    __shared__ double red[32 * NV + NV];
    __shared__ int s_last;
    block_sum<NV>(v, red);
    const unsigned G = gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) parts[(size_t)k * kMaxParts + blockIdx.x] = v[k];
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        s_last = (t == G - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (wid < NV) {
        const double t = warp_sum_range(parts + (size_t)wid * kMaxParts, 0, (int)G);
        if (lane == 0) red[32 * NV + wid] = t;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = red[32 * NV + k];
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

__device__ __forceinline__ void set_cond(const Args& a, unsigned v)
{
    if (a.cond) cudaGraphSetConditional((cudaGraphConditionalHandle)a.cond, v);
}

// The smoother steps written with 1 / D only.  With S = sum_j w_ij v_j, so
// that (A v)_i = D_i v_i - S_i, and x1 = omega b / D:
//   rho = b - A x1 = (1 - omega) b + S(x1)            (D > 0; rho = b + S if D = 0)
//   x = y + omega (b - A y) / D = (1 - omega) y + omega (b + S(y)) / D
__device__ __forceinline__ float rho_of(float b, float di, float om, float S)
{
    return (di > 0.f ? (1.f - om) * b : b) + S;
}
__device__ __forceinline__ float smooth_of(float y, float b, float di, float om, float S)
{
    return di > 0.f ? fmaf(om * di, b + S, (1.f - om) * y) : y;
}

// ---------------------------------------------------------------------------
// Outer PCG kernels (level 0)
// ---------------------------------------------------------------------------

// x += alpha p_new, r -= alpha q, partial r . r; the last CTA counts the
// iteration and asks for a true-residual replacement when it is due.  Four
// pixels per step (16-byte vectors; the pitch is a multiple of 8); lanes past
// W are written as zero and left out of the sum.
__global__ void __launch_bounds__(kThreads) mg_update_kernel(Args a)
{
    pdl_enter();
    State* st = a.st;
    if (st->done) return;
    const int W = a.W, H = a.H, P = a.P;
    const int it = st->iter;
    const double al = st->alpha;
    const float alf = (float)al;
    const float* pn = (it & 1) ? a.p0 : a.p1;
    const bool fold = st->fold_at == it;  // a replacement ran: move the increment into x
    double acc = 0.0;
    const int qpr = (W + 3) / 4;
    const size_t nq = (size_t)qpr * H;
    for (size_t qi = (size_t)blockIdx.x * kThreads + threadIdx.x; qi < nq; qi += (size_t)gridDim.x * kThreads) {
        const int y = (int)(qi / qpr), x = (int)(qi % qpr) * 4;
        const size_t o = (size_t)y * P + x;
        const float4 p = *reinterpret_cast<const float4*>(pn + o);
        const float4 q = *reinterpret_cast<const float4*>(a.q + o);
        float4 r = *reinterpret_cast<const float4*>(a.r + o);
        float4 xi = *reinterpret_cast<const float4*>(a.xinc + o);
        const bool v1 = x + 1 < W, v2 = x + 2 < W, v3 = x + 3 < W;
        if (fold) {
            double2 x01 = *reinterpret_cast<const double2*>(a.x + o);
            double2 x23 = *reinterpret_cast<const double2*>(a.x + o + 2);
            x01.x += (double)xi.x;
            x01.y = v1 ? x01.y + (double)xi.y : 0.0;
            x23.x = v2 ? x23.x + (double)xi.z : 0.0;
            x23.y = v3 ? x23.y + (double)xi.w : 0.0;
            *reinterpret_cast<double2*>(a.x + o) = x01;
            *reinterpret_cast<double2*>(a.x + o + 2) = x23;
            xi = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        xi.x = fmaf(alf, p.x, xi.x);
        xi.y = v1 ? fmaf(alf, p.y, xi.y) : 0.f;
        xi.z = v2 ? fmaf(alf, p.z, xi.z) : 0.f;
        xi.w = v3 ? fmaf(alf, p.w, xi.w) : 0.f;
        r.x = fmaf(-alf, q.x, r.x);
        r.y = v1 ? fmaf(-alf, q.y, r.y) : 0.f;
        r.z = v2 ? fmaf(-alf, q.z, r.z) : 0.f;
        r.w = v3 ? fmaf(-alf, q.w, r.w) : 0.f;
        *reinterpret_cast<float4*>(a.xinc + o) = xi;
        *reinterpret_cast<float4*>(a.r + o) = r;
        acc += (double)r.x * r.x + (double)r.y * r.y + ((double)r.z * r.z + (double)r.w * r.w);
    }
    double v[1] = {acc};
    if (last_cta_total<1>(v, a.parts + kMaxParts, &st->ticket[T_RR]) && threadIdx.x == 0) {
        const int k = it + 1;
        st->iter = k;
        st->rr = v[0];
        const bool conv = a.rtol > 0.0 && v[0] <= a.rtol * a.rtol * st->bn2;
        if (conv || (a.replace_every > 0 && k % a.replace_every == 0) || k >= a.max_iters || !isfinite(v[0]))
            st->need_replace = 1;
    }
}

// True residual r = b - A x with the FP32 planes in FP64 arithmetic (runs
// only when a replacement is due).  Also forms ||b||^2 on the first call.
__global__ void __launch_bounds__(kThreads, 3) mg_replace_kernel(Args a)
{
    pdl_enter();
    State* st = a.st;
    if (st->done || !st->need_replace) return;
    extern __shared__ __align__(16) unsigned char smem[];
    float* pt = reinterpret_cast<float*>(smem);
    double* xt = reinterpret_cast<double*>(smem + sizeof(float) * FineSten::NP * (kTY + kHalo) * kPW);
    const int W = a.W, H = a.H, P = a.P;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int tiles_x = (W + kTX - 1) / kTX, tiles = tiles_x * ((H + kTY - 1) / kTY);
    double rr = 0.0, bb = 0.0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int x0 = (t % tiles_x) * kTX, y0 = (t / tiles_x) * kTY;
        __syncthreads();
        load_planes<float, FineSten::NP, kTY + kHalo>(pt, a.w32, a.ps32, P, W, H, x0, y0);
        constexpr int XT = (kTY + 2 * kHalo) * kVW, XI = (XT + kThreads - 1) / kThreads;
        double xv[XI];
#pragma unroll
        for (int j = 0; j < XI; ++j) {
            const int i = threadIdx.x + j * kThreads;
            const int gx = x0 - kHalo + i % kVW, gy = y0 - kHalo + i / kVW;
            const size_t o = (size_t)gy * P + gx;
            xv[j] = (i < XT && gx >= 0 && gx < W && gy >= 0 && gy < H) ? a.x[o] + (double)a.xinc[o] : 0.0;
        }
#pragma unroll
        for (int j = 0; j < XI; ++j) {
            const int i = threadIdx.x + j * kThreads;
            if (i < XT) xt[i] = xv[j];
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int lx = tx + 32 * h, gx = x0 + lx, gy = y0 + ty;
            if (gx < W && gy < H) {
                const size_t o = (size_t)gy * P + gx;
                const int vc = (ty + kHalo) * kVW + lx + kHalo;
                const double xc = xt[vc];
                double y = (double)a.gamma[o] * xc;
#pragma unroll
                for (int k = 0; k < FineSten::NP; ++k) {
                    const int du = FineSten::du(k), dv = FineSten::dv(k);
                    const double wu = pt[((size_t)k * (kTY + kHalo) + ty + kHalo) * kPW + lx + 8];
                    const double wl = pt[((size_t)k * (kTY + kHalo) + ty + kHalo - dv) * kPW + lx + 8 - du];
                    y += wu * (xc - xt[vc + dv * kVW + du]) + wl * (xc - xt[vc - dv * kVW - du]);
                }
                const double bv = a.bvec[(size_t)gy * a.bpitch + gx];
                const double r = bv - y;
                a.r[o] = (float)r;
                rr += r * r;
                bb += bv * bv;
            }
        }
    }
    double v[2] = {rr, bb};
    if (last_cta_total<2>(v, a.parts + 2 * kMaxParts, &st->ticket[T_TRUE]) && threadIdx.x == 0) {
        if (st->replacements == 0) st->bn2 = v[1];
        st->replacements += 1;
        st->fold_at = st->iter;
        st->need_replace = 0;
        // A true residual well above the recurrence's (more than twice its
        // norm) means the FP32 recurrences drifted: from a zero guess the
        // first cycle can carry the whole solution in the FP32 increment.
        // The old direction is then conjugate to a residual that no longer
        // exists, and beta = true r.z / recurrence r.z would let it swamp
        // the new one (the iteration stalls), so the next direction restarts
        // from z.  Forward solves never open such a gap.
        st->restart = v[0] > 4.0 * st->rr;
        st->rr_true = v[0];
        st->rr = v[0];
        const double bn2 = st->bn2;
        if (!(bn2 > 0.0)) {
            st->done = 1;          // b = 0: the solution is 0
            st->status = GM_OK;
        } else if (!isfinite(v[0])) {
            st->done = 1;
            st->status = GM_ERR_BREAKDOWN;
        } else if (a.rtol > 0.0 && v[0] <= a.rtol * a.rtol * bn2) {
            st->done = 1;
            st->status = GM_OK;
        } else if (st->iter >= a.max_iters) {
            st->done = 1;
            st->status = a.rtol > 0.0 ? GM_ERR_NOT_CONVERGED : GM_OK;
        }
    }
}

// ---------------------------------------------------------------------------
// V-cycle kernels
// ---------------------------------------------------------------------------

// The small levels lt .. L of a V-cycle in ONE CTA: their operators and
// vectors are staged in shared memory (compact [H_l][W_l] arrays) and the
// phases (smoothing + restriction down to the coarsest level, the exact
// coarsest solve with the stored FP64 inverse, prolongation + smoothing back
// up) are separated by block barriers instead of kernel launches.  Reads
// b_lt, writes x_lt.
constexpr int kTailThreads = 1024;
constexpr int kTailSmem = 160 * 1024;

__device__ __forceinline__ float tail_sum(const float* c, const float* v, int W, int H, int n, int x, int y)
{
    const int i = y * W + x;
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int du = CoarseSten::du(k), dv = CoarseSten::dv(k);
        const int xu = x + du, yu = y + dv, xl = x - du, yl = y - dv;
        if (xu >= 0 && xu < W && yu < H) s = fmaf(c[k * n + i], v[yu * W + xu], s);
        if (xl >= 0 && xl < W && yl >= 0) s = fmaf(c[k * n + yl * W + xl], v[yl * W + xl], s);
    }
    return s;
}

__global__ void __launch_bounds__(kTailThreads) mg_tail_kernel(Args a)
{
    // The levels' operators and the coarsest inverse were written by the
    // set-up kernels, which completed before this kernel's predecessor
    // started (every other kernel waits before it triggers), so they are
    // staged before the wait, overlapping the predecessor; b_lt after it.
    pdl_trigger();
    extern __shared__ __align__(16) float sh[];
    const int lt = a.lt, L = a.L, tid = threadIdx.x;
    const float om = a.omega, sc = a.scale;
    // carve: per level c[4n], 1/D [n], b[n], x[n]; then tmp[n_lt]; then the
    // coarsest inverse (FP64, rounded up to an 8-byte boundary)
    auto base = [&](int l) {
        int off = 0;
        for (int m = lt; m < l; ++m) off += 7 * a.lev[m].W * a.lev[m].H;
        return sh + off;
    };
    float* tmp = base(L + 1);
    const int nL = a.lev[L].W * a.lev[L].H;
    double* minv = reinterpret_cast<double*>(sh + ((int)(tmp - sh) + a.lev[lt].W * a.lev[lt].H + 1) / 2 * 2);
    for (int l = lt; l <= L; ++l) {
        const Lev& G = a.lev[l];
        const int W = G.W, n = G.W * G.H;
        float* c = base(l);
        float* D = c + 4 * n;
        const float* gc = static_cast<const float*>(G.c);
        for (int i = tid; i < n; i += kTailThreads) {
            const size_t g = (size_t)(i / W) * G.P + i % W;
#pragma unroll
            for (int k = 0; k < 4; ++k) c[k * n + i] = gc[(size_t)k * G.ps + g];
            D[i] = G.Di[g];
        }
    }
    for (int i = tid; i < nL * nL; i += kTailThreads) minv[i] = a.minv[i];
    pdl_wait();
    if (a.st->done) return;
    {
        const Lev& G = a.lev[lt];
        const int n = G.W * G.H;
        float* b = base(lt) + 5 * n;
        for (int i = tid; i < n; i += kTailThreads) b[i] = G.b[(size_t)(i / G.W) * G.P + i % G.W];
    }
    __syncthreads();
    for (int l = lt; l < L; ++l) {
        const Lev& F = a.lev[l];
        const Lev& Cl = a.lev[l + 1];
        const int W = F.W, H = F.H, n = W * H;
        float* c = base(l);
        float* D = c + 4 * n;
        float* b = D + n;
        float* x = b + n;
        for (int i = tid; i < n; i += kTailThreads) x[i] = om * b[i] * D[i];
        __syncthreads();
        float* bc = base(l + 1) + 5 * Cl.W * Cl.H;
        for (int I = tid; I < Cl.W * Cl.H; I += kTailThreads) {
            const int X = I % Cl.W, Y = I / Cl.W;
            float sum = 0.f;
            for (int q = 0; q < 4; ++q) {
                const int xf = 2 * X + (q & 1), yf = 2 * Y + (q >> 1);
                if (xf < W && yf < H) {
                    const int i = yf * W + xf;
                    sum += rho_of(b[i], D[i], om, tail_sum(c, x, W, H, n, xf, yf));
                }
            }
            bc[I] = sum;
        }
        __syncthreads();
    }
    {
        const Lev& G = a.lev[L];
        const int n = G.W * G.H;
        float* b = base(L) + 5 * n;
        float* x = b + n;
        for (int i = tid; i < n; i += kTailThreads) {
            double s = 0.0;
#pragma unroll 8
            for (int j = 0; j < n; ++j) s += minv[j * n + i] * (double)b[j];
            x[i] = (float)s;
        }
        __syncthreads();
    }
    for (int l = L - 1; l >= lt; --l) {
        const Lev& F = a.lev[l];
        const Lev& Cl = a.lev[l + 1];
        const int W = F.W, H = F.H, n = W * H;
        float* c = base(l);
        float* D = c + 4 * n;
        float* b = D + n;
        float* x = b + n;
        const float* xc = base(l + 1) + 6 * Cl.W * Cl.H;
        for (int i = tid; i < n; i += kTailThreads) {
            const int xf = i % W, yf = i / W;
            x[i] = fmaf(sc, xc[(yf >> 1) * Cl.W + (xf >> 1)], om * b[i] * D[i]);
        }
        __syncthreads();
        for (int i = tid; i < n; i += kTailThreads) {
            tmp[i] = smooth_of(x[i], b[i], D[i], om, tail_sum(c, x, W, H, n, i % W, i / W));
        }
        __syncthreads();
        for (int i = tid; i < n; i += kTailThreads) x[i] = tmp[i];
        __syncthreads();
    }
    {
        const Lev& G = a.lev[lt];
        const int n = G.W * G.H;
        const float* x = base(lt) + 6 * n;
        for (int i = tid; i < n; i += kTailThreads) G.x[(size_t)(i / G.W) * G.P + i % G.W] = x[i];
    }
}

// Shared-memory bytes of the tail kernel for levels lt .. L.
static int tail_bytes(const int* Wl, const int* Hl, int lt, int L)
{
    long long f = 0;
    for (int l = lt; l <= L; ++l) f += 7LL * Wl[l] * Hl[l];
    f += (long long)Wl[lt] * Hl[lt];
    f = (f + 1) / 2 * 2;                        // the FP64 inverse starts 8-byte aligned
    f += 2LL * Wl[L] * Hl[L] * Wl[L] * Hl[L];
    return (int)(f * 4);
}

// ---------------------------------------------------------------------------
// Level-0 kernels: persistent CTAs streaming 128-column tiles through a
// two-stage TMA ring (the pattern of the standalone SpMV).  One elected
// thread issues, per tile, a 3-D box {144, TH + 2, 12} of the affinity planes
// (8 columns each side so the box starts on a 16-byte boundary, 2 rows above
// for the mirrored couplings) and 2-D boxes {144, TH + 4} of the vectors the
// stencil input is made of; TMA's zero fill stands in for everything outside
// the image.  After a stage lands, the CTA forms the stencil input in a
// shared tile, then each thread marches TH / 4 rows of a column pair with a
// 5 x 6 window of it in registers.
//   FM_SPMV  input z + beta p_old; q = A p_new with the FP32 planes and d32
//            (FP16 planes and d when Args::outer_low);
//            writes p_new and q, sums p_new . q (the last CTA forms alpha).
//   FM_DOWN  input x1 = omega b / d; rho = b - A x1, summed over 2 x 2 blocks
//            into the level-1 right-hand side.
//   FM_UP    input y = x1 + scale x_1[aggregate]; z = y + omega (b - A y) / d,
//            sums r . z (the last CTA forms beta and the loop condition).
// ---------------------------------------------------------------------------
enum { FM_SPMV = 0, FM_DOWN = 1, FM_UP = 2 };
constexpr int kFTW = 128;             // output columns per tile
constexpr int kFBW = kFTW + 16;       // box width
constexpr int kXBW = kFTW / 2 + 8;    // coarse box width (FM_UP)

// SPMV: m[0] w32 planes, m[1] z, m[2] p0, m[3] p1, m[4] d32 (tile rows only)
// DOWN: m[0] iteration planes, m[1] r, m[2] d
// UP:   m[0] iteration planes, m[1] r, m[2] d, m[3] level-1 x
struct TMaps {
    CUtensorMap m[5];
};

__host__ __device__ constexpr int fine_rows(int esize) { return esize == 2 ? 16 : 8; }
__host__ __device__ constexpr int b128(int x) { return (x + 127) & ~127; }

template <int MODE, int ES, int NP = 12>
struct FineLayout {
    static constexpr int TH = fine_rows(ES);
    static constexpr int THR = ES == 2 ? 512 : 256;  // threads: 64 column pairs x TH / 2 row pairs
    static constexpr int PB = NP * (TH + 2) * kFBW * ES;
    static constexpr int VB = (TH + 4) * kFBW * 4;
    static constexpr int XB = MODE == FM_UP ? (TH / 2 + 2) * kXBW * 4 : 0;
    static constexpr int DB = MODE == FM_SPMV ? TH * kFTW * 4 : 0;
    static constexpr int v0_off = b128(PB);
    static constexpr int v1_off = v0_off + b128(VB);
    static constexpr int x_off = v1_off + b128(VB);
    static constexpr int d_off = x_off + b128(XB);
    static constexpr int stage = d_off + b128(DB);
    static constexpr int vt_off = 2 * stage;
    static constexpr int bar_off = vt_off + b128(VB);
    static constexpr int total = bar_off + 64 + 128;  // + room to align the base to 128 bytes
    static constexpr uint32_t bytes = (uint32_t)(PB + 2 * VB + XB + DB);
};

// Element type of the planes a level-0 kernel streams: the iteration planes.
// The SpMV of a BF16 store reads the FP32 planes instead (a BF16 outer
// operator costs more iterations than its bytes save); so does an FP16
// store's when the tolerance is tight (Args::outer_low = 0), through the
// float instantiation.
template <int MODE, class T>
struct FinePlanes {
    using PT = typename std::conditional<MODE == FM_SPMV && !std::is_same<T, __half>::value, float, T>::type;
    static constexpr int ES = (int)sizeof(PT);
};

template <class T> __device__ __forceinline__ float2 ld2(const T* p);
template <> __device__ __forceinline__ float2 ld2<float>(const float* p) { return *reinterpret_cast<const float2*>(p); }
template <> __device__ __forceinline__ float2 ld2<__half>(const __half* p)
{
    return __half22float2(*reinterpret_cast<const __half2*>(p));
}
template <> __device__ __forceinline__ float2 ld2<__nv_bfloat16>(const __nv_bfloat16* p)
{
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}

// Adds expected TMA bytes to the current phase without arriving; and a plain
// arrival (the phase completes once its bytes have landed).
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive_only(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Waits for a TMA stage with a wall-clock limit (2 s); on expiry the solve
// ends with GM_ERR_TIMEOUT.
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t parity, State* st)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    unsigned spins = 0;
    while (!mbar_try_wait_hint(bar, parity, 100000u)) {
        if ((++spins & 15u) == 0 && globaltimer_ns() - t0 > 2000000000ull) {
            atomicCAS(&st->status, (int)GM_OK, (int)GM_ERR_TIMEOUT);
            st->done = 1;
            return false;
        }
    }
    return true;
}

template <int MODE, class S, class T>
__global__ void __launch_bounds__(FineLayout<MODE, FinePlanes<MODE, T>::ES, S::NP>::THR, 1)
    mg_fine_kernel(const __grid_constant__ TMaps tm, Args a, int l)
{
    constexpr int ES = FinePlanes<MODE, T>::ES;
    using PT = typename FinePlanes<MODE, T>::PT;
    using LY = FineLayout<MODE, ES, S::NP>;
    constexpr int TH = LY::TH, NT = LY::THR, RPT = TH / (NT / 64);
    static_assert(RPT == 2, "each thread covers one row pair");
    constexpr int PW = (TH + 2) * kFBW;  // elements per plane in the box
    // TMA destinations must be 128-byte aligned; the dynamic region follows
    // the reduction's static shared memory, so align its base by hand.
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + LY::bar_off);
    float* vt = reinterpret_cast<float*>(smem + LY::vt_off);
    const Lev& F = a.lev[l];
    const int W = F.W, H = F.H, P = F.P, tid = threadIdx.x, G = gridDim.x;
    const int ntx = (W + kFTW - 1) / kFTW, ntiles = ntx * ((H + TH - 1) / TH);
    const int t0 = blockIdx.x;
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue_planes = [&](int t, int s) {
        const int u0 = (t % ntx) * kFTW, v0 = (t / ntx) * TH;
        tma_load_3d(smem + s * LY::stage, &tm.m[0], u0 - 8, v0 - 2, 0, &full[s]);
    };
    // The planes are constant during a solve (written by the store's assembly
    // or the set-up kernels, which completed before this kernel's predecessor
    // began), so the first two stages' plane boxes are requested before the
    // wait for the predecessor; the stage's arrival comes with the vectors.
    const int npre = (t0 < ntiles ? 1 : 0) + (t0 + G < ntiles ? 1 : 0);
    if (tid == 0)
        for (int k = 0; k < npre; ++k) {
            mbar_expect_tx(&full[k], (uint32_t)LY::PB);
            issue_planes(t0 + k * G, k);
        }
    pdl_enter();
    State* st = a.st;
    if (st->done) {
        if (MODE == FM_UP && blockIdx.x == 0 && threadIdx.x == 0) set_cond(a, 0u);
        // complete the stages with no vectors and let the plane loads land
        if (tid == 0)
            for (int k = 0; k < npre; ++k) mbar_arrive_only(&full[k]);
        for (int k = 0; k < npre; ++k) stage_wait(&full[k], 0u, st);
        return;
    }
    const int it = st->iter;
    const bool first = it == 0;
    const float beta = (float)st->beta, om = a.omega, sc = a.scale;
    const CUtensorMap* mv1 = MODE == FM_SPMV ? ((it & 1) ? &tm.m[3] : &tm.m[2]) : &tm.m[2];
    float* pnew = (it & 1) ? a.p0 : a.p1;
    const Lev& C = a.lev[l + 1];
    auto issue_vectors = [&](int t, int s) {
        const int u0 = (t % ntx) * kFTW, v0 = (t / ntx) * TH;
        unsigned char* sp = smem + s * LY::stage;
        tma_load_2d(sp + LY::v0_off, &tm.m[1], u0 - 8, v0 - 2, &full[s]);
        tma_load_2d(sp + LY::v1_off, mv1, u0 - 8, v0 - 2, &full[s]);
        if (MODE == FM_UP) tma_load_2d(sp + LY::x_off, &tm.m[3], u0 / 2 - 4, v0 / 2 - 1, &full[s]);
        if (MODE == FM_SPMV) tma_load_2d(sp + LY::d_off, &tm.m[4], u0, v0, &full[s]);
    };
    auto issue = [&](int t, int s) {
        mbar_arrive_expect_tx(&full[s], LY::bytes);
        issue_planes(t, s);
        issue_vectors(t, s);
    };
    if (tid == 0)
        for (int k = 0; k < npre; ++k) {
            mbar_arrive_expect_tx(&full[k], LY::bytes - (uint32_t)LY::PB);
            issue_vectors(t0 + k * G, k);
        }
    const int cp = tid & 63, rg = tid >> 6;
    const int lu = 8 + 2 * cp;
    const int r0 = rg * RPT;
    double acc = 0.0;
    int s = 0;
    uint32_t phase = 0u;
    bool ok = true;
    for (int t = t0; t < ntiles; t += G) {
        if (!stage_wait(&full[s], (phase >> s) & 1u, st)) { ok = false; break; }
        phase ^= 1u << s;
        const unsigned char* sp = smem + s * LY::stage;
        const PT* wb = reinterpret_cast<const PT*>(sp);
        const float* v0b = reinterpret_cast<const float*>(sp + LY::v0_off);
        const float* v1b = reinterpret_cast<const float*>(sp + LY::v1_off);
        const int u0 = (t % ntx) * kFTW, v0 = (t / ntx) * TH;
        // stencil input tile
        for (int i = tid; i < (TH + 4) * kFBW; i += NT) {
            float v;
            if (MODE == FM_SPMV) {
                v = first ? v0b[i] : fmaf(beta, v1b[i], v0b[i]);
            } else {
                v = om * v0b[i] * v1b[i];  // x1 = omega b / d (v1 holds 1 / d)
                if (MODE == FM_UP) {
                    // 1/d is zero outside the image (zero fill) and on pixels
                    // with no coupling and no scribble: y = 0 there
                    const int row = i / kFBW, col = i - row * kFBW;
                    const float* xb = reinterpret_cast<const float*>(sp + LY::x_off);
                    v = v1b[i] > 0.f ? fmaf(sc, xb[(row >> 1) * kXBW + (col >> 1)], v) : 0.f;
                }
            }
            vt[i] = v;
        }
        __syncthreads();
        float xw[5][6];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float* xr = vt + (r0 + j) * kFBW + lu - 2;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float2 q = *reinterpret_cast<const float2*>(xr + 2 * c);
                xw[j + 1][2 * c] = q.x;
                xw[j + 1][2 * c + 1] = q.y;
            }
        }
        float cs = 0.f;  // FM_DOWN: 2 x 2 block sum
#pragma unroll
        for (int rr = 0; rr < RPT; ++rr) {
            const int r = r0 + rr;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int c = 0; c < 6; ++c) xw[j][c] = xw[j + 1][c];
            {
                const float* xr = vt + (r + 4) * kFBW + lu - 2;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float2 q = *reinterpret_cast<const float2*>(xr + 2 * c);
                    xw[4][2 * c] = q.x;
                    xw[4][2 * c + 1] = q.y;
                }
            }
            const float xi0 = xw[2][2], xi1 = xw[2][3];
            // S = sum_j w_ij x_j, two chains per pixel
            float a0[2] = {0.f, 0.f}, a1[2] = {0.f, 0.f};
#pragma unroll
            for (int k = 0; k < S::NP; ++k) {
                const int dv = S::dv(k), du = S::du(k);
                const PT* pk = wb + k * PW;
                const float2 wo = ld2<PT>(pk + (r + 2) * kFBW + lu);
                const PT* pm = pk + (r + 2 - dv) * kFBW + lu - du;
                const float wm0 = tof(pm[0]), wm1 = tof(pm[1]);
                a0[k & 1] = fmaf(wo.x, xw[2 + dv][2 + du], a0[k & 1]);
                a1[k & 1] = fmaf(wo.y, xw[2 + dv][3 + du], a1[k & 1]);
                a0[k & 1] = fmaf(wm0, xw[2 - dv][2 - du], a0[k & 1]);
                a1[k & 1] = fmaf(wm1, xw[2 - dv][3 - du], a1[k & 1]);
            }
            const float S0 = a0[0] + a0[1], S1 = a1[0] + a1[1];
            const int u = u0 + 2 * cp, v = v0 + r;
            if (MODE == FM_SPMV) {
                const float2 dg = *reinterpret_cast<const float2*>(sp + LY::d_off + (size_t)(r * kFTW + 2 * cp) * 4);
                const float q0 = fmaf(dg.x, xi0, -S0), q1 = fmaf(dg.y, xi1, -S1);
                if (v < H) {
                    const size_t o = (size_t)v * P + u;
                    if (u + 1 < W) {
                        *reinterpret_cast<float2*>(pnew + o) = make_float2(xi0, xi1);
                        *reinterpret_cast<float2*>(a.q + o) = make_float2(q0, q1);
                        acc += (double)xi0 * q0 + (double)xi1 * q1;
                    } else if (u < W) {
                        pnew[o] = xi0;
                        a.q[o] = q0;
                        acc += (double)xi0 * q0;
                    }
                }
            } else {
                const float2 bb = *reinterpret_cast<const float2*>(v0b + (r + 2) * kFBW + lu);
                const float2 dd = *reinterpret_cast<const float2*>(v1b + (r + 2) * kFBW + lu);  // 1 / d
                if (MODE == FM_DOWN) {
                    // rho = b - A x1; zero outside the image (zero fill)
                    cs += rho_of(bb.x, dd.x, om, S0) + rho_of(bb.y, dd.y, om, S1);
                    if (rr & 1) {
                        const int X = (u0 >> 1) + cp, Y = v >> 1;
                        if (X < C.W && Y < C.H) C.b[(size_t)Y * C.P + X] = cs;
                        cs = 0.f;
                    }
                } else {
                    const float z0 = smooth_of(xi0, bb.x, dd.x, om, S0);
                    const float z1 = smooth_of(xi1, bb.y, dd.y, om, S1);
                    if (v < H) {
                        float* zr = F.x + (size_t)v * P + u;
                        if (u + 1 < W) {
                            *reinterpret_cast<float2*>(zr) = make_float2(z0, z1);
                            acc += (double)bb.x * z0 + (double)bb.y * z1;
                        } else if (u < W) {
                            *zr = z0;
                            acc += (double)bb.x * z0;
                        }
                    }
                }
            }
        }
        __syncthreads();  // every thread is done with stage s and the input tile
        if (tid == 0 && t + 2 * G < ntiles) issue(t + 2 * G, s);
        s ^= 1;
    }
    if (!ok) return;
    static_assert(NT <= 1024, "");
    if (MODE == FM_SPMV) {
        double v[1] = {acc};
        if (last_cta_total<1>(v, a.parts, &st->ticket[T_PQ]) && threadIdx.x == 0) {
            st->pq = v[0];
            if (!(v[0] > 0.0) || !isfinite(v[0]) || !isfinite(st->rz)) {
                st->status = GM_ERR_BREAKDOWN;
                st->done = 1;
            } else {
                st->alpha = st->rz / v[0];
            }
        }
    } else if (MODE == FM_UP && l == 0) {
        double v[1] = {acc};
        if (last_cta_total<1>(v, a.parts + 4 * kMaxParts, &st->ticket[T_RZ]) && threadIdx.x == 0) {
            const double rz = v[0];
            if (st->iter > 0) st->beta = st->restart ? 0.0 : rz / st->rz;
            st->restart = 0;
            st->rz = rz;
            if (!isfinite(rz)) {
                st->status = GM_ERR_BREAKDOWN;
                st->done = 1;
            }
            const bool go = !st->done && st->iter < a.max_iters + 1;
            set_cond(a, go ? 1u : 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// Set-up kernels
// ---------------------------------------------------------------------------

// Galerkin coarsening of level l into l+1, one thread per coarse cell: the
// couplings of the cell's (up to 4) fine cells in both directions are
// summed per neighbouring aggregate (FP64), in a fixed order.
template <class S, class T>
__global__ void mg_build_kernel(Args a, int l, const float* fine_gamma, int gpitch)
{
    pdl_enter();
    const Lev& F = a.lev[l];
    const Lev& C = a.lev[l + 1];
    const T* w = static_cast<const T*>(F.c);
    const int n = C.W * C.H;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int X = i % C.W, Y = i / C.W;
        double c[4] = {0.0, 0.0, 0.0, 0.0};
        double ext = 0.0, gam = 0.0;
        for (int bq = 0; bq < 2; ++bq)
            for (int aq = 0; aq < 2; ++aq) {
                const int x = 2 * X + aq, y = 2 * Y + bq;
                if (x >= F.W || y >= F.H) continue;
                gam += fine_gamma[(size_t)y * gpitch + x];
                for (int k = 0; k < S::NP; ++k)
                    for (int dir = 0; dir < 2; ++dir) {
                        const int du = dir ? -S::du(k) : S::du(k), dv = dir ? -S::dv(k) : S::dv(k);
                        const int xj = x + du, yj = y + dv;
                        if (xj < 0 || xj >= F.W || yj < 0 || yj >= F.H) continue;
                        // the coupling is stored at the upper end of the pair
                        const int xs = dir ? xj : x, ys = dir ? yj : y;
                        const double wv = tof(w[(size_t)k * F.ps + (size_t)ys * F.P + xs]);
                        const int ox = (xj >> 1) - X, oy = (yj >> 1) - Y;
                        if (ox == 0 && oy == 0) continue;
                        ext += wv;
                        for (int o = 0; o < 4; ++o)
                            if (ox == CoarseSten::du(o) && oy == CoarseSten::dv(o)) c[o] += wv;
                    }
            }
        const size_t oc = (size_t)Y * C.P + X;
        float* cp = static_cast<float*>(C.c);
        for (int o = 0; o < 4; ++o) cp[(size_t)o * C.ps + oc] = (float)c[o];
        C.gam[oc] = (float)gam;
        C.D[oc] = (float)(gam + ext);
        C.Di[oc] = gam + ext > 0.0 ? (float)(1.0 / (gam + ext)) : 0.f;
    }
}

// Dense FP64 inverse of the coarsest operator by in-place Gauss-Jordan
// elimination (SPD: no pivoting), one CTA, matrix in shared memory.
__global__ void __launch_bounds__(kThreads) mg_inverse_kernel(Args a)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem[];
    const Lev& C = a.lev[a.L];
    const int n = C.W * C.H;
    double* A = reinterpret_cast<double*>(smem);
    double* row = A + (size_t)n * n;
    double* col = row + kCoarseMax;
    __shared__ int s_bad;
    for (int i = threadIdx.x; i < n * n; i += kThreads) A[i] = 0.0;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const float* cp = static_cast<const float*>(C.c);
    for (int I = threadIdx.x; I < n; I += kThreads) {
        const int X = I % C.W, Y = I / C.W;
        const size_t o = (size_t)Y * C.P + X;
        A[(size_t)I * n + I] = C.D[o];
        for (int k = 0; k < 4; ++k) {
            const int Xj = X + CoarseSten::du(k), Yj = Y + CoarseSten::dv(k);
            if (Xj < 0 || Xj >= C.W || Yj >= C.H) continue;
            const int J = Yj * C.W + Xj;
            const double v = -(double)cp[(size_t)k * C.ps + o];
            A[(size_t)I * n + J] = v;
            A[(size_t)J * n + I] = v;
        }
    }
    __syncthreads();
    // Zero rows (aggregates with no coupling and no scribble weight, as in
    // images less than 3 pixels wide or tall, where no 3x3 window exists) are
    // left out: for a positive semidefinite matrix a zero pivot means a zero
    // row and column, and the inverse on the remaining rows is exact.
    double dmax = 0.0;
    for (int i = 0; i < n; ++i) dmax = fmax(dmax, A[(size_t)i * n + i]);
    for (int k = 0; k < n; ++k) {
        const double piv = A[(size_t)k * n + k];
        if (!isfinite(piv) || piv < 0.0) {
            if (threadIdx.x == 0) s_bad = 1;
            break;
        }
        if (piv <= 1e-300 + 1e-14 * dmax) {
            for (int j = threadIdx.x; j < n; j += kThreads) {
                A[(size_t)k * n + j] = 0.0;
                A[(size_t)j * n + k] = 0.0;
            }
            __syncthreads();
            continue;
        }
        const double inv = 1.0 / piv;
        for (int j = threadIdx.x; j < n; j += kThreads) {
            row[j] = A[(size_t)k * n + j] * inv;
            col[j] = A[(size_t)j * n + k];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < n * n; e += kThreads) {
            const int i = e / n, j = e % n;
            double v;
            if (i == k && j == k) v = inv;
            else if (i == k) v = row[j];
            else if (j == k) v = -col[i] * inv;
            else v = A[e] - col[i] * row[j];
            A[e] = v;
        }
        __syncthreads();
    }
    __syncthreads();
    if (s_bad) {
        if (threadIdx.x == 0) {
            a.st->status = GM_ERR_BREAKDOWN;
            a.st->done = 1;
        }
        return;
    }
    for (int e = threadIdx.x; e < n * n; e += kThreads) a.minv[e] = A[e];
}

// 1 / d of the level-0 iteration diagonal (0 where d = 0).
__global__ void mg_diag0_kernel(Args a)
{
    pdl_enter();
    const int W = a.W, H = a.H, P = a.P;
    const size_t n = (size_t)W * H;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t o = (i / W) * P + i % W;
        const float d = a.lev[0].D[o];
        a.lev[0].Di[o] = d > 0.f ? 1.f / d : 0.f;
    }
}

// Initial state, FP64 solution from the FP32 guess.
__global__ void mg_init_kernel(Args a)
{
    pdl_enter();
    const int W = a.W, H = a.H, P = a.P;
    const size_t n = (size_t)W * H;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i % W);
        a.x[(size_t)y * P + x] = (double)a.alpha_in[(size_t)y * W + x];
        a.xinc[(size_t)y * P + x] = 0.f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        State* st = a.st;
        st->rz = st->pq = st->alpha = st->beta = st->rr = st->bn2 = st->rr_true = 0.0;
        st->iter = 0;
        st->done = 0;
        st->status = GM_OK;
        st->need_replace = 1;
        st->replacements = 0;
        st->fold_at = -1;
        st->restart = 0;
        for (int k = 0; k < 8; ++k) st->ticket[k] = 0u;
    }
}

// Solution out (FP32), zero when b = 0.
__global__ void mg_final_kernel(Args a)
{
    pdl_enter();
    const int W = a.W, H = a.H, P = a.P;
    const bool zero = !(a.st->bn2 > 0.0) && a.st->replacements > 0;
    const size_t n = (size_t)W * H;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i % W);
        const size_t o = (size_t)y * P + x;
        a.alpha_out[(size_t)y * W + x] = zero ? 0.f : (float)(a.x[o] + (double)a.xinc[o]);
    }
}

}  // namespace mg
}  // namespace gm

// ===========================================================================
// Host driver
// ===========================================================================
namespace gm {
namespace mg {

struct Plan {
    int L, lt;
    int W[kMaxLevels], H[kMaxLevels];
};

static int make_plan(int W, int H, Plan& pl)
{
    pl.W[0] = W;
    pl.H[0] = H;
    int l = 0;
    for (;;) {
        const int w = (pl.W[l] + 1) / 2, h = (pl.H[l] + 1) / 2;
        if (++l >= kMaxLevels) { gm_set_error_msg("multigrid: too many levels"); return GM_ERR_UNSUPPORTED; }
        pl.W[l] = w;
        pl.H[l] = h;
        if ((long long)w * h <= kCoarseMax) break;
    }
    pl.L = l;
    // the tail takes the deepest levels that fit its shared memory
    pl.lt = pl.L;
    while (pl.lt > 1 && tail_bytes(pl.W, pl.H, pl.lt - 1, pl.L) <= kTailSmem) --pl.lt;
    return GM_OK;
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Workspace carve: fine vectors r, q, p0, p1, z (FP32) and x (FP64) with the
// store's pitch; per coarse level 4 coupling planes, D, Gamma, b, x (FP32,
// pitch a multiple of 32); the coarsest inverse; reduction partials; state.
static size_t carve(const Plan& pl, int P0, char* base, Args* a)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char* { char* p = base ? base + off : nullptr; off += al256(bytes); return p; };
    const size_t n0 = (size_t)pl.H[0] * P0;
    float* r = (float*)take(n0 * 4);
    float* q = (float*)take(n0 * 4);
    float* p0 = (float*)take(n0 * 4);
    float* p1 = (float*)take(n0 * 4);
    float* z = (float*)take(n0 * 4);
    float* di0 = (float*)take(n0 * 4);
    float* xinc = (float*)take(n0 * 4);
    double* x = (double*)take(n0 * 8);
    if (a) {
        a->r = r; a->q = q; a->p0 = p0; a->p1 = p1; a->x = x; a->xinc = xinc;
        a->lev[0].b = r;
        a->lev[0].x = z;
        a->lev[0].Di = di0;
    }
    for (int l = 1; l <= pl.L; ++l) {
        const int P = (pl.W[l] + 31) & ~31;
        const size_t n = (size_t)pl.H[l] * P;
        char* c = take(4 * n * 4);
        float* D = (float*)take(n * 4);
        float* Di = (float*)take(n * 4);
        float* gam = (float*)take(n * 4);
        float* b = (float*)take(n * 4);
        float* xl = (float*)take(n * 4);
        if (a) {
            Lev& v = a->lev[l];
            v.W = pl.W[l]; v.H = pl.H[l]; v.P = P;
            v.c = c; v.ps = n; v.D = D; v.Di = Di; v.gam = gam; v.b = b; v.x = xl;
        }
    }
    double* minv = (double*)take((size_t)kCoarseMax * kCoarseMax * 8);
    double* parts = (double*)take((size_t)5 * kMaxParts * 8);
    State* st = (State*)take(sizeof(State));
    if (a) { a->minv = minv; a->parts = parts; a->st = st; }
    return off;
}

// Per-device solver slots: each has a grow-only workspace, capture streams,
// an execution stream (for batches), pinned state for the read-back, timing
// events and a cache of instantiated graphs.  Single solves use slot 0;
// gm_levin_solve_mg_many spreads its images over the slots.
struct Graph {
    Args key;
    int tcode;
    cudaGraphExec_t exec;
    unsigned long long used;
};

struct Dev {
    void* ws = nullptr;
    size_t ws_bytes = 0;
    cudaStream_t cap = nullptr, cap2 = nullptr, run = nullptr;
    State* host_state = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    std::vector<Graph> graphs;
    unsigned long long clock = 0;
    int sms = 0;
    int cond_ok = -1;  // conditional nodes usable (-1 unknown)
    State* pin = nullptr;  // slot 0 only: pinned result states of a batch
    int pin_n = 0;
};

constexpr int kSlots = 8;        // concurrent solves of gm_levin_solve_mg_many
constexpr int kGraphCache = 16;  // instantiated graphs kept per slot

// GM_MG_GRAPH=0 selects the host-driven loop (the same kernels launched
// one by one, the done flag read every 4 iterations), e.g. for profilers
// that do not look inside conditional graph nodes.
static bool graph_enabled()
{
    const char* e = getenv("GM_MG_GRAPH");
    return !(e && e[0] == '0');
}

static std::mutex g_mu;
static Dev g_dev[64][kSlots];

static void drop_graphs(Dev& d)
{
    for (Graph& g : d.graphs) cudaGraphExecDestroy(g.exec);
    d.graphs.clear();
}

static int dev_setup(Dev& d, size_t bytes)
{
    if (!d.cap) {
        GM_CUDA_TRY(cudaStreamCreateWithFlags(&d.cap, cudaStreamNonBlocking));
        GM_CUDA_TRY(cudaStreamCreateWithFlags(&d.cap2, cudaStreamNonBlocking));
        GM_CUDA_TRY(cudaStreamCreateWithFlags(&d.run, cudaStreamNonBlocking));
        GM_CUDA_TRY(cudaMallocHost((void**)&d.host_state, sizeof(State)));
        GM_CUDA_TRY(cudaEventCreate(&d.e0));
        GM_CUDA_TRY(cudaEventCreate(&d.e1));
        GM_CUDA_TRY(cudaEventCreate(&d.e2));
    }
    if (d.ws_bytes < bytes) {
        drop_graphs(d);
        if (d.ws) cudaFree(d.ws);
        d.ws = nullptr;
        d.ws_bytes = 0;
        if (cudaMalloc(&d.ws, bytes) != cudaSuccess) {
            cudaGetLastError();
            gm_set_error_msg("multigrid workspace allocation (%zu bytes) failed", bytes);
            return GM_ERR_NOMEM;
        }
        d.ws_bytes = bytes;
    }
    return GM_OK;
}

static int occupancy(const void* fn, int smem, int threads)
{
    struct E { const void* fn; int dev, smem, occ; };
    static std::vector<E> cache;  // guarded by g_mu
    int dev = 0;
    cudaGetDevice(&dev);
    for (const E& e : cache)
        if (e.fn == fn && e.dev == dev && e.smem == smem) return e.occ;
    if (smem > 48 * 1024) {
        // the largest size the kernel may ask for (opt-in maximum less its
        // static shared memory), so graphs captured with other sizes stay valid
        int optin = 0;
        cudaFuncAttributes fa;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, fn) == cudaSuccess)
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 std::max(smem, optin - (int)fa.sharedSizeBytes));
        cudaGetLastError();
    }
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, threads, smem) != cudaSuccess) o = 1;
    if (o < 1) o = 1;
    cache.push_back({fn, dev, smem, o});
    return o;
}

static int tiles_of(int W, int H, int ty) { return ((W + kTX - 1) / kTX) * ((H + ty - 1) / ty); }

// Enqueues kernels on one stream.  The template argument is the element type
// of the fine iteration planes.  A dry pass only computes the launch shapes
// (it sets the kernels' shared-memory limits before any stream capture).
// Tensor maps of the TMA-pipelined kernels: the level-0 SpMV, and the
// restriction / prolongation of every level below the tail.
struct FineMaps {
    TMaps spmv, down[kMaxLevels], up[kMaxLevels];
};

// Whether the outer SpMV streams the FP16 iteration planes (tcode 1) rather
// than the FP32 ones.  It saves 24 of ~180 B per pixel-iteration, and the
// FP16 outer operator costs 1 % more iterations at rtol 1e-6 (1080p: 87
// against 86).  Between replacements each cycle can refine less, so below
// 1e-7 the extra iterations outweigh it (1e-10: 408 against 331), and the
// FP32 planes stay.  rtol <= 0 (a fixed iteration count) takes the FP16 ones.
constexpr double kOuterLowMinRtol = 1e-7;
static int outer_low_for(int tcode, double rtol)
{
    return tcode == 1 && !(rtol > 0.0 && rtol < kOuterLowMinRtol) ? 1 : 0;
}

// Tensor maps of the level-0 kernels (es: bytes per element of the
// iteration planes).
static int make_maps(const Args& a, int es, CUtensorMapDataType dt, FineMaps& fm)
{
    const uint64_t W = (uint64_t)a.W, H = (uint64_t)a.H, P = (uint64_t)a.P;
    auto planes = [&](CUtensorMap* m, const void* base, CUtensorMapDataType t, uint64_t e, uint64_t ps, int th) {
        const uint64_t d3[3] = {W, H, 12};
        const uint64_t s3[2] = {P * e, ps * e};
        const uint32_t b3[3] = {(uint32_t)kFBW, (uint32_t)(th + 2), 12u};
        return gm_make_tmap(m, t, 3, const_cast<void*>(base), d3, s3, b3);
    };
    auto vec = [&](CUtensorMap* m, const float* base, uint64_t w, uint64_t h, uint64_t pitch, int bw, int bh) {
        const uint64_t d2[2] = {w, h};
        const uint64_t s2[1] = {pitch * 4};
        const uint32_t b2[2] = {(uint32_t)bw, (uint32_t)bh};
        return gm_make_tmap(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), d2, s2, b2);
    };
    const int t32 = fine_rows(4), tlo = fine_rows(es);
    const Lev& L0 = a.lev[0];
    // the SpMV streams the FP16 iteration planes and their diagonal d when
    // outer_low is set, else the FP32 planes and d32
    const bool lo16 = es == 2 && dt == CU_TENSOR_MAP_DATA_TYPE_FLOAT16 && a.outer_low;
    const int ts = lo16 ? tlo : t32;
    if (lo16) GM_TRY(planes(&fm.spmv.m[0], L0.c, dt, 2, L0.ps, ts));
    else GM_TRY(planes(&fm.spmv.m[0], a.w32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.ps32, ts));
    GM_TRY(vec(&fm.spmv.m[1], L0.x, W, H, P, kFBW, ts + 4));
    GM_TRY(vec(&fm.spmv.m[2], a.p0, W, H, P, kFBW, ts + 4));
    GM_TRY(vec(&fm.spmv.m[3], a.p1, W, H, P, kFBW, ts + 4));
    GM_TRY(vec(&fm.spmv.m[4], lo16 ? L0.D : a.d32, W, H, P, kFTW, ts));
    for (int l = 0; l < a.lt; ++l) {
        // level 0: the store's planes (12, iteration precision); below: 4 FP32 planes
        const Lev& F = a.lev[l];
        const Lev& Cl = a.lev[l + 1];
        const int np = l == 0 ? 12 : 4;
        const uint64_t e = l == 0 ? (uint64_t)es : 4;
        const int th = l == 0 ? tlo : t32;
        const uint64_t Wl = (uint64_t)F.W, Hl = (uint64_t)F.H, Pl = (uint64_t)F.P;
        const uint64_t d3[3] = {Wl, Hl, (uint64_t)np};
        const uint64_t s3[2] = {Pl * e, (uint64_t)F.ps * e};
        const uint32_t b3[3] = {(uint32_t)kFBW, (uint32_t)(th + 2), (uint32_t)np};
        GM_TRY(gm_make_tmap(&fm.down[l].m[0], l == 0 ? dt : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, F.c, d3, s3, b3));
        GM_TRY(vec(&fm.down[l].m[1], F.b, Wl, Hl, Pl, kFBW, th + 4));
        GM_TRY(vec(&fm.down[l].m[2], F.Di, Wl, Hl, Pl, kFBW, th + 4));
        fm.up[l] = fm.down[l];
        GM_TRY(vec(&fm.up[l].m[3], Cl.x, (uint64_t)Cl.W, (uint64_t)Cl.H, (uint64_t)Cl.P, kXBW, th / 2 + 2));
    }
    return GM_OK;
}

template <class T>
struct Enq {
    const Args& a;
    int sms;
    cudaStream_t s;
    bool dry;
    const FineMaps* fm;

    template <class K, class... X> void go(K fn, int tiles, int smem, int threads, X... args) const
    {
        int g = std::min(tiles, sms * occupancy((const void*)fn, smem, threads));
        g = std::max(1, std::min(g, kMaxParts));
        if (dry) return;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)g);
        cfg.blockDim = dim3((unsigned)threads);
        cfg.dynamicSmemBytes = (size_t)smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, fn, args...);
    }

    int pointwise_tiles() const
    {
        return (int)std::min<size_t>((size_t)sms * 4, ((size_t)(a.W + 3) / 4 * a.H + kThreads - 1) / kThreads);
    }

    // The TMA-pipelined kernels: level 0 with the store's 12 planes in the
    // iteration precision, the levels below with their 4 FP32 planes.
    template <int MODE> void fine(int l) const
    {
        const Lev& F = a.lev[l];
        const TMaps& m = MODE == FM_SPMV ? fm->spmv : (MODE == FM_DOWN ? fm->down[l] : fm->up[l]);
        if (l == 0 && MODE == FM_SPMV && !a.outer_low) {
            using LY = FineLayout<MODE, 4, 12>;
            const int tiles = ((F.W + kFTW - 1) / kFTW) * ((F.H + LY::TH - 1) / LY::TH);
            go(mg_fine_kernel<MODE, FineSten, float>, tiles, LY::total, LY::THR, m, a, 0);
        } else if (l == 0) {
            using LY = FineLayout<MODE, FinePlanes<MODE, T>::ES, 12>;
            const int tiles = ((F.W + kFTW - 1) / kFTW) * ((F.H + LY::TH - 1) / LY::TH);
            go(mg_fine_kernel<MODE, FineSten, T>, tiles, LY::total, LY::THR, m, a, 0);
        } else {
            using LY = FineLayout<MODE, 4, 4>;
            const int tiles = ((F.W + kFTW - 1) / kFTW) * ((F.H + LY::TH - 1) / LY::TH);
            go(mg_fine_kernel<MODE, CoarseSten, float>, tiles, LY::total, LY::THR, m, a, l);
        }
    }

    void down(int l) const { fine<FM_DOWN>(l); }
    void up(int l) const { fine<FM_UP>(l); }

    void vcycle() const
    {
        for (int l = 0; l < a.lt; ++l) down(l);
        int Wl[kMaxLevels], Hl[kMaxLevels];
        for (int l = 0; l <= a.L; ++l) { Wl[l] = a.lev[l].W; Hl[l] = a.lev[l].H; }
        go(mg_tail_kernel, 1, tail_bytes(Wl, Hl, a.lt, a.L), kTailThreads, a);
        for (int l = a.lt - 1; l >= 0; --l) up(l);
    }

    void replace() const
    {
        constexpr int sm = (int)(sizeof(float) * FineSten::NP * (kTY + kHalo) * kPW +
                                 sizeof(double) * (kTY + 2 * kHalo) * kVW);
        go(mg_replace_kernel, tiles_of(a.W, a.H, kTY), sm, kThreads, a);
    }

    void build() const
    {
        go(mg_diag0_kernel, pointwise_tiles() * 4, 0, kThreads, a);
        for (int l = 0; l < a.L; ++l) {
            const Lev& C = a.lev[l + 1];
            const int t = (C.W * C.H + 127) / 128;
            if (l == 0) go(mg_build_kernel<FineSten, T>, t, 0, 128, a, 0, (const float*)a.gamma, a.P);
            else go(mg_build_kernel<CoarseSten, float>, t, 0, 128, a, l, (const float*)a.lev[l].gam, a.lev[l].P);
        }
        const int n = a.lev[a.L].W * a.lev[a.L].H;
        const int sm = (int)(sizeof(double) * ((size_t)n * n + 2 * kCoarseMax));
        go(mg_inverse_kernel, 1, sm, kThreads, a);
    }

    void setup() const
    {
        go(mg_init_kernel, pointwise_tiles(), 0, kThreads, a);
        build();
        replace();
        vcycle();
    }

    void iteration() const
    {
        fine<FM_SPMV>(0);
        go(mg_update_kernel, pointwise_tiles(), 0, kThreads, a);
        replace();
        vcycle();
    }

    void finish() const { go(mg_final_kernel, pointwise_tiles(), 0, kThreads, a); }
};

// Captures set-up + WHILE(iteration) + finish into one graph.
template <class T>
static int build_graph(Dev& d, Args a, const FineMaps& fm, cudaGraphExec_t* exec)
{
    cudaGraph_t g = nullptr;
    a.cond = 0;
    {
        const Enq<T> dry{a, d.sms, d.cap, true, &fm};
        dry.setup();
        dry.iteration();
        dry.finish();
    }
    GM_CUDA_TRY(cudaStreamBeginCapture(d.cap, cudaStreamCaptureModeThreadLocal));
    Enq<T>{a, d.sms, d.cap, false, &fm}.setup();
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(d.cap, &cs, nullptr, &cg, &deps, &ndeps);
    cudaGraphConditionalHandle h = 0;
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&node, cg, deps, ndeps, &cp);
    }
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(d.cap, &node, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(d.cap2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            Args ab = a;
            ab.cond = (unsigned long long)h;
            Enq<T>{ab, d.sms, d.cap2, false, &fm}.iteration();
            cudaGraph_t bg = body;
            e = cudaStreamEndCapture(d.cap2, &bg);
        }
    }
    if (e == cudaSuccess) Enq<T>{a, d.sms, d.cap, false, &fm}.finish();
    cudaError_t e2 = cudaStreamEndCapture(d.cap, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm_set_error_msg("multigrid graph capture: %s", cudaGetErrorString(e));
        return GM_ERR_CUDA;
    }
    return GM_OK;
}

// The cached graph of this solve on slot d, captured on first use.
template <class T>
static int graph_for(Dev& d, const Args& a, const FineMaps& fm, int tcode, Graph** out)
{
    *out = nullptr;
    for (Graph& g : d.graphs)
        if (g.tcode == tcode && memcmp(&g.key, &a, sizeof(Args)) == 0) *out = &g;
    if (*out) {
        (*out)->used = ++d.clock;
        return GM_OK;
    }
    cudaGraphExec_t ex = nullptr;
    GM_TRY(build_graph<T>(d, a, fm, &ex));
    if (d.graphs.size() >= (size_t)kGraphCache) {
        auto old = std::min_element(d.graphs.begin(), d.graphs.end(),
                                    [](const Graph& x, const Graph& y) { return x.used < y.used; });
        cudaGraphExecDestroy(old->exec);
        d.graphs.erase(old);
    }
    Graph g;
    memcpy(&g.key, &a, sizeof(Args));
    g.tcode = tcode;
    g.exec = ex;
    g.used = ++d.clock;
    d.graphs.push_back(g);
    *out = &d.graphs.back();
    return GM_OK;
}

template <class T>
static int run(Dev& d, const Args& a0, const FineMaps& fm, int tcode, cudaStream_t st, float* ms)
{
    Args a = a0;
    if (d.cond_ok != 0 && graph_enabled()) {
        Graph* hit = nullptr;
        for (Graph& g : d.graphs)
            if (g.tcode == tcode && memcmp(&g.key, &a, sizeof(Args)) == 0) hit = &g;
        if (!hit) {
            cudaGraphExec_t ex = nullptr;
            const int rc = build_graph<T>(d, a, fm, &ex);
            if (rc == GM_OK) {
                if (d.graphs.size() >= (size_t)kGraphCache) {
                    auto old = std::min_element(d.graphs.begin(), d.graphs.end(),
                                                [](const Graph& x, const Graph& y) { return x.used < y.used; });
                    cudaGraphExecDestroy(old->exec);
                    d.graphs.erase(old);
                }
                Graph g;
                memcpy(&g.key, &a, sizeof(Args));
                g.tcode = tcode;
                g.exec = ex;
                g.used = 0;
                d.graphs.push_back(g);
                hit = &d.graphs.back();
                d.cond_ok = 1;
            } else if (d.cond_ok == -1) {
                d.cond_ok = 0;  // conditional nodes unavailable: host-driven loop from now on
                if (getenv("GM_MG_DEBUG")) fprintf(stderr, "gm_mg: graph path unavailable (%s)\n", gm_last_error());
            } else {
                return rc;
            }
        }
        if (hit) {
            hit->used = ++d.clock;
            GM_CUDA_TRY(cudaEventRecord(d.e0, st));
            GM_CUDA_TRY(cudaGraphLaunch(hit->exec, st));
            GM_CUDA_TRY(cudaEventRecord(d.e1, st));
            GM_CUDA_TRY(cudaMemcpyAsync(d.host_state, a.st, sizeof(State), cudaMemcpyDeviceToHost, st));
            GM_CUDA_TRY(cudaStreamSynchronize(st));
            cudaEventElapsedTime(ms, d.e0, d.e1);
            return GM_OK;
        }
    }
    // Host-driven loop: the same kernels, the done flag read every 4 iterations.
    a.cond = 0;
    Enq<T> q{a, d.sms, st, false, &fm};
    GM_CUDA_TRY(cudaEventRecord(d.e0, st));
    q.setup();
    for (int it = 0; it <= a.max_iters + 4; it += 4) {
        for (int k = 0; k < 4; ++k) q.iteration();
        GM_CUDA_TRY(cudaMemcpyAsync(d.host_state, a.st, sizeof(State), cudaMemcpyDeviceToHost, st));
        GM_CUDA_TRY(cudaStreamSynchronize(st));
        if (d.host_state->done) break;
    }
    q.finish();
    GM_CUDA_TRY(cudaEventRecord(d.e1, st));
    GM_CUDA_TRY(cudaMemcpyAsync(d.host_state, a.st, sizeof(State), cudaMemcpyDeviceToHost, st));
    GM_CUDA_TRY(cudaStreamSynchronize(st));
    GM_CUDA_TRY(cudaGetLastError());
    cudaEventElapsedTime(ms, d.e0, d.e1);
    return GM_OK;
}

// One image of gm_levin_solve_mg_many.
struct Item {
    Plan pl;
    Args a;
    size_t bytes;
    FineMaps fm;
    int slot;
};

// Launches every image's graph on the execution stream of its slot, forked
// from and joined back to st, and copies each
// image's final state to pinned memory on the same stream.  The images of one
// slot run one after another (they share its workspace); different slots run
// concurrently.  One host synchronisation for the whole batch.
template <class T>
static int run_many(Dev* slots, int K, std::vector<Item>& items, int tcode, cudaStream_t st, float* ms)
{
    const int n = (int)items.size();
    Dev& d0 = slots[0];
    std::vector<cudaGraphExec_t> ex(n);
    for (int k = 0; k < n; ++k) {
        Graph* g = nullptr;
        GM_TRY(graph_for<T>(slots[items[k].slot], items[k].a, items[k].fm, tcode, &g));
        ex[k] = g->exec;
    }
    if (d0.pin_n < n) {
        if (d0.pin) cudaFreeHost(d0.pin);
        d0.pin = nullptr;
        d0.pin_n = 0;
        GM_CUDA_TRY(cudaMallocHost((void**)&d0.pin, (size_t)n * sizeof(State)));
        d0.pin_n = n;
    }
    GM_CUDA_TRY(cudaEventRecord(d0.e0, st));
    for (int j = 0; j < K; ++j) GM_CUDA_TRY(cudaStreamWaitEvent(slots[j].run, d0.e0, 0));
    for (int k = 0; k < n; ++k) {
        Dev& d = slots[items[k].slot];
        GM_CUDA_TRY(cudaGraphLaunch(ex[k], d.run));
        GM_CUDA_TRY(cudaMemcpyAsync(d0.pin + k, items[k].a.st, sizeof(State), cudaMemcpyDeviceToHost, d.run));
    }
    for (int j = 0; j < K; ++j) {
        GM_CUDA_TRY(cudaEventRecord(slots[j].e1, slots[j].run));
        GM_CUDA_TRY(cudaStreamWaitEvent(st, slots[j].e1, 0));
    }
    GM_CUDA_TRY(cudaEventRecord(d0.e2, st));
    GM_CUDA_TRY(cudaStreamSynchronize(st));
    cudaEventElapsedTime(ms, d0.e0, d0.e2);
    return GM_OK;
}

// Fills the level-0 fields and the carve of an Args for the store.
static int prepare(const gm_levin_store* store, int use_low, Plan& pl, Args& a, size_t* bytes, int* tcode)
{
    const int W = store->W, H = store->H, P = store->pitch;
    if (W <= 0 || H <= 0 || P < W || (P & 7)) { gm_set_error_msg("multigrid: bad store shape"); return GM_ERR_INVALID; }
    GM_TRY(make_plan(W, H, pl));
    memset(&a, 0, sizeof(Args));
    const bool low = use_low && store->precision != GM_PREC_FP32;
    const size_t ps = store->plane_stride ? store->plane_stride : (size_t)H * P;
    const int esz = low ? 2 : 4;
    const void* wp = low ? store->w : (const void*)store->w32;
    if (((uintptr_t)wp & 15) || ((uintptr_t)store->w32 & 15) || ((ps * esz) & 15) || ((ps * 4) & 15)) {
        gm_set_error_msg("multigrid: planes must be 16-byte aligned");
        return GM_ERR_INVALID;
    }
    *tcode = low ? (store->precision == GM_PREC_FP16 ? 1 : 2) : 0;
    a.L = pl.L;
    a.lt = pl.lt;
    a.W = W; a.H = H; a.P = P;
    Lev& f = a.lev[0];
    f.W = W; f.H = H; f.P = P;
    f.c = const_cast<void*>(wp);
    f.ps = ps;
    f.D = low ? store->d : store->d32;
    a.w32 = store->w32;
    a.ps32 = ps;
    a.gamma = store->gamma;
    a.d32 = store->d32;
    *bytes = carve(pl, P, nullptr, nullptr);
    return GM_OK;
}

static CUtensorMapDataType tcode_dtype(int tcode)
{
    return tcode == 1 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                      : (tcode == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32);
}

static int dev_index(int* dev)
{
    GM_CUDA_TRY(cudaGetDevice(dev));
    if (*dev < 0 || *dev >= 64) { gm_set_error_msg("device index out of range"); return GM_ERR_UNSUPPORTED; }
    return GM_OK;
}

}  // namespace mg

// Solve with the multigrid-preconditioned CG (called from the store solvers).
int run_mg_solver(const gm_levin_store* store, const float* b, int bpitch, const float* alpha_in, float* alpha_out,
                  const gm_solve_params* p, gm_solve_info* info, cudaStream_t st)
{
    using namespace mg;
    int sms = 0;
    GM_TRY(gm_check_device(&sms));
    if (p->max_iters < 0) { gm_set_error_msg("max_iters must be >= 0"); return GM_ERR_INVALID; }
    Plan pl;
    Args a;
    size_t bytes = 0;
    int tcode = 0;
    GM_TRY(prepare(store, p->use_low, pl, a, &bytes, &tcode));
    int dev = 0;
    GM_TRY(dev_index(&dev));
    std::lock_guard<std::mutex> g(g_mu);
    Dev& d = g_dev[dev][0];
    d.sms = sms;
    GM_TRY(dev_setup(d, bytes));
    carve(pl, a.P, (char*)d.ws, &a);
    a.bvec = b;
    a.bpitch = bpitch;
    a.alpha_in = alpha_in;
    a.alpha_out = alpha_out;
    a.rtol = p->rtol;
    a.outer_low = outer_low_for(tcode, a.rtol);
    a.max_iters = p->max_iters;
    a.replace_every = p->replace_every;
    a.omega = p->mg_omega > 0.f ? p->mg_omega : kDefaultOmega;
    a.scale = p->mg_scale > 0.f ? p->mg_scale : kDefaultScale;
    FineMaps fm;
    GM_TRY(make_maps(a, tcode ? 2 : 4, tcode_dtype(tcode), fm));
    float ms = 0.f;
    int rc;
    if (tcode == 1) rc = run<__half>(d, a, fm, tcode, st, &ms);
    else if (tcode == 2) rc = run<__nv_bfloat16>(d, a, fm, tcode, st, &ms);
    else rc = run<float>(d, a, fm, tcode, st, &ms);
    if (rc != GM_OK) return rc;
    const State& s = *d.host_state;
    if (info) {
        memset(info, 0, sizeof(*info));
        info->status = s.status;
        info->iters = s.iter;
        info->replacements = s.replacements;
        info->bnorm = std::sqrt(s.bn2);
        info->rel_residual = s.bn2 > 0.0 ? std::sqrt(s.rr_true / s.bn2) : 0.0;
        info->kernel_ms = ms;
        info->grid = pl.L + 1;
        info->where = 0;
        info->solver = GM_SOLVER_MG;
    }
    if (s.status != GM_OK) {
        gm_set_error_msg(s.status == GM_ERR_NOT_CONVERGED ? "multigrid CG: max_iters reached above rtol"
                                                         : "multigrid CG: breakdown (non-positive curvature, "
                                                           "singular coarse operator or non-finite value)");
    }
    return s.status;
}

static void fill_info(gm_solve_info* info, const mg::State& s, float ms, int levels)
{
    memset(info, 0, sizeof(*info));
    info->status = s.status;
    info->iters = s.iter;
    info->replacements = s.replacements;
    info->bnorm = std::sqrt(s.bn2);
    info->rel_residual = s.bn2 > 0.0 ? std::sqrt(s.rr_true / s.bn2) : 0.0;
    info->kernel_ms = ms;
    info->grid = levels;
    info->where = 0;
    info->solver = GM_SOLVER_MG;
}

}  // namespace gm

// Many independent multigrid solves at once (see gpumat.h).
extern "C" int gm_levin_solve_mg_many(const gm_levin_store* const* stores, float* const* alphas, int count,
                                      const gm_solve_params* prm, gm_solve_info* infos, void* stream)
{
    using namespace gm;
    using namespace gm::mg;
    gm_solve_params p;
    if (prm) p = *prm; else gm_default_params(&p);
    if (count < 0 || (count > 0 && (!stores || !alphas))) {
        gm_set_error_msg("gm_levin_solve_mg_many: bad arguments");
        return GM_ERR_INVALID;
    }
    if (count == 0) return GM_OK;
    if (p.max_iters < 0) { gm_set_error_msg("max_iters must be >= 0"); return GM_ERR_INVALID; }
    int sms = 0;
    GM_TRY(gm_check_device(&sms));
    std::vector<Item> items((size_t)count);
    int tcode = -1;
    for (int k = 0; k < count; ++k) {
        if (!stores[k] || !stores[k]->w32 || !alphas[k]) {
            gm_set_error_msg("gm_levin_solve_mg_many: image %d has no store or alpha", k);
            return GM_ERR_INVALID;
        }
        int tc = 0;
        GM_TRY(prepare(stores[k], p.use_low, items[k].pl, items[k].a, &items[k].bytes, &tc));
        if (tcode >= 0 && tc != tcode) {
            gm_set_error_msg("gm_levin_solve_mg_many: all stores must have the same precision");
            return GM_ERR_INVALID;
        }
        tcode = tc;
    }
    int dev = 0;
    GM_TRY(dev_index(&dev));
    std::lock_guard<std::mutex> g(g_mu);
    Dev* slots = g_dev[dev];
    const bool graphs = graph_enabled() && slots[0].cond_ok != 0;
    const int K = graphs ? std::min(kSlots, count) : 1;
    // Deal the images to the slots largest first, each to the least-loaded
    // slot (a fixed per-solve cost plus the pixels); the deal depends only
    // on the shapes, so repeated calls reuse each slot's cached graphs.
    {
        std::vector<int> order(count);
        for (int k = 0; k < count; ++k) order[k] = k;
        auto cost = [&](int k) { return (double)items[k].a.W * items[k].a.H + 2.0e5; };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
        std::vector<double> load(K, 0.0);
        for (int k : order) {
            const int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            items[k].slot = j;
            load[j] += cost(k);
        }
    }
    for (int j = 0; j < K; ++j) {
        size_t need = 0;
        for (int k = 0; k < count; ++k)
            if (items[k].slot == j) need = std::max(need, items[k].bytes);
        slots[j].sms = sms;
        GM_TRY(dev_setup(slots[j], need));
    }
    for (int k = 0; k < count; ++k) {
        Args& a = items[k].a;
        carve(items[k].pl, a.P, (char*)slots[items[k].slot].ws, &a);
        a.bvec = stores[k]->b;
        a.bpitch = stores[k]->pitch;
        a.alpha_in = alphas[k];
        a.alpha_out = alphas[k];
        a.rtol = p.rtol;
        a.outer_low = outer_low_for(tcode, a.rtol);
        a.max_iters = p.max_iters;
        a.replace_every = p.replace_every;
        a.omega = p.mg_omega > 0.f ? p.mg_omega : kDefaultOmega;
        a.scale = p.mg_scale > 0.f ? p.mg_scale : kDefaultScale;
        GM_TRY(make_maps(a, tcode ? 2 : 4, tcode_dtype(tcode), items[k].fm));
    }
    cudaStream_t st = (cudaStream_t)stream;
    int worst = GM_OK;
    if (!graphs) {
        // no conditional graphs here: one solve after another on slot 0
        for (int k = 0; k < count; ++k) {
            float ms = 0.f;
            int rc;
            if (tcode == 1) rc = run<__half>(slots[0], items[k].a, items[k].fm, tcode, st, &ms);
            else if (tcode == 2) rc = run<__nv_bfloat16>(slots[0], items[k].a, items[k].fm, tcode, st, &ms);
            else rc = run<float>(slots[0], items[k].a, items[k].fm, tcode, st, &ms);
            if (rc != GM_OK) return rc;
            if (infos) fill_info(&infos[k], *slots[0].host_state, ms, items[k].pl.L + 1);
            worst = std::max(worst, slots[0].host_state->status);
        }
    } else {
        float ms = 0.f;
        int rc;
        if (tcode == 1) rc = run_many<__half>(slots, K, items, tcode, st, &ms);
        else if (tcode == 2) rc = run_many<__nv_bfloat16>(slots, K, items, tcode, st, &ms);
        else rc = run_many<float>(slots, K, items, tcode, st, &ms);
        if (rc != GM_OK && slots[0].cond_ok == -1) {
            // the first capture failed: no conditional graphs here, so solve
            // the images one after another with the host-driven loop
            slots[0].cond_ok = 0;
            if (getenv("GM_MG_DEBUG")) fprintf(stderr, "gm_mg: graph path unavailable (%s)\n", gm_last_error());
            for (int k = 0; k < count; ++k) {
                GM_TRY(dev_setup(slots[0], items[k].bytes));
                Args& a = items[k].a;
                carve(items[k].pl, a.P, (char*)slots[0].ws, &a);
                GM_TRY(make_maps(a, tcode ? 2 : 4, tcode_dtype(tcode), items[k].fm));
                float ms1 = 0.f;
                if (tcode == 1) rc = run<__half>(slots[0], a, items[k].fm, tcode, st, &ms1);
                else if (tcode == 2) rc = run<__nv_bfloat16>(slots[0], a, items[k].fm, tcode, st, &ms1);
                else rc = run<float>(slots[0], a, items[k].fm, tcode, st, &ms1);
                if (rc != GM_OK) return rc;
                if (infos) fill_info(&infos[k], *slots[0].host_state, ms1, items[k].pl.L + 1);
                worst = std::max(worst, slots[0].host_state->status);
            }
            if (worst != GM_OK) gm_set_error_msg("multigrid batch: an image ended with status %d", worst);
            return worst;
        }
        if (rc != GM_OK) return rc;
        slots[0].cond_ok = 1;
        for (int k = 0; k < count; ++k) {
            if (infos) fill_info(&infos[k], slots[0].pin[k], ms, items[k].pl.L + 1);
            worst = std::max(worst, slots[0].pin[k].status);
        }
    }
    if (worst != GM_OK) gm_set_error_msg("multigrid batch: an image ended with status %d", worst);
    return worst;
}

// ---------------------------------------------------------------------------
// C ABI: level shapes and an inspection entry for tests
// ---------------------------------------------------------------------------
extern "C" int gm_levin_mg_levels(int W, int H, int* nlevels, int* dims, int cap)
{
    using namespace gm::mg;
    if (W <= 0 || H <= 0 || !nlevels) { gm_set_error_msg("gm_levin_mg_levels: bad arguments"); return GM_ERR_INVALID; }
    Plan pl;
    GM_TRY(make_plan(W, H, pl));
    *nlevels = pl.L + 1;
    if (dims)
        for (int l = 0; l <= pl.L && l < cap; ++l) { dims[2 * l] = pl.W[l]; dims[2 * l + 1] = pl.H[l]; }
    return GM_OK;
}

extern "C" int gm_levin_mg_inspect(const gm_levin_store* store, int use_low, const float* r, float* z, int level,
                                   float* c_host, float* d_host, void* stream)
{
    using namespace gm;
    using namespace gm::mg;
    if (!store || !store->w32) { gm_set_error_msg("gm_levin_mg_inspect: bad arguments"); return GM_ERR_INVALID; }
    int sms = 0;
    GM_TRY(gm_check_device(&sms));
    Plan pl;
    Args a;
    size_t bytes = 0;
    int tcode = 0;
    GM_TRY(prepare(store, use_low, pl, a, &bytes, &tcode));
    if (level < 0 || level > pl.L) { gm_set_error_msg("gm_levin_mg_inspect: level out of range"); return GM_ERR_INVALID; }
    int dev = 0;
    GM_TRY(dev_index(&dev));
    std::lock_guard<std::mutex> g(g_mu);
    Dev& d = g_dev[dev][0];
    d.sms = sms;
    GM_TRY(dev_setup(d, bytes));
    carve(pl, a.P, (char*)d.ws, &a);
    a.omega = kDefaultOmega;
    a.scale = kDefaultScale;
    a.max_iters = 1;
    FineMaps fm;
    GM_TRY(make_maps(a, tcode ? 2 : 4, tcode_dtype(tcode), fm));
    cudaStream_t st = (cudaStream_t)stream;
    GM_CUDA_TRY(cudaMemsetAsync(a.st, 0, sizeof(State), st));
    auto go = [&](auto tag) {
        using T = decltype(tag);
        Enq<T> q{a, sms, st, false, &fm};
        q.build();
        if (r && z) {
            cudaMemcpy2DAsync(a.r, (size_t)a.P * 4, r, (size_t)a.W * 4, (size_t)a.W * 4, a.H, cudaMemcpyDeviceToDevice,
                              st);
            q.vcycle();
            cudaMemcpy2DAsync(z, (size_t)a.W * 4, a.lev[0].x, (size_t)a.P * 4, (size_t)a.W * 4, a.H,
                              cudaMemcpyDeviceToDevice, st);
        }
    };
    if (tcode == 1) go(__half());
    else if (tcode == 2) go(__nv_bfloat16());
    else go(0.0f);
    if (level >= 1 && (c_host || d_host)) {
        const Lev& v = a.lev[level];
        for (int k = 0; k < 4 && c_host; ++k)
            GM_CUDA_TRY(cudaMemcpy2DAsync(c_host + (size_t)k * v.W * v.H, (size_t)v.W * 4,
                                          static_cast<float*>(v.c) + (size_t)k * v.ps, (size_t)v.P * 4,
                                          (size_t)v.W * 4, v.H, cudaMemcpyDeviceToHost, st));
        if (d_host)
            GM_CUDA_TRY(cudaMemcpy2DAsync(d_host, (size_t)v.W * 4, v.D, (size_t)v.P * 4, (size_t)v.W * 4, v.H,
                                          cudaMemcpyDeviceToHost, st));
    }
    GM_CUDA_TRY(cudaMemcpyAsync(d.host_state, a.st, sizeof(State), cudaMemcpyDeviceToHost, st));
    GM_CUDA_TRY(cudaStreamSynchronize(st));
    GM_CUDA_TRY(cudaGetLastError());
    if (d.host_state->status != GM_OK) {
        gm_set_error_msg("multigrid: singular coarse operator");
        return d.host_state->status;
    }
    return GM_OK;
}
