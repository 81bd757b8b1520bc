// gm_apply.cu -- one streaming pass y = A x over the symmetric Levin store
// (the banded SpMV of BandedMatrix.cu:107-141, bmAx_k, on the 13-band
// symmetric layout instead of 25 explicit bands).
//
// Persistent kernel, one CTA per SM, 256 threads.  The image is cut into
// tiles of 128 columns x TH rows; CTA c takes tiles c, c + G, ... in row-major
// tile order, so the tiles in flight at any moment are neighbours and the
// halo rows they share come from L2.  For each tile one elected thread issues
// three TMA loads into a two-stage shared-memory ring:
//   bands: 3-D box {144, TH + 2, 12} of the 12 affinity planes (2 rows above
//          the tile for the mirrored couplings, 8 columns each side so the
//          box starts on a 16-byte boundary),
//   x:     2-D box {144, TH + 4} (2 rows and 8 columns of halo),
//   diag:  2-D box {128, TH} of d (iteration operator) or gamma (true one),
// and while the CTA computes one stage the other stage's loads are in flight.
// Each thread owns a column pair and marches TH/4 consecutive rows with a
// 5-row x 6-column window of x in registers.  Tiles past the image edge read
// TMA's zero fill; the store's planes are zero on couplings that leave the
// image, so edges need no special case.
#include "gm_internal.cuh"

namespace gm {

constexpr int kApplyThreads = 256;
constexpr int kApplyTW = 128;             // output columns per tile
constexpr int kApplyBoxW = kApplyTW + 16; // 8 halo columns each side

__host__ __device__ constexpr int apply_rows(int esize) { return esize == 2 ? 16 : 8; }

struct ApplyLayout {
    int w_off, x_off, d_off, stage, total;
    uint32_t bytes;  // TMA bytes per stage
};

__host__ __device__ constexpr int a128c(int x) { return (x + 127) & ~127; }

__host__ __device__ constexpr ApplyLayout apply_layout(int esize)
{
    ApplyLayout L{};
    const int th = apply_rows(esize);
    const int wb = 12 * (th + 2) * kApplyBoxW * esize;
    const int xb = (th + 4) * kApplyBoxW * 4;
    const int db = th * kApplyTW * 4;
    L.w_off = 0;
    L.x_off = a128c(wb);
    L.d_off = L.x_off + a128c(xb);
    L.stage = L.d_off + a128c(db);
    L.total = 2 * L.stage + 128;  // + mbarriers
    L.bytes = (uint32_t)(wb + xb + db);
    return L;
}

template <class T> __device__ __forceinline__ float2 ld_pair(const T* p);
template <> __device__ __forceinline__ float2 ld_pair<float>(const float* p) { return *reinterpret_cast<const float2*>(p); }
template <> __device__ __forceinline__ float2 ld_pair<__half>(const __half* p)
{
    return __half22float2(*reinterpret_cast<const __half2*>(p));
}
template <> __device__ __forceinline__ float2 ld_pair<__nv_bfloat16>(const __nv_bfloat16* p)
{
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}
template <class T> __device__ __forceinline__ float ld_one(const T* p) { return Cvt<T>::to_f(*p); }

// TRUE_OP = false: y_i = d_i x_i - sum_j w_ij x_j (the iteration operator of
// the store's precision); true: y_i = gamma_i x_i + sum_j w_ij (x_i - x_j).
template <class T, bool TRUE_OP>
__global__ void __launch_bounds__(kApplyThreads, 1)
    levin_apply_kernel(const __grid_constant__ CUtensorMap mw, const __grid_constant__ CUtensorMap mx,
                       const __grid_constant__ CUtensorMap md, float* __restrict__ y, int ypitch, int W, int H,
                       int ntx, int ntiles, GridBarrier* gb, uint64_t limit_ns)
{
    constexpr int TH = apply_rows(sizeof(T));
    constexpr int RPT = TH / 4;  // rows per thread
    constexpr ApplyLayout L = apply_layout(sizeof(T));
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + 2 * L.stage);
    const int tid = threadIdx.x;
    const int G = gridDim.x;
    int t0 = blockIdx.x;
    if (t0 >= ntiles) return;
    if (tid == 0) {
        prefetch_tmap(&mw);
        prefetch_tmap(&mx);
        prefetch_tmap(&md);
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int s) {
        const int u0 = (t % ntx) * kApplyTW, v0 = (t / ntx) * TH;
        unsigned char* st = smem + s * L.stage;
        mbar_arrive_expect_tx(&full[s], L.bytes);
        tma_load_3d(st + L.w_off, &mw, u0 - 8, v0 - 2, 0, &full[s]);
        tma_load_2d(st + L.x_off, &mx, u0 - 8, v0 - 2, &full[s]);
        tma_load_2d(st + L.d_off, &md, u0, v0, &full[s]);
    };
    if (tid == 0) {
        issue(t0, 0);
        if (t0 + G < ntiles) issue(t0 + G, 1);
    }
    const int cp = tid & 63, rg = tid >> 6;
    const int lu = 8 + 2 * cp;  // box column of the pair's first pixel
    constexpr int PW = (TH + 2) * kApplyBoxW;  // elements per band plane in the box
    int s = 0;
    uint32_t phase = 0u;  // bit s: parity of stage s
    for (int t = t0; t < ntiles; t += G) {
        if (!mbar_wait_bounded(&full[s], (phase >> s) & 1u, gb, limit_ns)) return;
        phase ^= 1u << s;
        const unsigned char* st = smem + s * L.stage;
        const T* wb = reinterpret_cast<const T*>(st + L.w_off);
        const float* xb = reinterpret_cast<const float*>(st + L.x_off);
        const float* db = reinterpret_cast<const float*>(st + L.d_off);
        const int u0 = (t % ntx) * kApplyTW, v0 = (t / ntx) * TH;
        const int r0 = rg * RPT;
        // x window: rows r-2 .. r+2 of output row r, columns lu-2 .. lu+3.
        float xw[5][6];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float* xr = xb + (r0 + j) * kApplyBoxW + lu - 2;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float2 q = *reinterpret_cast<const float2*>(xr + 2 * c);
                xw[j + 1][2 * c] = q.x;
                xw[j + 1][2 * c + 1] = q.y;
            }
        }
#pragma unroll
        for (int rr = 0; rr < RPT; ++rr) {
            const int r = r0 + rr;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int c = 0; c < 6; ++c) xw[j][c] = xw[j + 1][c];
            {
                const float* xr = xb + (r + 4) * kApplyBoxW + lu - 2;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float2 q = *reinterpret_cast<const float2*>(xr + 2 * c);
                    xw[4][2 * c] = q.x;
                    xw[4][2 * c + 1] = q.y;
                }
            }
            const float2 dg = *reinterpret_cast<const float2*>(db + r * kApplyTW + 2 * cp);
            const float xi0 = xw[2][2], xi1 = xw[2][3];
            // two independent accumulation chains per pixel
            float a0[2] = {0.f, 0.f}, a1[2] = {0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= 12; ++k) {
                const int dv = (k + 2) / 5, du = k - 5 * dv;
                const T* pk = wb + (k - 1) * PW;
                const float2 wo = ld_pair<T>(pk + (r + 2) * kApplyBoxW + lu);
                const T* pm = pk + (r + 2 - dv) * kApplyBoxW + lu - du;
                const float wm0 = ld_one<T>(pm), wm1 = ld_one<T>(pm + 1);
                const float xf0 = xw[2 + dv][2 + du], xf1 = xw[2 + dv][3 + du];
                const float xb0 = xw[2 - dv][2 - du], xb1 = xw[2 - dv][3 - du];
                if (TRUE_OP) {
                    a0[k & 1] = fmaf(wo.x, xi0 - xf0, a0[k & 1]);
                    a1[k & 1] = fmaf(wo.y, xi1 - xf1, a1[k & 1]);
                    a0[k & 1] = fmaf(wm0, xi0 - xb0, a0[k & 1]);
                    a1[k & 1] = fmaf(wm1, xi1 - xb1, a1[k & 1]);
                } else {
                    a0[k & 1] = fmaf(wo.x, xf0, a0[k & 1]);
                    a1[k & 1] = fmaf(wo.y, xf1, a1[k & 1]);
                    a0[k & 1] = fmaf(wm0, xb0, a0[k & 1]);
                    a1[k & 1] = fmaf(wm1, xb1, a1[k & 1]);
                }
            }
            float y0, y1;
            if (TRUE_OP) {
                y0 = fmaf(dg.x, xi0, a0[0] + a0[1]);
                y1 = fmaf(dg.y, xi1, a1[0] + a1[1]);
            } else {
                y0 = fmaf(dg.x, xi0, -(a0[0] + a0[1]));
                y1 = fmaf(dg.y, xi1, -(a1[0] + a1[1]));
            }
            const int u = u0 + 2 * cp, v = v0 + r;
            if (v < H) {
                float* yr = y + (size_t)v * ypitch + u;
                if (u + 1 < W) __stcs(reinterpret_cast<float2*>(yr), make_float2(y0, y1));
                else if (u < W) __stcs(yr, y0);
            }
        }
        __syncthreads();  // every thread is done with stage s
        if (tid == 0 && t + 2 * G < ntiles) issue(t + 2 * G, s);
        s ^= 1;
    }
}

__device__ GridBarrier g_apply_state;  // receives the bounded waits' verdict

}  // namespace gm

using namespace gm;

namespace {

template <class T, bool TRUE_OP>
int launch_apply(const CUtensorMap& mw, const CUtensorMap& mx, const CUtensorMap& md, float* y, int ypitch, int W,
                 int H, cudaStream_t st)
{
    constexpr ApplyLayout L = apply_layout(sizeof(T));
    constexpr int TH = apply_rows(sizeof(T));
    static int attr_done[64] = {};
    static int nsm_cache[64] = {};
    int dev = 0;
    GM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { gm_set_error_msg("device index out of range"); return GM_ERR_INVALID; }
    if (!attr_done[dev]) {
        GM_CUDA_TRY(cudaFuncSetAttribute(levin_apply_kernel<T, TRUE_OP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         L.total));
        GM_CUDA_TRY(cudaDeviceGetAttribute(&nsm_cache[dev], cudaDevAttrMultiProcessorCount, dev));
        attr_done[dev] = 1;
    }
    GridBarrier* gb = nullptr;
    GM_CUDA_TRY(cudaGetSymbolAddress((void**)&gb, g_apply_state));
    const int ntx = (W + kApplyTW - 1) / kApplyTW;
    const int nty = (H + TH - 1) / TH;
    const int ntiles = ntx * nty;
    const int grid = ntiles < nsm_cache[dev] ? ntiles : nsm_cache[dev];
    levin_apply_kernel<T, TRUE_OP><<<grid, kApplyThreads, L.total, st>>>(mw, mx, md, y, ypitch, W, H, ntx, ntiles, gb,
                                                                          2000000000ull);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

}  // namespace

extern "C" int gm_levin_apply(const gm_levin_store* stv, const float* x, int xpitch, float* y, int ypitch, int which,
                              void* stream)
{
    if (!stv || !stv->w32 || !x || !y || (which != 0 && which != 1)) {
        gm_set_error_msg("gm_levin_apply: bad arguments");
        return GM_ERR_INVALID;
    }
    const int W = stv->W, H = stv->H, P = stv->pitch;
    if (xpitch < W || ypitch < W || (xpitch * 4) % 16 || ((uintptr_t)x & 15) || (ypitch & 1) || ((uintptr_t)y & 7)) {
        gm_set_error_msg("gm_levin_apply: x needs a 16-byte aligned base and a pitch >= W that is a multiple of 4 "
                         "floats; y an 8-byte aligned base and an even pitch >= W");
        return GM_ERR_INVALID;
    }
    GM_TRY(gm_check_device(nullptr));
    const bool true_op = which == 1;
    const int prec = true_op ? GM_PREC_FP32 : stv->precision;
    const int es = prec == GM_PREC_FP32 ? 4 : 2;
    const int th = apply_rows(es);
    const CUtensorMapDataType dt = prec == GM_PREC_FP16   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                   : prec == GM_PREC_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                          : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const void* wbase = true_op || prec == GM_PREC_FP32 ? (const void*)stv->w32 : stv->w;
    const float* dbase = true_op ? stv->gamma : (prec == GM_PREC_FP32 ? stv->d32 : stv->d);
    CUtensorMap mw, mx, md;
    {
        const uint64_t d3[3] = {(uint64_t)W, (uint64_t)H, 12};
        const uint64_t ps = stv->plane_stride ? (uint64_t)stv->plane_stride : (uint64_t)H * P;
        const uint64_t s3[2] = {(uint64_t)P * es, ps * es};
        const uint32_t b3[3] = {(uint32_t)kApplyBoxW, (uint32_t)(th + 2), 12};
        GM_TRY(gm_make_tmap(&mw, dt, 3, const_cast<void*>(wbase), d3, s3, b3));
    }
    {
        const uint64_t d2[2] = {(uint64_t)W, (uint64_t)H};
        const uint64_t s2[1] = {(uint64_t)xpitch * 4};
        const uint32_t b2[2] = {(uint32_t)kApplyBoxW, (uint32_t)(th + 4)};
        GM_TRY(gm_make_tmap(&mx, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(x), d2, s2, b2));
    }
    {
        const uint64_t d2[2] = {(uint64_t)W, (uint64_t)H};
        const uint64_t s2[1] = {(uint64_t)P * 4};
        const uint32_t b2[2] = {(uint32_t)kApplyTW, (uint32_t)th};
        GM_TRY(gm_make_tmap(&md, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(dbase), d2, s2, b2));
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (true_op) return launch_apply<float, true>(mw, mx, md, y, ypitch, W, H, st);
    if (prec == GM_PREC_FP16) return launch_apply<__half, false>(mw, mx, md, y, ypitch, W, H, st);
    if (prec == GM_PREC_BF16) return launch_apply<__nv_bfloat16, false>(mw, mx, md, y, ypitch, W, H, st);
    return launch_apply<float, false>(mw, mx, md, y, ypitch, W, H, st);
}
