// gm_vector.cu -- reference vector API (Vector.cu) on sm_100a.
//
// Allocation mirrors Vector.cu:23-46 (zeroed, padded, pointer at element
// 0).  The dot product replaces innerProd_k (Vector.cu:195-265), whose
// blocks race on zeroing the result while others add into it: here every
// block writes an FP64 partial and a single-warp pass adds them in block
// order, so the result is deterministic and exact to FP64 rounding.
#include <climits>

#include "gm_internal.cuh"

int gm_note_status(int s);

namespace gm {

constexpr int kVecThreads = 256;

__global__ void vec_axpby_kernel(float* __restrict__ out, const float* __restrict__ x, const float* __restrict__ y,
                                 float a, float b, const float* __restrict__ dev_scale, int n)
{
    const float s = dev_scale ? *dev_scale : a;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = y ? s * x[i] + b * y[i] : s * x[i];
}

// Grid-stride loops index with 64 bits: n may come within one stride of
// INT_MAX, where a 32-bit i + stride would overflow.
__global__ void dot_partial_kernel(const float* __restrict__ x, const float* __restrict__ y, int n, double* part)
{
    __shared__ double red[32];
    double acc[1] = {0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        acc[0] += (double)x[i] * (double)y[i];
    block_sum<1>(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

__global__ void dot_finish_kernel(const double* part, int nparts, float* outf, double* outd)
{
    __shared__ double red[32];
    double t[1];
    grid_total<1>(part, nparts, t, red);
    if (threadIdx.x == 0) {
        if (outf) *outf = (float)t[0];
        if (outd) *outd = t[0];
    }
}

__global__ void mse_partial_kernel(const float* __restrict__ a, const float* __restrict__ g, int n, double* part)
{
    __shared__ double red[32];
    double acc[1] = {0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float av = a[i], gv = g[i];
        float d;
        if (av > 1.0f) d = 1.0f - gv;       // main.cu:567-572
        else if (av < 0.0f) d = gv;
        else d = av - gv;
        acc[0] += (double)(d * d);
    }
    block_sum<1>(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

int dot_blocks(int n)
{
    int nsm = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int nb = (n + kVecThreads * 4 - 1) / (kVecThreads * 4);
    if (nb > 4 * nsm) nb = 4 * nsm;
    if (nb < 1) nb = 1;
    return nb;
}

// Two-pass deterministic dot using caller-provided scratch of >= nb doubles.
int dot_with_scratch(const float* x, const float* y, int n, double* scratch, int nb, float* outf, double* outd,
                     cudaStream_t st)
{
    dot_partial_kernel<<<nb, kVecThreads, 0, st>>>(x, y, n, scratch);
    dot_finish_kernel<<<1, 32, 0, st>>>(scratch, nb, outf, outd);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

}  // namespace gm

using namespace gm;

static int vec_launch(float* out, const float* x, const float* y, float a, float b, const float* ds, int n,
                      void* stream)
{
    if (n < 0 || (n > 0 && (!out || !x))) { gm_set_error_msg("bad vector arguments"); return GM_ERR_INVALID; }
    if (n == 0) return GM_OK;
    int nb = (n + kVecThreads - 1) / kVecThreads;
    if (nb > 148 * 8) nb = 148 * 8;
    vec_axpby_kernel<<<nb, kVecThreads, 0, (cudaStream_t)stream>>>(out, x, y, a, b, ds, n);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_vec_add(float* r, const float* x, const float* y, int n, void* s) { return vec_launch(r, x, y, 1.f, 1.f, nullptr, n, s); }
extern "C" int gm_vec_sub(float* r, const float* x, const float* y, int n, void* s) { return vec_launch(r, x, y, 1.f, -1.f, nullptr, n, s); }
extern "C" int gm_vec_scale_const(float* r, const float* x, float a, int n, void* s) { return vec_launch(r, x, nullptr, a, 0.f, nullptr, n, s); }
extern "C" int gm_vec_scale(float* r, const float* x, const float* a, int n, void* s)
{
    if (!a) { gm_set_error_msg("device scale is NULL"); return GM_ERR_INVALID; }
    return vec_launch(r, x, nullptr, 0.f, 0.f, a, n, s);
}

static int inner_prod_impl(float* rf, double* rd, const float* x, const float* y, int len, void* stream)
{
    if (len < 0 || (!rf && !rd)) { gm_set_error_msg("bad inner product arguments"); return GM_ERR_INVALID; }
    cudaStream_t st = (cudaStream_t)stream;
    if (len == 0) {
        if (rf) GM_CUDA_TRY(cudaMemsetAsync(rf, 0, sizeof(float), st));
        if (rd) GM_CUDA_TRY(cudaMemsetAsync(rd, 0, sizeof(double), st));
        return GM_OK;
    }
    if (!x || !y) { gm_set_error_msg("NULL vector"); return GM_ERR_INVALID; }
    const int nb = dot_blocks(len);
    double* scratch = nullptr;
    GM_CUDA_TRY(gm_scratch_alloc((void**)&scratch, sizeof(double) * nb, st));
    int rc = dot_with_scratch(x, y, len, scratch, nb, rf, rd, st);
    cudaFreeAsync(scratch, st);
    return rc;
}

extern "C" int gm_inner_prod(float* result, const float* x, const float* y, int len, void* stream)
{
    return inner_prod_impl(result, nullptr, x, y, len, stream);
}

extern "C" int gm_inner_prod_f64(double* result, const float* x, const float* y, int len, void* stream)
{
    return inner_prod_impl(nullptr, result, x, y, len, stream);
}

extern "C" int gm_compute_error(double* mse_host, const float* alpha, const float* gt, int W, int H, void* stream)
{
    if (!mse_host || !alpha || !gt || W <= 0 || H <= 0) { gm_set_error_msg("bad compute_error arguments"); return GM_ERR_INVALID; }
    if ((long long)W * H > INT_MAX) {
        gm_set_error_msg("compute_error: W*H = %lld exceeds INT_MAX", (long long)W * H);
        return GM_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int n = W * H;
    const int nb = dot_blocks(n);
    double* scratch = nullptr;
    GM_CUDA_TRY(gm_scratch_alloc((void**)&scratch, sizeof(double) * (nb + 1), st));
    mse_partial_kernel<<<nb, kVecThreads, 0, st>>>(alpha, gt, n, scratch);
    dot_finish_kernel<<<1, 32, 0, st>>>(scratch, nb, nullptr, scratch + nb);
    double ssd = 0.0;
    cudaError_t e = cudaMemcpyAsync(&ssd, scratch + nb, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { gm_set_error_msg("compute_error: %s", cudaGetErrorString(e)); return GM_ERR_CUDA; }
    *mse_host = ssd / ((double)W * H);
    return GM_OK;
}

// ---- drop-ins (Vector.cu:23-46) ----
extern "C" void vecDeviceMalloc(float** dx, int length, int leftPadding, int rightPadding)
{
    if (!dx || length < 0 || leftPadding < 0 || rightPadding < 0) {
        gm_set_error_msg("vecDeviceMalloc: bad arguments");
        gm_note_status(GM_ERR_INVALID);
        return;
    }
    const size_t n = (size_t)length + leftPadding + rightPadding;
    float* p = nullptr;
    if (cudaMalloc((void**)&p, sizeof(float) * (n ? n : 1)) != cudaSuccess) {
        *dx = nullptr;
        gm_set_error_msg("vecDeviceMalloc: cudaMalloc of %zu floats failed", n);
        gm_note_status(GM_ERR_NOMEM);
        return;
    }
    cudaMemset(p, 0, sizeof(float) * (n ? n : 1));
    *dx = p + leftPadding;
    gm_note_status(GM_OK);
}

extern "C" void vecCopyToDevice(float** dx, const float* hx, int length, int leftPadding, int rightPadding)
{
    vecDeviceMalloc(dx, length, leftPadding, rightPadding);
    if (gm_last_status() != GM_OK) return;
    if (length > 0 && cudaMemcpy(*dx, hx, sizeof(float) * length, cudaMemcpyHostToDevice) != cudaSuccess) {
        gm_set_error_msg("vecCopyToDevice: copy failed");
        gm_note_status(GM_ERR_CUDA);
    }
}

extern "C" void vecDeviceFree(float* dx, int leftPadding)
{
    if (dx) cudaFree(dx - leftPadding);
    gm_note_status(GM_OK);
}

extern "C" void computeError(float* alpha, float* gtAlpha, int imW, int imH)
{
    const size_t n = (size_t)imW * imH;
    float* d = nullptr;
    double mse = 0.0;
    int rc = GM_OK;
    if (cudaMalloc((void**)&d, 2 * n * sizeof(float)) != cudaSuccess) rc = GM_ERR_NOMEM;
    if (rc == GM_OK && (cudaMemcpy(d, alpha, n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                        cudaMemcpy(d + n, gtAlpha, n * 4, cudaMemcpyHostToDevice) != cudaSuccess))
        rc = GM_ERR_CUDA;
    if (rc == GM_OK) rc = gm_compute_error(&mse, d, d + n, imW, imH, nullptr);
    if (d) cudaFree(d);
    gm_note_status(rc);
    if (rc == GM_OK) printf("Ground truth MSE: %.3e\n", mse);
}

// ---- CG building blocks over pitched row blocks (the row-slab solver) ----
//
// A host-driven CG over one slab of rows (the slab split of one image over
// several GPUs) needs, per iteration, the four FP64 sums of the single-
// reduction recurrence and one elementwise update; each is one launch here
// (plus a one-warp pass that adds the per-block sums in block order, so the
// sums are deterministic).  Rows are `rows` runs of W floats, `pitch` floats
// apart.
namespace gm {

constexpr int kCgThreads = 256;

__global__ void cg_dots4_kernel(const float* __restrict__ r, int rp, const float* __restrict__ p, int pp,
                                const float* __restrict__ q, int qp, int W, int rows, double* part)
{
    __shared__ double red[32 * 4];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long i = blockIdx.x; i < rows; i += gridDim.x) {
        const float* ri = r + i * rp;
        const float* pi = p + i * pp;
        const float* qi = q + i * qp;
        for (int j = threadIdx.x; j < W; j += blockDim.x) {
            const double rv = ri[j], pv = pi[j], qv = qi[j];
            acc[0] += rv * rv;
            acc[1] += pv * qv;
            acc[2] += rv * qv;
            acc[3] += qv * qv;
        }
    }
    block_sum<4>(acc, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) part[(size_t)k * gridDim.x + blockIdx.x] = acc[k];
}

__global__ void cg_dots4_finish(const double* part, int nb, double* out)
{
    __shared__ double red[32 * 4];
    double t[4];
    grid_total<4>(part, nb, t, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) out[k] = t[k];
}

// x += alpha p; r -= alpha q; then (update_p) p = r + beta p.
__global__ void cg_update_kernel(float* __restrict__ x, int xp, float* __restrict__ r, int rp, float* __restrict__ p,
                                 int pp, const float* __restrict__ q, int qp, int W, int rows, float alpha, float beta,
                                 int update_p)
{
    for (long long i = blockIdx.x; i < rows; i += gridDim.x) {
        float* xi = x + i * xp;
        float* ri = r + i * rp;
        float* pi = p + i * pp;
        const float* qi = q + i * qp;
        for (int j = threadIdx.x; j < W; j += blockDim.x) {
            const float pv = pi[j];
            xi[j] += alpha * pv;
            const float rn = ri[j] - alpha * qi[j];
            ri[j] = rn;
            if (update_p) pi[j] = rn + beta * pv;
        }
    }
}

// Device-side scalars of one iteration (one thread).  state: [0] threshold
// on the recurrence's next r.r (< 0: none), [1] r.r of this iteration, [2]
// the recurrence's next r.r, [3] iterations taken, [4] stop code, [5] the
// iteration count at which to stop for a residual replacement.  coef: alpha,
// beta, mode (0 nothing, 1 x and r, 2 x, r and p).
__global__ void cg_scalars_kernel(double* coef, double* state, const double* sums)
{
    double mode = 0.0, alpha = 0.0, beta = 0.0;
    if (state[4] == 0.0) {
        const double rr = sums[0], pq = sums[1], rq = sums[2], qq = sums[3];
        if (!(pq > 0.0) || rr != rr) {
            state[4] = 2.0;
        } else {
            alpha = rr / pq;
            const double nx = fmax(rr - 2.0 * alpha * rq + alpha * alpha * qq, 0.0);
            const double it = state[3] + 1.0;
            state[1] = rr;
            state[2] = nx;
            state[3] = it;
            if ((state[0] >= 0.0 && nx <= state[0]) || it >= state[5]) {
                state[4] = 1.0;
                mode = 1.0;
            } else {
                beta = nx / rr;
                mode = 2.0;
            }
        }
    }
    coef[0] = alpha;
    coef[1] = beta;
    coef[2] = mode;
}

// gm_cg_update with the coefficients read from the device.
__global__ void cg_update_dev_kernel(float* __restrict__ x, int xp, float* __restrict__ r, int rp,
                                     float* __restrict__ p, int pp, const float* __restrict__ q, int qp, int W,
                                     int rows, const double* __restrict__ coef)
{
    const double mode = coef[2];
    if (mode == 0.0) return;
    const float alpha = (float)coef[0], beta = (float)coef[1];
    const bool update_p = mode == 2.0;
    for (long long i = blockIdx.x; i < rows; i += gridDim.x) {
        float* xi = x + i * xp;
        float* ri = r + i * rp;
        float* pi = p + i * pp;
        const float* qi = q + i * qp;
        for (int j = threadIdx.x; j < W; j += blockDim.x) {
            const float pv = pi[j];
            xi[j] += alpha * pv;
            const float rn = ri[j] - alpha * qi[j];
            ri[j] = rn;
            if (update_p) pi[j] = rn + beta * pv;
        }
    }
}

static int cg_blocks(int rows)
{
    int nsm = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return rows < 4 * nsm ? (rows > 0 ? rows : 1) : 4 * nsm;
}

static int check_block(const void* a, int pitch, int W, const char* name)
{
    if (!a || pitch < W) {
        gm_set_error_msg("%s: NULL or pitch %d < W %d", name, pitch, W);
        return GM_ERR_INVALID;
    }
    return GM_OK;
}

}  // namespace gm

extern "C" int gm_cg_dots4(double* out4, const float* r, int r_pitch, const float* p, int p_pitch, const float* q,
                           int q_pitch, int W, int rows, void* stream)
{
    if (!out4 || W < 0 || rows < 0) {
        gm_set_error_msg("gm_cg_dots4: bad arguments");
        return GM_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if ((long long)W * rows == 0) {
        GM_CUDA_TRY(cudaMemsetAsync(out4, 0, 4 * sizeof(double), st));
        return GM_OK;
    }
    GM_TRY(gm::check_block(r, r_pitch, W, "r"));
    GM_TRY(gm::check_block(p, p_pitch, W, "p"));
    GM_TRY(gm::check_block(q, q_pitch, W, "q"));
    const int nb = gm::cg_blocks(rows);
    double* part = nullptr;
    GM_CUDA_TRY(gm_scratch_alloc((void**)&part, sizeof(double) * 4 * nb, st));
    gm::cg_dots4_kernel<<<nb, gm::kCgThreads, 0, st>>>(r, r_pitch, p, p_pitch, q, q_pitch, W, rows, part);
    gm::cg_dots4_finish<<<1, 128, 0, st>>>(part, nb, out4);
    cudaFreeAsync(part, st);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_cg_update(float* x, int x_pitch, float* r, int r_pitch, float* p, int p_pitch, const float* q,
                            int q_pitch, int W, int rows, float alpha, float beta, int update_p, void* stream)
{
    if (W < 0 || rows < 0) {
        gm_set_error_msg("gm_cg_update: bad arguments");
        return GM_ERR_INVALID;
    }
    if ((long long)W * rows == 0) return GM_OK;
    GM_TRY(gm::check_block(x, x_pitch, W, "x"));
    GM_TRY(gm::check_block(r, r_pitch, W, "r"));
    GM_TRY(gm::check_block(p, p_pitch, W, "p"));
    GM_TRY(gm::check_block(q, q_pitch, W, "q"));
    gm::cg_update_kernel<<<gm::cg_blocks(rows), gm::kCgThreads, 0, (cudaStream_t)stream>>>(
        x, x_pitch, r, r_pitch, p, p_pitch, q, q_pitch, W, rows, alpha, beta, update_p);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_cg_scalars(double* coef, double* state, const double* sums4, void* stream)
{
    if (!coef || !state || !sums4) {
        gm_set_error_msg("gm_cg_scalars: NULL argument");
        return GM_ERR_INVALID;
    }
    gm::cg_scalars_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(coef, state, sums4);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_cg_update_dev(float* x, int x_pitch, float* r, int r_pitch, float* p, int p_pitch,
                                const float* q, int q_pitch, int W, int rows, const double* coef, void* stream)
{
    if (W < 0 || rows < 0 || !coef) {
        gm_set_error_msg("gm_cg_update_dev: bad arguments");
        return GM_ERR_INVALID;
    }
    if ((long long)W * rows == 0) return GM_OK;
    GM_TRY(gm::check_block(x, x_pitch, W, "x"));
    GM_TRY(gm::check_block(r, r_pitch, W, "r"));
    GM_TRY(gm::check_block(p, p_pitch, W, "p"));
    GM_TRY(gm::check_block(q, q_pitch, W, "q"));
    gm::cg_update_dev_kernel<<<gm::cg_blocks(rows), gm::kCgThreads, 0, (cudaStream_t)stream>>>(
        x, x_pitch, r, r_pitch, p, p_pitch, q, q_pitch, W, rows, coef);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

// ---- allocation-free dot product ----
//
// For callers that may not allocate device memory while they run: code that
// hands all device memory to its own allocator or runs under a fixed memory
// budget, and latency-critical loops where a stream-ordered allocation that
// grows the pool would stall.  The partial sums live in a fixed file-scope
// device array instead of a cudaMallocAsync buffer.  Every block writes its
// own slot before the finishing pass reads it, so nothing has to start at
// zero.  Calls that overlap in time on one device (different streams or
// host threads) share the array and race; serialise them.
namespace gm {
constexpr int kStaticDotParts = 4096;  // 32 KB of partials per device
__device__ __align__(256) double g_static_dot_parts[kStaticDotParts];
}  // namespace gm

#include <mutex>

// Device address of the static partials in the current context of device
// dev.  Resolved once per context: a cudaDeviceReset (or any new context on
// the same ordinal) changes the context id and the address is looked up
// again, so a stale address from a destroyed context is never used.
static double* static_dot_parts(int dev)
{
    constexpr int kMaxDevices = 64;
    struct Entry { unsigned long long ctx; double* addr; };
    static std::mutex mu;
    static Entry cache[kMaxDevices] = {};
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    const unsigned long long ctx = gm_context_id();
    std::lock_guard<std::mutex> lock(mu);
    Entry& e = cache[dev];
    if (!e.addr || ctx == 0 || e.ctx != ctx) {
        void* p = nullptr;
        // The current device is dev, so the symbol resolves in its context
        // (the runtime makes the primary context current here if no call
        // has yet); the id is read again once that context exists.
        if (cudaGetSymbolAddress(&p, gm::g_static_dot_parts) != cudaSuccess) return nullptr;
        e.addr = static_cast<double*>(p);
        e.ctx = gm_context_id();
    }
    return e.addr;
}

extern "C" int gm_inner_prod_f64_noalloc(double* result, const float* x, const float* y, int len, void* stream)
{
    if (len < 0 || !result) { gm_set_error_msg("bad inner product arguments"); return GM_ERR_INVALID; }
    cudaStream_t st = (cudaStream_t)stream;
    if (len == 0) {
        GM_CUDA_TRY(cudaMemsetAsync(result, 0, sizeof(double), st));
        return GM_OK;
    }
    if (!x || !y) { gm_set_error_msg("NULL vector"); return GM_ERR_INVALID; }
    int dev = 0;
    GM_CUDA_TRY(cudaGetDevice(&dev));
    const int nb = dot_blocks(len);
    if (nb > kStaticDotParts) {
        gm_set_error_msg("inner product needs %d partial sums; the static scratch holds %d", nb, kStaticDotParts);
        return GM_ERR_INVALID;
    }
    double* parts = static_dot_parts(dev);
    if (!parts) {
        cudaGetLastError();
        gm_set_error_msg("cannot resolve the static dot-product scratch on device %d", dev);
        return GM_ERR_CUDA;
    }
    return dot_with_scratch(x, y, len, parts, nb, nullptr, result, st);
}
