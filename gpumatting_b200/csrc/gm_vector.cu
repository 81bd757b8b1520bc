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
    GM_CUDA_TRY(cudaMallocAsync((void**)&scratch, sizeof(double) * nb, st));
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
    GM_CUDA_TRY(cudaMallocAsync((void**)&scratch, sizeof(double) * (nb + 1), st));
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

// The driver's identifier of the current context (unique for the life of
// the process, never reused), or 0 when the driver cannot say.
static unsigned long long current_context_id()
{
    typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
    typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)p;
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)p;
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

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
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(mu);
    Entry& e = cache[dev];
    if (!e.addr || ctx == 0 || e.ctx != ctx) {
        void* p = nullptr;
        // The current device is dev, so the symbol resolves in its context
        // (the runtime makes the primary context current here if no call
        // has yet); the id is read again once that context exists.
        if (cudaGetSymbolAddress(&p, gm::g_static_dot_parts) != cudaSuccess) return nullptr;
        e.addr = static_cast<double*>(p);
        e.ctx = current_context_id();
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
