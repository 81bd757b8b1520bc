// gm_common.cu -- status plumbing, device checks and tensor-map encoding.
#include <stdarg.h>
#include <string.h>

#include <mutex>

#include "gm_internal.cuh"

static thread_local char g_msg[1024] = "";
static thread_local int g_status = GM_OK;

void gm_set_error_msg(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
}

// Records the status of a drop-in (void) entry point.
int gm_note_status(int s)
{
    g_status = s;
    if (s == GM_OK) g_msg[0] = 0;
    return s;
}

extern "C" int gm_last_status(void) { return g_status; }
extern "C" const char* gm_last_error(void) { return g_msg; }
extern "C" const char* gm_version(void) { return "gpumatting_b200 0.1 (sm_100a)"; }

// The driver's identifier of the current context (unique for the life of
// the process, never reused), or 0 when the driver cannot say.
unsigned long long gm_context_id()
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

// Stream-ordered scratch for the small per-call buffers (reduction partials).
// The device's default memory pool hands freed memory back to the driver at
// every synchronisation (release threshold 0), so a caller that synchronises
// between calls -- a host-driven iteration that reads each dot product --
// would pay a fresh mapping on every call.  A pool owned by the library, one
// per device and context, with a 64 MiB release threshold keeps these
// buffers mapped.  Under stream capture, or when the context id is unknown,
// the default pool is used.
static cudaMemPool_t scratch_pool()
{
    constexpr int kMaxDevices = 64;
    struct Entry { unsigned long long ctx; cudaMemPool_t pool; };
    static std::mutex mu;
    static Entry cache[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    const unsigned long long ctx = gm_context_id();
    if (ctx == 0) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    Entry& e = cache[dev];
    if (e.pool && e.ctx == ctx) return e.pool;
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = 64ull << 20;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    e.ctx = ctx;
    e.pool = pool;
    return pool;
}

cudaError_t gm_scratch_alloc(void** p, size_t bytes, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusActive;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
        if (cudaMemPool_t pool = scratch_pool()) return cudaMallocFromPoolAsync(p, bytes, pool, st);
    }
    cudaGetLastError();
    return cudaMallocAsync(p, bytes, st);
}

int gm_check_device(int* sm_count)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        gm_set_error_msg("no CUDA device: %s", cudaGetErrorString(e));
        return GM_ERR_CUDA;
    }
    int major = 0, minor = 0, nsm = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (major != 10) {
        gm_set_error_msg("libgpumat is built for sm_100a; device %d is sm_%d%d", dev, major, minor);
        return GM_ERR_UNSUPPORTED;
    }
    if (sm_count) *sm_count = nsm;
    return GM_OK;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

static int esize_of(CUtensorMapDataType t)
{
    switch (t) {
    case CU_TENSOR_MAP_DATA_TYPE_FLOAT16:
    case CU_TENSOR_MAP_DATA_TYPE_BFLOAT16: return 2;
    case CU_TENSOR_MAP_DATA_TYPE_FLOAT32: return 4;
    case CU_TENSOR_MAP_DATA_TYPE_FLOAT64: return 8;
    default: return 1;
    }
}

int gm_make_tmap(CUtensorMap* map, CUtensorMapDataType dtype, int rank, void* base, const uint64_t* dims,
                 const uint64_t* strides_bytes, const uint32_t* box)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        gm_set_error_msg("cuTensorMapEncodeTiled is not available from the driver");
        return GM_ERR_UNSUPPORTED;
    }
    const int es = esize_of(dtype);
    if (((uintptr_t)base & 15) != 0) {
        gm_set_error_msg("tensor base %p is not 16-byte aligned", base);
        return GM_ERR_INVALID;
    }
    for (int i = 0; i < rank - 1; ++i)
        if (strides_bytes[i] % 16 != 0) {
            gm_set_error_msg("tensor stride %llu bytes is not a multiple of 16", (unsigned long long)strides_bytes[i]);
            return GM_ERR_INVALID;
        }
    if ((box[0] * es) % 16 != 0) {
        gm_set_error_msg("tensor box inner extent %u x %d bytes is not a multiple of 16", box[0], es);
        return GM_ERR_INVALID;
    }
    cuuint64_t d[5];
    cuuint64_t s[4];
    cuuint32_t b[5], e[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        b[i] = box[i];
        e[i] = 1;
    }
    for (int i = 0; i < rank - 1; ++i) s[i] = strides_bytes[i];
    CUresult r = fn(map, dtype, (cuuint32_t)rank, base, d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        gm_set_error_msg("cuTensorMapEncodeTiled failed (%d) rank %d dims %llu x %llu", (int)r, rank,
                         (unsigned long long)dims[0], (unsigned long long)dims[1]);
        return GM_ERR_INVALID;
    }
    return GM_OK;
}

extern "C" void gm_default_params(gm_solve_params* p)
{
    memset(p, 0, sizeof(*p));
    p->solver = GM_SOLVER_CG;
    p->rtol = 1e-6;
    p->max_iters = 5000;
    p->restart = 0;
    p->replace_every = 50;
    p->omega = 2.0f / 3.0f;
    p->use_low = 1;
    p->timeout_s = 5.0;
    p->ctas_per_sm = 0;
    p->strip_width = 0;
}

extern "C" void gm_levin_band_offsets(int W, int offs[25])
{
    for (int dv = -2; dv <= 2; ++dv)
        for (int du = -2; du <= 2; ++du) offs[12 + du + 5 * dv] = du + W * dv;
}

extern "C" int gm_levin_pad(int W) { return ((2 * W + 2) / 32) * 32 + 32; }
