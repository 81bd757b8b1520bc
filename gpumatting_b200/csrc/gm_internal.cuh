// gm_internal.cuh -- shared device and host helpers of libgpumat.
//
// Device side: TMA (cp.async.bulk.tensor) row loads completed on mbarriers,
// a grid barrier with a wall-clock limit, and deterministic FP64 block
// reductions.  Host side: status plumbing and tensor-map encoding through the
// driver entry point (no libcuda link needed).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/gpumat.h"

#define GM_CUDA_TRY(expr)                                                     \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) {                                              \
            gm_set_error_msg("%s:%d: %s: %s", __FILE__, __LINE__, #expr,      \
                             cudaGetErrorString(_e));                         \
            return GM_ERR_CUDA;                                               \
        }                                                                     \
    } while (0)

#define GM_TRY(expr)                                                          \
    do {                                                                      \
        int _s = (expr);                                                      \
        if (_s != GM_OK) return _s;                                           \
    } while (0)

// Records a message for gm_last_error() (thread-local).
void gm_set_error_msg(const char* fmt, ...);

// Checks that the current device is sm_100 class; returns GM_ERR_UNSUPPORTED
// otherwise.
int gm_check_device(int* sm_count);

// The driver's identifier of the current context (unique for the life of
// the process, never reused), or 0 when the driver cannot say.
unsigned long long gm_context_id();

// Stream-ordered scratch from a library-owned pool that stays mapped across
// synchronisations (free with cudaFreeAsync).
cudaError_t gm_scratch_alloc(void** p, size_t bytes, cudaStream_t st);

// ---------------------------------------------------------------------------
// Tensor maps
// ---------------------------------------------------------------------------

// Encodes a tiled tensor map of rank 2 or 3 (dims innermost first, strides
// in bytes for dims 1..rank-1) with zero out-of-bounds fill and no swizzle.
int gm_make_tmap(CUtensorMap* map, CUtensorMapDataType dtype, int rank, void* base,
                 const uint64_t* dims, const uint64_t* strides_bytes,
                 const uint32_t* box);

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
namespace gm {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Orders this thread's earlier generic-proxy accesses (shared and global)
// before its later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile_int(const int* p)
{
    return *reinterpret_cast<const volatile int*>(p);
}

// Grid barrier state, zeroed before the launch.  `abort` carries the first
// error any CTA raised (GM_ERR_TIMEOUT from a wait that hit its limit, or a
// solver status); every wait also returns once it is set.
struct GridBarrier {
    unsigned long long count;  // arrivals so far in this launch (only grows)
    int abort;
    int where;  // which wait gave up: 1 = grid barrier, 2 = TMA row wait
};

__device__ __forceinline__ unsigned long long atom_add_release_u64(unsigned long long* p, unsigned long long v)
{
    unsigned long long old;
    asm volatile("atom.release.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Arrival half of the grid barrier, run by one thread per CTA.  The arrival
// counter only grows during a launch (it is zeroed before the launch): an
// arrival whose atomic returns `old` belongs to round old / G, which is
// complete once the count reaches (old / G + 1) * G, and `extra` more
// arrivals are awaited on top of that (the test hook's arrival that never
// comes).  Every CTA arrives once per round, so no CTA can start round k+1
// before the round-k arrival of every other CTA has landed.  The atomic's
// release covers every write the CTA made before the caller's
// __syncthreads; the acquire loads of the spin order the caller's later
// reads after all of them.  Compared with a last-arriver flag this saves the
// last arrival's round trip and the flag store (4.2 -> 3.0 us per barrier and
// all-reduce with 440 CTAs).  Returns 0 when the wait was abandoned (limit
// reached or abort set by any CTA).
__device__ __forceinline__ int grid_arrive_wait(GridBarrier* gb, unsigned G, uint64_t limit_ns, unsigned extra = 0u)
{
    const unsigned long long old = atom_add_release_u64(&gb->count, 1ull);
    const unsigned long long target = (old / G + 1ull) * G + extra;
    uint64_t t0 = 0;
    unsigned spins = 0;
    while (ld_acquire_u64(&gb->count) < target) {
        ++spins;
        if ((spins & 7u) == 0 && ld_volatile_int(&gb->abort)) return 0;
        if ((spins & 63u) == 0) {
            const uint64_t now = globaltimer_ns();
            if (t0 == 0) t0 = now;
            else if (now - t0 > limit_ns) {
                atomicCAS(&gb->abort, 0, (int)GM_ERR_TIMEOUT);
                atomicExch(&gb->where, 1);
                return 0;
            }
        }
    }
    return 1;
}

// All CTAs of the grid call this the same number of times.  Returns false
// when the barrier was abandoned (limit reached or abort set by any CTA).
__device__ __forceinline__ bool grid_sync(GridBarrier* gb, unsigned G, uint64_t limit_ns, unsigned extra = 0u)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = grid_arrive_wait(gb, G, limit_ns, extra);
        if (ld_volatile_int(&gb->abort)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// try_wait with a suspend-time hint: the warp parks in hardware until the
// phase completes or about hint_ns pass, instead of spinning.
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t hint_ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Waits for the mbarrier phase with a wall-clock limit; on expiry raises
// GM_ERR_TIMEOUT in the grid barrier state and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, GridBarrier* gb,
                                                  uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = globaltimer_ns();
    unsigned spins = 0;
    while (!mbar_try_wait_hint(bar, parity, 100000u)) {
        if ((++spins & 15u) == 0 && globaltimer_ns() - t0 > limit_ns) {
            atomicCAS(&gb->abort, 0, (int)GM_ERR_TIMEOUT);
            atomicExch(&gb->where, 2);
            return false;
        }
    }
    return true;
}

// Deterministic block sum of NV doubles: fixed shuffle tree per warp, then
// warp 0 adds the warp sums in warp order.  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch /* >= 32*NV */)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) scratch[wid * NV + k] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? scratch[lane * NV + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

// Sums the per-CTA partials p[k * n + i] (i < n) of each component k in a
// fixed order: thread t adds entries t, t + T, t + 2T, ... (T = blockDim.x),
// then a fixed shuffle tree and the warp sums in warp order.  Every CTA that
// calls this on the same data gets bit-identical results.  All loads are
// independent and coalesced; they bypass L1 (other CTAs wrote the data).
template <int NV>
__device__ __forceinline__ void grid_total(const double* p, int n, double (&out)[NV], double* scratch /* >= 32*NV */)
{
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    const int T = blockDim.x;
    int i = threadIdx.x;
    for (; i + T < n; i += 2 * T) {
        double a[NV], b[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            a[k] = __ldcg(p + (size_t)k * n + i);
            b[k] = __ldcg(p + (size_t)k * n + i + T);
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += a[k] + b[k];
    }
    if (i < n) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += __ldcg(p + (size_t)k * n + i);
    }
    block_sum<NV>(v, scratch);
    __shared__ double bc[NV];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) bc[k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = bc[k];
    __syncthreads();
}

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Sum of p[lo .. hi-1] by one warp in a fixed order: lane l adds entries
// l, l+32, l+64, ... in index order, then a fixed shuffle tree.  Every warp
// that calls it on the same data gets the same bits (result in all lanes).
// The loads of a chunk of 32 * 16 entries are all issued before any add, so a
// grid's partials (<= 512 per component) cost one L2 round trip.
__device__ __forceinline__ double warp_sum_range(const double* p, int lo, int hi)
{
    const int lane = threadIdx.x & 31;
    constexpr int kU = 16;
    double x = 0.0;
    for (int base = lo; base < hi; base += 32 * kU) {
        double v[kU];
#pragma unroll
        for (int j = 0; j < kU; ++j) {
            const int i = base + lane + 32 * j;
            v[j] = i < hi ? __ldcg(p + i) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < kU; ++j) x += v[j];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    return __shfl_sync(0xffffffffu, x, 0);
}

// Grid barrier fused with a deterministic all-reduce of NV doubles per
// thread.  On return every thread of every CTA holds the same bit-identical
// grid totals in v.  parts is [NV][G] global scratch for this call (callers
// alternate two copies so a fast CTA's next call cannot overwrite partials a
// slow CTA is still reading).  scratch: >= (warps + 1) * NV shared doubles.
// Components with index < NSEG are summed over CTAs lo .. hi-1 only (the
// CTAs of one image in a batched solve), the others over the whole grid.
// Warp 0 publishes the CTA sums and waits on the grid; after the release
// each warp sums its components (k = warp, warp + nwarps, ...) with all of
// its loads in flight at once.  Three __syncthreads per call.  Returns false
// when the barrier was abandoned (limit reached or abort set by any CTA).
template <int NV, int NSEG>
__device__ __forceinline__ bool grid_allreduce_impl(GridBarrier* gb, double* parts, unsigned G, int lo, int hi,
                                                    uint64_t limit_ns, double (&v)[NV], double* scratch)
{
    __shared__ int s_ok;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) scratch[wid * NV + k] = x;
    }
    __syncthreads();
    if (wid == 0) {
        double cs[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? scratch[lane * NV + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            cs[k] = x;
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) parts[(size_t)k * G + blockIdx.x] = cs[k];
            s_ok = grid_arrive_wait(gb, G, limit_ns);
        }
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    if (ok) {
        for (int k = wid; k < NV; k += nw) {
            const double t = k < NSEG ? warp_sum_range(parts + (size_t)k * G, lo, hi)
                                      : warp_sum_range(parts + (size_t)k * G, 0, (int)G);
            if (lane == 0) scratch[nw * NV + k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = scratch[nw * NV + k];
    return ok;
}

template <int NV>
__device__ __forceinline__ bool grid_allreduce(GridBarrier* gb, double* parts, unsigned G, uint64_t limit_ns,
                                               double (&v)[NV], double* scratch)
{
    return grid_allreduce_impl<NV, 0>(gb, parts, G, 0, (int)G, limit_ns, v, scratch);
}

// Batched form: components 0 .. NV-2 over the CTAs lo .. hi-1 (one image;
// lo == hi gives zeros), component NV-1 over the whole grid.
template <int NV>
__device__ __forceinline__ bool grid_allreduce_seg(GridBarrier* gb, double* parts, unsigned G, int lo, int hi,
                                                   uint64_t limit_ns, double (&v)[NV], double* scratch)
{
    return grid_allreduce_impl<NV, NV - 1>(gb, parts, G, lo, hi, limit_ns, v, scratch);
}

template <class T> struct Cvt;
template <> struct Cvt<float> {
    static __device__ __forceinline__ float to_f(float x) { return x; }
};
template <> struct Cvt<__half> {
    static __device__ __forceinline__ float to_f(__half x) { return __half2float(x); }
};
template <> struct Cvt<__nv_bfloat16> {
    static __device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
};

}  // namespace gm
