// gm_solver.cu -- persistent fused solvers for the Levin system
//     (L + diag(gamma)) x = b
// on a W x H pixel grid: conjugate gradient, steepest descent and damped
// Jacobi (the reference's cgSolve / gradSolve / jacobi, main.cu:406-556),
// each run as ONE cooperative kernel with no host round trip per iteration.
//
// Work decomposition.  The image is cut into column strips of 64 * NCOL
// pixels and each strip into row segments; one CTA owns one (strip,
// segment) unit and sweeps down it row by row.  A CTA is one TMA producer
// warp and kConsumers consumer warps:
//   * the producer (one lane) streams, per row step, one halo'd row
//     (kStrip + 16 columns from 8 left of the strip, zero fill outside the
//     image) of the input vectors and of the band planes into shared-memory
//     rings with cp.async.bulk.tensor (no multicast), each slot guarded by a
//     "full" mbarrier (transaction bytes) and an "empty" mbarrier (one
//     arrival per consumer warp) -- no block-wide barrier inside a sweep;
//   * consumer warp w owns 64 output columns, two adjacent pixels per lane,
//     and keeps rows v-2..v+2 of the stencil operand for its columns (+2 on
//     each side) in a private 6-row ring, so only __syncwarp is needed.
// Each band and vector element is read from HBM once per sweep (plus the
// 2-row and 8-column halos, shared with neighbouring CTAs through L2).
//
// Operators.  OP_SYMD (iteration operator of the symmetric store): 12 planes
// of upper affinities w_k (k = du + 5 dv) and a diagonal plane d = gamma +
// sum of the row's rounded affinities: y_i = d_i x_i - sum_j w_ij x_j, one
// FMA per neighbour, rows still summing exactly to gamma.  OP_SYMI (true
// operator, FP64 accumulation): y_i = gamma_i x_i + sum_j w_ij (x_i - x_j).
// The lower half is read from the rows above (w_k(u-du, v-dv)).  OP_REF25:
// the reference's 25 explicit FP32 bands (main.cu:164-194).
//
// CG iteration (one sweep, one grid barrier).  Sweep k, given alpha_{k-1}
// and beta_k from the previous barrier, forms on the fly (halo included)
//   r_k = r_{k-1} - alpha_{k-1} q_{k-1},  p_k = r_k + beta_k p_{k-1},
// applies q_k = A p_k, adds alpha_{k-1} p_{k-1} into the solution
// increment, and reduces <r_k,r_k>, <p_k,q_k>, <r_k,q_k>, <q_k,q_k> in FP64.
// After the barrier every CTA sums the per-CTA partials in the same fixed
// order (bit-identical scalars everywhere): alpha_k = r.r / p.q and
// ||r_{k+1}||^2 = r.r - 2 alpha r.q + alpha^2 q.q, which gives beta_{k+1}
// without a second barrier.  Steepest descent is the same sweep with
// beta = 0 (main.cu:424-449 computes the same exact line search).
//
// Replacement sweep (every replace_every iterations, at restarts, when the
// recursive residual drops below rtol, and at exit): folds the solution in
// FP64 (x = base + increment + alpha p, halo included), recomputes the true
// residual r = b - A x with FP64 accumulation over the FP32 planes, and
// writes alpha out.  With FP16/BF16 iteration planes this is the
// reliable-update scheme that keeps the iterate converging to the FP32
// operator's solution.
//
// Every wait (grid barrier, ring slot) has a wall-clock limit; on expiry the
// kernel records GM_ERR_TIMEOUT and all CTAs leave their loops.
#include <type_traits>

#include "gm_solver.cuh"

namespace gm {

__host__ __device__ constexpr int sym_dv(int k) { return (k + 2) / 5; }
__host__ __device__ constexpr int sym_du(int k) { return k - 5 * ((k + 2) / 5); }

// Two consecutive plane elements from an even index, as float2.
__device__ __forceinline__ float2 ld2(const float* p, int i) { return *reinterpret_cast<const float2*>(p + i); }
__device__ __forceinline__ float2 ld2(const __half* p, int i)
{
    return __half22float2(*reinterpret_cast<const __half2*>(p + i));
}
__device__ __forceinline__ float2 ld2(const __nv_bfloat16* p, int i)
{
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p + i));
}
// Two consecutive elements from an odd index: two aligned pair loads.
__device__ __forceinline__ float2 ld2o(const float* p, int i) { return make_float2(p[i], p[i + 1]); }
__device__ __forceinline__ float2 ld2o(const __half* p, int i)
{
    const __half2 a = *reinterpret_cast<const __half2*>(p + i - 1);
    const __half2 b = *reinterpret_cast<const __half2*>(p + i + 1);
    return __half22float2(__halves2half2(__high2half(a), __low2half(b)));
}
__device__ __forceinline__ float2 ld2o(const __nv_bfloat16* p, int i)
{
    const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(p + i - 1);
    const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(p + i + 1);
    return __bfloat1622float2(__halves2bfloat162(__high2bfloat16(a), __low2bfloat16(b)));
}
template <int DU, class T>
__device__ __forceinline__ float2 ld2s(const T* p, int i)
{
    if constexpr ((DU & 1) == 0) return ld2(p, i);
    else return ld2o(p, i);
}

template <class T>
__device__ __forceinline__ const T* plane(const unsigned char* slot, int k, int pstride)
{
    return reinterpret_cast<const T*>(slot + k * pstride);
}

// ---- operators on two adjacent output pixels (smem column c, c+1) ----
// X[d][m]: operand at row vbase + d - 2, local column 2*lane + m (output
// pixel e sits at m = 2 + e); the output row is vbase + RO, so rows
// RO..RO+4 of X are its stencil rows.  brow[d]: band slot of row v - d.
template <class T, int K, int RO, int BOX>
__device__ __forceinline__ void symd_term(float2& yu, float2& yl, const float (&X)[6][6],
                                          const unsigned char* const (&brow)[3], int c)
{
    constexpr int du = sym_du(K), dv = sym_dv(K);
    constexpr int pstride = BOX * (int)sizeof(T);
    const float2 wu = ld2(plane<T>(brow[0], K - 1, pstride), c);
    yu.x = fmaf(-wu.x, X[RO + 2 + dv][2 + du], yu.x);
    yu.y = fmaf(-wu.y, X[RO + 2 + dv][3 + du], yu.y);
    const float2 wl = ld2s<du>(plane<T>(brow[dv], K - 1, pstride), c - du);
    yl.x = fmaf(-wl.x, X[RO + 2 - dv][2 - du], yl.x);
    yl.y = fmaf(-wl.y, X[RO + 2 - dv][3 - du], yl.y);
}

// Four independent accumulation chains per pixel (upper/lower x two halves
// of the bands) keep the FMA dependency chains short.
template <class T, int RO, int BOX>
__device__ __forceinline__ float2 symd_apply(const float (&X)[6][6], const unsigned char* const (&brow)[3], int xoff,
                                             int c)
{
    const float2 dg = ld2(reinterpret_cast<const float*>(brow[0] + xoff), c);
    float2 a = make_float2(dg.x * X[RO + 2][2], dg.y * X[RO + 2][3]);
    float2 b = make_float2(0.f, 0.f), e = make_float2(0.f, 0.f), f = make_float2(0.f, 0.f);
    symd_term<T, 1, RO, BOX>(a, b, X, brow, c);
    symd_term<T, 2, RO, BOX>(e, f, X, brow, c);
    symd_term<T, 3, RO, BOX>(a, b, X, brow, c);
    symd_term<T, 4, RO, BOX>(e, f, X, brow, c);
    symd_term<T, 5, RO, BOX>(a, b, X, brow, c);
    symd_term<T, 6, RO, BOX>(e, f, X, brow, c);
    symd_term<T, 7, RO, BOX>(a, b, X, brow, c);
    symd_term<T, 8, RO, BOX>(e, f, X, brow, c);
    symd_term<T, 9, RO, BOX>(a, b, X, brow, c);
    symd_term<T, 10, RO, BOX>(e, f, X, brow, c);
    symd_term<T, 11, RO, BOX>(a, b, X, brow, c);
    symd_term<T, 12, RO, BOX>(e, f, X, brow, c);
    return make_float2((a.x + b.x) + (e.x + f.x), (a.y + b.y) + (e.y + f.y));
}

// True operator, implicit diagonal, accumulation type V (float or double);
// also returns the diagonal gamma + sum w (for Jacobi).
template <class V, int K, int RO, int BOX>
__device__ __forceinline__ void symi_term(V& y0, V& y1, V& d0, V& d1, const V (&X)[6][6],
                                          const unsigned char* const (&brow)[3], int c)
{
    constexpr int du = sym_du(K), dv = sym_dv(K);
    constexpr int pstride = BOX * 4;
    const float2 wu = ld2(plane<float>(brow[0], K - 1, pstride), c);
    const float2 wl = ld2s<du>(plane<float>(brow[dv], K - 1, pstride), c - du);
    y0 += (V)wu.x * (X[RO + 2][2] - X[RO + 2 + dv][2 + du]) + (V)wl.x * (X[RO + 2][2] - X[RO + 2 - dv][2 - du]);
    y1 += (V)wu.y * (X[RO + 2][3] - X[RO + 2 + dv][3 + du]) + (V)wl.y * (X[RO + 2][3] - X[RO + 2 - dv][3 - du]);
    d0 += (V)wu.x + (V)wl.x;
    d1 += (V)wu.y + (V)wl.y;
}

template <class V, int RO, int BOX>
__device__ __forceinline__ void symi_apply(V& y0, V& y1, V& d0, V& d1, const V (&X)[6][6],
                                           const unsigned char* const (&brow)[3], int xoff, int c)
{
    const float2 g = ld2(reinterpret_cast<const float*>(brow[0] + xoff), c);
    y0 = (V)g.x * X[RO + 2][2];
    y1 = (V)g.y * X[RO + 2][3];
    d0 = (V)g.x;
    d1 = (V)g.y;
    symi_term<V, 1, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 2, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 3, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 4, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 5, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 6, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 7, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 8, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 9, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 10, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 11, RO, BOX>(y0, y1, d0, d1, X, brow, c);
    symi_term<V, 12, RO, BOX>(y0, y1, d0, d1, X, brow, c);
}

// Reference layout: y = sum_j a_j x(u+du_j, v+dv_j), band j = 12 + du + 5 dv,
// in band order (BandedMatrix.cu:172-173); d = a_12.
template <class V, int RO, int BOX>
__device__ __forceinline__ void ref25_apply(V& y0, V& y1, V& d0, V& d1, const V (&X)[6][6],
                                            const unsigned char* b0, int c)
{
    constexpr int pstride = BOX * 4;
    V s0[3] = {0, 0, 0}, s1[3] = {0, 0, 0};  // three chains per pixel
#pragma unroll
    for (int j = 0; j < 25; ++j) {
        const int du = j % 5 - 2, dv = j / 5 - 2;
        const float2 a = ld2(plane<float>(b0, j, pstride), c);
        s0[j % 3] += (V)a.x * X[RO + 2 + dv][2 + du];
        s1[j % 3] += (V)a.y * X[RO + 2 + dv][3 + du];
        if (j == 12) {
            d0 = (V)a.x;
            d1 = (V)a.y;
        }
    }
    y0 = (s0[0] + s0[1]) + s0[2];
    y1 = (s1[0] + s1[1]) + s1[2];
}

struct KState {
    float af;        // alpha_{k-1} (float) for the r / x updates
    float bf;        // beta_k (float)
    double ad;       // alpha as double (fold)
    bool skipR;      // r_k = r_{k-1} (after a replacement)
    bool beta_zero;
    int c;           // vector side read this sweep
    int xsel;        // solution buffers read this sweep
};

// The solver state of one image (every CTA of the image holds the same copy
// in registers); batched solves publish it when CTAs are re-dealt.
struct ImgState {
    KState s;
    int status, it, nrep, kind, final_rep, restart_due;
    double rr_prev, bb, rr_true, rel, be_pred, jtol;
};

// Per-thread pipeline state that lives across sweeps: one bit per ring slot.
struct Pipe {
    uint32_t full_v, full_b;    // consumers: parity of the next full-barrier phase
    uint32_t empty_v, empty_b;  // producer: parity of the next empty-barrier phase
    uint32_t used_v, used_b;    // producer: slot has been filled before
};

__device__ __forceinline__ int ring_next(int s, int R) { return s + 1 == R ? 0 : s + 1; }
__device__ __forceinline__ int ring_prev(int s, int R) { return s == 0 ? R - 1 : s - 1; }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_n(uint64_t* bar, uint32_t n)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(n) : "memory");
}

// Rows vbase-2 .. vbase+3 of the operand sit in ring rows r0, r0+1, ...
// (mod NR); columns lc0 .. lc0+5.
template <class V, int NR>
__device__ __forceinline__ void load_rows(V (&X)[6][6], const V* ring, int r0, int lc0)
{
#pragma unroll
    for (int d = 0; d < 6; ++d) {
        const V* row = ring + ((r0 + d) & (NR - 1)) * kRingCols + lc0;
#pragma unroll
        for (int m = 0; m < 6; m += 2) {
            if constexpr (sizeof(V) == 4) {
                const float2 t = *reinterpret_cast<const float2*>(row + m);
                X[d][m] = t.x;
                X[d][m + 1] = t.y;
            } else {
                const double2 t = *reinterpret_cast<const double2*>(row + m);
                X[d][m] = t.x;
                X[d][m + 1] = t.y;
            }
        }
    }
}

template <class TLo, int OPLO, int OPHI, bool MIXED, int CFG, int KIND, bool PCG = false, bool FULLW = false>
__device__ __forceinline__ void run_sweep(const SolverArgs& A, const UnitGeo& geo, unsigned char* smem, int u0,
                                          int v0, int v1, const KState& s, double (&part)[kNPart], Pipe& pp)
{
    constexpr Layout L = make_layout(OPLO, OPLO == OP_REF25 ? 4 : (int)sizeof(TLo), OPHI, MIXED, CFG);
    constexpr KindLayout K = L.k[KIND];
    constexpr int NCONS = cfg_ncol(CFG);
    constexpr int BOX = cfg_box(CFG);
    constexpr int OPR = kOpRows, OWNR = kOwnRows;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nsteps = v1 - v0 + 4;
    const int nband = nsteps - 2;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
    unsigned char* vring = smem + K.vbase;
    unsigned char* bring = smem + K.bbase;
    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + L.red_off + cfg_red_bytes(CFG));
    constexpr bool kSymBand = (KIND == KIND_KRYLOV ? OPLO : OPHI) != OP_REF25;
    constexpr bool kEarly = kSymBand && KIND != KIND_KRYLOV;

    if (warp == NCONS) {
        // ------------------------------ producer ------------------------------
        if (lane != 0) return;
        const CUtensorMap* vm[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
        if (KIND == KIND_KRYLOV) {
            vm[0] = &A.m_r[s.c]; vm[1] = &A.m_q[s.c]; vm[2] = &A.m_p[s.c]; vm[3] = &A.m_xacc[s.xsel];
            if (PCG) vm[4] = &A.m_xlo;  // the diagonal, for z = r / d
        } else if (KIND == KIND_REPLACE) {
            vm[0] = MIXED ? &A.m_base[s.xsel] : nullptr; vm[1] = &A.m_xacc[s.xsel]; vm[2] = &A.m_p[s.c];
            vm[3] = &A.m_b;
        } else {
            vm[0] = &A.m_xacc[s.xsel]; vm[3] = &A.m_b;
        }
        const CUtensorMap* bm = KIND == KIND_KRYLOV ? &A.m_wlo : &A.m_whi;
        const CUtensorMap* xm = KIND == KIND_KRYLOV ? &A.m_xlo : &A.m_xhi;
        const uint32_t vbytes = K.vbytes[0] + K.vbytes[1] + K.vbytes[2] + K.vbytes[3] + (vm[4] ? K.vbytes[4] : 0);
        fence_proxy_async();
        // Issue in the consumers' order: super-step j takes vector rows j and
        // j+1, then band rows up to (its last step) - 2.  Matching the order
        // keeps the rings deadlock-free for any depth >= 1.
        int vs = 0, bs = 0, bnext = 0;
        auto issue_vec = [&](int t) -> bool {
            const uint32_t bit = 1u << vs;
            if (pp.used_v & bit) {
                if (!mbar_wait_bounded(&empty[vs], (pp.empty_v & bit) ? 1u : 0u, A.gb, A.tma_limit_ns)) return false;
                pp.empty_v ^= bit;
            }
            pp.used_v |= bit;
            unsigned char* dst = vring + vs * K.vslot;
            mbar_arrive_expect_tx(&full[vs], vbytes);
#pragma unroll
            for (int i = 0; i < 5; ++i)
                if (K.vbytes[i] && vm[i]) tma_load_2d(dst + K.voff[i], vm[i], u0 - 8, v0 - 2 + t, &full[vs]);
            vs = ring_next(vs, K.Rv);
            return true;
        };
        auto issue_band = [&](int m) -> bool {
            const uint32_t bit = 1u << bs;
            if (pp.used_b & bit) {
                if (!mbar_wait_bounded(&empty[kRvMax + bs], (pp.empty_b & bit) ? 1u : 0u, A.gb, A.tma_limit_ns))
                    return false;
                pp.empty_b ^= bit;
            }
            pp.used_b |= bit;
            unsigned char* dst = bring + bs * K.bslot;
            mbar_arrive_expect_tx(&full[kRvMax + bs], K.bbytes);
            tma_load_3d(dst, bm, u0 - 8, v0 - 2 + m, 0, &full[kRvMax + bs]);
            if (K.xoff >= 0) tma_load_2d(dst + K.xoff, xm, u0 - 8, v0 - 2 + m, &full[kRvMax + bs]);
            bs = ring_next(bs, K.Rb);
            return true;
        };
        for (int j = 0; j < nsteps; j += 2) {
            if (*s_abort) break;
            const bool two = j + 1 < nsteps;
            if (!issue_vec(j) || (two && !issue_vec(j + 1))) { *s_abort = 1; break; }
            const int mneed = (two ? j + 1 : j) - 2;
            bool ok = true;
            for (; bnext <= mneed && bnext < nband; ++bnext)
                if (!issue_band(bnext)) { ok = false; break; }
            if (!ok) { *s_abort = 1; break; }
        }
        return;
    }

    // -------------------------------- consumers --------------------------------
    // Rows are consumed in super-steps of two: phase A of steps j and j+1
    // (combine the incoming rows into the operand ring), one __syncwarp, then
    // phase B of both output rows from one shared 6-row operand window.
    const int w = warp;
    const int c = 8 + kWarpCols * w + 2 * lane;        // smem column of this lane's pixel pair
    const int lc0 = 2 * lane;                          // first operand column (local ring index)
    const int u = u0 + kWarpCols * w + 2 * lane;       // image column of pixel 0
    // FULLW: every column of the strip lies inside the image
    const bool in0 = FULLW || u < geo.W, in1 = FULLW || u + 1 < geo.W;
    // extra operand pair for the ring halo: lane 0 left, lane 1 right
    const bool has_x = lane < 2;
    const int cx = lane == 0 ? 6 + kWarpCols * w : 8 + kWarpCols * w + kWarpCols;
    const int lcx = lane == 0 ? 0 : kRingCols - 2;
    using RingT = std::conditional_t<MIXED, double, float>;  // replacement operand ring element
    float* ring_f = reinterpret_cast<float*>(smem + L.pring_off) + w * OPR * kRingCols;
    RingT* ring_d = reinterpret_cast<RingT*>(smem + L.pringd_off) + w * OPR * kRingCols;
    float* own_ring = reinterpret_cast<float*>(smem + L.rring_off) + w * OWNR * kWarpCols;  // r or b, own columns
    const int P = A.P;
    // Krylov outputs, read once from the parameter block (warp-uniform)
    float* const r_nx = A.r[s.c ^ 1];
    float* const p_nx = A.p[s.c ^ 1];
    float* const q_nx = A.q[s.c ^ 1];
    float* const x_cur = A.xacc[s.xsel];
    constexpr int Rb = K.Rb;
    constexpr bool pcg = PCG && OPLO == OP_SYMD && KIND == KIND_KRYLOV;  // Jacobi-preconditioned CG

    int vs = 0;     // vector slot of the next vector row
    int bs = 0;     // band slot of the next band step
    // band steps j-4 .. j-1 of super-step j: slot (low byte) and full-barrier
    // parity (bit 8), kept in registers as a sliding window
    uint32_t bw0 = 0u, bw1 = 0u, bw2 = 0u, bw3 = 0u;

    auto wait_rec = [&](uint32_t r) {
        if (!mbar_try_wait(&full[kRvMax + (r & 0xffu)], r >> 8) && !*s_abort &&
            !mbar_wait_bounded(&full[kRvMax + (r & 0xffu)], r >> 8, A.gb, A.tma_limit_ns))
            *s_abort = 1;
    };
    auto band_of = [&](uint32_t r) { return bring + (int)(r & 0xffu) * K.bslot; };
    // Band step m is read by the phase B of super-steps j (even, 4 <= j <
    // nsteps) with j-4 <= m <= j-1 (symmetric store: output row v reads rows
    // v, v-1, v-2) or m in {j-2, j-1} (reference layout: row v only).  Its
    // slot is released at its last read, by all NCONS warps (the empty
    // barrier takes 2 * NCONS arrivals, 2 per warp).
    auto release_rec = [&](uint32_t r) {
        if (lane == 0) mbar_arrive_n(&empty[kRvMax + (r & 0xffu)], 2u);
    };

    // phase A of step j (vector slot vsl, full parity vpar) into operand ring
    // row j mod 8 and own ring row j mod 4
    auto phase_a = [&](int j, int vsl, uint32_t vpar) {
        const int Lr = v0 - 2 + j;
        if (!mbar_try_wait(&full[vsl], vpar) && !*s_abort && !mbar_wait_bounded(&full[vsl], vpar, A.gb, A.tma_limit_ns))
            *s_abort = 1;
        const unsigned char* vsp = vring + vsl * K.vslot;
        const bool own_row = Lr >= v0 && Lr < v1;
        const size_t gi = (size_t)(own_row ? Lr : 0) * P + u;
        const int rr = j & (OPR - 1), orow = j & (OWNR - 1);
        if (KIND == KIND_KRYLOV) {
            const float* vr = reinterpret_cast<const float*>(vsp + K.voff[0]);
            const float* vq = reinterpret_cast<const float*>(vsp + K.voff[1]);
            const float* vp = reinterpret_cast<const float*>(vsp + K.voff[2]);
            const float* vx = reinterpret_cast<const float*>(vsp + K.voff[3]);
            const float* vd = reinterpret_cast<const float*>(vsp + K.voff[4]);
            // r' = r - alpha q; z' = r' / d (Jacobi PCG) or r'; p' = z' + beta p
            auto combine = [&](int cc, float2& rn, float2& zn, float2& pv) {
                const float2 rv = ld2(vr, cc);
                pv = ld2(vp, cc);
                // selects, not branches (skipR is uniform but costs a branch per row)
                const float2 qv = ld2(vq, cc);
                rn.x = s.skipR ? rv.x : fmaf(-s.af, qv.x, rv.x);
                rn.y = s.skipR ? rv.y : fmaf(-s.af, qv.y, rv.y);
                if constexpr (pcg) {
                    // d = 0 only outside the image (TMA zero fill), where r = 0 too
                    const float2 dv = ld2(vd, cc);
                    zn = make_float2(dv.x > 0.f ? __fdividef(rn.x, dv.x) : 0.f,
                                     dv.y > 0.f ? __fdividef(rn.y, dv.y) : 0.f);
                } else {
                    zn = rn;
                }
                return s.beta_zero ? zn : make_float2(fmaf(s.bf, pv.x, zn.x), fmaf(s.bf, pv.y, zn.y));
            };
            float2 rn, zn, pv;
            const float2 pn = combine(c, rn, zn, pv);
            *reinterpret_cast<float2*>(ring_f + rr * kRingCols + lc0 + 2) = pn;
            {
                // lanes 0 and 1 also form the ring's halo pairs (left, right);
                // the other lanes form their own pair again into its own place,
                // so the warp does not diverge here
                float2 rx, zx, px;
                *reinterpret_cast<float2*>(ring_f + rr * kRingCols + (has_x ? lcx : lc0 + 2)) =
                    combine(has_x ? cx : c, rx, zx, px);
            }
            if (own_row) {
                *reinterpret_cast<float2*>(own_ring + orow * kWarpCols + lc0) = zn;
                if (in1) {
                    *reinterpret_cast<float2*>(r_nx + gi) = rn;
                    *reinterpret_cast<float2*>(p_nx + gi) = pn;
                    if (!s.skipR) {
                        const float2 xv = ld2(vx, c);
                        *reinterpret_cast<float2*>(x_cur + gi) =
                            make_float2(fmaf(s.af, pv.x, xv.x), fmaf(s.af, pv.y, xv.y));
                    }
                    part[0] += (double)fmaf(rn.x, zn.x, rn.y * zn.y);
                    if constexpr (pcg) part[4] += (double)fmaf(rn.x, rn.x, rn.y * rn.y);
                } else if (in0) {
                    r_nx[gi] = rn.x;
                    p_nx[gi] = pn.x;
                    if (!s.skipR) x_cur[gi] = fmaf(s.af, pv.x, vx[c]);
                    part[0] += (double)rn.x * (double)zn.x;
                    if constexpr (pcg) part[4] += (double)rn.x * (double)rn.x;
                }
            }
        } else if (KIND == KIND_REPLACE) {
            // Jacobi keeps its iterate in the FP32 vector (its sweeps read no
            // FP64 base), so its fold goes back there with a zero base.
            const bool jfold = MIXED && A.solver == GM_SOLVER_JACOBI;
            const float* vx = reinterpret_cast<const float*>(vsp + K.voff[1]);
            const float* vp = reinterpret_cast<const float*>(vsp + K.voff[2]);
            const float* vb = reinterpret_cast<const float*>(vsp + K.voff[3]);
            auto fold = [&](int cc) {
                const float2 xv = ld2(vx, cc), pv = ld2(vp, cc);
                double2 xf;
                if (MIXED) {
                    const double2 bv = *reinterpret_cast<const double2*>(
                        reinterpret_cast<const double*>(vsp + K.voff[0]) + cc);
                    xf.x = bv.x + (double)xv.x + s.ad * (double)pv.x;
                    xf.y = bv.y + (double)xv.y + s.ad * (double)pv.y;
                } else {
                    xf.x = (double)fmaf(s.af, pv.x, xv.x);
                    xf.y = (double)fmaf(s.af, pv.y, xv.y);
                }
                return xf;
            };
            const double2 xf = fold(c);
            if constexpr (MIXED) {
                *reinterpret_cast<double2*>(ring_d + rr * kRingCols + lc0 + 2) = xf;
                if (has_x) *reinterpret_cast<double2*>(ring_d + rr * kRingCols + lcx) = fold(cx);
            } else {
                *reinterpret_cast<float2*>(ring_d + rr * kRingCols + lc0 + 2) = make_float2((float)xf.x, (float)xf.y);
                if (has_x) {
                    const double2 xx = fold(cx);
                    *reinterpret_cast<float2*>(ring_d + rr * kRingCols + lcx) = make_float2((float)xx.x, (float)xx.y);
                }
            }
            if (own_row) {
                *reinterpret_cast<float2*>(own_ring + orow * kWarpCols + lc0) = ld2(vb, c);
                if (in1) {
                    if (MIXED && !jfold) {
                        *reinterpret_cast<double2*>(A.base[s.xsel ^ 1] + gi) = xf;
                        *reinterpret_cast<float2*>(A.xacc[s.xsel ^ 1] + gi) = make_float2(0.f, 0.f);
                    } else if (MIXED) {
                        *reinterpret_cast<double2*>(A.base[s.xsel ^ 1] + gi) = make_double2(0.0, 0.0);
                        *reinterpret_cast<float2*>(A.xacc[s.xsel ^ 1] + gi) = make_float2((float)xf.x, (float)xf.y);
                    } else {
                        *reinterpret_cast<float2*>(A.xacc[s.xsel ^ 1] + gi) = make_float2((float)xf.x, (float)xf.y);
                    }
                } else if (in0) {
                    if (MIXED && !jfold) {
                        A.base[s.xsel ^ 1][gi] = xf.x;
                        A.xacc[s.xsel ^ 1][gi] = 0.f;
                    } else if (MIXED) {
                        A.base[s.xsel ^ 1][gi] = 0.0;
                        A.xacc[s.xsel ^ 1][gi] = (float)xf.x;
                    } else {
                        A.xacc[s.xsel ^ 1][gi] = (float)xf.x;
                    }
                }
            }
        } else {  // Jacobi
            const float* vx = reinterpret_cast<const float*>(vsp + K.voff[0]);
            const float* vb = reinterpret_cast<const float*>(vsp + K.voff[3]);
            *reinterpret_cast<float2*>(ring_f + rr * kRingCols + lc0 + 2) = ld2(vx, c);
            if (has_x) *reinterpret_cast<float2*>(ring_f + rr * kRingCols + lcx) = ld2(vx, cx);
            if (own_row) *reinterpret_cast<float2*>(own_ring + orow * kWarpCols + lc0) = ld2(vb, c);
        }
    };
    for (int j = 0; j < nsteps; j += 2) {
        const bool two = j + 1 < nsteps;
        const int vs0 = vs;
        const uint32_t vp0 = (pp.full_v >> vs0) & 1u;
        pp.full_v ^= 1u << vs0;
        vs = ring_next(vs, K.Rv);
        int vs1 = 0;
        uint32_t vp1 = 0u;
        if (two) {
            vs1 = vs;
            vp1 = (pp.full_v >> vs1) & 1u;
            pp.full_v ^= 1u << vs1;
            vs = ring_next(vs, K.Rv);
        }
        // band steps j-2 and j-1 enter the window
        bw0 = bw2;
        bw1 = bw3;
        if (j >= 2 && j - 2 < nband) {
            bw2 = (uint32_t)bs | (((pp.full_b >> bs) & 1u) << 8);
            pp.full_b ^= 1u << bs;
            bs = ring_next(bs, Rb);
        }
        if (j >= 2 && j - 1 < nband) {
            bw3 = (uint32_t)bs | (((pp.full_b >> bs) & 1u) << 8);
            pp.full_b ^= 1u << bs;
            bs = ring_next(bs, Rb);
        }
        phase_a(j, vs0, vp0);
        if (two) phase_a(j + 1, vs1, vp1);
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[vs0]);
            if (two) mbar_arrive(&empty[vs1]);
        }
        if (!kSymBand && j == 2) {
            // rows v0-2, v0-1: loaded but unused by the reference layout; released
            // as soon as their loads land, since a ring of two slots needs them back
            wait_rec(bw2);
            wait_rec(bw3);
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_n(&empty[kRvMax + (bw2 & 0xffu)], 2u);
                mbar_arrive_n(&empty[kRvMax + (bw3 & 0xffu)], 2u);
            }
        }
        if (j >= 4) {
            // ---------------- phase B: output rows v and v+1 ----------------
            const int v = v0 - 4 + j;
            const bool second = two && v + 1 < v1;
            if (kSymBand) {
                // steps j-4, j-3 were waited for at super-step j-2
                if (j == 4) {
                    wait_rec(bw0);
                    wait_rec(bw1);
                }
                wait_rec(bw2);
                if (second && !kEarly) wait_rec(bw3);  // early release: waited before row v + 1
            } else {
                wait_rec(bw2);
                if (second) wait_rec(bw3);
            }
            const unsigned char* bA[3] = {band_of(bw2), band_of(bw1), band_of(bw0)};
            const unsigned char* bB[3] = {band_of(bw3), bA[0], bA[1]};
            const int r0 = (j - 4) & (OPR - 1);   // ring row of operand row v - 2
            const int o0 = (j - 2) & (OWNR - 1);  // own ring row of output row v
            const int o1 = (j - 1) & (OWNR - 1);
            const size_t go = (size_t)v * P + u;
            // The rows of a replacement or Jacobi sweep (r0_: output row v,
            // r1_: row v + 1), each call loading the operand window itself.
            auto nk_rows = [&](bool r0_, bool r1_) {
                if constexpr (KIND == KIND_REPLACE) {
                    double X[6][6];
                    if constexpr (MIXED) {
                        load_rows<double, OPR>(X, ring_d, r0, lc0);
                    } else {
                        float Xf[6][6];
                        load_rows<float, OPR>(Xf, ring_d, r0, lc0);
#pragma unroll
                        for (int a = 0; a < 6; ++a)
#pragma unroll
                            for (int b2 = 0; b2 < 6; ++b2) X[a][b2] = (double)Xf[a][b2];
                    }
                    auto rep_row = [&](double y0, double y1, const float2 bv, size_t g, int vr, int ro) {
                        const float r0f = (float)((double)bv.x - y0), r1f = (float)((double)bv.y - y1);
                        float* ao = geo.aout + (size_t)(vr - geo.arow0) * geo.apitch + u;
                        ao[0] = (float)X[ro + 2][2];
                        A.r[s.c][g] = r0f;
                        part[0] += (double)r0f * (double)r0f;
                        part[1] += (double)bv.x * (double)bv.x;
                        if (in1) {
                            ao[1] = (float)X[ro + 2][3];
                            A.r[s.c][g + 1] = r1f;
                            part[0] += (double)r1f * (double)r1f;
                            part[1] += (double)bv.y * (double)bv.y;
                        }
                    };
                    double y0, y1, d0, d1;
                    if (r0_) {
                        if (OPHI == OP_REF25) ref25_apply<double, 0, BOX>(y0, y1, d0, d1, X, bA[0], c);
                        else symi_apply<double, 0, BOX>(y0, y1, d0, d1, X, bA, K.xoff, c);
                        rep_row(y0, y1, *reinterpret_cast<const float2*>(own_ring + o0 * kWarpCols + lc0), go, v, 0);
                    }
                    if (r1_) {
                        if (OPHI == OP_REF25) ref25_apply<double, 1, BOX>(y0, y1, d0, d1, X, bB[0], c);
                        else symi_apply<double, 1, BOX>(y0, y1, d0, d1, X, bB, K.xoff, c);
                        rep_row(y0, y1, *reinterpret_cast<const float2*>(own_ring + o1 * kWarpCols + lc0), go + P,
                                v + 1, 1);
                    }
                } else if constexpr (KIND == KIND_JACOBI) {
                    float X[6][6];
                    load_rows<float, OPR>(X, ring_f, r0, lc0);
                    auto jac_row = [&](float y0, float y1, float d0, float d1, const float2 bv, size_t g, int ro) {
                        const float rv0 = bv.x - y0, rv1 = bv.y - y1;
                        A.xacc[s.xsel ^ 1][g] = X[ro + 2][2] + A.omega * rv0 / d0;
                        part[0] += (double)rv0 * (double)rv0;
                        part[1] += (double)bv.x * (double)bv.x;
                        if (in1) {
                            A.xacc[s.xsel ^ 1][g + 1] = X[ro + 2][3] + A.omega * rv1 / d1;
                            part[0] += (double)rv1 * (double)rv1;
                            part[1] += (double)bv.y * (double)bv.y;
                        }
                    };
                    float y0, y1, d0, d1;
                    if (r0_) {
                        if (OPHI == OP_REF25) ref25_apply<float, 0, BOX>(y0, y1, d0, d1, X, bA[0], c);
                        else symi_apply<float, 0, BOX>(y0, y1, d0, d1, X, bA, K.xoff, c);
                        jac_row(y0, y1, d0, d1, *reinterpret_cast<const float2*>(own_ring + o0 * kWarpCols + lc0), go,
                                0);
                    }
                    if (r1_) {
                        if (OPHI == OP_REF25) ref25_apply<float, 1, BOX>(y0, y1, d0, d1, X, bB[0], c);
                        else symi_apply<float, 1, BOX>(y0, y1, d0, d1, X, bB, K.xoff, c);
                        jac_row(y0, y1, d0, d1, *reinterpret_cast<const float2*>(own_ring + o1 * kWarpCols + lc0),
                                go + P, 1);
                    }
                }
            };
            if (in0) {
                if (KIND == KIND_KRYLOV) {
                    float X[6][6];
                    load_rows<float, OPR>(X, ring_f, r0, lc0);
                    float2 q0, q1 = make_float2(0.f, 0.f);
                    if (OPLO == OP_SYMD) {
                        q0 = symd_apply<TLo, 0, BOX>(X, bA, K.xoff, c);
                        if (second) q1 = symd_apply<TLo, 1, BOX>(X, bB, K.xoff, c);
                    } else {
                        float d0, d1;
                        ref25_apply<float, 0, BOX>(q0.x, q0.y, d0, d1, X, bA[0], c);
                        if (second) ref25_apply<float, 1, BOX>(q1.x, q1.y, d0, d1, X, bB[0], c);
                    }
                    // own ring: z (= r for plain CG) of the output rows
                    const float2 rn0 = *reinterpret_cast<const float2*>(own_ring + o0 * kWarpCols + lc0);
                    const float2 rn1 = *reinterpret_cast<const float2*>(own_ring + o1 * kWarpCols + lc0);
                    // q M^-1 q: the diagonal of output rows v, v+1 sits in their band rows
                    float2 w0 = make_float2(1.f, 1.f), w1 = make_float2(1.f, 1.f);
                    if constexpr (pcg) {
                        {
                            const float2 d0 = ld2(reinterpret_cast<const float*>(bA[0] + K.xoff), c);
                            w0 = make_float2(d0.x > 0.f ? __fdividef(1.f, d0.x) : 0.f,
                                             d0.y > 0.f ? __fdividef(1.f, d0.y) : 0.f);
                            if (second) {
                                const float2 d1 = ld2(reinterpret_cast<const float*>(bB[0] + K.xoff), c);
                                w1 = make_float2(d1.x > 0.f ? __fdividef(1.f, d1.x) : 0.f,
                                                 d1.y > 0.f ? __fdividef(1.f, d1.y) : 0.f);
                            }
                        }
                    }
                    if (in1) {
                        *reinterpret_cast<float2*>(q_nx + go) = q0;
                        float spq = fmaf(X[2][2], q0.x, X[2][3] * q0.y);
                        float srq = fmaf(rn0.x, q0.x, rn0.y * q0.y);
                        float sqq = fmaf(q0.x * w0.x, q0.x, q0.y * w0.y * q0.y);
                        if (second) {
                            *reinterpret_cast<float2*>(q_nx + go + P) = q1;
                            if constexpr (OPLO == OP_SYMD) {
                                // both rows' products in FP32, one FP64 add per sum
                                spq = fmaf(X[3][2], q1.x, fmaf(X[3][3], q1.y, spq));
                                srq = fmaf(rn1.x, q1.x, fmaf(rn1.y, q1.y, srq));
                                sqq = fmaf(q1.x * w1.x, q1.x, fmaf(q1.y * w1.y, q1.y, sqq));
                            } else {
                                // the plain FP32 method (the reference's layout) keeps
                                // one FP64 add per row and partial sum
                                part[1] += (double)fmaf(X[3][2], q1.x, X[3][3] * q1.y);
                                part[2] += (double)fmaf(rn1.x, q1.x, rn1.y * q1.y);
                                part[3] += (double)fmaf(q1.x * w1.x, q1.x, q1.y * w1.y * q1.y);
                            }
                        }
                        part[1] += (double)spq;
                        part[2] += (double)srq;
                        part[3] += (double)sqq;
                    } else {
                        q_nx[go] = q0.x;
                        part[1] += (double)X[2][2] * (double)q0.x;
                        part[2] += (double)rn0.x * (double)q0.x;
                        part[3] += (double)q0.x * w0.x * (double)q0.x;
                        if (second) {
                            q_nx[go + P] = q1.x;
                            part[1] += (double)X[3][2] * (double)q1.x;
                            part[2] += (double)rn1.x * (double)q1.x;
                            part[3] += (double)q1.x * w1.x * (double)q1.x;
                        }
                    }
                } else {
                    nk_rows(true, second && !kEarly);
                }
            }
            if constexpr (kEarly) {
                // band row v - 2 is read by output row v only: its slot goes
                // back before row v + 1 is formed, so that the producer refills
                // it meanwhile (this kind's four band slots are exactly the two
                // rows' window and leave no room to load ahead otherwise)
                __syncwarp();
                release_rec(bw0);
                if (second) {
                    wait_rec(bw3);
                    if (in0) nk_rows(false, true);
                }
            }
            __syncwarp();
            // band steps read for the last time: j-4, j-3 (symmetric store)
            // and, at the last super-step, the rest
            if (kSymBand) {
                if (!kEarly) release_rec(bw0);
                release_rec(bw1);
                if (j + 2 >= nsteps) {
                    release_rec(bw2);
                    if (second) release_rec(bw3);
                }
            } else {
                release_rec(bw2);
                if (second) release_rec(bw3);
            }
        }
    }
    __syncwarp();
}

// The unit of CTA b after a re-deal (run by one warp; lane 0 writes out[]):
// the strip-row partition of the host (batch_partition, rmul 1) over the
// images that have not finished.  out = {img, u0, v0, v1, u0b, v0b, v1b, lo,
// hi}; img = -1 when b gets no work.  Every CTA computes the same partition.
__device__ __noinline__ void batch_redeal(const SolverArgs& A, int b, int G, int* out)
{
    const int kStrip = A.strip;
    const int lane = threadIdx.x & 31;
    auto running = [&](int k) { return __ldcg(A.img_done + k) == 0; };
    int maxT = 0;
    for (int k = lane; k < A.nimg; k += 32)
        if (running(k)) {
            const BatchImage I = A.imgs[k];
            maxT = max(maxT, ((I.W + kStrip - 1) / kStrip) * I.H);
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxT = max(maxT, __shfl_xor_sync(0xffffffffu, maxT, o));
    int R = max(maxT, 1);
    if (maxT > 0) {
        int rlo = 1, rhi = maxT;
        while (rlo < rhi) {
            const int mid = rlo + (rhi - rlo) / 2;
            long long c = 0;
            for (int k = lane; k < A.nimg; k += 32)
                if (running(k)) {
                    const BatchImage I = A.imgs[k];
                    const int sk = (I.W + kStrip - 1) / kStrip, T = sk * I.H;
                    c += max(sk, (T + mid - 1) / mid);
                }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (c <= G) rhi = mid; else rlo = mid + 1;
        }
        R = rlo;
    }
    if (lane != 0) return;
    int res[9] = {-1, 0, 0, 0, 0, 0, 0, 0, 0};
    int c0 = 0;
    for (int k = 0; k < A.nimg && maxT > 0; ++k) {
        if (!running(k)) continue;
        const BatchImage I = A.imgs[k];
        const int sk = (I.W + kStrip - 1) / kStrip, H = I.H;
        const long long T = (long long)sk * H;
        const long long nk = (T + R - 1) / R;
        const int n = (int)(nk > sk ? nk : (long long)sk);
        if (b >= c0 && b < c0 + n) {
            const int u = b - c0;
            const long long t0 = T * u / n, t1 = T * (u + 1) / n;
            const int sa = (int)(t0 / H), ra = (int)(t0 % H), sb = (int)((t1 - 1) / H);
            res[0] = k;
            res[1] = sa * kStrip;
            res[2] = I.y0 + ra;
            res[3] = I.y0 + (sb == sa ? (int)((t1 - 1) % H) + 1 : H);
            if (sb != sa) {
                res[4] = sb * kStrip;
                res[5] = I.y0;
                res[6] = I.y0 + (int)((t1 - 1) % H) + 1;
            }
            res[7] = c0;
            res[8] = c0 + n;
            break;
        }
        c0 += n;
    }
    for (int q = 0; q < 9; ++q) out[q] = res[q];
}

// Resident CTAs per SM the register budget is sized for: 3 (4 with
// 128-column strips) for the 2-byte symmetric stores with shallow rings, as
// their shared memory allows; 1 (no register cap) for the other
// configurations, which shared memory limits to 2.
template <class TLo, int OPLO, int CFG>
constexpr int solver_min_blocks()
{
    return (OPLO == OP_SYMD && sizeof(TLo) == 2 && CFG != 1) ? cfg_cps(CFG) : 1;
}

template <class TLo, int OPLO, int OPHI, bool MIXED, int CFG, bool BATCH>
__global__ void __launch_bounds__(cfg_threads(CFG), solver_min_blocks<TLo, OPLO, CFG>())
    solver_kernel(const __grid_constant__ SolverArgs A)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x;
    constexpr Layout L = make_layout(OPLO, OPLO == OP_REF25 ? 4 : (int)sizeof(TLo), OPHI, MIXED, CFG);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
    double* red = reinterpret_cast<double*>(smem + L.red_off);

    // This CTA's unit: a 192-column strip of a row segment of one image.
    int img = -1, u0 = 0, v0 = 0, v1 = 0, lo = 0, hi = 0;
    UnitGeo geo;
    int u0b = 0, v0b = 0, v1b = 0;  // second piece (batched units only)
    if constexpr (BATCH) {
        geo.W = 0; geo.arow0 = 0; geo.apitch = 0; geo.aout = nullptr; geo.ain = nullptr;
        const BatchUnit U = A.units[blockIdx.x];
        if (U.img >= 0 && U.img < A.nimg) {
            const BatchImage I = A.imgs[U.img];
            img = U.img;
            u0 = U.u0[0]; v0 = U.v0[0]; v1 = U.v1[0];
            u0b = U.u0[1]; v0b = U.v0[1]; v1b = U.v1[1];
            lo = I.c0;
            hi = I.c0 + I.units;
            geo.W = I.W; geo.arow0 = I.y0; geo.apitch = I.W; geo.aout = I.alpha; geo.ain = I.alpha;
        }
    } else {
        const int unit = blockIdx.x;
        if (unit < A.nunits) {
            const int st = unit % A.nstrips, sg = unit / A.nstrips;
            u0 = st * cfg_strip(CFG);
            v0 = (int)((long long)A.H * sg / A.nseg);
            v1 = (int)((long long)A.H * (sg + 1) / A.nseg);
        }
        geo.W = A.W; geo.arow0 = 0; geo.apitch = A.alpha_pitch; geo.aout = A.alpha_out; geo.ain = A.alpha_in;
    }

    if (tid == 0) {
        for (int i = 0; i < kRvMax + kRbMax; ++i) {
            mbar_init(&full[i], 1);
            // vector slots: one arrival per consumer warp; band slots: two
            // per consumer warp (see run_sweep)
            mbar_init(&empty[i], i < kRvMax ? cfg_ncol(CFG) : 2 * cfg_ncol(CFG));
        }
        *reinterpret_cast<volatile int*>(smem + L.red_off + cfg_red_bytes(CFG)) = 0;
        fence_mbar_init();
    }
    __syncthreads();
    Pipe pp = {0u, 0u, 0u, 0u, 0u, 0u};

    const bool jac = A.solver == GM_SOLVER_JACOBI;
    // Import the initial guess and the right-hand side; zero the first
    // search direction.
#pragma unroll 1
    for (int piece = 0; piece < (BATCH ? 2 : 1); ++piece) {
        const int pu0 = piece ? u0b : u0, pv0 = piece ? v0b : v0, pv1 = piece ? v1b : v1;
        for (int v = pv0; v < pv1; ++v)
            for (int cl = tid; cl < cfg_strip(CFG); cl += blockDim.x) {
                const int u = pu0 + cl;
                if (u >= geo.W) continue;
                const size_t i = (size_t)v * A.P + u;
                const float a0 = geo.ain[(size_t)(v - geo.arow0) * geo.apitch + u];
                if (MIXED) {
                    A.base[0][i] = jac ? 0.0 : (double)a0;
                    A.base[1][i] = 0.0;
                }
                A.xacc[0][i] = (MIXED && !jac) ? 0.f : a0;
                A.p[0][i] = 0.f;
                A.q[0][i] = 0.f;
                A.r[0][i] = 0.f;
                A.bw[i] = A.b[(size_t)v * A.bpitch + u];
            }
    }
    const unsigned G = gridDim.x;
    bool ok = grid_sync(A.gb, G, A.limit_ns, A.inject == 1 ? 1u : 0u);

    int status = GM_OK, it = 0, nrep = 0, parity = 0;
    int kind = jac ? KIND_JACOBI : KIND_REPLACE;
    KState s;
    s.af = 0.f; s.bf = 0.f; s.ad = 0.0; s.skipR = true; s.beta_zero = true; s.c = 0; s.xsel = 0;
    double rr_prev = 0.0, bb = -1.0, rr_true = 0.0, rel = 0.0, be_pred = 0.0;
    // Jacobi: target of the in-sweep (FP32) residual; lowered when the FP64
    // replacement finds the true residual still above rtol
    double jtol = A.rtol;
    bool final_rep = false, restart_due = false;
    const bool gd = A.solver == GM_SOLVER_GD;
    const bool pcg_mode = A.solver == GM_SOLVER_PCG;
    if (jac && A.max_iters <= 0) {
        kind = KIND_REPLACE;
        final_rep = true;
    }
    // Batched solves: a CTA whose image has converged (or that has no image)
    // keeps joining the grid barrier with no work until every image is done.
    bool done = BATCH && img < 0;
    // Batched solves re-deal the CTAs when images finish (the grid-wide count
    // of CTAs that worked in a sweep dropped): the images still running
    // publish their state, and after a barrier every CTA computes the same
    // strip-row partition over them and takes up its new image's state.
    bool redeal = false;
    double prev_running = -1.0;

    while (ok) {
        if constexpr (BATCH) {
            if (redeal) {
                redeal = false;
                ImgState* tab = reinterpret_cast<ImgState*>(A.states);
                if (img >= 0 && !done && (int)blockIdx.x == lo && tid == 0) {
                    ImgState t;
                    t.s = s; t.status = status; t.it = it; t.nrep = nrep; t.kind = kind;
                    t.final_rep = final_rep; t.restart_due = restart_due;
                    t.rr_prev = rr_prev; t.bb = bb; t.rr_true = rr_true; t.rel = rel; t.be_pred = be_pred;
                    t.jtol = jtol;
                    tab[img] = t;
                }
                ok = grid_sync(A.gb, G, A.limit_ns);
                if (!ok) break;
                __shared__ int s_unit[9];  // img, u0, v0, v1, u0b, v0b, v1b, lo, hi
                if (tid < 32) batch_redeal(A, (int)blockIdx.x, (int)G, s_unit);
                __syncthreads();
                img = s_unit[0];
                u0 = s_unit[1]; v0 = s_unit[2]; v1 = s_unit[3];
                u0b = s_unit[4]; v0b = s_unit[5]; v1b = s_unit[6];
                lo = s_unit[7]; hi = s_unit[8];
                __syncthreads();
                done = img < 0;
                if (!done) {
                    const BatchImage I = A.imgs[img];
                    geo.W = I.W; geo.arow0 = I.y0; geo.apitch = I.W; geo.aout = I.alpha; geo.ain = I.alpha;
                    // written by another CTA before the barrier: read past L1
                    ImgState tv;
                    const int* src = reinterpret_cast<const int*>(tab + img);
                    int* dst = reinterpret_cast<int*>(&tv);
#pragma unroll
                    for (int q = 0; q < (int)(sizeof(ImgState) / sizeof(int)); ++q) dst[q] = __ldcg(src + q);
                    s = tv.s; status = tv.status; it = tv.it; nrep = tv.nrep; kind = tv.kind;
                    final_rep = tv.final_rep != 0; restart_due = tv.restart_due != 0;
                    rr_prev = tv.rr_prev; bb = tv.bb; rr_true = tv.rr_true; rel = tv.rel; be_pred = tv.be_pred;
                    jtol = tv.jtol;
                }
            }
        }
        double part[kNPart] = {};
#pragma unroll 1
        for (int piece = 0; piece < (BATCH ? 2 : 1); ++piece) {
            const int pu0 = piece ? u0b : u0, pv0 = piece ? v0b : v0, pv1 = piece ? v1b : v1;
            if (!(pv1 > pv0) || done) continue;
            // every strip of the image full: one code path for the whole grid
            // (a grid that mixes both paths on one SM runs slower)
            const bool fullw = !BATCH && geo.W % cfg_strip(CFG) == 0;
            if (kind == KIND_KRYLOV && pcg_mode && fullw)
                run_sweep<TLo, OPLO, OPHI, MIXED, CFG, KIND_KRYLOV, OPLO == OP_SYMD, true>(A, geo, smem, pu0, pv0, pv1,
                                                                                          s, part, pp);
            else if (kind == KIND_KRYLOV && pcg_mode)
                run_sweep<TLo, OPLO, OPHI, MIXED, CFG, KIND_KRYLOV, OPLO == OP_SYMD>(A, geo, smem, pu0, pv0, pv1, s,
                                                                                    part, pp);
            else if (kind == KIND_KRYLOV && fullw)
                run_sweep<TLo, OPLO, OPHI, MIXED, CFG, KIND_KRYLOV, false, true>(A, geo, smem, pu0, pv0, pv1, s, part,
                                                                                 pp);
            else if (kind == KIND_KRYLOV)
                run_sweep<TLo, OPLO, OPHI, MIXED, CFG, KIND_KRYLOV>(A, geo, smem, pu0, pv0, pv1, s, part, pp);
            else if (kind == KIND_REPLACE)
                run_sweep<TLo, OPLO, OPHI, MIXED, CFG, KIND_REPLACE>(A, geo, smem, pu0, pv0, pv1, s, part, pp);
            else
                run_sweep<TLo, OPLO, OPHI, MIXED, CFG, KIND_JACOBI>(A, geo, smem, pu0, pv0, pv1, s, part, pp);
        }
        if constexpr (BATCH) {
            // per-image sums + "CTAs still working" over the grid (last component)
            double* parts = A.partials + (size_t)parity * G * (kNPart + 1);
            double running;
            if (pcg_mode) {
                double v6[kNPart + 1] = {part[0], part[1], part[2], part[3], part[4], done ? 0.0 : 1.0};
                ok = grid_allreduce_seg<kNPart + 1>(A.gb, parts, G, lo, hi, A.limit_ns, v6, red);
#pragma unroll
                for (int k = 0; k < kNPart; ++k) part[k] = v6[k];
                running = v6[kNPart];
            } else {
                double v5[kNPart] = {part[0], part[1], part[2], part[3], done ? 0.0 : 1.0};
                ok = grid_allreduce_seg<kNPart>(A.gb, parts, G, lo, hi, A.limit_ns, v5, red);
#pragma unroll
                for (int k = 0; k < 4; ++k) part[k] = v5[k];
                running = v5[4];
            }
            if (!ok) break;
            parity ^= 1;
            if (!(running > 0.0)) break;  // no CTA worked in this sweep: every image is done
            if (prev_running >= 0.0 && running < prev_running) redeal = true;
            prev_running = running;
            if (done) continue;
        } else {
            // four sums for CG, GD and Jacobi; PCG adds r.r
            double* parts = A.partials + (size_t)parity * G * kNPart;
            if (pcg_mode) ok = grid_allreduce<kNPart>(A.gb, parts, G, A.limit_ns, part, red);
            else ok = grid_allreduce<4>(A.gb, parts, G, A.limit_ns, *reinterpret_cast<double(*)[4]>(part), red);
            if (!ok) break;
            parity ^= 1;
        }
        const double (&tot)[kNPart] = part;

        if (kind == KIND_KRYLOV) {
            s.c ^= 1;
            ++it;
            // CG: rr = r.r, rq = r.q, qq = q.q.  Jacobi PCG: rr = r.z, rq = q.z,
            // qq = q.M^-1 q (z = M^-1 r, M = diag(d)); tot[4] = r.r.  The same
            // recurrence then predicts the next r.r (CG) or r.z (PCG).
            const double rr = tot[0], pq = tot[1], rq = tot[2], qq = tot[3];
            if (isfinite(rr) && !(rr > 1e-32 * bb)) {
                // residual at the end of FP64 precision (exactly 0 on tiny
                // systems iterated with rtol = 0): converged, not broken down
                s.ad = 0.0; s.af = 0.f;
                kind = KIND_REPLACE;
                final_rep = true;
                continue;
            }
            if (!(pq > 0.0) || !isfinite(pq) || !isfinite(rr)) {
                status = GM_ERR_BREAKDOWN;
                s.ad = 0.0; s.af = 0.f;
                kind = KIND_REPLACE;
                final_rep = true;
                continue;
            }
            const double al = rr / pq;
            double rr_pred = rr - 2.0 * al * rq + al * al * qq;
            if (rr_pred < 0.0) rr_pred = 0.0;
            rr_prev = rr;
            be_pred = rr_pred / rr;
            s.ad = al;
            s.af = (float)al;
            const bool rep_due = A.replace_every > 0 && it % A.replace_every == 0;
            restart_due = A.restart > 0 && it % A.restart == 0;
            // PCG tests the residual of this sweep (r.r is exact, one iteration
            // behind the CG prediction)
            const bool tol_hit = A.rtol > 0.0 && (A.solver == GM_SOLVER_PCG ? tot[4] : rr_pred) <= A.rtol * A.rtol * bb;
            if (rep_due || restart_due || tol_hit || it >= A.max_iters) {
                kind = KIND_REPLACE;
                final_rep = it >= A.max_iters;
            } else {
                kind = KIND_KRYLOV;
                s.skipR = false;
                const double be = gd ? 0.0 : rr_pred / rr;
                s.bf = (float)be;
                s.beta_zero = gd;
            }
        } else if (kind == KIND_REPLACE) {
            s.xsel ^= 1;
            ++nrep;
            if (bb < 0.0) {
                bb = tot[1];
                if (!(bb > 0.0)) bb = tot[0] > 0.0 ? tot[0] : 1.0;
            }
            rr_true = tot[0];
            rel = sqrt(rr_true / bb);
            if (!isfinite(rr_true)) status = GM_ERR_BREAKDOWN;
            if (final_rep || (A.rtol > 0.0 && rel <= A.rtol) || it >= A.max_iters || !isfinite(rr_true)) {
                if constexpr (BATCH) {
                    done = true;
                    if ((int)blockIdx.x == lo && tid == 0) {  // the image's lead reports it now
                        SolverOut* o = A.outs + img;
                        o->status = (status == GM_OK && A.rtol > 0.0 && !(rel <= A.rtol)) ? GM_ERR_NOT_CONVERGED : status;
                        o->iters = it;
                        o->replacements = nrep;
                        o->where = 0;
                        o->rr_true = rr_true;
                        o->bb = bb;
                        o->rel = rel;
                        A.img_done[img] = 1;
                    }
                    continue;
                } else {
                    break;
                }
            }
            if (jac) {
                // the in-sweep residual met its target but the true one did
                // not: go on iterating, aiming lower by the observed ratio
                jtol *= 0.98 * A.rtol / rel;
                kind = KIND_JACOBI;
                continue;
            }
            const bool bz = restart_due || gd || !(rr_prev > 0.0);
            // after a replacement CG rescales with the true residual; PCG keeps
            // the predicted r.z ratio (the replacement sweep has no diagonal)
            const double be = bz ? 0.0 : (A.solver == GM_SOLVER_PCG ? be_pred : rr_true / rr_prev);
            s.bf = (float)be;
            s.beta_zero = bz;
            s.skipR = true;
            s.af = 0.f;
            s.ad = 0.0;
            restart_due = false;
            kind = KIND_KRYLOV;
        } else {  // Jacobi
            s.xsel ^= 1;
            ++it;
            if (bb < 0.0) {
                bb = tot[1];
                if (!(bb > 0.0)) bb = tot[0] > 0.0 ? tot[0] : 1.0;
            }
            const double rl = sqrt(tot[0] / bb);
            if ((A.rtol > 0.0 && rl <= jtol) || it >= A.max_iters || !isfinite(tot[0])) {
                // the replacement sweep checks the true residual in FP64
                kind = KIND_REPLACE;
                final_rep = it >= A.max_iters || !isfinite(tot[0]);
                s.ad = 0.0; s.af = 0.f;
            }
        }
    }
    // batched images report when they finish; here only those cut short
    const bool reporter = BATCH ? (img >= 0 && !done && (int)blockIdx.x == lo) : blockIdx.x == 0;
    if (reporter && tid == 0) {
        SolverOut* o = BATCH ? A.outs + img : A.out;
        const int ab = ld_volatile_int(&A.gb->abort);
        if (ab) status = ab;
        else if (status == GM_OK && A.rtol > 0.0 && !(rel <= A.rtol)) status = GM_ERR_NOT_CONVERGED;
        o->status = status;
        o->iters = it;
        o->replacements = nrep;
        o->where = A.gb->where;
        o->rr_true = rr_true;
        o->bb = bb;
        o->rel = rel;
    }
    __syncthreads();
    if (tid == 0)
        for (int i = 0; i < kRvMax + kRbMax; ++i) {
            mbar_inval(&full[i]);
            mbar_inval(&empty[i]);
        }
}

}  // namespace gm

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
#include "gm_solver_host.inc"
#include "gm_batch_host.inc"
