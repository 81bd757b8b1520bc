// gm_solver.cu -- persistent fused solvers for the Levin system
//     (L + diag(gamma)) x = b
// on a W x H pixel grid: conjugate gradient, steepest descent and damped
// Jacobi (the reference's cgSolve / gradSolve / jacobi, main.cu:406-556),
// each run as ONE cooperative kernel with no host round trip per iteration.
//
// Work decomposition.  The image is cut into column strips of `cw` pixels
// and each strip into row segments; one CTA owns one (strip, segment) unit
// and sweeps down it row by row.  At every row step a single thread issues
// TMA loads (cp.async.bulk.tensor, no multicast) of one halo'd row
// (cw + 16 columns starting 8 left of the strip, zero fill outside the
// image) of the input vectors and, two rows behind, of the band planes into
// shared-memory rings completed on mbarriers.  Rows v-2..v+2 of the stencil
// operand stay in a 6-row ring, so each band element and each vector
// element is read from HBM once per sweep (plus the 2-row and 8-column
// halos, which neighbouring CTAs read too and normally hit in L2).
//
// Operators.  OP_SYM: 12 planes of upper affinities w_k (k = du + 5 dv) plus
// gamma; the lower half is read from the rows above (w_k(u-du, v-dv)) and
// the Laplacian diagonal is implicit: y_i = gamma_i x_i + sum_j w_ij (x_i -
// x_j), so rows sum to zero exactly whatever the storage precision.
// OP_REF25: the reference's 25 explicit FP32 bands (main.cu:164-194).
//
// CG iteration (one sweep, one grid barrier).  Sweep k, given alpha_{k-1}
// and beta_k from the previous barrier, forms on the fly (halo included)
//   r_k = r_{k-1} - alpha_{k-1} q_{k-1},  p_k = r_k + beta_k p_{k-1},
// applies q_k = A p_k, adds alpha_{k-1} p_{k-1} into the local solution
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
// residual r = b - A_hi x with FP64 accumulation over the FP32 planes, and
// writes alpha out.  With FP16/BF16 iteration planes this is the
// reliable-update scheme that keeps the iterate converging to the FP32
// operator's solution.
//
// Every wait (grid barrier, TMA row) has a wall-clock limit; on expiry the
// kernel records GM_ERR_TIMEOUT and all CTAs leave their loops.
#include "gm_solver.cuh"

namespace gm {

__host__ __device__ constexpr int sym_dv(int k) { return (k + 2) / 5; }
__host__ __device__ constexpr int sym_du(int k) { return k - 5 * ((k + 2) / 5); }

// y = gamma x0 + sum_k w_k(u,v)(x0 - x(u+du,v+dv)) + w_k(u-du,v-dv)(x0 - x(u-du,v-dv))
// prow[d]: operand row v+d-2; brow[d]: band slot of row v-d.
template <class T, class V, class Acc>
__device__ __forceinline__ Acc sym_apply(const V* const (&prow)[5], const unsigned char* const (&brow)[3],
                                         int pstride, int gamma_off, int cc)
{
    const Acc x0 = static_cast<Acc>(prow[2][cc]);
    const float* g = reinterpret_cast<const float*>(brow[0] + gamma_off);
    Acc y = static_cast<Acc>(g[cc]) * x0;
#pragma unroll
    for (int k = 1; k <= 12; ++k) {
        const int du = sym_du(k), dv = sym_dv(k);
        const T* wu = reinterpret_cast<const T*>(brow[0] + (k - 1) * pstride);
        const T* wl = reinterpret_cast<const T*>(brow[dv] + (k - 1) * pstride);
        const Acc w1 = static_cast<Acc>(Cvt<T>::to_f(wu[cc]));
        const Acc w2 = static_cast<Acc>(Cvt<T>::to_f(wl[cc - du]));
        y += w1 * (x0 - static_cast<Acc>(prow[2 + dv][cc + du]));
        y += w2 * (x0 - static_cast<Acc>(prow[2 - dv][cc - du]));
    }
    return y;
}

// Diagonal of the symmetric operator: gamma + sum of the row's affinities.
template <class T>
__device__ __forceinline__ float sym_diag(const unsigned char* const (&brow)[3], int pstride, int gamma_off,
                                          int cc)
{
    float d = reinterpret_cast<const float*>(brow[0] + gamma_off)[cc];
#pragma unroll
    for (int k = 1; k <= 12; ++k) {
        const int du = sym_du(k), dv = sym_dv(k);
        d += Cvt<T>::to_f(reinterpret_cast<const T*>(brow[0] + (k - 1) * pstride)[cc]);
        d += Cvt<T>::to_f(reinterpret_cast<const T*>(brow[dv] + (k - 1) * pstride)[cc - du]);
    }
    return d;
}

// y = sum_{band j} a_j(u,v) x(u+du_j, v+dv_j), band j = 12 + du + 5 dv, in
// band order (BandedMatrix.cu:172-173).
template <class V, class Acc>
__device__ __forceinline__ Acc ref25_apply(const V* const (&prow)[5], const unsigned char* b0, int pstride, int cc)
{
    Acc y = 0;
#pragma unroll
    for (int j = 0; j < 25; ++j) {
        const int du = j % 5 - 2;   // j = 12 + du + 5 dv
        const int dv = j / 5 - 2;
        const float a = reinterpret_cast<const float*>(b0 + j * pstride)[cc];
        y += static_cast<Acc>(a) * static_cast<Acc>(prow[2 + dv][cc + du]);
    }
    return y;
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

template <class TLo, int OPLO, int OPHI, bool MIXED, int KIND>
__device__ __forceinline__ void run_sweep(const SolverArgs& A, unsigned char* smem, int u0, int v0, int v1,
                                          const KState& s, double (&part)[kNPart], uint32_t& vphase,
                                          uint32_t& bphase)
{
    const Layout& L = A.lay;
    const KindLayout& K = L.k[KIND];
    const int tid = threadIdx.x;
    const int cw = L.cw, bw = L.bw;
    const int nsteps = v1 - v0 + 4;
    const int nband = nsteps - 2;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
    unsigned char* vring = smem + L.vring_off;
    unsigned char* bring = smem + L.bring_off;
    const int W = A.W, P = A.P;

    // Tensor maps of this sweep's row loads (slot order fixed by plan_layout).
    const CUtensorMap* vm[4] = {nullptr, nullptr, nullptr, nullptr};
    if (KIND == KIND_KRYLOV) {
        vm[0] = &A.m_r[s.c]; vm[1] = &A.m_q[s.c]; vm[2] = &A.m_p[s.c]; vm[3] = &A.m_xacc[s.xsel];
    } else if (KIND == KIND_REPLACE) {
        vm[0] = MIXED ? &A.m_base[s.xsel] : nullptr; vm[1] = &A.m_xacc[s.xsel]; vm[2] = &A.m_p[s.c];
        vm[3] = &A.m_b;
    } else {
        vm[0] = &A.m_xacc[s.xsel]; vm[3] = &A.m_b;
    }
    const bool use_hi = KIND != KIND_KRYLOV;
    const CUtensorMap* bm = use_hi ? &A.m_whi : &A.m_wlo;
    const bool sym = (use_hi ? OPHI : OPLO) == OP_SYM;

    auto issue_vec = [&](int j) {
        const int slot = j % K.Rv;
        uint64_t* bar = &bars[slot];
        uint32_t bytes = K.vbytes[0] + K.vbytes[1] + K.vbytes[2] + K.vbytes[3];
        mbar_arrive_expect_tx(bar, bytes);
        unsigned char* dst = vring + slot * K.vslot;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (K.vbytes[i]) tma_load_2d(dst + K.voff[i], vm[i], u0 - 8, v0 - 2 + j, bar);
    };
    auto issue_band = [&](int m) {
        const int slot = m % K.Rb;
        uint64_t* bar = &bars[kRvMax + slot];
        uint32_t bytes = K.bbytes + (sym ? bw * 4 : 0);
        mbar_arrive_expect_tx(bar, bytes);
        unsigned char* dst = bring + slot * K.bslot;
        tma_load_3d(dst, bm, u0 - 8, v0 - 2 + m, 0, bar);
        if (sym) tma_load_2d(dst + K.gamma_off, &A.m_gamma, u0 - 8, v0 - 2 + m, bar);
    };

    if (tid == 0) {
        fence_proxy_async();
        const int nv = K.D < nsteps ? K.D : nsteps;
        for (int j = 0; j < nv; ++j) issue_vec(j);
        for (int m = 0; m < K.D - 2 && m < nband; ++m) issue_band(m);
    }

    float* pring_f = reinterpret_cast<float*>(smem + L.pring_off);
    double* pring_d = reinterpret_cast<double*>(smem + L.pring_off);
    float* rring = reinterpret_cast<float*>(smem + L.rring_off);

    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + L.red_off + 32 * kNPart * 8);
    for (int j = 0; j < nsteps; ++j) {
        const int Lr = v0 - 2 + j;
        {
            const int vs = j % K.Rv;
            if (*s_abort || !mbar_wait_bounded(&bars[vs], (vphase >> vs) & 1u, A.gb, A.tma_limit_ns)) *s_abort = 1;
            vphase ^= 1u << vs;
        }
        const unsigned char* vs_ptr = vring + (j % K.Rv) * K.vslot;
        // ---------------- phase A: combine the incoming row ----------------
        if (tid < cw + 4) {
            const int cc = tid + 6;
            const int uo = u0 + tid - 2;
            const bool own = tid >= 2 && tid < cw + 2 && uo < W && Lr >= v0 && Lr < v1;
            const size_t gi = (size_t)Lr * P + uo;
            if (KIND == KIND_KRYLOV) {
                const float rv = reinterpret_cast<const float*>(vs_ptr + K.voff[0])[cc];
                const float qv = reinterpret_cast<const float*>(vs_ptr + K.voff[1])[cc];
                const float pv = reinterpret_cast<const float*>(vs_ptr + K.voff[2])[cc];
                const float rn = s.skipR ? rv : fmaf(-s.af, qv, rv);
                const float pn = s.beta_zero ? rn : fmaf(s.bf, pv, rn);
                pring_f[(j % 6) * bw + cc] = pn;
                if (own) {
                    rring[(j & 3) * cw + tid - 2] = rn;
                    A.r[s.c ^ 1][gi] = rn;
                    A.p[s.c ^ 1][gi] = pn;
                    if (!s.skipR)
                        A.xacc[s.xsel][gi] = fmaf(s.af, pv, reinterpret_cast<const float*>(vs_ptr + K.voff[3])[cc]);
                    part[0] += (double)rn * (double)rn;
                }
            } else if (KIND == KIND_REPLACE) {
                const float xv = reinterpret_cast<const float*>(vs_ptr + K.voff[1])[cc];
                const float pv = reinterpret_cast<const float*>(vs_ptr + K.voff[2])[cc];
                double xf;
                if (MIXED) {
                    const double bv = reinterpret_cast<const double*>(vs_ptr + K.voff[0])[cc];
                    xf = bv + (double)xv + s.ad * (double)pv;
                } else {
                    xf = (double)fmaf(s.af, pv, xv);
                }
                pring_d[(j % 6) * bw + cc] = xf;
                if (own) {
                    if (MIXED) {
                        A.base[s.xsel ^ 1][gi] = xf;
                        A.xacc[s.xsel ^ 1][gi] = 0.f;
                    } else {
                        A.xacc[s.xsel ^ 1][gi] = (float)xf;
                    }
                }
            } else {  // Jacobi
                pring_f[(j % 6) * bw + cc] = reinterpret_cast<const float*>(vs_ptr + K.voff[0])[cc];
            }
            if (KIND != KIND_KRYLOV && tid >= 2 && tid < cw + 2)
                rring[(j & 3) * cw + tid - 2] = reinterpret_cast<const float*>(vs_ptr + K.voff[3])[cc];
        }
        __syncthreads();
        if (*s_abort) return;  // uniform: read after the barrier by every thread
        if (tid == 0) {
            fence_proxy_async();
            if (j + K.D < nsteps) issue_vec(j + K.D);
            const int m = j + K.D - 2;
            if (m >= 0 && m < nband) issue_band(m);
        }
        if (j >= 2) {
            const int m = j - 2;
            const int bs = m % K.Rb;
            if (*s_abort || !mbar_wait_bounded(&bars[kRvMax + bs], (bphase >> bs) & 1u, A.gb, A.tma_limit_ns))
                *s_abort = 1;
            bphase ^= 1u << bs;
        }
        if (j < 4) continue;
        // ---------------- phase B: stencil on output row v ----------------
        const int v = Lr - 2;
        const int u = u0 + tid;
        if (tid < cw && u < W) {
            const int cc = tid + 8;
            const unsigned char* brow[3] = {bring + ((j - 2) % K.Rb) * K.bslot,
                                            bring + ((j - 3) % K.Rb) * K.bslot,
                                            bring + ((j - 4) % K.Rb) * K.bslot};
            const size_t go = (size_t)v * P + u;
            if (KIND == KIND_KRYLOV) {
                const float* prow[5];
#pragma unroll
                for (int d = 0; d < 5; ++d) prow[d] = pring_f + ((j - 4 + d) % 6) * bw;
                float qv;
                if (OPLO == OP_SYM)
                    qv = sym_apply<TLo, float, float>(prow, brow, K.pstride, K.gamma_off, cc);
                else
                    qv = ref25_apply<float, float>(prow, brow[0], K.pstride, cc);
                A.q[s.c ^ 1][go] = qv;
                const float pn = prow[2][cc];
                const float rn = rring[((j - 2) & 3) * cw + tid];
                part[1] += (double)pn * (double)qv;
                part[2] += (double)rn * (double)qv;
                part[3] += (double)qv * (double)qv;
            } else if (KIND == KIND_REPLACE) {
                const double* prow[5];
#pragma unroll
                for (int d = 0; d < 5; ++d) prow[d] = pring_d + ((j - 4 + d) % 6) * bw;
                double y;
                if (OPHI == OP_SYM)
                    y = sym_apply<float, double, double>(prow, brow, K.pstride, K.gamma_off, cc);
                else
                    y = ref25_apply<double, double>(prow, brow[0], K.pstride, cc);
                const double bv = (double)rring[((j - 2) & 3) * cw + tid];
                const float rf = (float)(bv - y);
                A.r[s.c][go] = rf;
                part[0] += (double)rf * (double)rf;
                part[1] += bv * bv;
                A.alpha_out[(size_t)v * A.alpha_pitch + u] = (float)prow[2][cc];
            } else {  // Jacobi
                const float* prow[5];
#pragma unroll
                for (int d = 0; d < 5; ++d) prow[d] = pring_f + ((j - 4 + d) % 6) * bw;
                float y, dg;
                if (OPHI == OP_SYM) {
                    y = sym_apply<float, float, float>(prow, brow, K.pstride, K.gamma_off, cc);
                    dg = sym_diag<float>(brow, K.pstride, K.gamma_off, cc);
                } else {
                    y = ref25_apply<float, float>(prow, brow[0], K.pstride, cc);
                    dg = reinterpret_cast<const float*>(brow[0] + 12 * K.pstride)[cc];
                }
                const float bv = rring[((j - 2) & 3) * cw + tid];
                const float rv = bv - y;
                const float x0 = prow[2][cc];
                A.xacc[s.xsel ^ 1][go] = x0 + A.omega * rv / dg;
                part[0] += (double)rv * (double)rv;
                part[1] += (double)bv * (double)bv;
            }
        }
    }
}

template <class TLo, int OPLO, int OPHI, bool MIXED>
__global__ void __launch_bounds__(kThreads) solver_kernel(const __grid_constant__ SolverArgs A)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x;
    const Layout& L = A.lay;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar_off);
    double* red = reinterpret_cast<double*>(smem + L.red_off);

    const int unit = blockIdx.x;
    int u0 = 0, v0 = 0, v1 = 0;
    if (unit < A.nunits) {
        const int st = unit % A.nstrips, sg = unit / A.nstrips;
        u0 = st * L.cw;
        v0 = (int)((long long)A.H * sg / A.nseg);
        v1 = (int)((long long)A.H * (sg + 1) / A.nseg);
    }
    const bool active = v1 > v0;

    if (tid == 0) {
        for (int i = 0; i < kRvMax + kRbMax; ++i) mbar_init(&bars[i], 1);
        *reinterpret_cast<volatile int*>(smem + L.red_off + 32 * kNPart * 8) = 0;
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t vphase = 0, bphase = 0;

    const bool jac = A.solver == GM_SOLVER_JACOBI;
    // Import the initial guess; zero the first search direction.
    if (active) {
        for (int v = v0; v < v1; ++v)
            for (int cl = tid; cl < L.cw; cl += blockDim.x) {
                const int u = u0 + cl;
                if (u >= A.W) continue;
                const size_t i = (size_t)v * A.P + u;
                const float a0 = A.alpha_in[(size_t)v * A.alpha_pitch + u];
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
    bool ok = grid_sync(A.gb, G + (A.inject == 1 ? 1u : 0u), A.limit_ns);

    int status = GM_OK, it = 0, nrep = 0, parity = 0;
    int kind = jac ? KIND_JACOBI : KIND_REPLACE;
    KState s;
    s.af = 0.f; s.bf = 0.f; s.ad = 0.0; s.skipR = true; s.beta_zero = true; s.c = 0; s.xsel = 0;
    double rr_prev = 0.0, bb = -1.0, rr_true = 0.0, rel = 0.0;
    bool final_rep = false, restart_due = false;
    const bool gd = A.solver == GM_SOLVER_GD;
    if (jac && A.max_iters <= 0) {
        kind = KIND_REPLACE;
        final_rep = true;
    }

    while (ok) {
        double part[kNPart] = {0.0, 0.0, 0.0, 0.0};
        if (active) {
            if (kind == KIND_KRYLOV)
                run_sweep<TLo, OPLO, OPHI, MIXED, KIND_KRYLOV>(A, smem, u0, v0, v1, s, part, vphase, bphase);
            else if (kind == KIND_REPLACE)
                run_sweep<TLo, OPLO, OPHI, MIXED, KIND_REPLACE>(A, smem, u0, v0, v1, s, part, vphase, bphase);
            else
                run_sweep<TLo, OPLO, OPHI, MIXED, KIND_JACOBI>(A, smem, u0, v0, v1, s, part, vphase, bphase);
        }
        block_sum<kNPart>(part, red);
        double* slot = A.partials + (size_t)parity * G * kNPart + blockIdx.x;
        if (tid == 0) {
#pragma unroll
            for (int k = 0; k < kNPart; ++k) slot[(size_t)k * G] = part[k];
        }
        ok = grid_sync(A.gb, G, A.limit_ns);
        if (!ok) break;
        double tot[kNPart];
        grid_total<kNPart>(A.partials + (size_t)parity * G * kNPart, (int)G, tot, red);
        parity ^= 1;

        if (kind == KIND_KRYLOV) {
            s.c ^= 1;
            ++it;
            const double rr = tot[0], pq = tot[1], rq = tot[2], qq = tot[3];
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
            s.ad = al;
            s.af = (float)al;
            const bool rep_due = A.replace_every > 0 && it % A.replace_every == 0;
            restart_due = A.restart > 0 && it % A.restart == 0;
            const bool tol_hit = A.rtol > 0.0 && rr_pred <= A.rtol * A.rtol * bb;
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
            if (final_rep || (A.rtol > 0.0 && rel <= A.rtol) || it >= A.max_iters || !isfinite(rr_true)) break;
            const bool bz = restart_due || gd || !(rr_prev > 0.0);
            const double be = bz ? 0.0 : rr_true / rr_prev;
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
            if ((A.rtol > 0.0 && rl <= A.rtol) || it >= A.max_iters || !isfinite(tot[0])) {
                kind = KIND_REPLACE;
                final_rep = true;
                s.ad = 0.0; s.af = 0.f;
            }
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        const int ab = ld_volatile_int(&A.gb->abort);
        if (ab) status = ab;
        else if (status == GM_OK && A.rtol > 0.0 && !(rel <= A.rtol)) status = GM_ERR_NOT_CONVERGED;
        A.out->status = status;
        A.out->iters = it;
        A.out->replacements = nrep;
        A.out->where = A.gb->where;
        A.out->rr_true = rr_true;
        A.out->bb = bb;
        A.out->rel = rel;
    }
    __syncthreads();
    if (tid == 0)
        for (int i = 0; i < kRvMax + kRbMax; ++i) mbar_inval(&bars[i]);
}

}  // namespace gm

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
#include "gm_solver_host.inc"
