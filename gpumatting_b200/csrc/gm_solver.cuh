// gm_solver.cuh -- argument blocks shared by the persistent solver kernel
// and its host driver.
#pragma once

#include "gm_internal.cuh"

namespace gm {

enum SweepKind { KIND_KRYLOV = 0, KIND_REPLACE = 1, KIND_JACOBI = 2, NKIND = 3 };
// OP_SYMD: 12 affinity planes + a diagonal plane, y = d x - sum w x_j
// OP_SYMI: 12 affinity planes + gamma, y = gamma x + sum w (x - x_j)
// OP_REF25: the reference's 25 explicit FP32 bands
enum OpKind { OP_SYMD = 0, OP_SYMI = 1, OP_REF25 = 2 };

// Launch configurations (the kernels' CFG template argument).  A CTA owns a
// strip of kWarpCols * NCOL columns: NCOL consumer warps side by side, each
// owning 64 columns (two adjacent pixels per lane), plus one TMA producer
// warp.
//   CFG  NCOL  strip  CTAs/SM  rings
//   0    3     192    3        shallow
//   1    3     192    2        deep
//   2    2     128    4        shallow
constexpr int kNumCfg = 3;
__host__ __device__ constexpr int cfg_ncol(int cfg) { return cfg == 2 ? 2 : 3; }
__host__ __device__ constexpr int cfg_cps(int cfg) { return cfg == 0 ? 3 : cfg == 1 ? 2 : 4; }
constexpr int kWarpCols = 64;                    // output columns per consumer warp (2 per lane)
__host__ __device__ constexpr int cfg_strip(int cfg) { return kWarpCols * cfg_ncol(cfg); }
// TMA box width: strip + 8 columns each side (every box x stays 16-byte aligned)
__host__ __device__ constexpr int cfg_box(int cfg) { return cfg_strip(cfg) + 16; }
__host__ __device__ constexpr int cfg_threads(int cfg) { return 32 * (cfg_ncol(cfg) + 1); }
// Operand ring rows (stencil operand of each consumer warp) and own-row ring
// rows (r or b of the rows being output).
constexpr int kOpRows = 8;
constexpr int kOwnRows = 4;
constexpr int kRingCols = kWarpCols + 4;         // private operand ring: warp columns + 2 each side
constexpr int kRvMax = 16;                       // vector ring slots
constexpr int kRbMax = 16;                       // band ring slots
constexpr int kNPart = 5;                        // FP64 partial sums per CTA per sweep
// reduction scratch: per-warp sums + grid totals of up to kNPart + 1 values
__host__ __device__ constexpr int cfg_red_bytes(int cfg) { return (cfg_threads(cfg) / 32 + 1) * (kNPart + 1) * 8; }

// Shared-memory carve of one sweep kind.  Everything here is a compile-time
// function of the operator types, so the hot loop indexes rings with
// constants; the host uses the same functions to size the launch.
struct KindLayout {
    int D;          // prefetch distance in rows
    int Rv, Rb;     // ring slots
    int vslot;      // bytes per vector slot
    int bslot;      // bytes per band slot
    int vbase;      // offset of the vector ring in the ring area
    int bbase;      // offset of the band ring in the ring area
    int voff[5];    // offsets of the vector rows inside a vector slot
    int vbytes[5];  // TMA bytes of each vector row (0 = unused)
    int planes;     // band planes loaded per row
    int pstride;    // bytes between planes inside a band slot (= box * elem)
    int xoff;       // offset of the extra plane row (diagonal or gamma), -1 none
    int bbytes;     // TMA bytes of one band row (planes + extra)
};

__host__ __device__ constexpr int a128(int x) { return (x + 127) & ~127; }

// Vector rows per step: Krylov r, q, p, x increment, and the diagonal d for
// the Jacobi preconditioner (symmetric store; loaded only by PCG solves);
// replacement base (FP64, mixed only), x increment, p, b; Jacobi x, -, -, b.
__host__ __device__ constexpr KindLayout kind_layout(int kind, int op, int esize, bool mixed, int Rv, int Rb, int box)
{
    KindLayout K{};
    const int vb4 = box * 4;
    int vb[5] = {0, 0, 0, 0, 0};
    if (kind == KIND_KRYLOV) {
        vb[0] = vb4; vb[1] = vb4; vb[2] = vb4; vb[3] = vb4;
        vb[4] = op == OP_SYMD ? vb4 : 0;
    }
    else if (kind == KIND_REPLACE) { vb[0] = mixed ? 2 * vb4 : 0; vb[1] = vb4; vb[2] = vb4; vb[3] = vb4; }
    else { vb[0] = vb4; vb[3] = vb4; }
    int off = 0;
    for (int i = 0; i < 5; ++i) {
        K.voff[i] = off;
        K.vbytes[i] = vb[i];
        off += a128(vb[i]);
    }
    K.vslot = off;
    const bool sym = op != OP_REF25;
    K.planes = sym ? 12 : 25;
    K.pstride = box * esize;
    const int pbytes = K.planes * K.pstride;
    K.xoff = sym ? a128(pbytes) : -1;
    K.bbytes = pbytes + (sym ? box * 4 : 0);
    K.bslot = sym ? a128(K.xoff + box * 4) : a128(pbytes);
    K.D = Rv - 1;
    K.Rv = Rv;
    K.Rb = Rb;
    K.vbase = 0;
    K.bbase = a128(Rv * K.vslot);
    return K;
}

// Ring slots per kind for a configuration.  A super-step holds two vector
// slots and (symmetric store) four band slots, so Rv >= 2 and Rb >= 4 (2 for
// the reference layout) always make progress; extra slots are prefetch.
// Configs 0 and 2 fit three (four) CTAs per SM with a 2-byte store, config 1
// trades one CTA per SM for rings about twice as deep.  Config 0's fifth
// Krylov vector slot is the room the replacement sweep's operand ring leaves
// by overlapping the Krylov rings (make_layout).
__host__ __device__ constexpr int rings_v(int kind, int oplo, int cfg)
{
    return kind == KIND_KRYLOV ? (cfg == 1 && oplo == OP_SYMD ? 8 : cfg == 0 && oplo == OP_SYMD ? 5 : 4)
                               : (cfg == 1 && oplo == OP_SYMD ? 3 : 2);
}
__host__ __device__ constexpr int rings_b(int kind, int oplo, int cfg)
{
    return kind == KIND_KRYLOV ? (oplo == OP_REF25 ? 4 : (cfg == 1 ? 10 : 7))
                               : (oplo == OP_REF25 ? 2 : (cfg == 1 ? 6 : 4));
}

// Element type of the operand ring in replacement sweeps: FP64 when the
// solution is kept in FP64 (mixed), FP32 otherwise.
__host__ __device__ constexpr int ring_esize(bool mixed) { return mixed ? 8 : 4; }

// The vector and band rings of a sweep share one area whose split depends on
// the sweep kind (a sweep starts with both rings drained).
struct Layout {
    int ring_bytes, pring_off, pringd_off, rring_off, full_off, empty_off, red_off, total;
    KindLayout k[NKIND];
};

__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }

__host__ __device__ constexpr Layout make_layout(int oplo, int esize_lo, int ophi, bool mixed, int cfg)
{
    Layout L{};
    const int box = cfg_box(cfg), ncol = cfg_ncol(cfg);
    for (int k = 0; k < NKIND; ++k)
        L.k[k] = kind_layout(k, k == KIND_KRYLOV ? oplo : ophi, k == KIND_KRYLOV ? esize_lo : 4, mixed,
                             rings_v(k, oplo, cfg), rings_b(k, oplo, cfg), box);
    int cap[NKIND] = {};
    for (int k = 0; k < NKIND; ++k) cap[k] = L.k[k].bbase + L.k[k].Rb * L.k[k].bslot;
    L.ring_bytes = a128(imax(cap[KIND_KRYLOV], imax(cap[KIND_REPLACE], cap[KIND_JACOBI])));
    // Operand rings: the float one (Krylov and Jacobi sweeps) after the larger
    // of those kinds' TMA rings; the replacement sweep's (FP64 when mixed)
    // after its own TMA rings, where it may overlap the Krylov rings and the
    // float ring, which a replacement sweep does not use (every load of a
    // sweep has landed and been read before the next sweep starts).
    const int pf = a128(ncol * kOpRows * kRingCols * 4);
    const int pd = a128(ncol * kOpRows * kRingCols * ring_esize(mixed));
    L.pring_off = a128(imax(cap[KIND_KRYLOV], cap[KIND_JACOBI]));
    L.pringd_off = a128(cap[KIND_REPLACE]);
    L.rring_off = imax(L.pring_off + pf, L.pringd_off + pd);
    L.full_off = L.rring_off + a128(ncol * kOwnRows * kWarpCols * 4);
    L.empty_off = L.full_off + a128((kRvMax + kRbMax) * 8);
    L.red_off = L.empty_off + a128((kRvMax + kRbMax) * 8);
    L.total = L.red_off + a128(cfg_red_bytes(cfg) + 16);  // + abort flag at red_off + cfg_red_bytes
    return L;
}

struct SolverOut {
    int status;
    int iters;
    int replacements;
    int where;
    double rr_true;
    double bb;
    double rel;
};

// One image of a batched solve.  Images are stacked in one canvas, image k
// occupying canvas rows y0 .. y0+H-1 (columns 0 .. W-1) with two zero rows
// between neighbours; its CTAs are c0 .. c0+units-1 (their rows are in the
// BatchUnit table).
struct BatchImage {
    int y0, W, H;
    int c0, units;
    int pad_[3];
    float* alpha;             // [H][W] device: initial guess in, solution out
};

// A CTA's share of a batched solve: rows of up to two strips of one image
// (a run of strip-rows that may continue from the bottom of one strip into
// the top of the next), so the CTAs of an image get equal row counts to
// within one row.  Rows are canvas rows; v1 <= v0 marks an absent piece.
struct BatchUnit {
    int img;                  // -1: no work
    int u0[2];                // strip start column
    int v0[2], v1[2];         // canvas rows [v0, v1)
    int pad_;
};

// Where a CTA's unit lives: image width for masking, and where its solution
// rows go (row vr of the canvas is row vr - arow0 of aout).
struct UnitGeo {
    int W;
    int arow0;
    int apitch;
    float* aout;
    const float* ain;
};

struct SolverArgs {
    // Tensor maps: vectors are 2-D {W, H}; bands 3-D {W, H, planes}.
    CUtensorMap m_r[2], m_q[2], m_p[2], m_xacc[2], m_base[2];
    CUtensorMap m_wlo, m_whi, m_xlo, m_xhi, m_b;  // planes; extra plane (d or gamma) of each op; rhs
    float* r[2];
    float* q[2];
    float* p[2];
    float* xacc[2];
    double* base[2];
    const float* b;           // caller's right-hand side
    int bpitch;               // elements
    float* bw;                // work copy of b, pitch P (read through m_b)
    const float* alpha_in;
    float* alpha_out;
    int alpha_pitch;          // elements
    int P;                    // pitch (elements) of the work vectors
    int W, H;
    int nstrips, nseg, nunits;
    int strip;                // strip width of the configuration (columns)
    double* partials;         // [2][kNPart][grid]
    GridBarrier* gb;
    SolverOut* out;
    // parameters
    int solver;
    double rtol;
    int max_iters;
    int restart;
    int replace_every;
    float omega;
    uint64_t limit_ns;       // grid-barrier wait limit
    uint64_t tma_limit_ns;   // TMA / ring wait limit (never below 2 s)
    int inject;              // 1: first grid barrier expects one extra arrival
    // batched solves (BATCH kernels only)
    const BatchImage* imgs;
    const BatchUnit* units;  // [grid]
    void* states;            // [nimg] solver state of each image, for re-deals
    int* img_done;           // [nimg] set when an image has finished (zeroed before launch)
    int nimg;
    SolverOut* outs;         // [nimg]
};

}  // namespace gm
