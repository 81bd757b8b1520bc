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

constexpr int kConsumers = 3;                    // consumer warps per CTA
constexpr int kThreads = 32 * (kConsumers + 1);  // + one TMA producer warp
constexpr int kWarpCols = 64;                    // output columns per consumer warp (2 per lane)
constexpr int kStrip = kWarpCols * kConsumers;   // strip width (192)
constexpr int kBox = kStrip + 16;                // TMA box width: strip + 8 columns each side
constexpr int kRingCols = kWarpCols + 4;         // private operand ring: warp columns + 2 each side
constexpr int kRvMax = 16;                       // vector ring slots
constexpr int kRbMax = 16;                       // band ring slots
constexpr int kNPart = 4;                        // FP64 partial sums per CTA per sweep

// Shared-memory carve of one sweep kind (bytes from the start of dynamic
// shared memory; every TMA destination is 128-byte aligned).
struct KindLayout {
    int D;          // prefetch distance in rows
    int Rv, Rb;     // ring slots
    int vslot;      // bytes per vector slot
    int bslot;      // bytes per band slot
    int voff[4];    // offsets of the vector rows inside a vector slot
    int vbytes[4];  // TMA bytes of each vector row (0 = unused)
    int planes;     // band planes loaded per row
    int pstride;    // bytes between planes inside a band slot (= kBox * elem)
    int xoff;       // offset of the extra plane row (diagonal or gamma), -1 none
    int bbytes;     // TMA bytes of one band row (planes + extra)
    int band_life;  // steps a band row stays in use after its first use (2 sym, 0 ref25)
};

struct Layout {
    int vring_off, bring_off, pring_off, rring_off, full_off, empty_off, red_off, total;
    KindLayout k[NKIND];
};

struct SolverOut {
    int status;
    int iters;
    int replacements;
    int where;
    double rr_true;
    double bb;
    double rel;
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
    Layout lay;
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
};

}  // namespace gm
