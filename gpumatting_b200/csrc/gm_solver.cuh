// gm_solver.cuh -- argument blocks shared by the persistent solver kernel
// and its host driver.
#pragma once

#include "gm_internal.cuh"

namespace gm {

enum SweepKind { KIND_KRYLOV = 0, KIND_REPLACE = 1, KIND_JACOBI = 2, NKIND = 3 };
enum OpKind { OP_SYM = 0, OP_REF25 = 1 };

constexpr int kThreads = 256;     // threads per CTA
constexpr int kMaxStrip = 240;    // strip width limit: box width cw+16 <= 256
constexpr int kRvMax = 16;        // vector ring slots
constexpr int kRbMax = 24;        // band ring slots
constexpr int kNPart = 4;         // FP64 partial sums per CTA per sweep

// Shared-memory carve of one sweep kind.  Offsets are bytes from the start
// of dynamic shared memory; every TMA destination is 128-byte aligned.
struct KindLayout {
    int D;          // prefetch distance in rows
    int Rv, Rb;     // ring slots
    int vslot;      // bytes per vector slot
    int bslot;      // bytes per band slot
    int voff[4];    // offsets of the vector arrays inside a vector slot
    int vbytes[4];  // TMA bytes of each vector row (0 = unused)
    int nvec;
    int planes;     // band planes loaded per row
    int pstride;    // bytes between planes inside a band slot (= bw * elem)
    int gamma_off;  // offset of the gamma row inside a band slot (-1 none)
    int bbytes;     // TMA bytes of the band planes of one row
};

struct Layout {
    int cw, bw;
    int vring_off, bring_off, pring_off, rring_off, bar_off, red_off, total;
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
    CUtensorMap m_wlo, m_whi, m_gamma, m_b;
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
    uint64_t tma_limit_ns;   // TMA row wait limit (never below 2 s)
    int inject;              // 1: first grid barrier expects one extra arrival
};

}  // namespace gm
