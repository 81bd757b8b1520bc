// gm_solver_api.h -- internal interface between the C-ABI front ends and the
// persistent solver driver (gm_solver.cu).
#pragma once

#include "gm_solver.cuh"

namespace gm {

// One operator source: band planes on the device, addressed as a 3-D tensor
// {W, H, planes} with byte strides between rows and between planes.
struct OpSource {
    int kind;                 // OP_SYMD, OP_SYMI (12 planes) or OP_REF25 (25 planes)
    CUtensorMapDataType dt;   // element type of the planes
    int esize;                // bytes per element
    const void* base;         // plane 0, row 0
    uint64_t row_stride;      // bytes, multiple of 16
    uint64_t plane_stride;    // bytes, multiple of 16
    int planes;
};

struct SolverSetup {
    int W, H;
    OpSource lo;              // operator of the Krylov / Jacobi sweeps
    OpSource hi;              // true operator (replacement sweeps)
    bool mixed;               // keep the solution in FP64 between replacements
    const float* xlo;         // OP_SYMD iteration operator: diagonal plane [H][xlo_pitch]
    int xlo_pitch;
    const float* xhi;         // OP_SYMI true operator: gamma plane [H][xhi_pitch]
    int xhi_pitch;
    const float* b;           // [H][bpitch]
    int bpitch;
    const float* alpha_in;    // [H][alpha_pitch]
    float* alpha_out;
    int alpha_pitch;
    void* workspace;          // optional caller-provided scratch (NULL: allocate)
    size_t workspace_bytes;
    bool no_sync;             // do not wait for / read back the result
};

int run_solver(const SolverSetup& S, const gm_solve_params* p, gm_solve_info* info, cudaStream_t st);

// Multigrid-preconditioned CG on the symmetric store (gm_mg.cu): b is
// [H][bpitch], alpha_in / alpha_out [H][W] (may alias).
int run_mg_solver(const gm_levin_store* store, const float* b, int bpitch, const float* alpha_in, float* alpha_out,
                  const gm_solve_params* p, gm_solve_info* info, cudaStream_t st);

}  // namespace gm
