// gm_capi.cu -- C-ABI front ends: the native solve entry points and the
// reference-named drop-ins (main.cu, Matting.cu, Solve.cpp).
#include <string.h>

#include <algorithm>
#include <vector>

#include "gm_solver_api.h"

int gm_note_status(int s);

namespace gm {
int generic_solve(const BandedMatrix& L, float* alpha, int pad, const float* b, const gm_solve_params& p,
                  gm_solve_info* info, cudaStream_t st);

// True when offs is the 25-band Levin stencil of an image W wide
// (main.cu:164-190) and rows is a whole number of image rows.
static bool levin_pattern(const int* offs, int nb, int rows, int* W_out)
{
    if (nb != 25) return false;
    const int W = offs[17];  // band 12 + 5: offset W
    if (W < 1 || rows % W != 0) return false;
    for (int dv = -2; dv <= 2; ++dv)
        for (int du = -2; du <= 2; ++du)
            if (offs[12 + du + 5 * dv] != du + W * dv) return false;
    *W_out = W;
    return true;
}

}  // namespace gm

using namespace gm;

static int read_offsets(const BandedMatrix& L, std::vector<int>& offs, cudaStream_t st)
{
    offs.resize(L.nbands > 0 ? L.nbands : 0);
    if (L.nbands <= 0 || !L.bands) { gm_set_error_msg("matrix has no bands"); return GM_ERR_INVALID; }
    GM_CUDA_TRY(cudaMemcpyAsync(offs.data(), L.bands, sizeof(int) * L.nbands, cudaMemcpyDeviceToHost, st));
    GM_CUDA_TRY(cudaStreamSynchronize(st));
    return GM_OK;
}

extern "C" int gm_banded_solve(BandedMatrix L, int W, float* alpha, int pad, const float* b,
                               const gm_solve_params* prm, gm_solve_info* info, void* stream)
{
    gm_solve_params p;
    if (prm) p = *prm; else gm_default_params(&p);
    cudaStream_t st = (cudaStream_t)stream;
    if (!alpha || !b || !L.a || L.rows <= 0) { gm_set_error_msg("gm_banded_solve: bad arguments"); return GM_ERR_INVALID; }
    if (p.solver == GM_SOLVER_PCG || p.solver == GM_SOLVER_MG) {
        gm_set_error_msg("GM_SOLVER_PCG / GM_SOLVER_MG run on the symmetric Levin store (gm_levin_solve), not on 25 bands");
        return GM_ERR_UNSUPPORTED;
    }
    std::vector<int> offs;
    GM_TRY(read_offsets(L, offs, st));
    int Wd = 0;
    const bool lev = levin_pattern(offs.data(), L.nbands, L.rows, &Wd) && (W <= 0 || W == Wd);
    if (!lev) {
        if (W > 0) { gm_set_error_msg("band offsets are not the Levin stencil of width %d", W); return GM_ERR_INVALID; }
        return generic_solve(L, alpha, pad, b, p, info, st);
    }
    W = Wd;
    const int H = L.rows / W;
    const int P = (W + 7) & ~7;
    SolverSetup S;
    memset(&S, 0, sizeof(S));
    S.W = W;
    S.H = H;
    float* tmp = nullptr;
    const float* planes = L.a;
    uint64_t rs = (uint64_t)W * 4, ps = (uint64_t)L.apitch * 4;
    if (W % 4 != 0 || L.apitch % 4 != 0 || ((uintptr_t)L.a & 15)) {
        // Repack into a pitched copy that tensor maps can address.
        GM_CUDA_TRY(cudaMallocAsync((void**)&tmp, (size_t)25 * H * P * 4, st));
        for (int k = 0; k < 25; ++k)
            GM_CUDA_TRY(cudaMemcpy2DAsync(tmp + (size_t)k * H * P, (size_t)P * 4, L.a + (size_t)k * L.apitch,
                                          (size_t)W * 4, (size_t)W * 4, H, cudaMemcpyDeviceToDevice, st));
        planes = tmp;
        rs = (uint64_t)P * 4;
        ps = (uint64_t)H * P * 4;
    }
    OpSource op;
    op.kind = OP_REF25;
    op.dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    op.esize = 4;
    op.base = planes;
    op.row_stride = rs;
    op.plane_stride = ps;
    op.planes = 25;
    S.lo = op;
    S.hi = op;
    S.mixed = false;
    S.b = b;
    S.bpitch = W;
    S.alpha_in = alpha;
    S.alpha_out = alpha;
    S.alpha_pitch = W;
    int rc = run_solver(S, &p, info, st);
    if (tmp) cudaFreeAsync(tmp, st);
    return rc;
}

// Solves the store's system for right-hand side b ([H][bpitch] floats).
static int levin_solve_impl(const gm_levin_store* store, const float* b, int bpitch, float* alpha,
                            const gm_solve_params* prm, gm_solve_info* info, void* stream)
{
    gm_solve_params p;
    if (prm) p = *prm; else gm_default_params(&p);
    if (!store || !store->w32 || !alpha || !b) { gm_set_error_msg("gm_levin_solve: bad arguments"); return GM_ERR_INVALID; }
    if (p.solver == GM_SOLVER_MG) return run_mg_solver(store, b, bpitch, alpha, alpha, &p, info, (cudaStream_t)stream);
    const int W = store->W, H = store->H, P = store->pitch;
    SolverSetup S;
    memset(&S, 0, sizeof(S));
    S.W = W;
    S.H = H;
    OpSource hi;
    hi.kind = OP_SYMI;
    hi.dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    hi.esize = 4;
    hi.base = store->w32;
    hi.row_stride = (uint64_t)P * 4;
    const uint64_t pstride = store->plane_stride ? (uint64_t)store->plane_stride : (uint64_t)H * P;
    hi.plane_stride = pstride * 4;
    hi.planes = 12;
    OpSource lo = hi;
    lo.kind = OP_SYMD;
    const bool low = p.use_low && store->precision != GM_PREC_FP32;
    if (low) {
        lo.dt = store->precision == GM_PREC_FP16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
        lo.esize = 2;
        lo.base = store->w;
        lo.row_stride = (uint64_t)P * 2;
        lo.plane_stride = pstride * 2;
    }
    S.lo = lo;
    S.hi = hi;
    S.mixed = true;
    S.xlo = low ? store->d : store->d32;
    S.xlo_pitch = P;
    S.xhi = store->gamma;
    S.xhi_pitch = P;
    S.b = b;
    S.bpitch = bpitch;
    S.alpha_in = alpha;
    S.alpha_out = alpha;
    S.alpha_pitch = W;
    return run_solver(S, &p, info, (cudaStream_t)stream);
}

extern "C" int gm_levin_solve(const gm_levin_store* store, float* alpha, const gm_solve_params* prm,
                              gm_solve_info* info, void* stream)
{
    if (!store) { gm_set_error_msg("gm_levin_solve: bad arguments"); return GM_ERR_INVALID; }
    return levin_solve_impl(store, store->b, store->pitch, alpha, prm, info, stream);
}

extern "C" int gm_levin_solve_rhs(const gm_levin_store* store, const float* rhs, float* x,
                                  const gm_solve_params* prm, gm_solve_info* info, void* stream)
{
    if (!store) { gm_set_error_msg("gm_levin_solve_rhs: bad arguments"); return GM_ERR_INVALID; }
    return levin_solve_impl(store, rhs, store->W, x, prm, info, stream);
}

int gm_levin_adjoint_grads(const gm_image* im, const gm_scribbles* sc, double eps, int W, int H,
                           const float* lam, const float* alpha, float* dimage, size_t dimage_pitch,
                           int dimage_channels, float* dgamma, cudaStream_t stream);

extern "C" int gm_levin_adjoint(const gm_levin_store* store, const gm_image* im, const gm_scribbles* sc,
                                double eps, const float* alpha, const float* dalpha, float* lambda,
                                float* dimage, size_t dimage_pitch, int dimage_channels, float* dgamma,
                                const gm_solve_params* prm, gm_solve_info* info, void* stream)
{
    if (!store || !store->w32 || !alpha || !dalpha || !lambda || !dimage) {
        gm_set_error_msg("gm_levin_adjoint: bad arguments");
        return GM_ERR_INVALID;
    }
    const int W = store->W, H = store->H;
    cudaStream_t st = (cudaStream_t)stream;
    gm_solve_params p;
    if (prm) p = *prm; else gm_default_params(&p);
    gm_solve_info first;
    gm_solve_info* inf = info ? info : &first;
    GM_CUDA_TRY(cudaMemsetAsync(lambda, 0, sizeof(float) * (size_t)W * H, st));
    int rc = levin_solve_impl(store, dalpha, W, lambda, &p, inf, stream);
    if (rc == GM_ERR_NOT_CONVERGED && p.solver != GM_SOLVER_MG) {
        // The right-hand side dloss/dalpha excites the smooth, weakly
        // constrained modes that a scribble-driven forward solve barely
        // touches; at small eps or large sizes CG and Jacobi PCG stall on
        // them.  Solve again with the multigrid-preconditioned CG from zero;
        // info->solver says so, kernel_ms counts both solves.
        const float ms0 = inf->kernel_ms;
        gm_solve_params q = p;
        q.solver = GM_SOLVER_MG;
        GM_CUDA_TRY(cudaMemsetAsync(lambda, 0, sizeof(float) * (size_t)W * H, st));
        rc = levin_solve_impl(store, dalpha, W, lambda, &q, inf, stream);
        inf->kernel_ms += ms0;
    }
    if (rc != GM_OK && rc != GM_ERR_NOT_CONVERGED) return rc;
    GM_TRY(gm_levin_adjoint_grads(im, sc, eps, W, H, lambda, alpha, dimage, dimage_pitch, dimage_channels, dgamma,
                                  st));
    return rc;
}

// ---------------------------------------------------------------------------
// Drop-ins
// ---------------------------------------------------------------------------

// main.cu:458-526
extern "C" void cgSolve(float* alpha, BandedMatrix L, float* b, int pad, int iterations, int restartInterval)
{
    gm_solve_params p;
    gm_default_params(&p);
    p.solver = GM_SOLVER_CG;
    p.rtol = 0.0;
    p.max_iters = iterations > 0 ? iterations : 0;
    p.restart = restartInterval > 0 ? restartInterval : 0;
    p.replace_every = 0;
    gm_solve_info info;
    gm_note_status(gm_banded_solve(L, 0, alpha, pad, b, &p, &info, nullptr));
}

// main.cu:406-456: the reference recomputes d = L alpha - b every iteration,
// so the drop-in replaces the residual every iteration too.
extern "C" void gradSolve(float* alpha, BandedMatrix L, float* b, int iterations, int pad)
{
    gm_solve_params p;
    gm_default_params(&p);
    p.solver = GM_SOLVER_GD;
    p.rtol = 0.0;
    p.max_iters = iterations > 0 ? iterations : 0;
    p.replace_every = 1;
    gm_solve_info info;
    gm_note_status(gm_banded_solve(L, 0, alpha, pad, b, &p, &info, nullptr));
}

// main.cu:528-556.  The reference swaps x and its scratch buffer each sweep,
// so after an odd count its last iterate sits in the freed scratch; here the
// last iterate is always returned in x.
extern "C" void jacobi(float* x, const BandedMatrix a, const float* b, float omega, int pad, int iterations)
{
    gm_solve_params p;
    gm_default_params(&p);
    p.solver = GM_SOLVER_JACOBI;
    p.rtol = 0.0;
    p.max_iters = iterations > 0 ? iterations : 0;
    p.omega = omega;
    gm_solve_info info;
    gm_note_status(gm_banded_solve(a, 0, x, pad, b, &p, &info, nullptr));
}

// Matting.cu:39-219 on the GPU with the reference's arithmetic.  The
// reference accumulates into a zeroed L.a; this writes the final values.
extern "C" void hostLevinLaplacian(BandedMatrix L, float* b, float lambda, gm_float4* im, unsigned char* scribs,
                                   int imW, int imH, size_t imPitch)
{
    if (!L.a || !b || !im || !scribs || imW <= 0 || imH <= 0 || imPitch < (size_t)imW || L.nbands != 25 ||
        L.rows != imW * imH || L.apitch < (size_t)L.rows) {
        gm_set_error_msg("hostLevinLaplacian: bad arguments (need 25 bands, rows = W*H)");
        gm_note_status(GM_ERR_INVALID);
        return;
    }
    const size_t N = (size_t)imW * imH;
    float4* dim = nullptr;
    unsigned char* dsc = nullptr;
    float* da = nullptr;
    float* db = nullptr;
    int rc = GM_OK;
    if (cudaMalloc((void**)&dim, imPitch * imH * sizeof(float4)) != cudaSuccess ||
        cudaMalloc((void**)&dsc, imPitch * imH) != cudaSuccess ||
        cudaMalloc((void**)&da, 25 * N * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&db, N * sizeof(float)) != cudaSuccess)
        rc = GM_ERR_NOMEM;
    if (rc == GM_OK && (cudaMemcpy(dim, im, imPitch * imH * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess ||
                        cudaMemcpy(dsc, scribs, imPitch * imH, cudaMemcpyHostToDevice) != cudaSuccess))
        rc = GM_ERR_CUDA;
    if (rc == GM_OK) {
        gm_image gi;
        gi.data = dim;
        gi.format = GM_IMAGE_RGBA32F;
        gi.pitch_bytes = imPitch * sizeof(float4);
        gm_scribbles sc;
        memset(&sc, 0, sizeof(sc));
        sc.map = dsc;
        sc.map_pitch = imPitch;
        sc.gamma_value = 1.0f;  // Matting.cu:48
        rc = gm_levin_assemble_bands25(da, N, db, &gi, &sc, lambda, imW, imH, GM_ASSEMBLY_REFERENCE, nullptr);
    }
    if (rc == GM_OK &&
        (cudaMemcpy2D(L.a, L.apitch * sizeof(float), da, N * sizeof(float), N * sizeof(float), 25,
                      cudaMemcpyDeviceToHost) != cudaSuccess ||
         cudaMemcpy(b, db, N * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = GM_ERR_CUDA;
    cudaFree(dim);
    cudaFree(dsc);
    cudaFree(da);
    cudaFree(db);
    gm_note_status(rc);
}
