// gm_hostsolve.cu -- the reference's CPU relaxations (Solve.cpp) as GPU
// drop-ins whose iterates are bit-identical to the reference's.
//
// Both take HOST vectors and a HOST BandedMatrix, as Solve.h:17,31 do; the
// matrix and vectors are copied to the device, the sweeps run there, and x
// is copied back.  Any band pattern is accepted.  The arithmetic is the
// reference's, operation for operation, in FP32: the middle band (nbands/2)
// is the diagonal and is skipped in the sum, the other bands are added in
// band order, products and sums are rounded separately (__fmul_rn /
// __fadd_rn: no FMA contraction, as in the reference's host build) and the
// division is IEEE-rounded.
//
// jacobi_host (Solve.cpp:35-85): row i of an iteration reads only the
// previous iterate, so one thread per row reproduces the sequential loop
// exactly.  Iterates ping-pong between two device buffers.  Unlike the
// reference, which frees the buffer holding the last iterate when the
// iteration count is odd (Solve.cpp:72-83), the last iterate always ends in
// x.
//
// gaussSeidel_host (Solve.cpp:3-33): the sequential in-place sweep.  When
// row i is updated it sees the values of rows i+o (o < 0) from the current
// sweep and those of rows i+o (o > 0) from the previous one.  A level
// schedule keeps exactly those reads in parallel:
//   level(i) = 1 + max { level(i+o) : o < 0, 0 <= i+o, a(i, o) != 0 }
// (0 when there is none); the rows of one level depend on none of each
// other, and every level only on earlier ones.  Each sweep reads forward
// neighbours from the previous sweep's buffer and backward neighbours from
// the current one, so the values used are the sequential loop's values for
// every non-zero coefficient (a zero coefficient adds +0 to the sum
// whatever it multiplies, for finite x).  For the 25-band Levin stencil,
// whose couplings that would cross the image edge are zero, the levels are
// the anti-diagonals u + 3v: W + 3H - 3 levels.  One CTA runs a sweep with
// a block barrier between levels; a pattern whose dependencies form one
// chain (a tridiagonal matrix, say) has one row per level and runs
// serially.
#include <string.h>

#include <algorithm>
#include <vector>

#include "gm_internal.cuh"

int gm_note_status(int s);

namespace gm {

constexpr int kHostSolveMaxBands = 128;
constexpr int kGsThreads = 1024;

// xx[i] = omega * (b_i - sum_{j != mid} a_ij x_{i+off_j}) / a_i,mid + (1 - omega) x_i
__global__ void jacobi_host_kernel(float* __restrict__ xx, const float* __restrict__ x, const float* __restrict__ a,
                                   size_t apitch, const int* __restrict__ bands, int nbands, int rows,
                                   const float* __restrict__ b, float omega, float omega1)
{
    __shared__ int off[kHostSolveMaxBands];
    for (int j = threadIdx.x; j < nbands; j += blockDim.x) off[j] = bands[j];
    __syncthreads();
    const int mid = nbands / 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride) {
        float t = 0.f;
        for (int j = 0; j < nbands; ++j) {
            if (j == mid) continue;
            t = __fadd_rn(t, __fmul_rn(a[i + (size_t)j * apitch], x[i + off[j]]));
        }
        t = __fsub_rn(b[i], t);
        // omega*tmp/a[mid] + omega1*x[i], evaluated left to right
        xx[i] = __fadd_rn(__fdiv_rn(__fmul_rn(omega, t), a[i + (size_t)mid * apitch]), __fmul_rn(omega1, x[i]));
    }
}

// One Gauss-Seidel sweep over the level schedule: perm holds the rows in
// level order, lstart[l] .. lstart[l+1]-1 are level l's.  xold: previous
// sweep; xnew: this sweep (rows not yet updated hold stale values that are
// only ever multiplied by zero coefficients).
__global__ void __launch_bounds__(kGsThreads) gs_level_kernel(float* xnew, const float* xold,
                                                              const float* __restrict__ a, size_t apitch,
                                                              const int* __restrict__ bands, int nbands,
                                                              const float* __restrict__ b,
                                                              const int* __restrict__ perm,
                                                              const int* __restrict__ lstart, int nlev)
{
    __shared__ int off[kHostSolveMaxBands];
    for (int j = threadIdx.x; j < nbands; j += blockDim.x) off[j] = bands[j];
    __syncthreads();
    const int mid = nbands / 2;
    for (int l = 0; l < nlev; ++l) {
        const int r0 = lstart[l], r1 = lstart[l + 1];
        for (int k = r0 + (int)threadIdx.x; k < r1; k += blockDim.x) {
            const long long i = perm[k];
            float t = 0.f;
            for (int j = 0; j < nbands; ++j) {
                if (j == mid) continue;
                // plain loads: xnew is written by this block between levels
                const float xv = off[j] < 0 ? xnew[i + off[j]] : xold[i + off[j]];
                t = __fadd_rn(t, __fmul_rn(a[i + (size_t)j * apitch], xv));
            }
            t = __fsub_rn(b[i], t);
            xnew[i] = __fdiv_rn(t, a[i + (size_t)mid * apitch]);
        }
        __syncthreads();  // orders this level's writes before the next level's reads
    }
}

// Level schedule of a host matrix (see the file comment).  Returns the
// number of levels; perm and lstart are filled.
static int gs_levels(const BandedMatrix& A, std::vector<int>& perm, std::vector<int>& lstart)
{
    const int n = A.rows;
    std::vector<int> lev((size_t)n, 0);
    std::vector<int> back;
    for (int j = 0; j < A.nbands; ++j)
        if (j != A.nbands / 2 && A.bands[j] < 0) back.push_back(j);
    int nlev = n > 0 ? 1 : 0;
    for (int i = 0; i < n; ++i) {
        int l = 0;
        for (int j : back) {
            const long long k = (long long)i + A.bands[j];
            if (k < 0) continue;
            if (A.a[(size_t)i + (size_t)j * A.apitch] != 0.f) l = std::max(l, lev[(size_t)k] + 1);
        }
        lev[(size_t)i] = l;
        nlev = std::max(nlev, l + 1);
    }
    lstart.assign((size_t)nlev + 1, 0);
    for (int i = 0; i < n; ++i) ++lstart[(size_t)lev[(size_t)i] + 1];
    for (int l = 0; l < nlev; ++l) lstart[(size_t)l + 1] += lstart[(size_t)l];
    perm.resize((size_t)n);
    std::vector<int> fill(lstart.begin(), lstart.end() - 1);
    for (int i = 0; i < n; ++i) perm[(size_t)fill[(size_t)lev[(size_t)i]]++] = i;
    return nlev;
}

// Reach of the pattern: the reference reads x[i + off] for every band, so
// x must be addressable from x - left to x + rows + right.
static void band_reach(const BandedMatrix& A, int* left, int* right)
{
    int l = 0, r = 0;
    for (int j = 0; j < A.nbands; ++j) {
        l = std::max(l, -A.bands[j]);
        r = std::max(r, A.bands[j]);
    }
    *left = l;
    *right = r;
}

static int check_host_matrix(const BandedMatrix* A, const char* who)
{
    if (!A || !A->a || !A->bands || A->nbands <= 0 || A->nbands > kHostSolveMaxBands || A->rows < 0 ||
        A->apitch < (size_t)A->rows) {
        gm_set_error_msg("%s: bad BandedMatrix (need host a and bands, 0 < nbands <= %d, apitch >= rows)", who,
                         kHostSolveMaxBands);
        return GM_ERR_INVALID;
    }
    return GM_OK;
}

// Device copies of what a host relaxation needs: the bands (nbands x rows,
// pitch rows), their offsets, b, and two padded x buffers, each holding the
// caller's x with `left` / `right` elements of the caller's padding.
struct HostSolveBufs {
    float* a = nullptr;
    int* bands = nullptr;
    float* b = nullptr;
    float* xbuf[2] = {nullptr, nullptr};
    ~HostSolveBufs()
    {
        cudaFree(a);
        cudaFree(bands);
        cudaFree(b);
        cudaFree(xbuf[0]);
        cudaFree(xbuf[1]);
    }
};

static int upload(const BandedMatrix& A, const float* x, const float* b, int left, int right, HostSolveBufs& B)
{
    const size_t n = (size_t)A.rows;
    const size_t nx = n + (size_t)left + (size_t)right;
    if (cudaMalloc((void**)&B.a, sizeof(float) * std::max<size_t>(1, n * A.nbands)) != cudaSuccess ||
        cudaMalloc((void**)&B.bands, sizeof(int) * A.nbands) != cudaSuccess ||
        cudaMalloc((void**)&B.b, sizeof(float) * std::max<size_t>(1, n)) != cudaSuccess ||
        cudaMalloc((void**)&B.xbuf[0], sizeof(float) * std::max<size_t>(1, nx)) != cudaSuccess ||
        cudaMalloc((void**)&B.xbuf[1], sizeof(float) * std::max<size_t>(1, nx)) != cudaSuccess) {
        gm_set_error_msg("host relaxation: device allocation failed");
        return GM_ERR_NOMEM;
    }
    if (n > 0) {
        GM_CUDA_TRY(cudaMemcpy2D(B.a, n * sizeof(float), A.a, A.apitch * sizeof(float), n * sizeof(float), A.nbands,
                                 cudaMemcpyHostToDevice));
        GM_CUDA_TRY(cudaMemcpy(B.b, b, n * sizeof(float), cudaMemcpyHostToDevice));
    }
    GM_CUDA_TRY(cudaMemcpy(B.bands, A.bands, sizeof(int) * A.nbands, cudaMemcpyHostToDevice));
    for (int k = 0; k < 2; ++k)
        GM_CUDA_TRY(cudaMemcpy(B.xbuf[k], x - left, nx * sizeof(float), cudaMemcpyHostToDevice));
    return GM_OK;
}

static int run_jacobi_host(float* x, const BandedMatrix* A, const float* b, size_t iterations, int xpad, float omega)
{
    GM_TRY(check_host_matrix(A, "jacobi_host"));
    if (!x || !b || xpad < 0) {
        gm_set_error_msg("jacobi_host: bad arguments");
        return GM_ERR_INVALID;
    }
    if (A->rows == 0 || iterations == 0) return GM_OK;
    int left = 0, right = 0;
    band_reach(*A, &left, &right);
    if (left > xpad || right > xpad) {
        // the reference would read outside the caller's buffer (Solve.cpp:45-47)
        gm_set_error_msg("jacobi_host: xpad %d is smaller than the band reach (%d left, %d right)", xpad, left, right);
        return GM_ERR_INVALID;
    }
    HostSolveBufs B;
    GM_TRY(upload(*A, x, b, left, right, B));
    const int n = A->rows;
    const float omega1 = 1.f - omega;  // Solve.cpp:38
    const int nb = std::max(1, std::min((n + 255) / 256, 148 * 8));
    int cur = 0;
    for (size_t it = 0; it < iterations; ++it) {
        jacobi_host_kernel<<<nb, 256>>>(B.xbuf[cur ^ 1] + left, B.xbuf[cur] + left, B.a, (size_t)n, B.bands,
                                        A->nbands, n, B.b, omega, omega1);
        GM_CUDA_TRY(cudaGetLastError());
        cur ^= 1;
    }
    GM_CUDA_TRY(cudaMemcpy(x, B.xbuf[cur] + left, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return GM_OK;
}

static int run_gauss_seidel_host(float* x, const BandedMatrix* A, const float* b, size_t iterations)
{
    GM_TRY(check_host_matrix(A, "gaussSeidel_host"));
    if (!x || !b) {
        gm_set_error_msg("gaussSeidel_host: bad arguments");
        return GM_ERR_INVALID;
    }
    if (A->rows == 0 || iterations == 0) return GM_OK;
    std::vector<int> perm, lstart;
    const int nlev = gs_levels(*A, perm, lstart);
    int left = 0, right = 0;
    band_reach(*A, &left, &right);
    HostSolveBufs B;
    GM_TRY(upload(*A, x, b, left, right, B));
    int* dperm = nullptr;
    int* dlst = nullptr;
    if (cudaMalloc((void**)&dperm, sizeof(int) * perm.size()) != cudaSuccess ||
        cudaMalloc((void**)&dlst, sizeof(int) * lstart.size()) != cudaSuccess) {
        cudaFree(dperm);
        gm_set_error_msg("gaussSeidel_host: device allocation failed");
        return GM_ERR_NOMEM;
    }
    int rc = GM_OK;
    if (cudaMemcpy(dperm, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dlst, lstart.data(), sizeof(int) * lstart.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = GM_ERR_CUDA;
    const int n = A->rows;
    int cur = 0;
    for (size_t it = 0; it < iterations && rc == GM_OK; ++it) {
        gs_level_kernel<<<1, kGsThreads>>>(B.xbuf[cur ^ 1] + left, B.xbuf[cur] + left, B.a, (size_t)n, B.bands,
                                           A->nbands, B.b, dperm, dlst, nlev);
        if (cudaGetLastError() != cudaSuccess) rc = GM_ERR_CUDA;
        cur ^= 1;
    }
    if (rc == GM_OK && cudaMemcpy(x, B.xbuf[cur] + left, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = GM_ERR_CUDA;
    if (rc == GM_ERR_CUDA) gm_set_error_msg("gaussSeidel_host: %s", cudaGetErrorString(cudaGetLastError()));
    cudaFree(dperm);
    cudaFree(dlst);
    return rc;
}

}  // namespace gm

// Solve.cpp:35-85.
extern "C" void jacobi_host(float* x, const BandedMatrix* A, const float* b, size_t iterations, int xpad,
                            float omega)
{
    gm_note_status(gm::run_jacobi_host(x, A, b, iterations, xpad, omega));
}

// Solve.cpp:3-33.
extern "C" void gaussSeidel_host(float* x, const BandedMatrix* A, const float* b, size_t iterations)
{
    gm_note_status(gm::run_gauss_seidel_host(x, A, b, iterations));
}

// Number of levels of the Gauss-Seidel schedule of a host matrix (its
// parallel depth per sweep); -1 on bad arguments.
extern "C" int gm_gs_host_levels(const BandedMatrix* A)
{
    if (gm::check_host_matrix(A, "gm_gs_host_levels") != GM_OK) return -1;
    std::vector<int> perm, lstart;
    return gm::gs_levels(*A, perm, lstart);
}
