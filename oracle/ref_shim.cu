/* ref_shim.cu -- C entry points onto the reference's own CPU code.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile from the reference
 * sources where they lie (the reference tree is put on the include path);
 * nothing of the reference is copied here.  Output goes to oracle/_ref/,
 * which stays out of version control.  Used to pin the oracle's
 * restatement and to generate the golden fixtures in tests/golden/.
 *
 * Wrapped functions:
 *   pgmread, ppmread    ppm.h:32-127, :178-278 (valid files only: the
 *                       reference exits on some malformed ones)
 *   ppmread_float4      ppm.h:309-333
 *   pgmwrite_float      ppm.h:430-451
 *   hostLevinLaplacian  Matting.cu:39-219
 *   gaussSeidel_host    Solve.cpp:3-33
 *   jacobi_host         Solve.cpp:35-85
 * The reference's GPU kernels are compiled along with Matting.cu but never
 * launched: with its 25-band store they index shared memory out of bounds
 * (BandedMatrix.cu:111,119).
 */
#include "Matting.cu"
#include "Solve.h"
#include "ppm.h"

extern "C" {

void ref_hostLevinLaplacian(float* a, size_t apitch, int* bands, float* b, float lambda,
                            const float* im4, const unsigned char* scribs,
                            int W, int H, size_t imPitch)
{
    BandedMatrix L;
    L.a = a;
    L.apitch = apitch;
    L.bands = bands;
    L.nbands = 25;
    L.rows = W * H;
    L.cols = W * H;
    hostLevinLaplacian(L, b, lambda, (float4*)im4, (unsigned char*)scribs, W, H, imPitch);
}

void ref_gaussSeidel_host(float* x, float* a, size_t apitch, int* bands, int nbands,
                          int rows, const float* b, size_t iterations)
{
    BandedMatrix A;
    A.a = a;
    A.apitch = apitch;
    A.bands = bands;
    A.nbands = nbands;
    A.rows = rows;
    A.cols = rows;
    gaussSeidel_host(x, A, b, iterations);
}

/* jacobi_host frees its caller's buffer after an odd number of iterations
 * (Solve.cpp:72-83), so only even counts are accepted here.  Returns 0 on
 * success, -1 when refused. */
int ref_jacobi_host(float* x, float* a, size_t apitch, int* bands, int nbands,
                    int rows, const float* b, size_t iterations, int xpad, float omega)
{
    if (iterations % 2 != 0) return -1;
    BandedMatrix A;
    A.a = a;
    A.apitch = apitch;
    A.bands = bands;
    A.nbands = nbands;
    A.rows = rows;
    A.cols = rows;
    jacobi_host(x, A, b, iterations, xpad, omega);
    return 0;
}


unsigned char* ref_pgmread(char* filename, int* w, int* h) { return pgmread(filename, w, h); }
unsigned char* ref_ppmread(char* filename, int* w, int* h, int* maxval) { return ppmread(filename, w, h, maxval); }
float* ref_ppmread_float4(char* filename, int* w, int* h)
{
    return reinterpret_cast<float*>(ppmread_float4(0, filename, w, h));
}
int ref_pgmwrite_float(char* filename, int w, int h, float* data, const char* comment, int binsave)
{
    return pgmwrite_float(filename, w, h, data, comment, binsave);
}
void ref_free(void* p) { free(p); }

}
