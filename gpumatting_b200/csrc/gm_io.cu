// gm_io.cu -- the data formats on either side of the solve.
//
// In:  PNM images (ppm.h:32-127 pgmread, :178-278 ppmread): the header is
//      parsed on the host, the pixel bytes go to the device as they are, and
//      the normalisation to [0,1] float4 with alpha = 1 (ppm.h:309-333
//      ppmread_float4) runs as a kernel.  The assembly also takes the bytes
//      directly (GM_IMAGE_RGB8), which is the same arithmetic for maxval 255.
// Out: the 8-bit matte (ppm.h:430-451 pgmwrite_float: clamp, then truncate
//      255 * alpha) as a kernel, and the PGM file (ppm.h:345-414 pgmwrite)
//      byte for byte; the A.bin band dump of main.cu:334-355 (nbands x rows
//      floats, band-major).
//
// Header rules follow the reference so that every file it reads is read the
// same way: the magic on the first line, comment lines ('#') before the
// size line, "w h" on one line, maxval on the next, pixel data right after
// that line.  ASCII samples are cast to bytes as the reference casts them.
// Files the reference would reject (or abort on) return GM_ERR_INVALID.
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "gm_internal.cuh"

namespace {

// One header line as fgets(256) would return it (without the newline), and
// the offset just past it.
bool next_line(const std::vector<unsigned char>& f, size_t& pos, std::string& line)
{
    if (pos >= f.size()) return false;
    line.clear();
    while (pos < f.size() && f[pos] != '\n' && line.size() < 255) line.push_back((char)f[pos++]);
    if (pos < f.size() && f[pos] == '\n') ++pos;
    return true;
}

bool read_file(const char* path, std::vector<unsigned char>& f)
{
    FILE* fp = fopen(path, "rb");
    if (!fp) return false;
    unsigned char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), fp)) > 0) f.insert(f.end(), buf, buf + n);
    fclose(fp);
    return true;
}

}  // namespace

extern "C" int gm_pnm_read(const char* path, gm_pnm* img)
{
    if (!path || !img) { gm_set_error_msg("gm_pnm_read: bad arguments"); return GM_ERR_INVALID; }
    memset(img, 0, sizeof(*img));
    std::vector<unsigned char> f;
    if (!read_file(path, f)) { gm_set_error_msg("cannot open %s", path); return GM_ERR_INVALID; }
    size_t pos = 0;
    std::string line;
    if (!next_line(f, pos, line) || line.size() < 2 || line[0] != 'P') {
        gm_set_error_msg("%s: not a PNM file", path);
        return GM_ERR_INVALID;
    }
    int channels = 0, binary = 0;
    switch (line[1]) {
    case '5': channels = 1; binary = 1; break;
    case '2': channels = 1; binary = 0; break;
    case '6': channels = 3; binary = 1; break;
    case '3': channels = 3; binary = 0; break;
    default: gm_set_error_msg("%s: unsupported PNM type %c%c", path, line[0], line[1]); return GM_ERR_INVALID;
    }
    do {
        if (!next_line(f, pos, line)) { gm_set_error_msg("%s: truncated header", path); return GM_ERR_INVALID; }
    } while (!line.empty() && line[0] == '#');
    int w = 0, h = 0, maxval = 0;
    if (sscanf(line.c_str(), "%d %d", &w, &h) != 2 || w <= 0 || h <= 0) {
        gm_set_error_msg("%s: bad size line", path);
        return GM_ERR_INVALID;
    }
    if (!next_line(f, pos, line) || sscanf(line.c_str(), "%d", &maxval) != 1) {
        gm_set_error_msg("%s: bad maxval line", path);
        return GM_ERR_INVALID;
    }
    if (channels == 3 && (maxval < 0 || maxval > 255)) {  // ppm.h:234-238
        gm_set_error_msg("%s: maximum value %d is bad", path, maxval);
        return GM_ERR_INVALID;
    }
    const size_t n = (size_t)w * h * channels;
    unsigned char* data = (unsigned char*)malloc(n ? n : 1);
    if (!data) { gm_set_error_msg("out of host memory"); return GM_ERR_NOMEM; }
    if (binary) {
        if (f.size() - pos < n) {
            free(data);
            gm_set_error_msg("%s: read %zu of %zu samples", path, f.size() - pos, n);
            return GM_ERR_INVALID;
        }
        memcpy(data, f.data() + pos, n);
    } else {
        f.push_back(0);  // strtol stops at the terminator
        const char* p = (const char*)f.data() + pos;
        for (size_t k = 0; k < n; ++k) {
            char* end = nullptr;
            const long v = strtol(p, &end, 10);
            if (end == p) {
                free(data);
                gm_set_error_msg("%s: ASCII sample %zu missing", path, k);
                return GM_ERR_INVALID;
            }
            data[k] = (unsigned char)v;  // the reference's (unsigned char) cast
            p = end;
        }
    }
    img->w = w;
    img->h = h;
    img->channels = channels;
    img->maxval = maxval;
    img->data = data;
    return GM_OK;
}

extern "C" void gm_pnm_free(gm_pnm* img)
{
    if (!img) return;
    free(img->data);
    memset(img, 0, sizeof(*img));
}

extern "C" int gm_pgm_write(const char* path, int w, int h, const unsigned char* data, const char* comment,
                            int binary)
{
    if (!path || !data || w <= 0 || h <= 0) { gm_set_error_msg("gm_pgm_write: bad arguments"); return GM_ERR_INVALID; }
    FILE* fp = fopen(path, "wb");
    if (!fp) { gm_set_error_msg("cannot create %s", path); return GM_ERR_INVALID; }
    fprintf(fp, binary ? "P5\n" : "P2\n");
    if (comment) fprintf(fp, "# %s \n", comment);
    fprintf(fp, "%d %d \n", w, h);
    fprintf(fp, "%d \n", 255);
    const size_t n = (size_t)w * h;
    bool ok = true;
    if (binary) {
        ok = fwrite(data, 1, n, fp) == n;
    } else {
        for (size_t k = 0; k < n && ok; ++k) ok = fprintf(fp, "%d ", (int)data[k]) > 0;
    }
    ok = (fclose(fp) == 0) && ok;
    if (!ok) { gm_set_error_msg("write to %s failed", path); return GM_ERR_INVALID; }
    return GM_OK;
}

namespace gm {

__global__ void rgb8_to_float4_kernel(float4* __restrict__ dst, const unsigned char* __restrict__ src, int n,
                                      float maxval)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned char* p = src + 3 * (size_t)i;
        dst[i] = make_float4(__fdiv_rn((float)p[0], maxval), __fdiv_rn((float)p[1], maxval),
                             __fdiv_rn((float)p[2], maxval), 1.0f);
    }
}

__global__ void alpha_to_gray8_kernel(unsigned char* __restrict__ dst, const float* __restrict__ a, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = a[i];
        dst[i] = v < 0.f ? 0 : (v > 1.f ? 255 : (unsigned char)__fmul_rn(255.f, v));
    }
}

static int grid_for(int n)
{
    int nb = (n + 255) / 256;
    return nb > 148 * 16 ? 148 * 16 : (nb < 1 ? 1 : nb);
}

}  // namespace gm

using namespace gm;

extern "C" int gm_rgb8_to_float4(gm_float4* dst, const unsigned char* src, int n, int maxval, void* stream)
{
    if (n < 0 || (n > 0 && (!dst || !src)) || maxval <= 0 || ((uintptr_t)dst & 15)) {
        gm_set_error_msg("gm_rgb8_to_float4: bad arguments");
        return GM_ERR_INVALID;
    }
    if (n == 0) return GM_OK;
    rgb8_to_float4_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<float4*>(dst), src, n,
                                                                          (float)maxval);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_alpha_to_gray8(unsigned char* dst, const float* alpha, int n, void* stream)
{
    if (n < 0 || (n > 0 && (!dst || !alpha))) { gm_set_error_msg("gm_alpha_to_gray8: bad arguments"); return GM_ERR_INVALID; }
    if (n == 0) return GM_OK;
    alpha_to_gray8_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dst, alpha, n);
    GM_CUDA_TRY(cudaGetLastError());
    return GM_OK;
}

extern "C" int gm_bands_dump(const char* path, BandedMatrix L, int on_device)
{
    if (!path || !L.a || L.nbands <= 0 || L.rows <= 0 || L.apitch < (size_t)L.rows) {
        gm_set_error_msg("gm_bands_dump: bad arguments");
        return GM_ERR_INVALID;
    }
    FILE* fp = fopen(path, "wb");
    if (!fp) { gm_set_error_msg("cannot create %s", path); return GM_ERR_INVALID; }
    std::vector<float> band(on_device ? (size_t)L.rows : 0);
    int rc = GM_OK;
    for (int i = 0; i < L.nbands && rc == GM_OK; ++i) {
        const float* src = L.a + (size_t)i * L.apitch;
        if (on_device) {
            if (cudaMemcpy(band.data(), src, sizeof(float) * L.rows, cudaMemcpyDeviceToHost) != cudaSuccess) {
                gm_set_error_msg("gm_bands_dump: device copy failed");
                rc = GM_ERR_CUDA;
                break;
            }
            src = band.data();
        }
        if (fwrite(src, sizeof(float), (size_t)L.rows, fp) != (size_t)L.rows) {
            gm_set_error_msg("write to %s failed", path);
            rc = GM_ERR_INVALID;
        }
    }
    if (fclose(fp) != 0 && rc == GM_OK) rc = GM_ERR_INVALID;
    return rc;
}
