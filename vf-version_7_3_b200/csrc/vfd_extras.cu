// vfd_extras.cu -- the steps either side of the diffusion path.
//
//  gradients_kernel  the attractant gradients WHChemical::update forms after
//                    the chemical update (WHChemical.cpp:433-441):
//                      grad = IL1 + TNF + TGF + FGF + collagen fragments
//                      fib  = TGF;  neu = grad + IL6 + IL8;  mac = grad + elastin fragments
//  sample_kernel     the compute part of sampleChem (volumeRender_kernel.cu:215-321):
//                    every stride-th voxel on each axis, times a per-chemical
//                    scale, clamped above at 1, into a plain device buffer of
//                    (nx/stride) x (ny/stride) x (nz/stride) (the reference
//                    writes a CUDA surface for its OpenGL renderer instead).
//  vfd_write_vtk     legacy-VTK ASCII STRUCTURED_POINTS writer of one field
//                    (the file layout util::outputChem produces,
//                    output_utils.h:813-854: scalars "Color", x fastest,
//                    one line per row).
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <stdio.h>

#include "vfd.h"
#include "vfd_internal.h"

namespace vfd {

__global__ void gradients_kernel(const float *tnf, const float *tgf, const float *fgf, const float *il1,
                                 const float *il6, const float *il8, const float *col, const float *ela,
                                 float *fib, float *neu, float *mac, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float t = tgf[i];
        const float grad = il1[i] + tnf[i] + t + fgf[i] + (col ? col[i] : 0.0f);
        if (fib) fib[i] = t;
        if (neu) neu[i] = grad + il6[i] + il8[i];
        if (mac) mac[i] = grad + (ela ? ela[i] : 0.0f);
    }
}

__global__ void sample_kernel(const float *src, int nx, int ny, int nz, int stride, float scale, float *out)
{
    const int sx = nx / stride, sy = ny / stride, sz = nz / stride;
    const int64_t n = (int64_t)sx * sy * sz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int dx = (int)(i % sx);
        const int64_t r = i / sx;
        const int dy = (int)(r % sy), dz = (int)(r / sy);
        float v = src[(int64_t)dx * stride + (int64_t)nx * ((int64_t)dy * stride + (int64_t)ny * dz * stride)] * scale;
        if (v > 1.0f) v = 1.0f;
        out[i] = v;
    }
}

static int grid_of(int64_t n)
{
    int64_t b = (n + 255) / 256;
    return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

cudaError_t launch_gradients(const float *const *chem, const float *col, const float *ela, float *fib, float *neu,
                             float *mac, int64_t n, cudaStream_t st)
{
    gradients_kernel<<<grid_of(n), 256, 0, st>>>(chem[0], chem[1], chem[2], chem[4], chem[5], chem[6], col, ela,
                                                  fib, neu, mac, n);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_sample(const float *src, int nx, int ny, int nz, int stride, float scale, float *out,
                          cudaStream_t st)
{
    const int64_t n = (int64_t)(nx / stride) * (ny / stride) * (nz / stride);
    if (n == 0) return cudaSuccess;
    sample_kernel<<<grid_of(n), 256, 0, st>>>(src, nx, ny, nz, stride, scale, out);
    note_launch();
    return cudaGetLastError();
}

}  // namespace vfd

extern "C" vfd_status vfd_write_vtk(const float *field, int nx, int ny, int nz, const char *path)
{
    if (!field || !path || nx < 1 || ny < 1 || nz < 1) return VFD_ERR_INVALID_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return VFD_ERR_INVALID_ARG;
    const long long n = (long long)nx * ny * nz;
    fprintf(f, "# vtk DataFile Version 2.0\ncytokine field\nASCII\nDATASET STRUCTURED_POINTS\n");
    fprintf(f, "DIMENSIONS %d %d %d\nORIGIN 0 0 0\nSPACING 1 1 1\nPOINT_DATA %lld\n", nx, ny, nz, n);
    fprintf(f, "SCALARS Color float 1\nLOOKUP_TABLE default\n");
    for (long long row = 0; row < (long long)ny * nz; ++row) {
        const float *p = field + row * nx;
        for (int x = 0; x < nx; ++x) fprintf(f, "%.9g ", (double)p[x]);
        fputc('\n', f);
    }
    const int bad = ferror(f);
    fclose(f);
    return bad ? VFD_ERR_INVALID_ARG : VFD_OK;
}

// The reference's raw field writers (output_utils.h:21-128), restated.
// Normalised 8-bit volume: every voxel v -> 255 if v >= 1, 0 if v <= 0, else
// floor(v * 256) (writeNormalizedFloatRaw; append = 1 adds a frame to an
// existing file, writeNormalizedFloatRawFrames).
extern "C" vfd_status vfd_write_raw_normalized(const float *field, int nx, int ny, int nz, const char *path,
                                               int append)
{
    if (!field || !path || nx < 1 || ny < 1 || nz < 1) return VFD_ERR_INVALID_ARG;
    FILE *f = fopen(path, append ? "ab" : "wb");
    if (!f) return VFD_ERR_INVALID_ARG;
    unsigned char buf[4096];
    const size_t n = (size_t)nx * ny * nz;
    size_t done = 0;
    bool ok = true;
    while (done < n && ok) {
        const size_t m = n - done < sizeof(buf) ? n - done : sizeof(buf);
        for (size_t i = 0; i < m; ++i) {
            const float v = field[done + i];
            buf[i] = v >= 1.0f ? 255 : (v <= 0.0f ? 0 : (unsigned char)floorf(v * 256.0f));
        }
        ok = fwrite(buf, 1, m, f) == m;
        done += m;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? VFD_OK : VFD_ERR_INVALID_ARG;
}

// Comma-separated values of a field (writeFloatCsv): one line per row (x
// fastest, each value followed by ", "), an empty line after each z plane,
// values with 6 significant digits (the iostream default).
extern "C" vfd_status vfd_write_csv(const float *field, int nx, int ny, int nz, const char *path)
{
    if (!field || !path || nx < 1 || ny < 1 || nz < 1) return VFD_ERR_INVALID_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return VFD_ERR_INVALID_ARG;
    bool ok = true;
    for (int z = 0; z < nz && ok; ++z) {
        for (int y = 0; y < ny && ok; ++y) {
            const float *r = field + (size_t)nx * (y + (size_t)ny * z);
            for (int x = 0; x < nx; ++x) ok = ok && fprintf(f, "%g, ", (double)r[x]) > 0;
            ok = ok && fputc('\n', f) != EOF;
        }
        ok = ok && fputc('\n', f) != EOF;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? VFD_OK : VFD_ERR_INVALID_ARG;
}
