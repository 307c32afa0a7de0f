/*
 * vfd_cpu_port.c -- FP32 OpenMP CPU port of the diffusion tick (timed CPU
 * baseline; also the `--impl reference` arm of bench.py).
 *
 * TEST/BENCH INFRASTRUCTURE ONLY: never linked into the product library.
 *
 * The reference has no runnable CPU diffusion: Diffuser::diffuseChemCPU
 * returns immediately under OPT_CHEM and does not compile without it
 * (src/Diffusion/Diffuser.cpp:477-654).  This port restates the GPU path's
 * method on the CPU in the reference's precision (FP32 values, FP64 totals as
 * in WHChemical::update, WHChemical.cpp:420-450): per substep a separable
 * direct convolution with the truncated Gaussian -- equal to the FFT
 * convolution with padding >= radius followed by the top-left crop
 * (unpadResult3D_kernel, convolutionFFT.cuh:152-171) -- then the decay
 * factor; per tick the source deposit and the FP64 total.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static void taps_f(double sigma, int r, float *t)
{
    double s = 0.0, g[64];
    for (int j = -r; j <= r; ++j) {
        g[j + r] = exp(-(double)j * j / (2.0 * sigma * sigma));
        s += g[j + r];
    }
    for (int j = 0; j <= 2 * r; ++j) t[j] = (float)(g[j] / s);
}

int vfp_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* In-place separable convolution of one fp32 field (zero padding), then
 * u <- keep * (b + conv(M (u - b))).  pad_mode 1 = constant-VF interior box. */
int vfp_substep(int nx, int ny, int nz, float *u, const double sigma[3], const int radius[3],
                double rate, float b, int pad_mode, int epi, int nthreads)
{
    int r[3];
    float t[3][64];
    for (int a = 0; a < 3; ++a) {
        r[a] = radius[a] > 0 ? radius[a] : (int)ceil(3.0 * sigma[a]);
        if (r[a] > 31) return -1;
        taps_f(sigma[a], r[a], t[a]);
    }
    const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
    const float keep = (float)(1.0 - rate);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    /* x pass with the padding rule applied on load */
#pragma omp parallel
    {
        float *line = (float *)malloc(sizeof(float) * (nx + 2 * 64));
#pragma omp for schedule(static)
        for (long long row = 0; row < (long long)ny * nz; ++row) {
            int y = (int)(row % ny), z = (int)(row / ny);
            float *p = u + (size_t)row * nx;
            const int rr = r[0];
            for (int i = 0; i < rr; ++i) { line[i] = 0.f; line[nx + rr + i] = 0.f; }
            int rowin = pad_mode != 1 || (y > 0 && y < ny - 1 && z > 0 && z < nz - 1);
            for (int x = 0; x < nx; ++x) {
                int in = rowin && (pad_mode != 1 || (x > 0 && x < epi));
                line[x + rr] = in ? p[x] - b : 0.f;
            }
            for (int x = 0; x < nx; ++x) {
                float s = 0.f;
                for (int j = -rr; j <= rr; ++j) s += t[0][j + rr] * line[x + rr - j];
                p[x] = s;
            }
        }
        free(line);
    }
    /* y pass: per z plane, blocks of x columns */
#pragma omp parallel
    {
        const int rr = r[1];
        float *col = (float *)malloc(sizeof(float) * (size_t)(ny + 2 * rr) * 64);
#pragma omp for schedule(static) collapse(2)
        for (int z = 0; z < nz; ++z)
            for (int xb = 0; xb < (nx + 63) / 64; ++xb) {
                int x0 = xb * 64, w = nx - x0 < 64 ? nx - x0 : 64;
                float *pl = u + (size_t)z * sz;
                memset(col, 0, sizeof(float) * (size_t)(ny + 2 * rr) * 64);
                for (int y = 0; y < ny; ++y)
                    memcpy(col + (size_t)(y + rr) * 64, pl + (size_t)y * sy + x0, sizeof(float) * w);
                for (int y = 0; y < ny; ++y) {
                    float acc[64];
                    for (int i = 0; i < w; ++i) acc[i] = 0.f;
                    for (int j = -rr; j <= rr; ++j) {
                        const float c = t[1][j + rr];
                        const float *src = col + (size_t)(y + rr - j) * 64;
                        for (int i = 0; i < w; ++i) acc[i] += c * src[i];
                    }
                    memcpy(pl + (size_t)y * sy + x0, acc, sizeof(float) * w);
                }
            }
        free(col);
    }
    /* z pass: per y, blocks of x columns; baseline + decay fused */
#pragma omp parallel
    {
        const int rr = r[2];
        float *col = (float *)malloc(sizeof(float) * (size_t)(nz + 2 * rr) * 64);
#pragma omp for schedule(static) collapse(2)
        for (int y = 0; y < ny; ++y)
            for (int xb = 0; xb < (nx + 63) / 64; ++xb) {
                int x0 = xb * 64, w = nx - x0 < 64 ? nx - x0 : 64;
                memset(col, 0, sizeof(float) * (size_t)(nz + 2 * rr) * 64);
                for (int z = 0; z < nz; ++z)
                    memcpy(col + (size_t)(z + rr) * 64, u + (size_t)z * sz + (size_t)y * sy + x0,
                           sizeof(float) * w);
                for (int z = 0; z < nz; ++z) {
                    float acc[64];
                    for (int i = 0; i < w; ++i) acc[i] = 0.f;
                    for (int j = -rr; j <= rr; ++j) {
                        const float c = t[2][j + rr];
                        const float *src = col + (size_t)(z + rr - j) * 64;
                        for (int i = 0; i < w; ++i) acc[i] += c * src[i];
                    }
                    float *dst = u + (size_t)z * sz + (size_t)y * sy + x0;
                    for (int i = 0; i < w; ++i) dst[i] = keep * (acc[i] + b);
                }
            }
        free(col);
    }
    return 0;
}

/* Source deposit + FP64 total of one field. */
double vfp_deposit_total(float *u, size_t V, const int32_t *idx, const float *amt, int64_t n)
{
    for (int64_t j = 0; j < n; ++j) u[idx[j]] += amt[j];
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long long i = 0; i < (long long)V; ++i) s += (double)u[i];
    return s;
}
