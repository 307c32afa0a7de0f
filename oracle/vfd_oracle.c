/*
 * vfd_oracle.c -- FP64 CPU oracle for the cytokine-diffusion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline leg of bench.py load it.
 * The product library (libvfd.so) never links, calls or falls back to it.
 *
 * Parity status: the reference ships no CPU diffusion path (its
 * Diffuser::diffuseChemCPU returns immediately under OPT_CHEM,
 * src/Diffusion/Diffuser.cpp:477-479), no test suite and no golden vectors.
 * This oracle is therefore a restatement of the reference's GPU algorithm in
 * FP64.  It is pinned (a) against the reference's own 2D CPU gold routine
 * convolutionClampToBorderCPU (src/Diffusion/convolutionFFT_gold.cpp:22-58),
 * compiled from the reference sources into oracle/_ref by oracle/Makefile,
 * for the kernel-centre/orientation convention of the direct sum, and
 * (b) against the reference's own CUDA kernels + cuFFT replayed in
 * fftDiffuse3D's call order on a B200 (oracle/ref_replay.cu), and (c)
 * against the known-answer properties listed in tests/test_oracle.py.
 *
 * Semantics restated here (reference file:line in each function):
 *   substep:  v = M .* (u - b)              (padDataConstantVF3D rule)
 *             t = crop(IDFT(DFT(pad0(v)) .* K) / N) + b
 *             u <- (1 - rate) * t           (first-order decay per substep)
 *   tick end: u[idx_j] += amt_j             (agents' dChem deposit)
 *             total = sum(u) in FP64        (WHChemical::update totals)
 *
 * Layout: x fastest, index = x + nx*(y + ny*z)  (WHChemical.cpp:424).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define VFO_PI 3.14159265358979323846264338327950288

/* ------------------------------------------------------------------ */
/* Gaussian heat-kernel taps.                                          */
/* Taps g[j], j in [-r, r], g ~ exp(-j^2 / (2 sigma^2)), normalised to  */
/* sum 1 in FP64.  The 3D kernel is the separable product gx*gy*gz over */
/* the cube [-r,r]^3, which is itself normalised to 1.                 */
/* Counterpart of the reference's kernel window (the stencil power     */
/* S^n, Diffusion.cu:1078-1531), whose per-axis variance is 2*lambda*n. */
/* ------------------------------------------------------------------ */
int vfo_gauss_taps(double sigma, int r, double *taps)
{
    if (!(sigma > 0.0) || r < 0) return -1;
    double s = 0.0;
    for (int j = -r; j <= r; ++j) {
        double v = exp(-((double)j * (double)j) / (2.0 * sigma * sigma));
        taps[j + r] = v;
        s += v;
    }
    for (int j = 0; j < 2 * r + 1; ++j) taps[j] /= s;
    return 0;
}

/* Real spectrum of the wrapped symmetric taps on an F-point grid:
 * G(k) = g0 + 2 sum_{j=1..r} g_j cos(2 pi j k / F).  Equal to the DFT of
 * padKernel3D's wrap of the 1D kernel (convolutionFFT.cuh:402-445). */
void vfo_gauss_spectrum(const double *taps, int r, int F, double *spec)
{
    for (int k = 0; k < F; ++k) {
        double s = taps[r];
        for (int j = 1; j <= r; ++j)
            s += 2.0 * taps[r + j] * cos(2.0 * VFO_PI * (double)j * (double)k / (double)F);
        spec[k] = s;
    }
}

/* ------------------------------------------------------------------ */
/* FP64 mixed-radix Stockham FFT (any length; each factor handled by a  */
/* direct DFT of that radix).  sign = -1 forward, +1 inverse, unscaled. */
/* Stands in for cuFFT's cufftExecR2C / cufftExecC2R                    */
/* (Diffusion.cu:1814, 1842), applied here to complex data.             */
/* ------------------------------------------------------------------ */
static int vfo_factor(int n, int *f)
{
    int k = 0;
    static const int pref[] = {8, 4, 2, 3, 5, 7};
    for (int i = 0; i < 6; ++i)
        while (n % pref[i] == 0 && n > 1) { f[k++] = pref[i]; n /= pref[i]; }
    for (int p = 11; n > 1; p += 2)
        while (n % p == 0) { f[k++] = p; n /= p; }
    return k;
}

void vfo_fft(int n, double *re, double *im, int sign)
{
    if (n <= 1) return;
    int fac[64];
    int nf = vfo_factor(n, fac);
    double *ar = re, *ai = im;
    double *br = (double *)malloc(sizeof(double) * n);
    double *bi = (double *)malloc(sizeof(double) * n);
    double vr[64], vi[64], wr[64], wi[64];
    int ns = 1;
    for (int s = 0; s < nf; ++s) {
        int R = fac[s], M = n / R;
        for (int j = 0; j < M; ++j) {
            int jm = j % ns;
            for (int q = 0; q < R; ++q) {
                double ang = sign * 2.0 * VFO_PI * (double)(jm * q) / (double)(ns * R);
                double c = cos(ang), sn = sin(ang);
                double xr = ar[j + q * M], xi = ai[j + q * M];
                vr[q] = xr * c - xi * sn;
                vi[q] = xr * sn + xi * c;
            }
            for (int k = 0; k < R; ++k) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < R; ++q) {
                    double ang = sign * 2.0 * VFO_PI * (double)((q * k) % R) / (double)R;
                    double c = cos(ang), sn = sin(ang);
                    sr += vr[q] * c - vi[q] * sn;
                    si += vr[q] * sn + vi[q] * c;
                }
                wr[k] = sr; wi[k] = si;
            }
            int d = (j / ns) * ns * R + jm;
            for (int k = 0; k < R; ++k) { br[d + k * ns] = wr[k]; bi[d + k * ns] = wi[k]; }
        }
        double *t;
        t = ar; ar = br; br = t;
        t = ai; ai = bi; bi = t;
        ns *= R;
    }
    if (ar != re) {
        memcpy(re, ar, sizeof(double) * n);
        memcpy(im, ai, sizeof(double) * n);
        free(ar); free(ai);
    } else {
        free(br); free(bi);
    }
}

/* ------------------------------------------------------------------ */
/* Boundary treatment.                                                 */
/* pad mode 0 (zero): the whole data grid is interior, outside is 0.   */
/* pad mode 1 (constant VF): padDataConstantVF3D_kernel                 */
/* (convolutionFFT.cuh:590-638) -- interior is 0<z<D-1, 0<y<H-1,       */
/* 0<x<epi; every other FFT-grid voxel (padding AND the outer data     */
/* shell AND x >= epi) holds the baseline b.                           */
/* The convolution of that padded grid equals b + conv(M .* (u - b))   */
/* because the kernel sums to one; v = M .* (u - b) is what is built.  */
/* ------------------------------------------------------------------ */
void vfo_prepare(int nx, int ny, int nz, const float *u, double b, int pad_mode,
                 int epi, double *v)
{
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
                int inside = 1;
                if (pad_mode == 1)
                    inside = (z > 0 && z < nz - 1 && y > 0 && y < ny - 1 && x > 0 && x < epi);
                v[i] = inside ? ((double)u[i] - b) : 0.0;
            }
}

/* ------------------------------------------------------------------ */
/* O2: separable direct linear convolution with zero padding, in place.*/
/* Exactly equal (in exact arithmetic) to the FFT circular convolution */
/* on any grid F >= n + r followed by the top-left crop                */
/* (unpadResult3D_kernel, convolutionFFT.cuh:152-171).                 */
/* leaked[a] (optional) gets the mass pushed outside [0,n) on axis a.  */
/* ------------------------------------------------------------------ */
static void conv_axis(int n, size_t stride, size_t count_outer, size_t outer_stride,
                      size_t count_inner, size_t inner_stride, double *v,
                      const double *taps, int r, double *leak)
{
    double *line = (double *)malloc(sizeof(double) * (n + 2 * r));
    double lk = 0.0;
    for (size_t o = 0; o < count_outer; ++o)
        for (size_t in = 0; in < count_inner; ++in) {
            double *base = v + o * outer_stride + in * inner_stride;
            for (int i = 0; i < n + 2 * r; ++i) line[i] = 0.0;
            for (int i = 0; i < n; ++i) line[i + r] = base[(size_t)i * stride];
            /* full linear convolution over output positions [-r, n+r) */
            for (int p = -r; p < n + r; ++p) {
                double s = 0.0;
                for (int j = -r; j <= r; ++j) {
                    int q = p - j;
                    if (q >= 0 && q < n) s += taps[j + r] * line[q + r];
                }
                if (p >= 0 && p < n) base[(size_t)p * stride] = s;
                else lk += s;
            }
        }
    if (leak) *leak += lk;
    free(line);
}

void vfo_conv_sep_direct(int nx, int ny, int nz, double *v,
                         const double *tx, int rx, const double *ty, int ry,
                         const double *tz, int rz, double *leaked3)
{
    double l[3] = {0, 0, 0};
    size_t sx = 1, sy = (size_t)nx, sz = (size_t)nx * ny;
    /* x lines: outer z, inner y */
    conv_axis(nx, sx, nz, sz, ny, sy, v, tx, rx, &l[0]);
    /* y lines: outer z, inner x */
    conv_axis(ny, sy, nz, sz, nx, sx, v, ty, ry, &l[1]);
    /* z lines: outer y, inner x */
    conv_axis(nz, sz, ny, sy, nx, sx, v, tz, rz, &l[2]);
    if (leaked3) { leaked3[0] = l[0]; leaked3[1] = l[1]; leaked3[2] = l[2]; }
}

/* ------------------------------------------------------------------ */
/* O2 again, the same sums in FP64, split over OpenMP threads and with  */
/* the strided y / z lines gathered B columns at a time, so that the   */
/* full-size configurations (50 M - 170 M voxels) run in seconds.      */
/* ------------------------------------------------------------------ */
/* taps j of output p that reach inputs q = p - j in [0, n) */
static inline void tap_range(int p, int n, int r, int *jlo, int *jhi)
{
    *jlo = (p - (n - 1) > -r) ? p - (n - 1) : -r;
    *jhi = (p < r) ? p : r;
}

/* contiguous rows of n (x lines) */
static double conv_rows_mt(int n, size_t nrows, double *v, const double *t, int r)
{
    double lk = 0.0;
#pragma omp parallel reduction(+ : lk)
    {
        double *line = (double *)malloc(sizeof(double) * (size_t)n);
#pragma omp for schedule(static)
        for (long long row = 0; row < (long long)nrows; ++row) {
            double *b = v + (size_t)row * n;
            for (int i = 0; i < n; ++i) line[i] = b[i];
            for (int p = -r; p < n + r; ++p) {
                int jlo, jhi;
                tap_range(p, n, r, &jlo, &jhi);
                double s = 0.0;
                for (int j = jlo; j <= jhi; ++j) s += t[j + r] * line[p - j];
                if (p >= 0 && p < n) b[p] = s;
                else lk += s;
            }
        }
        free(line);
    }
    return lk;
}

/* lines along a strided axis: element (col, pos, outer) at
 * v[col + pos*ps + outer*os], ncols contiguous columns per outer index */
static double conv_cols_mt(int n, size_t ps, size_t nouter, size_t os, int ncols, double *v, const double *t,
                           int r)
{
    enum { B = 64 };
    const long long nblk = (ncols + B - 1) / B;
    double lk = 0.0;
#pragma omp parallel reduction(+ : lk)
    {
        double *buf = (double *)malloc(sizeof(double) * (size_t)n * B);
        double acc[B];
#pragma omp for schedule(static)
        for (long long task = 0; task < (long long)nouter * nblk; ++task) {
            const size_t o = (size_t)(task / nblk);
            const int c0 = (int)(task % nblk) * B;
            const int w = (ncols - c0 < B) ? ncols - c0 : B;
            double *base = v + o * os + c0;
            for (int i = 0; i < n; ++i) memcpy(buf + (size_t)i * B, base + (size_t)i * ps, sizeof(double) * w);
            for (int p = -r; p < n + r; ++p) {
                int jlo, jhi;
                tap_range(p, n, r, &jlo, &jhi);
                for (int c = 0; c < w; ++c) acc[c] = 0.0;
                for (int j = jlo; j <= jhi; ++j) {
                    const double tj = t[j + r];
                    const double *src = buf + (size_t)(p - j) * B;
                    for (int c = 0; c < w; ++c) acc[c] += tj * src[c];
                }
                if (p >= 0 && p < n) memcpy(base + (size_t)p * ps, acc, sizeof(double) * w);
                else
                    for (int c = 0; c < w; ++c) lk += acc[c];
            }
        }
        free(buf);
    }
    return lk;
}

void vfo_conv_sep_direct_mt(int nx, int ny, int nz, double *v,
                            const double *tx, int rx, const double *ty, int ry,
                            const double *tz, int rz, double *leaked3)
{
    double l[3];
    const size_t sxy = (size_t)nx * ny;
    l[0] = conv_rows_mt(nx, (size_t)ny * nz, v, tx, rx);
    l[1] = conv_cols_mt(ny, (size_t)nx, (size_t)nz, sxy, nx, v, ty, ry);  /* (x, y, z) */
    l[2] = conv_cols_mt(nz, sxy, (size_t)ny, (size_t)nx, nx, v, tz, rz);  /* (x, z, y) */
    if (leaked3) { leaked3[0] = l[0]; leaked3[1] = l[1]; leaked3[2] = l[2]; }
}

/* ------------------------------------------------------------------ */
/* O3: full 3D FFT convolution on an Fx*Fy*Fz grid, FP64, own FFT.     */
/* Order of operations of fftDiffuse3D (Diffusion.cu:1622-1934):       */
/* pad (here v zero-padded), forward 3D DFT, pointwise multiply by the */
/* kernel spectrum with 1/N scaling (modulateAndNormalize_kernel,      */
/* convolutionFFT.cuh:696-716), inverse 3D DFT, top-left crop.         */
/* Kernel given either as a separable real spectrum (spec_x/y/z) or as */
/* a dense window w (kd*kh*kw, centre kz0,ky0,kx0) wrapped to index 0  */
/* like padKernel3D_kernel (convolutionFFT.cuh:402-445).               */
/* full_sum (optional) returns the sum over the whole FFT grid of the  */
/* convolved result (crop + leaked).                                   */
/* ------------------------------------------------------------------ */
static void fft3d(int Fx, int Fy, int Fz, double *re, double *im, int sign)
{
    int mx = Fx > Fy ? Fx : Fy;
    if (Fz > mx) mx = Fz;
    double *lr = (double *)malloc(sizeof(double) * mx);
    double *li = (double *)malloc(sizeof(double) * mx);
    size_t sy = (size_t)Fx, sz = (size_t)Fx * Fy;
    for (int z = 0; z < Fz; ++z)
        for (int y = 0; y < Fy; ++y) {
            double *pr = re + z * sz + y * sy, *pi = im + z * sz + y * sy;
            vfo_fft(Fx, pr, pi, sign);
        }
    for (int z = 0; z < Fz; ++z)
        for (int x = 0; x < Fx; ++x) {
            for (int y = 0; y < Fy; ++y) { lr[y] = re[z * sz + y * sy + x]; li[y] = im[z * sz + y * sy + x]; }
            vfo_fft(Fy, lr, li, sign);
            for (int y = 0; y < Fy; ++y) { re[z * sz + y * sy + x] = lr[y]; im[z * sz + y * sy + x] = li[y]; }
        }
    for (int y = 0; y < Fy; ++y)
        for (int x = 0; x < Fx; ++x) {
            for (int z = 0; z < Fz; ++z) { lr[z] = re[z * sz + y * sy + x]; li[z] = im[z * sz + y * sy + x]; }
            vfo_fft(Fz, lr, li, sign);
            for (int z = 0; z < Fz; ++z) { re[z * sz + y * sy + x] = lr[z]; im[z * sz + y * sy + x] = li[z]; }
        }
    free(lr); free(li);
}

int vfo_conv_fft3d(int nx, int ny, int nz, int Fx, int Fy, int Fz, double *v,
                   const double *spec_x, const double *spec_y, const double *spec_z,
                   const double *w, int kw, int kh, int kd, int kx0, int ky0, int kz0,
                   double *full_sum)
{
    if (Fx < nx || Fy < ny || Fz < nz) return -1;
    size_t N = (size_t)Fx * Fy * Fz;
    double *re = (double *)calloc(N, sizeof(double));
    double *im = (double *)calloc(N, sizeof(double));
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                re[(size_t)x + (size_t)Fx * (y + (size_t)Fy * z)] =
                    v[(size_t)x + (size_t)nx * (y + (size_t)ny * z)];
    fft3d(Fx, Fy, Fz, re, im, -1);
    if (w) {
        double *kr = (double *)calloc(N, sizeof(double));
        double *ki = (double *)calloc(N, sizeof(double));
        for (int z = 0; z < kd; ++z)
            for (int y = 0; y < kh; ++y)
                for (int x = 0; x < kw; ++x) {
                    int pz = z - kz0, py = y - ky0, px = x - kx0;
                    pz = ((pz % Fz) + Fz) % Fz; py = ((py % Fy) + Fy) % Fy; px = ((px % Fx) + Fx) % Fx;
                    kr[(size_t)px + (size_t)Fx * (py + (size_t)Fy * pz)] +=
                        w[(size_t)x + (size_t)kw * (y + (size_t)kh * z)];
                }
        fft3d(Fx, Fy, Fz, kr, ki, -1);
        for (size_t i = 0; i < N; ++i) {
            double ar = re[i], ai = im[i];
            re[i] = (ar * kr[i] - ai * ki[i]) / (double)N;
            im[i] = (ar * ki[i] + ai * kr[i]) / (double)N;
        }
        free(kr); free(ki);
    } else {
        for (int z = 0; z < Fz; ++z)
            for (int y = 0; y < Fy; ++y)
                for (int x = 0; x < Fx; ++x) {
                    size_t i = (size_t)x + (size_t)Fx * (y + (size_t)Fy * z);
                    double k = spec_x[x] * spec_y[y] * spec_z[z] / (double)N;
                    re[i] *= k; im[i] *= k;
                }
    }
    fft3d(Fx, Fy, Fz, re, im, +1);
    double fs = 0.0;
    for (size_t i = 0; i < N; ++i) fs += re[i];
    if (full_sum) *full_sum = fs;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                v[(size_t)x + (size_t)nx * (y + (size_t)ny * z)] =
                    re[(size_t)x + (size_t)Fx * (y + (size_t)Fy * z)];
    free(re); free(im);
    return 0;
}

/* ------------------------------------------------------------------ */
/* O1: literal 3D direct sum with a dense window, zero padding.        */
/* t(p) = sum_q w(q) v(p - q + K), the orientation of the reference's  */
/* gold routine convolutionClampToBorderCPU                            */
/* (convolutionFFT_gold.cpp:22-58) with zero instead of clamp outside. */
/* ------------------------------------------------------------------ */
void vfo_conv_direct3d(int nx, int ny, int nz, const double *v, double *out,
                       const double *w, int kw, int kh, int kd, int kx0, int ky0, int kz0)
{
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double s = 0.0;
                for (int qz = 0; qz < kd; ++qz) {
                    int sz = z - qz + kz0;
                    if (sz < 0 || sz >= nz) continue;
                    for (int qy = 0; qy < kh; ++qy) {
                        int sy = y - qy + ky0;
                        if (sy < 0 || sy >= ny) continue;
                        for (int qx = 0; qx < kw; ++qx) {
                            int sx = x - qx + kx0;
                            if (sx < 0 || sx >= nx) continue;
                            s += w[(size_t)qx + (size_t)kw * (qy + (size_t)kh * qz)] *
                                 v[(size_t)sx + (size_t)nx * (sy + (size_t)ny * sz)];
                        }
                    }
                }
                out[(size_t)x + (size_t)nx * (y + (size_t)ny * z)] = s;
            }
}

/* 2D clamp-to-border direct sum, the same contract as the reference's   */
/* convolutionClampToBorderCPU (convolutionFFT_gold.cpp:22-58), FP64 out. */
void vfo_conv_clamp2d(int h, int wd, const double *data, const double *ker,
                      int kh, int kw, int ky0, int kx0, double *out)
{
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < wd; ++x) {
            double s = 0.0;
            for (int qy = 0; qy < kh; ++qy)
                for (int qx = 0; qx < kw; ++qx) {
                    int sy = y - qy + ky0, sx = x - qx + kx0;
                    if (sy < 0) sy = 0;
                    if (sy >= h) sy = h - 1;
                    if (sx < 0) sx = 0;
                    if (sx >= wd) sx = wd - 1;
                    s += ker[qy * kw + qx] * data[sy * wd + sx];
                }
            out[y * wd + x] = s;
        }
}

/* ------------------------------------------------------------------ */
/* Reference-mode kernel: the 7-point explicit diffusion stencil       */
/* (centre 1 - 6*lambda - gamma*dt, six arms lambda;                    */
/* Diffusion.cu:1182-1195) applied n_steps times to a unit impulse,    */
/* then the centred (2R+1)^3 window is returned (extractCenter3D,       */
/* convolutionFFT.cuh:77-112).  The working grid is large enough that   */
/* nothing reaches its edge (support grows by one voxel per step).     */
/* ------------------------------------------------------------------ */
int vfo_stencil_power(double lambda, double gamma_dt, int n_steps, int R, double *w)
{
    int H = n_steps > R ? n_steps : R;
    int n = 2 * H + 3;
    size_t N = (size_t)n * n * n;
    double *a = (double *)calloc(N, sizeof(double));
    double *b = (double *)calloc(N, sizeof(double));
    if (!a || !b) { free(a); free(b); return -1; }
    size_t c = (size_t)(H + 1) * (1 + n + (size_t)n * n);
    a[c] = 1.0;
    double cc = 1.0 - 6.0 * lambda - gamma_dt;
    size_t sy = n, sz = (size_t)n * n;
    for (int s = 0; s < n_steps; ++s) {
        for (int z = 1; z < n - 1; ++z)
            for (int y = 1; y < n - 1; ++y)
                for (int x = 1; x < n - 1; ++x) {
                    size_t i = x + sy * y + sz * z;
                    b[i] = cc * a[i] + lambda * (a[i - 1] + a[i + 1] + a[i - sy] + a[i + sy] +
                                                  a[i - sz] + a[i + sz]);
                }
        double *t = a; a = b; b = t;
    }
    int k = 2 * R + 1;
    for (int z = 0; z < k; ++z)
        for (int y = 0; y < k; ++y)
            for (int x = 0; x < k; ++x)
                w[x + (size_t)k * (y + (size_t)k * z)] =
                    a[(x - R + H + 1) + sy * (y - R + H + 1) + sz * (z - R + H + 1)];
    free(a); free(b);
    return 0;
}

/* ------------------------------------------------------------------ */
/* One full substep on a float field, FP64 inside, result FP64.        */
/* method 0: separable direct (O2); 1: 3D FFT on grid F (O3).           */
/* out = (1 - rate) * (b + conv(M .* (u - b))).                         */
/* mass3 (optional): [sum v, leaked (full-grid or per-axis sum), 0].    */
/* ------------------------------------------------------------------ */
/* ------------------------------------------------------------------ */
/* The same window computed from the stencil's spectrum, FP64, for      */
/* step counts where explicit iteration is too large (the reference's   */
/* human-VF kernel: 894 steps).  S(k) = 1 - 6 lambda - gamma_dt +       */
/* 2 lambda (cos kx + cos ky + cos kz) on a periodic G^3 grid, raised   */
/* to n_steps (signed integer power), inverse 3D DFT / G^3, centred     */
/* window of half-width R.  Equal to the explicit iteration up to the   */
/* periodic images of the kernel, which reach the window from distance  */
/* G - R: below 1e-15 of the centre value for G - R >= 8.5 sigma,       */
/* sigma = sqrt(2 lambda n_steps) (G = 256 for the reference's 894      */
/* steps at lambda 0.1333, R = 73).                                     */
/* ------------------------------------------------------------------ */
int vfo_stencil_power_spectral(double lambda, double gamma_dt, int n_steps, int R, int G, double *w)
{
    if (G < 2 * R + 1) return -2;
    size_t N = (size_t)G * G * G;
    double *re = (double *)calloc(N, sizeof(double));
    double *im = (double *)calloc(N, sizeof(double));
    double *cs = (double *)malloc(sizeof(double) * G);
    if (!re || !im || !cs) { free(re); free(im); free(cs); return -1; }
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < G; ++k) cs[k] = cos(two_pi * (double)k / (double)G);
    const double c0 = 1.0 - 6.0 * lambda - gamma_dt;
    for (int z = 0; z < G; ++z)
        for (int y = 0; y < G; ++y)
            for (int x = 0; x < G; ++x) {
                double sk = c0 + 2.0 * lambda * (cs[x] + cs[y] + cs[z]);
                /* integer power by squaring keeps the sign of negative bins */
                double r = 1.0, b = sk;
                for (int e = n_steps; e > 0; e >>= 1) {
                    if (e & 1) r *= b;
                    b *= b;
                }
                re[x + (size_t)G * (y + (size_t)G * z)] = r;
            }
    fft3d(G, G, G, re, im, +1);
    const double inv = 1.0 / (double)N;
    int k = 2 * R + 1;
    for (int z = 0; z < k; ++z)
        for (int y = 0; y < k; ++y)
            for (int x = 0; x < k; ++x) {
                int gx = (x - R + G) % G, gy = (y - R + G) % G, gz = (z - R + G) % G;
                w[x + (size_t)k * (y + (size_t)k * z)] = re[gx + (size_t)G * (gy + (size_t)G * gz)] * inv;
            }
    free(re); free(im); free(cs);
    return 0;
}

int vfo_substep(int nx, int ny, int nz, const float *u, double *out,
                double sigma_x, double sigma_y, double sigma_z, int rx, int ry, int rz,
                double rate, double b, int pad_mode, int epi, int method,
                int Fx, int Fy, int Fz, double *mass3)
{
    size_t V = (size_t)nx * ny * nz;
    double *tx = (double *)malloc(sizeof(double) * (2 * rx + 1));
    double *ty = (double *)malloc(sizeof(double) * (2 * ry + 1));
    double *tz = (double *)malloc(sizeof(double) * (2 * rz + 1));
    if (vfo_gauss_taps(sigma_x, rx, tx) || vfo_gauss_taps(sigma_y, ry, ty) ||
        vfo_gauss_taps(sigma_z, rz, tz)) {
        free(tx); free(ty); free(tz);
        return -1;
    }
    vfo_prepare(nx, ny, nz, u, b, pad_mode, epi, out);
    double sv = 0.0;
    for (size_t i = 0; i < V; ++i) sv += out[i];
    double leaked = 0.0;
    int rc = 0;
    if (method == 0) {
        double l3[3];
        vfo_conv_sep_direct(nx, ny, nz, out, tx, rx, ty, ry, tz, rz, l3);
        leaked = l3[0] + l3[1] + l3[2];
    } else {
        double *sx = (double *)malloc(sizeof(double) * Fx);
        double *sy = (double *)malloc(sizeof(double) * Fy);
        double *sz = (double *)malloc(sizeof(double) * Fz);
        vfo_gauss_spectrum(tx, rx, Fx, sx);
        vfo_gauss_spectrum(ty, ry, Fy, sy);
        vfo_gauss_spectrum(tz, rz, Fz, sz);
        double fs = 0.0;
        rc = vfo_conv_fft3d(nx, ny, nz, Fx, Fy, Fz, out, sx, sy, sz, NULL, 0, 0, 0, 0, 0, 0, &fs);
        double sc = 0.0;
        for (size_t i = 0; i < V; ++i) sc += out[i];
        leaked = fs - sc;
        free(sx); free(sy); free(sz);
    }
    double keep = 1.0 - rate;
    for (size_t i = 0; i < V; ++i) out[i] = keep * (b + out[i]);
    if (mass3) { mass3[0] = sv; mass3[1] = leaked; mass3[2] = 0.0; }
    free(tx); free(ty); free(tz);
    return rc;
}

/* Source deposit u[idx_j] += amt_j (duplicates accumulate).  The agents'
 * dChem[ic][voxel] += inc (Agent.cpp:185) followed by the update's
 * p = d + t * decay (WHChemical.cpp:420-450). */
int vfo_deposit(double *u, size_t V, const int32_t *idx, const float *amt, int64_t n)
{
    for (int64_t j = 0; j < n; ++j) {
        if (idx[j] < 0 || (size_t)idx[j] >= V) return -1;
        u[idx[j]] += (double)amt[j];
    }
    return 0;
}

/* The reference's post-diffusion update, WHChemical::update(gpuUpdate)
 * (WHChemical.cpp:420-450): p = d + t * decay; d = 0; total = sum p (FP64). */
double vfo_update(size_t V, const float *t, float *d, float *p, double decay)
{
    double s = 0.0;
    for (size_t i = 0; i < V; ++i) {
        float level = (float)((double)d[i] + (double)t[i] * decay);
        d[i] = 0.0f;
        p[i] = level;
        s += (double)level;
    }
    return s;
}

double vfo_sum(const double *u, size_t V)
{
    double s = 0.0;
    for (size_t i = 0; i < V; ++i) s += u[i];
    return s;
}
