// vfd_general.cu -- the general 3D FFT convolution (any kernel spectrum).
//
// Used when a field's kernel is not a separable Gaussian (the reference's
// window: the 7-point stencil to the power n, Diffusion.cu:1078-1531, or any
// user window) and as the unfused "plain" per-field path.  Same order of
// operations as fftDiffuse3D (Diffusion.cu:1622-1934):
//   pad -> R2C along x -> C2C along y -> C2C along z -> multiply by K/N
//   -> inverse C2C z -> inverse C2C y -> C2R along x -> crop.
// The spectrum is laid out [z][y][kx] with Fxh = Fx/2 + 1 bins per row
// (the reference's fftD x fftH x (fftW/2 + 1), Diffusion.cu:1687).
//
// Kernels:
//   r2c_x_kernel   real rows -> half spectra.  Two real rows form one complex
//                  line z = a + i b; after the FFT, A(k) = (Z(k) + conj Z(-k))/2,
//                  B(k) = (Z(k) - conj Z(-k))/(2i).  Optional fused padding rule.
//   c2c_kernel     complex lines along y or z; forward, inverse, or forward +
//                  multiply by the stored spectrum + inverse (fused z pass).
//                  Positions >= nload are zero on input; only positions <
//                  nstore are written (pruning of the zero padding and crop).
//   c2r_x_kernel   half spectra -> real rows (z(k) = A(k) + i B(k) rebuilt
//                  from Hermitian symmetry); optional fused crop epilogue
//                  out = keep * (t + b * K0) with FP64 totals.
//   pad_kernel, modulate_kernel, crop_kernel: the unfused elementwise steps.
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_general.h"
#include "vfd_internal.h"

namespace vfd {

// Global loads each thread keeps in flight before their shared-memory
// stores in the load loops (the loops are otherwise bound by load latency).
constexpr int kGU = 6;

__device__ __forceinline__ double warp_sum_g(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int NT>
__device__ __forceinline__ void block_sum_atomic_g(double v, double *dst, double *red)
{
    v = warp_sum_g(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < NT / 32) ? red[l] : 0.0;
        v = warp_sum_g(v);
        if (l == 0 && v != 0.0 && dst) atomicAdd(dst, v);
    }
    __syncthreads();
}

// Shared layout of every general kernel: tile S[F][NL+1] (float2), then F twiddles.
template <int NL>
__device__ __forceinline__ void load_twiddles(float2 *tw, const float2 *src, int F, int NT)
{
    for (int i = threadIdx.x; i < F; i += NT) tw[i] = src[i];
}

// ---------------------------------------------------------------------------
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) r2c_x_kernel(const GenRowPass p)
{
    constexpr int NT = NL * TL, LS = NL + 1, NR = 2 * NL;
    extern __shared__ __align__(16) float2 gsm[];
    __shared__ double red[NT / 32];
    const int F = p.plan.F;
    float2 *S = gsm;
    float *Sf = reinterpret_cast<float *>(gsm);
    float2 *tw = S + F * LS;
    load_twiddles<NL>(tw, p.tw, F, NT);

    const int r0 = blockIdx.x * NR;
    // real rows: warp w takes tile rows w, w + NT/32, ...; its lanes walk the
    // row's positions, so every load instruction reads 128 contiguous bytes
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int q = warp; q < NR; q += NT / 32) {
        const int row = r0 + q;
        const int sidx = 2 * (q % NL) + q / NL;
        const bool ok = row < p.nrows;
        int r1 = 0, r2 = 0;
        if (ok) {
            r1 = row % p.rows_per_plane;
            r2 = row / p.rows_per_plane;
        }
        bool rowin = ok;
        if (ok && p.fuse_pad)
            rowin = r1 >= p.box_lo[1] && r1 < p.box_hi[1] && r2 >= p.box_lo[2] && r2 < p.box_hi[2];
        const float *src = p.rsrc + (int64_t)r1 * p.r_s1 + (int64_t)r2 * p.r_s2;
        // kGU loads in flight per lane before their shared-memory stores
        for (int x0 = lane; x0 < p.nload; x0 += 32 * kGU) {
            float v[kGU];
#pragma unroll
            for (int u = 0; u < kGU; ++u) {
                const int x = x0 + 32 * u;
                v[u] = (rowin && x < p.nload) ? __ldg(src + x) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < kGU; ++u) {
                const int x = x0 + 32 * u;
                if (x < p.nload) {
                    float w = v[u];
                    if (p.fuse_pad) w = (rowin && x >= p.box_lo[0] && x < p.box_hi[0]) ? w - p.b : 0.0f;
                    Sf[x * 2 * LS + sidx] = w;
                    acc += (double)w;
                }
            }
        }
    }
    for (int i = p.nload * LS + threadIdx.x; i < F * LS; i += NT) S[i] = make_float2(0.f, 0.f);
    __syncthreads();
    fft_lines<MAXP, TL, NL, false>(S, p.plan, threadIdx.x % NL, threadIdx.x / NL, tw);

    // split the two real rows' half spectra; lanes along k for coalesced rows
    const int Fh = F / 2 + 1;
    for (int i = threadIdx.x; i < NR * Fh; i += NT) {
        const int q = i / Fh, k = i - q * Fh;
        const int rr = r0 + q;
        if (rr >= p.nrows) continue;
        const int ln = q % NL;
        const float2 z = S[k * LS + ln];
        const float2 zc = S[((F - k) % F) * LS + ln];  // Z(-k)
        float2 o;
        if (q < NL) o = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));       // A(k)
        else o = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));              // B(k)
        const int s1 = rr % p.rows_per_plane, s2 = rr / p.rows_per_plane;
        p.cdst[(int64_t)s1 * p.c_s1 + (int64_t)s2 * p.c_s2 + k] = o;
    }
    block_sum_atomic_g<NT>(acc, p.mass_in, red);
}

// ---------------------------------------------------------------------------
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) c2r_x_kernel(const GenRowPass p)
{
    constexpr int NT = NL * TL, LS = NL + 1, NR = 2 * NL;
    extern __shared__ __align__(16) float2 gsm[];
    __shared__ double red[NT / 32];
    const int F = p.plan.F;
    const int Fh = F / 2 + 1;
    float2 *S = gsm;
    float *Sf = reinterpret_cast<float *>(gsm);
    float2 *tw = S + F * LS;
    load_twiddles<NL>(tw, p.tw, F, NT);

    const int r0 = blockIdx.x * NR;
    // rebuild z(k) = A(k) + i B(k) for every k from the Hermitian halves:
    // warp w takes line pairs w, w + NT/32, ...; its lanes walk k with kGU
    // loads of each row in flight
    {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int ln = warp; ln < NL; ln += NT / 32) {
            const int ra = r0 + ln, rb = r0 + NL + ln;
            const float2 *pa = nullptr, *pb = nullptr;
            if (ra < p.nrows)
                pa = p.csrc + (int64_t)(ra % p.rows_per_plane) * p.c_s1 + (int64_t)(ra / p.rows_per_plane) * p.c_s2;
            if (rb < p.nrows)
                pb = p.csrc + (int64_t)(rb % p.rows_per_plane) * p.c_s1 + (int64_t)(rb / p.rows_per_plane) * p.c_s2;
            for (int k0 = lane; k0 < Fh; k0 += 32 * kGU) {
                float2 A[kGU], B[kGU];
#pragma unroll
                for (int u = 0; u < kGU; ++u) {
                    const int k = k0 + 32 * u;
                    A[u] = (pa && k < Fh) ? pa[k] : make_float2(0.f, 0.f);
                    B[u] = (pb && k < Fh) ? pb[k] : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < kGU; ++u) {
                    const int k = k0 + 32 * u;
                    if (k < Fh) {
                        // z(k) = A + iB ; z(-k) = conj(A) + i conj(B)
                        S[k * LS + ln] = make_float2(A[u].x - B[u].y, A[u].y + B[u].x);
                        if (k > 0 && k < F - k) S[(F - k) * LS + ln] = make_float2(A[u].x + B[u].y, B[u].x - A[u].y);
                    }
                }
            }
        }
    }
    __syncthreads();
    fft_lines<MAXP, TL, NL, true>(S, p.plan, threadIdx.x % NL, threadIdx.x / NL, tw);

    double acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int i = threadIdx.x; i < (F - p.nstore) * NL; i += NT) {
        const float2 x = S[(p.nstore + i / NL) * LS + (i % NL)];
        acc_leak += (double)x.x + (double)x.y;
    }
    // real rows: warp w stores tile rows w, w + NT/32, ...; lanes walk positions
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = warp; q < NR; q += NT / 32) {
        const int row = r0 + q;
        if (row >= p.nrows) continue;
        const int sidx = 2 * (q % NL) + q / NL;
        const int r1 = row % p.rows_per_plane, r2 = row / p.rows_per_plane;
        float *dst = p.rdst + (int64_t)r1 * p.r_s1 + (int64_t)r2 * p.r_s2;
        // fused WHChemical::update: p = d + decay t, d = 0 (same row layout as the field)
        float *drow = (p.fuse_update && p.dchem) ? p.dchem + (int64_t)r1 * p.r_s1 + (int64_t)r2 * p.r_s2 : nullptr;
        for (int x = lane; x < p.nstore; x += 32) {
            float t = Sf[x * 2 * LS + sidx];
            if (p.fuse_crop) {
                acc_conv += (double)t;
                t = p.keep * (t + p.b * p.k0);
                if (p.fuse_update) {
                    t *= p.upd_scale;
                    if (drow) {
                        t += drow[x];
                        drow[x] = 0.0f;
                    }
                }
                acc_out += (double)t;
            }
            dst[x] = t;
        }
    }
    block_sum_atomic_g<NT>(acc_leak, p.mass_leak, red);
    block_sum_atomic_g<NT>(acc_conv, p.mass_conv, red);
    block_sum_atomic_g<NT>(acc_out, p.mass_out, red);
}

// ---------------------------------------------------------------------------
// Complex lines: element (line, outer, pos) at base + line + outer*outer_stride
// + pos*pos_stride (complex units); NL consecutive lines per tile.
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) c2c_kernel(const GenColPass p)
{
    constexpr int NT = NL * TL, LS = NL + 1, NPG = NT / NL;
    extern __shared__ __align__(16) float2 gsm[];
    const int F = p.plan.F;
    float2 *S = gsm;
    float2 *tw = S + F * LS;
    load_twiddles<NL>(tw, p.tw, F, NT);

    const int tiles_per_outer = (p.nlines + NL - 1) / NL;
    const int outer = blockIdx.x / tiles_per_outer;
    const int l0 = (blockIdx.x - outer * tiles_per_outer) * NL;
    const int ln = threadIdx.x % NL, pg = threadIdx.x / NL;
    const bool ok = (l0 + ln) < p.nlines;
    float2 *base = p.data + (int64_t)outer * p.outer_stride + l0 + ln;
    for (int x0 = pg; x0 < p.nload; x0 += NPG * kGU) {
        float2 v[kGU];
#pragma unroll
        for (int u = 0; u < kGU; ++u) {
            const int x = x0 + NPG * u;
            v[u] = (ok && x < p.nload) ? base[(int64_t)x * p.pos_stride] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < kGU; ++u) {
            const int x = x0 + NPG * u;
            if (x < p.nload) S[x * LS + ln] = v[u];
        }
    }
    for (int i = p.nload * LS + threadIdx.x; i < F * LS; i += NT) S[i] = make_float2(0.f, 0.f);
    __syncthreads();
    const int line = threadIdx.x % NL, tj = threadIdx.x / NL;
    if (p.mode != GEN_INVERSE) fft_lines<MAXP, TL, NL, false>(S, p.plan, line, tj, tw);
    if (p.mode == GEN_FWD_MUL_INV) {
        // K[kz][ky][kx]: this tile is ky = outer, kx = l0 + line
        for (int i = threadIdx.x; i < F * NL; i += NT) {
            const int k = i / NL, l = i % NL;
            if (l0 + l < p.nlines) {
                const float2 kk = p.kspec[(int64_t)k * p.k_s_pos + (int64_t)outer * p.k_s_outer + l0 + l];
                const float2 x = S[k * LS + l];
                S[k * LS + l] = make_float2(p.scale * (x.x * kk.x - x.y * kk.y),
                                            p.scale * (x.x * kk.y + x.y * kk.x));
            }
        }
        __syncthreads();
    }
    if (p.mode != GEN_FORWARD) fft_lines<MAXP, TL, NL, true>(S, p.plan, line, tj, tw);
    if (ok)
        for (int x = pg; x < p.nstore; x += NPG) base[(int64_t)x * p.pos_stride] = S[x * LS + ln];
}

// ---------------------------------------------------------------------------
// Unfused elementwise steps of the plain path.
// pad: P[z][y][x] on the Fx*Fy*Fz grid, the padDataConstantVF3D rule
// (interior box keeps u, every other voxel b) or zero padding (box = data,
// b = 0).  Writes every voxel, so no memset is needed.
__global__ void pad_kernel(float *P, const float *u, int nx, int ny, int nz, int Fx, int Fy, int Fz, int x0,
                           int x1, int y0, int y1, int z0, int z1, float b)
{
    const int64_t N = (int64_t)Fx * Fy * Fz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % Fx);
        const int64_t r = i / Fx;
        const int y = (int)(r % Fy), z = (int)(r / Fy);
        float v = b;
        if (x >= x0 && x < x1 && y >= y0 && y < y1 && z >= z0 && z < z1)
            v = u[(int64_t)x + (int64_t)nx * (y + (int64_t)ny * z)];
        P[i] = v;
    }
}

// C *= K * scale over Nc bins (modulateAndNormalize_kernel's job).
__global__ void modulate_kernel(float2 *C, const float2 *K, int64_t n, float scale)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = C[i], k = K[i];
        C[i] = make_float2(scale * (a.x * k.x - a.y * k.y), scale * (a.x * k.y + a.y * k.x));
    }
}

// u = keep * P[z][y][x] over the data region (unpadResult3D + the decay),
// with FP64 sums of the cropped convolution and of the output.
// With fuse_update: u = d + upd_scale * keep * P and d = 0 (WHChemical::update).
__global__ void crop_kernel(float *u, const float *P, int nx, int ny, int nz, int Fx, int Fy, float keep,
                            double *mass_conv, double *mass_out, int fuse_update, float upd_scale, float *dchem)
{
    __shared__ double red[8];
    const int64_t V = (int64_t)nx * ny * nz;
    double ac = 0.0, ao = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t r = i / nx;
        const int y = (int)(r % ny), z = (int)(r / ny);
        const float t = P[(int64_t)x + (int64_t)Fx * (y + (int64_t)Fy * z)];
        float o = keep * t;
        if (fuse_update) {
            o *= upd_scale;
            if (dchem) {
                o += dchem[i];
                dchem[i] = 0.0f;
            }
        }
        ac += (double)t;
        ao += (double)o;
        u[i] = o;
    }
    block_sum_atomic_g<256>(ac, mass_conv, red);
    block_sum_atomic_g<256>(ao, mass_out, red);
}

// p = d + scale p, d = 0 (d may be NULL): WHChemical::update after a
// separable tick; FP64 total of p.
__global__ void update_kernel(float *p, float *d, float scale, int64_t n, double *mass_out)
{
    __shared__ double red[8];
    double ao = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float o = scale * p[i];
        if (d) {
            o += d[i];
            d[i] = 0.0f;
        }
        p[i] = o;
        ao += (double)o;
    }
    block_sum_atomic_g<256>(ao, mass_out, red);
}

// Sum of P over the whole FFT grid (the plain path's input mass).
__global__ void sum_kernel(const float *P, int64_t n, double *out)
{
    __shared__ double red[8];
    double a = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a += (double)P[i];
    block_sum_atomic_g<256>(a, out, red);
}

// Wrap a window w (kd*kh*kw, centre c) onto the FFT grid so that its centre
// lands at index 0 (padKernel3D_kernel, convolutionFFT.cuh:402-445).  P must
// be zero beforehand.
__global__ void wrap_window_kernel(float *P, const float *w, int kw, int kh, int kd, int cx, int cy, int cz,
                                   int Fx, int Fy, int Fz)
{
    const int64_t n = (int64_t)kw * kh * kd;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % kw);
        const int64_t r = i / kw;
        const int y = (int)(r % kh), z = (int)(r / kh);
        int px = (x - cx) % Fx, py = (y - cy) % Fy, pz = (z - cz) % Fz;
        if (px < 0) px += Fx;
        if (py < 0) py += Fy;
        if (pz < 0) pz += Fz;
        atomicAdd(&P[(int64_t)px + (int64_t)Fx * (py + (int64_t)Fy * pz)], w[i]);
    }
}

// K[kz][ky][kx] = Gx(kx) Gy(ky) Gz(kz) for a separable Gaussian, from the
// per-axis multipliers G(k)/F (so the F factors are restored here).
__global__ void outer_spectrum_kernel(float2 *K, const float *sx, const float *sy, const float *sz, int Fx,
                                      int Fy, int Fz, int Fxh)
{
    const int64_t n = (int64_t)Fxh * Fy * Fz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(i % Fxh);
        const int64_t r = i / Fxh;
        const int ky = (int)(r % Fy), kz = (int)(r / Fy);
        const double v = (double)sx[kx] * Fx * (double)sy[ky] * Fy * (double)sz[kz] * Fz;
        K[i] = make_float2((float)v, 0.0f);
    }
}

// Half spectrum of the 7-point stencil to the power n on a periodic G^3 grid:
// S(k) = c + 2 lambda (cos kx + cos ky + cos kz), c = 1 - 6 lambda - gamma dt
// (the stencil of Diffusion.cu:1182-1195), FP64, stored FP32.
__global__ void stencil_spectrum_kernel(float2 *K, int G, double lambda, double centre, int n)
{
    const int Gh = G / 2 + 1;
    const int64_t total = (int64_t)Gh * G * G;
    const double w = 2.0 / (double)G;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(i % Gh);
        const int64_t r = i / Gh;
        const int ky = (int)(r % G), kz = (int)(r / G);
        const double s = centre + 2.0 * lambda * (cospi(w * kx) + cospi(w * ky) + cospi(w * kz));
        K[i] = make_float2((float)pow(s, (double)n), 0.0f);
    }
}

// Centred (2R+1)^3 window of the periodic grid P (index 0 = the impulse).
__global__ void crop_window_kernel(float *w, const float *P, int G, int R, float scale)
{
    const int k = 2 * R + 1;
    const int64_t total = (int64_t)k * k * k;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % k);
        const int64_t r = i / k;
        const int y = (int)(r % k), z = (int)(r / k);
        const int px = (x - R + G) % G, py = (y - R + G) % G, pz = (z - R + G) % G;
        w[i] = scale * P[(int64_t)px + (int64_t)G * (py + (int64_t)G * pz)];
    }
}

// window[z][y][x] = scale * P[(z - cz) mod Fz][(y - cy) mod Fy][(x - cx) mod Fx]:
// the window whose centre padKernel3D wrapped to index 0, read back from the
// real grid of an inverse transform.
__global__ void unwrap_window_kernel(float *w, const float *P, int kw, int kh, int kd, int cx, int cy, int cz,
                                     int Fx, int Fy, int Fz, float scale)
{
    const int64_t n = (int64_t)kw * kh * kd;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % kw);
        const int64_t r = i / kw;
        const int y = (int)(r % kh), z = (int)(r / kh);
        int px = (x - cx) % Fx, py = (y - cy) % Fy, pz = (z - cz) % Fz;
        if (px < 0) px += Fx;
        if (py < 0) py += Fy;
        if (pz < 0) pz += Fz;
        w[i] = scale * P[(int64_t)px + (int64_t)Fx * (py + (int64_t)Fy * pz)];
    }
}

// ---------------------------------------------------------------------------
// Launchers (variant = index into VFD_AXIS_VARIANTS, NL must be 16 for c2c
// coalescing; any variant works for the row passes).
template <int NL, int TL, int MAXP, int MINB>
static cudaError_t set_attrs()
{
    static thread_local int dev_done = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev_done == dev) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(r2c_x_kernel<NL, TL, MAXP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)axis_smem_limit())) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(c2r_x_kernel<NL, TL, MAXP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)axis_smem_limit())) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(c2c_kernel<NL, TL, MAXP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)axis_smem_limit())) != cudaSuccess)
        return e;
    dev_done = dev;
    return cudaSuccess;
}

static size_t gen_smem(int F, int NL) { return (size_t)F * (NL + 1) * sizeof(float2) + (size_t)F * sizeof(float2); }

template <int NL, int TL, int MAXP, int MINB>
static cudaError_t launch_rows_t(const GenRowPass &p, bool inverse, cudaStream_t st)
{
    cudaError_t e = set_attrs<NL, TL, MAXP, MINB>();
    if (e != cudaSuccess) return e;
    const int blocks = (p.nrows + 2 * NL - 1) / (2 * NL);
    if (blocks <= 0) return cudaSuccess;
    if (inverse) c2r_x_kernel<NL, TL, MAXP, MINB><<<blocks, NL * TL, gen_smem(p.plan.F, NL), st>>>(p);
    else r2c_x_kernel<NL, TL, MAXP, MINB><<<blocks, NL * TL, gen_smem(p.plan.F, NL), st>>>(p);
    note_launch();
    return cudaGetLastError();
}

template <int NL, int TL, int MAXP, int MINB>
static cudaError_t launch_cols_t(const GenColPass &p, cudaStream_t st)
{
    cudaError_t e = set_attrs<NL, TL, MAXP, MINB>();
    if (e != cudaSuccess) return e;
    const int blocks = p.nouter * ((p.nlines + NL - 1) / NL);
    if (blocks <= 0) return cudaSuccess;
    c2c_kernel<NL, TL, MAXP, MINB><<<blocks, NL * TL, gen_smem(p.plan.F, NL), st>>>(p);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_gen_rows(int variant, const GenRowPass &p, bool inverse, cudaStream_t st)
{
    switch (variant) {
#define VFD_GEN_ROW_CASE(i, NL, TL, MAXP, MINB) \
    case i: return launch_rows_t<NL, TL, MAXP, MINB>(p, inverse, st);
        VFD_AXIS_VARIANTS(VFD_GEN_ROW_CASE)
#undef VFD_GEN_ROW_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_gen_cols(int variant, const GenColPass &p, cudaStream_t st)
{
    switch (variant) {
#define VFD_GEN_COL_CASE(i, NL, TL, MAXP, MINB) \
    case i: return launch_cols_t<NL, TL, MAXP, MINB>(p, st);
        VFD_AXIS_VARIANTS(VFD_GEN_COL_CASE)
#undef VFD_GEN_COL_CASE
    default: return cudaErrorInvalidValue;
    }
}

static int grid_for(int64_t n)
{
    int64_t b = (n + 255) / 256;
    return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

cudaError_t launch_pad(float *P, const float *u, int nx, int ny, int nz, int Fx, int Fy, int Fz, const int *lo,
                       const int *hi, float b, cudaStream_t st)
{
    pad_kernel<<<grid_for((int64_t)Fx * Fy * Fz), 256, 0, st>>>(P, u, nx, ny, nz, Fx, Fy, Fz, lo[0], hi[0], lo[1],
                                                                 hi[1], lo[2], hi[2], b);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_modulate(float2 *C, const float2 *K, int64_t n, float scale, cudaStream_t st)
{
    modulate_kernel<<<grid_for(n), 256, 0, st>>>(C, K, n, scale);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_crop(float *u, const float *P, int nx, int ny, int nz, int Fx, int Fy, float keep,
                        double *mass_conv, double *mass_out, cudaStream_t st, int fuse_update, float upd_scale,
                        float *dchem)
{
    crop_kernel<<<grid_for((int64_t)nx * ny * nz), 256, 0, st>>>(u, P, nx, ny, nz, Fx, Fy, keep, mass_conv,
                                                                  mass_out, fuse_update, upd_scale, dchem);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_update(float *p, float *d, float scale, int64_t n, double *mass_out, cudaStream_t st)
{
    update_kernel<<<grid_for(n), 256, 0, st>>>(p, d, scale, n, mass_out);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_sum(const float *P, int64_t n, double *out, cudaStream_t st)
{
    sum_kernel<<<grid_for(n), 256, 0, st>>>(P, n, out);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_outer_spectrum(float2 *K, const float *sx, const float *sy, const float *sz, int Fx, int Fy,
                                  int Fz, cudaStream_t st)
{
    const int Fxh = Fx / 2 + 1;
    outer_spectrum_kernel<<<grid_for((int64_t)Fxh * Fy * Fz), 256, 0, st>>>(K, sx, sy, sz, Fx, Fy, Fz, Fxh);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_stencil_spectrum(float2 *K, int G, double lambda, double centre, int n, cudaStream_t st)
{
    stencil_spectrum_kernel<<<grid_for((int64_t)(G / 2 + 1) * G * G), 256, 0, st>>>(K, G, lambda, centre, n);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_crop_window(float *w, const float *P, int G, int R, float scale, cudaStream_t st)
{
    const int64_t k = 2 * R + 1;
    crop_window_kernel<<<grid_for(k * k * k), 256, 0, st>>>(w, P, G, R, scale);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_unwrap_window(float *w, const float *P, int kw, int kh, int kd, int cx, int cy, int cz, int Fx,
                                 int Fy, int Fz, float scale, cudaStream_t st)
{
    unwrap_window_kernel<<<grid_for((int64_t)kw * kh * kd), 256, 0, st>>>(w, P, kw, kh, kd, cx, cy, cz, Fx, Fy, Fz,
                                                                          scale);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_wrap_window(float *P, const float *w, int kw, int kh, int kd, int cx, int cy, int cz, int Fx,
                               int Fy, int Fz, cudaStream_t st)
{
    wrap_window_kernel<<<grid_for((int64_t)kw * kh * kd), 256, 0, st>>>(P, w, kw, kh, kd, cx, cy, cz, Fx, Fy, Fz);
    note_launch();
    return cudaGetLastError();
}

}  // namespace vfd
