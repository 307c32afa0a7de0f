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
// The row and column passes run on the two-pass register FFT
// (vfd_gen_tpr.cu) when the line length splits as f1 * f2 with f1, f2 <= 32;
// the Stockham kernels below serve every other length (and all lengths with
// VFD_GEN_ENGINE=stockham).  launch_gen_rows / launch_gen_cols choose.
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
#include <stdlib.h>
#include <string.h>

#include "vfd_general.h"
#include "vfd_internal.h"

namespace vfd {

// Tiles are fetched with cp.async: every element of a tile is in flight at
// once without holding registers (the loads are otherwise bound by latency
// at the one or two CTAs per SM that the FFT tiles allow).  The issuing
// thread sees its own copies after cp.async.wait_group, so a pass that
// touches only the elements it fetched needs no barrier.
__device__ __forceinline__ void g_cp4(float *smem, const float *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void g_cp8(float2 *smem, const float2 *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void g_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void g_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ double warp_sum_g(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of v over the block added to *dst (skipped when dst is NULL or the
// sum is zero); red holds one double per warp.
__device__ __forceinline__ void block_sum_atomic_g(double v, double *dst, double *red)
{
    v = warp_sum_g(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        v = warp_sum_g(v);
        if (l == 0 && v != 0.0 && dst) atomicAdd(dst, v);
    }
    __syncthreads();
}

// Shared layout of the Stockham row and column kernels: the tile (F
// positions of NL + 1 complex values), the F twiddles, then the c2r side
// buffer [2][NL] or the fused z pass's spectrum tile [F][NL] (when staged).
// These kernels serve the lengths the register engine (vfd_gen_tpr.cu)
// cannot split.
__host__ __device__ __forceinline__ int tile_elems(int F, int NL) { return F * (NL + 1); }
__device__ __forceinline__ void load_twiddles(float2 *tw, const float2 *src, int F)
{
    for (int i = threadIdx.x; i < F; i += blockDim.x) tw[i] = src[i];
}

// ---------------------------------------------------------------------------
// R2C along x: 2 NL real rows per CTA, rows r0 + l (real parts) and
// r0 + NL + l (imaginary parts) of complex line l.
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) r2c_x_kernel(const GenRowPass p)
{
    constexpr int NT = NL * TL, NW = NT / 32, LS = NL + 1, NR = 2 * NL;
    extern __shared__ __align__(16) float2 gsm[];
    __shared__ double red[32];
    const int F = p.plan.F;
    float2 *S = gsm;
    float *Sf = reinterpret_cast<float *>(gsm);
    float2 *tw = S + tile_elems(F, NL);
    load_twiddles(tw, p.tw, F);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = blockIdx.x * NR;

    // real rows: warp w takes tile rows w, w + NW, ...; its lanes walk the
    // row's positions (128 contiguous bytes per load); positions >= nload
    // and rows outside the padding box are zero-filled
    for (int q = warp; q < NR; q += NW) {
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
        for (int x = lane; x < F; x += 32) {
            const bool v = rowin && x < p.nload;
            g_cp4(&Sf[x * 2 * LS + sidx], v ? src + x : p.rsrc, v);
        }
    }
    g_commit();
    g_wait<0>();
    // padding rule and input mass over this thread's own elements
    double acc = 0.0;
    if (p.fuse_pad || p.mass_in) {
        for (int q = warp; q < NR; q += NW) {
            const int row = r0 + q;
            const int sidx = 2 * (q % NL) + q / NL;
            bool rowin = row < p.nrows;
            if (rowin && p.fuse_pad) {
                const int r1 = row % p.rows_per_plane, r2 = row / p.rows_per_plane;
                rowin = r1 >= p.box_lo[1] && r1 < p.box_hi[1] && r2 >= p.box_lo[2] && r2 < p.box_hi[2];
            }
            for (int x = lane; x < p.nload; x += 32) {
                float w = Sf[x * 2 * LS + sidx];
                if (p.fuse_pad) {
                    w = (rowin && x >= p.box_lo[0] && x < p.box_hi[0]) ? w - p.b : 0.0f;
                    Sf[x * 2 * LS + sidx] = w;
                }
                acc += (double)w;
            }
        }
    }
    __syncthreads();
    fft_lines<MAXP, TL, NL, false>(S, p.plan, threadIdx.x % NL, threadIdx.x / NL, tw);

    // split the two real rows' half spectra: warp per output row, lanes along k
    const int Fh = F / 2 + 1;
    for (int q = warp; q < NR; q += NW) {
        const int rr = r0 + q;
        if (rr >= p.nrows) continue;
        const int ln = q % NL;
        const int s1 = rr % p.rows_per_plane, s2 = rr / p.rows_per_plane;
        float2 *dst = p.cdst + (int64_t)s1 * p.c_s1 + (int64_t)s2 * p.c_s2;
        for (int k = lane; k < Fh; k += 32) {
            const float2 z = S[k * LS + ln];
            const float2 zc = S[(k == 0 ? 0 : F - k) * LS + ln];  // Z(-k)
            dst[k] = q < NL ? make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y))    // A(k)
                            : make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));  // B(k)
        }
    }
    block_sum_atomic_g(acc, p.mass_in, red);
}

// C2R along x with the optional crop / update epilogue.
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) c2r_x_kernel(const GenRowPass p)
{
    constexpr int NT = NL * TL, NW = NT / 32, LS = NL + 1, NR = 2 * NL;
    extern __shared__ __align__(16) float2 gsm[];
    __shared__ double red[32];
    const int F = p.plan.F;
    const int Fh = F / 2 + 1;
    float2 *S = gsm;
    const float *Sf = reinterpret_cast<const float *>(gsm);
    float2 *tw = S + tile_elems(F, NL);
    float2 *Sb = tw + F;  // [2][NL]
    load_twiddles(tw, p.tw, F);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = blockIdx.x * NR;

    // z(k) = A(k) + i B(k) for every k from the Hermitian halves.  Warp w
    // takes line pairs w, w + NW, ...; its lanes walk k.  A(k) is fetched
    // into slot k and B(k) into slot F - k, which z(-k) takes (B(0) and
    // B(F/2), whose slots A holds, into the side buffer Sb); after the wait
    // each thread combines the pairs it fetched.
    for (int ln = warp; ln < NL; ln += NW) {
        const int ra = r0 + ln, rb = r0 + NL + ln;
        const float2 *pa = nullptr, *pb = nullptr;
        if (ra < p.nrows)
            pa = p.csrc + (int64_t)(ra % p.rows_per_plane) * p.c_s1 + (int64_t)(ra / p.rows_per_plane) * p.c_s2;
        if (rb < p.nrows)
            pb = p.csrc + (int64_t)(rb % p.rows_per_plane) * p.c_s1 + (int64_t)(rb / p.rows_per_plane) * p.c_s2;
        for (int k = lane; k < Fh; k += 32) {
            float2 *db = k == 0 ? &Sb[ln] : (2 * k == F ? &Sb[NL + ln] : &S[(F - k) * LS + ln]);
            g_cp8(&S[k * LS + ln], pa ? pa + k : p.csrc, pa != nullptr);
            g_cp8(db, pb ? pb + k : p.csrc, pb != nullptr);
        }
    }
    g_commit();
    g_wait<0>();
    for (int ln = warp; ln < NL; ln += NW) {
        for (int k = lane; k < Fh; k += 32) {
            float2 *da = &S[k * LS + ln];
            float2 *db = k == 0 ? &Sb[ln] : (2 * k == F ? &Sb[NL + ln] : &S[(F - k) * LS + ln]);
            const float2 A = *da, B = *db;
            // z(k) = A + iB ; z(-k) = conj(A) + i conj(B)
            *da = make_float2(A.x - B.y, A.y + B.x);
            if (k > 0 && k < F - k) *db = make_float2(A.x + B.y, B.x - A.y);
        }
    }
    __syncthreads();
    fft_lines<MAXP, TL, NL, true>(S, p.plan, threadIdx.x % NL, threadIdx.x / NL, tw);

    double acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int j = threadIdx.x; j < (F - p.nstore) * NL; j += NT) {
        const float2 x = S[(p.nstore + j / NL) * LS + (j % NL)];
        acc_leak += (double)x.x + (double)x.y;
    }
    // real rows: warp w stores tile rows w, w + NW, ...; lanes walk positions
    for (int q = warp; q < NR; q += NW) {
        const int row = r0 + q;
        if (row >= p.nrows) continue;
        const int sidx = 2 * (q % NL) + q / NL;
        const int r1 = row % p.rows_per_plane, r2 = row / p.rows_per_plane;
        float *dst = p.rdst + (int64_t)r1 * p.r_s1 + (int64_t)r2 * p.r_s2;
        // fused WHChemical::update: p = d + decay t, d = 0 (same row layout as the field)
        float *drow = (p.fuse_update && p.dchem) ? p.dchem + (int64_t)r1 * p.r_s1 + (int64_t)r2 * p.r_s2 : nullptr;
        for (int x = lane; x < p.nstore; x += 32) {
            float v = Sf[x * 2 * LS + sidx];
            if (p.fuse_crop) {
                acc_conv += (double)v;
                v = p.keep * (v + p.b * p.k0);
                if (p.fuse_update) {
                    v *= p.upd_scale;
                    if (drow) {
                        v += drow[x];
                        drow[x] = 0.0f;
                    }
                }
                acc_out += (double)v;
            }
            dst[x] = v;
        }
    }
    block_sum_atomic_g(acc_leak, p.mass_leak, red);
    block_sum_atomic_g(acc_conv, p.mass_conv, red);
    block_sum_atomic_g(acc_out, p.mass_out, red);
}

// Complex lines: element (line, outer, pos) at base + line + outer*outer_stride
// + pos*pos_stride (complex units); NL consecutive lines per tile.
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) c2c_kernel(const GenColPass p)
{
    constexpr int NT = NL * TL, LS = NL + 1;
    extern __shared__ __align__(16) float2 gsm[];
    const int F = p.plan.F;
    float2 *S = gsm;
    float2 *tw = S + tile_elems(F, NL);
    load_twiddles(tw, p.tw, F);

    const int tiles_per_outer = (p.nlines + NL - 1) / NL;
    const int outer = blockIdx.x / tiles_per_outer;
    const int l0 = (blockIdx.x - outer * tiles_per_outer) * NL;
    // thread (ln, pg): line ln of the tile, positions pg, pg + TL, ...
    const int ln = threadIdx.x % NL, pg = threadIdx.x / NL;
    const bool ok = (l0 + ln) < p.nlines;
    float2 *base = p.data + (int64_t)outer * p.outer_stride + l0 + ln;
    for (int x = pg; x < F; x += TL) {
        const bool v = ok && x < p.nload;
        g_cp8(&S[x * LS + ln], v ? base + (int64_t)x * p.pos_stride : p.data, v);
    }
    g_commit();
    // fused z pass: the spectrum tile K[kz][ky = outer][kx = l0 + l] (F x NL,
    // after the twiddles) is fetched as a second group, in flight during the
    // forward transform
    float2 *Ks = tw + F;
    const bool ks = p.mode == GEN_FWD_MUL_INV && p.kspec_smem;
    if (ks) {
        for (int j = threadIdx.x; j < F * NL; j += NT) {
            const int k = j / NL, l = j % NL;
            const bool v = l0 + l < p.nlines;
            g_cp8(&Ks[j], v ? p.kspec + (int64_t)k * p.k_s_pos + (int64_t)outer * p.k_s_outer + l0 + l : p.kspec, v);
        }
        g_commit();
    }
    if (ks) g_wait<1>();
    else g_wait<0>();
    __syncthreads();
    const int line = threadIdx.x % NL, tj = threadIdx.x / NL;
    if (p.mode != GEN_INVERSE) fft_lines<MAXP, TL, NL, false>(S, p.plan, line, tj, tw);
    if (p.mode == GEN_FWD_MUL_INV) {
        g_wait<0>();  // this thread's own spectrum elements
        for (int j = threadIdx.x; j < F * NL; j += NT) {
            const int k = j / NL, l = j % NL;
            if (l0 + l >= p.nlines) continue;
            const float2 kk = ks ? Ks[j] : p.kspec[(int64_t)k * p.k_s_pos + (int64_t)outer * p.k_s_outer + l0 + l];
            const float2 x = S[k * LS + l];
            S[k * LS + l] = make_float2(p.scale * (x.x * kk.x - x.y * kk.y), p.scale * (x.x * kk.y + x.y * kk.x));
        }
        __syncthreads();
    }
    if (p.mode != GEN_FORWARD) fft_lines<MAXP, TL, NL, true>(S, p.plan, line, tj, tw);
    if (ok)
        for (int x = pg; x < p.nstore; x += TL) base[(int64_t)x * p.pos_stride] = S[x * LS + ln];
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
    block_sum_atomic_g(ac, mass_conv, red);
    block_sum_atomic_g(ao, mass_out, red);
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
    block_sum_atomic_g(ao, mass_out, red);
}

// Sum of P over the whole FFT grid (the plain path's input mass).
__global__ void sum_kernel(const float *P, int64_t n, double *out)
{
    __shared__ double red[8];
    double a = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a += (double)P[i];
    block_sum_atomic_g(a, out, red);
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
// Launchers.  A pass runs on the register engine (vfd_gen_tpr.cu) when its
// length splits as F = f1 * f2 with f1, f2 <= 32, else on the Stockham kernel
// variant given (index into VFD_AXIS_VARIANTS; NL 16 for c2c coalescing).
// VFD_GEN_ENGINE=stockham keeps every pass on the Stockham kernels.
template <int NL, int TL, int MAXP, int MINB>
static cudaError_t set_attrs()
{
    // once per CUDA context (a device reset starts a new one)
    static thread_local unsigned long long ctx_done = 0;
    const unsigned long long ctx = current_context_id();
    if (ctx != 0 && ctx == ctx_done) return cudaSuccess;
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
    ctx_done = ctx;
    return cudaSuccess;
}

// the tile, the twiddles, then the c2r side buffer [2][NL] or the fused z
// pass's spectrum tile [F][NL]
static size_t gen_smem(int F, int NL, bool spectrum = false)
{
    return ((size_t)tile_elems(F, NL) + F + (spectrum ? (size_t)F * NL : (size_t)2 * NL)) * sizeof(float2);
}

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
    // the fused z pass stages its spectrum tile when it fits beside the data
    GenColPass q = p;
    q.kspec_smem = p.mode == GEN_FWD_MUL_INV && gen_smem(p.plan.F, NL, true) <= axis_smem_limit();
    c2c_kernel<NL, TL, MAXP, MINB><<<blocks, NL * TL, gen_smem(p.plan.F, NL, q.kspec_smem != 0), st>>>(q);
    note_launch();
    return cudaGetLastError();
}

static bool tpr_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_GEN_ENGINE");
        on = !(e && strcmp(e, "stockham") == 0);
    }
    return on == 1;
}

cudaError_t launch_gen_rows(int variant, const GenRowPass &p, bool inverse, cudaStream_t st)
{
    const int f1 = tpr_enabled() ? tpr_split(p.plan.F) : 0;
    if (f1 > 0) return launch_tpr_rows(p, f1, inverse, st);
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
    const int f1 = tpr_enabled() ? tpr_split(p.plan.F) : 0;
    if (f1 > 0) {
        // a pass whose register-engine tile would not fit in shared memory
        // runs on the Stockham kernels
        const cudaError_t e = launch_tpr_cols(p, f1, st);
        if (e != cudaErrorInvalidConfiguration) return e;
    }
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
