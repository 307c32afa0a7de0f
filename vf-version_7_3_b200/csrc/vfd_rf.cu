// vfd_rf.cu -- one axis of the separable FFT convolution, overlap-save with
// 64-point blocks, each block's FFT held by ONE thread in registers.
//
// Same method as vfd_os.cu (blocks of L = 64 - 2r outputs; forward FFT-64,
// multiply by the kernel's 64-point spectrum, inverse FFT-64, keep L samples
// -- the reference's pad / R2C / modulate / C2R / crop, Diffusion.cu:1731-1859,
// per block; two lines ride in one complex FFT as its real and imaginary
// parts: rows 2q and 2q+1 in the x pass, lines k and k+32 of a tile in the
// y and z passes).  What changes is who holds a block: a thread owns a line
// pair and walks its blocks in order.
//
// Register layout ("split pairs"): the 64 complex samples x[0..63] of a block
// sit in 32 slots of two float2 registers, slot j = {re: (Re x[2j], Re x[2j+1]),
// im: (Im x[2j], Im x[2j+1])}.  Lane .x of every slot is the even-sample
// sequence, lane .y the odd one, so ONE packed FFT-32 (radix 8 x 4; every
// add, subtract and twiddle multiply a packed FP32x2 instruction on both
// sequences, the transposes register renaming, the twiddles constant-bank
// pairs) transforms both.  The radix-2 step that joins them into the 64-point
// spectrum, the spectrum multiply and the radix-2 step that splits it again
// for the inverse are one 2x2 map per bin pair (k, k + 32) (s_middle); the
// inverse FFT-32 then leaves outputs 2m, 2m+1 side by side in slot m.
//
//   y and z passes (lines contiguous in x): a warp owns a tile of 64
//   adjacent lines, lane k the pair (k, k + 32); at each position the warp
//   loads and stores two runs of 128 contiguous bytes straight from and to
//   global memory.  A CTA of W warps takes W
//   tiles of one job and meets at one barrier per block.
//   x pass (positions contiguous): a warp owns 64 rows; each block's window
//   is copied row by row with 16-byte cp.async into a shared tile, each
//   thread reads its pair's two rows (16-byte reads land whole slots), and
//   outputs go back the same way with 16-byte stores (rows 16-byte aligned
//   and n a multiple of 4; otherwise the x pass uses the overlap-save kernel).
//
// In place: block b's window starts r positions before its first output, so
// it overlaps the previous block's last r outputs.  Those r outputs are held
// back (in shared memory) and stored only after the next block has loaded
// its window; everything else is stored as soon as it is computed.  Blocks
// cover outputs [-r, n + r); outputs outside [0, n) are the leak.  The radius
// is a template parameter (1..8): register indices stay compile-time.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "vfd_fft.cuh"
#include "vfd_internal.h"
#include "vfd_rf.h"
#include "vfd_tma.h"

namespace vfd {

// Set when a pass's bounded wait for a bulk copy gave up (read and cleared by
// rf_take_timeout).
__device__ int g_rf_timeout = 0;

__constant__ float2 c_rfw64[64];  // exp(-2 pi i m / 64), FP64-generated on the host
// w = exp(-2 pi i m / 32) = wr + i wi as packed pairs: (wr, wr), (wi, wi), (-wi, -wi)
__constant__ float2 c_spc[32], c_sps[32], c_spn[32];

namespace {

__device__ __forceinline__ float2 r_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 r_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

__device__ __forceinline__ double r_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Two complex values side by side: lane .x and lane .y of re and im.
struct sp2 {
    float2 re, im;
};

__device__ __forceinline__ sp2 s_add(sp2 a, sp2 b) { return {r_add(a.re, b.re), r_add(a.im, b.im)}; }
__device__ __forceinline__ sp2 s_sub(sp2 a, sp2 b) { return {r_sub(a.re, b.re), r_sub(a.im, b.im)}; }
// a + (-i) b (forward) or a + i b (inverse); -i b = (b.im, -b.re)
template <bool INV>
__device__ __forceinline__ sp2 s_add_rot(sp2 a, sp2 b)
{
    return INV ? sp2{r_sub(a.re, b.im), r_add(a.im, b.re)} : sp2{r_add(a.re, b.im), r_sub(a.im, b.re)};
}
// a - (-i) b (forward) or a - i b (inverse)
template <bool INV>
__device__ __forceinline__ sp2 s_sub_rot(sp2 a, sp2 b)
{
    return INV ? sp2{r_add(a.re, b.im), r_sub(a.im, b.re)} : sp2{r_sub(a.re, b.im), r_add(a.im, b.re)};
}

// DFT-4 in place: a_k <- sum_n a_n w4^(+-nk).
template <bool INV>
__device__ __forceinline__ void s_dft4(sp2 &a0, sp2 &a1, sp2 &a2, sp2 &a3)
{
    const sp2 t0 = s_add(a0, a2), t1 = s_sub(a0, a2), t2 = s_add(a1, a3), d = s_sub(a1, a3);
    a0 = s_add(t0, t2);
    a2 = s_sub(t0, t2);
    a1 = s_add_rot<INV>(t1, d);
    a3 = s_sub_rot<INV>(t1, d);
}

// DFT-8 in place (v_k <- X_k), radix 2 x 4: X_k = E_k + w8^k O_k,
// X_{k+4} = E_k - w8^k O_k with E, O the DFT-4 of the even and odd inputs.
template <bool INV>
__device__ __forceinline__ void s_dft8(sp2 &v0, sp2 &v1, sp2 &v2, sp2 &v3, sp2 &v4, sp2 &v5, sp2 &v6, sp2 &v7)
{
    const float h = 0.707106781186547524400844362105f;
    const float2 H = make_float2(h, h), NH = make_float2(-h, -h);
    sp2 e0 = v0, e1 = v2, e2 = v4, e3 = v6, o0 = v1, o1 = v3, o2 = v5, o3 = v7;
    s_dft4<INV>(e0, e1, e2, e3);
    s_dft4<INV>(o0, o1, o2, o3);
    v0 = s_add(e0, o0);
    v4 = s_sub(e0, o0);
    v2 = s_add_rot<INV>(e2, o2);
    v6 = s_sub_rot<INV>(e2, o2);
    if (!INV) {
        // w8 z = h ((zr + zi) + i (zi - zr)); w8^3 z = h ((zi - zr) - i (zr + zi))
        const float2 p = r_add(o1.re, o1.im), q = r_sub(o1.im, o1.re);
        v1 = sp2{__ffma2_rn(p, H, e1.re), __ffma2_rn(q, H, e1.im)};
        v5 = sp2{__ffma2_rn(p, NH, e1.re), __ffma2_rn(q, NH, e1.im)};
        const float2 u = r_sub(o3.im, o3.re), s = r_add(o3.re, o3.im);
        v3 = sp2{__ffma2_rn(u, H, e3.re), __ffma2_rn(s, NH, e3.im)};
        v7 = sp2{__ffma2_rn(u, NH, e3.re), __ffma2_rn(s, H, e3.im)};
    } else {
        // conj(w8) z = h ((zr - zi) + i (zr + zi)); conj(w8^3) z = h (-(zr + zi) + i (zr - zi))
        const float2 p = r_sub(o1.re, o1.im), q = r_add(o1.re, o1.im);
        v1 = sp2{__ffma2_rn(p, H, e1.re), __ffma2_rn(q, H, e1.im)};
        v5 = sp2{__ffma2_rn(p, NH, e1.re), __ffma2_rn(q, NH, e1.im)};
        const float2 s = r_add(o3.re, o3.im), u = r_sub(o3.re, o3.im);
        v3 = sp2{__ffma2_rn(s, NH, e3.re), __ffma2_rn(u, H, e3.im)};
        v7 = sp2{__ffma2_rn(s, H, e3.re), __ffma2_rn(u, NH, e3.im)};
    }
}

// z * w32^m (forward) or z * conj(w32^m) (inverse), both lanes.
template <bool INV>
__device__ __forceinline__ sp2 s_tw(sp2 z, int m)
{
    const float2 c = c_spc[m], s = c_sps[m], n = c_spn[m];
    if (!INV) return sp2{__ffma2_rn(z.re, c, __fmul2_rn(z.im, n)), __ffma2_rn(z.re, s, __fmul2_rn(z.im, c))};
    return sp2{__ffma2_rn(z.re, c, __fmul2_rn(z.im, s)), __ffma2_rn(z.re, n, __fmul2_rn(z.im, c))};
}

// Packed FFT-32 of both lanes.  In: sample n = 4 n1 + n2 in slot n.  Out:
// bin k = k1 + 8 k2 in slot 4 k1 + k2.
//   DFT-8 over n1 for each n2        -> A(n2, k1) in slot 4 k1 + n2
//   twiddle w32^(n2 k1)
//   DFT-4 over n2 for each k1        -> X(k1 + 8 k2) in slot 4 k1 + k2
__device__ __forceinline__ void s_fft32_fwd(sp2 (&P)[32])
{
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2)
        s_dft8<false>(P[n2], P[4 + n2], P[8 + n2], P[12 + n2], P[16 + n2], P[20 + n2], P[24 + n2], P[28 + n2]);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1)
#pragma unroll
        for (int n2 = 1; n2 < 4; ++n2) P[4 * k1 + n2] = s_tw<false>(P[4 * k1 + n2], n2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) s_dft4<false>(P[4 * k1], P[4 * k1 + 1], P[4 * k1 + 2], P[4 * k1 + 3]);
}

// Inverse of s_fft32_fwd (unnormalised): bins in its output slots, samples
// back in natural slots.
__device__ __forceinline__ void s_fft32_inv(sp2 (&P)[32])
{
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) s_dft4<true>(P[4 * k1], P[4 * k1 + 1], P[4 * k1 + 2], P[4 * k1 + 3]);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1)
#pragma unroll
        for (int n2 = 1; n2 < 4; ++n2) P[4 * k1 + n2] = s_tw<true>(P[4 * k1 + n2], n2 * k1);
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2)
        s_dft8<true>(P[n2], P[4 + n2], P[8 + n2], P[12 + n2], P[16 + n2], P[20 + n2], P[24 + n2], P[28 + n2]);
}

// Between the packed FFT-32s.  With E, O the 32-point spectra of the even and
// odd samples (lanes .x, .y of bin k's slot), t = w64^k and H the kernel's
// 64-point spectrum (1/64 folded in):
//   X[k] = E + t O,  X[k+32] = E - t O            (radix-2 join)
//   Y = H X                                        (spectrum multiply)
//   E' = Y[k] + Y[k+32],  O' = (Y[k] - Y[k+32]) conj(t)   (radix-2 split)
// i.e. E' = Hs E + Hd t O,  O' = Hs O + Hd conj(t) E  with Hs = H[k] + H[k+32],
// Hd = H[k] - H[k+32].  Per bin k the table holds
//   mt[2k] = (Hs, Hs, Hd C, Hd C),  mt[2k+1] = (Hd S, -Hd S, -Hd S, Hd S),
// t = C - i S.  The inverse FFT-32 of E' gives outputs 2m, of O' outputs 2m+1.
__device__ __forceinline__ void s_middle(sp2 (&P)[32], const float4 *mt)
{
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        sp2 &q = P[4 * (k & 7) + (k >> 3)];
        const float4 m0 = mt[2 * k], m1 = mt[2 * k + 1];
        const float2 A = make_float2(m0.x, m0.y), B = make_float2(m0.z, m0.w);
        const float2 D = make_float2(m1.x, m1.y), ND = make_float2(m1.z, m1.w);
        const float2 sre = make_float2(q.re.y, q.re.x), sim = make_float2(q.im.y, q.im.x);
        const float2 re = __ffma2_rn(sim, D, __ffma2_rn(sre, B, __fmul2_rn(q.re, A)));
        const float2 im = __ffma2_rn(sre, ND, __ffma2_rn(sim, B, __fmul2_rn(q.im, A)));
        q.re = re;
        q.im = im;
    }
}

// The middle table of a job from its spectrum HH (HH[k].x = H[k]) times
// `scale`; threads t, t + nthreads, ... of the CTA each fill bins.
__device__ __forceinline__ void s_fill_middle(float4 *mt, const float2 *HH, int t, int nthreads, float scale = 1.0f)
{
    for (int k = t; k < 32; k += nthreads) {
        const float a = scale * HH[k].x, b = scale * HH[k + 32].x;
        const float hs = a + b, hd = a - b;
        const float2 w = c_rfw64[k];  // (C, -S)
        const float dc = hd * w.x, ds = -hd * w.y;
        mt[2 * k] = make_float4(hs, hs, dc, dc);
        mt[2 * k + 1] = make_float4(ds, -ds, -ds, ds);
    }
}

// Sample i of a block (lane i & 1 of slot i / 2) as (line a, line b).
__device__ __forceinline__ float2 s_get(const sp2 (&P)[32], int i)
{
    return (i & 1) ? make_float2(P[i >> 1].re.y, P[i >> 1].im.y) : make_float2(P[i >> 1].re.x, P[i >> 1].im.x);
}
__device__ __forceinline__ void s_set(sp2 (&P)[32], int i, float2 v)
{
    if (i & 1) {
        P[i >> 1].re.y = v.x;
        P[i >> 1].im.y = v.y;
    } else {
        P[i >> 1].re.x = v.x;
        P[i >> 1].im.x = v.y;
    }
}

// ---------------------------------------------------------------------------
// y / z passes: one warp = one tile of 64 lines (32 pairs) of one outer index.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rf_prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

template <int R, int W, bool ZL>
__device__ __forceinline__ void rf_col_body(const OsJob &J, const OsTileInfo &T, int nreal, const float4 *mt,
                                            float (*held)[64])
{
    constexpr int L = 64 - 2 * R;
    const int lane = threadIdx.x & 31;
    const bool va = lane < nreal, vb = lane + 32 < nreal;
    const int n = J.n;
    const int64_t ps = J.pos_stride;
    // line a = tile line `lane`, line b = tile line `lane + 32`: lines are
    // adjacent (line stride 1), so b sits 128 bytes after a
    constexpr int lb = 32;
    float *const base = J.data + T.outer * J.outer_stride + (T.l0 + lane);
    constexpr bool zlast = ZL;
    const float keep = J.keep, b = J.b;
    const int nblocks = (n + 2 * R + L - 1) / L;
    // outputs of the pair at position pointer d
    auto put = [&](float *d, float va_, float vb_) {
        d[0] = va_;
        if (vb) d[lb] = vb_;
    };

    float2 lk = make_float2(0.0f, 0.0f), ot = lk;
    // W > 1: every warp of the CTA walks the same job, so all run nblocks
    // iterations and meet at one barrier per block (warps of an SM
    // sub-partition stay on the same instructions)
    for (int bi = 0; bi < nblocks; ++bi) {
        if (W > 1) __syncthreads();
        if (va) {
            const int c = -R + bi * L;  // first output of the block
            const int p0 = c - R;       // first input
            const bool inner = p0 >= 0 && p0 + 64 <= n;  // window and outputs inside the line
            float *const w0 = base + (int64_t)p0 * ps;
            sp2 P[32];
            {
                const float *sp = w0;
                if (inner) {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps) s_set(P, i, make_float2(sp[0], vb ? sp[lb] : 0.0f));
                } else {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps) {
                        const bool in = (unsigned)(p0 + i) < (unsigned)n;
                        s_set(P, i, make_float2(in ? sp[0] : 0.0f, (in && vb) ? sp[lb] : 0.0f));
                    }
                }
            }
            // the next block's new samples start for L2 while this one is
            // transformed: lane k covers bytes 8k .. 8k + 7 of the tile's 256
            if (bi + 1 < nblocks) {
                const int q0 = p0 + 64, q1 = min(p0 + L + 64, n);
                const float *pp = base + lane + (int64_t)q0 * ps;  // tile line 2 lane
                if (2 * lane < nreal)
                    for (int q = q0; q < q1; ++q, pp += ps) rf_prefetch_l2(pp);
            }
            // the previous block's held-back outputs: positions p0 .. p0 + R - 1,
            // just loaded above as this window's first inputs
            if (bi > 0) {
#pragma unroll
                for (int i = 0; i < R; ++i)
                    if ((unsigned)(p0 + i) < (unsigned)n) put(w0 + (int64_t)i * ps, held[i][lane], held[i][32 + lane]);
            }
            s_fft32_fwd(P);
            s_middle(P, mt);
            if (zlast) {
                // + keep b on every output: on the DC bins of both inverse FFT-32s
                // (keep itself is folded into the z pass's spectrum table)
                const float2 kb = make_float2(keep * b, keep * b);
                P[0].re = r_add(P[0].re, kb);
                P[0].im = r_add(P[0].im, kb);
            }
            s_fft32_inv(P);
            if (!inner) {
                // outputs past the line ends within the kernel's reach: the leak
#pragma unroll
                for (int i = R; i < R + L; ++i) {
                    const int o = c + i - R;
                    if (!((unsigned)o < (unsigned)n) && o >= -R && o < n + R) lk = r_add(lk, s_get(P, i));
                }
            }
            if (zlast && inner) {
                // FP32 total of the kept outputs (lane .x: sample 2j, .y: 2j + 1)
                float2 sa = make_float2(0.0f, 0.0f), sb = sa;
#pragma unroll
                for (int j = R / 2; j <= (R + L - 1) / 2; ++j) {
                    const int i0 = 2 * j, i1 = 2 * j + 1;
                    const bool k0 = i0 >= R && i0 < R + L, k1 = i1 >= R && i1 < R + L;
                    const float2 ra = P[j].re, rb = P[j].im;
                    sa = r_add(sa, make_float2(k0 ? ra.x : 0.0f, k1 ? ra.y : 0.0f));
                    sb = r_add(sb, make_float2(k0 ? rb.x : 0.0f, k1 ? rb.y : 0.0f));
                }
                ot = r_add(ot, make_float2(sa.x + sa.y, sb.x + sb.y));
            }
            float *d = w0 + (int64_t)R * ps;  // position of sample R = first output c
            if (inner) {
#pragma unroll
                for (int i = R; i < R + L; ++i, d += ps) {
                    const float2 v = s_get(P, i);
                    if (i >= L) {  // stored after the next block's loads
                        held[i - L][lane] = v.x;
                        held[i - L][32 + lane] = v.y;
                    } else {
                        put(d, v.x, v.y);
                    }
                }
            } else {
#pragma unroll
                for (int i = R; i < R + L; ++i, d += ps) {
                    const int o = c + i - R;
                    if ((unsigned)o < (unsigned)n) {
                        const float2 v = s_get(P, i);
                        if (zlast) ot = r_add(ot, v);
                        if (i >= L) {
                            held[i - L][lane] = v.x;
                            held[i - L][32 + lane] = v.y;
                        } else {
                            put(d, v.x, v.y);
                        }
                    }
                }
            }
        }
    }
    if (va) {
        // the last block's held-back outputs
        const int clast = -R + (nblocks - 1) * L;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int o = clast + L - R + i;
            if ((unsigned)o < (unsigned)n) put(base + (int64_t)o * ps, held[i][lane], held[i][32 + lane]);
        }
    }
    double *mass = J.mass;
    double s_lk = r_warp_sum((double)(va ? lk.x : 0.0f) + (double)(vb ? lk.y : 0.0f));
    if (!zlast) {
        if (lane == 0 && s_lk != 0.0) atomicAdd(mass + MS_LEAK_Y, s_lk);
    } else {
        // z outputs are keep (v + b): n kept and 2r leaked per line give back
        // the convolution's kept total (cv) and leak
        const double s_ot = r_warp_sum((double)(va ? ot.x : 0.0f) + (double)(vb ? ot.y : 0.0f));
        const double lines = (double)min(max(nreal, 0), 64);
        const double s_cv = s_ot / (double)keep - (double)b * n * lines;
        s_lk = s_lk / (double)keep - (double)b * (2 * R) * lines;
        if (lane == 0) {
            if (s_lk != 0.0) atomicAdd(mass + MS_LEAK_Z, s_lk);
            if (s_cv != 0.0) atomicAdd(mass + MS_CONV, s_cv);
            if (s_ot != 0.0) atomicAdd(mass + MS_OUT, s_ot);
        }
    }
}

// One launch covers tiles of every radius: the CTA's job picks the variant.
// A CTA of W warps takes W consecutive tiles, all of one job (the host pads
// each job's tiles to a multiple of W with empty ones); a tile of another
// job than the CTA's first is treated as empty, so every warp runs the same
// number of blocks and barriers.
// ZL: the z pass (decay, baseline and the output totals applied).
template <int W, bool ZL>
__global__ void __launch_bounds__(32 * W, 12 / W) rf_col_kernel(const OsJob *__restrict__ jobs,
                                                                const OsTileInfo *__restrict__ tiles)
{
    __shared__ __align__(16) float4 mt[64];
    __shared__ float held[W][RF_RMAX][64];  // held-back outputs [warp][i][line]
    const int warp = threadIdx.x >> 5;
    const int job = tiles[(size_t)blockIdx.x * W].job;
    const OsTileInfo T = tiles[(size_t)blockIdx.x * W + warp];
    const int nreal = T.job == job ? (T.flags & 255) : 0;
    const OsJob &J = jobs[job];
    s_fill_middle(mt, J.HH, threadIdx.x, 32 * W, ZL ? J.keep : 1.0f);
    if (W > 1) __syncthreads();
    else __syncwarp();
    switch (J.r) {
    case 1: rf_col_body<1, W, ZL>(J, T, nreal, mt, held[warp]); break;
    case 2: rf_col_body<2, W, ZL>(J, T, nreal, mt, held[warp]); break;
    case 3: rf_col_body<3, W, ZL>(J, T, nreal, mt, held[warp]); break;
    case 4: rf_col_body<4, W, ZL>(J, T, nreal, mt, held[warp]); break;
    case 5: rf_col_body<5, W, ZL>(J, T, nreal, mt, held[warp]); break;
    case 6: rf_col_body<6, W, ZL>(J, T, nreal, mt, held[warp]); break;
    case 7: rf_col_body<7, W, ZL>(J, T, nreal, mt, held[warp]); break;
    default: rf_col_body<8, W, ZL>(J, T, nreal, mt, held[warp]); break;
    }
}

// ---------------------------------------------------------------------------
// y / z passes with TMA staging.  Same blocks, same FFT; what changes is how
// a block's window reaches the registers: each warp owns a 64 x 64 float
// window buffer in shared memory (positions x lines, 16 KB) and an mbarrier.
// Lane 0 issues one 3D bulk tensor copy per window (the field seen as the
// tensor {nx, ny, nz}; box {64 lines, 64 positions} along y or z); the
// hardware fills positions outside the line with zeros, so loads need no
// range tests.  Per block:
//   wait for window b; every lane reads its pair's 64 samples (conflict-free
//   4-byte reads: lane k reads columns k and k + 32); lane 0 issues the copy
//   of window b + 1 into the same buffer; FFT, multiply, inverse FFT;
//   outputs [c, c + L - r) go straight to global memory; the last r outputs
//   -- positions that window b + 1 reads -- are stored once that copy has
//   landed (it was in flight during the transform).
// The waits are bounded (kTmaWaitCycles): a wait that gives up sets
// g_rf_timeout and the warp stops.
// ---------------------------------------------------------------------------
template <int R, bool ZL>
__device__ __forceinline__ void rf_col_tma_body(const OsJob &J, const CUtensorMap *map, const OsTileInfo &T,
                                                int nreal, const float4 *mt, float *win, uint64_t *bar)
{
    constexpr int L = 64 - 2 * R;
    const int lane = threadIdx.x & 31;
    const bool va = lane < nreal, vb = lane + 32 < nreal;
    const int n = J.n;
    const int64_t ps = J.pos_stride;
    constexpr int lb = 32;
    float *const base = J.data + T.outer * J.outer_stride + (T.l0 + lane);
    const float keep = J.keep, b = J.b;
    const int nblocks = (n + 2 * R + L - 1) / L;
    auto put = [&](float *d, float va_, float vb_) {
        d[0] = va_;
        if (vb) d[lb] = vb_;
    };
    // window of block bi: positions [-2R + bi L, -2R + bi L + 64) of lines [l0, l0 + 64)
    auto issue = [&](int bi) {
        const int p0 = -2 * R + bi * L;
        mbar_arrive_expect_tx(bar, 64 * 64 * 4);
        if (ZL) tma_load_3d(win, map, T.l0, T.outer, p0, bar);
        else tma_load_3d(win, map, T.l0, p0, T.outer, bar);
    };
    if (lane == 0) issue(0);
    float2 lk = make_float2(0.0f, 0.0f), ot = lk;
    int issued = 0;  // last window issued
    bool ok = true;
    for (int bi = 0; bi < nblocks && ok; ++bi) {
        // warp-uniform outcome: a lane whose wait gave up stops the whole warp
        if (!__all_sync(0xffffffffu, mbar_wait(bar, bi & 1))) {
            ok = false;
            break;
        }
        const int c = -R + bi * L;  // first output of the block
        const int p0 = c - R;       // first input
        const bool inner = p0 >= 0 && p0 + 64 <= n;
        sp2 P[32];
#pragma unroll
        for (int i = 0; i < 64; ++i) s_set(P, i, make_float2(win[i * 64 + lane], win[i * 64 + 32 + lane]));
        __syncwarp();
        const bool more = bi + 1 < nblocks;
        if (more && lane == 0) {
            fence_proxy_async_smem();  // the reads above before the copy overwrites the buffer
            issue(bi + 1);
        }
        if (more) issued = bi + 1;
        s_fft32_fwd(P);
        s_middle(P, mt);
        if (ZL) {
            const float2 kb = make_float2(keep * b, keep * b);
            P[0].re = r_add(P[0].re, kb);
            P[0].im = r_add(P[0].im, kb);
        }
        s_fft32_inv(P);
        if (!inner) {
#pragma unroll
            for (int i = R; i < R + L; ++i) {
                const int o = c + i - R;
                if (!((unsigned)o < (unsigned)n) && o >= -R && o < n + R) lk = r_add(lk, s_get(P, i));
            }
        }
        if (ZL && inner) {
            float2 sa = make_float2(0.0f, 0.0f), sb = sa;
#pragma unroll
            for (int j = R / 2; j <= (R + L - 1) / 2; ++j) {
                const int i0 = 2 * j, i1 = 2 * j + 1;
                const bool k0 = i0 >= R && i0 < R + L, k1 = i1 >= R && i1 < R + L;
                const float2 ra = P[j].re, rb = P[j].im;
                sa = r_add(sa, make_float2(k0 ? ra.x : 0.0f, k1 ? ra.y : 0.0f));
                sb = r_add(sb, make_float2(k0 ? rb.x : 0.0f, k1 ? rb.y : 0.0f));
            }
            ot = r_add(ot, make_float2(sa.x + sa.y, sb.x + sb.y));
        }
        float *d = base + (int64_t)(p0 + R) * ps;  // position of sample R = first output c
        // samples [R, L): positions no later window reads
        if (va) {
            if (inner) {
#pragma unroll
                for (int i = R; i < L; ++i, d += ps) {
                    const float2 v = s_get(P, i);
                    put(d, v.x, v.y);
                }
            } else {
#pragma unroll
                for (int i = R; i < L; ++i, d += ps) {
                    const int o = c + i - R;
                    if ((unsigned)o < (unsigned)n) {
                        const float2 v = s_get(P, i);
                        if (ZL) ot = r_add(ot, v);
                        put(d, v.x, v.y);
                    }
                }
            }
        }
        // samples [L, L + R): positions window bi + 1 reads; store after it landed
        if (more && !__all_sync(0xffffffffu, mbar_wait(bar, (bi + 1) & 1))) {
            ok = false;
            break;
        }
        if (va) {
#pragma unroll
            for (int i = L; i < L + R; ++i, d += ps) {
                const int o = c + i - R;
                if (inner || (unsigned)o < (unsigned)n) {
                    const float2 v = s_get(P, i);
                    if (ZL && !inner) ot = r_add(ot, v);
                    put(d, v.x, v.y);
                }
            }
        }
    }
    if (!ok) {
        if (lane == 0) atomicExch(&g_rf_timeout, 1);
        mbar_wait(bar, issued & 1);  // bounded: the copy still in flight, if any
        return;
    }
    double *mass = J.mass;
    double s_lk = r_warp_sum((double)(va ? lk.x : 0.0f) + (double)(vb ? lk.y : 0.0f));
    if (!ZL) {
        if (lane == 0 && s_lk != 0.0) atomicAdd(mass + MS_LEAK_Y, s_lk);
    } else {
        const double s_ot = r_warp_sum((double)(va ? ot.x : 0.0f) + (double)(vb ? ot.y : 0.0f));
        const double lines = (double)min(max(nreal, 0), 64);
        const double s_cv = s_ot / (double)keep - (double)b * n * lines;
        s_lk = s_lk / (double)keep - (double)b * (2 * R) * lines;
        if (lane == 0) {
            if (s_lk != 0.0) atomicAdd(mass + MS_LEAK_Z, s_lk);
            if (s_cv != 0.0) atomicAdd(mass + MS_CONV, s_cv);
            if (s_ot != 0.0) atomicAdd(mass + MS_OUT, s_ot);
        }
    }
}

constexpr int RF_WIN_FLOATS = 64 * 64;  // one warp's window buffer

// W warps per CTA, each on its own tile (tiles of other jobs than the CTA's
// first are empty, as in rf_col_kernel); no CTA barrier after set-up.
template <int W, bool ZL, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) rf_col_tma_kernel(const OsJob *__restrict__ jobs,
                                                                    const CUtensorMap *__restrict__ maps,
                                                                    const OsTileInfo *__restrict__ tiles)
{
    extern __shared__ __align__(16) unsigned char rf_dyn[];
    __shared__ __align__(16) float4 mt[64];
    __shared__ __align__(8) uint64_t bars[W];
    const int warp = threadIdx.x >> 5;
    const int job = tiles[(size_t)blockIdx.x * W].job;
    const OsTileInfo T = tiles[(size_t)blockIdx.x * W + warp];
    const int nreal = T.job == job ? (T.flags & 255) : 0;
    const OsJob &J = jobs[job];
    if (threadIdx.x < W) mbar_init(&bars[threadIdx.x], 1);
    if (threadIdx.x < W) mbar_fence_init();
    s_fill_middle(mt, J.HH, threadIdx.x, 32 * W, ZL ? J.keep : 1.0f);
    __syncthreads();
    if (nreal == 0) return;
    // window buffers on a 1024-byte boundary (the launch adds 1 KB of slack)
    const uint32_t s0 = smem_u32(rf_dyn);
    float *win = reinterpret_cast<float *>(rf_dyn + (((s0 + 1023u) & ~1023u) - s0)) + warp * RF_WIN_FLOATS;
    const CUtensorMap *map = maps + job;
    switch (J.r) {
    case 1: rf_col_tma_body<1, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    case 2: rf_col_tma_body<2, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    case 3: rf_col_tma_body<3, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    case 4: rf_col_tma_body<4, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    case 5: rf_col_tma_body<5, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    case 6: rf_col_tma_body<6, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    case 7: rf_col_tma_body<7, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    default: rf_col_tma_body<8, ZL>(J, map, T, nreal, mt, win, &bars[warp]); break;
    }
}

// ---------------------------------------------------------------------------
// x pass: one warp = 64 rows (32 pairs).  Rows hold positions contiguously,
// so blocks are moved through a shared tile with 16-byte copies:
//   * chunks start on multiples of 4: the first output is -Rh (Rh = r
//     rounded up to 4) and blocks keep L4 outputs (L4 = L rounded down to a
//     multiple of 4); a block's window is the 68 positions from c - Rh;
//   * the FFT input starts e = (Rh - r) & ~1 positions into the window (an
//     even offset, so 16-byte reads of a row land whole slots), which puts
//     the first output in sample R2 = Rh - e (r or r + 1; L4 <= L - 2 when
//     r is odd keeps the last output at most 63 - r);
//   * tile rows are 68 floats; line row 2q sits in tile row q and row 2q+1
//     in tile row 32 + q, so a warp's 16-byte column reads (lane = pair) fall
//     on distinct bank quads (68 floats = 272 bytes = 16 mod 128);
//   * the last Rh outputs of a block are the first Rh positions of the next
//     window: they are held back and stored after that window has landed.
// Needs rows 16-byte aligned and n a multiple of 4.
// ---------------------------------------------------------------------------
constexpr int RF_TS = 68;  // floats per tile row (17 chunks of 4)

__device__ __forceinline__ void rf_cp16(float *smem, const float *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0)
                 : "memory");
}

__device__ __forceinline__ int rf_trow(int row) { return (row & 1) * 32 + (row >> 1); }

template <int R>
__device__ __forceinline__ void rf_row_body(const OsJob &J, const OsTileInfo &T, const float4 *mt, float *A,
                                            float *held)
{
    constexpr int L = 64 - 2 * R;
    constexpr int L4 = L & ~3;          // outputs kept per block
    constexpr int RH = (R + 3) & ~3;    // held-back outputs per block (multiple of 4)
    constexpr int E = (RH - R) & ~1;    // FFT input offset in the window (even)
    constexpr int R2 = RH - E;          // sample of the first output (even)
    constexpr int NST = (L4 - RH) / 4;  // chunks stored at once per row
    constexpr int NHD = RH / 4;         // held chunks per row
    static_assert(R2 % 2 == 0 && R2 >= R && R2 + L4 - 1 + R <= 63, "x-pass block geometry");
    const int lane = threadIdx.x;
    const int nreal = T.flags & 255;
    const int n = J.n;
    const int64_t ls = J.line_stride;
    float *const base = J.data + (int64_t)T.l0 * ls;
    const float b = J.b;
    const bool masked = J.mask != 0;
    bool in_a = 2 * lane < nreal, in_b = 2 * lane + 1 < nreal;
    const bool va = in_a, vb = in_b;
    int xlo = 0, xhi = n;
    if (masked) {
        xlo = J.box_lo[0];
        xhi = J.box_hi[0];
        if (va) {
            const int rr = T.l0 + 2 * lane, y = rr % J.ny, z = rr / J.ny;
            in_a = y >= J.box_lo[1] && y < J.box_hi[1] && z >= J.box_lo[2] && z < J.box_hi[2];
        }
        if (vb) {
            const int rr = T.l0 + 2 * lane + 1, y = rr % J.ny, z = rr / J.ny;
            in_b = y >= J.box_lo[1] && y < J.box_hi[1] && z >= J.box_lo[2] && z < J.box_hi[2];
        }
    }
    const int nblocks = (n + R + RH + L4 - 1) / L4;
    const int hw = lane >> 4, cq = lane & 15;  // half-warp, 16-byte chunk
    float *const rowp = base + (int64_t)hw * ls;  // row hw of the tile
    static_assert(NST <= 16, "one chunk per lane of a half-warp");
    // stores the held-back outputs (positions pa .. pa + RH - 1) of every row
    auto put_held = [&](int pa) {
        for (int k = lane; k < nreal * NHD; k += 32) {
            const int row = k / NHD, cc = k - row * NHD;
            const int o = pa + 4 * cc;
            if ((unsigned)o < (unsigned)n)
                *reinterpret_cast<float4 *>(base + (int64_t)row * ls + o) =
                    *reinterpret_cast<const float4 *>(held + row * RH + 4 * cc);
        }
    };

    double acc_in = 0.0;
    float2 lk = make_float2(0.0f, 0.0f);
    for (int bi = 0; bi < nblocks; ++bi) {
        const int c = -RH + bi * L4;  // first output, a multiple of 4
        const int pa = c - RH;        // window start, a multiple of 4
        // ---- window [pa, pa + 64 + e) of every row, 16-byte chunks -----------
        // half-warp h copies chunk `cq` of rows h, h + 2, ...: row 2t + h lands
        // in tile row 32 h + t (a chunk lies wholly inside or outside the line)
        {
            const int p = pa + 4 * cq;
            const bool v = (unsigned)p < (unsigned)n;
            const float *src = rowp + (v ? p : 0);
            float *dst = A + (32 * hw) * RF_TS + 4 * cq;
            for (int r = hw; r < nreal; r += 2, src += 2 * ls, dst += RF_TS) rf_cp16(dst, src, v);
            if (E > 0) {  // chunk 16: positions pa + 64 .. pa + 67
                const int p16 = pa + 64;
                const bool v16 = (unsigned)p16 < (unsigned)n;
                for (int r = lane; r < nreal; r += 32) {
                    const float *s16 = base + (int64_t)r * ls;
                    rf_cp16(A + rf_trow(r) * RF_TS + 64, v16 ? s16 + p16 : s16, v16);
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncwarp();
        // the previous block's held-back outputs are this window's first RH positions
        if (bi > 0) put_held(pa);
        // ---- this lane's pair: slots from 16-byte reads of its two rows ---------
        sp2 P[32];
        {
            const float4 *ra = reinterpret_cast<const float4 *>(A + lane * RF_TS);
            const float4 *rb = reinterpret_cast<const float4 *>(A + (32 + lane) * RF_TS);
#pragma unroll
            for (int m = 0; m < 17; ++m) {
                const int j0 = (4 * m - E) / 2;  // slot of the chunk's first two positions
                if (j0 + 1 < 0 || j0 >= 32) continue;
                const float4 u = ra[m], w = rb[m];
                if (j0 >= 0) P[j0] = sp2{make_float2(u.x, u.y), make_float2(w.x, w.y)};
                if (j0 + 1 < 32) P[j0 + 1] = sp2{make_float2(u.z, u.w), make_float2(w.z, w.w)};
            }
        }
        __syncwarp();  // every lane has its columns: the tile is free for outputs
        if (!vb) {
            // tile rows past the tile's lines hold stale data: zero the pair's missing line
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                P[j].im = make_float2(0.0f, 0.0f);
                if (!va) P[j].re = make_float2(0.0f, 0.0f);
            }
        }
        if (masked) {
#pragma unroll
            for (int i = 0; i < 64; ++i) {
                const int p = c - R2 + i;
                const bool px = p >= xlo && p < xhi;
                float2 v = s_get(P, i);
                v.x = (in_a && px) ? v.x - b : 0.0f;
                v.y = (in_b && px) ? v.y - b : 0.0f;
                s_set(P, i, v);
            }
        }
        {
            // input mass: the block outputs' positions (slots R2 / 2 .. (R2 + L4) / 2)
            float2 sa = make_float2(0.0f, 0.0f), sb = sa;
#pragma unroll
            for (int j = R2 / 2; j < (R2 + L4) / 2; ++j) {
                sa = r_add(sa, P[j].re);
                sb = r_add(sb, P[j].im);
            }
            acc_in += (double)(va ? sa.x + sa.y : 0.0f) + (double)(vb ? sb.x + sb.y : 0.0f);
        }
        s_fft32_fwd(P);
        s_middle(P, mt);
        s_fft32_inv(P);
#pragma unroll
        for (int i = R2; i < R2 + L4; ++i) {
            const int o = c + i - R2;
            if (!((unsigned)o < (unsigned)n) && o >= -R && o < n + R) lk = r_add(lk, s_get(P, i));
        }
        {
            float4 *wa = reinterpret_cast<float4 *>(A + lane * RF_TS);
            float4 *wb = reinterpret_cast<float4 *>(A + (32 + lane) * RF_TS);
#pragma unroll
            for (int m = 0; m < L4 / 4; ++m) {
                const int j = R2 / 2 + 2 * m;
                wa[m] = make_float4(P[j].re.x, P[j].re.y, P[j + 1].re.x, P[j + 1].re.y);
                wb[m] = make_float4(P[j].im.x, P[j].im.y, P[j + 1].im.x, P[j + 1].im.y);
            }
        }
        __syncwarp();
        // ---- outputs [c, c + L4 - RH) of every row; the rest is held back ------
        {
            const int o = c + 4 * cq;
            if (cq < NST && (unsigned)o < (unsigned)n) {
                float *dst = rowp + o;
                const float *src = A + (32 * hw) * RF_TS + 4 * cq;
                for (int r = hw; r < nreal; r += 2, dst += 2 * ls, src += RF_TS)
                    *reinterpret_cast<float4 *>(dst) = *reinterpret_cast<const float4 *>(src);
            }
        }
        for (int k = lane; k < nreal * NHD; k += 32) {
            const int row = k / NHD, cc = k - row * NHD;
            *reinterpret_cast<float4 *>(held + row * RH + 4 * cc) =
                *reinterpret_cast<const float4 *>(A + rf_trow(row) * RF_TS + (L4 - RH) + 4 * cc);
        }
        __syncwarp();  // the tile is refilled by the next block
    }
    put_held(-RH + (nblocks - 1) * L4 + L4 - RH);
    double *mass = J.mass;
    const double s_in = r_warp_sum(acc_in);
    const double s_lk = r_warp_sum((double)(va ? lk.x : 0.0f) + (double)(vb ? lk.y : 0.0f));
    if (lane == 0) {
        if (s_in != 0.0) atomicAdd(mass + MS_INPUT, s_in);
        if (s_lk != 0.0) atomicAdd(mass + MS_LEAK_X, s_lk);
    }
}

__global__ void __launch_bounds__(32, 12) rf_row_kernel(const OsJob *__restrict__ jobs,
                                                        const OsTileInfo *__restrict__ tiles)
{
    __shared__ __align__(16) float A[64 * RF_TS];
    __shared__ __align__(16) float held[64 * 8];  // held-back outputs [row][RH]
    __shared__ __align__(16) float4 mt[64];
    const OsTileInfo T = tiles[blockIdx.x];
    const OsJob &J = jobs[T.job];
    s_fill_middle(mt, J.HH, threadIdx.x, 32);
    __syncwarp();
    switch (J.r) {
    case 1: rf_row_body<1>(J, T, mt, A, held); break;
    case 2: rf_row_body<2>(J, T, mt, A, held); break;
    case 3: rf_row_body<3>(J, T, mt, A, held); break;
    case 4: rf_row_body<4>(J, T, mt, A, held); break;
    case 5: rf_row_body<5>(J, T, mt, A, held); break;
    case 6: rf_row_body<6>(J, T, mt, A, held); break;
    case 7: rf_row_body<7>(J, T, mt, A, held); break;
    default: rf_row_body<8>(J, T, mt, A, held); break;
    }
}


// ---------------------------------------------------------------------------
// x pass with TMA staging.  Same blocks, tiles and register layout as
// rf_row_body; the window of every block arrives by two 3D bulk tensor
// copies (the field's rows seen as two tensors {nx, rows / 2} with row
// stride 2 nx: even rows land in tile rows 0..31, odd rows in 32..63, the
// conflict-free layout of rf_trow), one block ahead, into a per-warp input
// tile.  Outputs go to global memory through a per-warp 32-row output tile,
// even rows then odd rows, as coalesced 16-byte stores; they are stored once
// the next window has landed, because its first Rh positions are this
// block's last outputs.  26 KB of shared memory per warp: 8 warps per SM.
// ---------------------------------------------------------------------------
constexpr int RF_XTILE_FLOATS = 64 * RF_TS;        // the 64-row input tile
constexpr int RF_XOUT_FLOATS = 32 * RF_TS;         // the 32-row output tile
constexpr int RF_XWARP_BYTES = 26 * 1024;          // per-warp stride (input + output tiles, 1 KB aligned)
static_assert((RF_XTILE_FLOATS + RF_XOUT_FLOATS) * 4 <= RF_XWARP_BYTES, "x-pass tiles");

template <int R>
__device__ __forceinline__ void rf_row_tma_body(const OsJob &J, const CUtensorMap *maps, const OsTileInfo &T,
                                                const float4 *mt, float *IN, float *OUT, uint64_t *bar)
{
    constexpr int L = 64 - 2 * R;
    constexpr int L4 = L & ~3;
    constexpr int RH = (R + 3) & ~3;
    constexpr int E = (RH - R) & ~1;
    constexpr int R2 = RH - E;
    static_assert(R2 % 2 == 0 && R2 >= R && R2 + L4 - 1 + R <= 63, "x-pass block geometry");
    static_assert(L4 / 4 <= 16, "one chunk per lane of a half-warp");
    const int lane = threadIdx.x & 31;
    const int nreal = T.flags & 255;
    const int n = J.n;
    const int64_t ls = J.line_stride;
    float *const base = J.data + (int64_t)T.l0 * ls;
    const float b = J.b;
    const bool masked = J.mask != 0;
    bool in_a = 2 * lane < nreal, in_b = 2 * lane + 1 < nreal;
    const bool va = in_a, vb = in_b;
    int xlo = 0, xhi = n;
    if (masked) {
        xlo = J.box_lo[0];
        xhi = J.box_hi[0];
        if (va) {
            const int rr = T.l0 + 2 * lane, y = rr % J.ny, z = rr / J.ny;
            in_a = y >= J.box_lo[1] && y < J.box_hi[1] && z >= J.box_lo[2] && z < J.box_hi[2];
        }
        if (vb) {
            const int rr = T.l0 + 2 * lane + 1, y = rr % J.ny, z = rr / J.ny;
            in_b = y >= J.box_lo[1] && y < J.box_hi[1] && z >= J.box_lo[2] && z < J.box_hi[2];
        }
    }
    const int nblocks = (n + R + RH + L4 - 1) / L4;
    const int hw = lane >> 4, cq = lane & 15;
    const int pair0 = T.l0 >> 1;  // first row pair of the tile
    // window of block bi: positions [pa, pa + 68), pa = -2 Rh + bi L4 (a multiple of 4)
    auto issue = [&](int bi) {
        const int pa = -2 * RH + bi * L4;
        mbar_arrive_expect_tx(bar, 64 * RF_TS * 4);
        tma_load_3d(IN, maps, pa, pair0, 0, bar);                  // even rows
        tma_load_3d(IN + 32 * RF_TS, maps + 1, pa, pair0, 0, bar);  // odd rows
    };
    // stores the block's outputs of the rows of parity `par` (tile row t =
    // line row 2t + par) from the output tile: half-warp hw takes t = hw,
    // hw + 2, ..., lane cq the 16-byte chunk cq of each
    auto store_rows = [&](int c, int par) {
        const int o = c + 4 * cq;
        if (cq < L4 / 4 && (unsigned)o < (unsigned)n) {
            float *dst = base + (int64_t)(2 * hw + par) * ls + o;
            const float *src = OUT + hw * RF_TS + 4 * cq;
            for (int t = hw; 2 * t + par < nreal; t += 2, dst += 4 * ls, src += 2 * RF_TS)
                *reinterpret_cast<float4 *>(dst) = *reinterpret_cast<const float4 *>(src);
        }
    };
    if (lane == 0) issue(0);
    double acc_in = 0.0;
    float2 lk = make_float2(0.0f, 0.0f);
    int issued = 0;
    bool ok = true;
    for (int bi = 0; bi < nblocks; ++bi) {
        const int c = -RH + bi * L4;  // first output, a multiple of 4
        if (!__all_sync(0xffffffffu, mbar_wait(bar, bi & 1))) {
            ok = false;
            break;
        }
        sp2 P[32];
        {
            const float4 *ra = reinterpret_cast<const float4 *>(IN + lane * RF_TS);
            const float4 *rb = reinterpret_cast<const float4 *>(IN + (32 + lane) * RF_TS);
#pragma unroll
            for (int m = 0; m < 17; ++m) {
                const int j0 = (4 * m - E) / 2;
                if (j0 + 1 < 0 || j0 >= 32) continue;
                const float4 u = ra[m], w = rb[m];
                if (j0 >= 0) P[j0] = sp2{make_float2(u.x, u.y), make_float2(w.x, w.y)};
                if (j0 + 1 < 32) P[j0 + 1] = sp2{make_float2(u.z, u.w), make_float2(w.z, w.w)};
            }
        }
        __syncwarp();
        const bool more = bi + 1 < nblocks;
        if (more && lane == 0) {
            fence_proxy_async_smem();
            issue(bi + 1);
        }
        if (more) issued = bi + 1;
        if (!vb) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                P[j].im = make_float2(0.0f, 0.0f);
                if (!va) P[j].re = make_float2(0.0f, 0.0f);
            }
        }
        if (masked) {
#pragma unroll
            for (int i = 0; i < 64; ++i) {
                const int p = c - R2 + i;
                const bool px = p >= xlo && p < xhi;
                float2 v = s_get(P, i);
                v.x = (in_a && px) ? v.x - b : 0.0f;
                v.y = (in_b && px) ? v.y - b : 0.0f;
                s_set(P, i, v);
            }
        }
        {
            float2 sa = make_float2(0.0f, 0.0f), sb = sa;
#pragma unroll
            for (int j = R2 / 2; j < (R2 + L4) / 2; ++j) {
                sa = r_add(sa, P[j].re);
                sb = r_add(sb, P[j].im);
            }
            acc_in += (double)(va ? sa.x + sa.y : 0.0f) + (double)(vb ? sb.x + sb.y : 0.0f);
        }
        s_fft32_fwd(P);
        s_middle(P, mt);
        s_fft32_inv(P);
#pragma unroll
        for (int i = R2; i < R2 + L4; ++i) {
            const int o = c + i - R2;
            if (!((unsigned)o < (unsigned)n) && o >= -R && o < n + R) lk = r_add(lk, s_get(P, i));
        }
        // the next window holds this block's last Rh outputs' positions
        if (more && !__all_sync(0xffffffffu, mbar_wait(bar, (bi + 1) & 1))) {
            ok = false;
            break;
        }
        {
            float4 *wa = reinterpret_cast<float4 *>(OUT + lane * RF_TS);
#pragma unroll
            for (int m = 0; m < L4 / 4; ++m) {
                const int j = R2 / 2 + 2 * m;
                wa[m] = make_float4(P[j].re.x, P[j].re.y, P[j + 1].re.x, P[j + 1].re.y);
            }
        }
        __syncwarp();
        store_rows(c, 0);
        __syncwarp();
        {
            float4 *wb = reinterpret_cast<float4 *>(OUT + lane * RF_TS);
#pragma unroll
            for (int m = 0; m < L4 / 4; ++m) {
                const int j = R2 / 2 + 2 * m;
                wb[m] = make_float4(P[j].im.x, P[j].im.y, P[j + 1].im.x, P[j + 1].im.y);
            }
        }
        __syncwarp();
        store_rows(c, 1);
        __syncwarp();  // the output tile is rewritten by the next block
    }
    if (!ok) {
        if (lane == 0) atomicExch(&g_rf_timeout, 1);
        mbar_wait(bar, issued & 1);
        return;
    }
    double *mass = J.mass;
    const double s_in = r_warp_sum(acc_in);
    const double s_lk = r_warp_sum((double)(va ? lk.x : 0.0f) + (double)(vb ? lk.y : 0.0f));
    if (lane == 0) {
        if (s_in != 0.0) atomicAdd(mass + MS_INPUT, s_in);
        if (s_lk != 0.0) atomicAdd(mass + MS_LEAK_X, s_lk);
    }
}

// W warps per CTA, each on its own 64-row tile (tiles of other jobs than the
// CTA's first are empty); maps: two per job (even rows, odd rows).
template <int W>
__global__ void __launch_bounds__(32 * W, 8 / W) rf_row_tma_kernel(const OsJob *__restrict__ jobs,
                                                                   const CUtensorMap *__restrict__ maps,
                                                                   const OsTileInfo *__restrict__ tiles)
{
    extern __shared__ __align__(16) unsigned char rf_dyn[];
    __shared__ __align__(16) float4 mt[64];
    __shared__ __align__(8) uint64_t bars[W];
    const int warp = threadIdx.x >> 5;
    const int job = tiles[(size_t)blockIdx.x * W].job;
    const OsTileInfo T = tiles[(size_t)blockIdx.x * W + warp];
    const bool real = T.job == job && (T.flags & 255) > 0;
    const OsJob &J = jobs[job];
    if (threadIdx.x < W) mbar_init(&bars[threadIdx.x], 1);
    if (threadIdx.x < W) mbar_fence_init();
    s_fill_middle(mt, J.HH, threadIdx.x, 32 * W);
    __syncthreads();
    if (!real) return;
    const uint32_t s0 = smem_u32(rf_dyn);
    float *IN = reinterpret_cast<float *>(rf_dyn + (((s0 + 1023u) & ~1023u) - s0) + warp * RF_XWARP_BYTES);
    float *OUT = IN + RF_XTILE_FLOATS;
    const CUtensorMap *m = maps + 2 * job;
    switch (J.r) {
    case 1: rf_row_tma_body<1>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    case 2: rf_row_tma_body<2>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    case 3: rf_row_tma_body<3>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    case 4: rf_row_tma_body<4>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    case 5: rf_row_tma_body<5>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    case 6: rf_row_tma_body<6>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    case 7: rf_row_tma_body<7>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    default: rf_row_tma_body<8>(J, m, T, mt, IN, OUT, &bars[warp]); break;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
static bool rf_row_enabled();

bool rf_eligible(const OsJob &j)
{
    if (j.r < 1 || j.r > RF_RMAX) return false;
    if (j.kind == PASS_X)
        return rf_row_enabled() && (j.n & 3) == 0 && (j.line_stride & 3) == 0 &&
               (reinterpret_cast<uintptr_t>(j.data) & 15) == 0;
    return j.line_stride == 1;
}

void rf_append_tiles(const OsJob &j, int job, std::vector<OsTileInfo> &out)
{
    const int tpo = (j.nlines + RF_LINES - 1) / RF_LINES;
    for (int outer = 0; outer < j.nouter; ++outer)
        for (int lt = 0; lt < tpo; ++lt) {
            OsTileInfo ti;
            ti.job = job;
            ti.outer = outer;
            ti.l0 = lt * RF_LINES;
            ti.flags = std::min(RF_LINES, j.nlines - ti.l0);  // real lines
            out.push_back(ti);
        }
}

// VFD_RF_X=0 keeps the x pass on the overlap-save kernel.
static bool rf_row_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_RF_X");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1;
}

// Warps per CTA of the y/z kernel (VFD_RF_W: 1, 2, 4, 6 or 12; default 4:
// on B200 the 512x256x384 world's y and z passes took 0.737 / 0.761 ms with
// 4, 0.766 / 0.794 with 1, 0.768 / 0.775 with 12); the x kernel takes two
// warps per CTA when its windows are staged by TMA, else one.
int rf_cta_warps(int axis)
{
    static int w = -1;
    if (w < 0) {
        const char *e = getenv("VFD_RF_W");
        const int v = e ? atoi(e) : 4;
        w = (v == 1 || v == 2 || v == 4 || v == 6 || v == 12) ? v : 4;
    }
    if (axis == PASS_X) return rf_tma_enabled() && rf_row_enabled() ? 2 : 1;
    return w;
}

static std::mutex g_rf_mu;
static bool g_rf_done[64];

cudaError_t rf_prepare()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_rf_mu);
    if (g_rf_done[dev]) return cudaSuccess;
    float2 tw[64], pc[32], ps[32], pn[32];
    for (int m = 0; m < 64; ++m) {
        const double a = 6.283185307179586476925286766559 * m / 64.0;
        tw[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    for (int m = 0; m < 32; ++m) {
        const double a = 6.283185307179586476925286766559 * m / 32.0;
        const float wr = (float)std::cos(a), wi = (float)-std::sin(a);
        pc[m] = make_float2(wr, wr);
        ps[m] = make_float2(wi, wi);
        pn[m] = make_float2(-wi, -wi);
    }
    e = cudaMemcpyToSymbol(c_rfw64, tw, sizeof(tw));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_spc, pc, sizeof(pc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_sps, ps, sizeof(ps));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_spn, pn, sizeof(pn));
    if (e == cudaSuccess) g_rf_done[dev] = true;
    return e;
}

// The bounded wait of the passes on a barrier that no copy will complete:
// one warp arms the barrier for 1 KB that never arrives (no copy is issued,
// so nothing is left in flight), waits `limit` cycles and records the
// give-up in g_rf_timeout exactly as the passes do.
__global__ void rf_wait_probe_kernel(long long limit, int *gave_up)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncwarp();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 1024);
    __syncwarp();
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar, 0, limit));
    if (!ok && threadIdx.x == 0) {
        atomicExch(&g_rf_timeout, 1);
        *gave_up = 1;
    }
}

cudaError_t rf_wait_probe(long long limit, int *gave_up_device, cudaStream_t st)
{
    rf_wait_probe_kernel<<<1, 32, 0, st>>>(limit, gave_up_device);
    note_launch();
    return cudaGetLastError();
}

bool rf_take_timeout()
{
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_rf_timeout, sizeof(int)) != cudaSuccess) return false;
    if (v) {
        const int z = 0;
        cudaMemcpyToSymbol(g_rf_timeout, &z, sizeof(int));
    }
    return v != 0;
}

// VFD_RF_TMA=0 keeps the y and z passes on direct global loads.
bool rf_tma_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_RF_TMA");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1 && tma_available();
}

bool rf_encode_map(const OsJob &j, CUtensorMap *m)
{
    if (j.kind == PASS_X) {
        // rows of n positions, row stride line_stride: even rows and odd rows
        // as two tensors {n, rows / 2} with row stride 2 line_stride
        const uint64_t n = (uint64_t)j.n, rows = (uint64_t)j.nlines * j.nouter;
        const uint64_t rs = (uint64_t)j.line_stride * 4;
        if (j.nouter != 1 || rows < 2 || (j.n & 3) != 0 || (rs & 15) != 0) return false;
        const uint64_t ne = (rows + 1) / 2, no = rows / 2;
        return tma_encode_3d(&m[0], j.data, n, ne, 1, 2 * rs, 2 * rs * ne, RF_TS, 32, 1) &&
               tma_encode_3d(&m[1], j.data + j.line_stride, n, no, 1, 2 * rs, 2 * rs * no, RF_TS, 32, 1);
    }
    if (j.line_stride != 1) return false;
    // the field as the tensor {nx, ny, nz}: y pass (lines x, positions y,
    // outer z), z pass (lines x, outer y, positions z)
    const uint64_t nx = (uint64_t)j.nlines;
    const uint64_t ny = j.kind == PASS_Y ? (uint64_t)j.n : (uint64_t)j.nouter;
    const uint64_t nz = j.kind == PASS_Y ? (uint64_t)j.nouter : (uint64_t)j.n;
    const uint64_t sy = (uint64_t)(j.kind == PASS_Y ? j.pos_stride : j.outer_stride) * 4;
    const uint64_t sz = (uint64_t)(j.kind == PASS_Y ? j.outer_stride : j.pos_stride) * 4;
    if (sy != nx * 4 || sz != nx * ny * 4) return false;
    if (j.kind == PASS_Y) return tma_encode_3d(m, j.data, nx, ny, nz, sy, sz, 64, 64, 1);
    return tma_encode_3d(m, j.data, nx, ny, nz, sy, sz, 64, 1, 64);
}

template <int W, bool Z, int MINB>
static cudaError_t launch_col_tma(const OsJob *jobs, const CUtensorMap *maps, const OsTileInfo *tiles, int nb,
                                  cudaStream_t st)
{
    const size_t dyn = (size_t)W * RF_WIN_FLOATS * sizeof(float) + 1024;
    static int done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && !done[dev]) {
        e = cudaFuncSetAttribute(rf_col_tma_kernel<W, Z, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dyn);
        if (e != cudaSuccess) return e;
        done[dev] = 1;
    }
    rf_col_tma_kernel<W, Z, MINB><<<nb, 32 * W, dyn, st>>>(jobs, maps, tiles);
    return cudaSuccess;
}

// Resident 4-warp CTAs per SM the TMA y/z kernel is compiled for
// (VFD_RF_YZ_MINB: 2 = 8 warps, 220 registers and no spills, the default:
// on B200 the 512x256x384 world's y and z passes took 0.584 / 0.590 ms
// against 0.608 / 0.656 with 3 = 12 warps at 168 registers, which spill).
static int rf_yz_minb()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("VFD_RF_YZ_MINB");
        v = (e && e[0] == '3') ? 3 : 2;
    }
    return v;
}

cudaError_t launch_rf(const OsJob *jobs, const OsTileInfo *tiles, int ntiles, int axis, cudaStream_t st,
                      const CUtensorMap *maps)
{
    if (ntiles <= 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    bool ready;
    {
        std::lock_guard<std::mutex> lk(g_rf_mu);
        ready = dev >= 0 && dev < 64 && g_rf_done[dev];
    }
    if (!ready && (e = rf_prepare()) != cudaSuccess) return e;
    const int W = rf_cta_warps(axis);
    if (ntiles % W != 0) return cudaErrorInvalidValue;
    const int nb = ntiles / W;
    if (axis == PASS_X && maps && W == 2) {
        const size_t dyn = (size_t)2 * RF_XWARP_BYTES + 1024;
        static int done[64] = {};
        if (dev >= 0 && dev < 64 && !done[dev]) {
            e = cudaFuncSetAttribute(rf_row_tma_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            if (e != cudaSuccess) return e;
            done[dev] = 1;
        }
        rf_row_tma_kernel<2><<<nb, 64, dyn, st>>>(jobs, maps, tiles);
    } else if (axis == PASS_X) {
        rf_row_kernel<<<ntiles, 32, 0, st>>>(jobs, tiles);
    } else if (maps && W == 4) {
        if (rf_yz_minb() == 2)
            e = axis == PASS_Z ? launch_col_tma<4, true, 2>(jobs, maps, tiles, nb, st)
                               : launch_col_tma<4, false, 2>(jobs, maps, tiles, nb, st);
        else
            e = axis == PASS_Z ? launch_col_tma<4, true, 3>(jobs, maps, tiles, nb, st)
                               : launch_col_tma<4, false, 3>(jobs, maps, tiles, nb, st);
        if (e != cudaSuccess) return e;
    } else {
        const bool z = axis == PASS_Z;
        switch (W) {
        case 2:
            if (z) rf_col_kernel<2, true><<<nb, 64, 0, st>>>(jobs, tiles);
            else rf_col_kernel<2, false><<<nb, 64, 0, st>>>(jobs, tiles);
            break;
        case 4:
            if (z) rf_col_kernel<4, true><<<nb, 128, 0, st>>>(jobs, tiles);
            else rf_col_kernel<4, false><<<nb, 128, 0, st>>>(jobs, tiles);
            break;
        case 6:
            if (z) rf_col_kernel<6, true><<<nb, 192, 0, st>>>(jobs, tiles);
            else rf_col_kernel<6, false><<<nb, 192, 0, st>>>(jobs, tiles);
            break;
        case 12:
            if (z) rf_col_kernel<12, true><<<nb, 384, 0, st>>>(jobs, tiles);
            else rf_col_kernel<12, false><<<nb, 384, 0, st>>>(jobs, tiles);
            break;
        default:
            if (z) rf_col_kernel<1, true><<<nb, 32, 0, st>>>(jobs, tiles);
            else rf_col_kernel<1, false><<<nb, 32, 0, st>>>(jobs, tiles);
            break;
        }
    }
    note_launch();
    return cudaGetLastError();
}

}  // namespace vfd
