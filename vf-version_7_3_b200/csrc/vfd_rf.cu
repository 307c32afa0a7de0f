// vfd_rf.cu -- one axis of the separable FFT convolution, overlap-save with
// 64-point blocks, each block's FFT held by ONE thread in 64 complex
// registers.
//
// Same method as vfd_os.cu (blocks of L = 64 - 2r outputs; forward FFT-64,
// multiply by the kernel's 64-point spectrum, inverse FFT-64, keep L samples
// -- the reference's pad / R2C / modulate / C2R / crop, Diffusion.cu:1731-1859,
// per block; lines 2p and 2p+1 ride in one complex FFT).  What changes is who
// holds a block: a thread owns a line pair and walks its blocks in order.
// The FFT-64 is radix 8 x 8 entirely in registers: its transpose is register
// renaming and its twiddles are constant-bank operands, so a block costs no
// shared-memory traffic beyond its input and output.
//
//   y and z passes (lines contiguous in x): a warp owns 32 adjacent pairs
//   (64 lines); at each position the warp loads and stores 256 contiguous
//   bytes straight from and to global memory.
//   x pass (positions contiguous): a warp owns 64 rows; each block's window
//   is copied row by row with 16-byte cp.async into a shared tile, each
//   thread reads its pair's two rows, and outputs go back the same way with
//   16-byte stores (rows 16-byte aligned and n a multiple of 4; otherwise
//   the x pass uses the overlap-save kernel).
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

namespace vfd {

__constant__ float2 c_rfw64[64];  // exp(-2 pi i m / 64), FP64-generated on the host

namespace {

__device__ __forceinline__ float2 r_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 r_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 r_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }

__device__ __forceinline__ double r_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <bool INV>
__device__ __forceinline__ void r_dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3)
{
    const float2 t0 = r_add(a0, a2), t1 = r_sub(a0, a2);
    const float2 t2 = r_add(a1, a3), d = r_sub(a1, a3);
    a0 = r_add(t0, t2);
    a2 = r_sub(t0, t2);
    if (!INV) {  // t3 = -i d
        a1 = make_float2(t1.x + d.y, t1.y - d.x);
        a3 = make_float2(t1.x - d.y, t1.y + d.x);
    } else {  // t3 = +i d
        a1 = make_float2(t1.x - d.y, t1.y + d.x);
        a3 = make_float2(t1.x + d.y, t1.y - d.x);
    }
}

// DFT-8 of (v0 .. v7) in place, radix 2 x 4, w8 = exp(-+ i pi / 4).
template <bool INV>
__device__ __forceinline__ void r_dft8(float2 &v0, float2 &v1, float2 &v2, float2 &v3, float2 &v4, float2 &v5,
                                       float2 &v6, float2 &v7)
{
    const float h = 0.707106781186547524400844362105f;
    float2 e0 = v0, e1 = v2, e2 = v4, e3 = v6;
    float2 o0 = v1, o1 = v3, o2 = v5, o3 = v7;
    r_dft4<INV>(e0, e1, e2, e3);
    r_dft4<INV>(o0, o1, o2, o3);
    if (!INV) {
        o1 = r_mul(make_float2(o1.x + o1.y, o1.y - o1.x), make_float2(h, h));
        o3 = r_mul(make_float2(o3.y - o3.x, o3.x + o3.y), make_float2(h, -h));
        v2 = make_float2(e2.x + o2.y, e2.y - o2.x);  // o2 * -i
        v6 = make_float2(e2.x - o2.y, e2.y + o2.x);
    } else {
        o1 = r_mul(make_float2(o1.x - o1.y, o1.x + o1.y), make_float2(h, h));
        o3 = r_mul(make_float2(o3.x + o3.y, o3.x - o3.y), make_float2(-h, h));
        v2 = make_float2(e2.x - o2.y, e2.y + o2.x);  // o2 * +i
        v6 = make_float2(e2.x + o2.y, e2.y - o2.x);
    }
    v0 = r_add(e0, o0);
    v4 = r_sub(e0, o0);
    v1 = r_add(e1, o1);
    v5 = r_sub(e1, o1);
    v3 = r_add(e3, o3);
    v7 = r_sub(e3, o3);
}

// Forward FFT-64 in registers.  In: x[n], n = 8 n1 + n2.  Out: bin
// k = k1 + 8 k2 in slot 8 k1 + k2.
//   DFT-8 over n1 for each n2 (slots n2 + 8 n1)  -> A(n2, k1) in slot 8 k1 + n2
//   twiddle w64^(n2 k1)
//   DFT-8 over n2 for each k1 (slots 8 k1 + n2)  -> X(k1 + 8 k2) in slot 8 k1 + k2
__device__ __forceinline__ void r_fft64_fwd(float2 (&x)[64])
{
#pragma unroll
    for (int n2 = 0; n2 < 8; ++n2)
        r_dft8<false>(x[n2], x[8 + n2], x[16 + n2], x[24 + n2], x[32 + n2], x[40 + n2], x[48 + n2], x[56 + n2]);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1)
#pragma unroll
        for (int n2 = 1; n2 < 8; ++n2) x[8 * k1 + n2] = c_mul(x[8 * k1 + n2], c_rfw64[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1)
        r_dft8<false>(x[8 * k1], x[8 * k1 + 1], x[8 * k1 + 2], x[8 * k1 + 3], x[8 * k1 + 4], x[8 * k1 + 5],
                      x[8 * k1 + 6], x[8 * k1 + 7]);
}

// Inverse of r_fft64_fwd (unnormalised): bins in its output order, x[n] out.
__device__ __forceinline__ void r_fft64_inv(float2 (&x)[64])
{
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1)
        r_dft8<true>(x[8 * k1], x[8 * k1 + 1], x[8 * k1 + 2], x[8 * k1 + 3], x[8 * k1 + 4], x[8 * k1 + 5],
                     x[8 * k1 + 6], x[8 * k1 + 7]);
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1)
#pragma unroll
        for (int n2 = 1; n2 < 8; ++n2) {
            const float2 w = c_rfw64[n2 * k1];
            x[8 * k1 + n2] = c_mul(x[8 * k1 + n2], make_float2(w.x, -w.y));
        }
#pragma unroll
    for (int n2 = 0; n2 < 8; ++n2)
        r_dft8<true>(x[n2], x[8 + n2], x[16 + n2], x[24 + n2], x[32 + n2], x[40 + n2], x[48 + n2], x[56 + n2]);
}

// Spectrum multiply: bin k sits in slot 8 (k mod 8) + k / 8.
__device__ __forceinline__ void r_modulate(float2 (&x)[64], const float2 *hh)
{
#pragma unroll
    for (int k = 0; k < 64; ++k) x[8 * (k & 7) + (k >> 3)] = r_mul(x[8 * (k & 7) + (k >> 3)], hh[k]);
}

}  // namespace

// ---------------------------------------------------------------------------
// y / z passes: one warp = one tile of 64 lines (32 pairs) of one outer index.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rf_prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

template <int R, bool V2>
__device__ __forceinline__ void rf_col_body(const OsJob &J, const OsTileInfo &T, const float2 *hh,
                                            float2 (*held)[32])
{
    constexpr int L = 64 - 2 * R;
    const int lane = threadIdx.x;
    const int nreal = T.flags & 255;
    const int line = 2 * lane;
    const bool va = line < nreal, vb = line + 1 < nreal;
    const int n = J.n;
    const int64_t ps = J.pos_stride;
    float *const base = J.data + T.outer * J.outer_stride + (int64_t)(T.l0 + line) * J.line_stride;
    const bool zlast = J.kind == PASS_Z;
    const float keep = J.keep, b = J.b;
    const int nblocks = (n + 2 * R + L - 1) / L;
    // one output (or held-back output) of the pair at position o
    auto put = [&](float *d, float2 v) {
        if (V2) {
            *reinterpret_cast<float2 *>(d) = v;
        } else {
            d[0] = v.x;
            if (vb) d[1] = v.y;
        }
    };

    float2 lk = make_float2(0.0f, 0.0f), cv = lk, ot = lk;
    if (va) {
        for (int bi = 0; bi < nblocks; ++bi) {
            const int c = -R + bi * L;  // first output of the block
            const int p0 = c - R;       // first input
            const bool inner = p0 >= 0 && p0 + 64 <= n;  // window and outputs inside the line
            float *const w0 = base + (int64_t)p0 * ps;
            float2 x[64];
            {
                const float *sp = w0;
                if (inner) {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps)
                        x[i] = V2 ? *reinterpret_cast<const float2 *>(sp) : make_float2(sp[0], vb ? sp[1] : 0.0f);
                } else if (V2) {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps)
                        x[i] = ((unsigned)(p0 + i) < (unsigned)n) ? *reinterpret_cast<const float2 *>(sp)
                                                                  : make_float2(0.0f, 0.0f);
                } else {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps) {
                        const bool in = (unsigned)(p0 + i) < (unsigned)n;
                        x[i] = make_float2(in ? sp[0] : 0.0f, (in && vb) ? sp[1] : 0.0f);
                    }
                }
            }
            // the next block's new samples start for L2 while this one is transformed
            if (bi + 1 < nblocks) {
                const int q0 = p0 + 64, q1 = min(p0 + L + 64, n);
                const float *pp = base + (int64_t)q0 * ps;
                for (int q = q0; q < q1; ++q, pp += ps) rf_prefetch_l2(pp);
            }
            // the previous block's held-back outputs: positions p0 .. p0 + R - 1,
            // just loaded above as this window's first inputs
            if (bi > 0) {
#pragma unroll
                for (int i = 0; i < R; ++i)
                    if ((unsigned)(p0 + i) < (unsigned)n) put(w0 + (int64_t)i * ps, held[i][lane]);
            }
            r_fft64_fwd(x);
            r_modulate(x, hh);
            r_fft64_inv(x);
            float *d = w0 + (int64_t)R * ps;  // position of sample R = first output c
#pragma unroll
            for (int i = R; i < R + L; ++i, d += ps) {
                const int o = c + i - R;
                if (inner || (unsigned)o < (unsigned)n) {
                    float2 v = x[i];
                    if (zlast) {
                        cv = r_add(cv, v);
                        v = r_mul(r_add(v, make_float2(b, b)), make_float2(keep, keep));
                        ot = r_add(ot, v);
                    }
                    if (i >= L) held[i - L][lane] = v;  // stored after the next block's loads
                    else put(d, v);
                } else if (o >= -R && o < n + R) {
                    lk = r_add(lk, x[i]);
                }
            }
        }
        // the last block's held-back outputs
        const int clast = -R + (nblocks - 1) * L;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int o = clast + L - R + i;
            if ((unsigned)o < (unsigned)n) put(base + (int64_t)o * ps, held[i][lane]);
        }
    }
    double *mass = J.mass;
    const double s_lk = r_warp_sum((double)(va ? lk.x : 0.0f) + (double)(vb ? lk.y : 0.0f));
    if (J.kind == PASS_Y) {
        if (lane == 0 && s_lk != 0.0) atomicAdd(mass + MS_LEAK_Y, s_lk);
    } else {
        const double s_cv = r_warp_sum((double)(va ? cv.x : 0.0f) + (double)(vb ? cv.y : 0.0f));
        const double s_ot = r_warp_sum((double)(va ? ot.x : 0.0f) + (double)(vb ? ot.y : 0.0f));
        if (lane == 0) {
            if (s_lk != 0.0) atomicAdd(mass + MS_LEAK_Z, s_lk);
            if (s_cv != 0.0) atomicAdd(mass + MS_CONV, s_cv);
            if (s_ot != 0.0) atomicAdd(mass + MS_OUT, s_ot);
        }
    }
}

// The same walk with the radius read from the job at run time: register
// indices stay compile-time (every slot is tested against [r, r + L)), the
// held-back outputs are indexed in shared memory.  One code body for every
// radius keeps the kernel small enough for the instruction cache when warps
// of different radii share an SM.
template <bool V2>
__device__ __forceinline__ void rf_col_body_rt(const OsJob &J, const OsTileInfo &T, const float2 *hh,
                                               float2 (*held)[32])
{
    const int R = J.r, L = 64 - 2 * R;
    const int lane = threadIdx.x;
    const int nreal = T.flags & 255;
    const int line = 2 * lane;
    const bool va = line < nreal, vb = line + 1 < nreal;
    const int n = J.n;
    const int64_t ps = J.pos_stride;
    float *const base = J.data + T.outer * J.outer_stride + (int64_t)(T.l0 + line) * J.line_stride;
    const bool zlast = J.kind == PASS_Z;
    const float keep = J.keep, b = J.b;
    const int nblocks = (n + 2 * R + L - 1) / L;
    auto put = [&](int o, float2 v) {
        float *d = base + (int64_t)o * ps;
        if (V2) {
            *reinterpret_cast<float2 *>(d) = v;
        } else {
            d[0] = v.x;
            if (vb) d[1] = v.y;
        }
    };

    float2 lk = make_float2(0.0f, 0.0f), cv = lk, ot = lk;
    if (va) {
        for (int bi = 0; bi < nblocks; ++bi) {
            const int c = -R + bi * L;
            const int p0 = c - R;
            float2 x[64];
            {
                const float *sp = base + (int64_t)p0 * ps;
                if (V2) {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps)
                        x[i] = ((unsigned)(p0 + i) < (unsigned)n) ? *reinterpret_cast<const float2 *>(sp)
                                                                  : make_float2(0.0f, 0.0f);
                } else {
#pragma unroll
                    for (int i = 0; i < 64; ++i, sp += ps) {
                        const bool in = (unsigned)(p0 + i) < (unsigned)n;
                        x[i] = make_float2(in ? sp[0] : 0.0f, (in && vb) ? sp[1] : 0.0f);
                    }
                }
            }
            if (bi > 0)
                for (int i = 0; i < R; ++i)
                    if ((unsigned)(p0 + i) < (unsigned)n) put(p0 + i, held[i][lane]);
            r_fft64_fwd(x);
            r_modulate(x, hh);
            r_fft64_inv(x);
#pragma unroll
            for (int i = 1; i < 63; ++i) {  // kept samples: i in [R, R + L), R in 1 .. 8
                if (i < R || i >= R + L) continue;
                const int o = c + i - R;
                if ((unsigned)o < (unsigned)n) {
                    float2 v = x[i];
                    if (zlast) {
                        cv = r_add(cv, v);
                        v = r_mul(r_add(v, make_float2(b, b)), make_float2(keep, keep));
                        ot = r_add(ot, v);
                    }
                    if (i >= L) held[i - L][lane] = v;  // stored after the next block's loads
                    else put(o, v);
                } else if (o >= -R && o < n + R) {
                    lk = r_add(lk, x[i]);
                }
            }
        }
        const int clast = -R + (nblocks - 1) * L;
        for (int i = 0; i < R; ++i) {
            const int o = clast + L - R + i;
            if ((unsigned)o < (unsigned)n) put(o, held[i][lane]);
        }
    }
    double *mass = J.mass;
    const double s_lk = r_warp_sum((double)(va ? lk.x : 0.0f) + (double)(vb ? lk.y : 0.0f));
    if (J.kind == PASS_Y) {
        if (lane == 0 && s_lk != 0.0) atomicAdd(mass + MS_LEAK_Y, s_lk);
    } else {
        const double s_cv = r_warp_sum((double)(va ? cv.x : 0.0f) + (double)(vb ? cv.y : 0.0f));
        const double s_ot = r_warp_sum((double)(va ? ot.x : 0.0f) + (double)(vb ? ot.y : 0.0f));
        if (lane == 0) {
            if (s_lk != 0.0) atomicAdd(mass + MS_LEAK_Z, s_lk);
            if (s_cv != 0.0) atomicAdd(mass + MS_CONV, s_cv);
            if (s_ot != 0.0) atomicAdd(mass + MS_OUT, s_ot);
        }
    }
}

template <bool V2>
__global__ void __launch_bounds__(32, 12) rf_col_rt_kernel(const OsJob *__restrict__ jobs,
                                                           const OsTileInfo *__restrict__ tiles)
{
    __shared__ __align__(16) float2 hh[64];
    __shared__ float2 held[RF_RMAX][32];
    const OsTileInfo T = tiles[blockIdx.x];
    const OsJob &J = jobs[T.job];
    hh[threadIdx.x] = J.HH[threadIdx.x];
    hh[threadIdx.x + 32] = J.HH[threadIdx.x + 32];
    __syncwarp();
    rf_col_body_rt<V2>(J, T, hh, held);
}

// One launch covers tiles of every radius: the CTA's job picks the variant.
template <bool V2>
__global__ void __launch_bounds__(32, 12) rf_col_kernel(const OsJob *__restrict__ jobs,
                                                        const OsTileInfo *__restrict__ tiles)
{
    __shared__ __align__(16) float2 hh[64];
    __shared__ float2 held[RF_RMAX][32];  // held-back outputs [i][lane]
    const OsTileInfo T = tiles[blockIdx.x];
    const OsJob &J = jobs[T.job];
    hh[threadIdx.x] = J.HH[threadIdx.x];
    hh[threadIdx.x + 32] = J.HH[threadIdx.x + 32];
    __syncwarp();
    switch (J.r) {
    case 1: rf_col_body<1, V2>(J, T, hh, held); break;
    case 2: rf_col_body<2, V2>(J, T, hh, held); break;
    case 3: rf_col_body<3, V2>(J, T, hh, held); break;
    case 4: rf_col_body<4, V2>(J, T, hh, held); break;
    case 5: rf_col_body<5, V2>(J, T, hh, held); break;
    case 6: rf_col_body<6, V2>(J, T, hh, held); break;
    case 7: rf_col_body<7, V2>(J, T, hh, held); break;
    default: rf_col_body<8, V2>(J, T, hh, held); break;
    }
}

// ---------------------------------------------------------------------------
// x pass: one warp = 64 rows (32 pairs).  Rows hold positions contiguously,
// so blocks are moved through a shared tile with 16-byte copies:
//   * chunks start on multiples of 4: the first output is -Rh (Rh = r
//     rounded up to 4) and blocks keep L4 outputs (L4 = L rounded down to a
//     multiple of 4); a block's window is the 68 positions from c - Rh, and
//     its FFT input starts e = Rh - r positions into it;
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
__device__ __forceinline__ void rf_row_body(const OsJob &J, const OsTileInfo &T, const float2 *hh, float *A,
                                            float *held)
{
    constexpr int L = 64 - 2 * R;
    constexpr int L4 = L & ~3;          // outputs kept per block
    constexpr int RH = (R + 3) & ~3;    // held-back outputs per block (multiple of 4)
    constexpr int E = RH - R;           // FFT input offset in the window
    constexpr int NST = (L4 - RH) / 4;  // chunks stored at once per row
    constexpr int NHD = RH / 4;         // held chunks per row
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
        // ---- window [pa, pa + 68) of every row, 16-byte chunks ---------------
        {
            int row = lane / 17, cc = lane - 17 * (lane / 17);
            for (int k = lane; k < nreal * 17; k += 32) {
                const int p = pa + 4 * cc;
                const bool v = (unsigned)p < (unsigned)n;  // a chunk lies wholly inside or outside
                const float *src = base + (int64_t)row * ls;
                rf_cp16(A + rf_trow(row) * RF_TS + 4 * cc, v ? src + p : src, v);
                cc += 15;
                row += 1;
                if (cc >= 17) {
                    cc -= 17;
                    row += 1;
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncwarp();
        // the previous block's held-back outputs are this window's first RH positions
        if (bi > 0) put_held(pa);
        // ---- this lane's pair: FFT-64 in registers ------------------------------
        float2 x[64];
        {
            const float4 *ra = reinterpret_cast<const float4 *>(A + lane * RF_TS);
            const float4 *rb = reinterpret_cast<const float4 *>(A + (32 + lane) * RF_TS);
#pragma unroll
            for (int m = 0; m < 17; ++m) {
                const float4 u = ra[m], w = rb[m];
                const float ua[4] = {u.x, u.y, u.z, u.w}, wa[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int i = 4 * m + k - E;
                    if (i >= 0 && i < 64) x[i] = make_float2(ua[k], wa[k]);
                }
            }
        }
        __syncwarp();  // every lane has its column: the tile is free for outputs
        if (!vb) {
            // tile rows past the tile's lines hold stale data: zero the pair's missing line
#pragma unroll
            for (int i = 0; i < 64; ++i) x[i] = make_float2(va ? x[i].x : 0.0f, 0.0f);
        }
        if (masked) {
#pragma unroll
            for (int i = 0; i < 64; ++i) {
                const int p = c - R + i;
                const bool px = p >= xlo && p < xhi;
                x[i].x = (in_a && px) ? x[i].x - b : 0.0f;
                x[i].y = (in_b && px) ? x[i].y - b : 0.0f;
            }
        }
        {
            float2 s2 = make_float2(0.0f, 0.0f);  // input mass: block outputs' positions
#pragma unroll
            for (int i = R; i < R + L4; ++i) s2 = r_add(s2, x[i]);
            acc_in += (double)(va ? s2.x : 0.0f) + (double)(vb ? s2.y : 0.0f);
        }
        r_fft64_fwd(x);
        r_modulate(x, hh);
        r_fft64_inv(x);
#pragma unroll
        for (int i = R; i < R + L4; ++i) {
            const int o = c + i - R;
            if (!((unsigned)o < (unsigned)n) && o >= -R && o < n + R) lk = r_add(lk, x[i]);
        }
        {
            float4 *wa = reinterpret_cast<float4 *>(A + lane * RF_TS);
            float4 *wb = reinterpret_cast<float4 *>(A + (32 + lane) * RF_TS);
#pragma unroll
            for (int m = 0; m < L4 / 4; ++m) {
                wa[m] = make_float4(x[R + 4 * m].x, x[R + 4 * m + 1].x, x[R + 4 * m + 2].x, x[R + 4 * m + 3].x);
                wb[m] = make_float4(x[R + 4 * m].y, x[R + 4 * m + 1].y, x[R + 4 * m + 2].y, x[R + 4 * m + 3].y);
            }
        }
        __syncwarp();
        // ---- outputs [c, c + L4 - RH) of every row; the rest is held back ------
        for (int k = lane; k < nreal * NST; k += 32) {
            const int row = k / NST, cc = k - row * NST;
            const int o = c + 4 * cc;
            if ((unsigned)o < (unsigned)n)
                *reinterpret_cast<float4 *>(base + (int64_t)row * ls + o) =
                    *reinterpret_cast<const float4 *>(A + rf_trow(row) * RF_TS + 4 * cc);
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
    __shared__ __align__(16) float2 hh[64];
    const OsTileInfo T = tiles[blockIdx.x];
    const OsJob &J = jobs[T.job];
    hh[threadIdx.x] = J.HH[threadIdx.x];
    hh[threadIdx.x + 32] = J.HH[threadIdx.x + 32];
    __syncwarp();
    switch (J.r) {
    case 1: rf_row_body<1>(J, T, hh, A, held); break;
    case 2: rf_row_body<2>(J, T, hh, A, held); break;
    case 3: rf_row_body<3>(J, T, hh, A, held); break;
    case 4: rf_row_body<4>(J, T, hh, A, held); break;
    case 5: rf_row_body<5>(J, T, hh, A, held); break;
    case 6: rf_row_body<6>(J, T, hh, A, held); break;
    case 7: rf_row_body<7>(J, T, hh, A, held); break;
    default: rf_row_body<8>(J, T, hh, A, held); break;
    }
}

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
            const int nreal = std::min(RF_LINES, j.nlines - ti.l0);
            // 8-byte pair accesses: every (pair, position) address even
            const uintptr_t base = reinterpret_cast<uintptr_t>(j.data) +
                                   sizeof(float) * (uintptr_t)(outer * j.outer_stride + (int64_t)ti.l0 * j.line_stride);
            const bool v2 = j.kind != PASS_X && (base & 7) == 0 && (j.pos_stride & 1) == 0 && (nreal & 1) == 0;
            ti.flags = nreal | (v2 ? 1 << 8 : 0);
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

// VFD_RF_RT=1 selects the y/z kernel that reads the radius at run time (one
// code body) instead of the one with a compiled variant per radius.
static bool rf_col_runtime_radius()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_RF_RT");
        on = (e && e[0] == '1') ? 1 : 0;
    }
    return on == 1;
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
    float2 tw[64];
    for (int m = 0; m < 64; ++m) {
        const double a = 6.283185307179586476925286766559 * m / 64.0;
        tw[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    e = cudaMemcpyToSymbol(c_rfw64, tw, sizeof(tw));
    if (e == cudaSuccess) g_rf_done[dev] = true;
    return e;
}

cudaError_t launch_rf(const OsJob *jobs, const OsTileInfo *tiles, int ntiles, int axis, bool pairs8, cudaStream_t st)
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
    if (axis == PASS_X) rf_row_kernel<<<ntiles, 32, 0, st>>>(jobs, tiles);
    else if (rf_col_runtime_radius()) {
        if (pairs8) rf_col_rt_kernel<true><<<ntiles, 32, 0, st>>>(jobs, tiles);
        else rf_col_rt_kernel<false><<<ntiles, 32, 0, st>>>(jobs, tiles);
    } else if (pairs8) rf_col_kernel<true><<<ntiles, 32, 0, st>>>(jobs, tiles);
    else rf_col_kernel<false><<<ntiles, 32, 0, st>>>(jobs, tiles);
    note_launch();
    return cudaGetLastError();
}

}  // namespace vfd
