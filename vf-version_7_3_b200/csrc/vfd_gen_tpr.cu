// vfd_gen_tpr.cu -- the general 3D FFT convolution's row and column passes
// on the two-pass register engine (vfd_tpr.cuh).
//
// Same passes, arguments and results as the Stockham kernels of
// vfd_general.cu (R2C along x, C2C along y or z with the fused z multiply,
// C2R along x with the crop / update epilogue), for lengths F = F1 * F2 with
// F1, F2 <= 32.  The first pass of a tile reads its groups straight from
// global memory into registers and the last pass writes its groups straight
// back, so a tile crosses shared memory once:
//
//   c2c forward   A: global -> regs -> smem | B: smem -> regs -> global
//   c2c fused z   A | B, times K/N, B' in the same registers -> smem | A' -> global
//   c2c inverse   B': global -> regs -> smem | A' -> global
//   r2c           A: two real rows per complex line | B -> smem, natural order
//                 | split into the two half spectra -> global
//   c2r           B': z(k) = A(k) + i B(k) from the Hermitian halves | A' ->
//                 two real rows with the crop / update epilogue -> global
//
// Lanes walk the axis that is contiguous in memory: lines for the column
// passes (NL consecutive lines, 128 bytes for NL = 16), positions n2 (the
// first pass) or bins k1 (the C2R first pass) for the row passes.
//
// Shared memory: the tile, then (unused room for tw[m] = w_F^m) the pass
// twiddles w_F^(k1 n2) in both orders (T[k1 F2 + n2] for lanes along n2,
// Tt[n2 F1 + k1] for lanes along k1, so that neither gather conflicts).  The
// first pass's global loads are issued before the twiddle staging and its
// barrier, so they overlap.  The fused z pass reads its spectrum K straight
// from global memory in pass B (lanes along lines: coalesced), which leaves
// the shared memory to the tile and more CTAs per SM (measured on B200, the
// 512x256x384 world: 2.23 -> 1.96 ms per tick against staging K by
// cp.async).
// Tile: slot n2 + F2 k1 of line l at S[n2 * LS + k1 * GS + l] with
// LS = NL + 1 and GS = F2 * LS + pad, pad = 1 when F2 is even (an odd GS
// keeps the walks along k1 free of bank conflicts); the R2C pass B leaves
// bin k at S[k * LS + l].
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include "vfd_general.h"
#include "vfd_internal.h"
#include "vfd_tpr.cuh"

namespace vfd {

__device__ __forceinline__ double tpr_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum added to *dst (skipped when dst is NULL or the sum is zero).
__device__ __forceinline__ void tpr_block_sum(double v, double *dst, double *red)
{
    v = tpr_warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        v = tpr_warp_sum(v);
        if (l == 0 && v != 0.0 && dst) atomicAdd(dst, v);
    }
    __syncthreads();
}

__device__ __forceinline__ float2 c_conj_mul(float2 a, float2 w) { return c_mul(a, make_float2(w.x, -w.y)); }

struct TprSmem {
    float2 *S, *tw, *T, *Tt;
};
__device__ __forceinline__ TprSmem tpr_smem_layout(float2 *base, int F, int NL)
{
    TprSmem m;
    m.S = base;
    m.tw = base + F * (NL + 1) + TPR_MAX;
    m.T = m.tw + F;
    m.Tt = m.T + F;
    return m;
}
// T and Tt from the global table (no barrier: the caller's follows; the
// small DFTs take their twiddles as immediates, so tw is not staged).
// i / d as (i * ceil(2^21 / d)) >> 21, exact for i < 65536 and d <= 32.
__device__ __forceinline__ void stage_twiddles(const TprSmem &m, const float2 *__restrict__ g, int F, int F1, int F2)
{
    const int m1 = ((1 << 21) + F1 - 1) / F1, m2 = ((1 << 21) + F2 - 1) / F2;
    for (int i = threadIdx.x; i < F; i += blockDim.x) {
        const int a = (i * m2) >> 21, b = i - a * F2;  // T: k1 = a, n2 = b
        m.T[i] = g[a * b];
        const int c = (i * m1) >> 21, d = i - c * F1;  // Tt: n2 = c, k1 = d
        m.Tt[i] = g[c * d];
    }
}

__device__ __forceinline__ void tpr_cp8(float2 *smem, const float2 *gmem, bool valid)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void tpr_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void tpr_cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Kernel variants <NL, MAXT, MINB, MAXN>: NL lines per tile, up to MAXT
// threads, registers bounded for MINB resident CTAs, DFT lengths up to MAXN:
// <8, 256, 3 or 4, 24> for the lengths the general methods choose, <16, 512,
// 1, 32> for factors above 24.

// ---------------------------------------------------------------------------
// Column passes.  Element (line, outer, pos) at data + line + outer *
// outer_stride + pos * pos_stride; col points at (l0 + l, outer, 0).

// A (first pass): strided group n2 (positions n2 + F2 n1 < nload) loaded,
// twiddles staged, barrier, DFT F1, times w^(k1 n2), slots.
template <int N, int NL>
__device__ __forceinline__ void col_a(const GenColPass &p, const TprSmem &m, const float2 *col, int n2, int F2, int GS,
                                      bool lok, int l, bool active)
{
    const int F1 = N, F = F1 * F2;
    float2 v[N];
    if (active) {
#pragma unroll
        for (int n1 = 0; n1 < N; ++n1) {
            const int x = n2 + F2 * n1;
            v[n1] = (lok && x < p.nload) ? col[(int64_t)x * p.pos_stride] : make_float2(0.f, 0.f);
        }
    }
    stage_twiddles(m, p.tw, F, F1, F2);
    __syncthreads();
    if (!active) return;
    tpr_dft<N, false>(v);
    const float2 *t = m.T + n2;  // T[k1 F2 + n2]
#pragma unroll
    for (int k1 = 1; k1 < N; ++k1) v[k1] = c_mul(v[k1], t[k1 * F2]);
    float2 *d = m.S + n2 * (NL + 1) + l;
#pragma unroll
    for (int k1 = 0; k1 < N; ++k1) d[k1 * GS] = v[k1];
}

// B' tail: inverse DFT F2 of group k1 -> times conj w^(n2 k1) -> slots.
template <int N, int NL>
__device__ __forceinline__ void col_b_inverse(const TprSmem &m, float2 (&v)[N], int k1, int F1, int GS, int l)
{
    tpr_dft<N, true>(v);
    const float2 *t = m.T + k1 * N;  // T[k1 F2 + n2]
#pragma unroll
    for (int n2 = 1; n2 < N; ++n2) v[n2] = c_conj_mul(v[n2], t[n2]);
    float2 *grp = m.S + k1 * GS + l;
#pragma unroll
    for (int n2 = 0; n2 < N; ++n2) grp[n2 * (NL + 1)] = v[n2];
}

// B of group k1 (after A): slots -> DFT F2 -> bins k1 + F1 k2 to global
// (GEN_FORWARD), or times K/N (K[kz = bin][ky = outer][kx = l0 + l] from
// global memory) and B'.
template <int N, int NL>
__device__ __forceinline__ void col_b(const GenColPass &p, const TprSmem &m, float2 *col, int k1, int F1, int GS,
                                      bool lok, int l, int outer, int l0, bool active)
{
    if (!active) return;
    float2 v[N];
    const float2 *grp = m.S + k1 * GS + l;  // slot F2 k1 + n2 at grp[n2 * LS]
#pragma unroll
    for (int n2 = 0; n2 < N; ++n2) v[n2] = grp[n2 * (NL + 1)];
    tpr_dft<N, false>(v);
    if (p.mode == GEN_FORWARD) {
        if (lok) {
#pragma unroll
            for (int k2 = 0; k2 < N; ++k2) {
                const int bin = k1 + F1 * k2;
                if (bin < p.nstore) col[(int64_t)bin * p.pos_stride] = v[k2];
            }
        }
        return;
    }
    const float2 *kp = p.kspec + (int64_t)outer * p.k_s_outer + l0 + l;
#pragma unroll
    for (int k2 = 0; k2 < N; ++k2) {
        const float2 kk = lok ? kp[(int64_t)(k1 + F1 * k2) * p.k_s_pos] : make_float2(0.f, 0.f);
        const float2 x = v[k2];
        v[k2] = make_float2(p.scale * (x.x * kk.x - x.y * kk.y), p.scale * (x.x * kk.y + x.y * kk.x));
    }
    col_b_inverse<N, NL>(m, v, k1, F1, GS, l);
}

// B' as the first pass (inverse only): bins k1 + F1 k2 < nload loaded,
// twiddles staged, barrier, inverse DFT F2 -> slots.
template <int N, int NL>
__device__ __forceinline__ void col_bi(const GenColPass &p, const TprSmem &m, const float2 *col, int k1, int F1,
                                       int GS, bool lok, int l, bool active)
{
    const int F2 = N, F = F1 * F2;
    float2 v[N];
    if (active) {
#pragma unroll
        for (int k2 = 0; k2 < N; ++k2) {
            const int bin = k1 + F1 * k2;
            v[k2] = (lok && bin < p.nload) ? col[(int64_t)bin * p.pos_stride] : make_float2(0.f, 0.f);
        }
    }
    stage_twiddles(m, p.tw, F, F1, F2);
    __syncthreads();
    if (active) col_b_inverse<N, NL>(m, v, k1, F1, GS, l);
}

// A': slots of group n2 -> inverse DFT F1 -> positions n2 + F2 n1 < nstore.
template <int N, int NL>
__device__ __forceinline__ void col_ai(const GenColPass &p, const TprSmem &m, float2 *col, int n2, int F2, int GS,
                                       bool lok, int l)
{
    float2 v[N];
    const float2 *s = m.S + n2 * (NL + 1) + l;
#pragma unroll
    for (int k1 = 0; k1 < N; ++k1) v[k1] = s[k1 * GS];
    tpr_dft<N, true>(v);
    if (lok) {
#pragma unroll
        for (int n1 = 0; n1 < N; ++n1) {
            const int x = n2 + F2 * n1;
            if (x < p.nstore) col[(int64_t)x * p.pos_stride] = v[n1];
        }
    }
}

// One tile = NL consecutive lines of one outer index; thread (l, g) with the
// line fastest takes group g of each pass.
template <int NL, int MAXT, int MINB, int MAXN>
__global__ void __launch_bounds__(MAXT, MINB) c2c_tpr_kernel(const GenColPass p, int f1)
{
    constexpr int LS = NL + 1;
    extern __shared__ __align__(16) float2 tsm[];
    const int F = p.plan.F, F1 = f1, F2 = F / f1;
    const int GS = F2 * LS + ((F2 & 1) ^ 1);
    const TprSmem m = tpr_smem_layout(tsm, F, NL);

    const int tiles_per_outer = (p.nlines + NL - 1) / NL;
    const int outer = blockIdx.x / tiles_per_outer;
    const int l0 = (blockIdx.x - outer * tiles_per_outer) * NL;
    const int l = threadIdx.x % NL, g = threadIdx.x / NL;
    const bool lok = l0 + l < p.nlines;
    float2 *col = p.data + (int64_t)outer * p.outer_stride + l0 + l;

    if (p.mode != GEN_INVERSE) {
        switch (F1) {
#define VFD_COL_A(n) \
    case n: if constexpr (n <= MAXN) col_a<n, NL>(p, m, col, g, F2, GS, lok, l, g < F2); break;
            VFD_TPR_SIZES(VFD_COL_A)
#undef VFD_COL_A
        default: break;
        }
        __syncthreads();
        switch (F2) {
#define VFD_COL_B(n) \
    case n: if constexpr (n <= MAXN) col_b<n, NL>(p, m, col, g, F1, GS, lok, l, outer, l0, g < F1); break;
            VFD_TPR_SIZES(VFD_COL_B)
#undef VFD_COL_B
        default: break;
        }
    } else {
        switch (F2) {
#define VFD_COL_BI(n) \
    case n: if constexpr (n <= MAXN) col_bi<n, NL>(p, m, col, g, F1, GS, lok, l, g < F1); break;
            VFD_TPR_SIZES(VFD_COL_BI)
#undef VFD_COL_BI
        default: break;
        }
    }
    if (p.mode != GEN_FORWARD) {
        __syncthreads();
        if (g < F2) {
            switch (F1) {
#define VFD_COL_AI(n) \
    case n: if constexpr (n <= MAXN) col_ai<n, NL>(p, m, col, g, F2, GS, lok, l); break;
                VFD_TPR_SIZES(VFD_COL_AI)
#undef VFD_COL_AI
            default: break;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row passes: 2 NL real rows per tile; complex line l holds row r0 + l
// (real part) and row r0 + NL + l (imaginary part).

struct RowRef {
    bool ok;     // row < nrows
    bool in;     // ok, and inside the padding box in (r1, r2) when padding is fused
    int64_t off; // r1 * s1 + r2 * s2
};
__device__ __forceinline__ RowRef row_ref(const GenRowPass &p, int row, int64_t s1, int64_t s2)
{
    RowRef r{row < p.nrows, false, 0};
    if (r.ok) {
        const int r1 = row % p.rows_per_plane, r2 = row / p.rows_per_plane;
        r.off = (int64_t)r1 * s1 + (int64_t)r2 * s2;
        r.in = !p.fuse_pad || (r1 >= p.box_lo[1] && r1 < p.box_hi[1] && r2 >= p.box_lo[2] && r2 < p.box_hi[2]);
    }
    return r;
}

// R2C A (first pass): positions n2 + F2 n1 of rows a and b (the padding
// rule v = u - b inside the box, 0 outside, when fused) loaded, twiddles
// staged, barrier, DFT F1, times w^(k1 n2), slots.  Returns the FP64 sum of
// the values (the input mass).
template <int N, int NL>
__device__ __forceinline__ double r2c_a(const GenRowPass &p, const TprSmem &m, int r0, int l, int n2, int F2, int GS,
                                        bool active)
{
    const int F1 = N, F = F1 * F2;
    float2 v[N];
    double acc_a = 0.0, acc_b = 0.0;
    if (active) {
        const RowRef ra = row_ref(p, r0 + l, p.r_s1, p.r_s2), rb = row_ref(p, r0 + NL + l, p.r_s1, p.r_s2);
        const float *sa = p.rsrc + ra.off, *sb = p.rsrc + rb.off;
#pragma unroll
        for (int n1 = 0; n1 < N; ++n1) {
            const int x = n2 + F2 * n1;
            const bool xin = x < p.nload && (!p.fuse_pad || (x >= p.box_lo[0] && x < p.box_hi[0]));
            v[n1].x = (ra.in && xin) ? sa[x] : 0.0f;
            v[n1].y = (rb.in && xin) ? sb[x] : 0.0f;
        }
        if (p.fuse_pad) {
#pragma unroll
            for (int n1 = 0; n1 < N; ++n1) {
                const int x = n2 + F2 * n1;
                const bool xin = x < p.nload && x >= p.box_lo[0] && x < p.box_hi[0];
                v[n1].x = (ra.in && xin) ? v[n1].x - p.b : 0.0f;
                v[n1].y = (rb.in && xin) ? v[n1].y - p.b : 0.0f;
            }
        }
        if (p.mass_in) {
            // FP32 pairwise partial sums (error <= ceil(log2 N) ulp of the sum
            // of magnitudes), widened once
            float ta[N], tb[N];
#pragma unroll
            for (int n1 = 0; n1 < N; ++n1) {
                ta[n1] = v[n1].x;
                tb[n1] = v[n1].y;
            }
#pragma unroll
            for (int w = 1; w < N; w *= 2)
#pragma unroll
                for (int i = 0; i + w < N; i += 2 * w) {
                    ta[i] += ta[i + w];
                    tb[i] += tb[i + w];
                }
            acc_a = (double)ta[0];
            acc_b = (double)tb[0];
        }
    }
    stage_twiddles(m, p.tw, F, F1, F2);
    __syncthreads();
    if (active) {
        tpr_dft<N, false>(v);
        const float2 *t = m.T + n2;  // T[k1 F2 + n2], lanes along n2
#pragma unroll
        for (int k1 = 1; k1 < N; ++k1) v[k1] = c_mul(v[k1], t[k1 * F2]);
        float2 *d = m.S + n2 * (NL + 1) + l;
#pragma unroll
        for (int k1 = 0; k1 < N; ++k1) d[k1 * GS] = v[k1];
    }
    return acc_a + acc_b;
}

// R2C B: group k1 -> DFT F2 -> bins k1 + F1 k2 in natural order (after every
// thread has read its group).
template <int N, int NL>
__device__ __forceinline__ void r2c_b(const TprSmem &m, int l, int k1, int F1, int GS, bool active)
{
    float2 v[N];
    if (active) {
        const float2 *grp = m.S + k1 * GS + l;
#pragma unroll
        for (int n2 = 0; n2 < N; ++n2) v[n2] = grp[n2 * (NL + 1)];
        tpr_dft<N, false>(v);
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int k2 = 0; k2 < N; ++k2) m.S[(k1 + F1 * k2) * (NL + 1) + l] = v[k2];
    }
}

template <int NL, int MAXT, int MINB, int MAXN>
__global__ void __launch_bounds__(MAXT, MINB) r2c_tpr_kernel(const GenRowPass p, int f1)
{
    constexpr int LS = NL + 1, NR = 2 * NL;
    extern __shared__ __align__(16) float2 tsm[];
    __shared__ double red[32];
    const int F = p.plan.F, F1 = f1, F2 = F / f1;
    const int GS = F2 * LS + ((F2 & 1) ^ 1);
    const TprSmem m = tpr_smem_layout(tsm, F, NL);
    const int r0 = blockIdx.x * NR;

    double acc = 0.0;
    {
        // A: thread (n2, l), positions fastest (coalesced row segments)
        const int n2 = threadIdx.x % F2, l = threadIdx.x / F2;
        switch (F1) {
#define VFD_R2C_A(n) \
    case n: if constexpr (n <= MAXN) acc = r2c_a<n, NL>(p, m, r0, l, n2, F2, GS, l < NL); break;
            VFD_TPR_SIZES(VFD_R2C_A)
#undef VFD_R2C_A
        default: break;
        }
    }
    __syncthreads();
    {
        // B: thread (l, k1), lines fastest
        const int l = threadIdx.x % NL, k1 = threadIdx.x / NL;
        switch (F2) {
#define VFD_R2C_B(n) \
    case n: if constexpr (n <= MAXN) r2c_b<n, NL>(m, l, k1, F1, GS, k1 < F1); break;
            VFD_TPR_SIZES(VFD_R2C_B)
#undef VFD_R2C_B
        default: break;
        }
    }
    __syncthreads();

    // split the two real rows' half spectra: warp per output row, lanes along k
    const int Fh = F / 2 + 1, NW = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = warp; q < NR; q += NW) {
        const int rr = r0 + q;
        if (rr >= p.nrows) continue;
        const int ln = q % NL;
        const int s1 = rr % p.rows_per_plane, s2 = rr / p.rows_per_plane;
        float2 *dst = p.cdst + (int64_t)s1 * p.c_s1 + (int64_t)s2 * p.c_s2;
        for (int k = lane; k < Fh; k += 32) {
            const float2 z = m.S[k * LS + ln];
            const float2 zc = m.S[(k == 0 ? 0 : F - k) * LS + ln];  // Z(-k)
            dst[k] = q < NL ? make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y))    // A(k)
                            : make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));  // B(k)
        }
    }
    tpr_block_sum(acc, p.mass_in, red);
}

// C2R B' (first pass).  The half spectra of the tile's 2 NL rows are first
// fetched with cp.async into the tile's own space as St[q][k] (row q < NL:
// row a of line q; else row b of line q - NL; Fh bins each): every load is in
// flight at once without holding registers.  Then thread (k1, l) builds the
// bins k1 + F1 k2 of z(k) = A(k) + i B(k) (z(k) = conj A(F-k) + i conj B(F-k)
// above F/2) from St, runs the inverse DFT F2 and the times conj w^(n2 k1)
// in registers, and after a barrier (St and the slots share the space)
// writes its slots.
template <int N, int NL>
__device__ __forceinline__ void c2r_b(const GenRowPass &p, const TprSmem &m, int r0, int l, int k1, int F1, int GS,
                                      bool active)
{
    const int F2 = N, F = F1 * F2, H = F / 2, Fh = H + 1;
    const int NW = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2 *St = m.S;
    for (int q = warp; q < 2 * NL; q += NW) {
        const RowRef r = row_ref(p, r0 + q, p.c_s1, p.c_s2);
        const float2 *src = p.csrc + r.off;
        for (int k = lane; k < Fh; k += 32) tpr_cp8(&St[q * Fh + k], r.ok ? src + k : p.csrc, r.ok);
    }
    tpr_cp_commit();
    stage_twiddles(m, p.tw, F, F1, F2);
    tpr_cp_wait_all();
    __syncthreads();
    float2 v[N];
    if (active) {
        const float2 *sa = St + l * Fh, *sb = St + (NL + l) * Fh;
#pragma unroll
        for (int k2 = 0; k2 < N; ++k2) {
            const int k = k1 + F1 * k2;
            const bool up = k > H;
            const int kk = up ? F - k : k;
            const float2 A = sa[kk], B = sb[kk];
            v[k2] = up ? make_float2(A.x + B.y, B.x - A.y) : make_float2(A.x - B.y, A.y + B.x);
        }
        tpr_dft<N, true>(v);
        const float2 *t = m.Tt + k1;  // Tt[n2 F1 + k1], lanes along k1
#pragma unroll
        for (int n2 = 1; n2 < N; ++n2) v[n2] = c_conj_mul(v[n2], t[n2 * F1]);
    }
    __syncthreads();
    if (active) {
        float2 *grp = m.S + k1 * GS + l;
#pragma unroll
        for (int n2 = 0; n2 < N; ++n2) grp[n2 * (NL + 1)] = v[n2];
    }
}

struct C2rSums {
    double leak = 0.0, conv = 0.0, out = 0.0;
};

// One real output value at x of a row: the crop / update epilogue; the
// values for the mass totals are added to the FP32 group sums gc and go.
__device__ __forceinline__ void c2r_store(const GenRowPass &p, float t, float *dst, float *drow, int x, float &gc,
                                          float &go)
{
    if (p.fuse_crop) {
        gc += t;
        t = p.keep * (t + p.b * p.k0);
        if (p.fuse_update) {
            t *= p.upd_scale;
            if (drow) {
                t += drow[x];
                drow[x] = 0.0f;
            }
        }
        go += t;
    }
    dst[x] = t;
}

// C2R A': slots of group n2 -> inverse DFT F1 -> positions n2 + F2 n1 of rows
// a (real part) and b (imaginary part); positions >= nstore go to the leak
// sum.  The mass sums run in FP32 over groups of 4 positions, each group
// widened once into the FP64 totals.
template <int N, int NL>
__device__ __forceinline__ void c2r_a(const GenRowPass &p, const TprSmem &m, int r0, int l, int n2, int F2, int GS,
                                      C2rSums &s)
{
    float2 v[N];
    const float2 *src = m.S + n2 * (NL + 1) + l;
#pragma unroll
    for (int k1 = 0; k1 < N; ++k1) v[k1] = src[k1 * GS];
    tpr_dft<N, true>(v);
    const RowRef ra = row_ref(p, r0 + l, p.r_s1, p.r_s2), rb = row_ref(p, r0 + NL + l, p.r_s1, p.r_s2);
    float *da = p.rdst + ra.off, *db = p.rdst + rb.off;
    float *ua = (p.fuse_update && p.dchem) ? p.dchem + ra.off : nullptr;
    float *ub = (p.fuse_update && p.dchem) ? p.dchem + rb.off : nullptr;
    float gc = 0.0f, go = 0.0f, gl = 0.0f;
#pragma unroll
    for (int n1 = 0; n1 < N; ++n1) {
        const int x = n2 + F2 * n1;
        if (x < p.nstore) {
            if (ra.ok) c2r_store(p, v[n1].x, da, ua, x, gc, go);
            if (rb.ok) c2r_store(p, v[n1].y, db, ub, x, gc, go);
        } else {
            gl += v[n1].x + v[n1].y;
        }
        if ((n1 & 3) == 3 || n1 == N - 1) {
            s.conv += (double)gc;
            s.out += (double)go;
            s.leak += (double)gl;
            gc = go = gl = 0.0f;
        }
    }
}

template <int NL, int MAXT, int MINB, int MAXN>
__global__ void __launch_bounds__(MAXT, MINB) c2r_tpr_kernel(const GenRowPass p, int f1)
{
    constexpr int NR = 2 * NL;
    extern __shared__ __align__(16) float2 tsm[];
    __shared__ double red[32];
    const int F = p.plan.F, F1 = f1, F2 = F / f1;
    const int GS = F2 * (NL + 1) + ((F2 & 1) ^ 1);
    const TprSmem m = tpr_smem_layout(tsm, F, NL);
    const int r0 = blockIdx.x * NR;
    {
        // B': thread (k1, l), bins fastest (coalesced half-spectrum segments)
        const int k1 = threadIdx.x % F1, l = threadIdx.x / F1;
        switch (F2) {
#define VFD_C2R_B(n) \
    case n: if constexpr (n <= MAXN) c2r_b<n, NL>(p, m, r0, l, k1, F1, GS, l < NL); break;
            VFD_TPR_SIZES(VFD_C2R_B)
#undef VFD_C2R_B
        default: break;
        }
    }
    __syncthreads();
    C2rSums s;
    {
        // A': thread (n2, l), positions fastest (coalesced row segments)
        const int n2 = threadIdx.x % F2, l = threadIdx.x / F2;
        if (l < NL) {
            switch (F1) {
#define VFD_C2R_A(n) \
    case n: if constexpr (n <= MAXN) c2r_a<n, NL>(p, m, r0, l, n2, F2, GS, s); break;
                VFD_TPR_SIZES(VFD_C2R_A)
#undef VFD_C2R_A
            default: break;
            }
        }
    }
    tpr_block_sum(s.leak, p.mass_leak, red);
    tpr_block_sum(s.conv, p.mass_conv, red);
    tpr_block_sum(s.out, p.mass_out, red);
}

// ---------------------------------------------------------------------------
// Host side.

static bool tpr_len(int n)
{
    switch (n) {
#define VFD_TPR_LEN(x) case x:
        VFD_TPR_SIZES(VFD_TPR_LEN)
#undef VFD_TPR_LEN
        return true;
    default: return false;
    }
}

int tpr_split(int F)
{
    int best = 0;
    for (int a = 2; a <= TPR_MAX && a * a <= F; ++a)
        if (F % a == 0 && tpr_len(a) && tpr_len(F / a)) best = a;  // largest f1 <= sqrt(F): smallest f2
    return best;
}

// Lines per tile: 8 (measured on B200, 512x256x384 world: 8-line tiles at 3
// resident CTAs beat 16-line tiles at one for the row and the column
// passes); VFD_TPR_ROW_NL / VFD_TPR_COL_NL = 16 select the 16-line kernels.
static int tpr_nl(bool rows)
{
    static int nl[2] = {-1, -1};
    if (nl[rows] < 0) {
        const char *e = getenv(rows ? "VFD_TPR_ROW_NL" : "VFD_TPR_COL_NL");
        nl[rows] = (e && atoi(e) == 16) ? 16 : 8;
    }
    return nl[rows];
}

// every pass gives each thread at most one group: NL * max(f1, f2) threads
static int tpr_threads(int F, int f1, int NL)
{
    const int g = f1 > F / f1 ? f1 : F / f1;
    return (NL * g + 31) / 32 * 32;
}

// the tile, tw, T and Tt
static size_t tpr_smem(int F, int NL) { return ((size_t)F * (NL + 1) + TPR_MAX + 3 * (size_t)F) * sizeof(float2); }

// The largest dynamic shared memory, once per kernel (one instantiation per
// kernel, so one flag each) and CUDA context.
template <auto KERNEL>
static cudaError_t tpr_attr()
{
    static thread_local unsigned long long ctx_done = 0;
    const unsigned long long ctx = current_context_id();
    if (ctx != 0 && ctx == ctx_done) return cudaSuccess;
    const cudaError_t e =
        cudaFuncSetAttribute(KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axis_smem_limit());
    if (e == cudaSuccess) ctx_done = ctx;
    return e;
}

template <int NL, int MAXT, int MINB, int MAXN>
static cudaError_t rows_nl(const GenRowPass &p, int f1, bool inverse, cudaStream_t st)
{
    cudaError_t e = inverse ? tpr_attr<c2r_tpr_kernel<NL, MAXT, MINB, MAXN>>() : tpr_attr<r2c_tpr_kernel<NL, MAXT, MINB, MAXN>>();
    if (e != cudaSuccess) return e;
    const int blocks = (p.nrows + 2 * NL - 1) / (2 * NL);
    if (blocks <= 0) return cudaSuccess;
    const int nt = tpr_threads(p.plan.F, f1, NL);
    const size_t sm = tpr_smem(p.plan.F, NL);
    if (nt > MAXT || sm > axis_smem_limit()) return cudaErrorInvalidConfiguration;
    if (inverse) c2r_tpr_kernel<NL, MAXT, MINB, MAXN><<<blocks, nt, sm, st>>>(p, f1);
    else r2c_tpr_kernel<NL, MAXT, MINB, MAXN><<<blocks, nt, sm, st>>>(p, f1);
    note_launch();
    return cudaGetLastError();
}

template <int NL, int MAXT, int MINB, int MAXN>
static cudaError_t cols_nl(const GenColPass &p, int f1, cudaStream_t st)
{
    cudaError_t e = tpr_attr<c2c_tpr_kernel<NL, MAXT, MINB, MAXN>>();
    if (e != cudaSuccess) return e;
    const int64_t blocks = (int64_t)p.nouter * ((p.nlines + NL - 1) / NL);
    if (blocks <= 0) return cudaSuccess;
    const int nt = tpr_threads(p.plan.F, f1, NL);
    const size_t sm = tpr_smem(p.plan.F, NL);
    if (nt > MAXT || sm > axis_smem_limit()) return cudaErrorInvalidConfiguration;
    c2c_tpr_kernel<NL, MAXT, MINB, MAXN><<<(unsigned)blocks, nt, sm, st>>>(p, f1);
    note_launch();
    return cudaGetLastError();
}

static bool tpr_split_ok(int F, int f1) { return f1 >= 2 && F % f1 == 0 && tpr_len(f1) && tpr_len(F / f1); }

// the 8-line kernels carry the DFT lengths up to 24 (what the general
// methods' length choice prefers); longer factors run on the 16-line kernels
static bool tpr_use16(bool rows, int F, int f1)
{
    const int g = f1 > F / f1 ? f1 : F / f1;
    return tpr_nl(rows) == 16 || g > 24;
}

cudaError_t launch_tpr_rows(const GenRowPass &p, int f1, bool inverse, cudaStream_t st)
{
    if (!tpr_split_ok(p.plan.F, f1)) return cudaErrorInvalidValue;
    if (tpr_use16(true, p.plan.F, f1)) return rows_nl<16, 512, 1, 32>(p, f1, inverse, st);
    return rows_nl<8, 256, 3, 24>(p, f1, inverse, st);
}

cudaError_t launch_tpr_cols(const GenColPass &p, int f1, cudaStream_t st)
{
    if (!tpr_split_ok(p.plan.F, f1)) return cudaErrorInvalidValue;
    if (tpr_use16(false, p.plan.F, f1)) return cols_nl<16, 512, 1, 32>(p, f1, st);
    // measured on B200 (512x256x384 world): the forward-only and inverse-only
    // passes run best at 4 resident CTAs (64 registers), the fused z pass and
    // the row passes at 3 (85 registers)
    return p.mode == GEN_FWD_MUL_INV ? cols_nl<8, 256, 3, 24>(p, f1, st) : cols_nl<8, 256, 4, 24>(p, f1, st);
}

}  // namespace vfd
