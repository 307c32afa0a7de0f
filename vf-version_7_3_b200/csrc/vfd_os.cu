// vfd_os.cu -- one axis of the separable FFT convolution by overlap-save
// with 64-point FFT blocks held in registers.
//
// A line of n samples convolved with a radius-r kernel is cut into blocks of
// L = 64 - 2r outputs.  Block b takes the 64 input samples starting r before
// its first output (zero outside [0, n)); the 64-point circular convolution
// of that segment with the wrapped kernel equals the linear convolution on
// the segment's samples r .. r+L-1 (no wrap reaches them), so each block is:
// forward FFT-64, multiply by the kernel's 64-point spectrum, inverse
// FFT-64, keep L samples -- the reference's pad / R2C / modulate / C2R / crop
// (Diffusion.cu:1731-1859) applied per block.  Blocks cover output positions
// [ofirst, n + r) with ofirst <= -r; outputs in [-r, 0) and [n, n + r) are
// the mass pushed past the crop and are summed as the leak instead of being
// stored (outputs further out are zero: no input reaches them).
//
// Work split: a CTA owns 32 real lines of one outer index over their whole
// length, processed in chunks of 2 blocks (C = 2L outputs).  Lines 2p and
// 2p+1 form complex pair p (real and imaginary part): the kernel spectrum is
// real and even, so one complex FFT convolves both independently.  A group
// of 8 lanes computes one (pair, block) FFT; the 32 groups of a CTA cover
// the 16 pairs x 2 blocks of a chunk.
//
// Pipeline and in-place update: while chunk ch is transformed, chunk ch+1's
// input (its whole window, halo included) is fetched with cp.async into the
// second staging buffer; every thread waits for those copies and the CTA
// synchronises before chunk ch's outputs are stored.  So no sample is read
// after a chunk of the same lines overwrote it, and no two CTAs share a line.
//
// Staging layouts (what keeps a voxel's cost close to its FFT's):
//   * y/z passes stage position rows of 36 floats (32 lines + 4 pad, 144
//     bytes): one 16-byte cp.async moves 4 lines of one position, one
//     16-byte store writes 4 lines back (the lines are contiguous in x);
//   * the x pass stages line rows (positions contiguous) from a window that
//     starts on a 16-byte boundary, `delta` positions before the chunk's
//     first input, and its chunks start on multiples of 4 (ofirst), so both
//     the copies in and the stores out move 16 bytes along x;
//   * line-row strides are = 4 (mod 16) floats, so the 4 groups of a warp
//     (consecutive pairs, one block) touch disjoint bank octets;
//   * the constant-VF padding rule of the x pass is applied in registers as
//     samples enter the FFT.
//
// FFT-64 of one pair, by a group of 8 lanes: lane t holds samples t + 8q;
//   forward : DFT-8 over q in registers, twiddle w64^(t k1), transpose
//             through a swizzled per-group scratch (__syncwarp only), DFT-8
//             over t;  lane k1 then holds bins k1 + 8 k2
//   multiply: by G64(k) / 64 (FP64-generated, stored FP32)
//   inverse : the mirror steps, back to samples t + 8q.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "vfd_internal.h"
#include "vfd_os.h"

namespace vfd {

constexpr int OS_NT = 256;      // threads per CTA: 32 groups of 8 lanes
constexpr int OS_SCR = 72;      // float2 per group scratch: 8 rows of 9
constexpr int OS_RS = 36;       // y/z staging: floats per position row

__constant__ float2 c_tw64[64];  // exp(-2 pi i m / 64), FP64-generated on the host

__device__ __forceinline__ double os_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void os_block_sum(double v, double *dst, double *red)
{
    v = os_warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < OS_NT / 32) ? red[l] : 0.0;
        v = os_warp_sum(v);
        if (l == 0 && v != 0.0) atomicAdd(dst, v);
    }
    __syncthreads();
}

// ---- packed FP32x2 complex arithmetic (one instruction per complex add,
// subtract or real scale; a - b is fma(b, -1, a), rounded once like a - b) --
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }

// DFT-4 in place; forward uses w4 = -i, inverse +i.
template <bool INV>
__device__ __forceinline__ void dft4p(float2 &a0, float2 &a1, float2 &a2, float2 &a3)
{
    const float2 t0 = p_add(a0, a2), t1 = p_sub(a0, a2);
    const float2 t2 = p_add(a1, a3), d = p_sub(a1, a3);
    a0 = p_add(t0, t2);
    a2 = p_sub(t0, t2);
    if (!INV) {  // t3 = -i d
        a1 = make_float2(t1.x + d.y, t1.y - d.x);
        a3 = make_float2(t1.x - d.y, t1.y + d.x);
    } else {     // t3 = +i d
        a1 = make_float2(t1.x - d.y, t1.y + d.x);
        a3 = make_float2(t1.x + d.y, t1.y - d.x);
    }
}

// DFT-8 in place (radix 2 x 4), w8 = exp(-+ i pi / 4).
template <bool INV>
__device__ __forceinline__ void dft8p(float2 (&v)[8])
{
    const float h = 0.707106781186547524400844362105f;
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4p<INV>(e0, e1, e2, e3);
    dft4p<INV>(o0, o1, o2, o3);
    if (!INV) {
        o1 = p_mul(make_float2(o1.x + o1.y, o1.y - o1.x), make_float2(h, h));
        o3 = p_mul(make_float2(o3.y - o3.x, o3.x + o3.y), make_float2(h, -h));
        v[2] = make_float2(e2.x + o2.y, e2.y - o2.x);  // o2 * -i
        v[6] = make_float2(e2.x - o2.y, e2.y + o2.x);
    } else {
        o1 = p_mul(make_float2(o1.x - o1.y, o1.x + o1.y), make_float2(h, h));
        o3 = p_mul(make_float2(o3.x + o3.y, o3.x - o3.y), make_float2(-h, h));
        v[2] = make_float2(e2.x - o2.y, e2.y + o2.x);  // o2 * +i
        v[6] = make_float2(e2.x + o2.y, e2.y - o2.x);
    }
    v[0] = p_add(e0, o0);
    v[4] = p_sub(e0, o0);
    v[1] = p_add(e1, o1);
    v[5] = p_sub(e1, o1);
    v[3] = p_add(e3, o3);
    v[7] = p_sub(e3, o3);
}

// Forward FFT-64 of the 8 samples x[q] = s[t + 8q] of lane t of a group;
// on return lane t holds bins t + 8 k2 in x[k2].  The group's scratch is 8
// rows of 9 float2; lane t writes column t (wr = scr + t) and reads row t
// (rd = scr + 9t), so every access is a base plus a constant offset.  All 32
// lanes of the warp call it together (__syncwarp).
__device__ __forceinline__ void fft64_fwd(float2 (&x)[8], float2 *wr, const float2 *rd, const float2 *w)
{
    dft8p<false>(x);
#pragma unroll
    for (int k = 1; k < 8; ++k) x[k] = c_mul(x[k], w[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) wr[9 * k] = x[k];
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 8; ++s) x[s] = rd[s];
    __syncwarp();
    dft8p<false>(x);
}

// Inverse of fft64_fwd (unnormalised): lane t, x[k2] = bin t + 8 k2 in,
// samples t + 8q out in x[q].
__device__ __forceinline__ void fft64_inv(float2 (&x)[8], float2 *wr, const float2 *rd, const float2 *w)
{
    dft8p<true>(x);
#pragma unroll
    for (int s = 0; s < 8; ++s) wr[9 * s] = x[s];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = rd[k];
    __syncwarp();
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        const float2 wk = w[k];
        x[k] = c_mul(x[k], make_float2(wk.x, -wk.y));
    }
    dft8p<true>(x);
}

// ---- asynchronous copies (zero-filled past the source size) ---------------
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async16(float *smem, const float *gmem, int bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared-memory geometry of one job (floats).
struct OsGeom {
    int NP;     // input positions of a full chunk: C + 2r
    int delta;  // x pass: the staged window starts delta positions before the chunk's first input
    int RS;     // x pass: floats per staged line row
    int stage;  // floats per staging buffer
};

__host__ __device__ inline int os_round4mod16(int v) { return v + ((4 - v) % 16 + 16) % 16; }

__host__ __device__ inline OsGeom os_geom(int r, int C, bool xpass)
{
    OsGeom g;
    g.NP = C + 2 * r;
    g.delta = xpass ? ((-r) & 3) : 0;  // x: chunk inputs start at ofirst - r + ch C = -(r + delta) mod 4
    g.RS = os_round4mod16((g.delta + g.NP + 3) & ~3);
    g.stage = xpass ? 32 * g.RS : g.NP * OS_RS;
    return g;
}

// Issues the asynchronous copies of staging slots [sfirst, send) for a chunk
// whose slot 0 is position pa.  Lines >= nreal and positions outside [0, n)
// are zero-filled.  x pass with vec: rows 16-byte aligned, pa, sfirst and n
// multiples of 4 (a 4-position quad then lies wholly inside or outside the
// line).  y/z with vec: positions 16-byte aligned.
template <bool XP>
__device__ __forceinline__ void os_stage(float *stage, const OsJob &j, const float *base, int nreal, int pa,
                                         int sfirst, int send, bool vec)
{
    const int n = j.n;
    const int64_t ls = j.line_stride, ps = j.pos_stride;
    if (XP) {
        if (vec) {
            // 8 threads per line row, 16 bytes (4 positions) each
            const int row = threadIdx.x >> 3, k = threadIdx.x & 7;
            const bool rok = row < nreal;
            const float *src = base + (rok ? row : 0) * ls + pa;
            float *dst = stage + row * j.RS;
            if (rok && pa + sfirst >= 0 && pa + send <= n) {
#pragma unroll 2
                for (int s = sfirst + 4 * k; s < send; s += 32) cp_async16(dst + s, src + s, 16);
            } else {
#pragma unroll 2
                for (int s = sfirst + 4 * k; s < send; s += 32) {
                    const bool v = rok && (unsigned)(pa + s) < (unsigned)n;
                    cp_async16(dst + s, v ? src + s : base, v ? 16 : 0);
                }
            }
        } else {
            const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
            for (int row = wp; row < 32; row += OS_NT / 32) {
                const bool rok = row < nreal;
                const float *src = base + (rok ? row : 0) * ls + pa;
                float *dst = stage + row * j.RS;
                for (int s = sfirst + lane; s < send; s += 32) {
                    const bool v = rok && (unsigned)(pa + s) < (unsigned)n;
                    cp_async4(dst + s, v ? src + s : base, v);
                }
            }
        }
    } else {
        if (vec) {
            // 8 threads per position row, 16 bytes (4 lines) each
            constexpr int STEP = OS_NT / 8;
            const int k = threadIdx.x & 7, sub = threadIdx.x >> 3;
            const int vb = 4 * min(max(nreal - 4 * k, 0), 4);
            int i = sfirst + sub;
            const float *src = base + 4 * k + (int64_t)(pa + i) * ps;
            float *dst = stage + i * OS_RS + 4 * k;
            const int64_t gstep = STEP * ps;
            if (vb == 16 && pa + sfirst >= 0 && pa + send <= n) {
#pragma unroll 2
                for (; i < send; i += STEP, src += gstep, dst += STEP * OS_RS) cp_async16(dst, src, 16);
            } else {
#pragma unroll 2
                for (; i < send; i += STEP, src += gstep, dst += STEP * OS_RS) {
                    const bool v = vb > 0 && (unsigned)(pa + i) < (unsigned)n;
                    cp_async16(dst, v ? src : base, v ? vb : 0);
                }
            }
        } else {
            const int col = threadIdx.x & 31, wp = threadIdx.x >> 5;
            const bool cok = col < nreal;
            const float *src = base + (cok ? col : 0) * ls;
            for (int i = sfirst + wp; i < send; i += OS_NT / 32) {
                const int p = pa + i;
                const bool v = cok && (unsigned)p < (unsigned)n;
                cp_async4(stage + i * OS_RS + col, v ? src + (int64_t)p * ps : base, v);
            }
        }
    }
}

// Staging slots a chunk of nb blocks reads.
__device__ __forceinline__ int os_slots(const OsJob &J, int nb, bool xpass)
{
    return xpass ? ((J.delta + nb * J.L + 2 * J.r + 3) & ~3) : nb * J.L + 2 * J.r;
}

__device__ __forceinline__ float *os_tile_base(const OsJob &J, const OsTileInfo &T)
{
    return J.data + T.outer * J.outer_stride + (int64_t)T.l0 * J.line_stride;
}

// Persistent pass: CTA c takes tiles c, c + grid, c + 2 grid, ... and walks
// their chunks as one stream of steps.  At the top of each step the next
// step's input is requested (the next chunk of this tile, or the first chunk
// of the next tile), so a tile's first load overlaps the previous tile's last
// chunk.  Tile records and job descriptors live in a ring of three shared
// slots (the CTA's k-th tile in slot k % 3); warp 0 fetches tile k + 2's
// during tile k's first step, when slot (k + 2) % 3 = (k - 1) % 3 is free.
// Mass partial sums are flushed per warp (warp reduction, one atomic per
// value) whenever the job changes.
template <bool XP, int MINB>
__global__ void __launch_bounds__(OS_NT, MINB)
    os_pass_kernel(const OsJob *__restrict__ jobs, const OsTileInfo *__restrict__ tiles, int ntiles, int stage_floats)
{
    extern __shared__ __align__(16) float osm[];
    __shared__ __align__(16) OsJob sj[3];
    __shared__ __align__(16) OsTileInfo st[3];
    __shared__ float2 tws[8 * 9];  // twiddles w64^(t k), row t padded to 9 (conflict-free rows)

    const int grid = gridDim.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int tile = blockIdx.x;
    if (tile >= ntiles) return;

    // warp 0: tile record and job descriptor of a tile into a slot
    auto fetch = [&](int slot, const OsTileInfo &ti) {
        if (lane == 0) st[slot] = ti;
        const float *src = reinterpret_cast<const float *>(jobs + ti.job);
        float *dst = reinterpret_cast<float *>(&sj[slot]);
        for (int i = lane; i < (int)(sizeof(OsJob) / 16); i += 32) cp_async16(dst + 4 * i, src + 4 * i, 16);
    };
    if (threadIdx.x < 64) tws[(threadIdx.x >> 3) * 9 + (threadIdx.x & 7)] = c_tw64[(threadIdx.x >> 3) * (threadIdx.x & 7)];
    if (warp == 0) {
        fetch(0, tiles[tile]);
        if (tile + grid < ntiles) fetch(1, tiles[tile + grid]);
        cp_async_commit();
    }
    cp_async_wait_all();
    __syncthreads();

    // ---- per-lane constants: group g = (pair, block) ----------------------
    // The 4 groups of a warp share the block, so block-uniform branches are
    // warp-uniform (fft64_* synchronise the whole warp).
    const int g = threadIdx.x >> 3, t = threadIdx.x & 7;
    const int pair = g & 15, blk = g >> 4;
    float2 *const gs = reinterpret_cast<float2 *>(osm + 2 * stage_floats) + g * OS_SCR;
    float2 *const wr = gs + t;
    const float2 *const rd = gs + 9 * t;
    const float2 *const w = tws + 9 * t;  // w[k] = w64^(t k)

    // first step: chunk 0 of the first tile
    {
        const OsJob &J = sj[0];
        const OsTileInfo T = st[0];
        os_stage<XP>(osm, J, os_tile_base(J, T), T.flags & 63, J.ofirst - J.r - J.delta, 0,
                     os_slots(J, min(OS_M, J.nblocks), XP), (T.flags >> 8) & 1);
        cp_async_commit();
    }

    double acc_in = 0.0, acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    auto flush = [&](const OsJob &J) {
        double *mass = J.mass;
        const double a0 = os_warp_sum(acc_in), a1 = os_warp_sum(acc_leak);
        const double a2 = os_warp_sum(acc_conv), a3 = os_warp_sum(acc_out);
        if (lane == 0) {
            if (XP) {
                if (a0 != 0.0) atomicAdd(mass + MS_INPUT, a0);
                if (a1 != 0.0) atomicAdd(mass + MS_LEAK_X, a1);
            } else if (J.kind == PASS_Y) {
                if (a1 != 0.0) atomicAdd(mass + MS_LEAK_Y, a1);
            } else {
                if (a1 != 0.0) atomicAdd(mass + MS_LEAK_Z, a1);
                if (a2 != 0.0) atomicAdd(mass + MS_CONV, a2);
                if (a3 != 0.0) atomicAdd(mass + MS_OUT, a3);
            }
        }
        acc_in = acc_leak = acc_conv = acc_out = 0.0;
    };

    int slot = 0, ch = 0, buf = 0;
    for (;;) {
        const OsJob &J = sj[slot];
        const int slot1 = slot == 2 ? 0 : slot + 1, slot2 = slot1 == 2 ? 0 : slot1 + 1;
        // this step's input has landed (copies and carried slots), every
        // thread is done with the previous step, and records fetched during
        // the previous step are visible
        cp_async_wait_all();
        __syncthreads();
        // warp 0: record of the CTA's tile after next (fetched after the FFT phase)
        OsTileInfo ti2;
        ti2.job = -1;
        if (warp == 0 && ch == 0 && tile + 2 * grid < ntiles) ti2 = tiles[tile + 2 * grid];

        const OsTileInfo T = st[slot];
        float *const base = os_tile_base(J, T);
        const int nreal = T.flags & 63;
        const int r = J.r, L = J.L, C = J.C, n = J.n;
        const int c0 = J.ofirst + ch * C, p0 = c0 - r;
        const int nb = min(OS_M, J.nblocks - ch * OS_M);
        float *const in = osm + buf * stage_floats;
        float *const nxt = osm + (buf ^ 1) * stage_floats;
        const bool same = ch + 1 < J.nchunks;
        const bool has_next = same || tile + grid < ntiles;

        // ---- this step's samples into registers first (their shared-memory
        // latency overlaps the requests below) ----------------------------
        const int seg0 = blk * L;
        const int64_t ls = J.line_stride, ps = J.pos_stride;
        const float b = J.b;
        const bool va = 2 * pair < nreal, vb = 2 * pair + 1 < nreal;  // real lines of this pair
        const unsigned qmask = J.qmask[t];  // samples t + 8q that are outputs of the block
        float2 x[8];
        if (blk < nb) {
            if (XP) {
                const float *ra = in + (2 * pair) * J.RS + J.delta + seg0 + t;
                const float *rb = ra + J.RS;
#pragma unroll
                for (int q = 0; q < 8; ++q) x[q] = make_float2(ra[8 * q], rb[8 * q]);
                if (J.mask) {
                    // constant-VF padding rule: rows inside the y/z box, positions inside [lo, hi)
                    bool in_a = false, in_b = false;
                    if (va) {
                        const int rr = T.l0 + 2 * pair, y = rr % J.ny, z = rr / J.ny;
                        in_a = y >= J.box_lo[1] && y < J.box_hi[1] && z >= J.box_lo[2] && z < J.box_hi[2];
                    }
                    if (vb) {
                        const int rr = T.l0 + 2 * pair + 1, y = rr % J.ny, z = rr / J.ny;
                        in_b = y >= J.box_lo[1] && y < J.box_hi[1] && z >= J.box_lo[2] && z < J.box_hi[2];
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int p = p0 + seg0 + t + 8 * q;
                        const bool px = p >= J.box_lo[0] && p < J.box_hi[0];
                        x[q].x = (in_a && px) ? x[q].x - b : 0.0f;
                        x[q].y = (in_b && px) ? x[q].y - b : 0.0f;
                    }
                }
                // input mass: each position of a line is one block's output once
                float2 s2 = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if ((qmask >> q) & 1u) s2 = p_add(s2, x[q]);
                acc_in += (double)((va ? s2.x : 0.0f) + (vb ? s2.y : 0.0f));
            } else {
                const float2 *sp = reinterpret_cast<const float2 *>(in + (seg0 + t) * OS_RS) + pair;
#pragma unroll
                for (int q = 0; q < 8; ++q) x[q] = sp[q * 8 * (OS_RS / 2)];
            }
        }

        // ---- request the next step's input ---------------------------------
        if (same) {
            // this tile's next chunk, slots [hs, ..): positions >= c0 + C,
            // which this step does not store
            const int hs = J.hs;
            os_stage<XP>(nxt, J, base, nreal, p0 + C - J.delta, hs, os_slots(J, min(OS_M, J.nblocks - (ch + 1) * OS_M), XP),
                         (T.flags >> 8) & 1);
            cp_async_commit();
            // slots [0, hs): inputs this step overwrites, carried in shared memory
            if (XP) {
                const int row = threadIdx.x >> 3, c = threadIdx.x & 7;  // hs <= 16: 4 float4 per row
                if (4 * c < hs)
                    reinterpret_cast<float4 *>(nxt + row * J.RS)[c] =
                        reinterpret_cast<const float4 *>(in + row * J.RS + C)[c];
            } else {
                const float4 *hsrc = reinterpret_cast<const float4 *>(in + C * OS_RS);
                float4 *hdst = reinterpret_cast<float4 *>(nxt);
                for (int i = threadIdx.x; i < hs * (OS_RS / 4); i += OS_NT) hdst[i] = hsrc[i];
            }
        } else if (has_next) {
            // first chunk of the next tile (other lines: no overlap with this step's stores)
            const OsJob &Jn = sj[slot1];
            const OsTileInfo Tn = st[slot1];
            os_stage<XP>(nxt, Jn, os_tile_base(Jn, Tn), Tn.flags & 63, Jn.ofirst - Jn.r - Jn.delta, 0,
                         os_slots(Jn, min(OS_M, Jn.nblocks), XP), (Tn.flags >> 8) & 1);
            cp_async_commit();
        }

        // ---- one block of one pair per group: FFT-64, multiply, inverse,
        // outputs straight to global memory -------------------------------
        if (blk < nb) {
            fft64_fwd(x, wr, rd, w);
#pragma unroll
            for (int q = 0; q < 8; ++q) x[q] = p_mul(x[q], J.HH[t + 8 * q]);
            fft64_inv(x, wr, rd, w);

            const int ob = c0 + seg0 + t - r;  // position of sample t (q = 0)
            const bool inside = c0 + seg0 >= 0 && c0 + seg0 + L <= n;
            const bool zlast = !XP && J.kind == PASS_Z;
            // y/z outputs of a pair go out as one 8-byte store when aligned
            const bool st2 = !XP && vb && ((reinterpret_cast<uintptr_t>(base) & 7) == 0) && ((ps & 1) == 0);
            const float2 keep2 = make_float2(J.keep, J.keep), b2 = make_float2(b, b);
            float2 lk2 = make_float2(0.0f, 0.0f), cv2 = lk2, ot2 = lk2;
            if (inside) {
                // every kept sample is stored: addresses are a base plus constants
                if (XP) {
                    float *da = base + (2 * pair) * ls + ob;
                    float *db = da + ls;
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (!((qmask >> q) & 1u)) continue;
                        if (va) da[8 * q] = x[q].x;
                        if (vb) db[8 * q] = x[q].y;
                    }
                } else {
                    float *d = base + 2 * pair + (int64_t)ob * ps;
                    const int64_t step = 8 * ps;
#pragma unroll
                    for (int q = 0; q < 8; ++q, d += step) {
                        if (!((qmask >> q) & 1u)) continue;
                        float2 v = x[q];
                        if (zlast) {
                            cv2 = p_add(cv2, v);
                            v = p_mul(p_add(v, b2), keep2);
                            ot2 = p_add(ot2, v);
                        }
                        if (st2) {
                            *reinterpret_cast<float2 *>(d) = v;
                        } else {
                            if (va) d[0] = v.x;
                            if (vb) d[1] = v.y;
                        }
                    }
                }
            } else if (XP) {
                float *da = base + (2 * pair) * ls;
                float *db = da + ls;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (!((qmask >> q) & 1u)) continue;
                    const int o = ob + 8 * q;
                    if (o >= 0 && o < n) {
                        if (va) da[o] = x[q].x;
                        if (vb) db[o] = x[q].y;
                    } else if (o >= -r && o < n + r) {
                        lk2 = p_add(lk2, x[q]);
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (!((qmask >> q) & 1u)) continue;
                    const int o = ob + 8 * q;
                    if (o >= 0 && o < n) {
                        float *d = base + 2 * pair + (int64_t)o * ps;
                        float2 v = x[q];
                        if (zlast) {
                            cv2 = p_add(cv2, v);
                            v = p_mul(p_add(v, b2), keep2);
                            ot2 = p_add(ot2, v);
                        }
                        if (st2) {
                            *reinterpret_cast<float2 *>(d) = v;
                        } else {
                            if (va) d[0] = v.x;
                            if (vb) d[1] = v.y;
                        }
                    } else if (o >= -r && o < n + r) {
                        lk2 = p_add(lk2, x[q]);
                    }
                }
            }
            acc_leak += (double)((va ? lk2.x : 0.0f) + (vb ? lk2.y : 0.0f));
            if (zlast) {
                acc_conv += (double)((va ? cv2.x : 0.0f) + (vb ? cv2.y : 0.0f));
                acc_out += (double)((va ? ot2.x : 0.0f) + (vb ? ot2.y : 0.0f));
            }
        }

        if (ti2.job >= 0) {  // warp 0: the tile after next into the free slot
            fetch(slot2, ti2);
            cp_async_commit();
        }
        if (!has_next) {
            flush(J);
            break;
        }
        if (same) {
            ++ch;
        } else {
            if (sj[slot1].mass != J.mass) flush(J);
            slot = slot1;
            tile += grid;
            ch = 0;
        }
        buf ^= 1;
    }
}

void os_finish_job(OsJob &j)
{
    const OsGeom g = os_geom(j.r, j.C, j.kind == PASS_X);
    j.delta = g.delta;
    j.RS = g.RS;
    j.hs = j.r + g.delta;
    for (int t = 0; t < 8; ++t) {
        unsigned m = 0;
        for (int q = 0; q < 8; ++q) {
            const int i = t + 8 * q;
            if (i >= j.r && i < j.r + j.L) m |= 1u << q;
        }
        j.qmask[t] = (unsigned char)m;
    }
}

void os_append_tiles(const OsJob &j, int job, std::vector<OsTileInfo> &out)
{
    const bool xpass = j.kind == PASS_X;
    for (int outer = 0; outer < j.nouter; ++outer)
        for (int lt = 0; lt < j.tiles_per_outer; ++lt) {
            OsTileInfo ti;
            ti.job = job;
            ti.outer = outer;
            ti.l0 = lt * 32;
            const int nreal = std::min(32, j.nlines - ti.l0);
            const uintptr_t base = reinterpret_cast<uintptr_t>(j.data) +
                                   sizeof(float) * (uintptr_t)(outer * j.outer_stride + (int64_t)ti.l0 * j.line_stride);
            const bool aligned = (base & 15) == 0;
            const bool vec = xpass ? (aligned && (j.line_stride & 3) == 0 && (j.n & 3) == 0 && (j.ofirst & 3) == 0)
                                   : (aligned && j.line_stride == 1 && (j.pos_stride & 3) == 0);
            ti.flags = nreal | (vec ? 1 << 8 : 0);
            out.push_back(ti);
        }
}

static std::mutex g_tw_mu;
static bool g_tw_done[64];

cudaError_t os_prepare()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_tw_mu);
    if (g_tw_done[dev]) return cudaSuccess;
    float2 tw[64];
    for (int m = 0; m < 64; ++m) {
        const double a = 6.283185307179586476925286766559 * m / 64.0;
        tw[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    e = cudaMemcpyToSymbol(c_tw64, tw, sizeof(tw));
    if (e == cudaSuccess) g_tw_done[dev] = true;
    return e;
}

size_t os_smem_bytes(int rmin, int axis)
{
    size_t best = 0;
    for (int r = std::max(rmin, 0); r <= OS_RMAX; ++r) {
        const OsGeom g = os_geom(r, OS_M * (OS_N - 2 * r), axis == PASS_X);
        const size_t bytes = (size_t)(2 * g.stage) * sizeof(float) + (size_t)(OS_NT / 8) * OS_SCR * sizeof(float2);
        best = std::max(best, bytes);
    }
    return best;
}

static int os_min_blocks()
{
    static int m = -1;
    if (m < 0) {
        const char *ev = getenv("VFD_OS_MINB");
        m = (ev && ev[0] == '4') ? 4 : 3;
    }
    return m;
}

int os_default_ctas_per_sm() { return os_min_blocks(); }

template <bool XP, int MINB>
static cudaError_t launch_os_t(const OsJob *jobs, const OsTileInfo *tiles, int ntiles, int rmin, cudaStream_t st)
{
    static std::mutex mu;
    static int configured[64] = {};  // 1 + resident CTAs per SM at the configured size
    static size_t configured_smem[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    const size_t smem = os_smem_bytes(rmin, XP ? PASS_X : PASS_Y);
    int per_sm = 0, nsm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (configured[dev] == 0 || configured_smem[dev] != smem) {
            e = cudaFuncSetAttribute(os_pass_kernel<XP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)axis_smem_limit());
            if (e != cudaSuccess) return e;
            int b = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, os_pass_kernel<XP, MINB>, OS_NT, smem);
            if (e != cudaSuccess) return e;
            configured[dev] = 1 + std::max(b, 1);
            configured_smem[dev] = smem;
        }
        per_sm = configured[dev] - 1;
    }
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int grid = std::min(ntiles, per_sm * nsm);
    int stage_floats = 0;
    for (int r = std::max(rmin, 0); r <= OS_RMAX; ++r)
        stage_floats = std::max(stage_floats, os_geom(r, OS_M * (OS_N - 2 * r), XP).stage);
    os_pass_kernel<XP, MINB><<<grid, OS_NT, smem, st>>>(jobs, tiles, ntiles, stage_floats);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_os(const OsJob *jobs, const OsTileInfo *tiles, int ntiles, int rmin, int axis, cudaStream_t st,
                      int ctas_per_sm)
{
    if (ntiles <= 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    bool ready;
    {
        std::lock_guard<std::mutex> lk(g_tw_mu);
        ready = dev >= 0 && dev < 64 && g_tw_done[dev];
    }
    if (!ready && (e = os_prepare()) != cudaSuccess) return e;
    if ((ctas_per_sm > 0 ? ctas_per_sm : os_min_blocks()) == 4) {
        if (axis == PASS_X) return launch_os_t<true, 4>(jobs, tiles, ntiles, rmin, st);
        return launch_os_t<false, 4>(jobs, tiles, ntiles, rmin, st);
    }
    if (axis == PASS_X) return launch_os_t<true, 3>(jobs, tiles, ntiles, rmin, st);
    return launch_os_t<false, 3>(jobs, tiles, ntiles, rmin, st);
}

}  // namespace vfd
