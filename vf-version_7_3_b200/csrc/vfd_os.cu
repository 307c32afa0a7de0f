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
// [-r, n + r); outputs outside [0, n) are the mass pushed past the crop and
// are summed as the leak instead of being stored.
//
// Work split: a CTA owns 32 real lines (16 complex pairs: line q is the real
// part of pair q % 16 for q < 16, the imaginary part otherwise -- the kernel
// spectrum is real and even, so the pair's parts are convolved independently)
// over their whole length, processed in chunks of M consecutive blocks.  The
// field is updated in place: a chunk's 2r-sample input halo that overlaps
// the previous chunk's outputs is carried forward in shared memory before
// those outputs are stored, so no CTA ever reads a sample another chunk has
// already overwritten (and no two CTAs share a line).  A group of 8 lanes
// computes one (pair, block) FFT: lane t holds samples t + 8q (q = 0..7);
//   forward : DFT-8 over q in registers, twiddle w64^(t k1), transpose
//             through a swizzled per-group scratch (__syncwarp only), DFT-8
//             over t;  lane k1 then holds bins k1 + 8 k2 (k2 = 0..7)
//   multiply: by G64(k) / 64 (FP64-generated, stored FP32)
//   inverse : the mirror steps, back to samples t + 8q.
// Global <-> shared traffic uses the same interleaved [position][17] complex
// staging as the full-line kernel (conflict-free for the group pattern used).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include "vfd_internal.h"
#include "vfd_os.h"

namespace vfd {

constexpr int OS_NT = 256;             // threads per CTA: 32 groups of 8 lanes
constexpr int OS_PAIRS = 16;
constexpr int OS_LS = OS_PAIRS + 1;    // float2 per staged position
constexpr int OS_SCR = 64 + 8;         // float2 per group scratch (64 + pad)

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

// Forward FFT-64 of the 8 samples x[q] = s[t + 8q] of lane t of a group;
// on return lane t holds bins t + 8 k2 in x[k2].  scr: the group's scratch.
__device__ __forceinline__ void fft64_fwd(float2 (&x)[8], int t, float2 *scr, const float2 (&w)[8])
{
    Dft<8, false>::run(x);
#pragma unroll
    for (int k = 1; k < 8; ++k) x[k] = c_mul(x[k], w[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) scr[k * 8 + ((t + k) & 7)] = x[k];
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 8; ++s) x[s] = scr[t * 8 + ((s + t) & 7)];
    __syncwarp();
    Dft<8, false>::run(x);
}

// Inverse of fft64_fwd (unnormalised): lane t, x[k2] = bin t + 8 k2 in,
// samples t + 8q out in x[q].
__device__ __forceinline__ void fft64_inv(float2 (&x)[8], int t, float2 *scr, const float2 (&w)[8])
{
    Dft<8, true>::run(x);
#pragma unroll
    for (int s = 0; s < 8; ++s) scr[t * 8 + ((s + t) & 7)] = x[s];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = scr[k * 8 + ((t + k) & 7)];
    __syncwarp();
#pragma unroll
    for (int k = 1; k < 8; ++k) x[k] = c_mul(x[k], make_float2(w[k].x, -w[k].y));
    Dft<8, true>::run(x);
}

template <int M, int MINB>
__global__ void __launch_bounds__(OS_NT, MINB) os_pass_kernel(const OsJob *__restrict__ jobs, int njobs)
{
    extern __shared__ __align__(16) float2 osm[];
    __shared__ double red[OS_NT / 32];
    __shared__ OsJob sj;
    __shared__ float2 tw64[64];

    const int tile = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].tile_begin <= tile) lo = mid;
            else hi = mid - 1;
        }
        sj = jobs[lo];
    }
    if (threadIdx.x < 64) {
        double sn, cs;
        sincospi((double)threadIdx.x / 32.0, &sn, &cs);
        tw64[threadIdx.x] = make_float2((float)cs, (float)-sn);
    }
    __syncthreads();

    const int n = sj.n, r = sj.r, L = sj.L, C = sj.C;
    const int NP = C + 2 * r;                 // staged input positions per chunk
    float2 *in = osm;                         // [NP][OS_LS]
    float2 *out = in + NP * OS_LS;            // [C][OS_LS]
    float2 *scr = out + C * OS_LS;            // [32 groups][OS_SCR]
    float *inf = reinterpret_cast<float *>(in);
    float *outf = reinterpret_cast<float *>(out);

    // this CTA owns 32 lines of one outer index, whole length, all chunks
    const int local = tile - sj.tile_begin;
    const int outer = local / sj.tiles_per_outer;
    const int lt = local - outer * sj.tiles_per_outer;
    const int l0 = lt * 32;
    const int nreal = min(32, sj.nlines - l0);
    float *base = sj.data + outer * sj.outer_stride + (int64_t)l0 * sj.line_stride;
    const int kind = sj.kind;
    const float b = sj.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = OS_NT / 32;

    // per-lane constants of the FFT phase
    const int g = threadIdx.x >> 3, t = threadIdx.x & 7;
    float2 *gs = scr + g * OS_SCR;
    float2 w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = tw64[(t * k) & 63];
    unsigned qmask = 0;  // samples t + 8q that are outputs of a block
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int i = t + 8 * q;
        if (i >= r && i < r + L) qmask |= 1u << q;
    }

    // x-pass row state (lane = position; rows = lines of the tile)
    int xlo = 0, xhi = 0;
    unsigned rowin_mask = 0;  // bit row: row inside the padding rule's y/z range
    if (kind == PASS_X) {
        xlo = sj.box_lo[0];
        xhi = sj.box_hi[0];
        for (int row = 0; row < nreal; ++row) {
            const int rr = l0 + row;
            const int y = rr % sj.ny, z = rr / sj.ny;
            if (y >= sj.box_lo[1] && y < sj.box_hi[1] && z >= sj.box_lo[2] && z < sj.box_hi[2])
                rowin_mask |= 1u << row;
        }
    }
    const int64_t ps = sj.pos_stride;

    double acc_in = 0.0, acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int ch = 0; ch < sj.nchunks; ++ch) {
        const int c0 = -r + ch * C;           // first output position of the chunk
        const int p0 = c0 - r;                // first staged input position
        // positions [p0, p0 + 2r) were staged by the previous chunk (its last
        // 2r slots) before it overwrote anything; bring them forward and load
        // only the rest from global memory
        int ifirst = 0;
        if (ch > 0) {
            for (int i = threadIdx.x; i < 2 * r * OS_LS; i += OS_NT) in[i] = in[C * OS_LS + i];
            ifirst = 2 * r;
            __syncthreads();
        }
        const bool in_inside = p0 + ifirst >= 0 && p0 + NP <= n;
        // ---- stage the chunk's new input positions -------------------------
        if (kind == PASS_X) {
            // lane = position along the row: 128-byte coalesced reads
            for (int row = warp; row < 32; row += NW) {
                const bool rowin = (rowin_mask >> row) & 1u;
                const int sidx = 2 * (row & 15) + (row >> 4);
                const float *src = base + (int64_t)row * sj.line_stride + p0;
                float *dst = inf + sidx;
                const bool fast = rowin && p0 + ifirst >= xlo && p0 + NP <= xhi;
                constexpr int U = 4;
                for (int i0 = ifirst + lane; i0 < NP; i0 += 32 * U) {
                    float v[U];
                    if (fast) {
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            const int i = i0 + 32 * u;
                            v[u] = i < NP ? __ldg(src + i) - b : 0.0f;
                        }
                    } else {
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            const int i = i0 + 32 * u, p = p0 + i;
                            v[u] = (rowin && i < NP && p >= xlo && p < xhi) ? __ldg(src + i) - b : 0.0f;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + 32 * u;
                        if (i < NP) {
                            dst[i * 2 * OS_LS] = v[u];
                            acc_in += (double)v[u];  // every position is staged once
                        }
                    }
                }
            }
        } else {
            // lane = column: 128-byte coalesced reads of one position
            const int sidx = 2 * (lane & 15) + (lane >> 4);
            const bool ok = lane < nreal;
            const float *src = base + (int64_t)lane * sj.line_stride + (int64_t)(p0 + ifirst + warp) * ps;
            const int64_t step = (int64_t)NW * ps;
            float *dst = inf + (ifirst + warp) * 2 * OS_LS + sidx;
            constexpr int DST = NW * 2 * OS_LS;
            constexpr int U = 8;
            for (int i0 = ifirst + warp; i0 < NP; i0 += NW * U) {
                float v[U];
                if (in_inside) {
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        v[u] = (ok && i0 + NW * u < NP) ? __ldg(src + u * step) : 0.0f;
                } else {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int p = p0 + i0 + NW * u;
                        v[u] = (ok && i0 + NW * u < NP && p >= 0 && p < n) ? __ldg(src + u * step) : 0.0f;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (i0 + NW * u < NP) dst[u * DST] = v[u];
                src += U * step;
                dst += U * DST;
            }
        }
        __syncthreads();

        // ---- blocks: FFT-64, multiply, inverse, keep L samples -------------
        const bool out_inside = c0 >= 0 && c0 + C <= n;
        for (int u = g; u < OS_PAIRS * M; u += OS_NT / 8) {
            // groups 2j, 2j+1 of a warp take pairs p, p + 8 (conflict-free staging reads)
            const int pair = ((u & 1) << 3) | ((u >> 1) & 7);
            const int seg0 = (u >> 4) * L;
            const float2 *sp = in + (seg0 + t) * OS_LS + pair;
            float2 x[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) x[q] = sp[q * 8 * OS_LS];
            fft64_fwd(x, t, gs, w);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float h = sj.H[t + 8 * k];
                x[k] = make_float2(x[k].x * h, x[k].y * h);
            }
            fft64_inv(x, t, gs, w);
            float2 *op = out + (seg0 + t - r) * OS_LS + pair;  // sample t + 8q -> out row seg0 + t + 8q - r
            if (out_inside) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if ((qmask >> q) & 1u) op[q * 8 * OS_LS] = x[q];
            } else {
                const int o0 = c0 + seg0 + t - r;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if ((qmask >> q) & 1u) {
                        const int o = o0 + 8 * q;
                        if (o >= 0 && o < n) op[q * 8 * OS_LS] = x[q];
                        else acc_leak += (double)x[q].x + (double)x[q].y;
                    }
                }
            }
        }
        __syncthreads();

        // ---- store the chunk's outputs (baseline + decay + mass in the z pass)
        const int jlo = max(0, -c0), jhi = min(C, n - c0);
        if (kind == PASS_X) {
            for (int row = warp; row < nreal; row += NW) {
                float *dst = base + (int64_t)row * sj.line_stride + c0;
                const float *sv = outf + 2 * (row & 15) + (row >> 4);
                for (int j = jlo + lane; j < jhi; j += 32) dst[j] = sv[j * 2 * OS_LS];
            }
        } else if (lane < nreal) {
            const float *sv = outf + (jlo + warp) * 2 * OS_LS + 2 * (lane & 15) + (lane >> 4);
            float *dst = base + (int64_t)lane * sj.line_stride + (int64_t)(c0 + jlo + warp) * ps;
            const int64_t step = (int64_t)NW * ps;
            if (kind == PASS_Z) {
                const float keep = sj.keep;
                for (int j = jlo + warp; j < jhi; j += NW) {
                    float v = *sv;
                    acc_conv += (double)v;
                    v = keep * (v + b);
                    acc_out += (double)v;
                    *dst = v;
                    sv += NW * 2 * OS_LS;
                    dst += step;
                }
            } else {
                for (int j = jlo + warp; j < jhi; j += NW) {
                    *dst = *sv;
                    sv += NW * 2 * OS_LS;
                    dst += step;
                }
            }
        }
        // the next chunk's halo copy reads `in` (no longer read by the FFT
        // phase) and its FFT phase writes `out` only after the next barrier
    }

    double *mass = sj.mass;
    if (kind == PASS_X) {
        os_block_sum(acc_in, mass + MS_INPUT, red);
        os_block_sum(acc_leak, mass + MS_LEAK_X, red);
    } else if (kind == PASS_Y) {
        os_block_sum(acc_leak, mass + MS_LEAK_Y, red);
    } else {
        os_block_sum(acc_leak, mass + MS_LEAK_Z, red);
        os_block_sum(acc_conv, mass + MS_CONV, red);
        os_block_sum(acc_out, mass + MS_OUT, red);
    }
}

// ---------------------------------------------------------------------------
// Pipelined variant: the next chunk's new input positions are fetched with
// cp.async (4-byte, zero-filled outside the line) into the second of two
// staging buffers while the current chunk's FFTs run.  Used when staging
// needs no transform on load (zero padding: v = u); the input mass of the x
// pass is summed from the samples that are block outputs (each staged
// position inside the chunk's output range exactly once).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Issues the asynchronous staging of positions [ifirst, NP) of chunk (p0) into
// stage (float view).  Rows/columns beyond nreal and positions outside
// [0, n) are zero-filled.
__device__ __forceinline__ void os_stage_async(float *stage, const OsJob &j, float *base, int nreal, int p0,
                                               int ifirst, int NP)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = OS_NT / 32;
    const int n = j.n;
    if (j.kind == PASS_X) {
        for (int row = warp; row < 32; row += NW) {
            const bool ok = row < nreal;
            const float *src = base + (int64_t)(ok ? row : 0) * j.line_stride;
            float *dst = stage + 2 * (row & 15) + (row >> 4);
            for (int i = ifirst + lane; i < NP; i += 32) {
                const int p = p0 + i;
                const bool v = ok && p >= 0 && p < n;
                cp_async4(dst + i * 2 * OS_LS, v ? src + p : src, v);
            }
        }
    } else {
        const int64_t ps = j.pos_stride;
        const bool ok = lane < nreal;
        const float *src = base + (int64_t)(ok ? lane : 0) * j.line_stride;
        float *dst = stage + 2 * (lane & 15) + (lane >> 4);
        for (int i = ifirst + warp; i < NP; i += NW) {
            const int p = p0 + i;
            const bool v = ok && p >= 0 && p < n;
            cp_async4(dst + i * 2 * OS_LS, v ? src + (int64_t)p * ps : src, v);
        }
    }
}

template <int M, int MINB>
__global__ void __launch_bounds__(OS_NT, MINB) os_pass_pipe_kernel(const OsJob *__restrict__ jobs, int njobs)
{
    extern __shared__ __align__(16) float2 osm[];
    __shared__ double red[OS_NT / 32];
    __shared__ OsJob sj;
    __shared__ float2 tw64[64];

    const int tile = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].tile_begin <= tile) lo = mid;
            else hi = mid - 1;
        }
        sj = jobs[lo];
    }
    if (threadIdx.x < 64) {
        double sn, cs;
        sincospi((double)threadIdx.x / 32.0, &sn, &cs);
        tw64[threadIdx.x] = make_float2((float)cs, (float)-sn);
    }
    __syncthreads();

    const int n = sj.n, r = sj.r, L = sj.L, C = sj.C;
    const int NP = C + 2 * r;
    // two staging buffers [NP][OS_LS] at osm and osm + NP * OS_LS
    float2 *out = osm + 2 * NP * OS_LS;        // [C][OS_LS]
    float2 *scr = out + C * OS_LS;             // [32 groups][OS_SCR]
    float *outf = reinterpret_cast<float *>(out);

    const int local = tile - sj.tile_begin;
    const int outer = local / sj.tiles_per_outer;
    const int lt = local - outer * sj.tiles_per_outer;
    const int l0 = lt * 32;
    const int nreal = min(32, sj.nlines - l0);
    float *base = sj.data + outer * sj.outer_stride + (int64_t)l0 * sj.line_stride;
    const int kind = sj.kind;
    const float b = sj.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = OS_NT / 32;

    const int g = threadIdx.x >> 3, t = threadIdx.x & 7;
    float2 *gs = scr + g * OS_SCR;
    float2 w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = tw64[(t * k) & 63];
    unsigned qmask = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int i = t + 8 * q;
        if (i >= r && i < r + L) qmask |= 1u << q;
    }
    const int64_t ps = sj.pos_stride;
    const int nch = sj.nchunks;

    os_stage_async(reinterpret_cast<float *>(osm), sj, base, nreal, -2 * r, 0, NP);
    cp_async_commit();

    double acc_in = 0.0, acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int ch = 0; ch < nch; ++ch) {
        const int c0 = -r + ch * C, p0 = c0 - r;
        float2 *in = osm + (ch & 1) * NP * OS_LS;
        float2 *nxt = osm + ((ch & 1) ^ 1) * NP * OS_LS;
        // this chunk's samples have landed; every thread has also finished the
        // previous iteration (its halo copy out of `nxt` and its reads of `out`)
        cp_async_wait<0>();
        __syncthreads();
        if (ch + 1 < nch) {
            // next chunk: positions [2r, NP) from global memory (not yet
            // overwritten: this chunk stores only outputs below p0 + C + 2r)
            os_stage_async(reinterpret_cast<float *>(nxt), sj, base, nreal, p0 + C, 2 * r, NP);
            cp_async_commit();
        }

        const bool out_inside = c0 >= 0 && c0 + C <= n;
        for (int u = g; u < OS_PAIRS * M; u += OS_NT / 8) {
            const int pair = ((u & 1) << 3) | ((u >> 1) & 7);
            const int seg0 = (u >> 4) * L;
            const float2 *sp = in + (seg0 + t) * OS_LS + pair;
            float2 x[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) x[q] = sp[q * 8 * OS_LS];
            if (kind == PASS_X) {
                // input mass: the samples this block outputs (own positions)
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if ((qmask >> q) & 1u) acc_in += (double)x[q].x + (double)x[q].y;
            }
            fft64_fwd(x, t, gs, w);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float h = sj.H[t + 8 * k];
                x[k] = make_float2(x[k].x * h, x[k].y * h);
            }
            fft64_inv(x, t, gs, w);
            float2 *op = out + (seg0 + t - r) * OS_LS + pair;
            if (out_inside) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if ((qmask >> q) & 1u) op[q * 8 * OS_LS] = x[q];
            } else {
                const int o0 = c0 + seg0 + t - r;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if ((qmask >> q) & 1u) {
                        const int o = o0 + 8 * q;
                        if (o >= 0 && o < n) op[q * 8 * OS_LS] = x[q];
                        else acc_leak += (double)x[q].x + (double)x[q].y;
                    }
                }
            }
        }
        __syncthreads();
        // carry the next chunk's first 2r positions (disjoint from its async part)
        if (ch + 1 < nch)
            for (int i = threadIdx.x; i < 2 * r * OS_LS; i += OS_NT) nxt[i] = in[C * OS_LS + i];

        const int jlo = max(0, -c0), jhi = min(C, n - c0);
        if (kind == PASS_X) {
            for (int row = warp; row < nreal; row += NW) {
                float *dst = base + (int64_t)row * sj.line_stride + c0;
                const float *sv = outf + 2 * (row & 15) + (row >> 4);
                for (int j = jlo + lane; j < jhi; j += 32) dst[j] = sv[j * 2 * OS_LS];
            }
        } else if (lane < nreal) {
            const float *sv = outf + (jlo + warp) * 2 * OS_LS + 2 * (lane & 15) + (lane >> 4);
            float *dst = base + (int64_t)lane * sj.line_stride + (int64_t)(c0 + jlo + warp) * ps;
            const int64_t step = (int64_t)NW * ps;
            if (kind == PASS_Z) {
                const float keep = sj.keep;
                for (int j = jlo + warp; j < jhi; j += NW) {
                    float v = *sv;
                    acc_conv += (double)v;
                    v = keep * (v + b);
                    acc_out += (double)v;
                    *dst = v;
                    sv += NW * 2 * OS_LS;
                    dst += step;
                }
            } else {
                for (int j = jlo + warp; j < jhi; j += NW) {
                    *dst = *sv;
                    sv += NW * 2 * OS_LS;
                    dst += step;
                }
            }
        }
    }

    double *mass = sj.mass;
    if (kind == PASS_X) {
        os_block_sum(acc_in, mass + MS_INPUT, red);
        os_block_sum(acc_leak, mass + MS_LEAK_X, red);
    } else if (kind == PASS_Y) {
        os_block_sum(acc_leak, mass + MS_LEAK_Y, red);
    } else {
        os_block_sum(acc_leak, mass + MS_LEAK_Z, red);
        os_block_sum(acc_conv, mass + MS_CONV, red);
        os_block_sum(acc_out, mass + MS_OUT, red);
    }
}

int os_blocks_per_chunk()
{
    static int m = -1;
    if (m < 0) {
        const char *e = getenv("VFD_OS_M");
        m = (e && e[0] == '4') ? 4 : 2;
    }
    return m;
}

size_t os_smem_bytes(int rmin, int M)
{
    const int L = OS_N - 2 * rmin, C = M * L;
    return ((size_t)(C + 2 * rmin) * OS_LS + (size_t)C * OS_LS + (size_t)(OS_NT / 8) * OS_SCR) * sizeof(float2);
}

template <int M, int MINB>
static cudaError_t launch_os_t(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st)
{
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(os_pass_kernel<M, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)axis_smem_limit());
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    os_pass_kernel<M, MINB><<<tiles, OS_NT, os_smem_bytes(rmin, M), st>>>(jobs, njobs);
    note_launch();
    return cudaGetLastError();
}

static int os_min_blocks()
{
    static int m = -1;
    if (m < 0) {
        const char *e = getenv("VFD_OS_MINB");
        m = (e && e[0] == '3') ? 3 : 4;  // 4 blocks per SM (64 registers) measured faster on B200
    }
    return m;
}

size_t os_pipe_smem_bytes(int rmin, int M)
{
    const int L = OS_N - 2 * rmin, C = M * L;
    return ((size_t)2 * (C + 2 * rmin) * OS_LS + (size_t)C * OS_LS + (size_t)(OS_NT / 8) * OS_SCR) *
           sizeof(float2);
}

template <int M, int MINB>
static cudaError_t launch_os_pipe_t(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st)
{
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(os_pass_pipe_kernel<M, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)axis_smem_limit());
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    os_pass_pipe_kernel<M, MINB><<<tiles, OS_NT, os_pipe_smem_bytes(rmin, M), st>>>(jobs, njobs);
    note_launch();
    return cudaGetLastError();
}

bool os_pipe_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_OS_PIPE");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1;
}

cudaError_t launch_os_pipe(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st)
{
    if (tiles <= 0) return cudaSuccess;
    // the pipelined kernel measured fastest at 3 blocks per SM (80 registers)
    if (os_blocks_per_chunk() == 4) return launch_os_pipe_t<4, 2>(jobs, njobs, tiles, rmin, st);
    return launch_os_pipe_t<2, 3>(jobs, njobs, tiles, rmin, st);
}

cudaError_t launch_os(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st)
{
    if (tiles <= 0) return cudaSuccess;
    if (os_blocks_per_chunk() == 4) return launch_os_t<4, 2>(jobs, njobs, tiles, rmin, st);
    if (os_min_blocks() == 4) return launch_os_t<2, 4>(jobs, njobs, tiles, rmin, st);
    return launch_os_t<2, 3>(jobs, njobs, tiles, rmin, st);
}

}  // namespace vfd
