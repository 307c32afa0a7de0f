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
constexpr int OS_SCR = 64 + 8;  // float2 per group scratch (64 + pad)
constexpr int OS_RS = 36;       // y/z staging: floats per position row
constexpr int OS_MINB = 3;      // CTAs per SM (80 registers per thread)

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

// Forward FFT-64 of the 8 samples x[q] = s[t + 8q] of lane t of a group;
// on return lane t holds bins t + 8 k2 in x[k2].  scr: the group's scratch.
// All 32 lanes of the warp call it together (__syncwarp).
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
    int NPA;    // x pass: staged positions per line row (delta + NP, rounded up to 4)
    int RS;     // x pass: floats per staged line row
    int CS;     // x pass: floats per output line row
    int stage;  // floats per staging buffer
    int out;    // floats of the output staging
};

__host__ __device__ inline int os_round4mod16(int v) { return v + ((4 - v) % 16 + 16) % 16; }

__host__ __device__ inline OsGeom os_geom(int r, int C, bool xpass)
{
    OsGeom g;
    g.NP = C + 2 * r;
    g.delta = xpass ? ((-r) & 3) : 0;  // x: chunk inputs start at ofirst - r + ch C = -(r + delta) mod 4
    g.NPA = (g.delta + g.NP + 3) & ~3;
    g.RS = os_round4mod16(g.NPA);
    g.CS = os_round4mod16(C);
    g.stage = xpass ? 32 * g.RS : g.NP * OS_RS;
    g.out = xpass ? 32 * g.CS : C * OS_RS;
    return g;
}

// Issues the asynchronous copies of staging slots [0, send) for a chunk
// whose slot 0 is position pa.  Lines >= nreal and positions outside [0, n)
// are zero-filled.  x pass with vec: rows 16-byte aligned, pa and n
// multiples of 4 (a 4-position quad then lies wholly inside or outside the
// line).  y/z with vec: positions 16-byte aligned.
template <bool XP>
__device__ __forceinline__ void os_stage(float *stage, const OsJob &j, const OsGeom &G, const float *base,
                                         int nreal, int pa, int send, bool vec)
{
    const int n = j.n;
    const int64_t ls = j.line_stride, ps = j.pos_stride;
    if (XP) {
        if (vec) {
            const int row = threadIdx.x >> 3, k = threadIdx.x & 7;
            const bool rok = row < nreal;
            const float *src = base + (rok ? row : 0) * ls;
            float *dst = stage + row * G.RS;
#pragma unroll 2
            for (int s = 4 * k; s < send; s += 32) {
                const int p = pa + s;
                const bool v = rok && p >= 0 && p < n;
                cp_async16(dst + s, v ? src + p : base, v ? 16 : 0);
            }
        } else {
            const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
            for (int row = wp; row < 32; row += OS_NT / 32) {
                const bool rok = row < nreal;
                const float *src = base + (rok ? row : 0) * ls;
                float *dst = stage + row * G.RS;
                for (int s = lane; s < send; s += 32) {
                    const int p = pa + s;
                    const bool v = rok && p >= 0 && p < n;
                    cp_async4(dst + s, v ? src + p : base, v);
                }
            }
        }
    } else {
        if (vec) {
            const int k = threadIdx.x & 7, sub = threadIdx.x >> 3;
            const int vb = 4 * min(max(nreal - 4 * k, 0), 4);
            const float *src = base + 4 * k;
            float *dst = stage + 4 * k;
#pragma unroll 2
            for (int i = sub; i < send; i += OS_NT / 8) {
                const int p = pa + i;
                const bool v = vb > 0 && p >= 0 && p < n;
                cp_async16(dst + i * OS_RS, v ? src + (int64_t)p * ps : base, v ? vb : 0);
            }
        } else {
            const int col = threadIdx.x & 31, wp = threadIdx.x >> 5;
            const bool cok = col < nreal;
            const float *src = base + (cok ? col : 0) * ls;
            for (int i = wp; i < send; i += OS_NT / 32) {
                const int p = pa + i;
                const bool v = cok && p >= 0 && p < n;
                cp_async4(stage + i * OS_RS + col, v ? src + (int64_t)p * ps : base, v);
            }
        }
    }
}

template <bool XP>
__global__ void __launch_bounds__(OS_NT, OS_MINB) os_pass_kernel(const OsJob *__restrict__ jobs, int njobs)
{
    extern __shared__ __align__(16) float osm[];
    __shared__ double red[OS_NT / 32];
    __shared__ __align__(16) OsJob sj;
    __shared__ int sjob;

    // ---- job descriptor: found by one lane, copied by its warp -------------
    const int tile = blockIdx.x;
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = njobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (jobs[mid].tile_begin <= tile) lo = mid;
                else hi = mid - 1;
            }
            sjob = lo;
        }
        __syncwarp();
        const int *src = reinterpret_cast<const int *>(jobs + sjob);
        int *dst = reinterpret_cast<int *>(&sj);
        for (int i = threadIdx.x; i < (int)(sizeof(OsJob) / sizeof(int)); i += 32) dst[i] = src[i];
    }
    __syncthreads();

    const int n = sj.n, r = sj.r, L = sj.L, C = sj.C;
    const OsGeom G = os_geom(r, C, XP);
    float *const outs = osm + 2 * G.stage;
    float2 *const scr = reinterpret_cast<float2 *>(outs + G.out);

    const int local = tile - sj.tile_begin;
    const int outer = local / sj.tiles_per_outer;
    const int l0 = (local - outer * sj.tiles_per_outer) * 32;
    const int nreal = min(32, sj.nlines - l0);
    float *const base = sj.data + outer * sj.outer_stride + (int64_t)l0 * sj.line_stride;
    const float b = sj.b;
    const int64_t ls = sj.line_stride, ps = sj.pos_stride;
    const int nch = sj.nchunks, nblocks = sj.nblocks, ofirst = sj.ofirst;
    const bool aligned = (reinterpret_cast<uintptr_t>(base) & 15) == 0;
    const bool vec = XP ? (aligned && (ls & 3) == 0 && (n & 3) == 0 && (ofirst & 3) == 0)
                        : (aligned && ls == 1 && (ps & 3) == 0);

    // ---- per-lane constants of the FFT phase: group g = (pair, block) ------
    // The 4 groups of a warp share the block, so block-uniform branches are
    // warp-uniform (fft64_* synchronise the whole warp).
    const int g = threadIdx.x >> 3, t = threadIdx.x & 7;
    const int pair = g & 15, blk = g >> 4, seg0 = blk * L;
    float2 *const gs = scr + g * OS_SCR;
    float2 w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = c_tw64[(t * k) & 63];
    unsigned qmask = 0;  // samples t + 8q that are outputs of the block
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int i = t + 8 * q;
        if (i >= r && i < r + L) qmask |= 1u << q;
    }
    // constant-VF padding rule (x pass): rows of this pair inside the y/z box
    const bool masked = XP && sj.mask;
    bool in_a = false, in_b = false;
    if (masked) {
        const int la = 2 * pair;
        if (la < nreal) {
            const int rr = l0 + la, y = rr % sj.ny, z = rr / sj.ny;
            in_a = y >= sj.box_lo[1] && y < sj.box_hi[1] && z >= sj.box_lo[2] && z < sj.box_hi[2];
        }
        if (la + 1 < nreal) {
            const int rr = l0 + la + 1, y = rr % sj.ny, z = rr / sj.ny;
            in_b = y >= sj.box_lo[1] && y < sj.box_hi[1] && z >= sj.box_lo[2] && z < sj.box_hi[2];
        }
    }

    // staging slots a chunk of nb blocks needs
    auto slots = [&](int nb) { return XP ? ((G.delta + nb * L + 2 * r + 3) & ~3) : nb * L + 2 * r; };

    os_stage<XP>(osm, sj, G, base, nreal, ofirst - r - G.delta, slots(min(OS_M, nblocks)), vec);
    cp_async_commit();

    double acc_in = 0.0, acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int ch = 0; ch < nch; ++ch) {
        const int c0 = ofirst + ch * C, p0 = c0 - r;
        const int nb = min(OS_M, nblocks - ch * OS_M);
        float *const in = osm + (ch & 1) * G.stage;
        float *const nxt = osm + ((ch & 1) ^ 1) * G.stage;
        // chunk ch has landed, and every thread is done with the previous
        // chunk's outputs in `outs`
        cp_async_wait_all();
        __syncthreads();
        if (ch + 1 < nch) {
            const int pn = p0 + C;
            os_stage<XP>(nxt, sj, G, base, nreal, pn - G.delta, slots(min(OS_M, nblocks - (ch + 1) * OS_M)), vec);
            cp_async_commit();
        }

        // ---- one block of one pair per group: FFT-64, multiply, inverse ----
        if (blk < nb) {
            float2 x[8];
            if (XP) {
                const float *ra = in + (2 * pair) * G.RS + G.delta + seg0 + t;
                const float *rb = ra + G.RS;
#pragma unroll
                for (int q = 0; q < 8; ++q) x[q] = make_float2(ra[8 * q], rb[8 * q]);
            } else {
                const float2 *sp = reinterpret_cast<const float2 *>(in + (seg0 + t) * OS_RS) + pair;
#pragma unroll
                for (int q = 0; q < 8; ++q) x[q] = sp[q * 8 * (OS_RS / 2)];
            }
            if (masked) {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int p = p0 + seg0 + t + 8 * q;
                    const bool px = p >= sj.box_lo[0] && p < sj.box_hi[0];
                    x[q].x = (in_a && px) ? x[q].x - b : 0.0f;
                    x[q].y = (in_b && px) ? x[q].y - b : 0.0f;
                }
            }
            if (XP) {
                // input mass: each position of a line is one block's output once
                float s = 0.0f;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if ((qmask >> q) & 1u) s += x[q].x + x[q].y;
                acc_in += (double)s;
            }
            fft64_fwd(x, t, gs, w);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float h = sj.H[t + 8 * k];
                x[k] = make_float2(x[k].x * h, x[k].y * h);
            }
            fft64_inv(x, t, gs, w);
            const bool out_inside = c0 + seg0 >= 0 && c0 + seg0 + L <= n;
            const int j0 = seg0 + t - r;  // chunk output index of sample t (q = 0)
            float leak = 0.0f;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                if (!((qmask >> q) & 1u)) continue;
                const int j = j0 + 8 * q;
                if (!out_inside) {
                    const int o = c0 + j;
                    if (o < 0 || o >= n) {
                        if (o >= -r && o < n + r) leak += x[q].x + x[q].y;
                        continue;
                    }
                }
                if (XP) {
                    outs[(2 * pair) * G.CS + j] = x[q].x;
                    outs[(2 * pair + 1) * G.CS + j] = x[q].y;
                } else {
                    reinterpret_cast<float2 *>(outs + j * OS_RS)[pair] = x[q];
                }
            }
            acc_leak += (double)leak;
        }
        // chunk ch+1's reads of global memory are complete (every thread)
        // before any output of chunk ch overwrites its inputs
        cp_async_wait_all();
        __syncthreads();

        // ---- store outputs [max(c0, 0), min(c0 + nb L, n)) ------------------
        const int olo = max(c0, 0), ohi = min(c0 + nb * L, n);
        if (XP) {
            const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
            if (vec) {
                // olo is a multiple of 4, and so is ohi (n, or c0 + C)
                for (int row = wp; row < nreal; row += OS_NT / 32) {
                    float *dst = base + row * ls;
                    const float *sv = outs + row * G.CS;  // sv[o - c0]: output at position o
                    for (int o = olo + 4 * lane; o < ohi; o += 128) {
                        if (o + 4 <= ohi) {
                            *reinterpret_cast<float4 *>(dst + o) = *reinterpret_cast<const float4 *>(sv + (o - c0));
                        } else {
                            for (int k = o; k < ohi; ++k) dst[k] = sv[k - c0];
                        }
                    }
                }
            } else {
                for (int row = wp; row < nreal; row += OS_NT / 32) {
                    float *dst = base + row * ls;
                    const float *sv = outs + row * G.CS;
                    for (int o = olo + lane; o < ohi; o += 32) dst[o] = sv[o - c0];
                }
            }
        } else {
            const int jlo = olo - c0, jhi = ohi - c0;
            const bool last = sj.kind == PASS_Z;
            const float keep = sj.keep;
            if (vec) {
                const int k = threadIdx.x & 7, sub = threadIdx.x >> 3;
                const int valid = min(max(nreal - 4 * k, 0), 4);
                if (valid > 0) {
                    float *dq = base + 4 * k;
                    for (int j = jlo + sub; j < jhi; j += OS_NT / 8) {
                        float4 v = *reinterpret_cast<const float4 *>(outs + j * OS_RS + 4 * k);
                        float *dst = dq + (int64_t)(c0 + j) * ps;
                        if (last) {
                            float sc = v.x;
                            if (valid > 1) sc += v.y;
                            if (valid > 2) sc += v.z;
                            if (valid > 3) sc += v.w;
                            acc_conv += (double)sc;
                            v.x = keep * (v.x + b);
                            v.y = keep * (v.y + b);
                            v.z = keep * (v.z + b);
                            v.w = keep * (v.w + b);
                            float so = v.x;
                            if (valid > 1) so += v.y;
                            if (valid > 2) so += v.z;
                            if (valid > 3) so += v.w;
                            acc_out += (double)so;
                        }
                        if (valid == 4) {
                            *reinterpret_cast<float4 *>(dst) = v;
                        } else {
                            dst[0] = v.x;
                            if (valid > 1) dst[1] = v.y;
                            if (valid > 2) dst[2] = v.z;
                        }
                    }
                }
            } else {
                const int col = threadIdx.x & 31, wp = threadIdx.x >> 5;
                if (col < nreal) {
                    for (int j = jlo + wp; j < jhi; j += OS_NT / 32) {
                        float v = outs[j * OS_RS + col];
                        if (last) {
                            acc_conv += (double)v;
                            v = keep * (v + b);
                            acc_out += (double)v;
                        }
                        base[col + (int64_t)(c0 + j) * ps] = v;
                    }
                }
            }
        }
    }

    double *mass = sj.mass;
    if (XP) {
        os_block_sum(acc_in, mass + MS_INPUT, red);
        os_block_sum(acc_leak, mass + MS_LEAK_X, red);
    } else if (sj.kind == PASS_Y) {
        os_block_sum(acc_leak, mass + MS_LEAK_Y, red);
    } else {
        os_block_sum(acc_leak, mass + MS_LEAK_Z, red);
        os_block_sum(acc_conv, mass + MS_CONV, red);
        os_block_sum(acc_out, mass + MS_OUT, red);
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
        const size_t bytes =
            (size_t)(2 * g.stage + g.out) * sizeof(float) + (size_t)(OS_NT / 8) * OS_SCR * sizeof(float2);
        best = std::max(best, bytes);
    }
    return best;
}

template <bool XP>
static cudaError_t launch_os_t(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st)
{
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(os_pass_kernel<XP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)axis_smem_limit());
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    os_pass_kernel<XP><<<tiles, OS_NT, os_smem_bytes(rmin, XP ? PASS_X : PASS_Y), st>>>(jobs, njobs);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_os(const OsJob *jobs, int njobs, int tiles, int rmin, int axis, cudaStream_t st)
{
    if (tiles <= 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    bool ready;
    {
        std::lock_guard<std::mutex> lk(g_tw_mu);
        ready = dev >= 0 && dev < 64 && g_tw_done[dev];
    }
    if (!ready && (e = os_prepare()) != cudaSuccess) return e;
    if (axis == PASS_X) return launch_os_t<true>(jobs, njobs, tiles, rmin, st);
    return launch_os_t<false>(jobs, njobs, tiles, rmin, st);
}

}  // namespace vfd
