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
// and a chunk of OS_M consecutive blocks of those lines.  A group of 8 lanes
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

__global__ void __launch_bounds__(OS_NT, 2) os_pass_kernel(const OsJob *__restrict__ jobs, int njobs)
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
        double s, c;
        sincospi((double)threadIdx.x / 32.0, &s, &c);
        tw64[threadIdx.x] = make_float2((float)c, (float)-s);
    }
    __syncthreads();

    const int n = sj.n, r = sj.r, L = sj.L, C = sj.C;
    const int NP = C + 2 * r;                 // staged input positions
    float2 *in = osm;                         // [NP][OS_LS]
    float2 *out = in + NP * OS_LS;            // [C][OS_LS]
    float2 *scr = out + C * OS_LS;            // [32 groups][OS_SCR]
    float *inf = reinterpret_cast<float *>(in);
    float *outf = reinterpret_cast<float *>(out);

    const int local = tile - sj.tile_begin;
    const int outer = local / sj.tiles_per_outer;
    const int q0 = local - outer * sj.tiles_per_outer;
    const int lt = q0 / sj.nchunks, ch = q0 - lt * sj.nchunks;
    const int l0 = lt * 32;
    const int nreal = min(32, sj.nlines - l0);
    const int c0 = -r + ch * C;               // first output position of the chunk
    const int p0 = c0 - r;                    // first staged input position
    float *base = sj.data + outer * sj.outer_stride + (int64_t)l0 * sj.line_stride;
    const int kind = sj.kind;
    const float b = sj.b;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // ---- stage the input chunk (padding rule fused into the x pass) -----
    double acc_in = 0.0;
    if (kind == PASS_X) {
        // lane = position along the row: 128-byte coalesced reads
        const int xlo = sj.box_lo[0], xhi = sj.box_hi[0];
        for (int row = warp; row < 32; row += OS_NT / 32) {
            bool rowin = false;
            if (row < nreal) {
                const int rr = l0 + row;
                const int y = rr % sj.ny, z = rr / sj.ny;
                rowin = y >= sj.box_lo[1] && y < sj.box_hi[1] && z >= sj.box_lo[2] && z < sj.box_hi[2];
            }
            const float *src = base + (int64_t)row * sj.line_stride;
            const int sidx = 2 * (row & 15) + (row >> 4);
            constexpr int U = 4;
            for (int i0 = lane; i0 < NP; i0 += 32 * U) {
                float v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + 32 * u, p = p0 + i;
                    v[u] = (rowin && i < NP && p >= 0 && p < n) ? __ldg(src + p) : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + 32 * u, p = p0 + i;
                    if (i < NP) {
                        const float x = (rowin && p >= xlo && p < xhi) ? v[u] - b : 0.0f;
                        inf[i * 2 * OS_LS + sidx] = x;
                        if (p >= c0 && p < c0 + C) acc_in += (double)x;
                    }
                }
            }
        }
    } else {
        // lane = column: 128-byte coalesced reads of one position
        const int64_t ps = sj.pos_stride;
        const int sidx = 2 * (lane & 15) + (lane >> 4);
        const bool ok = lane < nreal;
        const float *src = base + (int64_t)lane * sj.line_stride;
        constexpr int U = 8;
        for (int i0 = warp; i0 < NP; i0 += (OS_NT / 32) * U) {
            float v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + (OS_NT / 32) * u, p = p0 + i;
                v[u] = (ok && i < NP && p >= 0 && p < n) ? __ldg(src + p * ps) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + (OS_NT / 32) * u;
                if (i < NP) inf[i * 2 * OS_LS + sidx] = v[u];
            }
        }
    }
    __syncthreads();

    // ---- blocks: FFT-64, multiply, inverse, keep L samples ----------------
    const int g = threadIdx.x >> 3, t = threadIdx.x & 7;
    float2 *gs = scr + g * OS_SCR;
    float2 w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = tw64[(t * k) & 63];
    float H[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) H[k] = sj.H[t + 8 * k];
    double acc_leak = 0.0;
    const int nitems = OS_PAIRS * OS_M;
    for (int u = g; u < nitems; u += OS_NT / 8) {
        // groups 2j, 2j+1 of a warp take pairs p, p + 8 (conflict-free staging reads)
        const int pair = ((u & 1) << 3) | ((u >> 1) & 7);
        const int blk = u >> 4;
        const int seg0 = blk * L;
        float2 x[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = in[(seg0 + t + 8 * q) * OS_LS + pair];
        fft64_fwd(x, t, gs, w);
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = make_float2(x[k].x * H[k], x[k].y * H[k]);
        fft64_inv(x, t, gs, w);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int i = t + 8 * q;
            if (i >= r && i < r + L) {
                const int j = seg0 + i - r;   // chunk output index
                const int o = c0 + j;
                if (o >= 0 && o < n) out[j * OS_LS + pair] = x[q];
                else acc_leak += (double)x[q].x + (double)x[q].y;
            }
        }
    }
    __syncthreads();

    // ---- store the chunk's outputs (baseline + decay + mass in the z pass) -
    double acc_conv = 0.0, acc_out = 0.0;
    const int jlo = max(0, -c0), jhi = min(C, n - c0);
    if (kind == PASS_X) {
        for (int row = warp; row < nreal; row += OS_NT / 32) {
            float *dst = base + (int64_t)row * sj.line_stride + c0;
            const int sidx = 2 * (row & 15) + (row >> 4);
            for (int j = jlo + lane; j < jhi; j += 32) dst[j] = outf[j * 2 * OS_LS + sidx];
        }
    } else if (lane < nreal) {
        const int64_t ps = sj.pos_stride;
        const int sidx = 2 * (lane & 15) + (lane >> 4);
        float *dst = base + (int64_t)lane * sj.line_stride;
        const bool last = kind == PASS_Z;
        const float keep = sj.keep;
        for (int j = jlo + warp; j < jhi; j += OS_NT / 32) {
            float v = outf[j * 2 * OS_LS + sidx];
            if (last) {
                acc_conv += (double)v;
                v = keep * (v + b);
                acc_out += (double)v;
            }
            dst[(int64_t)(c0 + j) * ps] = v;
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

size_t os_smem_bytes(int rmin)
{
    const int L = OS_N - 2 * rmin, C = OS_M * L;
    return ((size_t)(C + 2 * rmin) * OS_LS + (size_t)C * OS_LS + (size_t)(OS_NT / 8) * OS_SCR) * sizeof(float2);
}

cudaError_t launch_os(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st)
{
    if (tiles <= 0) return cudaSuccess;
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(os_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)axis_smem_limit());
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    os_pass_kernel<<<tiles, OS_NT, os_smem_bytes(rmin), st>>>(jobs, njobs);
    note_launch();
    return cudaGetLastError();
}

}  // namespace vfd
