// vfd_kernels.cu -- device kernels of the diffusion path.
//
//  axis_pass_kernel  one axis of the separable FFT convolution for a list of
//                    (field, axis) jobs: load (with the padding rule fused),
//                    forward FFT, multiply by the real heat-kernel spectrum,
//                    inverse FFT, crop (with baseline, decay and FP64 mass
//                    fused into the z pass).  Replaces, for one axis,
//                    padDataConstantVF3D + cufftExecR2C + modulateAndNormalize3D
//                    + cufftExecC2R + unpadResult3D (Diffusion.cu:1731-1859).
//  deposit_kernel    agents' point sources u[idx] += amt with warp-aggregated
//                    atomics and FP64 per-field source totals (the dChem part
//                    of WHChemical::update, WHChemical.cpp:420-450).
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_axis.cuh"
#include "vfd_internal.h"

namespace vfd {

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide FP64 sum, one atomicAdd per block into *dst (skipped when 0).
template <int NT>
__device__ __forceinline__ void block_sum_atomic(double v, double *dst, double *red)
{
    v = warp_sum_d(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < NT / 32) ? red[l] : 0.0;
        v = warp_sum_d(v);
        if (l == 0 && v != 0.0) atomicAdd(dst, v);
    }
    __syncthreads();
}

template <int TL, int MAXP>
__global__ void __launch_bounds__(NL *TL) axis_pass_kernel(const AxisJob *__restrict__ jobs, int njobs)
{
    constexpr int NT = NL * TL;
    extern __shared__ __align__(16) float smem[];
    __shared__ double red[NT / 32];
    __shared__ AxisJob sj;

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
    __syncthreads();

    const int F = sj.plan.F;
    const int n = sj.n;
    float *re = smem;
    float *im = re + F * LS;
    float2 *tw = reinterpret_cast<float2 *>(im + F * LS);
    float *G = reinterpret_cast<float *>(tw + F);
    for (int i = threadIdx.x; i < F; i += NT) {
        tw[i] = sj.tw[i];
        G[i] = sj.spec[i];
    }

    const int local = tile - sj.tile_begin;
    const int outer = local / sj.tiles_per_outer;
    const int l0 = (local - outer * sj.tiles_per_outer) * (2 * NL);
    const int nreal = min(2 * NL, sj.nlines - l0);
    float *base = sj.data + outer * sj.outer_stride + (int64_t)l0 * sj.line_stride;
    const int kind = sj.kind;
    const float b = sj.b;

    // ---- load (padding rule fused) ---------------------------------------
    double acc_in = 0.0;
    if (kind == PASS_X) {
        const int ny = sj.ny;
        for (int q = 0; q < 2 * NL; ++q) {
            float *plane = (q < NL) ? re : im;
            const int ln = q & (NL - 1);
            bool rowin = false;
            if (q < nreal) {
                const int row = l0 + q;
                const int y = row % ny, z = row / ny;
                rowin = y >= sj.box_lo[1] && y < sj.box_hi[1] && z >= sj.box_lo[2] && z < sj.box_hi[2];
            }
            const float *src = base + (int64_t)q * sj.line_stride;
            for (int pos = threadIdx.x; pos < n; pos += NT) {
                float v = 0.0f;
                if (rowin && pos >= sj.box_lo[0] && pos < sj.box_hi[0]) v = src[pos] - b;
                plane[pos * LS + ln] = v;
                acc_in += (double)v;
            }
        }
    } else {
        const int64_t ps = sj.pos_stride;
        for (int idx = threadIdx.x; idx < n * 2 * NL; idx += NT) {
            const int q = idx & (2 * NL - 1);
            const int pos = idx >> 5;
            const float v = (q < nreal) ? base[q * sj.line_stride + pos * ps] : 0.0f;
            ((q < NL) ? re : im)[pos * LS + (q & (NL - 1))] = v;
        }
    }
    for (int i = n * LS + threadIdx.x; i < F * LS; i += NT) {
        re[i] = 0.0f;
        im[i] = 0.0f;
    }
    __syncthreads();

    // ---- forward FFT, spectrum multiply, inverse FFT ---------------------
    const int line = threadIdx.x & (NL - 1);
    const int tj = threadIdx.x / NL;
    fft_lines<MAXP, TL, false>(re, im, sj.plan, line, tj, tw);
    for (int i = threadIdx.x; i < F * NL; i += NT) {
        const int k = i / NL, l = i & (NL - 1);
        const float g = G[k];
        re[k * LS + l] *= g;
        im[k * LS + l] *= g;
    }
    __syncthreads();
    fft_lines<MAXP, TL, true>(re, im, sj.plan, line, tj, tw);

    // ---- crop / store (baseline + decay + mass fused into the z pass) ----
    double acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int i = threadIdx.x; i < (F - n) * NL; i += NT) {
        const int p = (n + i / NL) * LS + (i & (NL - 1));
        acc_leak += (double)re[p] + (double)im[p];
    }
    if (kind == PASS_X) {
        for (int q = 0; q < nreal; ++q) {
            const float *plane = (q < NL) ? re : im;
            const int ln = q & (NL - 1);
            float *dst = base + (int64_t)q * sj.line_stride;
            for (int pos = threadIdx.x; pos < n; pos += NT) dst[pos] = plane[pos * LS + ln];
        }
    } else {
        const int64_t ps = sj.pos_stride;
        const bool last = (kind == PASS_Z);
        const float keep = sj.keep;
        for (int idx = threadIdx.x; idx < n * 2 * NL; idx += NT) {
            const int q = idx & (2 * NL - 1);
            const int pos = idx >> 5;
            if (q < nreal) {
                float t = ((q < NL) ? re : im)[pos * LS + (q & (NL - 1))];
                if (last) {
                    acc_conv += (double)t;
                    t = keep * (t + b);
                    acc_out += (double)t;
                }
                base[q * sj.line_stride + pos * ps] = t;
            }
        }
    }

    double *mass = sj.mass;
    if (kind == PASS_X) {
        block_sum_atomic<NT>(acc_in, mass + MS_INPUT, red);
        block_sum_atomic<NT>(acc_leak, mass + MS_LEAK_X, red);
    } else if (kind == PASS_Y) {
        block_sum_atomic<NT>(acc_leak, mass + MS_LEAK_Y, red);
    } else {
        block_sum_atomic<NT>(acc_leak, mass + MS_LEAK_Z, red);
        block_sum_atomic<NT>(acc_conv, mass + MS_CONV, red);
        block_sum_atomic<NT>(acc_out, mass + MS_OUT, red);
    }
}

// ---------------------------------------------------------------------------
// Source deposit.  Thread i handles source i of the concatenated list; its
// job (field) is found by binary search on the jobs' begin offsets.  Lanes of
// a warp that hit the same (field, voxel) are combined before one atomicAdd.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) deposit_kernel(const DepositJob *__restrict__ jobs, int njobs,
                                                      const int32_t *__restrict__ idx,
                                                      const float *__restrict__ amt, int64_t total,
                                                      int *__restrict__ err)
{
    __shared__ double fsum[8];
    __shared__ int fbase;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 8) fsum[threadIdx.x] = 0.0;

    bool active = i < total;
    int j = 0;
    int32_t vox = 0;
    float a = 0.0f;
    if (active) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].begin <= i) lo = mid;
            else hi = mid - 1;
        }
        j = lo;
        vox = idx[i];
        a = amt[i];
        if (vox < 0 || (int64_t)vox >= jobs[j].nvox) {
            atomicOr(err, 1);
            active = false;
        }
    }
    if (threadIdx.x == 0) {
        int lo = 0, hi = njobs - 1;
        const int64_t i0 = (int64_t)blockIdx.x * blockDim.x;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].begin <= i0) lo = mid;
            else hi = mid - 1;
        }
        fbase = lo;
    }
    __syncthreads();

    const unsigned long long key =
        active ? (((unsigned long long)(unsigned)j << 32) | (unsigned)vox) : ~0ull;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    float s = a;
    if (__any_sync(0xffffffffu, active && __popc(peers) > 1)) {
        s = 0.0f;
        for (int src = 0; src < 32; ++src) {
            const float v = __shfl_sync(0xffffffffu, a, src);
            if ((peers >> src) & 1u) s += v;
        }
    }
    const int leader = __ffs(peers) - 1;
    if (active && lane == leader) {
        atomicAdd(jobs[j].data + vox, s);
        const int slot = j - fbase;
        if (slot >= 0 && slot < 8) atomicAdd(&fsum[slot], (double)s);
        else atomicAdd(jobs[j].mass + MS_SOURCES, (double)s);
    }
    __syncthreads();
    if (threadIdx.x < 8 && fbase + (int)threadIdx.x < njobs && fsum[threadIdx.x] != 0.0)
        atomicAdd(jobs[fbase + threadIdx.x].mass + MS_SOURCES, fsum[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
template <int TL, int MAXP>
static cudaError_t launch_axis_t(const AxisJob *jobs, int njobs, int tiles, int Fmax, cudaStream_t st)
{
    const size_t sm = axis_smem_bytes(Fmax);
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(axis_pass_kernel<TL, MAXP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)axis_smem_limit());
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    axis_pass_kernel<TL, MAXP><<<tiles, NL * TL, sm, st>>>(jobs, njobs);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_axis(int variant, const AxisJob *jobs, int njobs, int tiles, int Fmax, cudaStream_t st)
{
    if (tiles <= 0) return cudaSuccess;
    switch (variant) {
    case 0: return launch_axis_t<16, 24>(jobs, njobs, tiles, Fmax, st);
    case 1: return launch_axis_t<32, 16>(jobs, njobs, tiles, Fmax, st);
    case 2: return launch_axis_t<32, 24>(jobs, njobs, tiles, Fmax, st);
    case 3: return launch_axis_t<16, 40>(jobs, njobs, tiles, Fmax, st);
    case 4: return launch_axis_t<32, 40>(jobs, njobs, tiles, Fmax, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_deposit(const DepositJob *jobs, int njobs, const int32_t *idx, const float *amt,
                           int64_t total, int *err, cudaStream_t st)
{
    if (total <= 0) return cudaSuccess;
    const int64_t blocks = (total + 255) / 256;
    deposit_kernel<<<(unsigned)blocks, 256, 0, st>>>(jobs, njobs, idx, amt, total, err);
    note_launch();
    return cudaGetLastError();
}

}  // namespace vfd
