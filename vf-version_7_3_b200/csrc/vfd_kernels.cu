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

// Loads / stores map one real line of the tile to each lane (NR = 2*NL real
// lines), position groups to the rest of the block, and keep U loads in
// flight per thread.  Real line rl of the tile is complex line rl % NL,
// component rl / NL.
template <int NL, int TL, int MAXP, int MINB>
__global__ void __launch_bounds__(NL *TL, MINB) axis_pass_kernel(const AxisJob *__restrict__ jobs, int njobs)
{
    constexpr int NT = NL * TL;
    constexpr int LS = NL + 1;
    constexpr int NR = 2 * NL;
    constexpr int NPG = NT / NR;
    constexpr int U = 8;
    extern __shared__ __align__(16) float2 smem2[];
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
    float2 *S = smem2;
    float *Sf = reinterpret_cast<float *>(smem2);
    float2 *tw = S + F * LS;
    float *G = reinterpret_cast<float *>(tw + F);
    for (int i = threadIdx.x; i < F; i += NT) {
        tw[i] = sj.tw[i];
        G[i] = sj.spec[i];
    }

    const int local = tile - sj.tile_begin;
    const int outer = local / sj.tiles_per_outer;
    const int l0 = (local - outer * sj.tiles_per_outer) * NR;
    const int nreal = min(NR, sj.nlines - l0);
    float *base = sj.data + outer * sj.outer_stride + (int64_t)l0 * sj.line_stride;
    const int kind = sj.kind;
    const float b = sj.b;
    const int rl = threadIdx.x % NR;       // real line of this lane
    const int pg = threadIdx.x / NR;       // position group
    const int sidx = 2 * (rl % NL) + rl / NL;  // float offset of (line, component)
    const bool lane_ok = rl < nreal;
    float *lsrc = base + (int64_t)rl * sj.line_stride;

    // ---- load (padding rule fused) ---------------------------------------
    double acc_in = 0.0;
    if (kind == PASS_X) {
        // positions contiguous: float4 along the line when aligned
        bool rowin = false;
        if (lane_ok) {
            const int row = l0 + rl;
            const int y = row % sj.ny, z = row / sj.ny;
            rowin = y >= sj.box_lo[1] && y < sj.box_hi[1] && z >= sj.box_lo[2] && z < sj.box_hi[2];
        }
        const int xlo = sj.box_lo[0], xhi = sj.box_hi[0];
        const bool vec = ((n & 3) == 0) && ((sj.line_stride & 3) == 0) &&
                         ((reinterpret_cast<uintptr_t>(sj.data) & 15) == 0);
        if (vec) {
            const int nc = n >> 2;
            for (int c0 = pg; c0 < nc; c0 += NPG * U) {
                float4 r[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int c = c0 + u * NPG;
                    r[u] = (rowin && c < nc) ? __ldg(reinterpret_cast<const float4 *>(lsrc) + c)
                                             : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int c = c0 + u * NPG;
                    if (c < nc) {
                        const float e[4] = {r[u].x, r[u].y, r[u].z, r[u].w};
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int pos = 4 * c + i;
                            const float v = (rowin && pos >= xlo && pos < xhi) ? e[i] - b : 0.0f;
                            Sf[pos * 2 * LS + sidx] = v;
                            acc_in += (double)v;
                        }
                    }
                }
            }
        } else {
            for (int p0 = pg; p0 < n; p0 += NPG * U) {
                float r[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int p = p0 + u * NPG;
                    r[u] = (rowin && p < n) ? __ldg(lsrc + p) : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int p = p0 + u * NPG;
                    if (p < n) {
                        const float v = (rowin && p >= xlo && p < xhi) ? r[u] - b : 0.0f;
                        Sf[p * 2 * LS + sidx] = v;
                        acc_in += (double)v;
                    }
                }
            }
        }
    } else {
        const int64_t ps = sj.pos_stride;
        for (int p0 = pg; p0 < n; p0 += NPG * U) {
            float r[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int p = p0 + u * NPG;
                r[u] = (lane_ok && p < n) ? __ldg(lsrc + p * ps) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int p = p0 + u * NPG;
                if (p < n) Sf[p * 2 * LS + sidx] = r[u];
            }
        }
    }
    for (int i = n * LS + threadIdx.x; i < F * LS; i += NT) S[i] = make_float2(0.f, 0.f);
    __syncthreads();

    // ---- forward FFT, spectrum multiply, inverse FFT ---------------------
    const int line = threadIdx.x % NL;
    const int tj = threadIdx.x / NL;
    fft_lines<MAXP, TL, NL, false>(S, sj.plan, line, tj, tw);
    for (int i = threadIdx.x; i < F * NL; i += NT) {
        const int k = i / NL, l = i % NL;
        const float g = G[k];
        float2 &x = S[k * LS + l];
        x.x *= g;
        x.y *= g;
    }
    __syncthreads();
    fft_lines<MAXP, TL, NL, true>(S, sj.plan, line, tj, tw);

    // ---- crop / store (baseline + decay + mass fused into the z pass) ----
    double acc_leak = 0.0, acc_conv = 0.0, acc_out = 0.0;
    for (int i = threadIdx.x; i < (F - n) * NL; i += NT) {
        const float2 x = S[(n + i / NL) * LS + (i % NL)];
        acc_leak += (double)x.x + (double)x.y;
    }
    if (lane_ok) {
        if (kind == PASS_X) {
            float *dst = lsrc;
            const bool vec = ((n & 3) == 0) && ((sj.line_stride & 3) == 0) &&
                             ((reinterpret_cast<uintptr_t>(sj.data) & 15) == 0);
            if (vec) {
                const int nc = n >> 2;
                for (int c = pg; c < nc; c += NPG) {
                    float4 o;
                    o.x = Sf[(4 * c + 0) * 2 * LS + sidx];
                    o.y = Sf[(4 * c + 1) * 2 * LS + sidx];
                    o.z = Sf[(4 * c + 2) * 2 * LS + sidx];
                    o.w = Sf[(4 * c + 3) * 2 * LS + sidx];
                    reinterpret_cast<float4 *>(dst)[c] = o;
                }
            } else {
                for (int p = pg; p < n; p += NPG) dst[p] = Sf[p * 2 * LS + sidx];
            }
        } else {
            const int64_t ps = sj.pos_stride;
            const bool last = (kind == PASS_Z);
            const float keep = sj.keep;
            for (int p = pg; p < n; p += NPG) {
                float t = Sf[p * 2 * LS + sidx];
                if (last) {
                    acc_conv += (double)t;
                    t = keep * (t + b);
                    acc_out += (double)t;
                }
                lsrc[p * ps] = t;
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
    const bool lead = active && lane == leader;
    if (lead) atomicAdd(jobs[j].data + vox, s);
    // FP64 source totals: one shared add per warp when the warp's sources
    // belong to one field (the common case), else one per leader
    const int j0 = __shfl_sync(0xffffffffu, j, 0);
    if (__all_sync(0xffffffffu, !active || j == j0)) {
        const double ws = warp_sum_d(lead ? (double)s : 0.0);
        if (lane == 0 && ws != 0.0) {
            const int slot = j0 - fbase;
            if (slot >= 0 && slot < 8) atomicAdd(&fsum[slot], ws);
            else atomicAdd(jobs[j0].mass + MS_SOURCES, ws);
        }
    } else if (lead) {
        const int slot = j - fbase;
        if (slot >= 0 && slot < 8) atomicAdd(&fsum[slot], (double)s);
        else atomicAdd(jobs[j].mass + MS_SOURCES, (double)s);
    }
    __syncthreads();
    if (threadIdx.x < 8 && fbase + (int)threadIdx.x < njobs && fsum[threadIdx.x] != 0.0)
        atomicAdd(jobs[fbase + threadIdx.x].mass + MS_SOURCES, fsum[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Device copy of the synthetic field generator (vfd_synth_field): the same
// splitmix64 stream and the same IEEE double operations (no contraction), so
// host and device produce identical fields.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t d_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__global__ void synth_field_kernel(uint64_t key, double lo, double span, float *out, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t z = d_mix64(key + ((uint64_t)i + 1) * 0x9e3779b97f4a7c15ULL);
        const double u = __dmul_rn((double)(z >> 11), 1.0 / 9007199254740992.0);
        out[i] = (float)__dadd_rn(lo, __dmul_rn(span, u));
    }
}

cudaError_t launch_synth_field(uint64_t key, double lo, double span, float *out, int64_t n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    synth_field_kernel<<<(unsigned)blocks, 256, 0, st>>>(key, lo, span, out, n);
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
template <int NL, int TL, int MAXP, int MINB>
static cudaError_t launch_axis_t(const AxisJob *jobs, int njobs, int tiles, int Fmax, cudaStream_t st)
{
    const size_t sm = axis_smem_bytes(Fmax, NL);
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(axis_pass_kernel<NL, TL, MAXP, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)axis_smem_limit());
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    axis_pass_kernel<NL, TL, MAXP, MINB><<<tiles, NL * TL, sm, st>>>(jobs, njobs);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_axis(int variant, const AxisJob *jobs, int njobs, int tiles, int Fmax, cudaStream_t st)
{
    if (tiles <= 0) return cudaSuccess;
    switch (variant) {
#define VFD_VARIANT_CASE(i, NL, TL, MAXP, MINB) \
    case i: return launch_axis_t<NL, TL, MAXP, MINB>(jobs, njobs, tiles, Fmax, st);
        VFD_AXIS_VARIANTS(VFD_VARIANT_CASE)
#undef VFD_VARIANT_CASE
    default: return cudaErrorInvalidValue;
    }
}

// Zeroes the FP64 accounting blocks of many worlds in one launch (block b:
// blocks[b], counts[b] doubles) -- a batch's per-substep reset.
__global__ void zero_blocks_kernel(double *const *blocks, const int *counts, int n)
{
    for (int b = blockIdx.x; b < n; b += gridDim.x)
        for (int i = threadIdx.x; i < counts[b]; i += blockDim.x) blocks[b][i] = 0.0;
}

cudaError_t launch_zero_blocks(double *const *blocks, const int *counts, int n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    zero_blocks_kernel<<<n < 1024 ? n : 1024, 64, 0, st>>>(blocks, counts, n);
    note_launch();
    return cudaGetLastError();
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
