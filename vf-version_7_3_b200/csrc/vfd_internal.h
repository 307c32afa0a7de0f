// vfd_internal.h -- declarations shared by the host code and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_axis.cuh"

namespace vfd {

// One field's share of a source-deposit launch.
struct DepositJob {
    float *data;      // field (V floats)
    double *mass;     // MS_COUNT accounting doubles of the field
    int64_t begin;    // first source of this field in the concatenated list
    int64_t nvox;     // V, to reject out-of-range voxel indices
};

// Dynamic shared memory of one axis-pass CTA for FFT length F:
// two planes of F*LS floats, F twiddles (float2) and F multipliers.
inline size_t axis_smem_bytes(int F)
{
    return (size_t)F * LS * 2 * sizeof(float) + (size_t)F * sizeof(float2) + (size_t)F * sizeof(float);
}
inline size_t axis_smem_limit() { return 220 * 1024; }

// Kernel variants (threads per line TL, max points per thread MAXP):
//   0: (16, 24)  1: (32, 16)  2: (32, 24)  3: (16, 40)  4: (32, 40)
constexpr int kNumAxisVariants = 5;
inline int variant_tl(int v) { return (v == 0 || v == 3) ? 16 : 32; }
inline int variant_maxp(int v) { return v == 0 ? 24 : v == 1 ? 16 : v == 2 ? 24 : 40; }

cudaError_t launch_axis(int variant, const AxisJob *jobs, int njobs, int tiles, int Fmax,
                        cudaStream_t st);
cudaError_t launch_deposit(const DepositJob *jobs, int njobs, const int32_t *idx, const float *amt,
                           int64_t total, int *err, cudaStream_t st);

void note_launch();

}  // namespace vfd
