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

// Dynamic shared memory of one axis-pass CTA for FFT length F and NL lines:
// F*(NL+1) interleaved complex values, F twiddles (float2), F multipliers.
inline size_t axis_smem_bytes(int F, int NL)
{
    return (size_t)F * (NL + 1) * sizeof(float2) + (size_t)F * sizeof(float2) + (size_t)F * sizeof(float);
}
inline size_t axis_smem_limit() { return 220 * 1024; }

// Kernel variants: (index, lines per tile NL, threads per line TL, max points
// per thread MAXP, min resident blocks per SM for the register budget).
#define VFD_AXIS_VARIANTS(X) \
    X(0, 8, 32, 24, 2)       \
    X(1, 8, 64, 16, 2)       \
    X(2, 16, 32, 16, 2)      \
    X(3, 16, 32, 24, 1)      \
    X(4, 8, 32, 40, 1)       \
    X(5, 16, 32, 40, 1)

struct AxisVariant {
    int nl, tl, maxp, minb;
};
constexpr AxisVariant kAxisVariants[] = {
#define VFD_VARIANT_ROW(i, NL, TL, MAXP, MINB) {NL, TL, MAXP, MINB},
    VFD_AXIS_VARIANTS(VFD_VARIANT_ROW)
#undef VFD_VARIANT_ROW
};
constexpr int kNumAxisVariants = sizeof(kAxisVariants) / sizeof(kAxisVariants[0]);

cudaError_t launch_axis(int variant, const AxisJob *jobs, int njobs, int tiles, int Fmax,
                        cudaStream_t st);
cudaError_t launch_deposit(const DepositJob *jobs, int njobs, const int32_t *idx, const float *amt,
                           int64_t total, int *err, cudaStream_t st);

// Zeroes blocks[b][0 .. counts[b]) for b < n (device arrays of pointers and counts).
cudaError_t launch_zero_blocks(double *const *blocks, const int *counts, int n, cudaStream_t st);

cudaError_t launch_synth_field(uint64_t key, double lo, double span, float *out, int64_t n, cudaStream_t st);

// FFT plan of length F (radices 8,7,5,4,3,2) that some kernel variant can run,
// and the preferred variant for it (need_nl = 0: any tile width).
bool plan_for_length(int F, FftPlan *p);
int variant_for_plan(const FftPlan &p, int need_nl);

cudaError_t launch_gradients(const float *const *chem, const float *col, const float *ela, float *fib, float *neu,
                             float *mac, int64_t n, cudaStream_t st);
cudaError_t launch_sample(const float *src, int nx, int ny, int nz, int stride, float scale, float *out,
                          cudaStream_t st);

void note_launch();

// Unique id of the calling thread's current CUDA context (0 when the driver
// does not tell): caches of device pointers are keyed by it, because a
// device reset loads the library into a new context.
unsigned long long current_context_id();

}  // namespace vfd
