// vfd_os.h -- job descriptor of the overlap-save axis pass (vfd_os.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_axis.cuh"

namespace vfd {

constexpr int OS_N = 64;      // FFT length of one overlap-save block
constexpr int OS_RMAX = 16;   // largest kernel radius (L = 64 - 2r >= 32)
constexpr int OS_M = 2;       // blocks per chunk

// One (field, axis) pass; line addressing as in AxisJob.  A tile is 32 real
// lines of one outer index over their whole length (all chunks, in order).
struct OsJob {
    float *data;
    double *mass;
    int64_t line_stride, outer_stride, pos_stride;
    int n, nlines, nouter;
    int r, L, C;           // kernel radius, outputs per block (64 - 2r), outputs per chunk (OS_M L)
    int ofirst;            // first output position of chunk 0: -r, or below -r so that chunks
                           // start on multiples of 4 (x pass)
    int nblocks;           // ceil((n + r - ofirst) / L): blocks cover outputs [ofirst, n + r)
    int nchunks;           // ceil(nblocks / OS_M)
    int tiles_per_outer;   // ceil(nlines / 32)
    int tile_begin;
    int kind;              // PassKind
    int mask;              // x pass applies the constant-VF padding rule (b, box) to its samples
    float b, keep;
    int nx, ny;
    int box_lo[3], box_hi[3];
    float H[OS_N];         // G64(k) / 64, FP64-generated
};

// First output position of chunk 0 for a pass of radius r along `axis`.
inline int os_first_output(int r, int axis) { return axis == PASS_X ? -(r + ((-r) & 3)) : -r; }

// Uploads the FFT-64 twiddles to the current device; call outside any stream
// capture before the first launch on a device (world and batch creation do).
cudaError_t os_prepare();
// Dynamic shared memory of a launch whose jobs have radius >= rmin.
size_t os_smem_bytes(int rmin, int axis);
// All jobs of a launch belong to `axis`.
cudaError_t launch_os(const OsJob *jobs, int njobs, int tiles, int rmin, int axis, cudaStream_t st);

}  // namespace vfd
