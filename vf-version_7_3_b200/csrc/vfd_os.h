// vfd_os.h -- job descriptor of the overlap-save axis pass (vfd_os.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_axis.cuh"

namespace vfd {

constexpr int OS_N = 64;      // FFT length of one overlap-save block
constexpr int OS_M = 4;       // blocks per CTA chunk
constexpr int OS_RMAX = 16;   // largest kernel radius (L = 64 - 2r >= 32)

// One (field, axis) pass; line addressing as in AxisJob.  A tile is 32 real
// lines x one chunk of OS_M blocks; tiles are ordered (outer, line tile, chunk).
struct OsJob {
    float *data;
    double *mass;
    int64_t line_stride, outer_stride, pos_stride;
    int n, nlines, nouter;
    int r, L, C;           // kernel radius, outputs per block (64 - 2r), outputs per chunk
    int nchunks;           // ceil((n + 2r) / C): chunks cover outputs [-r, n + r)
    int tiles_per_outer;   // ceil(nlines / 32) * nchunks
    int tile_begin;
    int kind;              // PassKind
    float b, keep;
    int nx, ny;
    int box_lo[3], box_hi[3];
    float H[OS_N];         // G64(k) / 64, FP64-generated
};

size_t os_smem_bytes(int rmin);
cudaError_t launch_os(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st);

}  // namespace vfd
