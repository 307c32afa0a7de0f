// vfd_os.h -- job descriptor of the overlap-save axis pass (vfd_os.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_axis.cuh"

namespace vfd {

constexpr int OS_N = 64;      // FFT length of one overlap-save block
constexpr int OS_RMAX = 16;   // largest kernel radius (L = 64 - 2r >= 32)

// One (field, axis) pass; line addressing as in AxisJob.  A tile is 32 real
// lines of one outer index over their whole length (all chunks, in order).
struct OsJob {
    float *data;
    double *mass;
    int64_t line_stride, outer_stride, pos_stride;
    int n, nlines, nouter;
    int r, L, C;           // kernel radius, outputs per block (64 - 2r), outputs per chunk
    int nchunks;           // ceil((n + 2r) / C): chunks cover outputs [-r, n + r)
    int tiles_per_outer;   // ceil(nlines / 32)
    int tile_begin;
    int kind;              // PassKind
    float b, keep;
    int nx, ny;
    int box_lo[3], box_hi[3];
    float H[OS_N];         // G64(k) / 64, FP64-generated
};

// Blocks per CTA chunk (2 by default, 4 with VFD_OS_M=4); jobs must be built
// with the same value.
int os_blocks_per_chunk();
size_t os_smem_bytes(int rmin, int M);
cudaError_t launch_os(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st);
// Pipelined variant for jobs whose staging needs no transform (zero padding);
// VFD_OS_PIPE=0 disables it.
bool os_pipe_enabled();
cudaError_t launch_os_pipe(const OsJob *jobs, int njobs, int tiles, int rmin, cudaStream_t st);

}  // namespace vfd
