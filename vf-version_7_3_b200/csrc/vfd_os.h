// vfd_os.h -- job descriptor of the overlap-save axis pass (vfd_os.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "vfd_axis.cuh"

namespace vfd {

constexpr int OS_N = 64;      // FFT length of one overlap-save block
constexpr int OS_RMAX = 16;   // largest kernel radius (L = 64 - 2r >= 32)
constexpr int OS_M = 2;       // blocks per chunk

// One (field, axis) pass; line addressing as in AxisJob.  A tile is 32 real
// lines of one outer index over their whole length (all chunks, in order).
struct alignas(16) OsJob {
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
    // shared-memory geometry (host-computed, see os_geom in vfd_os.cu)
    int delta;             // x pass: staged window starts delta positions before a chunk's first input
    int RS;                // x pass: floats per staged line row
    int hs;                // staging slots carried from one chunk to the next: r + delta
    unsigned char qmask[8];  // lane t of a group: bit q set when sample t + 8q is a block output
    float2 HH[OS_N];       // (G64(k) / 64) twice, FP64-generated
};
static_assert(sizeof(OsJob) % 16 == 0, "OsJob is copied in 16-byte pieces");

// First output position of chunk 0 for a pass of radius r along `axis`.
inline int os_first_output(int r, int axis) { return axis == PASS_X ? -(r + ((-r) & 3)) : -r; }

// A tile of a persistent launch: its job, position and lines.
struct OsTileInfo {
    int job;    // index into the launch's job array
    int outer;  // outer index of the tile's lines
    int l0;     // first line within the outer index
    int flags;  // bits 0-5: real lines (1..32); bit 8: 16-byte copies apply
};

// Fills the host-computed geometry fields of a job whose other fields are set.
void os_finish_job(OsJob &j);
// Appends the tiles of job `job` (j) to `out`.
void os_append_tiles(const OsJob &j, int job, std::vector<OsTileInfo> &out);

// Uploads the FFT-64 twiddles to the current device; call outside any stream
// capture before the first launch on a device (world and batch creation do).
cudaError_t os_prepare();
// Dynamic shared memory of a launch whose jobs have radius >= rmin.
size_t os_smem_bytes(int rmin, int axis);
// Resident CTAs per SM a launch uses when none is asked for.
int os_default_ctas_per_sm();
// One persistent launch over `ntiles` tiles (tiles[i]) of jobs that all
// belong to `axis` and have radius >= rmin.
// ctas_per_sm: resident CTAs per SM the kernel is compiled for (3 or 4; 0:
// the default, 3, or VFD_OS_MINB=4).
cudaError_t launch_os(const OsJob *jobs, const OsTileInfo *tiles, int ntiles, int rmin, int axis, cudaStream_t st,
                      int ctas_per_sm = 0);

}  // namespace vfd
