// vfd_rf.h -- axis pass with the FFT-64 of each block held by one thread
// (vfd_rf.cu).  Jobs are overlap-save jobs (vfd_os.h) of radius <= RF_RMAX;
// tiles are 64 lines.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "vfd_os.h"

namespace vfd {

constexpr int RF_RMAX = 8;    // largest radius of the register-FFT pass
constexpr int RF_LINES = 64;  // lines per tile (32 line pairs, one warp)

// Whether job j (its other fields set) can use the register-FFT pass.
bool rf_eligible(const OsJob &j);
// Appends the 64-line tiles of job `job` to `out` (flags: real lines).
void rf_append_tiles(const OsJob &j, int job, std::vector<OsTileInfo> &out);
// Warps per CTA of the pass along `axis`: a launch's tile list holds a
// multiple of this many tiles, each CTA's tiles of one job (padded with
// empty tiles, flags 0).
int rf_cta_warps(int axis);
// Uploads the FFT-64 twiddles to the current device (outside stream capture).
cudaError_t rf_prepare();
// One launch over `ntiles` tiles of jobs (any radius <= RF_RMAX) that all
// belong to `axis`.  maps (y / z passes): one TMA tensor map per job, indexed
// like `jobs`; the windows are then staged by bulk tensor copies.
cudaError_t launch_rf(const OsJob *jobs, const OsTileInfo *tiles, int ntiles, int axis, cudaStream_t st,
                      const CUtensorMap *maps = nullptr);
// Whether the y / z passes stage their windows with TMA (VFD_RF_TMA=0: no).
bool rf_tma_enabled();
// Encodes job j's tensor maps for a TMA-staged launch (x pass: two, m[0]
// and m[1]; y / z: one); false if the job's layout does not allow it (then
// the launch uses the kernels without TMA).
bool rf_encode_map(const OsJob &j, CUtensorMap *m);
// Reads and clears the flag a pass sets when a bounded wait for a bulk copy
// gave up.
bool rf_take_timeout();
// Runs the passes' bounded barrier wait against a barrier nothing completes
// (limit in cycles); sets *gave_up_device and the pass timeout flag.
cudaError_t rf_wait_probe(long long limit, int *gave_up_device, cudaStream_t st);

}  // namespace vfd
