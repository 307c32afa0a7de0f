// vfd_noalloc.cu -- an entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that manages every byte of
// device memory itself (a preallocated arena or pool shared with other
// components), and per-tick loops that must not trigger the device-wide
// synchronisation cudaMalloc / cudaFree can cause while other work is in
// flight.  vfd_fft_diffuse3d_noalloc serves them: the caller passes the field
// and the kernel spectrum already on the device, and the only scratch the
// transform needs -- the pruned spectrum of the field and three twiddle
// tables -- lives in one file-scope __device__ array of fixed size
// (kNoAllocScratchBytes, 32 MiB), which every GPU that loads the library
// holds until the process exits.
//
// Host code cannot use the array's name as a device address (it is a
// host-side stand-in), so the first call on each device looks the address up
// with cudaGetSymbolAddress while that device is current and caches it.
// That first call therefore performs set-up work; make it before any stream
// capture.  The cache is keyed by the device's current CUDA context (its
// unique id): after cudaDeviceReset the library's module is loaded into a
// new context, and the next call looks the address up again (that call, too,
// belongs outside stream capture).  Every call shares the same array and
// overwrites it: calls that overlap on the GPU (other streams, other host
// threads, the same device) race on it, so serialise them.  Nothing in the
// array has to start at zero: every element a call reads was written by the
// same call, or -- the twiddle tables -- by an earlier call of the same FFT
// lengths in the same context, which later calls reuse.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "vfd.h"
#include "vfd_general.h"
#include "vfd_internal.h"

namespace vfd {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
// per device: the scratch address, the context it belongs to, and the FFT
// lengths (with nz, which places the tables) whose twiddles it holds
struct NoAllocSlot {
    unsigned char *ptr = nullptr;
    unsigned long long ctx = 0;
    int tw_key[4] = {0, 0, 0, 0};
};
static NoAllocSlot g_noalloc[kMaxDevices];

// Unique id of the calling thread's current context (0 when unavailable).
unsigned long long current_context_id()
{
    static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess)
            get_cur = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(a);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(b);
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Twiddles exp(-2 pi i m / F), FP64, stored FP32.
__global__ void noalloc_twiddle_kernel(float2 *tw, int F)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < F; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)m / (double)F, &s, &c);
        tw[m] = make_float2((float)c, (float)-s);
    }
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace vfd

using namespace vfd;

extern "C" vfd_status vfd_fft_diffuse3d_noalloc(float *field, const float *kspec, int nx, int ny, int nz, int fx,
                                                int fy, int fz, int pad_mode, int epi_boundary, float baseline,
                                                float kernel_sum, float keep, void *stream)
{
    if (!field || !kspec || nx < 1 || ny < 1 || nz < 1) return VFD_ERR_INVALID_ARG;
    if (fx < nx || fy < ny || fz < nz || (fx & 1)) return VFD_ERR_INVALID_ARG;
    if (pad_mode != VFD_PAD_ZERO && pad_mode != VFD_PAD_CONSTANT_VF) return VFD_ERR_INVALID_ARG;
    FftPlan plan[3];
    const int F[3] = {fx, fy, fz};
    for (int a = 0; a < 3; ++a)
        if (!plan_for_length(F[a], &plan[a])) return VFD_ERR_NOT_SUPPORTED;
    const int vrow = variant_for_plan(plan[0], 0);
    const int vy = variant_for_plan(plan[1], 16), vz = variant_for_plan(plan[2], 16);
    if (vrow < 0 || vy < 0 || vz < 0) return VFD_ERR_NOT_SUPPORTED;

    // scratch layout: pruned spectrum [nz][fy][fx/2+1], then the twiddles of x, y, z
    const int fxh = fx / 2 + 1;
    const size_t spec_bytes = align256(sizeof(float2) * (size_t)nz * fy * fxh);
    const size_t tw_bytes[3] = {align256(sizeof(float2) * fx), align256(sizeof(float2) * fy),
                                align256(sizeof(float2) * fz)};
    if (spec_bytes + tw_bytes[0] + tw_bytes[1] + tw_bytes[2] > kNoAllocScratchBytes)
        return VFD_ERR_INVALID_ARG;  // larger than the fixed 32 MiB scratch

    // an error left pending by the caller's earlier launches is not this call's
    (void)cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return VFD_ERR_CUDA;
    unsigned char *base = nullptr;
    bool need_tw = true;
    const int tw_key[4] = {fx, fy, fz, nz};
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        NoAllocSlot &slot = g_noalloc[dev];
        if (cudaSetDevice(dev) != cudaSuccess) return VFD_ERR_CUDA;  // the device's context, current on this thread
        const unsigned long long ctx = current_context_id();
        if (!slot.ptr || ctx == 0 || ctx != slot.ctx) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return VFD_ERR_CUDA;
            slot.ptr = static_cast<unsigned char *>(p);
            slot.ctx = ctx;
            for (int i = 0; i < 4; ++i) slot.tw_key[i] = 0;
        }
        base = slot.ptr;
        need_tw = !(slot.tw_key[0] == fx && slot.tw_key[1] == fy && slot.tw_key[2] == fz && slot.tw_key[3] == nz);
        // later calls of these lengths reuse the tables this call writes
        for (int i = 0; i < 4; ++i) slot.tw_key[i] = need_tw ? 0 : tw_key[i];
    }
    float2 *C = reinterpret_cast<float2 *>(base);
    float2 *tw[3];
    tw[0] = reinterpret_cast<float2 *>(base + spec_bytes);
    tw[1] = reinterpret_cast<float2 *>(base + spec_bytes + tw_bytes[0]);
    tw[2] = reinterpret_cast<float2 *>(base + spec_bytes + tw_bytes[0] + tw_bytes[1]);

    cudaStream_t st = (cudaStream_t)stream;
    if (need_tw) {
        for (int a = 0; a < 3; ++a) {
            noalloc_twiddle_kernel<<<(F[a] + 255) / 256, 256, 0, st>>>(tw[a], F[a]);
            note_launch();
        }
        if (cudaGetLastError() != cudaSuccess) return VFD_ERR_CUDA;
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        for (int i = 0; i < 4; ++i) g_noalloc[dev].tw_key[i] = tw_key[i];
    }

    int lo[3], hi[3];
    if (pad_mode == VFD_PAD_CONSTANT_VF) {
        lo[0] = 1; hi[0] = epi_boundary < nx ? epi_boundary : nx;
        lo[1] = 1; hi[1] = ny - 1;
        lo[2] = 1; hi[2] = nz - 1;
    } else {
        lo[0] = 0; hi[0] = nx;
        lo[1] = 0; hi[1] = ny;
        lo[2] = 0; hi[2] = nz;
    }
    const float b = pad_mode == VFD_PAD_CONSTANT_VF ? baseline : 0.0f;

    // the same five fused passes as VFD_METHOD_FFT3D, without mass accounting
    GenRowPass r = {};
    r.plan = plan[0];
    r.tw = tw[0];
    r.nrows = ny * nz;
    r.rows_per_plane = ny;
    r.r_s1 = nx;
    r.r_s2 = (int64_t)nx * ny;
    r.c_s1 = fxh;
    r.c_s2 = (int64_t)fxh * fy;
    r.nload = nx;
    r.nstore = nx;
    r.rsrc = field;
    r.rdst = field;
    r.cdst = C;
    r.csrc = C;
    r.fuse_pad = 1;
    for (int i = 0; i < 3; ++i) {
        r.box_lo[i] = lo[i];
        r.box_hi[i] = hi[i];
    }
    r.b = b;
    if (launch_gen_rows(vrow, r, false, st) != cudaSuccess) return VFD_ERR_CUDA;

    GenColPass c = {};
    c.plan = plan[1];
    c.tw = tw[1];
    c.data = C;
    c.nlines = fxh;
    c.nouter = nz;
    c.outer_stride = (int64_t)fy * fxh;
    c.pos_stride = fxh;
    c.nload = ny;
    c.nstore = fy;
    c.mode = GEN_FORWARD;
    c.scale = 1.0f;
    if (launch_gen_cols(vy, c, st) != cudaSuccess) return VFD_ERR_CUDA;

    GenColPass z = {};
    z.plan = plan[2];
    z.tw = tw[2];
    z.data = C;
    z.nlines = fxh;
    z.nouter = fy;
    z.outer_stride = fxh;
    z.pos_stride = (int64_t)fy * fxh;
    z.nload = nz;
    z.nstore = nz;
    z.mode = GEN_FWD_MUL_INV;
    z.kspec = reinterpret_cast<const float2 *>(kspec);
    z.k_s_outer = fxh;
    z.k_s_pos = (int64_t)fxh * fy;
    z.scale = (float)(1.0 / ((double)fx * fy * fz));
    if (launch_gen_cols(vz, z, st) != cudaSuccess) return VFD_ERR_CUDA;

    c.nload = fy;
    c.nstore = ny;
    c.mode = GEN_INVERSE;
    if (launch_gen_cols(vy, c, st) != cudaSuccess) return VFD_ERR_CUDA;

    r.fuse_pad = 0;
    r.fuse_crop = 1;
    r.keep = keep;
    r.k0 = kernel_sum;
    if (launch_gen_rows(vrow, r, true, st) != cudaSuccess) return VFD_ERR_CUDA;
    return VFD_OK;
}
