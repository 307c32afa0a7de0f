// vfd_world.cu -- host side of the C ABI (include/vfd.h): FFT planning,
// spectrum/twiddle tables, device residency of the fields, tick sequencing,
// the pipelined host-buffer entry point and the synthetic-input generator.
//
// Reference counterparts: c_ctx sizing and allocation
// (src/Diffusion/DiffusionHelper.cpp:29-163, 381-647), kernel spectrum
// preparation (computeKernelSpectrum3D, Diffusion.cu:1533-1619), the per-tick
// loop of Diffuser::diffuseChemGPU (Diffuser.cpp:221-470) and fftDiffuse3D
// (Diffusion.cu:1622-1934).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "vfd.h"
#include "vfd_internal.h"

namespace vfd {

static std::atomic<uint64_t> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static thread_local std::string g_thread_error = "";

// ---------------------------------------------------------------------------
// FFT planning.  Length F >= n + r makes the circular convolution of the
// zero-extended line with a radius-r kernel equal to the linear one on
// [0, n) (the reference instead rounds n + window - 1 up to a power of two,
// snapTransformSize, Diffusion.cu:39-70).  Among 7-smooth lengths the cheapest
// by a per-stage cost model is taken; radices 8,7,5,4,3,2.
// ---------------------------------------------------------------------------
static bool make_plan(int F, FftPlan *p)
{
    int n = F, k = 0;
    static const int order[] = {8, 7, 5, 4, 3, 2};
    for (int r : order) {
        while (n % r == 0) {
            if (k >= MAX_STAGES) return false;
            p->radix[k++] = r;
            n /= r;
        }
    }
    if (n != 1 || F < 2) return false;
    p->F = F;
    p->nst = k;
    for (int i = k; i < MAX_STAGES; ++i) p->radix[i] = 1;
    return true;
}

static bool variant_fits(int v, const FftPlan &p)
{
    const int TL = variant_tl(v), MAXP = variant_maxp(v);
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.radix[s];
        const int M = p.F / R;
        if ((M + TL - 1) / TL > MAXP / R) return false;
    }
    return axis_smem_bytes(p.F) <= axis_smem_limit();
}

static double plan_cost(const FftPlan &p)
{
    double c = 2.0;
    for (int s = 0; s < p.nst; ++s) {
        switch (p.radix[s]) {
        case 2: c += 1.0; break;
        case 3: c += 1.3; break;
        case 4: c += 1.15; break;
        case 5: c += 1.5; break;
        case 7: c += 1.9; break;
        case 8: c += 1.35; break;
        default: c += 3.0; break;
        }
    }
    return c * p.F;
}

static bool any_variant_fits(const FftPlan &p)
{
    for (int v = 0; v < kNumAxisVariants; ++v)
        if (variant_fits(v, p)) return true;
    return false;
}

static int choose_fft_len(int n, int r)
{
    const int lo = n + r;
    int best = -1;
    double best_cost = 0.0;
    for (int F = lo; F <= 2 * lo + 16; ++F) {
        FftPlan p;
        if (!make_plan(F, &p) || !any_variant_fits(p)) continue;
        const double c = plan_cost(p);
        if (best < 0 || c < best_cost) {
            best = F;
            best_cost = c;
        }
    }
    return best;
}

static int pick_variant(const std::vector<FftPlan> &plans)
{
    static int forced = -2;
    if (forced == -2) {
        const char *e = getenv("VFD_AXIS_VARIANT");
        forced = e ? atoi(e) : -1;
    }
    if (forced >= 0 && forced < kNumAxisVariants) {
        bool ok = true;
        for (const auto &p : plans) ok = ok && variant_fits(forced, p);
        if (ok) return forced;
    }
    static const int pref[] = {0, 1, 2, 3, 4};
    for (int v : pref) {
        bool ok = true;
        for (const auto &p : plans) ok = ok && variant_fits(v, p);
        if (ok) return v;
    }
    return -1;
}

// Real multipliers G(k)/F of the wrapped normalised Gaussian taps, FP64.
static void gauss_spectrum(double sigma, int r, int F, std::vector<float> &out)
{
    std::vector<double> g(2 * r + 1);
    double s = 0.0;
    for (int j = -r; j <= r; ++j) {
        g[j + r] = std::exp(-(double)j * j / (2.0 * sigma * sigma));
        s += g[j + r];
    }
    for (auto &x : g) x /= s;
    out.resize(F);
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < F; ++k) {
        double acc = g[r];
        for (int j = 1; j <= r; ++j) {
            const long long m = ((long long)j * k) % F;
            acc += 2.0 * g[r + j] * std::cos(two_pi * (double)m / (double)F);
        }
        out[k] = (float)(acc / (double)F);
    }
}

static void twiddles(int F, std::vector<float2> &out)
{
    out.resize(F);
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < F; ++m) {
        const double a = two_pi * (double)m / (double)F;
        out[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
}

}  // namespace vfd

using namespace vfd;

struct vfd_world {
    int device = 0;
    int nx = 0, ny = 0, nz = 0, nf = 0;
    int64_t V = 0;
    int pad_mode = 0, epi = 0;
    std::vector<vfd_field_params> params;
    int F[3] = {0, 0, 0};
    FftPlan plan[3];
    int variant[3] = {0, 0, 0};
    int tiles_per_field[3] = {0, 0, 0};

    float *d_fields = nullptr;
    float2 *d_tw[3] = {nullptr, nullptr, nullptr};
    float *d_spec = nullptr;   // [f][axis][Fmax]
    int Fmax = 0;
    double *d_mass = nullptr;  // [f][MS_COUNT]
    AxisJob *d_jobs = nullptr; // [pass][nf] all-field jobs, then [pass][nf] single-field jobs
    int *d_err = nullptr;

    // sources
    std::vector<std::vector<int32_t>> src_idx;
    std::vector<std::vector<float>> src_amt;
    bool src_dirty = false;
    int32_t *d_src_idx = nullptr;
    float *d_src_amt = nullptr;
    int64_t src_cap = 0, src_total = 0;
    DepositJob *d_dep = nullptr;     // [nf] all-field jobs (compacted) then [nf] single
    int dep_njobs = 0;
    std::vector<int64_t> src_begin;  // per field begin in concatenated list
    std::vector<int64_t> src_count;

    // optional per-launch event timing
    bool profiling = false;
    struct TimedLaunch {
        int kind;
        cudaEvent_t start, stop;
    };
    std::vector<TimedLaunch> timed;   // recorded, not yet read
    std::vector<cudaEvent_t> ev_pool; // free events

    cudaStream_t s_in = nullptr, s_cmp = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> ev_in, ev_cmp;

    std::string err;
};

static vfd_status fail(vfd_world *w, vfd_status s, const std::string &msg)
{
    if (w) w->err = msg;
    else g_thread_error = msg;
    return s;
}

#define VFD_CUDA(w, call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((w), e_ == cudaErrorMemoryAllocation ? VFD_ERR_OUT_OF_MEMORY         \
                                                              : VFD_ERR_CUDA,                 \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)

static void release(vfd_world *w)
{
    if (!w) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(w->device);
    cudaFree(w->d_fields);
    for (int a = 0; a < 3; ++a) cudaFree(w->d_tw[a]);
    cudaFree(w->d_spec);
    cudaFree(w->d_mass);
    cudaFree(w->d_jobs);
    cudaFree(w->d_err);
    cudaFree(w->d_src_idx);
    cudaFree(w->d_src_amt);
    cudaFree(w->d_dep);
    for (auto &t : w->timed) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    for (auto e : w->ev_pool) cudaEventDestroy(e);
    for (auto e : w->ev_in) cudaEventDestroy(e);
    for (auto e : w->ev_cmp) cudaEventDestroy(e);
    if (w->s_in) cudaStreamDestroy(w->s_in);
    if (w->s_cmp) cudaStreamDestroy(w->s_cmp);
    if (w->s_out) cudaStreamDestroy(w->s_out);
    cudaSetDevice(prev);
}

// Builds the AxisJob of (field f, axis a).
static AxisJob make_job(const vfd_world *w, int f, int a, int tile_begin)
{
    AxisJob j;
    memset(&j, 0, sizeof(j));
    const int64_t nx = w->nx, ny = w->ny;
    j.data = w->d_fields + (int64_t)f * w->V;
    j.tw = w->d_tw[a];
    j.spec = w->d_spec + ((int64_t)f * 3 + a) * w->Fmax;
    j.mass = w->d_mass + (int64_t)f * MS_COUNT;
    j.kind = a;
    j.plan = w->plan[a];
    j.nx = w->nx;
    j.ny = w->ny;
    j.b = w->pad_mode == VFD_PAD_CONSTANT_VF ? w->params[f].baseline : 0.0f;
    j.keep = (float)(1.0 - w->params[f].decay_rate);
    if (w->pad_mode == VFD_PAD_CONSTANT_VF) {
        // padDataConstantVF3D_kernel interior: 0<x<epi, 0<y<H-1, 0<z<D-1
        j.box_lo[0] = 1; j.box_hi[0] = std::min(w->epi, w->nx);
        j.box_lo[1] = 1; j.box_hi[1] = w->ny - 1;
        j.box_lo[2] = 1; j.box_hi[2] = w->nz - 1;
    } else {
        j.box_lo[0] = 0; j.box_hi[0] = w->nx;
        j.box_lo[1] = 0; j.box_hi[1] = w->ny;
        j.box_lo[2] = 0; j.box_hi[2] = w->nz;
    }
    if (a == PASS_X) {
        j.n = w->nx;
        j.line_stride = nx;
        j.outer_stride = 0;
        j.pos_stride = 1;
        j.nlines = w->ny * w->nz;
        j.nouter = 1;
    } else if (a == PASS_Y) {
        j.n = w->ny;
        j.line_stride = 1;
        j.outer_stride = nx * ny;
        j.pos_stride = nx;
        j.nlines = w->nx;
        j.nouter = w->nz;
    } else {
        j.n = w->nz;
        j.line_stride = 1;
        j.outer_stride = nx;
        j.pos_stride = nx * ny;
        j.nlines = w->nx;
        j.nouter = w->ny;
    }
    j.tiles_per_outer = (j.nlines + 2 * NL - 1) / (2 * NL);
    j.tile_begin = tile_begin;
    return j;
}

extern "C" {

const char *vfd_status_string(vfd_status s)
{
    switch (s) {
    case VFD_OK: return "ok";
    case VFD_ERR_INVALID_ARG: return "invalid argument";
    case VFD_ERR_OUT_OF_MEMORY: return "out of device memory";
    case VFD_ERR_BUDGET: return "HBM budget exceeded";
    case VFD_ERR_CUDA: return "CUDA error";
    case VFD_ERR_TIMEOUT: return "device wait timed out";
    case VFD_ERR_DEVICE_FAULT: return "device reported a bad argument";
    case VFD_ERR_NOT_SUPPORTED: return "not supported";
    case VFD_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char *vfd_last_error(const vfd_world *w)
{
    return w ? w->err.c_str() : g_thread_error.c_str();
}

uint64_t vfd_kernel_launch_count(void) { return g_launches.load(); }

vfd_status vfd_world_create(const vfd_world_desc *d, int device, vfd_world **out)
{
    if (!out) return fail(nullptr, VFD_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!d || !d->fields) return fail(nullptr, VFD_ERR_INVALID_ARG, "desc or desc->fields is NULL");
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->n_fields < 1)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "grid dims and n_fields must be >= 1");
    if ((int64_t)d->nx * d->ny * d->nz > ((int64_t)1 << 31) - 1)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "grid larger than 2^31-1 voxels");
    if (d->pad_mode != VFD_PAD_ZERO && d->pad_mode != VFD_PAD_CONSTANT_VF)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "unknown pad_mode");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, VFD_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev) return fail(nullptr, VFD_ERR_INVALID_ARG, "device ordinal out of range");

    vfd_world *w = new vfd_world();
    w->device = device;
    w->nx = d->nx; w->ny = d->ny; w->nz = d->nz; w->nf = d->n_fields;
    w->V = (int64_t)d->nx * d->ny * d->nz;
    w->pad_mode = d->pad_mode;
    w->epi = d->epi_boundary;
    w->params.assign(d->fields, d->fields + d->n_fields);
    const int dims[3] = {d->nx, d->ny, d->nz};
    // per-axis radius: the largest over fields (one FFT grid per world)
    int rmax[3] = {0, 0, 0};
    for (int f = 0; f < w->nf; ++f) {
        vfd_field_params &p = w->params[f];
        for (int a = 0; a < 3; ++a) {
            if (!(p.sigma[a] > 0.0) || !std::isfinite(p.sigma[a])) {
                delete w;
                return fail(nullptr, VFD_ERR_INVALID_ARG, "sigma must be finite and > 0");
            }
            if (p.radius[a] <= 0) p.radius[a] = (int)std::ceil(3.0 * p.sigma[a]);
            rmax[a] = std::max(rmax[a], p.radius[a]);
        }
        if (!(p.decay_rate >= 0.0 && p.decay_rate < 1.0)) {
            delete w;
            return fail(nullptr, VFD_ERR_INVALID_ARG, "decay_rate must be in [0, 1)");
        }
    }
    for (int a = 0; a < 3; ++a) {
        int F = d->fft[a];
        if (F > 0) {
            if (F < dims[a] + rmax[a]) {
                delete w;
                return fail(nullptr, VFD_ERR_INVALID_ARG, "fft length shorter than n + radius");
            }
            if (!make_plan(F, &w->plan[a]) || !any_variant_fits(w->plan[a])) {
                delete w;
                return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "fft length not 7-smooth or too long");
            }
        } else {
            F = choose_fft_len(dims[a], rmax[a]);
            if (F < 0) {
                delete w;
                return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "axis too long for the shared-memory FFT");
            }
            make_plan(F, &w->plan[a]);
        }
        w->F[a] = F;
        w->Fmax = std::max(w->Fmax, F);
        w->variant[a] = pick_variant(std::vector<FftPlan>{w->plan[a]});
    }
    w->tiles_per_field[0] = (w->ny * w->nz + 2 * NL - 1) / (2 * NL);
    w->tiles_per_field[1] = w->nz * ((w->nx + 2 * NL - 1) / (2 * NL));
    w->tiles_per_field[2] = w->ny * ((w->nx + 2 * NL - 1) / (2 * NL));

    int prev = 0;
    cudaGetDevice(&prev);
    auto bail = [&](cudaError_t e, const char *what) {
        std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
        release(w);
        delete w;
        cudaSetDevice(prev);
        return fail(nullptr, e == cudaErrorMemoryAllocation ? VFD_ERR_OUT_OF_MEMORY : VFD_ERR_CUDA, msg);
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaMalloc(&w->d_fields, sizeof(float) * w->V * w->nf)) != cudaSuccess) return bail(e, "cudaMalloc fields");
    if ((e = cudaMemset(w->d_fields, 0, sizeof(float) * w->V * w->nf)) != cudaSuccess) return bail(e, "cudaMemset fields");
    for (int a = 0; a < 3; ++a) {
        std::vector<float2> tw;
        twiddles(w->F[a], tw);
        if ((e = cudaMalloc(&w->d_tw[a], sizeof(float2) * w->F[a])) != cudaSuccess) return bail(e, "cudaMalloc twiddles");
        if ((e = cudaMemcpy(w->d_tw[a], tw.data(), sizeof(float2) * w->F[a], cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e, "cudaMemcpy twiddles");
    }
    {
        std::vector<float> spec((size_t)w->nf * 3 * w->Fmax, 0.0f), tmp;
        for (int f = 0; f < w->nf; ++f)
            for (int a = 0; a < 3; ++a) {
                gauss_spectrum(w->params[f].sigma[a], w->params[f].radius[a], w->F[a], tmp);
                std::copy(tmp.begin(), tmp.end(), spec.begin() + ((size_t)f * 3 + a) * w->Fmax);
            }
        if ((e = cudaMalloc(&w->d_spec, sizeof(float) * spec.size())) != cudaSuccess) return bail(e, "cudaMalloc spectra");
        if ((e = cudaMemcpy(w->d_spec, spec.data(), sizeof(float) * spec.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e, "cudaMemcpy spectra");
    }
    if ((e = cudaMalloc(&w->d_mass, sizeof(double) * MS_COUNT * w->nf)) != cudaSuccess) return bail(e, "cudaMalloc mass");
    if ((e = cudaMemset(w->d_mass, 0, sizeof(double) * MS_COUNT * w->nf)) != cudaSuccess) return bail(e, "cudaMemset mass");
    if ((e = cudaMalloc(&w->d_err, sizeof(int))) != cudaSuccess) return bail(e, "cudaMalloc err");
    if ((e = cudaMemset(w->d_err, 0, sizeof(int))) != cudaSuccess) return bail(e, "cudaMemset err");
    {
        std::vector<AxisJob> jobs;
        for (int a = 0; a < 3; ++a) {
            int tb = 0;
            for (int f = 0; f < w->nf; ++f) {
                jobs.push_back(make_job(w, f, a, tb));
                tb += w->tiles_per_field[a];
            }
        }
        for (int a = 0; a < 3; ++a)
            for (int f = 0; f < w->nf; ++f) jobs.push_back(make_job(w, f, a, 0));
        if ((e = cudaMalloc(&w->d_jobs, sizeof(AxisJob) * jobs.size())) != cudaSuccess) return bail(e, "cudaMalloc jobs");
        if ((e = cudaMemcpy(w->d_jobs, jobs.data(), sizeof(AxisJob) * jobs.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e, "cudaMemcpy jobs");
    }
    if ((e = cudaMalloc(&w->d_dep, sizeof(DepositJob) * 2 * w->nf)) != cudaSuccess) return bail(e, "cudaMalloc deposit jobs");
    if ((e = cudaStreamCreateWithFlags(&w->s_in, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&w->s_cmp, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&w->s_out, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    w->ev_in.resize(w->nf);
    w->ev_cmp.resize(w->nf);
    for (int f = 0; f < w->nf; ++f) {
        if ((e = cudaEventCreateWithFlags(&w->ev_in[f], cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
        if ((e = cudaEventCreateWithFlags(&w->ev_cmp[f], cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    }
    w->src_idx.resize(w->nf);
    w->src_amt.resize(w->nf);
    w->src_begin.assign(w->nf, 0);
    w->src_count.assign(w->nf, 0);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(e, "cudaDeviceSynchronize");
    cudaSetDevice(prev);
    *out = w;
    return VFD_OK;
}

vfd_status vfd_world_destroy(vfd_world *w)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    release(w);
    delete w;
    return VFD_OK;
}

vfd_status vfd_world_fft_dims(const vfd_world *w, int *fft3)
{
    if (!w || !fft3) return VFD_ERR_INVALID_ARG;
    for (int a = 0; a < 3; ++a) fft3[a] = w->F[a];
    return VFD_OK;
}

vfd_status vfd_world_device_bytes(const vfd_world *w, size_t *bytes)
{
    if (!w || !bytes) return VFD_ERR_INVALID_ARG;
    size_t b = sizeof(float) * (size_t)w->V * w->nf;
    for (int a = 0; a < 3; ++a) b += sizeof(float2) * w->F[a];
    b += sizeof(float) * (size_t)w->nf * 3 * w->Fmax + sizeof(double) * MS_COUNT * w->nf;
    b += sizeof(AxisJob) * 6 * w->nf + sizeof(DepositJob) * 2 * w->nf;
    b += (sizeof(int32_t) + sizeof(float)) * (size_t)w->src_cap;
    *bytes = b;
    return VFD_OK;
}

class DeviceGuard {
  public:
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev_);
        cudaSetDevice(dev);
    }
    ~DeviceGuard() { cudaSetDevice(prev_); }

  private:
    int prev_ = 0;
};

vfd_status vfd_upload_field(vfd_world *w, int field, const float *host, void *stream)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (field < 0 || field >= w->nf || !host) return fail(w, VFD_ERR_INVALID_ARG, "bad field index or NULL host pointer");
    DeviceGuard g(w->device);
    VFD_CUDA(w, cudaMemcpyAsync(w->d_fields + (int64_t)field * w->V, host, sizeof(float) * w->V,
                                cudaMemcpyHostToDevice, (cudaStream_t)stream));
    return VFD_OK;
}

vfd_status vfd_download_field(vfd_world *w, int field, float *host, void *stream)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (field < 0 || field >= w->nf || !host) return fail(w, VFD_ERR_INVALID_ARG, "bad field index or NULL host pointer");
    DeviceGuard g(w->device);
    VFD_CUDA(w, cudaMemcpyAsync(host, w->d_fields + (int64_t)field * w->V, sizeof(float) * w->V,
                                cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    VFD_CUDA(w, cudaStreamSynchronize((cudaStream_t)stream));
    return VFD_OK;
}

vfd_status vfd_field_device_ptr(vfd_world *w, int field, float **dptr)
{
    if (!w || !dptr) return VFD_ERR_INVALID_ARG;
    if (field < 0 || field >= w->nf) return fail(w, VFD_ERR_INVALID_ARG, "bad field index");
    *dptr = w->d_fields + (int64_t)field * w->V;
    return VFD_OK;
}

vfd_status vfd_set_sources(vfd_world *w, int field, const int32_t *idx, const float *amt, int64_t n)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (field < 0 || field >= w->nf || n < 0 || (n > 0 && (!idx || !amt)))
        return fail(w, VFD_ERR_INVALID_ARG, "bad field index, count or NULL arrays");
    for (int64_t j = 0; j < n; ++j)
        if (idx[j] < 0 || (int64_t)idx[j] >= w->V)
            return fail(w, VFD_ERR_INVALID_ARG, "source voxel index out of range");
    w->src_idx[field].assign(idx, idx + n);
    w->src_amt[field].assign(amt, amt + n);
    w->src_dirty = true;
    return VFD_OK;
}

// Uploads the concatenated source list and deposit jobs when they changed.
static vfd_status sync_sources(vfd_world *w)
{
    if (!w->src_dirty) return VFD_OK;
    int64_t total = 0;
    for (int f = 0; f < w->nf; ++f) {
        w->src_begin[f] = total;
        w->src_count[f] = (int64_t)w->src_idx[f].size();
        total += w->src_count[f];
    }
    if (total > w->src_cap) {
        cudaFree(w->d_src_idx);
        cudaFree(w->d_src_amt);
        w->d_src_idx = nullptr;
        w->d_src_amt = nullptr;
        w->src_cap = 0;
        VFD_CUDA(w, cudaMalloc(&w->d_src_idx, sizeof(int32_t) * total));
        VFD_CUDA(w, cudaMalloc(&w->d_src_amt, sizeof(float) * total));
        w->src_cap = total;
    }
    std::vector<int32_t> hi(total);
    std::vector<float> ha(total);
    for (int f = 0; f < w->nf; ++f) {
        std::copy(w->src_idx[f].begin(), w->src_idx[f].end(), hi.begin() + w->src_begin[f]);
        std::copy(w->src_amt[f].begin(), w->src_amt[f].end(), ha.begin() + w->src_begin[f]);
    }
    if (total > 0) {
        VFD_CUDA(w, cudaMemcpy(w->d_src_idx, hi.data(), sizeof(int32_t) * total, cudaMemcpyHostToDevice));
        VFD_CUDA(w, cudaMemcpy(w->d_src_amt, ha.data(), sizeof(float) * total, cudaMemcpyHostToDevice));
    }
    std::vector<DepositJob> jobs;
    for (int f = 0; f < w->nf; ++f) {
        if (w->src_count[f] == 0) continue;
        DepositJob j;
        j.data = w->d_fields + (int64_t)f * w->V;
        j.mass = w->d_mass + (int64_t)f * MS_COUNT;
        j.begin = w->src_begin[f];
        j.nvox = w->V;
        jobs.push_back(j);
    }
    // [0, dep_njobs): fields with sources, for the all-field launch;
    // [nf, 2 nf): one job per field (begin 0) for single-field launches.
    w->dep_njobs = (int)jobs.size();
    jobs.resize(w->nf);
    for (int f = 0; f < w->nf; ++f) {
        DepositJob j;
        j.data = w->d_fields + (int64_t)f * w->V;
        j.mass = w->d_mass + (int64_t)f * MS_COUNT;
        j.begin = 0;
        j.nvox = w->V;
        jobs.push_back(j);
    }
    VFD_CUDA(w, cudaMemcpy(w->d_dep, jobs.data(), sizeof(DepositJob) * jobs.size(), cudaMemcpyHostToDevice));
    w->src_total = total;
    w->src_dirty = false;
    return VFD_OK;
}

static cudaEvent_t pool_event(vfd_world *w)
{
    if (!w->ev_pool.empty()) {
        cudaEvent_t e = w->ev_pool.back();
        w->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when profiling is on.
struct LaunchTimer {
    vfd_world *w;
    int kind;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    LaunchTimer(vfd_world *w_, int kind_, cudaStream_t st_) : w(w_), kind(kind_), st(st_)
    {
        if (w->profiling) {
            a = pool_event(w);
            cudaEventRecord(a, st);
        }
    }
    void done()
    {
        if (!a) return;
        cudaEvent_t b = pool_event(w);
        cudaEventRecord(b, st);
        w->timed.push_back({kind, a, b});
        a = nullptr;
    }
};

// Enqueues n_substeps of one field (field >= 0) or of all fields (field < 0).
static vfd_status enqueue_tick(vfd_world *w, int field, int n_substeps, cudaStream_t st)
{
    const int nj = field < 0 ? w->nf : 1;
    for (int s = 0; s < n_substeps; ++s) {
        if (field < 0)
            VFD_CUDA(w, cudaMemsetAsync(w->d_mass, 0, sizeof(double) * MS_COUNT * w->nf, st));
        else
            VFD_CUDA(w, cudaMemsetAsync(w->d_mass + (int64_t)field * MS_COUNT, 0, sizeof(double) * MS_COUNT, st));
        for (int a = 0; a < 3; ++a) {
            const AxisJob *jobs = field < 0 ? w->d_jobs + a * w->nf : w->d_jobs + 3 * w->nf + a * w->nf + field;
            const int tiles = w->tiles_per_field[a] * nj;
            LaunchTimer lt(w, a, st);
            VFD_CUDA(w, launch_axis(w->variant[a], jobs, nj, tiles, w->F[a], st));
            lt.done();
        }
    }
    if (field < 0) {
        if (w->dep_njobs > 0) {
            LaunchTimer lt(w, 3, st);
            VFD_CUDA(w, launch_deposit(w->d_dep, w->dep_njobs, w->d_src_idx, w->d_src_amt, w->src_total, w->d_err, st));
            lt.done();
        }
    } else if (w->src_count[field] > 0) {
        LaunchTimer lt(w, 3, st);
        VFD_CUDA(w, launch_deposit(w->d_dep + w->nf + field, 1, w->d_src_idx + w->src_begin[field],
                                   w->d_src_amt + w->src_begin[field], w->src_count[field], w->d_err, st));
        lt.done();
    }
    return VFD_OK;
}

vfd_status vfd_tick(vfd_world *w, int n_substeps, void *stream)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (n_substeps < 1) return fail(w, VFD_ERR_INVALID_ARG, "n_substeps must be >= 1");
    DeviceGuard g(w->device);
    vfd_status s = sync_sources(w);
    if (s != VFD_OK) return s;
    return enqueue_tick(w, -1, n_substeps, (cudaStream_t)stream);
}

vfd_status vfd_read_mass(vfd_world *w, vfd_mass *out, void *stream)
{
    if (!w || !out) return VFD_ERR_INVALID_ARG;
    DeviceGuard g(w->device);
    std::vector<double> h((size_t)MS_COUNT * w->nf);
    int herr = 0;
    VFD_CUDA(w, cudaMemcpyAsync(h.data(), w->d_mass, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                                (cudaStream_t)stream));
    VFD_CUDA(w, cudaMemcpyAsync(&herr, w->d_err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    VFD_CUDA(w, cudaStreamSynchronize((cudaStream_t)stream));
    for (int f = 0; f < w->nf; ++f) {
        const double *m = h.data() + (size_t)f * MS_COUNT;
        out[f].input_sum = m[MS_INPUT];
        out[f].leaked[0] = m[MS_LEAK_X];
        out[f].leaked[1] = m[MS_LEAK_Y];
        out[f].leaked[2] = m[MS_LEAK_Z];
        out[f].conv_sum = m[MS_CONV];
        out[f].sources = m[MS_SOURCES];
        out[f].total = m[MS_OUT] + m[MS_SOURCES];
        out[f].reserved = 0.0;
    }
    if (herr) return fail(w, VFD_ERR_DEVICE_FAULT, "a kernel rejected an out-of-range index");
    return VFD_OK;
}

vfd_status vfd_world_set_profiling(vfd_world *w, int enable)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    w->profiling = enable != 0;
    return VFD_OK;
}

vfd_status vfd_read_profile(vfd_world *w, double *ms4, int64_t *launches4)
{
    if (!w || !ms4 || !launches4) return VFD_ERR_INVALID_ARG;
    DeviceGuard g(w->device);
    for (int k = 0; k < 4; ++k) {
        ms4[k] = 0.0;
        launches4[k] = 0;
    }
    for (auto &t : w->timed) {
        VFD_CUDA(w, cudaEventSynchronize(t.stop));
        float ms = 0.0f;
        VFD_CUDA(w, cudaEventElapsedTime(&ms, t.start, t.stop));
        ms4[t.kind] += ms;
        launches4[t.kind] += 1;
        w->ev_pool.push_back(t.start);
        w->ev_pool.push_back(t.stop);
    }
    w->timed.clear();
    return VFD_OK;
}

vfd_status vfd_diffuse_host(vfd_world *w, const float *const *host_in, float *const *host_out, int n_substeps)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (!host_in || !host_out || n_substeps < 1) return fail(w, VFD_ERR_INVALID_ARG, "NULL buffers or n_substeps < 1");
    for (int f = 0; f < w->nf; ++f)
        if (!host_in[f] || !host_out[f]) return fail(w, VFD_ERR_INVALID_ARG, "NULL host buffer");
    DeviceGuard g(w->device);
    vfd_status s = sync_sources(w);
    if (s != VFD_OK) return s;
    const size_t bytes = sizeof(float) * w->V;
    for (int f = 0; f < w->nf; ++f) {
        float *dev = w->d_fields + (int64_t)f * w->V;
        VFD_CUDA(w, cudaMemcpyAsync(dev, host_in[f], bytes, cudaMemcpyHostToDevice, w->s_in));
        VFD_CUDA(w, cudaEventRecord(w->ev_in[f], w->s_in));
        VFD_CUDA(w, cudaStreamWaitEvent(w->s_cmp, w->ev_in[f], 0));
        s = enqueue_tick(w, f, n_substeps, w->s_cmp);
        if (s != VFD_OK) return s;
        VFD_CUDA(w, cudaEventRecord(w->ev_cmp[f], w->s_cmp));
        VFD_CUDA(w, cudaStreamWaitEvent(w->s_out, w->ev_cmp[f], 0));
        VFD_CUDA(w, cudaMemcpyAsync(host_out[f], dev, bytes, cudaMemcpyDeviceToHost, w->s_out));
    }
    VFD_CUDA(w, cudaStreamSynchronize(w->s_out));
    VFD_CUDA(w, cudaStreamSynchronize(w->s_cmp));
    int herr = 0;
    VFD_CUDA(w, cudaMemcpy(&herr, w->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(w, VFD_ERR_DEVICE_FAULT, "a kernel rejected an out-of-range index");
    return VFD_OK;
}

// ---------------------------------------------------------------------------
// Synthetic inputs: counter-based splitmix64 (Steele, Lea, Flood 2014
// finaliser) keyed by (seed, world, field, stream).
// ---------------------------------------------------------------------------
static inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline uint64_t stream_key(uint64_t seed, int world, int field, int stream)
{
    uint64_t k = mix64(seed + 0x9e3779b97f4a7c15ULL);
    k = mix64(k ^ (0x632be59bd9b4e019ULL * (uint64_t)(world + 1)));
    k = mix64(k ^ (0x85157af5ULL * (uint64_t)(field + 1)));
    k = mix64(k ^ (0xd6e8feb86659fd93ULL * (uint64_t)(stream + 1)));
    return k;
}
static inline double u01(uint64_t key, uint64_t i)
{
    return (double)(mix64(key + (i + 1) * 0x9e3779b97f4a7c15ULL) >> 11) * (1.0 / 9007199254740992.0);
}

vfd_status vfd_synth_field(uint64_t seed, int world, int field, float lo, float hi, float *out, size_t n)
{
    if (!out && n) return fail(nullptr, VFD_ERR_INVALID_ARG, "out is NULL");
    const uint64_t key = stream_key(seed, world, field, 0);
    const double a = lo, span = (double)hi - (double)lo;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) out[i] = (float)(a + span * u01(key, (uint64_t)i));
    return VFD_OK;
}

vfd_status vfd_synth_sources(uint64_t seed, int world, int field, int64_t n, int64_t n_voxels, double mu,
                             double sigma, int32_t *idx, float *amt)
{
    if (n < 0 || n_voxels < 1 || n_voxels > 2147483647LL || (n > 0 && (!idx || !amt)))
        return fail(nullptr, VFD_ERR_INVALID_ARG, "bad source request");
    const uint64_t k1 = stream_key(seed, world, field, 1), k2 = stream_key(seed, world, field, 2);
    const double two_pi = 6.283185307179586476925286766559;
    for (int64_t j = 0; j < n; ++j) {
        int64_t v = (int64_t)(u01(k1, (uint64_t)j) * (double)n_voxels);
        if (v >= n_voxels) v = n_voxels - 1;
        idx[j] = (int32_t)v;
        const double u1 = u01(k2, 2 * (uint64_t)j), u2 = u01(k2, 2 * (uint64_t)j + 1);
        const double z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(two_pi * u2);
        amt[j] = (float)std::exp(mu + sigma * z);
    }
    return VFD_OK;
}

}  // extern "C"
