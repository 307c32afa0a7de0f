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
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "vfd.h"
#include "vfd_general.h"
#include "vfd_internal.h"
#include "vfd_os.h"
#include "vfd_rf.h"

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
// Radix orders for the Stockham stages: 0 takes radix 8 first, 1 radix 4
// (more, cheaper stages); the autotuner times both.
constexpr int kPlanOrders = 2;

static bool make_plan_order(int F, int order_id, FftPlan *p)
{
    int n = F, k = 0;
    static const int orders[kPlanOrders][6] = {{8, 7, 5, 4, 3, 2}, {4, 7, 5, 8, 3, 2}};
    const int *order = orders[(order_id >= 0 && order_id < kPlanOrders) ? order_id : 0];
    for (int i = 0; i < 6; ++i) {
        const int r = order[i];
        while (n % r == 0) {
            if (k >= MAX_STAGES) return false;
            p->radix[k++] = r;
            n /= r;
        }
    }
    if (n != 1 || F < 2 || F > 2047) return false;
    p->F = F;
    p->nst = k;
    int ns = 1;
    for (int i = 0; i < MAX_STAGES; ++i) {
        if (i >= k) p->radix[i] = 1;
        p->ns[i] = ns;
        p->ns_magic[i] = (int)(((1 << 21) + ns - 1) / ns);
        ns *= p->radix[i];
    }
    return true;
}

static bool make_plan(int F, FftPlan *p) { return make_plan_order(F, 0, p); }

static bool variant_fits(int v, const FftPlan &p)
{
    const int TL = kAxisVariants[v].tl, MAXP = kAxisVariants[v].maxp;
    for (int s = 0; s < p.nst; ++s) {
        const int R = p.radix[s];
        const int M = p.F / R;
        if ((M + TL - 1) / TL > MAXP / R) return false;
    }
    return axis_smem_bytes(p.F, kAxisVariants[v].nl) <= axis_smem_limit();
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

static int choose_fft_len(int n, int r, bool even)
{
    const int lo = n + r;
    int best = -1;
    double best_cost = 0.0;
    for (int F = lo; F <= 2 * lo + 16; ++F) {
        FftPlan p;
        if (even && (F & 1)) continue;
        if (!make_plan(F, &p) || !any_variant_fits(p)) continue;
        const double c = plan_cost(p);
        if (best < 0 || c < best_cost) {
            best = F;
            best_cost = c;
        }
    }
    return best;
}

// FFT length of a general-method axis: the shortest length >= n + r that the
// register engine splits into two factors <= 24 (measured on B200 at the
// 512x256x384 world: x 576 = 24 x 24 runs its row passes in 3.43 ms per tick,
// 540 = 18 x 30 in 3.98 ms and 560 = 20 x 28 in 4.03 ms), else <= 32, else
// the Stockham choice.
static int choose_general_len(int n, int r, bool even)
{
    const int lo = n + r;
    for (int cap : {24, 32}) {
        for (int F = lo; F <= 2 * lo + 16; ++F) {
            if (even && (F & 1)) continue;
            const int f1 = tpr_split(F);
            FftPlan p;
            if (f1 > 0 && F / f1 <= cap && make_plan(F, &p) && any_variant_fits(p)) return F;
        }
    }
    return choose_fft_len(n, r, even);
}

static int pick_variant(const std::vector<FftPlan> &plans, int need_nl = 0)
{
    static int forced = -2;
    if (forced == -2) {
        const char *e = getenv("VFD_AXIS_VARIANT");
        forced = e ? atoi(e) : -1;
    }
    if (forced >= 0 && forced < kNumAxisVariants && (need_nl == 0 || kAxisVariants[forced].nl == need_nl)) {
        bool ok = true;
        for (const auto &p : plans) ok = ok && variant_fits(forced, p);
        if (ok) return forced;
    }
    // measured on B200 (512x256x384 world, 8 fields): 16-line tiles with 32
    // threads per line and 2 resident blocks first
    static const int pref[] = {2, 3, 1, 0, 5, 4};
    for (int v : pref) {
        if (need_nl && kAxisVariants[v].nl != need_nl) continue;
        bool ok = true;
        for (const auto &p : plans) ok = ok && variant_fits(v, p);
        if (ok) return v;
    }
    return -1;
}

// Plan and kernel-variant lookup without heap use, for the allocation-free
// entry point (vfd_noalloc.cu); same radices and variant preference as above.
bool plan_for_length(int F, FftPlan *p) { return make_plan(F, p) && any_variant_fits(*p); }

int variant_for_plan(const FftPlan &p, int need_nl)
{
    static const int pref[] = {2, 3, 1, 0, 5, 4};
    for (int v : pref) {
        if (need_nl && kAxisVariants[v].nl != need_nl) continue;
        if (variant_fits(v, p)) return v;
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

// A register-FFT launch of one axis (tiles of every radius).
struct RfGroup {
    int r = 0;  // unused: the kernel reads each tile's radius from its job
    int ntiles = 0;
    OsTileInfo *d_tiles = nullptr;
    CUtensorMap *d_maps = nullptr;  // y / z: one TMA map per job (NULL: direct loads)
    bool owned = true;              // false: the arrays live in their owner's arena
};

// A register-FFT launch's arrays on the host, before they are placed.
struct RfGroupHost {
    std::vector<OsTileInfo> tiles;
    std::vector<CUtensorMap> maps;
};

// Device arrays of one object in a single allocation: staged on the host,
// then one cudaMalloc and one copy (a server builds a batch every time its
// active set changes; one allocation and copy instead of a dozen).
struct ArenaBuilder {
    std::vector<unsigned char> host;
    size_t add(const void *p, size_t bytes, size_t align = 256)
    {
        const size_t off = (host.size() + align - 1) & ~(align - 1);
        host.resize(off + bytes);
        if (bytes) memcpy(host.data() + off, p, bytes);
        return off;
    }
};

static bool rf_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_RF");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1;
}

// Tiles (and TMA maps) of jobs[0..n) (all rf-eligible) for one launch, on
// the host.  Job indices in the tiles are positions in `jobs`.
static void rf_group_host(const OsJob *jobs, int n, RfGroupHost &h)
{
    // CTAs start in tile order: grouping tiles by radius keeps the warps
    // resident together on one compiled variant (instruction-cache locality);
    // jobs are bucketed by radius (1..RF_RMAX), job order kept within a radius
    std::vector<OsTileInfo> t;
    for (int r = 1; r <= RF_RMAX; ++r)
        for (int i = 0; i < n; ++i)
            if (jobs[i].r == r || (r == RF_RMAX && (jobs[i].r < 1 || jobs[i].r > RF_RMAX))) rf_append_tiles(jobs[i], i, t);
    if (t.empty()) return;
    // CTAs of W warps: each job's run of tiles padded to a multiple of W
    const int W = rf_cta_warps(jobs[0].kind);
    if (W > 1) {
        std::vector<OsTileInfo> p;
        p.reserve(t.size() + (size_t)n * W);
        for (size_t i = 0; i < t.size(); ++i) {
            p.push_back(t[i]);
            if (i + 1 == t.size() || t[i + 1].job != t[i].job)
                while (p.size() % W) p.push_back(OsTileInfo{t[i].job, 0, 0, 0});
        }
        t.swap(p);
    }
    // TMA tensor maps (x: two per job, y / z: one) when every job's layout
    // allows them; the CTA widths the TMA kernels take (x 2 warps, y / z 4)
    std::vector<CUtensorMap> maps;
    const bool xpass = jobs[0].kind == PASS_X;
    const int per = xpass ? 2 : 1;
    if (rf_tma_enabled() && W == (xpass ? 2 : 4)) {
        maps.resize((size_t)n * per);
        for (int i = 0; i < n && !maps.empty(); ++i)
            if (!rf_encode_map(jobs[i], &maps[(size_t)i * per])) maps.clear();
    }
    h.tiles.swap(t);
    h.maps.swap(maps);
}

// rf_group_host, uploaded to arrays of its own.
static cudaError_t build_rf_groups(const OsJob *jobs, int n, std::vector<RfGroup> &out)
{
    RfGroupHost h;
    rf_group_host(jobs, n, h);
    if (h.tiles.empty()) return cudaSuccess;
    const std::vector<OsTileInfo> &t = h.tiles;
    const std::vector<CUtensorMap> &maps = h.maps;
    RfGroup g;
    g.r = 0;
    g.ntiles = (int)t.size();
    cudaError_t e = cudaMalloc(&g.d_tiles, sizeof(OsTileInfo) * t.size());
    if (e == cudaSuccess) e = cudaMemcpy(g.d_tiles, t.data(), sizeof(OsTileInfo) * t.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !maps.empty()) {
        e = cudaMalloc(&g.d_maps, sizeof(CUtensorMap) * maps.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(g.d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(g.d_tiles);
        cudaFree(g.d_maps);
        return e;
    }
    out.push_back(g);
    return cudaSuccess;
}

static void free_rf_groups(std::vector<RfGroup> &g)
{
    for (auto &x : g)
        if (x.owned) {
            cudaFree(x.d_tiles);
            cudaFree(x.d_maps);
        }
    g.clear();
}

static cudaError_t launch_rf_groups(const OsJob *jobs, const std::vector<RfGroup> &g, int axis, cudaStream_t st)
{
    for (const auto &x : g) {
        cudaError_t e = launch_rf(jobs, x.d_tiles, x.ntiles, axis, st, x.d_maps);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

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
    // overlap-save passes (kernel radius <= OS_RMAX): per axis
    bool use_os[3] = {false, false, false};
    int rmin[3] = {0, 0, 0};
    OsJob *d_osjobs = nullptr;             // [pass][nf] all-field, then [pass][nf] single-field
    std::vector<int> os_tiles[3];          // per field
    OsTileInfo *d_os_tiles[3] = {nullptr, nullptr, nullptr};    // all-field launches
    OsTileInfo *d_os_ftiles[3] = {nullptr, nullptr, nullptr};   // single-field launches, [field][tiles]
    bool use_rf[3] = {false, false, false};       // register-FFT pass (radius <= RF_RMAX)
    bool allow_rf[3] = {true, true, true};        // tuning may keep an axis off the register-FFT pass
    int os_minb[3] = {0, 0, 0};                   // overlap-save CTAs per SM (0: default)
    int plan_order[3] = {0, 0, 0};                // full-line radix order
    float tuned_ms[3] = {0.0f, 0.0f, 0.0f};       // tuned pass times (0: not tuned)
    std::vector<RfGroup> rf[3];                   // all-field launches
    std::vector<std::vector<RfGroup>> rf_field[3];  // single-field launches

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
    uint64_t src_gen = 0;            // bumped whenever the device source lists change

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

    // general 3D methods (VFD_METHOD_FFT3D / VFD_METHOD_PLAIN)
    int method = VFD_METHOD_SEPARABLE;
    int Fxh = 0;
    int gvar[3] = {0, 0, 0};         // kernel variants of the x rows, y and z columns
    float2 *d_kspec = nullptr;       // [f][Fz][Fy][Fxh], unscaled K
    float2 *d_C = nullptr;           // spectrum scratch
    float *d_P = nullptr;            // full real grid scratch (plain)
    std::vector<float> k0;           // K(0,0,0) = sum of the window, per field
    float *d_upd = nullptr;          // vfd_diffuse_update_host: the fields' dChem on the device
    std::vector<OsJob> oj_host;      // [axis][nf] overlap-save jobs (host copy, reused by batches)

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
    cudaFree(w->d_osjobs);
    for (int a = 0; a < 3; ++a) {
        cudaFree(w->d_os_tiles[a]);
        cudaFree(w->d_os_ftiles[a]);
        free_rf_groups(w->rf[a]);
        for (auto &g : w->rf_field[a]) free_rf_groups(g);
        w->rf_field[a].clear();
    }
    cudaFree(w->d_err);
    cudaFree(w->d_src_idx);
    cudaFree(w->d_src_amt);
    cudaFree(w->d_dep);
    cudaFree(w->d_kspec);
    cudaFree(w->d_C);
    cudaFree(w->d_P);
    cudaFree(w->d_upd);
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
// Tiles of one field for axis a when a launch uses nl lines per tile.
static int field_tiles(const vfd_world *w, int a, int nl)
{
    const int nr = 2 * nl;
    if (a == PASS_X) return (w->ny * w->nz + nr - 1) / nr;
    if (a == PASS_Y) return w->nz * ((w->nx + nr - 1) / nr);
    return w->ny * ((w->nx + nr - 1) / nr);
}

static AxisJob make_job(const vfd_world *w, int f, int a, int tile_begin, int nl)
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
    const int nr = 2 * nl;
    j.tiles_per_outer = (j.nlines + nr - 1) / nr;
    j.tile_begin = tile_begin;
    return j;
}

static bool os_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_OS");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1;
}

static bool os_plain_staging(const OsJob &j);

// Copies v to a new device array (at least one element).
template <class T>
static cudaError_t upload_vec(T **d, const std::vector<T> &v)
{
    cudaError_t e = cudaMalloc(d, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
}

static OsJob make_os_job(const vfd_world *w, int f, int a, int tile_begin)
{
    const AxisJob aj = make_job(w, f, a, 0, 16);
    OsJob j;
    memset(&j, 0, sizeof(j));
    j.data = aj.data;
    j.mass = aj.mass;
    j.line_stride = aj.line_stride;
    j.outer_stride = aj.outer_stride;
    j.pos_stride = aj.pos_stride;
    j.n = aj.n;
    j.nlines = aj.nlines;
    j.nouter = aj.nouter;
    j.r = w->params[f].radius[a];
    j.L = OS_N - 2 * j.r;
    j.C = OS_M * j.L;
    j.ofirst = os_first_output(j.r, a);
    j.nblocks = (j.n + j.r - j.ofirst + j.L - 1) / j.L;
    j.nchunks = (j.nblocks + OS_M - 1) / OS_M;
    j.tiles_per_outer = (j.nlines + 31) / 32;
    j.tile_begin = tile_begin;
    j.kind = a;
    j.b = aj.b;
    j.keep = aj.keep;
    j.nx = aj.nx;
    j.ny = aj.ny;
    for (int i = 0; i < 3; ++i) {
        j.box_lo[i] = aj.box_lo[i];
        j.box_hi[i] = aj.box_hi[i];
    }
    j.mask = os_plain_staging(j) ? 0 : 1;
    os_finish_job(j);
    std::vector<float> h;
    gauss_spectrum(w->params[f].sigma[a], j.r, OS_N, h);
    for (int k = 0; k < OS_N; ++k) j.HH[k] = make_float2(h[k], h[k]);
    return j;
}

static int os_field_tiles(const OsJob &j) { return j.nouter * j.tiles_per_outer; }

// True when the pass stages samples unchanged (no padding-rule transform).
static bool os_plain_staging(const OsJob &j)
{
    if (j.kind != PASS_X) return true;
    return j.b == 0.0f && j.box_lo[0] == 0 && j.box_hi[0] == j.nx && j.box_lo[1] == 0 && j.box_hi[1] == j.ny &&
           j.box_lo[2] == 0 && j.box_hi[2] == j.nlines / j.ny;
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

// ---------------------------------------------------------------------------
// Autotuning: per axis, the pass (register FFT, overlap-save at 3 or 4 CTAs
// per SM, full-line Stockham with a chosen FFT length, radix order and kernel
// variant), timed on a temporary world of the same shape and cached per
// shape; vfd_world_create applies a cached choice.
// ---------------------------------------------------------------------------
enum { PASS_METHOD_AUTO = -1, PASS_METHOD_RF = 0, PASS_METHOD_OS = 1, PASS_METHOD_FULL = 2 };

struct AxisChoice {
    int method = PASS_METHOD_AUTO;
    int minb = 0;      // overlap-save CTAs per SM
    int F = 0;         // full line: FFT length
    int order = 0;     // full line: radix order
    int variant = -1;  // full line: kernel variant
    float ms = 0.0f;
};
struct ShapeChoice {
    AxisChoice ax[3];
};

static std::mutex g_tune_mu;
static std::map<std::string, ShapeChoice> g_tune_cache;

// Cache key: device, grid, padding rule and every field's radius per axis.
static std::string shape_key(const vfd_world_desc *d, int device)
{
    std::string k = std::to_string(device) + ":" + std::to_string(d->nx) + "x" + std::to_string(d->ny) + "x" +
                    std::to_string(d->nz) + ":p" + std::to_string(d->pad_mode) + ":e" +
                    std::to_string(d->pad_mode == VFD_PAD_CONSTANT_VF ? d->epi_boundary : 0) + ":m" +
                    std::to_string(d->method) + ":r";
    for (int f = 0; f < d->n_fields; ++f)
        for (int a = 0; a < 3; ++a) {
            int r = d->fields[f].radius[a];
            if (r <= 0) r = (int)std::ceil(3.0 * d->fields[f].sigma[a]);
            k += std::to_string(r) + ",";
        }
    return k;
}

static bool cached_choice(const vfd_world_desc *d, int device, ShapeChoice *out)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(shape_key(d, device));
    if (it == g_tune_cache.end()) return false;
    *out = it->second;
    return true;
}

static vfd_status world_create(const vfd_world_desc *d, int device, const ShapeChoice *ch, vfd_world **out);
static vfd_status tune_shape(const vfd_world_desc *d, int device, int reps, ShapeChoice *out);

static bool autotune_on_create()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VFD_AUTOTUNE");
        on = (e && e[0] == '1') ? 1 : 0;
    }
    return on == 1;
}

vfd_status vfd_world_create(const vfd_world_desc *d, int device, vfd_world **out)
{
    if (!out) return fail(nullptr, VFD_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!d || !d->fields) return fail(nullptr, VFD_ERR_INVALID_ARG, "desc or desc->fields is NULL");
    ShapeChoice ch;
    bool have = d->method == VFD_METHOD_SEPARABLE && cached_choice(d, device, &ch);
    if (!have && d->method == VFD_METHOD_SEPARABLE && autotune_on_create() && d->nx >= 1 && d->ny >= 1 &&
        d->nz >= 1 && d->n_fields >= 1 && tune_shape(d, device, 3, &ch) == VFD_OK) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[shape_key(d, device)] = ch;
        have = true;
    }
    return world_create(d, device, have ? &ch : nullptr, out);
}

static vfd_status world_create(const vfd_world_desc *d, int device, const ShapeChoice *ch, vfd_world **out)
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
    w->method = d->method;
    if (w->method < VFD_METHOD_SEPARABLE || w->method > VFD_METHOD_PLAIN) {
        delete w;
        return fail(nullptr, VFD_ERR_INVALID_ARG, "unknown method");
    }
    const bool general = w->method != VFD_METHOD_SEPARABLE;
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
        const int order = ch ? ch->ax[a].order : 0;
        if (F <= 0 && ch && ch->ax[a].F >= dims[a] + rmax[a]) F = ch->ax[a].F;
        if (F > 0) {
            if (F < dims[a] + rmax[a]) {
                delete w;
                return fail(nullptr, VFD_ERR_INVALID_ARG, "fft length shorter than n + radius");
            }
            if (general && a == 0 && (F & 1)) {
                delete w;
                return fail(nullptr, VFD_ERR_INVALID_ARG, "the general 3D methods need an even x FFT length");
            }
            if (!make_plan_order(F, order, &w->plan[a]) || !any_variant_fits(w->plan[a])) {
                delete w;
                return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "fft length not 7-smooth or too long");
            }
            w->plan_order[a] = order;
        } else {
            F = general ? choose_general_len(dims[a], rmax[a], a == 0) : choose_fft_len(dims[a], rmax[a], false);
            if (F < 0) {
                delete w;
                return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "axis too long for the shared-memory FFT");
            }
            make_plan(F, &w->plan[a]);
            FftPlan q;
            if (order != 0 && make_plan_order(F, order, &q) && any_variant_fits(q)) {
                w->plan[a] = q;
                w->plan_order[a] = order;
            }
        }
        w->F[a] = F;
        w->Fmax = std::max(w->Fmax, F);
        w->variant[a] = pick_variant(std::vector<FftPlan>{w->plan[a]});
        if (ch && ch->ax[a].variant >= 0 && ch->ax[a].variant < kNumAxisVariants &&
            variant_fits(ch->ax[a].variant, w->plan[a]))
            w->variant[a] = ch->ax[a].variant;
    }
    for (int a = 0; a < 3; ++a) {
        if (w->variant[a] < 0) {
            delete w;
            return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "no kernel variant fits the FFT plan");
        }
    }
    for (int a = 0; a < 3; ++a) w->tiles_per_field[a] = field_tiles(w, a, kAxisVariants[w->variant[a]].nl);
    if (!general && os_enabled()) {
        for (int a = 0; a < 3; ++a) {
            int rmn = 1 << 30;
            for (int f = 0; f < w->nf; ++f) rmn = std::min(rmn, w->params[f].radius[a]);
            w->use_os[a] = rmax[a] <= OS_RMAX;
            w->rmin[a] = rmn;
        }
    }
    if (ch && !general)
        for (int a = 0; a < 3; ++a) {
            if (ch->ax[a].method == PASS_METHOD_FULL) w->use_os[a] = false;
            if (ch->ax[a].method == PASS_METHOD_OS || ch->ax[a].method == PASS_METHOD_FULL) w->allow_rf[a] = false;
            w->os_minb[a] = ch->ax[a].minb;
            w->tuned_ms[a] = ch->ax[a].ms;
        }
    if (general) {
        w->Fxh = w->F[0] / 2 + 1;
        w->gvar[0] = w->variant[0];
        for (int a = 1; a < 3; ++a) {
            w->gvar[a] = pick_variant(std::vector<FftPlan>{w->plan[a]}, 16);
            if (w->gvar[a] < 0) {
                delete w;
                return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "no 16-line kernel variant fits the FFT plan");
            }
        }
    }

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
                jobs.push_back(make_job(w, f, a, tb, kAxisVariants[w->variant[a]].nl));
                tb += w->tiles_per_field[a];
            }
        }
        for (int a = 0; a < 3; ++a)
            for (int f = 0; f < w->nf; ++f) jobs.push_back(make_job(w, f, a, 0, kAxisVariants[w->variant[a]].nl));
        if ((e = cudaMalloc(&w->d_jobs, sizeof(AxisJob) * jobs.size())) != cudaSuccess) return bail(e, "cudaMalloc jobs");
        if ((e = cudaMemcpy(w->d_jobs, jobs.data(), sizeof(AxisJob) * jobs.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e, "cudaMemcpy jobs");
    }
    if (w->use_os[0] || w->use_os[1] || w->use_os[2]) {
        std::vector<OsJob> oj;
        for (int a = 0; a < 3; ++a) {
            int tb = 0;
            w->os_tiles[a].assign(w->nf, 0);
            for (int f = 0; f < w->nf; ++f) {
                oj.push_back(make_os_job(w, f, a, tb));
                w->os_tiles[a][f] = os_field_tiles(oj.back());
                tb += w->os_tiles[a][f];
            }
        }
        w->oj_host.assign(oj.begin(), oj.end());
        for (int a = 0; a < 3; ++a)
            for (int f = 0; f < w->nf; ++f) oj.push_back(make_os_job(w, f, a, 0));
        if ((e = os_prepare()) != cudaSuccess) return bail(e, "overlap-save twiddles");
        if ((e = cudaMalloc(&w->d_osjobs, sizeof(OsJob) * oj.size())) != cudaSuccess) return bail(e, "cudaMalloc os jobs");
        if ((e = cudaMemcpy(w->d_osjobs, oj.data(), sizeof(OsJob) * oj.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e, "cudaMemcpy os jobs");
        for (int a = 0; a < 3; ++a) {
            std::vector<OsTileInfo> all, one;
            for (int f = 0; f < w->nf; ++f) {
                os_append_tiles(oj[(size_t)a * w->nf + f], f, all);
                os_append_tiles(oj[(size_t)(3 + a) * w->nf + f], 0, one);
            }
            if ((e = upload_vec(&w->d_os_tiles[a], all)) != cudaSuccess ||
                (e = upload_vec(&w->d_os_ftiles[a], one)) != cudaSuccess)
                return bail(e, "os tiles");
        }
        for (int a = 0; a < 3 && rf_enabled(); ++a) {
            bool ok = w->use_os[a] && w->allow_rf[a];
            for (int f = 0; f < w->nf; ++f) ok = ok && rf_eligible(oj[(size_t)a * w->nf + f]);
            if (!ok) continue;
            if ((e = rf_prepare()) != cudaSuccess) return bail(e, "register-FFT twiddles");
            if ((e = build_rf_groups(&oj[(size_t)a * w->nf], w->nf, w->rf[a])) != cudaSuccess) return bail(e, "rf tiles");
            w->rf_field[a].resize(w->nf);
            for (int f = 0; f < w->nf; ++f)
                if ((e = build_rf_groups(&oj[(size_t)(3 + a) * w->nf + f], 1, w->rf_field[a][f])) != cudaSuccess)
                    return bail(e, "rf tiles");
            w->use_rf[a] = true;
        }
    }
    if ((e = cudaMalloc(&w->d_dep, sizeof(DepositJob) * 2 * w->nf)) != cudaSuccess) return bail(e, "cudaMalloc deposit jobs");
    if (general) {
        const int64_t nk = (int64_t)w->Fxh * w->F[1] * w->F[2];
        if ((e = cudaMalloc(&w->d_kspec, sizeof(float2) * nk * w->nf)) != cudaSuccess) return bail(e, "cudaMalloc spectra");
        for (int f = 0; f < w->nf; ++f) {
            const float *sp = w->d_spec + (int64_t)f * 3 * w->Fmax;
            if ((e = launch_outer_spectrum(w->d_kspec + nk * f, sp, sp + w->Fmax, sp + 2 * w->Fmax, w->F[0], w->F[1],
                                           w->F[2], 0)) != cudaSuccess)
                return bail(e, "outer spectrum");
        }
        w->k0.assign(w->nf, 1.0f);
        const int64_t nc = (w->method == VFD_METHOD_PLAIN) ? nk : (int64_t)w->Fxh * w->F[1] * w->nz;
        if ((e = cudaMalloc(&w->d_C, sizeof(float2) * nc)) != cudaSuccess) return bail(e, "cudaMalloc spectrum scratch");
        if (w->method == VFD_METHOD_PLAIN) {
            if ((e = cudaMalloc(&w->d_P, sizeof(float) * (int64_t)w->F[0] * w->F[1] * w->F[2])) != cudaSuccess)
                return bail(e, "cudaMalloc padded grid");
        }
    }
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
    // the set-up above ran on the legacy stream; work on other streams (a
    // batch running on this device) is not waited for
    if ((e = cudaStreamSynchronize(0)) != cudaSuccess) return bail(e, "cudaStreamSynchronize");
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
    if (w->method != VFD_METHOD_SEPARABLE) {
        const size_t nk = (size_t)w->Fxh * w->F[1] * w->F[2];
        b += sizeof(float2) * nk * w->nf;
        b += sizeof(float2) * ((w->method == VFD_METHOD_PLAIN) ? nk : (size_t)w->Fxh * w->F[1] * w->nz);
        if (w->method == VFD_METHOD_PLAIN) b += sizeof(float) * (size_t)w->F[0] * w->F[1] * w->F[2];
    }
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

static void interior_box(const vfd_world *w, int *lo, int *hi)
{
    if (w->pad_mode == VFD_PAD_CONSTANT_VF) {
        lo[0] = 1; hi[0] = std::min(w->epi, w->nx);
        lo[1] = 1; hi[1] = w->ny - 1;
        lo[2] = 1; hi[2] = w->nz - 1;
    } else {
        lo[0] = 0; hi[0] = w->nx;
        lo[1] = 0; hi[1] = w->ny;
        lo[2] = 0; hi[2] = w->nz;
    }
}

static GenColPass col_pass(const vfd_world *w, int a, float2 *data, int nouter, int nload, int nstore, int mode)
{
    GenColPass c;
    memset(&c, 0, sizeof(c));
    c.plan = w->plan[a];
    c.tw = w->d_tw[a];
    c.data = data;
    c.nlines = w->Fxh;
    c.nouter = nouter;
    if (a == PASS_Y) {
        c.outer_stride = (int64_t)w->F[1] * w->Fxh;
        c.pos_stride = w->Fxh;
    } else {
        c.outer_stride = w->Fxh;
        c.pos_stride = (int64_t)w->F[1] * w->Fxh;
    }
    c.nload = nload;
    c.nstore = nstore;
    c.mode = mode;
    c.scale = 1.0f;
    return c;
}

vfd_status vfd_set_window(vfd_world *w, int field, const float *window, int kw, int kh, int kd, int cx, int cy,
                          int cz)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (w->method == VFD_METHOD_SEPARABLE)
        return fail(w, VFD_ERR_NOT_SUPPORTED, "dense windows need VFD_METHOD_FFT3D or VFD_METHOD_PLAIN");
    if (field < 0 || field >= w->nf || !window || kw < 1 || kh < 1 || kd < 1 || cx < 0 || cx >= kw || cy < 0 ||
        cy >= kh || cz < 0 || cz >= kd)
        return fail(w, VFD_ERR_INVALID_ARG, "bad field, window dims or centre");
    const int Fx = w->F[0], Fy = w->F[1], Fz = w->F[2];
    // the wrapped window must not alias onto the data: half-widths within F - n
    if (std::max(cx, kw - 1 - cx) > Fx - w->nx || std::max(cy, kh - 1 - cy) > Fy - w->ny ||
        std::max(cz, kd - 1 - cz) > Fz - w->nz)
        return fail(w, VFD_ERR_INVALID_ARG, "window wider than the FFT padding; pass larger fft lengths");
    DeviceGuard g(w->device);
    const int64_t nk = (int64_t)w->Fxh * Fy * Fz;
    const int64_t np = (int64_t)Fx * Fy * Fz;
    const int64_t nwin = (int64_t)kw * kh * kd;
    float *P = nullptr, *dw = nullptr;
    VFD_CUDA(w, cudaMalloc(&P, sizeof(float) * np));
    cudaError_t e = cudaMalloc(&dw, sizeof(float) * nwin);
    if (e != cudaSuccess) {
        cudaFree(P);
        return fail(w, VFD_ERR_OUT_OF_MEMORY, "cudaMalloc window");
    }
    float2 *K = w->d_kspec + nk * field;
    double wsum = 0.0;
    for (int64_t i = 0; i < nwin; ++i) wsum += window[i];
    auto run = [&]() -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpy(dw, window, sizeof(float) * nwin, cudaMemcpyHostToDevice)) != cudaSuccess) return r;
        if ((r = cudaMemset(P, 0, sizeof(float) * np)) != cudaSuccess) return r;
        if ((r = launch_wrap_window(P, dw, kw, kh, kd, cx, cy, cz, Fx, Fy, Fz, 0)) != cudaSuccess) return r;
        GenRowPass rp;
        memset(&rp, 0, sizeof(rp));
        rp.plan = w->plan[0];
        rp.tw = w->d_tw[0];
        rp.nrows = Fy * Fz;
        rp.rows_per_plane = Fy;
        rp.r_s1 = Fx;
        rp.r_s2 = (int64_t)Fx * Fy;
        rp.c_s1 = w->Fxh;
        rp.c_s2 = (int64_t)w->Fxh * Fy;
        rp.nload = Fx;
        rp.rsrc = P;
        rp.cdst = K;
        if ((r = launch_gen_rows(w->gvar[0], rp, false, 0)) != cudaSuccess) return r;
        if ((r = launch_gen_cols(w->gvar[1], col_pass(w, PASS_Y, K, Fz, Fy, Fy, GEN_FORWARD), 0)) != cudaSuccess)
            return r;
        if ((r = launch_gen_cols(w->gvar[2], col_pass(w, PASS_Z, K, Fy, Fz, Fz, GEN_FORWARD), 0)) != cudaSuccess)
            return r;
        return cudaDeviceSynchronize();
    };
    e = run();
    cudaFree(P);
    cudaFree(dw);
    if (e != cudaSuccess) return fail(w, VFD_ERR_CUDA, std::string("window spectrum: ") + cudaGetErrorString(e));
    w->k0[field] = (float)wsum;
    return VFD_OK;
}

vfd_status vfd_check_wait_timeout(int device, long long limit_cycles)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, VFD_ERR_NO_DEVICE, "no device");
    if (device < 0 || device >= ndev || limit_cycles < 1 || limit_cycles > 4000000000ll)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "bad device or wait limit");
    DeviceGuard g(device);
    int *d = nullptr;
    int h = 0;
    cudaError_t e = cudaMalloc(&d, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(int));
    if (e == cudaSuccess) e = rf_wait_probe(limit_cycles, d, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(nullptr, VFD_ERR_CUDA, std::string("wait probe: ") + cudaGetErrorString(e));
    const bool flagged = rf_take_timeout();
    if (h && flagged) return fail(nullptr, VFD_ERR_TIMEOUT, "the bounded wait gave up and reported it");
    return fail(nullptr, VFD_ERR_CUDA, "the bounded wait did not report giving up");
}

vfd_status vfd_window_spectrum(const float *window, int kw, int kh, int kd, int cx, int cy, int cz, int fx, int fy,
                               int fz, float *out, int device)
{
    if (!window || !out || kw < 1 || kh < 1 || kd < 1 || cx < 0 || cx >= kw || cy < 0 || cy >= kh || cz < 0 ||
        cz >= kd)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "bad window, centre or output");
    const int rx = std::max(1, std::max(cx, kw - 1 - cx)), ry = std::max(1, std::max(cy, kh - 1 - cy)),
              rz = std::max(1, std::max(cz, kd - 1 - cz));
    if (fx - rx < 1 || fy - ry < 1 || fz - rz < 1 || (fx & 1))
        return fail(nullptr, VFD_ERR_INVALID_ARG, "FFT grid smaller than the window (or odd x length)");
    // a one-field world whose FFT grid is (fx, fy, fz): its set-up computes the
    // spectrum with this library's transform
    vfd_field_params p;
    memset(&p, 0, sizeof(p));
    p.sigma[0] = p.sigma[1] = p.sigma[2] = 1.0;
    p.radius[0] = rx;
    p.radius[1] = ry;
    p.radius[2] = rz;
    vfd_world_desc d;
    memset(&d, 0, sizeof(d));
    d.nx = fx - rx;
    d.ny = fy - ry;
    d.nz = fz - rz;
    d.n_fields = 1;
    d.fields = &p;
    d.fft[0] = fx;
    d.fft[1] = fy;
    d.fft[2] = fz;
    d.method = VFD_METHOD_FFT3D;
    vfd_world *w = nullptr;
    vfd_status st = vfd_world_create(&d, device, &w);
    if (st != VFD_OK) return st;
    st = vfd_set_window(w, 0, window, kw, kh, kd, cx, cy, cz);
    if (st == VFD_OK) {
        DeviceGuard g(w->device);
        const int64_t nk = (int64_t)w->Fxh * fy * fz;
        cudaError_t e = cudaMemcpy(out, w->d_kspec, sizeof(float2) * nk, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            g_thread_error = std::string("window spectrum: ") + cudaGetErrorString(e);
            st = VFD_ERR_CUDA;
        }
    } else {
        g_thread_error = w->err;
    }
    vfd_world_destroy(w);
    return st;
}

vfd_status vfd_spectrum_window(const float *kspec, int fx, int fy, int fz, int kw, int kh, int kd, int cx, int cy,
                               int cz, float *window, int device)
{
    if (!kspec || !window || kw < 1 || kh < 1 || kd < 1 || cx < 0 || cx >= kw || cy < 0 || cy >= kh || cz < 0 ||
        cz >= kd || kw > fx || kh > fy || kd > fz)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "bad spectrum grid, window or centre");
    // a one-field world on the (fx, fy, fz) grid: its plans, twiddles and
    // kernel variants run the inverse transform
    vfd_field_params p;
    memset(&p, 0, sizeof(p));
    p.sigma[0] = p.sigma[1] = p.sigma[2] = 1.0;
    p.radius[0] = p.radius[1] = p.radius[2] = 1;
    vfd_world_desc d;
    memset(&d, 0, sizeof(d));
    d.nx = fx - 1;
    d.ny = fy - 1;
    d.nz = fz - 1;
    d.n_fields = 1;
    d.fields = &p;
    d.fft[0] = fx;
    d.fft[1] = fy;
    d.fft[2] = fz;
    d.method = VFD_METHOD_FFT3D;
    vfd_world *w = nullptr;
    vfd_status st = vfd_world_create(&d, device, &w);
    if (st != VFD_OK) return st;
    st = vfd_set_spectrum(w, 0, kspec, fx, fy, fz);
    if (st != VFD_OK) {
        g_thread_error = w->err;
        vfd_world_destroy(w);
        return st;
    }
    DeviceGuard g(w->device);
    const int64_t np = (int64_t)fx * fy * fz;
    float *P = nullptr, *dw = nullptr;
    cudaError_t e = cudaMalloc(&P, sizeof(float) * np);
    if (e == cudaSuccess) e = cudaMalloc(&dw, sizeof(float) * (int64_t)kw * kh * kd);
    if (e == cudaSuccess) {
        // inverse z, inverse y (in place on the stored spectrum), C2R along x
        float2 *K = w->d_kspec;
        e = launch_gen_cols(w->gvar[2], col_pass(w, PASS_Z, K, fy, fz, fz, GEN_INVERSE), 0);
        if (e == cudaSuccess) e = launch_gen_cols(w->gvar[1], col_pass(w, PASS_Y, K, fz, fy, fy, GEN_INVERSE), 0);
        if (e == cudaSuccess) {
            GenRowPass rp;
            memset(&rp, 0, sizeof(rp));
            rp.plan = w->plan[0];
            rp.tw = w->d_tw[0];
            rp.nrows = fy * fz;
            rp.rows_per_plane = fy;
            rp.r_s1 = fx;
            rp.r_s2 = (int64_t)fx * fy;
            rp.c_s1 = w->Fxh;
            rp.c_s2 = (int64_t)w->Fxh * fy;
            rp.nstore = fx;
            rp.rdst = P;
            rp.csrc = K;
            e = launch_gen_rows(w->gvar[0], rp, true, 0);
        }
        if (e == cudaSuccess)
            e = launch_unwrap_window(dw, P, kw, kh, kd, cx, cy, cz, fx, fy, fz, (float)(1.0 / (double)np), 0);
        if (e == cudaSuccess)
            e = cudaMemcpy(window, dw, sizeof(float) * (int64_t)kw * kh * kd, cudaMemcpyDeviceToHost);
    }
    cudaFree(P);
    cudaFree(dw);
    vfd_world_destroy(w);
    if (e != cudaSuccess) return fail(nullptr, VFD_ERR_CUDA, std::string("spectrum window: ") + cudaGetErrorString(e));
    return VFD_OK;
}

vfd_status vfd_set_spectrum(vfd_world *w, int field, const float *kspec, int fx, int fy, int fz)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (w->method == VFD_METHOD_SEPARABLE)
        return fail(w, VFD_ERR_NOT_SUPPORTED, "stored spectra need VFD_METHOD_FFT3D or VFD_METHOD_PLAIN");
    if (field < 0 || field >= w->nf || !kspec) return fail(w, VFD_ERR_INVALID_ARG, "bad field or NULL spectrum");
    if (fx != w->F[0] || fy != w->F[1] || fz != w->F[2])
        return fail(w, VFD_ERR_INVALID_ARG,
                    "spectrum grid " + std::to_string(fx) + "x" + std::to_string(fy) + "x" + std::to_string(fz) +
                        " differs from the world's FFT grid " + std::to_string(w->F[0]) + "x" +
                        std::to_string(w->F[1]) + "x" + std::to_string(w->F[2]) +
                        " (create the world with desc.fft = {FFTW, FFTH, FFTD})");
    DeviceGuard g(w->device);
    const int64_t nk = (int64_t)w->Fxh * w->F[1] * w->F[2];
    float2 *K = w->d_kspec + nk * field;
    // cudaMemcpyDefault: host (pinned or pageable) or device source
    VFD_CUDA(w, cudaMemcpy(K, kspec, sizeof(float2) * nk, cudaMemcpyDefault));
    float2 dc;
    VFD_CUDA(w, cudaMemcpy(&dc, K, sizeof(float2), cudaMemcpyDeviceToHost));
    w->k0[field] = dc.x;
    return VFD_OK;
}

vfd_status vfd_set_boundary(vfd_world *w, int epi_boundary, const float *baselines)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (w->method == VFD_METHOD_SEPARABLE)
        return fail(w, VFD_ERR_NOT_SUPPORTED, "separable worlds fix their padding at creation");
    if (baselines)
        for (int f = 0; f < w->nf; ++f)
            if (!std::isfinite(baselines[f])) return fail(w, VFD_ERR_INVALID_ARG, "baseline must be finite");
    w->epi = epi_boundary;
    if (baselines)
        for (int f = 0; f < w->nf; ++f) w->params[f].baseline = baselines[f];
    return VFD_OK;
}

// Uploads the concatenated source list and deposit jobs when they changed,
// ordered on stream `st` before the tick that follows.  The lists grow by
// stream-ordered allocation (cudaMallocAsync / cudaFreeAsync), so a world
// whose sources grow does not wait for work in flight on other streams (a
// server reusing worlds keeps several rounds queued on the device).
static vfd_status sync_sources(vfd_world *w, cudaStream_t st)
{
    if (!w->src_dirty) return VFD_OK;
    int64_t total = 0;
    for (int f = 0; f < w->nf; ++f) {
        w->src_begin[f] = total;
        w->src_count[f] = (int64_t)w->src_idx[f].size();
        total += w->src_count[f];
    }
    if (total > w->src_cap) {
        if (w->d_src_idx) VFD_CUDA(w, cudaFreeAsync(w->d_src_idx, st));
        if (w->d_src_amt) VFD_CUDA(w, cudaFreeAsync(w->d_src_amt, st));
        w->d_src_idx = nullptr;
        w->d_src_amt = nullptr;
        w->src_cap = 0;
        const int64_t cap = std::max<int64_t>(total, 2 * w->src_total);
        VFD_CUDA(w, cudaMallocAsync(&w->d_src_idx, sizeof(int32_t) * cap, st));
        VFD_CUDA(w, cudaMallocAsync(&w->d_src_amt, sizeof(float) * cap, st));
        w->src_cap = cap;
    }
    std::vector<int32_t> hi(total);
    std::vector<float> ha(total);
    for (int f = 0; f < w->nf; ++f) {
        std::copy(w->src_idx[f].begin(), w->src_idx[f].end(), hi.begin() + w->src_begin[f]);
        std::copy(w->src_amt[f].begin(), w->src_amt[f].end(), ha.begin() + w->src_begin[f]);
    }
    // pageable sources: each copy returns once its data is staged
    if (total > 0) {
        VFD_CUDA(w, cudaMemcpyAsync(w->d_src_idx, hi.data(), sizeof(int32_t) * total, cudaMemcpyHostToDevice, st));
        VFD_CUDA(w, cudaMemcpyAsync(w->d_src_amt, ha.data(), sizeof(float) * total, cudaMemcpyHostToDevice, st));
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
    VFD_CUDA(w, cudaMemcpyAsync(w->d_dep, jobs.data(), sizeof(DepositJob) * jobs.size(), cudaMemcpyHostToDevice, st));
    w->src_total = total;
    w->src_dirty = false;
    w->src_gen++;
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

// The WHChemical::update epilogue of vfd_tick_update: per field the device
// array d (NULL: zero) and the retention factor of p = d + decay * t.
struct UpdateArgs {
    float *const *dchem;  // n_fields entries, or NULL
    const float *decay;   // n_fields entries
};

// One substep of field f with the general 3D transform; with `upd` the crop
// store applies the update epilogue.
static vfd_status enqueue_general_substep(vfd_world *w, int f, cudaStream_t st, const UpdateArgs *upd = nullptr)
{
    const int Fx = w->F[0], Fy = w->F[1], Fz = w->F[2];
    const int64_t nk = (int64_t)w->Fxh * Fy * Fz;
    float *u = w->d_fields + (int64_t)f * w->V;
    double *mass = w->d_mass + (int64_t)f * MS_COUNT;
    const float2 *K = w->d_kspec + nk * f;
    const float invN = (float)(1.0 / ((double)Fx * Fy * Fz));
    const float b = w->pad_mode == VFD_PAD_CONSTANT_VF ? w->params[f].baseline : 0.0f;
    const float keep = (float)(1.0 - w->params[f].decay_rate);
    int lo[3], hi[3];
    interior_box(w, lo, hi);
    GenRowPass r;
    memset(&r, 0, sizeof(r));
    r.plan = w->plan[0];
    r.tw = w->d_tw[0];
    r.c_s1 = w->Fxh;
    r.c_s2 = (int64_t)w->Fxh * Fy;
    if (w->method == VFD_METHOD_FFT3D) {
        // pruned + fused: rows of the data only; C holds z < nz
        r.nrows = w->ny * w->nz;
        r.rows_per_plane = w->ny;
        r.r_s1 = w->nx;
        r.r_s2 = (int64_t)w->nx * w->ny;
        r.nload = w->nx;
        r.nstore = w->nx;
        r.rsrc = u;
        r.rdst = u;
        r.cdst = w->d_C;
        r.csrc = w->d_C;
        r.fuse_pad = 1;
        for (int i = 0; i < 3; ++i) {
            r.box_lo[i] = lo[i];
            r.box_hi[i] = hi[i];
        }
        r.b = b;
        r.mass_in = mass + MS_INPUT;
        {
            LaunchTimer lt(w, 0, st);
            VFD_CUDA(w, launch_gen_rows(w->gvar[0], r, false, st));
            lt.done();
        }
        {
            LaunchTimer lt(w, 1, st);
            VFD_CUDA(w, launch_gen_cols(w->gvar[1], col_pass(w, PASS_Y, w->d_C, w->nz, w->ny, Fy, GEN_FORWARD), st));
            lt.done();
        }
        {
            GenColPass c = col_pass(w, PASS_Z, w->d_C, Fy, w->nz, w->nz, GEN_FWD_MUL_INV);
            c.kspec = K;
            c.k_s_outer = w->Fxh;
            c.k_s_pos = (int64_t)w->Fxh * Fy;
            c.scale = invN;
            LaunchTimer lt(w, 2, st);
            VFD_CUDA(w, launch_gen_cols(w->gvar[2], c, st));
            lt.done();
        }
        {
            LaunchTimer lt(w, 1, st);
            VFD_CUDA(w, launch_gen_cols(w->gvar[1], col_pass(w, PASS_Y, w->d_C, w->nz, Fy, w->ny, GEN_INVERSE), st));
            lt.done();
        }
        r.fuse_pad = 0;
        r.fuse_crop = 1;
        r.keep = keep;
        r.k0 = w->k0[f];
        if (upd) {
            r.fuse_update = 1;
            r.upd_scale = upd->decay[f];
            r.dchem = upd->dchem ? upd->dchem[f] : nullptr;
        }
        r.mass_in = nullptr;
        r.mass_leak = mass + MS_LEAK_X;
        r.mass_conv = mass + MS_CONV;
        r.mass_out = mass + MS_OUT;
        LaunchTimer lt(w, 0, st);
        VFD_CUDA(w, launch_gen_rows(w->gvar[0], r, true, st));
        lt.done();
        return VFD_OK;
    }
    // plain: unfused kernels on the full grid, the reference's order
    VFD_CUDA(w, launch_pad(w->d_P, u, w->nx, w->ny, w->nz, Fx, Fy, Fz, lo, hi, b, st));
    VFD_CUDA(w, launch_sum(w->d_P, (int64_t)Fx * Fy * Fz, mass + MS_INPUT, st));
    r.nrows = Fy * Fz;
    r.rows_per_plane = Fy;
    r.r_s1 = Fx;
    r.r_s2 = (int64_t)Fx * Fy;
    r.nload = Fx;
    r.nstore = Fx;
    r.rsrc = w->d_P;
    r.rdst = w->d_P;
    r.cdst = w->d_C;
    r.csrc = w->d_C;
    VFD_CUDA(w, launch_gen_rows(w->gvar[0], r, false, st));
    VFD_CUDA(w, launch_gen_cols(w->gvar[1], col_pass(w, PASS_Y, w->d_C, Fz, Fy, Fy, GEN_FORWARD), st));
    VFD_CUDA(w, launch_gen_cols(w->gvar[2], col_pass(w, PASS_Z, w->d_C, Fy, Fz, Fz, GEN_FORWARD), st));
    VFD_CUDA(w, launch_modulate(w->d_C, K, nk, invN, st));
    VFD_CUDA(w, launch_gen_cols(w->gvar[2], col_pass(w, PASS_Z, w->d_C, Fy, Fz, Fz, GEN_INVERSE), st));
    VFD_CUDA(w, launch_gen_cols(w->gvar[1], col_pass(w, PASS_Y, w->d_C, Fz, Fy, Fy, GEN_INVERSE), st));
    VFD_CUDA(w, launch_gen_rows(w->gvar[0], r, true, st));
    VFD_CUDA(w, launch_sum(w->d_P, (int64_t)Fx * Fy * Fz, mass + MS_LEAK_X, st));  // full-grid sum, see read_mass
    VFD_CUDA(w, launch_crop(u, w->d_P, w->nx, w->ny, w->nz, Fx, Fy, keep, mass + MS_CONV, mass + MS_OUT, st,
                            upd ? 1 : 0, upd ? upd->decay[f] : 1.0f,
                            (upd && upd->dchem) ? upd->dchem[f] : nullptr));
    return VFD_OK;
}

// Enqueues n_substeps of one field (field >= 0) or of all fields (field < 0).
// One axis pass of every field (field < 0) or of one field, with the pass
// the world uses for that axis.
static vfd_status enqueue_axis(vfd_world *w, int a, int field, cudaStream_t st)
{
    const int nj = field < 0 ? w->nf : 1;
    if (w->use_rf[a]) {
        if (field < 0)
            VFD_CUDA(w, launch_rf_groups(w->d_osjobs + a * w->nf, w->rf[a], a, st));
        else
            VFD_CUDA(w, launch_rf_groups(w->d_osjobs + 3 * w->nf + a * w->nf + field, w->rf_field[a][field], a, st));
    } else if (w->use_os[a]) {
        const OsJob *jobs = field < 0 ? w->d_osjobs + a * w->nf : w->d_osjobs + 3 * w->nf + a * w->nf + field;
        int tiles = 0;
        if (field < 0)
            for (int f = 0; f < w->nf; ++f) tiles += w->os_tiles[a][f];
        else
            tiles = w->os_tiles[a][field];
        const OsTileInfo *ti = w->d_os_tiles[a];
        if (field >= 0) {
            ti = w->d_os_ftiles[a];
            for (int f = 0; f < field; ++f) ti += w->os_tiles[a][f];
        }
        VFD_CUDA(w, launch_os(jobs, ti, tiles, w->rmin[a], a, st, w->os_minb[a]));
    } else {
        const AxisJob *jobs = field < 0 ? w->d_jobs + a * w->nf : w->d_jobs + 3 * w->nf + a * w->nf + field;
        const int tiles = w->tiles_per_field[a] * nj;
        VFD_CUDA(w, launch_axis(w->variant[a], jobs, nj, tiles, w->F[a], st));
    }
    return VFD_OK;
}

static vfd_status enqueue_tick(vfd_world *w, int field, int n_substeps, cudaStream_t st,
                               const UpdateArgs *upd = nullptr)
{
    if (w->method != VFD_METHOD_SEPARABLE) {
        const int f0 = field < 0 ? 0 : field, f1 = field < 0 ? w->nf : field + 1;
        for (int s = 0; s < n_substeps; ++s)
            for (int f = f0; f < f1; ++f) {
                VFD_CUDA(w, cudaMemsetAsync(w->d_mass + (int64_t)f * MS_COUNT, 0, sizeof(double) * MS_COUNT, st));
                vfd_status r = enqueue_general_substep(w, f, st, s + 1 == n_substeps ? upd : nullptr);
                if (r != VFD_OK) return r;
            }
        if (field < 0) {
            if (w->dep_njobs > 0)
                VFD_CUDA(w, launch_deposit(w->d_dep, w->dep_njobs, w->d_src_idx, w->d_src_amt, w->src_total,
                                           w->d_err, st));
        } else if (w->src_count[field] > 0) {
            VFD_CUDA(w, launch_deposit(w->d_dep + w->nf + field, 1, w->d_src_idx + w->src_begin[field],
                                       w->d_src_amt + w->src_begin[field], w->src_count[field], w->d_err, st));
        }
        return VFD_OK;
    }
    for (int s = 0; s < n_substeps; ++s) {
        if (field < 0)
            VFD_CUDA(w, cudaMemsetAsync(w->d_mass, 0, sizeof(double) * MS_COUNT * w->nf, st));
        else
            VFD_CUDA(w, cudaMemsetAsync(w->d_mass + (int64_t)field * MS_COUNT, 0, sizeof(double) * MS_COUNT, st));
        for (int a = 0; a < 3; ++a) {
            LaunchTimer lt(w, a, st);
            vfd_status r = enqueue_axis(w, a, field, st);
            if (r != VFD_OK) return r;
            lt.done();
        }
    }
    if (upd) {
        // the update as one pass per field after the z pass (whose output
        // total it replaces by the total of p)
        const int f0 = field < 0 ? 0 : field, f1 = field < 0 ? w->nf : field + 1;
        for (int f = f0; f < f1; ++f) {
            double *m = w->d_mass + (int64_t)f * MS_COUNT + MS_OUT;
            VFD_CUDA(w, cudaMemsetAsync(m, 0, sizeof(double), st));
            VFD_CUDA(w, launch_update(w->d_fields + (int64_t)f * w->V, upd->dchem ? upd->dchem[f] : nullptr,
                                      upd->decay[f], w->V, m, st));
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
    vfd_status s = sync_sources(w, (cudaStream_t)stream);
    if (s != VFD_OK) return s;
    return enqueue_tick(w, -1, n_substeps, (cudaStream_t)stream);
}

vfd_status vfd_tick_update(vfd_world *w, int n_substeps, float *const *dchem, const float *decay, void *stream)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (n_substeps < 1) return fail(w, VFD_ERR_INVALID_ARG, "n_substeps must be >= 1");
    if (!decay) return fail(w, VFD_ERR_INVALID_ARG, "decay is NULL");
    for (int f = 0; f < w->nf; ++f)
        if (!std::isfinite(decay[f])) return fail(w, VFD_ERR_INVALID_ARG, "decay must be finite");
    DeviceGuard g(w->device);
    vfd_status s = sync_sources(w, (cudaStream_t)stream);
    if (s != VFD_OK) return s;
    const UpdateArgs upd{dchem, decay};
    return enqueue_tick(w, -1, n_substeps, (cudaStream_t)stream, &upd);
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
        if (w->method == VFD_METHOD_PLAIN) {
            // MS_LEAK_X holds the full-grid sum of the inverse transform
            out[f].leaked[0] = m[MS_LEAK_X] - m[MS_CONV];
            out[f].leaked[1] = out[f].leaked[2] = 0.0;
        } else if (w->method == VFD_METHOD_FFT3D) {
            // pruned transform: the y/z spill is not materialised; report the
            // total beyond the crop implied by the kernel sum K0
            out[f].leaked[0] = m[MS_INPUT] * w->k0[f] - m[MS_CONV];
            out[f].leaked[1] = out[f].leaked[2] = 0.0;
        }
        out[f].conv_sum = m[MS_CONV];
        out[f].sources = m[MS_SOURCES];
        out[f].total = m[MS_OUT] + m[MS_SOURCES];
        out[f].reserved = 0.0;
    }
    if (herr) return fail(w, VFD_ERR_DEVICE_FAULT, "a kernel rejected an out-of-range index");
    if (rf_take_timeout()) return fail(w, VFD_ERR_TIMEOUT, "an axis pass gave up waiting for a bulk copy");
    return VFD_OK;
}

vfd_status vfd_update_gradients(vfd_world *w, const float *collagen, const float *elastin, float *fib, float *neu,
                                float *mac, void *stream)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (w->nf < 7) return fail(w, VFD_ERR_INVALID_ARG, "gradients need the TNF..IL8 fields (n_fields >= 7)");
    DeviceGuard g(w->device);
    const float *chem[8];
    for (int f = 0; f < 7; ++f) chem[f] = w->d_fields + (int64_t)f * w->V;
    VFD_CUDA(w, launch_gradients(chem, collagen, elastin, fib, neu, mac, w->V, (cudaStream_t)stream));
    return VFD_OK;
}

vfd_status vfd_sample_field(vfd_world *w, int field, int stride, float scale, float *out, void *stream)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (field < 0 || field >= w->nf || stride < 1 || !out)
        return fail(w, VFD_ERR_INVALID_ARG, "bad field, stride or output pointer");
    DeviceGuard g(w->device);
    VFD_CUDA(w, launch_sample(w->d_fields + (int64_t)field * w->V, w->nx, w->ny, w->nz, stride, scale, out,
                              (cudaStream_t)stream));
    return VFD_OK;
}

// ---- autotuning -------------------------------------------------------------
// The `k` cheapest FFT lengths (plan_cost order) for a line of n with radius r.
static int fft_len_candidates(int n, int r, int k, int *out)
{
    std::vector<std::pair<double, int>> c;
    const int lo = n + r;
    for (int F = lo; F <= 2 * lo + 16; ++F) {
        FftPlan p;
        if (!make_plan(F, &p) || !any_variant_fits(p)) continue;
        c.push_back({plan_cost(p), F});
    }
    std::stable_sort(c.begin(), c.end(), [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
        return x.first < y.first;
    });
    const int m = std::min(k, (int)c.size());
    for (int i = 0; i < m; ++i) out[i] = c[i].second;
    return m;
}

static bool same_radices(const FftPlan &p, const FftPlan &q)
{
    if (p.nst != q.nst) return false;
    for (int s = 0; s < p.nst; ++s)
        if (p.radix[s] != q.radix[s]) return false;
    return true;
}

// Mean time of one pass of axis a over every field (ms), or < 0 on error.
static float time_axis(vfd_world *w, int a, int reps, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1)
{
    if (enqueue_axis(w, a, -1, st) != VFD_OK) return -1.0f;
    if (cudaEventRecord(e0, st) != cudaSuccess) return -1.0f;
    for (int i = 0; i < reps; ++i)
        if (enqueue_axis(w, a, -1, st) != VFD_OK) return -1.0f;
    if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) return -1.0f;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return -1.0f;
    return ms / reps;
}

// Times the candidates of each axis on worlds built from `proto` and keeps
// the fastest in best (candidates whose world does not run the asked pass
// on an axis are not timed there).
struct TuneRun {
    const vfd_world_desc *d;
    int device, reps;
    cudaStream_t st;
    cudaEvent_t e0, e1;
    ShapeChoice best;
    bool have[3] = {false, false, false};
};

static vfd_status tune_candidate(TuneRun &T, const ShapeChoice &proto, const bool *axes)
{
    vfd_world *w = nullptr;
    vfd_status s = world_create(T.d, T.device, &proto, &w);
    if (s == VFD_ERR_NOT_SUPPORTED || s == VFD_ERR_OUT_OF_MEMORY) return VFD_OK;  // candidate does not fit
    if (s != VFD_OK) return s;
    for (int a = 0; a < 3 && s == VFD_OK; ++a) {
        if (!axes[a]) continue;
        const AxisChoice &c = proto.ax[a];
        int method = w->use_rf[a] ? PASS_METHOD_RF : w->use_os[a] ? PASS_METHOD_OS : PASS_METHOD_FULL;
        if (c.method != PASS_METHOD_AUTO && method != c.method) continue;
        if (method == PASS_METHOD_FULL && c.variant >= 0 && w->variant[a] != c.variant) continue;
        const float ms = time_axis(w, a, T.reps, T.st, T.e0, T.e1);
        if (ms < 0.0f) {
            s = VFD_ERR_CUDA;
            break;
        }
        if (!T.have[a] || ms < T.best.ax[a].ms) {
            AxisChoice b;
            b.method = method;
            b.minb = method == PASS_METHOD_OS ? (c.minb > 0 ? c.minb : os_default_ctas_per_sm()) : 0;
            b.F = method == PASS_METHOD_FULL ? w->F[a] : 0;
            b.order = method == PASS_METHOD_FULL ? w->plan_order[a] : 0;
            b.variant = method == PASS_METHOD_FULL ? w->variant[a] : -1;
            b.ms = ms;
            T.best.ax[a] = b;
            T.have[a] = true;
        }
    }
    vfd_world_destroy(w);
    return s;
}

static vfd_status tune_shape(const vfd_world_desc *d, int device, int reps, ShapeChoice *out)
{
    if (!d || !d->fields || d->n_fields < 1 || d->nx < 1 || d->ny < 1 || d->nz < 1)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "invalid world description");
    if (d->method != VFD_METHOD_SEPARABLE)
        return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "autotuning covers VFD_METHOD_SEPARABLE worlds");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, VFD_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev) return fail(nullptr, VFD_ERR_INVALID_ARG, "device ordinal out of range");
    DeviceGuard g(device);
    TuneRun T;
    T.d = d;
    T.device = device;
    T.reps = std::max(1, std::min(reps, 100));
    if (cudaStreamCreateWithFlags(&T.st, cudaStreamNonBlocking) != cudaSuccess)
        return fail(nullptr, VFD_ERR_CUDA, "autotune: stream");
    cudaEventCreate(&T.e0);
    cudaEventCreate(&T.e1);
    const bool all[3] = {true, true, true};
    const int dims[3] = {d->nx, d->ny, d->nz};
    int rmax[3] = {0, 0, 0};
    for (int f = 0; f < d->n_fields; ++f)
        for (int a = 0; a < 3; ++a) {
            int r = d->fields[f].radius[a];
            if (r <= 0) r = (int)std::ceil(3.0 * d->fields[f].sigma[a]);
            rmax[a] = std::max(rmax[a], r);
        }
    vfd_status s = VFD_OK;
    // register FFT (where the world would take it)
    {
        ShapeChoice c;
        for (int a = 0; a < 3; ++a) c.ax[a].method = PASS_METHOD_RF;
        s = tune_candidate(T, c, all);
    }
    // overlap-save at 3 and 4 resident CTAs per SM
    for (int minb = 3; minb <= 4 && s == VFD_OK; ++minb) {
        ShapeChoice c;
        for (int a = 0; a < 3; ++a) {
            c.ax[a].method = PASS_METHOD_OS;
            c.ax[a].minb = minb;
        }
        s = tune_candidate(T, c, all);
    }
    // full line: FFT length x radix order x kernel variant; the FFT length of
    // an axis that has fewer candidates stays at its cheapest
    int cand[3][3], ncand[3];
    for (int a = 0; a < 3; ++a) ncand[a] = d->fft[a] > 0 ? 0 : fft_len_candidates(dims[a], rmax[a], 3, cand[a]);
    for (int k = 0; k < 3 && s == VFD_OK; ++k)
        for (int order = 0; order < kPlanOrders && s == VFD_OK; ++order)
            for (int v = 0; v < kNumAxisVariants && s == VFD_OK; ++v) {
                ShapeChoice c;
                bool axes[3] = {false, false, false}, any = false;
                for (int a = 0; a < 3; ++a) {
                    c.ax[a].method = PASS_METHOD_FULL;
                    c.ax[a].order = order;
                    c.ax[a].variant = v;
                    const int F = d->fft[a] > 0 ? d->fft[a] : (ncand[a] > 0 ? cand[a][std::min(k, ncand[a] - 1)] : 0);
                    c.ax[a].F = d->fft[a] > 0 ? 0 : F;
                    if (F <= 0 || (k > 0 && k >= ncand[a])) continue;
                    FftPlan p, p0;
                    if (!make_plan_order(F, order, &p) || !variant_fits(v, p)) continue;
                    if (order > 0 && make_plan_order(F, 0, &p0) && same_radices(p, p0)) continue;
                    axes[a] = any = true;
                }
                if (any) s = tune_candidate(T, c, axes);
            }
    cudaEventDestroy(T.e0);
    cudaEventDestroy(T.e1);
    cudaStreamDestroy(T.st);
    if (s != VFD_OK) return s;
    for (int a = 0; a < 3; ++a)
        if (!T.have[a]) return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "autotune: no pass runs this shape");
    *out = T.best;
    return VFD_OK;
}

static void to_public(const AxisChoice &c, vfd_axis_tuning *o)
{
    o->method = c.method == PASS_METHOD_RF   ? VFD_PASS_REGISTER_FFT
                : c.method == PASS_METHOD_OS ? VFD_PASS_OVERLAP_SAVE
                                             : VFD_PASS_FULL_LINE;
    o->ctas_per_sm = c.minb;
    o->fft_len = c.F;
    o->radix_order = c.order;
    o->variant = c.variant;
    o->ms = c.ms;
}

vfd_status vfd_autotune(const vfd_world_desc *desc, int device, int reps, vfd_axis_tuning *out3)
{
    if (!out3) return fail(nullptr, VFD_ERR_INVALID_ARG, "out3 is NULL");
    ShapeChoice ch;
    vfd_status s = tune_shape(desc, device, reps, &ch);
    if (s != VFD_OK) return s;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[shape_key(desc, device)] = ch;
    }
    for (int a = 0; a < 3; ++a) to_public(ch.ax[a], &out3[a]);
    return VFD_OK;
}

vfd_status vfd_world_tuning(const vfd_world *w, vfd_axis_tuning *out3)
{
    if (!w || !out3) return VFD_ERR_INVALID_ARG;
    if (w->method != VFD_METHOD_SEPARABLE) return VFD_ERR_NOT_SUPPORTED;
    for (int a = 0; a < 3; ++a) {
        AxisChoice c;
        c.method = w->use_rf[a] ? PASS_METHOD_RF : w->use_os[a] ? PASS_METHOD_OS : PASS_METHOD_FULL;
        c.minb = c.method == PASS_METHOD_OS ? (w->os_minb[a] > 0 ? w->os_minb[a] : os_default_ctas_per_sm()) : 0;
        c.F = c.method == PASS_METHOD_FULL ? w->F[a] : 0;
        c.order = c.method == PASS_METHOD_FULL ? w->plan_order[a] : 0;
        c.variant = c.method == PASS_METHOD_FULL ? w->variant[a] : -1;
        c.ms = w->tuned_ms[a];
        to_public(c, &out3[a]);
    }
    return VFD_OK;
}

vfd_status vfd_autotune_set(const vfd_world_desc *desc, int device, const vfd_axis_tuning *in3)
{
    if (!desc || !desc->fields || !in3 || desc->n_fields < 1)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "desc, desc->fields or in3 is NULL");
    if (desc->method != VFD_METHOD_SEPARABLE)
        return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "tunings cover VFD_METHOD_SEPARABLE worlds");
    const int dims[3] = {desc->nx, desc->ny, desc->nz};
    ShapeChoice ch;
    for (int a = 0; a < 3; ++a) {
        const vfd_axis_tuning &t = in3[a];
        AxisChoice &c = ch.ax[a];
        if (t.method < VFD_PASS_REGISTER_FFT || t.method > VFD_PASS_FULL_LINE)
            return fail(nullptr, VFD_ERR_INVALID_ARG, "unknown pass method");
        c.method = t.method == VFD_PASS_REGISTER_FFT ? PASS_METHOD_RF
                   : t.method == VFD_PASS_OVERLAP_SAVE ? PASS_METHOD_OS
                                                        : PASS_METHOD_FULL;
        c.ms = t.ms;
        if (c.method == PASS_METHOD_OS) {
            if (t.ctas_per_sm != 0 && t.ctas_per_sm != 3 && t.ctas_per_sm != 4)
                return fail(nullptr, VFD_ERR_INVALID_ARG, "ctas_per_sm must be 0, 3 or 4");
            c.minb = t.ctas_per_sm;
        }
        if (c.method == PASS_METHOD_FULL) {
            if (t.radix_order < 0 || t.radix_order >= kPlanOrders)
                return fail(nullptr, VFD_ERR_INVALID_ARG, "radix_order out of range");
            if (t.variant < -1 || t.variant >= kNumAxisVariants)
                return fail(nullptr, VFD_ERR_INVALID_ARG, "variant out of range");
            int rmax = 0;
            for (int f = 0; f < desc->n_fields; ++f) {
                int r = desc->fields[f].radius[a];
                if (r <= 0) r = (int)std::ceil(3.0 * desc->fields[f].sigma[a]);
                rmax = std::max(rmax, r);
            }
            FftPlan p;
            if (t.fft_len != 0 && (t.fft_len < dims[a] + rmax || !make_plan_order(t.fft_len, t.radix_order, &p) ||
                                   !any_variant_fits(p)))
                return fail(nullptr, VFD_ERR_INVALID_ARG, "fft_len is shorter than n + radius or has no plan");
            if (t.fft_len != 0 && t.variant >= 0 && !variant_fits(t.variant, p))
                return fail(nullptr, VFD_ERR_INVALID_ARG, "the kernel variant does not fit fft_len");
            c.F = t.fft_len;
            c.order = t.radix_order;
            c.variant = t.variant;
        }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[shape_key(desc, device)] = ch;
    return VFD_OK;
}

vfd_status vfd_autotune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache.clear();
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
    vfd_status s = VFD_OK;
    const size_t bytes = sizeof(float) * w->V;
    for (int f = 0; f < w->nf; ++f) {
        float *dev = w->d_fields + (int64_t)f * w->V;
        VFD_CUDA(w, cudaMemcpyAsync(dev, host_in[f], bytes, cudaMemcpyHostToDevice, w->s_in));
        VFD_CUDA(w, cudaEventRecord(w->ev_in[f], w->s_in));
        // the sources go up on the compute stream (ahead of every tick)
        // while the first field is in flight: their pageable copies hold the
        // host until staged
        if (f == 0 && (s = sync_sources(w, w->s_cmp)) != VFD_OK) return s;
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

vfd_status vfd_diffuse_update_host(vfd_world *w, float *const *host_p, float *const *host_d, const float *decay,
                                   int n_substeps)
{
    if (!w) return VFD_ERR_INVALID_ARG;
    if (!host_p || !decay || n_substeps < 1)
        return fail(w, VFD_ERR_INVALID_ARG, "NULL buffers, NULL decay or n_substeps < 1");
    for (int f = 0; f < w->nf; ++f) {
        if (!host_p[f]) return fail(w, VFD_ERR_INVALID_ARG, "NULL host buffer");
        if (!std::isfinite(decay[f])) return fail(w, VFD_ERR_INVALID_ARG, "decay must be finite");
    }
    DeviceGuard g(w->device);
    vfd_status s = VFD_OK;
    const size_t bytes = sizeof(float) * w->V;
    if (host_d && !w->d_upd) VFD_CUDA(w, cudaMalloc(&w->d_upd, bytes * w->nf));
    std::vector<float *> dptr(w->nf, nullptr);
    for (int f = 0; f < w->nf; ++f)
        if (host_d && host_d[f]) dptr[f] = w->d_upd + (int64_t)f * w->V;
    for (int f = 0; f < w->nf; ++f) {
        float *dev = w->d_fields + (int64_t)f * w->V;
        VFD_CUDA(w, cudaMemcpyAsync(dev, host_p[f], bytes, cudaMemcpyHostToDevice, w->s_in));
        if (dptr[f]) VFD_CUDA(w, cudaMemcpyAsync(dptr[f], host_d[f], bytes, cudaMemcpyHostToDevice, w->s_in));
        VFD_CUDA(w, cudaEventRecord(w->ev_in[f], w->s_in));
        // sources ahead of every tick, staged while the first field is in flight
        if (f == 0 && (s = sync_sources(w, w->s_cmp)) != VFD_OK) return s;
        VFD_CUDA(w, cudaStreamWaitEvent(w->s_cmp, w->ev_in[f], 0));
        // the update reads decay[f] and dchem[f] only for field f
        const UpdateArgs upd{dptr.data(), decay};
        s = enqueue_tick(w, f, n_substeps, w->s_cmp, &upd);
        if (s != VFD_OK) return s;
        VFD_CUDA(w, cudaEventRecord(w->ev_cmp[f], w->s_cmp));
        VFD_CUDA(w, cudaStreamWaitEvent(w->s_out, w->ev_cmp[f], 0));
        VFD_CUDA(w, cudaMemcpyAsync(host_p[f], dev, bytes, cudaMemcpyDeviceToHost, w->s_out));
    }
    // dChem = 0 on the host (WHChemical.cpp:427) once its copy has landed on the device
    VFD_CUDA(w, cudaStreamSynchronize(w->s_in));
    for (int f = 0; f < w->nf; ++f)
        if (dptr[f]) std::memset(host_d[f], 0, bytes);
    VFD_CUDA(w, cudaStreamSynchronize(w->s_out));
    VFD_CUDA(w, cudaStreamSynchronize(w->s_cmp));
    int herr = 0;
    VFD_CUDA(w, cudaMemcpy(&herr, w->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(w, VFD_ERR_DEVICE_FAULT, "a kernel rejected an out-of-range index");
    return VFD_OK;
}

// ---------------------------------------------------------------------------
// Batched ensembles: every field of every world goes through one launch per
// axis pass per substep; the whole tick is captured once into a CUDA graph
// and replayed (re-captured when the substep count or any world's source
// lists change).
// ---------------------------------------------------------------------------
}  // extern "C"

struct vfd_batch {
    int device = 0;
    std::vector<vfd_world *> worlds;
    int variant[3] = {0, 0, 0};
    int tiles[3] = {0, 0, 0};
    int Fmax[3] = {0, 0, 0};
    int njobs = 0;
    AxisJob *d_jobs = nullptr;  // [3][njobs]
    bool use_os[3] = {false, false, false};
    int rmin[3] = {0, 0, 0};
    OsJob *d_osjobs = nullptr;  // [3][njobs]
    int os_tiles[3] = {0, 0, 0};
    OsTileInfo *d_os_tiles[3] = {nullptr, nullptr, nullptr};
    int os_minb[3] = {0, 0, 0};
    bool use_rf[3] = {false, false, false};
    std::vector<RfGroup> rf[3];
    cudaStream_t st = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_substeps = -1;
    uint64_t graph_launches = 0;
    int same_ticks = 0;  // ticks in a row with the current substep count and sources
    std::vector<uint64_t> gens;
    double **d_mass_ptrs = nullptr;  // every world's accounting block, zeroed per substep in one launch
    int *d_mass_counts = nullptr;
    unsigned char *d_arena = nullptr;  // the arrays set up at creation, in one allocation
    bool os_tiles_owned[3] = {true, true, true};
    std::vector<OsJob> oj;       // host copy of the overlap-save jobs ([axis][njobs])
    bool can_os[3] = {false, false, false};
    float tuned_ms[3] = {0.0f, 0.0f, 0.0f};
    std::string err;
};

static vfd_status bfail(vfd_batch *b, vfd_status s, const std::string &msg)
{
    if (b) b->err = msg;
    else g_thread_error = msg;
    return s;
}

#define VFD_BCUDA(b, call)                                                                  \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? VFD_ERR_OUT_OF_MEMORY        \
                                                               : VFD_ERR_CUDA,                \
                         std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// Arenas and streams of destroyed batches, kept per device for the next
// batch (a server creates a batch at every change of its active set):
// destroying a batch frees nothing on the device, creating one allocates
// only when no kept arena is large enough.
struct BatchCache {
    std::mutex mu;
    unsigned long long ctx[64] = {};                    // context the kept items belong to
    std::multimap<size_t, unsigned char *> arenas[64];  // by capacity
    std::vector<std::array<void *, 3>> streams[64];     // stream, ev_in, ev_out
};
static BatchCache g_bcache;
// capacity and context of every arena handed out (under g_bcache.mu)
static std::map<unsigned char *, std::pair<size_t, unsigned long long>> g_arena_cap;

// Forgets what was kept for `dev` if it belongs to another context than the
// current one (after a device reset; the memory went with that context).
static void bcache_check_context(int dev)
{
    const unsigned long long c = current_context_id();
    if (c == 0 || g_bcache.ctx[dev] == c) return;
    for (auto &kv : g_bcache.arenas[dev]) g_arena_cap.erase(kv.second);
    g_bcache.arenas[dev].clear();
    g_bcache.streams[dev].clear();
    g_bcache.ctx[dev] = c;
}

static cudaError_t take_arena(int dev, size_t bytes, unsigned char **out)
{
    {
        std::lock_guard<std::mutex> lk(g_bcache.mu);
        if (dev >= 0 && dev < 64) {
            bcache_check_context(dev);
            auto &m = g_bcache.arenas[dev];
            auto it = m.lower_bound(bytes);
            if (it != m.end() && it->first <= 4 * bytes + (1 << 20)) {
                *out = it->second;
                m.erase(it);
                return cudaSuccess;
            }
        }
    }
    const size_t cap = bytes + bytes / 4 + 4096;
    cudaError_t e = cudaMalloc(out, cap);
    if (e == cudaSuccess) {
        const unsigned long long c = current_context_id();
        std::lock_guard<std::mutex> lk(g_bcache.mu);
        g_arena_cap[*out] = {cap, c};
    }
    return e;
}

static void give_arena(int dev, unsigned char *p)
{
    if (!p) return;
    const unsigned long long c = current_context_id();
    std::lock_guard<std::mutex> lk(g_bcache.mu);
    auto it = g_arena_cap.find(p);
    const bool keep = dev >= 0 && dev < 64 && it != g_arena_cap.end() && it->second.second == c && c != 0 &&
                      g_bcache.ctx[dev] == c && g_bcache.arenas[dev].size() < 64;
    if (!keep) {
        if (it != g_arena_cap.end()) g_arena_cap.erase(it);
        cudaFree(p);
        return;
    }
    g_bcache.arenas[dev].insert({it->second.first, p});
}

static void batch_release(vfd_batch *b)
{
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (int a = 0; a < 3; ++a) {
        if (b->os_tiles_owned[a]) cudaFree(b->d_os_tiles[a]);
        free_rf_groups(b->rf[a]);
    }
    // d_jobs, d_osjobs, the mass arrays and the arena-placed tiles: the
    // arena is kept for the next batch on this device (the batch's work is
    // complete when it is destroyed)
    if (b->d_arena) cudaStreamSynchronize(b->st);
    give_arena(b->device, b->d_arena);
    bool kept = false;
    if (b->st && b->ev_in && b->ev_out && b->device >= 0 && b->device < 64) {
        const unsigned long long c = current_context_id();
        std::lock_guard<std::mutex> lk(g_bcache.mu);
        if (c != 0 && g_bcache.ctx[b->device] == c && g_bcache.streams[b->device].size() < 64) {
            g_bcache.streams[b->device].push_back({(void *)b->st, (void *)b->ev_in, (void *)b->ev_out});
            kept = true;
        }
    }
    if (!kept) {
        if (b->ev_in) cudaEventDestroy(b->ev_in);
        if (b->ev_out) cudaEventDestroy(b->ev_out);
        if (b->st) cudaStreamDestroy(b->st);
    }
    cudaSetDevice(prev);
}

extern "C" {

// Whether every job of axis a (oj: [axis][njobs]) can take the register-FFT
// pass and every world allows it there.
static bool batch_rf_possible(const vfd_batch *b, const std::vector<OsJob> &oj, int a)
{
    if (!rf_enabled() || !b->use_os[a]) return false;
    for (auto *w : b->worlds)
        if (!w->allow_rf[a]) return false;
    for (int i = 0; i < b->njobs; ++i)
        if (!rf_eligible(oj[(size_t)a * b->njobs + i])) return false;
    return true;
}



// The batch's stream and events: kept ones of this device, or new.
static cudaError_t take_stream(vfd_batch *b)
{
    if (b->device >= 0 && b->device < 64) {
        std::lock_guard<std::mutex> lk(g_bcache.mu);
        bcache_check_context(b->device);
        auto &v = g_bcache.streams[b->device];
        if (!v.empty()) {
            b->st = (cudaStream_t)v.back()[0];
            b->ev_in = (cudaEvent_t)v.back()[1];
            b->ev_out = (cudaEvent_t)v.back()[2];
            v.pop_back();
            return cudaSuccess;
        }
    }
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

vfd_status vfd_batch_create(vfd_world *const *worlds, int n_worlds, vfd_batch **out)
{
    if (!out) return bfail(nullptr, VFD_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!worlds || n_worlds < 1) return bfail(nullptr, VFD_ERR_INVALID_ARG, "no worlds");
    for (int i = 0; i < n_worlds; ++i) {
        if (!worlds[i]) return bfail(nullptr, VFD_ERR_INVALID_ARG, "NULL world");
        if (worlds[i]->device != worlds[0]->device)
            return bfail(nullptr, VFD_ERR_INVALID_ARG, "worlds of a batch must share one device");
        if (worlds[i]->method != VFD_METHOD_SEPARABLE)
            return bfail(nullptr, VFD_ERR_NOT_SUPPORTED, "batches take VFD_METHOD_SEPARABLE worlds");
    }
    vfd_batch *b = new vfd_batch();
    b->device = worlds[0]->device;
    b->worlds.assign(worlds, worlds + n_worlds);
    for (int a = 0; a < 3; ++a) {
        std::vector<FftPlan> plans;
        for (auto *w : b->worlds) {
            plans.push_back(w->plan[a]);
            b->Fmax[a] = std::max(b->Fmax[a], w->F[a]);
        }
        b->variant[a] = pick_variant(plans);
        if (b->variant[a] < 0) {
            delete b;
            return bfail(nullptr, VFD_ERR_NOT_SUPPORTED, "no kernel variant fits every world's FFT plan");
        }
    }
    std::vector<AxisJob> jobs;
    for (int a = 0; a < 3; ++a) {
        const int nl = kAxisVariants[b->variant[a]].nl;
        int tb = 0;
        for (auto *w : b->worlds)
            for (int f = 0; f < w->nf; ++f) {
                jobs.push_back(make_job(w, f, a, tb, nl));
                tb += field_tiles(w, a, nl);
            }
        b->tiles[a] = tb;
    }
    b->njobs = (int)jobs.size() / 3;
    std::vector<OsJob> oj;
    std::vector<OsTileInfo> tile_info[3];
    for (int a = 0; a < 3; ++a) {
        bool all = true;
        int rmn = 1 << 30;
        for (auto *w : b->worlds) {
            all = all && w->use_os[a];
            for (int f = 0; f < w->nf; ++f) rmn = std::min(rmn, w->params[f].radius[a]);
        }
        b->use_os[a] = all;
        b->can_os[a] = all;
        b->rmin[a] = rmn;
        b->os_minb[a] = b->worlds[0]->os_minb[a];
        for (auto *w : b->worlds)
            if (w->os_minb[a] != b->os_minb[a]) b->os_minb[a] = 0;
    }
    if (b->use_os[0] || b->use_os[1] || b->use_os[2]) {
        for (int a = 0; a < 3; ++a) {
            int tb = 0;
            for (auto *w : b->worlds)
                for (int f = 0; f < w->nf; ++f) {
                    if (w->oj_host.size() == (size_t)3 * w->nf) {
                        oj.push_back(w->oj_host[(size_t)a * w->nf + f]);  // the world's own job, re-based
                        oj.back().tile_begin = tb;
                    } else {
                        oj.push_back(make_os_job(w, f, a, tb));
                    }
                    tb += os_field_tiles(oj.back());
                }
            b->os_tiles[a] = tb;
        }
    }
    // Per axis: the register-FFT pass when every job and world allows it,
    // else the overlap-save pass (its tile list built only then: a server
    // rebuilds its batch whenever the active set changes; autotuning builds
    // the others when it times that pass), else the full-line pass.
    RfGroupHost rfh[3];
    for (int a = 0; a < 3 && !oj.empty(); ++a) {
        if (batch_rf_possible(b, oj, a)) {
            rf_group_host(&oj[(size_t)a * b->njobs], b->njobs, rfh[a]);
            if (!rfh[a].tiles.empty()) continue;
        }
        if (b->use_os[a])
            for (int i = 0; i < b->njobs; ++i) os_append_tiles(oj[(size_t)a * b->njobs + i], i, tile_info[a]);
    }
    std::vector<double *> mp;
    std::vector<int> mc;
    for (auto *w : b->worlds) {
        mp.push_back(w->d_mass);
        mc.push_back(MS_COUNT * w->nf);
    }
    ArenaBuilder ar;
    const size_t o_jobs = ar.add(jobs.data(), sizeof(AxisJob) * jobs.size());
    const size_t o_oj = ar.add(oj.data(), sizeof(OsJob) * oj.size());
    size_t o_ost[3], o_rft[3], o_rfm[3];
    for (int a = 0; a < 3; ++a) {
        o_ost[a] = ar.add(tile_info[a].data(), sizeof(OsTileInfo) * tile_info[a].size());
        o_rft[a] = ar.add(rfh[a].tiles.data(), sizeof(OsTileInfo) * rfh[a].tiles.size());
        o_rfm[a] = ar.add(rfh[a].maps.data(), sizeof(CUtensorMap) * rfh[a].maps.size());
    }
    const size_t o_mp = ar.add(mp.data(), sizeof(double *) * mp.size());
    const size_t o_mc = ar.add(mc.data(), sizeof(int) * mc.size());
    DeviceGuard g(b->device);
    cudaError_t e = cudaSuccess;
    if ((!oj.empty() && (e = os_prepare()) != cudaSuccess) ||
        ((rfh[0].tiles.size() + rfh[1].tiles.size() + rfh[2].tiles.size()) > 0 && (e = rf_prepare()) != cudaSuccess) ||
        (e = take_arena(b->device, ar.host.size(), &b->d_arena)) != cudaSuccess ||
        (e = cudaMemcpy(b->d_arena, ar.host.data(), ar.host.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = take_stream(b)) != cudaSuccess) {
        std::string msg = std::string("batch setup: ") + cudaGetErrorString(e);
        batch_release(b);
        delete b;
        return bfail(nullptr, e == cudaErrorMemoryAllocation ? VFD_ERR_OUT_OF_MEMORY : VFD_ERR_CUDA, msg);
    }
    unsigned char *base = b->d_arena;
    b->d_jobs = reinterpret_cast<AxisJob *>(base + o_jobs);
    b->d_osjobs = oj.empty() ? nullptr : reinterpret_cast<OsJob *>(base + o_oj);
    for (int a = 0; a < 3; ++a) {
        if (!tile_info[a].empty()) {
            b->d_os_tiles[a] = reinterpret_cast<OsTileInfo *>(base + o_ost[a]);
            b->os_tiles_owned[a] = false;
        }
        if (!rfh[a].tiles.empty()) {
            RfGroup rg;
            rg.ntiles = (int)rfh[a].tiles.size();
            rg.d_tiles = reinterpret_cast<OsTileInfo *>(base + o_rft[a]);
            rg.d_maps = rfh[a].maps.empty() ? nullptr : reinterpret_cast<CUtensorMap *>(base + o_rfm[a]);
            rg.owned = false;
            b->rf[a].push_back(rg);
            b->use_rf[a] = true;
        }
    }
    b->d_mass_ptrs = reinterpret_cast<double **>(base + o_mp);
    b->d_mass_counts = reinterpret_cast<int *>(base + o_mc);
    b->gens.assign(n_worlds, ~0ull);
    b->oj.swap(oj);
    *out = b;
    return VFD_OK;
}

// Times one axis pass of the whole batch as configured now (one warm-up,
// `reps` timed launches, CUDA events on the batch stream).
static vfd_status batch_time_axis(vfd_batch *b, int a, int reps, cudaEvent_t e0, cudaEvent_t e1, float *ms)
{
    for (int it = -1; it < reps; ++it) {
        if (it == 0) VFD_BCUDA(b, cudaEventRecord(e0, b->st));
        if (b->use_rf[a])
            VFD_BCUDA(b, launch_rf_groups(b->d_osjobs + a * b->njobs, b->rf[a], a, b->st));
        else if (b->use_os[a])
            VFD_BCUDA(b, launch_os(b->d_osjobs + a * b->njobs, b->d_os_tiles[a], b->os_tiles[a], b->rmin[a], a, b->st,
                                   b->os_minb[a]));
        else
            VFD_BCUDA(b, launch_axis(b->variant[a], b->d_jobs + a * b->njobs, b->njobs, b->tiles[a], b->Fmax[a],
                                     b->st));
    }
    VFD_BCUDA(b, cudaEventRecord(e1, b->st));
    VFD_BCUDA(b, cudaEventSynchronize(e1));
    VFD_BCUDA(b, cudaEventElapsedTime(ms, e0, e1));
    *ms /= (float)reps;
    return VFD_OK;
}

vfd_status vfd_batch_autotune(vfd_batch *b, int reps, vfd_axis_tuning *out3)
{
    if (!b) return VFD_ERR_INVALID_ARG;
    if (reps < 1) reps = 3;
    DeviceGuard g(b->device);
    VFD_BCUDA(b, cudaStreamSynchronize(b->st));
    // the passes run on the worlds' own fields: save them, restore after
    std::vector<float *> saved(b->worlds.size(), nullptr);
    auto restore = [&](bool copy) {
        for (size_t i = 0; i < b->worlds.size(); ++i) {
            vfd_world *w = b->worlds[i];
            if (copy && saved[i])
                cudaMemcpyAsync(w->d_fields, saved[i], sizeof(float) * w->V * w->nf, cudaMemcpyDeviceToDevice, b->st);
        }
        cudaStreamSynchronize(b->st);
        for (auto p : saved) cudaFree(p);
    };
    for (size_t i = 0; i < b->worlds.size(); ++i) {
        vfd_world *w = b->worlds[i];
        cudaError_t e = cudaMalloc(&saved[i], sizeof(float) * w->V * w->nf);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(saved[i], w->d_fields, sizeof(float) * w->V * w->nf, cudaMemcpyDeviceToDevice, b->st);
        if (e != cudaSuccess) {
            restore(false);
            return bfail(b, e == cudaErrorMemoryAllocation ? VFD_ERR_OUT_OF_MEMORY : VFD_ERR_CUDA,
                         std::string("autotune backup: ") + cudaGetErrorString(e));
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    vfd_status st = VFD_OK;
    for (int a = 0; a < 3 && st == VFD_OK; ++a) {
        // register-FFT groups for this axis if every job allows them
        bool rf_ok = !b->rf[a].empty();
        if (!rf_ok && b->can_os[a] && rf_enabled() && !b->oj.empty()) {
            bool ok = true;
            for (int i = 0; i < b->njobs; ++i) ok = ok && rf_eligible(b->oj[(size_t)a * b->njobs + i]);
            if (ok && rf_prepare() == cudaSuccess &&
                build_rf_groups(&b->oj[(size_t)a * b->njobs], b->njobs, b->rf[a]) == cudaSuccess)
                rf_ok = !b->rf[a].empty();
        }
        struct Cand {
            int method, minb;
        };
        if (b->can_os[a] && !b->d_os_tiles[a] && !b->oj.empty()) {
            std::vector<OsTileInfo> ti;
            for (int i = 0; i < b->njobs; ++i) os_append_tiles(b->oj[(size_t)a * b->njobs + i], i, ti);
            if (upload_vec(&b->d_os_tiles[a], ti) != cudaSuccess) b->d_os_tiles[a] = nullptr;
            b->os_tiles_owned[a] = true;
        }
        std::vector<Cand> cands;
        if (rf_ok) cands.push_back({PASS_METHOD_RF, 0});
        if (b->can_os[a] && b->d_os_tiles[a]) {
            cands.push_back({PASS_METHOD_OS, 3});
            cands.push_back({PASS_METHOD_OS, 4});
        }
        cands.push_back({PASS_METHOD_FULL, 0});
        float best = 0.0f;
        Cand bc = cands.back();
        for (const Cand &c : cands) {
            b->use_rf[a] = c.method == PASS_METHOD_RF;
            b->use_os[a] = c.method == PASS_METHOD_OS;
            b->os_minb[a] = c.minb;
            float ms = 0.0f;
            st = batch_time_axis(b, a, reps, e0, e1, &ms);
            if (st != VFD_OK) break;
            if (best == 0.0f || ms < best) {
                best = ms;
                bc = c;
            }
        }
        b->use_rf[a] = bc.method == PASS_METHOD_RF;
        b->use_os[a] = bc.method == PASS_METHOD_OS;
        b->os_minb[a] = bc.minb;
        b->tuned_ms[a] = best;
        if (out3) {
            out3[a].method = bc.method == PASS_METHOD_RF ? VFD_PASS_REGISTER_FFT
                             : bc.method == PASS_METHOD_OS ? VFD_PASS_OVERLAP_SAVE
                                                           : VFD_PASS_FULL_LINE;
            out3[a].ctas_per_sm = bc.minb;
            out3[a].fft_len = bc.method == PASS_METHOD_FULL ? b->Fmax[a] : 64;
            out3[a].radix_order = 0;
            out3[a].variant = bc.method == PASS_METHOD_FULL ? b->variant[a] : -1;
            out3[a].ms = best;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    restore(true);
    // the next tick runs directly and re-captures its graph with the chosen passes
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_substeps = -1;
    b->same_ticks = 0;
    return st;
}

vfd_status vfd_batch_destroy(vfd_batch *b)
{
    if (!b) return VFD_ERR_INVALID_ARG;
    batch_release(b);
    delete b;
    return VFD_OK;
}

static vfd_status batch_enqueue(vfd_batch *b, int n_substeps)
{
    for (int s = 0; s < n_substeps; ++s) {
        VFD_BCUDA(b, launch_zero_blocks(b->d_mass_ptrs, b->d_mass_counts, (int)b->worlds.size(), b->st));
        for (int a = 0; a < 3; ++a) {
            if (b->use_rf[a])
                VFD_BCUDA(b, launch_rf_groups(b->d_osjobs + a * b->njobs, b->rf[a], a, b->st));
            else if (b->use_os[a])
                VFD_BCUDA(b, launch_os(b->d_osjobs + a * b->njobs, b->d_os_tiles[a], b->os_tiles[a], b->rmin[a], a,
                                       b->st, b->os_minb[a]));
            else
                VFD_BCUDA(b, launch_axis(b->variant[a], b->d_jobs + a * b->njobs, b->njobs, b->tiles[a],
                                         b->Fmax[a], b->st));
        }
    }
    for (auto *w : b->worlds)
        if (w->dep_njobs > 0)
            VFD_BCUDA(b, launch_deposit(w->d_dep, w->dep_njobs, w->d_src_idx, w->d_src_amt, w->src_total,
                                        w->d_err, b->st));
    return VFD_OK;
}

vfd_status vfd_batch_tick(vfd_batch *b, int n_substeps, void *stream)
{
    if (!b) return VFD_ERR_INVALID_ARG;
    if (n_substeps < 1) return bfail(b, VFD_ERR_INVALID_ARG, "n_substeps must be >= 1");
    DeviceGuard g(b->device);
    // The tick is captured into a CUDA graph once the same configuration
    // (substep count, source lists) has run twice in a row; a batch that
    // lives for a single tick (a server round whose active set changes)
    // launches its kernels directly and pays no capture.
    bool stale = b->graph_substeps != n_substeps;
    for (size_t i = 0; i < b->worlds.size(); ++i) {
        vfd_status st = sync_sources(b->worlds[i], b->st);
        if (st != VFD_OK) return bfail(b, st, b->worlds[i]->err);
        if (b->gens[i] != b->worlds[i]->src_gen) stale = true;
    }
    if (stale) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->graph) cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
        b->graph_substeps = n_substeps;
        for (size_t i = 0; i < b->worlds.size(); ++i) b->gens[i] = b->worlds[i]->src_gen;
        b->same_ticks = 0;
    }
    ++b->same_ticks;
    VFD_BCUDA(b, cudaEventRecord(b->ev_in, (cudaStream_t)stream));
    VFD_BCUDA(b, cudaStreamWaitEvent(b->st, b->ev_in, 0));
    if (!b->exec && b->same_ticks < 2) {
        vfd_status st = batch_enqueue(b, n_substeps);
        if (st != VFD_OK) return st;
    } else {
        if (!b->exec) {
            const uint64_t before = g_launches.load();
            VFD_BCUDA(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
            vfd_status st = batch_enqueue(b, n_substeps);
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(b->st, &graph);
            if (st != VFD_OK) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (ce != cudaSuccess) return bfail(b, VFD_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
            b->graph = graph;
            b->graph_launches = g_launches.load() - before;
            g_launches.fetch_sub(b->graph_launches);  // captured, not executed
            VFD_BCUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
        }
        VFD_BCUDA(b, cudaGraphLaunch(b->exec, b->st));
        g_launches.fetch_add(b->graph_launches);
    }
    VFD_BCUDA(b, cudaEventRecord(b->ev_out, b->st));
    VFD_BCUDA(b, cudaStreamWaitEvent((cudaStream_t)stream, b->ev_out, 0));
    return VFD_OK;
}

const char *vfd_batch_last_error(const vfd_batch *b) { return b ? b->err.c_str() : g_thread_error.c_str(); }

// ---------------------------------------------------------------------------
// Reference-mode kernel construction (computeKernel3D, Diffusion.cu:1078-1531).
// The reference raises the 7-point stencil to the power n by repeated FFT
// convolution (niter rounds of complexPower on a 616^3 grid with a 299^3
// crop between rounds) and keeps the centred window.  Here the power is
// taken once in the frequency domain on a periodic G^3 grid, G >= 2R + 1 +
// 16 sigma (sigma^2 = 2 lambda n per axis), so the wrapped tails that reach
// the window are below FP32 resolution, then one inverse 3D FFT and the crop.
// (The reference's complexPower uses atanf(b/a), which drops the sign of
// bins with a negative real part; those bins have |S|^n < 1e-30 at the
// reference's lambda, so the two agree to FP32 resolution.)
// ---------------------------------------------------------------------------
vfd_status vfd_stencil_window(double lambda, double gamma_dt, int n_steps, int R, float *out, int device)
{
    if (!out || R < 0 || n_steps < 0 || !(lambda >= 0.0) || lambda > 1.0 / 6.0)
        return fail(nullptr, VFD_ERR_INVALID_ARG, "bad stencil parameters (0 <= lambda <= 1/6, R >= 0)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, VFD_ERR_NO_DEVICE, "no device");
    const double sigma = std::sqrt(2.0 * lambda * (double)n_steps);
    int G = -1;
    for (int g = 2 * R + 2 + 2 * (int)std::ceil(8.0 * sigma); g < 4096; ++g) {
        if (g & 1) continue;
        FftPlan p;
        if (make_plan(g, &p) && any_variant_fits(p) && pick_variant(std::vector<FftPlan>{p}, 16) >= 0) {
            G = g;
            break;
        }
    }
    if (G < 0) return fail(nullptr, VFD_ERR_NOT_SUPPORTED, "stencil window too wide for the device FFT");
    DeviceGuard dg(device);
    FftPlan plan;
    make_plan(G, &plan);
    const int vrow = pick_variant(std::vector<FftPlan>{plan});
    const int vcol = pick_variant(std::vector<FftPlan>{plan}, 16);
    const int Gh = G / 2 + 1;
    const int64_t nk = (int64_t)Gh * G * G, np = (int64_t)G * G * G, nw = (int64_t)(2 * R + 1) * (2 * R + 1) * (2 * R + 1);
    float2 *K = nullptr, *tw = nullptr;
    float *P = nullptr, *W = nullptr;
    std::vector<float2> htw;
    twiddles(G, htw);
    cudaError_t e = cudaSuccess;
    auto run = [&]() -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMalloc(&K, sizeof(float2) * nk)) != cudaSuccess) return r;
        if ((r = cudaMalloc(&P, sizeof(float) * np)) != cudaSuccess) return r;
        if ((r = cudaMalloc(&W, sizeof(float) * nw)) != cudaSuccess) return r;
        if ((r = cudaMalloc(&tw, sizeof(float2) * G)) != cudaSuccess) return r;
        if ((r = cudaMemcpy(tw, htw.data(), sizeof(float2) * G, cudaMemcpyHostToDevice)) != cudaSuccess) return r;
        if ((r = launch_stencil_spectrum(K, G, lambda, 1.0 - 6.0 * lambda - gamma_dt, n_steps, 0)) != cudaSuccess)
            return r;
        GenColPass c;
        memset(&c, 0, sizeof(c));
        c.plan = plan;
        c.tw = tw;
        c.data = K;
        c.nlines = Gh;
        c.scale = 1.0f;
        c.mode = GEN_INVERSE;
        c.nload = c.nstore = G;
        // z lines: outer = y
        c.nouter = G;
        c.outer_stride = Gh;
        c.pos_stride = (int64_t)G * Gh;
        if ((r = launch_gen_cols(vcol, c, 0)) != cudaSuccess) return r;
        // y lines: outer = z
        c.outer_stride = (int64_t)G * Gh;
        c.pos_stride = Gh;
        if ((r = launch_gen_cols(vcol, c, 0)) != cudaSuccess) return r;
        GenRowPass rp;
        memset(&rp, 0, sizeof(rp));
        rp.plan = plan;
        rp.tw = tw;
        rp.nrows = G * G;
        rp.rows_per_plane = G;
        rp.r_s1 = G;
        rp.r_s2 = (int64_t)G * G;
        rp.c_s1 = Gh;
        rp.c_s2 = (int64_t)Gh * G;
        rp.nstore = G;
        rp.rdst = P;
        rp.csrc = K;
        if ((r = launch_gen_rows(vrow, rp, true, 0)) != cudaSuccess) return r;
        if ((r = launch_crop_window(W, P, G, R, (float)(1.0 / (double)np), 0)) != cudaSuccess) return r;
        return cudaMemcpy(out, W, sizeof(float) * nw, cudaMemcpyDeviceToHost);
    };
    e = run();
    cudaFree(K);
    cudaFree(P);
    cudaFree(W);
    cudaFree(tw);
    if (e != cudaSuccess) return fail(nullptr, e == cudaErrorMemoryAllocation ? VFD_ERR_OUT_OF_MEMORY : VFD_ERR_CUDA,
                                      std::string("stencil window: ") + cudaGetErrorString(e));
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
    for (long long i = 0; i < (long long)n; ++i) {
        volatile double prod = span * u01(key, (uint64_t)i);  // rounded product, then the sum
        out[i] = (float)(a + prod);
    }
    return VFD_OK;
}

vfd_status vfd_synth_field_device(uint64_t seed, int world, int field, float lo, float hi, float *dptr, size_t n,
                                  void *stream)
{
    if (!dptr && n) return fail(nullptr, VFD_ERR_INVALID_ARG, "dptr is NULL");
    const uint64_t key = stream_key(seed, world, field, 0);
    cudaError_t e = launch_synth_field(key, (double)lo, (double)hi - (double)lo, dptr, (int64_t)n, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(nullptr, VFD_ERR_CUDA, std::string("synth: ") + cudaGetErrorString(e));
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
