/*
 * vfd.h -- C ABI of the B200 cytokine-diffusion library (libvfd.so).
 *
 * Replaces the diffusion layer of the vocal-fold ABM (src/Diffusion/ in the
 * reference): the per-tick FFT-convolution diffusion of the chemical fields
 * that WHWorld::diffuseCytokines() drives through
 * Diffuser::diffuseChemGPU(int rightWallIndex)
 * (src/World/Usr_World/woundHealingWorld.cpp:2403-2407,
 *  src/Diffusion/Diffuser.cpp:221-470).
 *
 * Plain C types only: pointers, sizes, ints, doubles.  A CUDA stream is
 * passed as void* (cudaStream_t); NULL means the legacy default stream.
 * Every entry point returns a vfd_status; none exits, aborts or traps.
 *
 * Data layout (unchanged from the reference): one fp32 array of nx*ny*nz
 * voxels per field, index = x + nx*(y + ny*z), x fastest
 * (src/FieldVariable/Usr_FieldVariables/WHChemical.cpp:424).
 *
 * Threading: a world is bound to one device.  Calls on different worlds are
 * thread-safe; calls on one world must be serialised by the caller (the
 * reference calls its Diffuser from one OpenMP thread,
 * woundHealingWorld.cpp:2013-2026).
 */
#ifndef VFD_H_
#define VFD_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference has none: checkCudaErrors() exits the
 * process and fftDiffuse3D's bool is ignored (Diffuser.cpp:139-148). */
typedef enum vfd_status {
    VFD_OK = 0,
    VFD_ERR_INVALID_ARG = 1,
    VFD_ERR_OUT_OF_MEMORY = 2,
    VFD_ERR_BUDGET = 3,       /* admission refused by an HBM budget      */
    VFD_ERR_CUDA = 4,         /* a CUDA runtime call failed              */
    VFD_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up      */
    VFD_ERR_DEVICE_FAULT = 6, /* a kernel reported a bad index/argument  */
    VFD_ERR_NOT_SUPPORTED = 7,
    VFD_ERR_NO_DEVICE = 8
} vfd_status;

/* Boundary treatment of the padded FFT grid.
 * VFD_PAD_ZERO: the field is zero-extended (the benchmark configurations).
 * VFD_PAD_CONSTANT_VF: the reference's padDataConstantVF3D rule
 *   (src/Diffusion/convolutionFFT.cuh:590-638): only 0<z<nz-1, 0<y<ny-1,
 *   0<x<epi_boundary keeps the field value; every other voxel of the FFT
 *   grid (padding, outer data shell, x >= epi_boundary) holds `baseline`. */
typedef enum vfd_pad_mode {
    VFD_PAD_ZERO = 0,
    VFD_PAD_CONSTANT_VF = 1
} vfd_pad_mode;

/* How a substep's 3D FFT convolution is evaluated.
 * VFD_METHOD_SEPARABLE (default): the Gaussian spectrum is separable, so the
 *   3D transform factorises into three fused per-axis FFT convolutions
 *   (forward FFT, multiply, inverse FFT, crop) with one HBM read and write of
 *   the field per axis.
 * VFD_METHOD_FFT3D: the full 3D R2C FFT, multiply by a stored 3D spectrum,
 *   C2R, with the padding rule fused into the R2C pass, the multiply fused
 *   between the forward and inverse z transforms and the crop fused into the
 *   C2R pass; zero padding and cropped outputs are pruned.  Any kernel
 *   (vfd_set_window) -- the reference's stencil-power window included.
 * VFD_METHOD_PLAIN: the same 3D transform as unfused per-field kernels in the
 *   reference's order (pad, R2C, C2C y, C2C z, multiply, C2C z, C2C y, C2R,
 *   crop) on the full FFT grid -- fftDiffuse3D's structure, Diffusion.cu:1622-1934. */
typedef enum vfd_method {
    VFD_METHOD_SEPARABLE = 0,
    VFD_METHOD_FFT3D = 1,
    VFD_METHOD_PLAIN = 2
} vfd_method;

/* Per-field diffusion parameters.
 * Kernel: normalised sampled Gaussian exp(-j^2/(2 sigma^2)) per axis,
 * truncated to [-radius, radius] on each axis and normalised in FP64 (the
 * product over the cube is therefore normalised too).  This is the
 * heat-kernel counterpart of the reference's window (the explicit 7-point
 * stencil raised to a power, src/Diffusion/Diffusion.cu:1078-1531).
 * Substep: u <- (1 - decay_rate) * (baseline + conv(M .* (u - baseline))). */
typedef struct vfd_field_params {
    double sigma[3];    /* x, y, z, in voxels; > 0                       */
    int radius[3];      /* <= 0 selects ceil(3 sigma)                    */
    double decay_rate;  /* first-order decay per substep, in [0, 1)      */
    float baseline;     /* reference pbaseline[ic] (woundHealingWorld.cpp:969);
                           ignored by VFD_PAD_ZERO                        */
} vfd_field_params;

/* One world (one set of co-located fields on one grid).  The reference
 * sizes this through c_ctx (src/Diffusion/convolutionFFT_common.h:305-346)
 * and diffusion_helper::initChemDimensions (DiffusionHelper.cpp:381-461). */
typedef struct vfd_world_desc {
    int nx, ny, nz;
    int n_fields;
    const vfd_field_params *fields; /* n_fields entries                   */
    int pad_mode;                   /* vfd_pad_mode                       */
    int epi_boundary;               /* constant-VF x bound (rightWallIndex) */
    int fft[3];                     /* FFT length per axis; 0 = planner   */
    int method;                     /* vfd_method                         */
} vfd_world_desc;

typedef struct vfd_world vfd_world;

/* Mass accounting per field, FP64 (WHChemical::update sums per-field totals
 * in double, WHChemical.cpp:420-450).  Values refer to the last substep run
 * (input_sum, leaked, conv_sum) and to the last tick (total, sources). */
typedef struct vfd_mass {
    double input_sum;   /* sum of M .* (u - b) entering the last substep  */
    double leaked[3];   /* mass the kernel pushed past the crop, per axis */
    double conv_sum;    /* sum of the cropped convolution (before +b, decay) */
    double total;       /* sum of the field after the tick (incl. sources) */
    double sources;     /* sum of the amounts deposited in the last tick  */
    double reserved;
} vfd_mass;

/* ---- world lifetime (Diffuser ctor + diffusion_helper::alloc*Buffers,
 *      Diffuser.cpp:27-35, DiffusionHelper.cpp:464-647) ------------------ */
vfd_status vfd_world_create(const vfd_world_desc *desc, int device, vfd_world **out);
vfd_status vfd_world_destroy(vfd_world *w);

/* FFT grid the planner chose (Fx, Fy, Fz) -- the reference's FFTW/H/D. */
vfd_status vfd_world_fft_dims(const vfd_world *w, int *fft3);
/* Device bytes this world holds. */
vfd_status vfd_world_device_bytes(const vfd_world *w, size_t *bytes);

/* ---- autotuning (VFD_METHOD_SEPARABLE worlds) ---------------------------
 * Per axis, the pass that runs it: the register FFT (kernel radius <= 8),
 * overlap-save FFT-64 blocks (radius <= 16) at 3 or 4 resident CTAs per SM,
 * or a full-line FFT with a chosen padded length (the three cheapest
 * 7-smooth lengths >= n + r), radix order and kernel variant.  The reference
 * leaves the padded sizes to diffusion_helper::initChemDimensions
 * (DiffusionHelper.cpp:381-461) and its transforms to cuFFT's planner. */
typedef enum {
    VFD_PASS_REGISTER_FFT = 0,
    VFD_PASS_OVERLAP_SAVE = 1,
    VFD_PASS_FULL_LINE = 2
} vfd_pass_method;

typedef struct vfd_axis_tuning {
    int method;        /* vfd_pass_method                                */
    int ctas_per_sm;   /* overlap-save: resident CTAs per SM (3 or 4)    */
    int fft_len;       /* full line: padded FFT length                   */
    int radix_order;   /* full line: 0 = radix 8 first, 1 = radix 4 first */
    int variant;       /* full line: kernel variant (tile shape)         */
    float ms;          /* tuned time of the pass over every field, or 0  */
} vfd_axis_tuning;

/* Times every candidate of each axis on temporary worlds of desc's shape
 * (zero fields, `reps` timed launches each after one warm-up; the device
 * needs room for one extra world), caches the fastest per shape (device,
 * grid, padding rule, per-field radii) and writes it to out[3].  Later
 * vfd_world_create calls with that shape use the cached choice; with the
 * environment variable VFD_AUTOTUNE=1 they tune an uncached shape first. */
vfd_status vfd_autotune(const vfd_world_desc *desc, int device, int reps, vfd_axis_tuning *out3);
/* The pass each axis of this world runs (ms: the tuned time, 0 if the
 * world was not created from a tuned choice). */
vfd_status vfd_world_tuning(const vfd_world *w, vfd_axis_tuning *out3);
/* Stores a choice for desc's shape in the cache (a saved tuning, or a pinned
 * pass): later worlds of the shape run it.  An axis whose world cannot run
 * the stored method (register FFT beyond radius 8 or on an unaligned x
 * line, overlap-save beyond radius 16) falls back to the default pass. */
vfd_status vfd_autotune_set(const vfd_world_desc *desc, int device, const vfd_axis_tuning *in3);
/* Empties the per-shape cache. */
vfd_status vfd_autotune_clear(void);

/* ---- field transfer (H2D / D2H, Diffusion.cu:72-122) ------------------ */
vfd_status vfd_upload_field(vfd_world *w, int field, const float *host, void *stream);
vfd_status vfd_download_field(vfd_world *w, int field, float *host, void *stream);
/* Device pointer of a resident field (V floats, valid until destroy). */
vfd_status vfd_field_device_ptr(vfd_world *w, int field, float **dptr);

/* ---- sources (Agent::produce_* -> dChem[ic][voxel] += inc, Agent.cpp:185)
 * Registers this field's point sources for every following tick: the
 * arrays are copied to the device; idx are voxel indices in [0, V),
 * duplicates accumulate.  n = 0 clears them. */
vfd_status vfd_set_sources(vfd_world *w, int field, const int32_t *idx,
                           const float *amt, int64_t n);

/* ---- reference-mode kernel (computeKernelSpectrum3D, Diffusion.cu:1533-1619)
 * Replaces field `field`'s Gaussian by a dense real window w (kd*kh*kw,
 * x fastest) whose centre (cx, cy, cz) is wrapped to index 0 like
 * padKernel3D (convolutionFFT.cuh:402-445); its 3D spectrum is computed on the
 * device with this library's FFT.  Worlds created with VFD_METHOD_FFT3D or
 * VFD_METHOD_PLAIN only (VFD_ERR_NOT_SUPPORTED otherwise).  The window must
 * fit the FFT grid: the planner grid covers n + max(radius); pass explicit
 * fft lengths >= n + window half-width for wider windows. */
vfd_status vfd_set_window(vfd_world *w, int field, const float *window, int kw, int kh, int kd,
                          int cx, int cy, int cz);

/* Reference-mode kernel given as its stored spectrum.  The reference keeps
 * each chemical's kernel only as chem_cctx->h_kernelspectrum[ic]: the
 * unscaled R2C transform of the wrapped window (padKernel3D) on the chemical
 * FFT grid, FFTD x FFTH x (FFTW/2+1) complex values laid out [z][y][kx] as
 * interleaved (re, im) floats, filled once by computeKernelSpectrum3D
 * (Diffusion.cu:1540-1610) into a buffer allocated per chemical
 * (DiffusionHelper.cpp:556-592).  kspec may be a host (pinned or pageable)
 * or a device pointer; it is copied, so the caller may free it on return.
 * (fx, fy, fz) must equal the world's FFT grid: create the world with
 * desc.fft = {FFTW, FFTH, FFTD}.  The kernel sum K0 (used by the constant-VF
 * rule) is Re kspec[0].  Worlds created with VFD_METHOD_FFT3D or
 * VFD_METHOD_PLAIN only (VFD_ERR_NOT_SUPPORTED otherwise). */
vfd_status vfd_set_spectrum(vfd_world *w, int field, const float *kspec, int fx, int fy, int fz);

/* computeKernelSpectrum3D (Diffusion.cu:1533-1619) without cuFFT: the
 * unscaled R2C spectrum of the window (kd*kh*kw, x fastest) wrapped with its
 * centre (cx, cy, cz) at index 0 (padKernel3D, convolutionFFT.cuh:402-445) on
 * the fx*fy*fz grid, computed on `device` with this library's FFT and written
 * to out (host, fz*fy*(fx/2+1) interleaved (re, im) floats: the layout of
 * chem_cctx->h_kernelspectrum[ic]).  fx even, 7-smooth lengths. */
vfd_status vfd_window_spectrum(const float *window, int kw, int kh, int kd, int cx, int cy, int cz,
                               int fx, int fy, int fz, float *out, int device);

/* The inverse of vfd_window_spectrum: the window (kd*kh*kw floats, x
 * fastest, centre (cx, cy, cz)) whose wrapped copy has the unscaled R2C
 * spectrum kspec (host or device, fz*fy*(fx/2+1) interleaved (re, im), the
 * reference's h_kernelspectrum[ic] layout) on the fx*fy*fz grid, computed on
 * `device` with this library's inverse transform.  With it a stored spectrum
 * can be used on any other FFT grid (vfd_set_window): the reference's
 * power-of-two grid always holds n + window - 1 points per axis, so its
 * circular convolution is the linear one and the grid can be swapped for
 * the cheapest one that also avoids wrap-around. */
vfd_status vfd_spectrum_window(const float *kspec, int fx, int fy, int fz, int kw, int kh, int kd,
                               int cx, int cy, int cz, float *window, int device);

/* Changes the constant-VF padding of a VFD_METHOD_FFT3D / VFD_METHOD_PLAIN
 * world between ticks: the x bound (the reference passes rightWallIndex =
 * bmcx - 1 to every diffuseChemGPU call, woundHealingWorld.cpp:2407) and,
 * when baselines is not NULL, each field's baseline (pbaseline[ic],
 * woundHealingWorld.cpp:970-975).  VFD_ERR_NOT_SUPPORTED for separable
 * worlds, whose passes carry the padding box in their job records. */
vfd_status vfd_set_boundary(vfd_world *w, int epi_boundary, const float *baselines);

/* Reference-mode tick epilogue on the device (WHChemical::update,
 * WHChemical.cpp:420-450): one tick of n_substeps substeps in which the last
 * substep's output t becomes
 *     p = d + decay[f] * t,    d = 0,    total[f] = sum(p) (FP64)
 * for every field f (the reference's pChem = dChem + tChem*cytokineDecay[ic],
 * dChem = 0; its decay table is woundHealingWorld.cpp:2640-2648).  dchem
 * holds n_fields device pointers of V floats (an entry, or dchem itself, may
 * be NULL: d = 0).  In VFD_METHOD_FFT3D / VFD_METHOD_PLAIN worlds the update
 * is fused into the crop store of the inverse x transform; separable worlds
 * run it as one extra pass over the fields.  Registered sources
 * (vfd_set_sources) are deposited after the update.  vfd_read_mass then
 * reports total = sum(p) + sources.  Asynchronous on `stream`. */
vfd_status vfd_tick_update(vfd_world *w, int n_substeps, float *const *dchem, const float *decay, void *stream);

/* Reference-mode window itself (computeKernel3D, Diffusion.cu:1078-1531):
 * the 7-point stencil (centre 1 - 6 lambda - gamma_dt, six arms lambda)
 * applied n_steps times to a unit impulse; out receives the centred window
 * of half-width R ((2R+1)^3 floats, x fastest, centre at (R, R, R)).
 * Computed on `device` as the inverse 3D FFT of the stencil spectrum to the
 * power n_steps.  The reference's human-VF setting is lambda = 2*15/15^2,
 * n_steps = 894, R = 73 (DiffusionHelper.cpp:48-100). */
vfd_status vfd_stencil_window(double lambda, double gamma_dt, int n_steps, int R, float *out, int device);

/* ---- one tick: n_substeps diffusion substeps of every field, then the
 * registered sources are deposited and the FP64 totals are formed.
 * Replaces fftDiffuse3D (Diffusion.cu:1622-1934) for every chemical plus
 * the deposit/total part of WHChemical::update (WHChemical.cpp:420-450).
 * Fields stay on the device; asynchronous on `stream`. -------------------- */
vfd_status vfd_tick(vfd_world *w, int n_substeps, void *stream);

/* Mass accounting of each field (n_fields entries); synchronises `stream`. */
vfd_status vfd_read_mass(vfd_world *w, vfd_mass *out, void *stream);

/* ---- drop-in of Diffuser::diffuseChemGPU (Diffuser.cpp:221-470):
 * for every field, host_in[f] -> device, one tick, device -> host_out[f]
 * (the reference's h_ibuffs / h_obuffs, DiffusionHelper.cpp:529-531).
 * Copies are pipelined against the compute of the other fields.  Host
 * buffers may be pinned or pageable; host_out may equal host_in.
 * Synchronous: returns when host_out holds the result. */
vfd_status vfd_diffuse_host(vfd_world *w, const float *const *host_in,
                            float *const *host_out, int n_substeps);

/* ---- drop-in of diffuseChemGPU followed by WHChemical::update
 * (WHChemical.cpp:420-450) with the update on the device: for every field,
 * host_p[f] (pChem) and host_d[f] (dChem) -> device, one tick whose last
 * substep's crop stores p = d + decay[f] * t (vfd_tick_update), p -> host_p[f];
 * host_d[f] is zeroed.  host_d (or an entry) may be NULL: d = 0.  FP64 totals
 * through vfd_read_mass.  Synchronous. */
vfd_status vfd_diffuse_update_host(vfd_world *w, float *const *host_p, float *const *host_d,
                                   const float *decay, int n_substeps);

/* ---- batched ensembles (sensitivity-analysis ensembles of many worlds) --
 * A batch references (does not own) n_worlds worlds on one device; they
 * must outlive it.  vfd_batch_tick is vfd_tick on every world, but every
 * field of every world goes through one persistent kernel launch per axis
 * pass per substep.  Once the same n_substeps and source lists have run two
 * ticks in a row the tick is captured into a CUDA graph and replayed
 * (re-captured when n_substeps or a world's sources change); a batch used
 * for a single tick launches directly.
 * The reference runs worlds one at a time and its chemicals one at a time
 * (Diffuser.cpp:300-341); it has no batched form. */
typedef struct vfd_batch vfd_batch;
vfd_status vfd_batch_create(vfd_world *const *worlds, int n_worlds, vfd_batch **out);
vfd_status vfd_batch_tick(vfd_batch *b, int n_substeps, void *stream);
/* Per-axis pass choice for the batch as a whole: times every candidate
 * (register FFT, overlap-save at 3 and at 4 resident CTAs per SM, full-line
 * FFT) over all the batch's fields -- one warm-up and `reps` timed launches
 * each, CUDA events -- and keeps the fastest per axis (out3, may be NULL).
 * The passes run on the worlds' own fields, which are saved to temporary
 * device buffers and restored.  The next tick re-captures the graph. */
vfd_status vfd_batch_autotune(vfd_batch *b, int reps, vfd_axis_tuning *out3);
vfd_status vfd_batch_destroy(vfd_batch *b);
const char *vfd_batch_last_error(const vfd_batch *b);

/* ---- serving: a request loop with continuous batching --------------------
 * Requests are queued from any thread.  One scheduler thread per server
 * admits them in FIFO order while a slot (max_active) is free and the
 * request's device bytes fit hbm_budget_bytes; admitted fields stay resident
 * on the device for all the request's ticks.  Each round advances every
 * active request by one tick (substeps_per_tick substeps) with all their
 * fields in one launch per axis pass; up to four rounds are queued on the
 * device at a time, so the host prepares the next rounds (admissions, batch
 * set-up) while the device works.  Finished requests are retired (totals,
 * optional download) once their last round has completed and free their
 * slot; their device memory is returned in bulk (device memory is freed
 * while the device is idle, or when the budget needs it, since freeing waits
 * for the device).
 * A request's results do not depend on which other requests share its
 * rounds (each field's lines stay in their own tiles).
 * Host buffers named by a request (init, result, mass) must stay valid until
 * the request completes; source arrays are copied at submit. */
typedef struct vfd_server vfd_server;

typedef struct vfd_request_desc {
    int nx, ny, nz, n_fields;
    const vfd_field_params *fields;    /* n_fields                          */
    int pad_mode, epi_boundary;
    int ticks;                          /* ticks while resident               */
    const float *const *init;           /* n_fields host fields, or NULL      */
    uint64_t synth_seed;                /* init == NULL: vfd_synth_field_device */
    int synth_world;                    /*   with (seed, world, field)         */
    float synth_lo, synth_hi;
    const int32_t *const *src_idx;      /* per field, or NULL (no sources)    */
    const float *const *src_amt;
    const int64_t *n_src;
    float *const *result;               /* n_fields host buffers, or NULL     */
    vfd_mass *mass;                     /* n_fields, or NULL                  */
} vfd_request_desc;

typedef struct vfd_request_info {
    uint64_t id;
    int status;                         /* vfd_status; -1 while pending       */
    double t_submit, t_admit, t_done;   /* seconds on the server clock        */
    double voxel_steps;
} vfd_request_info;

typedef struct vfd_server_stats {
    int64_t submitted, admitted, completed, rejected, active, queued, rounds;
    double busy_s;                      /* time with at least one active request */
    double voxel_steps_done;
    /* submit -> done over every submitted request: one still queued or
     * resident counts with the time it has waited so far (a lower bound of
     * its latency; `censored` of them) */
    double p50_latency_s, p99_latency_s, mean_latency_s;
    size_t hbm_in_use, hbm_peak;
    double device_s;                    /* device time of the rounds (CUDA events) */
    double p50_completed_s, p99_completed_s;  /* over completed requests only */
    int64_t censored;
    /* scheduler-thread time spent building batches, admitting requests
     * (world creation or reuse, field and source set-up), and waiting for
     * rounds to complete */
    double host_batch_s, host_admit_s, host_wait_s;
} vfd_server_stats;

vfd_status vfd_server_create(int device, size_t hbm_budget_bytes, int max_active, int substeps_per_tick,
                             vfd_server **out);
vfd_status vfd_server_submit(vfd_server *s, const vfd_request_desc *req, uint64_t *id);
/* Waits for request id; returns its status (VFD_ERR_TIMEOUT if not done). */
vfd_status vfd_server_wait(vfd_server *s, uint64_t id, double timeout_s, vfd_request_info *info);
vfd_status vfd_server_drain(vfd_server *s, double timeout_s);
vfd_status vfd_server_get_stats(vfd_server *s, vfd_server_stats *out);
double vfd_server_clock(const vfd_server *s);
/* Stops the scheduler; requests still queued or resident are dropped. */
vfd_status vfd_server_destroy(vfd_server *s);

/* ---- allocation-free single-field transform -------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (they manage all device memory in their own arena or pool, or must not
 * trigger the device-wide synchronisation that cudaMalloc / cudaFree can
 * cause inside a per-tick loop): one substep of the general 3D FFT
 * convolution of one field, in place,
 *     field <- keep * (baseline * kernel_sum + conv(M .* (field - baseline)))
 * (the VFD_METHOD_FFT3D transform; M and baseline as in vfd_pad_mode), where
 * kspec is the unscaled spectrum of the wrapped kernel window on the
 * fx * fy * fz grid, laid out [fz][fy][fx/2 + 1] as interleaved (re, im)
 * floats -- the layout of the reference's d_KernelSpectrum -- and
 * kernel_sum = Re kspec[0].  field and kspec are device pointers; fx must be
 * even and each F >= n + the window's half-width; lengths 7-smooth.
 * Allocates nothing: its scratch (the pruned field spectrum, nz*fy*(fx/2+1)
 * complex values, plus twiddles) lives in a fixed 32 MiB __device__ array
 * held by every GPU that loads the library; larger problems return
 * VFD_ERR_INVALID_ARG.  The first call on a device looks up that array's
 * address (make it before any stream capture).  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * Asynchronous on `stream`. */
vfd_status vfd_fft_diffuse3d_noalloc(float *field, const float *kspec, int nx, int ny, int nz,
                                     int fx, int fy, int fz, int pad_mode, int epi_boundary,
                                     float baseline, float kernel_sum, float keep, void *stream);

/* ---- per-kernel timing (the reference's PROFILE_GPU stage timers,
 * Diffusion.cu:1908-1912, as CUDA events) ---------------------------------
 * When enabled, every launch of this world is bracketed by CUDA events on
 * its stream.  vfd_read_profile synchronises, returns per kernel kind
 * (0 = x pass, 1 = y pass, 2 = z pass, 3 = source deposit) the summed
 * milliseconds and launch counts since the last read, and resets them. */
vfd_status vfd_world_set_profiling(vfd_world *w, int enable);
vfd_status vfd_read_profile(vfd_world *w, double *ms4, int64_t *launches4);

/* ---- steps either side of the diffusion -----------------------------------
 * Attractant gradients of WHChemical::update (WHChemical.cpp:433-441) from a
 * world whose fields are in the reference's chemical order (TNF, TGF, FGF,
 * MMP8, IL1, IL6, IL8, IL10; src/enums.h:124-138):
 *   grad = IL1 + TNF + TGF + FGF + collagen;  fib = TGF;
 *   neu = grad + IL6 + IL8;  mac = grad + elastin.
 * All pointers are device arrays of nx*ny*nz floats; collagen / elastin
 * (the ECM fragment counts) may be NULL (zero); any output may be NULL. */
vfd_status vfd_update_gradients(vfd_world *w, const float *collagen, const float *elastin,
                                float *fib, float *neu, float *mac, void *stream);
/* The compute part of sampleChem (volumeRender_kernel.cu:215-321): out
 * (device, (nx/stride)*(ny/stride)*(nz/stride) floats, x fastest) receives
 * min(field[stride*dx, stride*dy, stride*dz] * scale, 1).  The reference uses
 * stride 3 and scales 5e4, 1e4, 1e6, 100, 1e4, 1e5, 1e5, 1e4 per chemical. */
vfd_status vfd_sample_field(vfd_world *w, int field, int stride, float scale, float *out, void *stream);
/* Legacy-VTK ASCII STRUCTURED_POINTS file of one host field (scalars
 * "Color", x fastest, one line per row: the layout of util::outputChem,
 * output_utils.h:813-854), values with 9 significant digits. */
vfd_status vfd_write_vtk(const float *field, int nx, int ny, int nz, const char *path);

/* The reference's raw field writers (output_utils.h:21-128) for one host
 * field: an 8-bit volume, v -> 255 if v >= 1, 0 if v <= 0, else floor(256 v)
 * (writeNormalizedFloatRaw; append != 0 adds a frame to the file,
 * writeNormalizedFloatRawFrames), and comma-separated values, one line per
 * row and an empty line per z plane, 6 significant digits (writeFloatCsv). */
vfd_status vfd_write_raw_normalized(const float *field, int nx, int ny, int nz, const char *path, int append);
vfd_status vfd_write_csv(const float *field, int nx, int ny, int nz, const char *path);

/* ---- diagnostics ------------------------------------------------------ */
/* Exercises the bounded wait the TMA-staged passes use for their bulk copies,
 * on `device`, against a barrier that no copy will ever complete (none is
 * issued, so nothing is left in flight): the wait gives up after
 * limit_cycles SM cycles, records it in the flag the passes use, and this
 * call returns VFD_ERR_TIMEOUT -- the status vfd_read_mass reports after a
 * pass's wait gave up.  Any other status means the mechanism is broken. */
vfd_status vfd_check_wait_timeout(int device, long long limit_cycles);

const char *vfd_status_string(vfd_status s);
/* Last error message of this world (or of the last failed create when
 * w == NULL, per calling thread).  Never NULL. */
const char *vfd_last_error(const vfd_world *w);
/* Number of kernels this library launched since load (all worlds). */
uint64_t vfd_kernel_launch_count(void);

/* ---- deterministic synthetic inputs (workload generator) -------------
 * Counter-based splitmix64 stream keyed by (seed, world, field, stream):
 * field values uniform in [lo, hi); sources = n voxels drawn uniformly with
 * replacement, strengths lognormal(mu, sigma) through FP64 Box-Muller. */
vfd_status vfd_synth_field(uint64_t seed, int world, int field, float lo, float hi,
                           float *out, size_t n);
/* Same values as vfd_synth_field, generated on the device into dptr. */
vfd_status vfd_synth_field_device(uint64_t seed, int world, int field, float lo, float hi,
                                  float *dptr, size_t n, void *stream);
vfd_status vfd_synth_sources(uint64_t seed, int world, int field, int64_t n,
                             int64_t n_voxels, double mu, double sigma,
                             int32_t *idx, float *amt);

#ifdef __cplusplus
}
#endif

#endif /* VFD_H_ */
