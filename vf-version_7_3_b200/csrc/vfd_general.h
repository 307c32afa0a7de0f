// vfd_general.h -- parameter blocks of the general 3D FFT convolution kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vfd_fft.cuh"

namespace vfd {

enum GenMode { GEN_FORWARD = 0, GEN_INVERSE = 1, GEN_FWD_MUL_INV = 2 };

// Row pass along x (R2C forward or C2R inverse).  Row r of nrows splits into
// (r1, r2) = (r % rows_per_plane, r / rows_per_plane); its real data start at
// rsrc/rdst + r1*r_s1 + r2*r_s2 and its half spectrum at c + r1*c_s1 + r2*c_s2.
struct GenRowPass {
    FftPlan plan;
    const float2 *tw;
    int nrows, rows_per_plane;
    int64_t r_s1, r_s2, c_s1, c_s2;
    int nload;   // R2C: real positions read (others zero)
    int nstore;  // C2R: real positions written
    const float *rsrc;
    float *rdst;
    float2 *cdst;
    const float2 *csrc;
    // fused padding rule on load (R2C): v = box ? u - b : 0 with (x, r1, r2)
    int fuse_pad;
    int box_lo[3], box_hi[3];
    float b;
    // fused crop epilogue on store (C2R): out = keep * (t + b * k0); with
    // fuse_update additionally out <- d + upd_scale * out and d <- 0 (the
    // WHChemical::update epilogue; dchem NULL means d = 0)
    int fuse_crop;
    float keep, k0;
    int fuse_update;
    float upd_scale;
    float *dchem;
    double *mass_in, *mass_leak, *mass_conv, *mass_out;  // may be NULL
};

// Column pass along y or z over complex data: element (line, outer, pos) at
// data + line + outer*outer_stride + pos*pos_stride.
struct GenColPass {
    FftPlan plan;
    const float2 *tw;
    float2 *data;
    int nlines, nouter;
    int64_t outer_stride, pos_stride;
    int nload, nstore;
    int mode;                 // GenMode
    const float2 *kspec;      // GEN_FWD_MUL_INV: spectrum, element (kx, ky, kz) at
    int64_t k_s_outer, k_s_pos;  //   kspec + kx + ky*k_s_outer + kz*k_s_pos
    float scale;
    int kspec_smem;           // set by the Stockham launcher: spectrum tile staged in shared memory
};

// Register engine (vfd_gen_tpr.cu).  tpr_split: F = f1 * f2 with
// f1 <= f2 <= 32 both lengths the engine runs (f2 as small as possible), 0
// when F has no such split.  The launchers take the split to use; they
// return cudaErrorInvalidConfiguration, without launching, when the tile
// does not fit in shared memory.
int tpr_split(int F);
cudaError_t launch_tpr_rows(const GenRowPass &p, int f1, bool inverse, cudaStream_t st);
cudaError_t launch_tpr_cols(const GenColPass &p, int f1, cudaStream_t st);

cudaError_t launch_gen_rows(int variant, const GenRowPass &p, bool inverse, cudaStream_t st);
cudaError_t launch_gen_cols(int variant, const GenColPass &p, cudaStream_t st);
cudaError_t launch_pad(float *P, const float *u, int nx, int ny, int nz, int Fx, int Fy, int Fz, const int *lo,
                       const int *hi, float b, cudaStream_t st);
cudaError_t launch_modulate(float2 *C, const float2 *K, int64_t n, float scale, cudaStream_t st);
cudaError_t launch_crop(float *u, const float *P, int nx, int ny, int nz, int Fx, int Fy, float keep,
                        double *mass_conv, double *mass_out, cudaStream_t st, int fuse_update = 0,
                        float upd_scale = 1.0f, float *dchem = nullptr);
// p = d + scale * p, d = 0 (d may be NULL), FP64 total of p added to mass_out.
cudaError_t launch_update(float *p, float *d, float scale, int64_t n, double *mass_out, cudaStream_t st);
cudaError_t launch_sum(const float *P, int64_t n, double *out, cudaStream_t st);
cudaError_t launch_outer_spectrum(float2 *K, const float *sx, const float *sy, const float *sz, int Fx, int Fy,
                                  int Fz, cudaStream_t st);
cudaError_t launch_stencil_spectrum(float2 *K, int G, double lambda, double centre, int n, cudaStream_t st);
cudaError_t launch_crop_window(float *w, const float *P, int G, int R, float scale, cudaStream_t st);
cudaError_t launch_wrap_window(float *P, const float *w, int kw, int kh, int kd, int cx, int cy, int cz, int Fx,
                               int Fy, int Fz, cudaStream_t st);
cudaError_t launch_unwrap_window(float *w, const float *P, int kw, int kh, int kd, int cx, int cy, int cz, int Fx,
                                 int Fy, int Fz, float scale, cudaStream_t st);

}  // namespace vfd
