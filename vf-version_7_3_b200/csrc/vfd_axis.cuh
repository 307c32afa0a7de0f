// vfd_axis.cuh -- job descriptor of one axis pass of the separable FFT
// convolution (shared by the kernel and the host planner).
#pragma once
#include <stdint.h>
#include "vfd_fft.cuh"

namespace vfd {

// Slots of the per-field FP64 accounting block (8 doubles per field).
enum MassSlot {
    MS_INPUT = 0,   // sum of M .* (u - b) loaded by the x pass
    MS_LEAK_X = 1,  // mass beyond the crop, per axis
    MS_LEAK_Y = 2,
    MS_LEAK_Z = 3,
    MS_CONV = 4,    // sum of the cropped convolution (z pass, before +b / decay)
    MS_OUT = 5,     // sum of the stored field after the substep
    MS_SOURCES = 6, // sum of deposited amounts
    MS_COUNT = 8
};

enum PassKind { PASS_X = 0, PASS_Y = 1, PASS_Z = 2 };

// One (field, axis) pass.  Real lines of the field are addressed as
//   base + line*line_stride + outer*outer_stride + pos*pos_stride,
// line in [0, nlines), outer in [0, nouter), pos in [0, n).
// A tile takes 2*NL consecutive lines of one outer index (NL of the kernel
// variant the launch uses); line l0+q goes to complex line q % NL, real part
// for q < NL, imaginary part otherwise.
struct AxisJob {
    float *data;
    const float2 *tw;     // F twiddles exp(-2 pi i m / F), FP64-generated
    const float *spec;    // F real multipliers: G(k) / F
    double *mass;         // MS_COUNT doubles for this field
    int64_t line_stride;
    int64_t outer_stride;
    int64_t pos_stride;
    int n;                // data length along the axis
    int nlines;           // real lines per outer index
    int nouter;
    int tiles_per_outer;  // ceil(nlines / (2*NL))
    int tile_begin;       // first tile of this job in the launch
    int kind;             // PassKind
    float b;              // baseline (constant-VF padding value)
    float keep;           // 1 - decay_rate (z pass)
    int nx, ny;           // grid dims, to recover (y, z) of an x-pass row
    int box_lo[3], box_hi[3];  // interior box of the padding rule (x, y, z)
    FftPlan plan;
};

}  // namespace vfd
