// vfd_fft.cuh -- shared-memory mixed-radix Stockham FFT building blocks.
//
// Replaces cuFFT's 3D R2C / C2R (src/Diffusion/Diffusion.cu:1814, 1842 in the
// reference) on the product path.  Lines of one axis are transformed in
// batches of NL complex lines held in shared memory as interleaved complex
// values laid out [position][line] with an odd line stride LS = NL + 1, so
// that
//   * during butterflies each half-warp addresses NL consecutive lines of one
//     position (conflict-free 64-bit accesses, twiddles uniform per line set),
//   * transposing loads (one real line per lane) hit distinct banks.
// Each complex line carries two real lines of the field (real part and
// imaginary part).  Because the Gaussian heat-kernel spectrum is real and
// even, multiplying the spectrum of (a + i b) by it convolves a and b
// independently, so no R2C post-processing pass is needed.
//
// Twiddles are generated on the host in FP64 and stored in FP32.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vfd {

constexpr int MAX_STAGES = 12;
constexpr int NL_MAX = 16;      // largest lines-per-tile of any kernel variant

// A mixed-radix plan: F = prod(radix[s]); ns[s] = prod(radix[0..s-1]);
// ns_magic[s] = ceil(2^21 / ns[s]) gives j / ns = (j * magic) >> 21 exactly
// for j < 2048 and ns < 1024.
struct FftPlan {
    int F;
    int nst;
    int radix[MAX_STAGES];
    int ns[MAX_STAGES];
    int ns_magic[MAX_STAGES];
};

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 c_rot(float2 a)
{
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// cos / sin of 2*pi*m/R for the odd radices (mathematical constants).
template <int R>
__device__ __forceinline__ constexpr float cos_r(int m);
template <int R>
__device__ __forceinline__ constexpr float sin_r(int m);

template <>
__device__ __forceinline__ constexpr float cos_r<3>(int m)
{
    return m == 0 ? 1.0f : -0.5f;
}
template <>
__device__ __forceinline__ constexpr float sin_r<3>(int m)
{
    return m == 0 ? 0.0f : (m == 1 ? 0.866025403784438646763723170753f : -0.866025403784438646763723170753f);
}
template <>
__device__ __forceinline__ constexpr float cos_r<5>(int m)
{
    return m == 0 ? 1.0f
         : (m == 1 || m == 4) ? 0.309016994374947424102293417183f
                              : -0.809016994374947424102293417183f;
}
template <>
__device__ __forceinline__ constexpr float sin_r<5>(int m)
{
    return m == 0 ? 0.0f
         : m == 1 ? 0.951056516295153572116439333379f
         : m == 2 ? 0.587785252292473129168705954639f
         : m == 3 ? -0.587785252292473129168705954639f
                  : -0.951056516295153572116439333379f;
}
template <>
__device__ __forceinline__ constexpr float cos_r<7>(int m)
{
    return m == 0 ? 1.0f
         : (m == 1 || m == 6) ? 0.623489801858733530525004884004f
         : (m == 2 || m == 5) ? -0.222520933956314404288902564497f
                              : -0.900968867902419126236102319507f;
}
template <>
__device__ __forceinline__ constexpr float sin_r<7>(int m)
{
    return m == 0 ? 0.0f
         : m == 1 ? 0.781831482468029808708444526674f
         : m == 2 ? 0.974927912181823607018131682993f
         : m == 3 ? 0.433883739117558120475768332849f
         : m == 4 ? -0.433883739117558120475768332849f
         : m == 5 ? -0.974927912181823607018131682993f
                  : -0.781831482468029808708444526674f;
}

// In-register DFT of R points, forward (e^{-2 pi i qk/R}) or inverse.
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = c_add(a, b);
        v[1] = c_sub(a, b);
    }
};

template <bool INV>
struct Dft<4, INV> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
        float2 t2 = c_add(v[1], v[3]), t3 = c_rot<INV>(c_sub(v[1], v[3]));
        v[0] = c_add(t0, t2);
        v[2] = c_sub(t0, t2);
        v[1] = c_add(t1, t3);
        v[3] = c_sub(t1, t3);
    }
};

template <bool INV>
struct Dft<8, INV> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float h = 0.707106781186547524400844362105f;
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, INV>::run(e);
        Dft<4, INV>::run(o);
        // o[k] *= w8^k, w8 = e^{-+ i pi/4}
        o[1] = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                   : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
        o[2] = c_rot<INV>(o[2]);
        o[3] = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                   : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = c_add(e[k], o[k]);
            v[k + 4] = c_sub(e[k], o[k]);
        }
    }
};

// Odd radix: X_k = a0 + C_k -/+ i S_k, X_{R-k} = a0 + C_k +/- i S_k with
// C_k = sum_q (a_q + a_{R-q}) cos(2 pi qk/R), S_k = sum_q (a_q - a_{R-q}) sin(2 pi qk/R).
template <int R, bool INV>
struct DftOdd {
    __device__ __forceinline__ static void run(float2 *v)
    {
        constexpr int H = (R - 1) / 2;
        float2 sp[H], sm[H];
        float2 a0 = v[0];
        float2 x0 = a0;
#pragma unroll
        for (int q = 1; q <= H; ++q) {
            sp[q - 1] = c_add(v[q], v[R - q]);
            sm[q - 1] = c_sub(v[q], v[R - q]);
            x0 = c_add(x0, sp[q - 1]);
        }
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            float2 C = a0, S = make_float2(0.f, 0.f);
#pragma unroll
            for (int q = 1; q <= H; ++q) {
                const float c = cos_r<R>((q * k) % R), s = sin_r<R>((q * k) % R);
                C.x = fmaf(sp[q - 1].x, c, C.x);
                C.y = fmaf(sp[q - 1].y, c, C.y);
                S.x = fmaf(sm[q - 1].x, s, S.x);
                S.y = fmaf(sm[q - 1].y, s, S.y);
            }
            if (!INV) {
                v[k] = make_float2(C.x + S.y, C.y - S.x);
                v[R - k] = make_float2(C.x - S.y, C.y + S.x);
            } else {
                v[k] = make_float2(C.x - S.y, C.y + S.x);
                v[R - k] = make_float2(C.x + S.y, C.y - S.x);
            }
        }
        v[0] = x0;
    }
};
template <bool INV>
struct Dft<3, INV> : DftOdd<3, INV> {};
template <bool INV>
struct Dft<5, INV> : DftOdd<5, INV> {};
template <bool INV>
struct Dft<7, INV> : DftOdd<7, INV> {};

// One radix-R Stockham stage, in place on the interleaved complex tile.
// Thread (line, tj) handles butterflies j = tj, tj + TL, ...  All reads of
// the stage complete (barrier) before any write.  MAXP bounds the points a
// thread holds; buf is one register buffer shared by all radices.
//   inputs  a[j + r*M], twiddled by w_F^{(j mod Ns) * r * F/(Ns*R)}
//   outputs b[(j - j mod Ns)*R + j mod Ns + r*Ns]
template <int R, int MAXP, int TL, int NL, bool INV>
__device__ __forceinline__ void stockham_stage(float2 *__restrict__ S, int F, int Ns, int magic, int line,
                                               int tj, const float2 *__restrict__ tw, float2 (&buf)[MAXP])
{
    constexpr int LS = NL + 1;
    constexpr int MB = MAXP / R;
    const int M = F / R;
    const int step = M / Ns;
    float2(*v)[R] = reinterpret_cast<float2(*)[R]>(buf);
#pragma unroll
    for (int b = 0; b < MB; ++b) {
        const int j = tj + b * TL;
        if (j < M) {
            const int q = (j * magic) >> 21;
            const int jm = j - q * Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) v[b][r] = S[(j + r * M) * LS + line];
            if (jm != 0) {
                const int t1 = jm * step;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = tw[t1 * r];
                    if (INV) w.y = -w.y;
                    v[b][r] = c_mul(v[b][r], w);
                }
            }
            Dft<R, INV>::run(v[b]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < MB; ++b) {
        const int j = tj + b * TL;
        if (j < M) {
            const int q = (j * magic) >> 21;
            const int d = q * Ns * (R - 1) + j;  // (j - jm) * R + jm
#pragma unroll
            for (int r = 0; r < R; ++r) S[(d + r * Ns) * LS + line] = v[b][r];
        }
    }
    __syncthreads();
}

template <int MAXP, int TL, int NL, bool INV>
__device__ __forceinline__ void fft_lines(float2 *S, const FftPlan &pl, int line, int tj, const float2 *tw)
{
    float2 buf[MAXP];
#pragma unroll 1
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.radix[s], Ns = pl.ns[s], mg = pl.ns_magic[s];
        switch (R) {
        case 8: stockham_stage<8, MAXP, TL, NL, INV>(S, pl.F, Ns, mg, line, tj, tw, buf); break;
        case 4: stockham_stage<4, MAXP, TL, NL, INV>(S, pl.F, Ns, mg, line, tj, tw, buf); break;
        case 2: stockham_stage<2, MAXP, TL, NL, INV>(S, pl.F, Ns, mg, line, tj, tw, buf); break;
        case 3: stockham_stage<3, MAXP, TL, NL, INV>(S, pl.F, Ns, mg, line, tj, tw, buf); break;
        case 5: stockham_stage<5, MAXP, TL, NL, INV>(S, pl.F, Ns, mg, line, tj, tw, buf); break;
        case 7: stockham_stage<7, MAXP, TL, NL, INV>(S, pl.F, Ns, mg, line, tj, tw, buf); break;
        default: break;
        }
    }
}

}  // namespace vfd
