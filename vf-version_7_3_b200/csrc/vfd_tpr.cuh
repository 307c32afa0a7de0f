// vfd_tpr.cuh -- in-register DFTs of the two-pass register FFT engine.
//
// A line of length F = F1 * F2 (F1, F2 <= 32, 7-smooth) is transformed in two
// passes instead of one Stockham stage per radix (vfd_fft.cuh):
//
//   forward  A: for every n2 < F2, the strided group x[n2 + F2 n1] (n1 < F1)
//               -> DFT of length F1 in registers -> times w_F^(n2 k1);
//            B: for every k1 < F1, the F2 values A left for that k1
//               -> DFT of length F2 in registers -> X[k1 + F1 k2] (k2 < F2).
//   inverse  B': for every k1, the bins k1 + F1 k2 -> inverse DFT of length
//               F2 -> times conj(w_F^(n2 k1));  A': for every n2, the F1
//               values B' left for that n2 -> inverse DFT of length F1
//               -> y[n2 + F2 n1].
//
// Every butterfly of a group runs in one thread's registers (fully unrolled
// small DFTs built recursively from the radix-2/3/4/5/7/8 kernels of
// vfd_fft.cuh).  The twiddles inside a small DFT of length N, w_N^e, depend
// only on N and e, both known at compile time: they are FP32 immediates of
// the multiply instructions (values computed by the compiler in FP64, below),
// multiples of a quarter turn are sign changes and swaps, odd eighths of a
// turn use the sqrt(1/2) form.  The pass twiddles w_F^(k1 n2) depend on the
// runtime length F and come from shared-memory tables staged by the caller.
// Unnormalised in both directions, as fft_lines.
#pragma once
#include <utility>

#include "vfd_fft.cuh"

namespace vfd {

// ---------------------------------------------------------------------------
// cos / sin of 2 pi e / n in FP64, for constant expressions only (twiddle
// immediates).  Quadrant reduction in integers (4e = q n + rem, angle =
// q pi/2 + psi with psi = (pi/2) rem / n in [0, pi/2)), then the Taylor
// series of sin and cos at psi to 16 terms (the last term is below 1e-22).
__host__ __device__ constexpr double tpr_series(double x, bool sine)
{
    double term = sine ? x : 1.0, sum = term;
    const double x2 = x * x;
    for (int k = sine ? 2 : 1; k < 34; k += 2) {
        term = -term * x2 / (double)(k * (k + 1));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double tpr_trig2pi(int e, int n, bool sine)
{
    const int t = ((e % n) + n) % n;
    const int q = (4 * t) / n, rem = 4 * t - q * n;
    const double psi = 1.57079632679489661923132169163975 * (double)rem / (double)n;
    const double c = tpr_series(psi, false), s = tpr_series(psi, true);
    // cos(q pi/2 + psi), sin(q pi/2 + psi)
    if (!sine) return q == 0 ? c : q == 1 ? -s : q == 2 ? -c : s;
    return q == 0 ? s : q == 1 ? c : q == 2 ? -s : -c;
}

// a * w_N^E (forward, w = e^{-2 pi i / N}) or a * conj(w_N^E) (inverse).
template <int N, bool INV, int E>
__device__ __forceinline__ float2 tpr_twiddle(float2 a)
{
    constexpr int e = E % N;
    if constexpr (e == 0) {
        return a;
    } else if constexpr ((4 * e) % N == 0) {
        constexpr int q = 4 * e / N;  // quarter turns: 1 -> -i, 2 -> -1, 3 -> +i (forward)
        if constexpr (q == 2) return make_float2(-a.x, -a.y);
        else if constexpr (q == 1) return c_rot<INV>(a);
        else return c_rot<!INV>(a);
    } else if constexpr ((8 * e) % N == 0) {
        // odd eighth turns: w = (cx + i sy) sqrt(1/2) with cx, sy = +-1
        constexpr float h = 0.707106781186547524400844362105f;
        constexpr int o = 8 * e / N;  // 1, 3, 5, 7
        constexpr float cx = (o == 1 || o == 7) ? 1.0f : -1.0f;
        constexpr float sf = (o == 1 || o == 3) ? -1.0f : 1.0f;  // sign of Im w (forward)
        constexpr float sy = INV ? -sf : sf;
        // (a.x + i a.y)(cx + i sy) h
        return make_float2(h * (cx * a.x - sy * a.y), h * (cx * a.y + sy * a.x));
    } else {
        constexpr float c = (float)tpr_trig2pi(e, N, false);
        constexpr float s = INV ? (float)tpr_trig2pi(e, N, true) : -(float)tpr_trig2pi(e, N, true);
        return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
    }
}

// y[r][k2] *= w_N^(r k2) for every r < R, k2 < M (I = r M + k2).
template <int N, bool INV, int R, int M, int... I>
__device__ __forceinline__ void tpr_twiddle_all(float2 (&y)[R][M], std::integer_sequence<int, I...>)
{
    ((y[I / M][I % M] = tpr_twiddle<N, INV, (I / M) * (I % M)>(y[I / M][I % M])), ...);
}

template <int N>
__device__ __forceinline__ constexpr bool tpr_is_base()
{
    return N == 2 || N == 3 || N == 4 || N == 5 || N == 7 || N == 8;
}
template <int N>
__device__ __forceinline__ constexpr int tpr_radix()
{
    return N % 8 == 0 ? 8 : N % 7 == 0 ? 7 : N % 5 == 0 ? 5 : N % 4 == 0 ? 4 : N % 3 == 0 ? 3 : 2;
}

// In-register DFT of N points (forward e^{-2 pi i nk/N}, or inverse), by
// decimation in time N = R * M: x[R m + r] -> M-point DFTs per r -> times
// w_N^(r k2) (compile-time immediates) -> R-point DFTs -> X[k2 + M k1].
template <int N, bool INV>
__device__ __forceinline__ void tpr_dft(float2 *x)
{
    if constexpr (tpr_is_base<N>()) {
        Dft<N, INV>::run(x);
    } else {
        constexpr int R = tpr_radix<N>(), M = N / R;
        float2 y[R][M];
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) y[r][m] = x[R * m + r];
#pragma unroll
        for (int r = 0; r < R; ++r) tpr_dft<M, INV>(y[r]);
        tpr_twiddle_all<N, INV>(y, std::make_integer_sequence<int, R * M>{});
#pragma unroll
        for (int k2 = 0; k2 < M; ++k2) {
            float2 t[R];
#pragma unroll
            for (int r = 0; r < R; ++r) t[r] = y[r][k2];
            Dft<R, INV>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) x[k2 + M * k1] = t[k1];
        }
    }
}

// Lengths a pass can take (F1 and F2); TPR_MAX bounds both.
#define VFD_TPR_SIZES(X) \
    X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(12) X(14) X(15) X(16) X(18) X(20) X(21) X(24) X(25) X(27) \
    X(28) X(30) X(32)
constexpr int TPR_MAX = 32;

}  // namespace vfd
