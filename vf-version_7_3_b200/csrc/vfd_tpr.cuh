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
// vfd_fft.cuh).  Twiddles come from the FP32 table tw[m] = e^{-2 pi i m / F}
// (generated in FP64 on the host): the small DFTs of length N use
// tw[e * F / N].  Unnormalised in both directions, as fft_lines.
#pragma once
#include "vfd_fft.cuh"

namespace vfd {

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
// w_N^(r k2) -> R-point DFTs -> X[k2 + M k1].  ts = F / N (twiddle stride).
template <int N, bool INV>
__device__ __forceinline__ void tpr_dft(float2 *x, const float2 *__restrict__ tw, int ts)
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
        for (int r = 0; r < R; ++r) tpr_dft<M, INV>(y[r], tw, ts * R);
#pragma unroll
        for (int r = 1; r < R; ++r)
#pragma unroll
            for (int k2 = 1; k2 < M; ++k2) {
                float2 w = tw[r * k2 * ts];
                if (INV) w.y = -w.y;
                y[r][k2] = c_mul(y[r][k2], w);
            }
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
