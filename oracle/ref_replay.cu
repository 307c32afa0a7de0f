// ref_replay.cu -- replays the reference's per-field GPU diffusion with the
// reference's OWN kernels (src/Diffusion/convolutionFFT.cu, compiled from the
// reference tree by oracle/Makefile) and cuFFT, in the call order of
// computeKernelSpectrum3D (Diffusion.cu:1533-1619) and fftDiffuse3D
// (Diffusion.cu:1622-1934):
//   memset pad; padDataConstantVF3D; cufftExecR2C; modulateAndNormalize3D
//   (padding 1, scale 1/(fftD*fftH*fftW)); cufftExecC2R; unpadResult3D.
//
// TEST INFRASTRUCTURE ONLY: it pins the oracle and the product against the
// reference's real GPU path on a B200.  Never linked into libvfd.so.
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdio.h>
#include <stdlib.h>

extern "C" void padKernel3D(float *d_Dst, float *d_Src, int fftD, int fftH, int fftW, int kernelD,
                            int kernelH, int kernelW, int kernelZ, int kernelY, int kernelX);
extern "C" void padDataConstantVF3D(float *d_Dst, float *d_Src, int fftD, int fftH, int fftW, int dataD,
                                    int dataH, int dataW, int kernelD, int kernelH, int kernelW,
                                    int kernelZ, int kernelY, int kernelX, int epiBoundary,
                                    float baseChem);
extern "C" void modulateAndNormalize3D(float2 *d_Dst, float2 *d_Src, int fftD, int fftH, int fftW,
                                       int padding);
extern "C" void unpadResult3D(float *d_Dst, float *d_Src, int dataD, int dataH, int dataW, int fftD,
                              int fftH, int fftW);
extern "C" void padDataClampToBorder3D(float *d_Dst, float *d_Src, int fftD, int fftH, int fftW, int dataD,
                                       int dataH, int dataW, int kernelD, int kernelH, int kernelW, int kernelZ,
                                       int kernelY, int kernelX);
extern "C" void complexPower(float2 *d_Dst, int fftD, int fftH, int fftW, int padding, int n);
extern "C" void extractCenter3D(float *d_Dst, float *d_Src, int dataD, int dataH, int dataW, int windowD,
                                int windowH, int windowW);

#define RR_CHECK(x)                                                                    \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            snprintf(g_err, sizeof(g_err), "%s: %s", #x, cudaGetErrorString(e_));      \
            rc = -1;                                                                   \
            goto done;                                                                 \
        }                                                                              \
    } while (0)
#define RR_CUFFT(x)                                                                    \
    do {                                                                               \
        cufftResult r_ = (x);                                                          \
        if (r_ != CUFFT_SUCCESS) {                                                     \
            snprintf(g_err, sizeof(g_err), "%s: cufft error %d", #x, (int)r_);         \
            rc = -2;                                                                   \
            goto done;                                                                 \
        }                                                                              \
    } while (0)

static char g_err[512] = "";

extern "C" const char *ref_replay_error(void) { return g_err; }

// One field: h_in (D*H*W, x fastest) -> h_out, kernel window h_win
// (kD*kH*kW, centre kZ,kY,kX) on an fftD*fftH*fftW grid.
extern "C" int ref_replay_fft_diffuse3d(const float *h_in, float *h_out, int D, int H, int W, int fftD,
                                        int fftH, int fftW, const float *h_win, int kD, int kH, int kW,
                                        int kZ, int kY, int kX, int epi, float baseChem)
{
    int rc = 0;
    float *d_data = nullptr, *d_win = nullptr, *d_pk = nullptr, *d_pad = nullptr;
    float2 *d_ks = nullptr, *d_ds = nullptr;
    cufftHandle fwd = 0, inv = 0;
    bool have_fwd = false, have_inv = false;
    const size_t dsz = (size_t)D * H * W, fsz = (size_t)fftD * fftH * fftW;
    const size_t ssz = (size_t)fftD * fftH * (fftW / 2 + 1);
    const size_t wsz = (size_t)kD * kH * kW;
    RR_CHECK(cudaMalloc(&d_data, dsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_win, wsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_pk, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_pad, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_ks, ssz * sizeof(float2)));
    RR_CHECK(cudaMalloc(&d_ds, ssz * sizeof(float2)));
    RR_CHECK(cudaMemcpy(d_data, h_in, dsz * sizeof(float), cudaMemcpyHostToDevice));
    RR_CHECK(cudaMemcpy(d_win, h_win, wsz * sizeof(float), cudaMemcpyHostToDevice));
    RR_CUFFT(cufftPlan3d(&fwd, fftD, fftH, fftW, CUFFT_R2C));
    have_fwd = true;
    RR_CUFFT(cufftPlan3d(&inv, fftD, fftH, fftW, CUFFT_C2R));
    have_inv = true;
    // kernel spectrum (computeKernelSpectrum3D)
    RR_CHECK(cudaMemset(d_pk, 0, fsz * sizeof(float)));
    padKernel3D(d_pk, d_win, fftD, fftH, fftW, kD, kH, kW, kZ, kY, kX);
    RR_CHECK(cudaGetLastError());
    RR_CUFFT(cufftExecR2C(fwd, (cufftReal *)d_pk, (cufftComplex *)d_ks));
    // fftDiffuse3D
    RR_CHECK(cudaMemset(d_pad, 0, fsz * sizeof(float)));
    padDataConstantVF3D(d_pad, d_data, fftD, fftH, fftW, D, H, W, kD, kH, kW, kZ, kY, kX, epi, baseChem);
    RR_CHECK(cudaGetLastError());
    RR_CUFFT(cufftExecR2C(fwd, (cufftReal *)d_pad, (cufftComplex *)d_ds));
    modulateAndNormalize3D(d_ds, d_ks, fftD, fftH, fftW, 1);
    RR_CHECK(cudaGetLastError());
    RR_CUFFT(cufftExecC2R(inv, (cufftComplex *)d_ds, (cufftReal *)d_pad));
    unpadResult3D(d_data, d_pad, D, H, W, fftD, fftH, fftW);
    RR_CHECK(cudaGetLastError());
    RR_CHECK(cudaMemcpy(h_out, d_data, dsz * sizeof(float), cudaMemcpyDeviceToHost));
done:
    if (have_fwd) cufftDestroy(fwd);
    if (have_inv) cufftDestroy(inv);
    cudaFree(d_data);
    cudaFree(d_win);
    cudaFree(d_pk);
    cudaFree(d_pad);
    cudaFree(d_ks);
    cudaFree(d_ds);
    return rc;
}

// computeKernelSpectrum3D (Diffusion.cu:1533-1619) replayed: the window
// (kD*kH*kW, centre kZ,kY,kX) wrapped onto the fftD*fftH*fftW grid by the
// reference's padKernel3D, transformed by cuFFT R2C, copied to h_spec
// (fftD*fftH*(fftW/2+1) complex values, interleaved) -- the reference's
// h_kernelspectrum[ic].
extern "C" int ref_kernel_spectrum(const float *h_win, int kD, int kH, int kW, int kZ, int kY, int kX, int fftD,
                                   int fftH, int fftW, float *h_spec)
{
    int rc = 0;
    float *d_win = nullptr, *d_pk = nullptr;
    float2 *d_ks = nullptr;
    cufftHandle fwd = 0;
    bool have_fwd = false;
    const size_t fsz = (size_t)fftD * fftH * fftW;
    const size_t ssz = (size_t)fftD * fftH * (fftW / 2 + 1);
    const size_t wsz = (size_t)kD * kH * kW;
    RR_CHECK(cudaMalloc(&d_win, wsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_pk, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_ks, ssz * sizeof(float2)));
    RR_CHECK(cudaMemcpy(d_win, h_win, wsz * sizeof(float), cudaMemcpyHostToDevice));
    RR_CUFFT(cufftPlan3d(&fwd, fftD, fftH, fftW, CUFFT_R2C));
    have_fwd = true;
    RR_CHECK(cudaMemset(d_pk, 0, fsz * sizeof(float)));
    padKernel3D(d_pk, d_win, fftD, fftH, fftW, kD, kH, kW, kZ, kY, kX);
    RR_CHECK(cudaGetLastError());
    RR_CUFFT(cufftExecR2C(fwd, (cufftReal *)d_pk, (cufftComplex *)d_ks));
    RR_CHECK(cudaMemcpy(h_spec, d_ks, ssz * sizeof(float2), cudaMemcpyDeviceToHost));
done:
    if (have_fwd) cufftDestroy(fwd);
    cudaFree(d_win);
    cudaFree(d_pk);
    cudaFree(d_ks);
    return rc;
}

// computeKernel3D (Diffusion.cu:1078-1401) replayed with the reference's own
// kernels and cuFFT: the 3x3x3 stencil (centre 1 - 6 lambda - gamma_dt, six
// arms lambda) placed at the centre of a D^3 data cube (D = 2 (kernelRadius -
// 1) + 1); niter rounds of padKernel3D(stencil) + padDataClampToBorder3D(data)
// on the F^3 grid, R2C of both, complexPower(K, kernelRadius - 1 - [first
// round]), modulateAndNormalize3D, C2R, unpadResult3D; then the centred
// window^3 (extractCenter3D) into h_window.  The reference's human-VF setting
// is kernelRadius 150, niter 6, F 616, window 147 (DiffusionHelper.cpp:48-100).
extern "C" int ref_compute_kernel3d(float lambda, float gamma_dt, int kernelRadius, int niter, int F, int window,
                                    float *h_window)
{
    int rc = 0;
    const int D = (kernelRadius - 1) * 2 + 1;
    const size_t dsz = (size_t)D * D * D, fsz = (size_t)F * F * F, ssz = (size_t)F * F * (F / 2 + 1);
    const size_t wsz = (size_t)window * window * window;
    float *d_data = nullptr, *d_kern = nullptr, *d_pdata = nullptr, *d_pkern = nullptr, *d_win = nullptr;
    float2 *d_kspec = nullptr, *d_dspec = nullptr;
    float *h_data = nullptr;
    cufftHandle fwd = 0, inv = 0;
    bool have_fwd = false, have_inv = false;
    float h_kern[27];
    for (int i = 0; i < 27; ++i) h_kern[i] = 0.0f;
    // Diffusion.cu:1182-1195: z-arms, y-arms, x-arms and the centre
    h_kern[0 * 9 + 1 * 3 + 1] = lambda;
    h_kern[2 * 9 + 1 * 3 + 1] = lambda;
    h_kern[1 * 9 + 0 * 3 + 1] = lambda;
    h_kern[1 * 9 + 2 * 3 + 1] = lambda;
    h_kern[1 * 9 + 1 * 3 + 0] = lambda;
    h_kern[1 * 9 + 1 * 3 + 2] = lambda;
    h_kern[1 * 9 + 1 * 3 + 1] = 1.0f - 6.0f * lambda - gamma_dt;
    h_data = (float *)calloc(dsz, sizeof(float));
    if (!h_data) return -3;
    // the stencil at the centre of the data cube (Diffusion.cu:1207-1226)
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                h_data[((size_t)(D / 2 - 1 + k) * D + (D / 2 - 1 + i)) * D + (D / 2 - 1 + j)] = h_kern[k * 9 + i * 3 + j];
    RR_CHECK(cudaMalloc(&d_data, dsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_kern, 27 * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_pdata, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_pkern, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_kspec, ssz * sizeof(float2)));
    RR_CHECK(cudaMalloc(&d_dspec, ssz * sizeof(float2)));
    RR_CHECK(cudaMalloc(&d_win, wsz * sizeof(float)));
    RR_CHECK(cudaMemcpy(d_kern, h_kern, 27 * sizeof(float), cudaMemcpyHostToDevice));
    RR_CHECK(cudaMemcpy(d_data, h_data, dsz * sizeof(float), cudaMemcpyHostToDevice));
    RR_CHECK(cudaMemset(d_pkern, 0, fsz * sizeof(float)));
    RR_CHECK(cudaMemset(d_pdata, 0, fsz * sizeof(float)));
    RR_CUFFT(cufftPlan3d(&fwd, F, F, F, CUFFT_R2C));
    have_fwd = true;
    RR_CUFFT(cufftPlan3d(&inv, F, F, F, CUFFT_C2R));
    have_inv = true;
    for (int it = 0; it < niter; ++it) {
        padKernel3D(d_pkern, d_kern, F, F, F, 3, 3, 3, 1, 1, 1);
        padDataClampToBorder3D(d_pdata, d_data, F, F, F, D, D, D, 3, 3, 3, 1, 1, 1);
        RR_CHECK(cudaGetLastError());
        RR_CUFFT(cufftExecR2C(fwd, (cufftReal *)d_pkern, (cufftComplex *)d_kspec));
        RR_CUFFT(cufftExecR2C(fwd, (cufftReal *)d_pdata, (cufftComplex *)d_dspec));
        complexPower(d_kspec, F, F, F, 1, kernelRadius - (it == 0 ? 1 : 0) - 1);
        modulateAndNormalize3D(d_dspec, d_kspec, F, F, F, 1);
        RR_CHECK(cudaGetLastError());
        RR_CUFFT(cufftExecC2R(inv, (cufftComplex *)d_dspec, (cufftReal *)d_pdata));
        unpadResult3D(d_data, d_pdata, D, D, D, F, F, F);
        RR_CHECK(cudaGetLastError());
    }
    extractCenter3D(d_win, d_data, D, D, D, window, window, window);
    RR_CHECK(cudaGetLastError());
    RR_CHECK(cudaMemcpy(h_window, d_win, wsz * sizeof(float), cudaMemcpyDeviceToHost));
done:
    if (have_fwd) cufftDestroy(fwd);
    if (have_inv) cufftDestroy(inv);
    cudaFree(d_data);
    cudaFree(d_kern);
    cudaFree(d_pdata);
    cudaFree(d_pkern);
    cudaFree(d_kspec);
    cudaFree(d_dspec);
    cudaFree(d_win);
    free(h_data);
    return rc;
}

// Times the reference's per-field diffusion on the device, window spectrum
// prepared once.  ms[0]: the kernels + cuFFT of one fftDiffuse3D call
// (memset, padDataConstantVF3D, R2C, modulateAndNormalize3D, C2R,
// unpadResult3D) with buffers and plans reused; ms[1]: the same call as the
// reference makes it each tick -- cufftPlan3d x2 (Diffuser.cpp:273-274),
// cudaMalloc of the padded and spectrum buffers (Diffusion.cu:1686-1687),
// the kernels, cudaFree and cufftDestroy.  Averages over `iters` calls.
extern "C" int ref_replay_time(int D, int H, int W, int fftD, int fftH, int fftW, const float *h_win, int kD,
                               int kH, int kW, int kZ, int kY, int kX, int epi, float baseChem, int iters,
                               double *ms)
{
    int rc = 0;
    float *d_data = nullptr, *d_win = nullptr, *d_pk = nullptr, *d_pad = nullptr;
    float2 *d_ks = nullptr, *d_ds = nullptr;
    cufftHandle fwd = 0, inv = 0;
    bool have_fwd = false, have_inv = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const size_t dsz = (size_t)D * H * W, fsz = (size_t)fftD * fftH * fftW;
    const size_t ssz = (size_t)fftD * fftH * (fftW / 2 + 1);
    const size_t wsz = (size_t)kD * kH * kW;
    float t = 0.0f;
    RR_CHECK(cudaEventCreate(&e0));
    RR_CHECK(cudaEventCreate(&e1));
    RR_CHECK(cudaMalloc(&d_data, dsz * sizeof(float)));
    RR_CHECK(cudaMemset(d_data, 0, dsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_win, wsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_pk, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_ks, ssz * sizeof(float2)));
    RR_CHECK(cudaMemcpy(d_win, h_win, wsz * sizeof(float), cudaMemcpyHostToDevice));
    RR_CUFFT(cufftPlan3d(&fwd, fftD, fftH, fftW, CUFFT_R2C));
    have_fwd = true;
    RR_CUFFT(cufftPlan3d(&inv, fftD, fftH, fftW, CUFFT_C2R));
    have_inv = true;
    RR_CHECK(cudaMemset(d_pk, 0, fsz * sizeof(float)));
    padKernel3D(d_pk, d_win, fftD, fftH, fftW, kD, kH, kW, kZ, kY, kX);
    RR_CUFFT(cufftExecR2C(fwd, (cufftReal *)d_pk, (cufftComplex *)d_ks));
    RR_CHECK(cudaMalloc(&d_pad, fsz * sizeof(float)));
    RR_CHECK(cudaMalloc(&d_ds, ssz * sizeof(float2)));
    for (int pass = 0; pass < 2; ++pass) {
        for (int it = -1; it < iters; ++it) {  // it = -1: warm-up
            if (it == 0) RR_CHECK(cudaEventRecord(e0));
            cufftHandle f2 = fwd, i2 = inv;
            float *pad = d_pad;
            float2 *ds = d_ds;
            if (pass == 1) {
                RR_CUFFT(cufftPlan3d(&f2, fftD, fftH, fftW, CUFFT_R2C));
                RR_CUFFT(cufftPlan3d(&i2, fftD, fftH, fftW, CUFFT_C2R));
                RR_CHECK(cudaMalloc(&pad, fsz * sizeof(float)));
                RR_CHECK(cudaMalloc(&ds, ssz * sizeof(float2)));
            }
            RR_CHECK(cudaMemset(pad, 0, fsz * sizeof(float)));
            padDataConstantVF3D(pad, d_data, fftD, fftH, fftW, D, H, W, kD, kH, kW, kZ, kY, kX, epi, baseChem);
            RR_CUFFT(cufftExecR2C(f2, (cufftReal *)pad, (cufftComplex *)ds));
            modulateAndNormalize3D(ds, d_ks, fftD, fftH, fftW, 1);
            RR_CUFFT(cufftExecC2R(i2, (cufftComplex *)ds, (cufftReal *)pad));
            unpadResult3D(d_data, pad, D, H, W, fftD, fftH, fftW);
            if (pass == 1) {
                RR_CHECK(cudaDeviceSynchronize());
                cudaFree(pad);
                cudaFree(ds);
                cufftDestroy(f2);
                cufftDestroy(i2);
            }
        }
        RR_CHECK(cudaEventRecord(e1));
        RR_CHECK(cudaEventSynchronize(e1));
        RR_CHECK(cudaEventElapsedTime(&t, e0, e1));
        ms[pass] = (double)t / iters;
    }
done:
    if (have_fwd) cufftDestroy(fwd);
    if (have_inv) cufftDestroy(inv);
    cudaFree(d_data);
    cudaFree(d_win);
    cudaFree(d_pk);
    cudaFree(d_pad);
    cudaFree(d_ks);
    cudaFree(d_ds);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return rc;
}
