// ref_shim_harness.cpp -- drives the Diffuser drop-in
// (vf-version_7_3_b200/host/vfd_diffuser.hpp) the way WHWorld drives the
// reference's Diffuser, with the reference's OWN context type c_ctx
// (src/Diffusion/convolutionFFT_common.h, included from the reference tree by
// oracle/Makefile, never copied) and the reference's own allocation pattern:
//
//   * chem_cctx is heap-allocated and lives on (woundHealingWorld.cpp:1014);
//     h_ibuffs[ic] / h_obuffs[ic] alias the chemical's pChem / tChem arrays
//     (DiffusionHelper.cpp:529-531); dev_id[ic] from gpu_id = ic % N_GPU
//     (DiffusionHelper.cpp:386-392; both GPUs map to device 0 here);
//   * h_kernelspectrum[ic] is one host buffer per chemical
//     (DiffusionHelper.cpp:556-592), filled by replaying the reference's
//     computeKernelSpectrum3D (its padKernel3D kernel + cuFFT R2C,
//     oracle/ref_replay.cu) from the chemical's window;
//   * the kernel context is a LOCAL of the init function
//     (woundHealingWorld.cpp:1010) whose h_data is one window buffer per GPU,
//     shared by chemicals ic and ic + N_GPU and overwritten chemical by
//     chemical (DiffusionHelper.cpp:218-247); after the Diffuser is
//     constructed its buffers are freed (deallocConvCtxBuffers,
//     woundHealingWorld.cpp:1038), the struct is poisoned here, and the
//     function returns -- before the first diffuseChemGPU.
//
// WHChemical itself drags in the whole agent model, so a stand-in carries the
// public members the drop-in reads (pbaseline, pChem, dChem, tChem, total).
//
// TEST INFRASTRUCTURE ONLY (tests/test_diffuser_shim_gpu.py).
#include <cstdlib>
#include <cstring>
#include <string>

#include "convolutionFFT_common.h"
#include "vfd_diffuser.hpp"

extern "C" int ref_kernel_spectrum(const float *h_win, int kD, int kH, int kW, int kZ, int kY, int kX, int fftD,
                                   int fftH, int fftW, float *h_spec);
extern "C" const char *ref_replay_error(void);

namespace {

struct ChemStandIn {
    float *pbaseline = nullptr;
    float *pChem[N_CHEM] = {};
    float *dChem[N_CHEM] = {};
    float *tChem[N_CHEM] = {};
    float total[N_CHEM] = {};
};

using Diffuser = vfd::DiffuserShim<c_ctx, ChemStandIn>;

// WHWorld::initializeChemGPU's kernel part: returns the constructed Diffuser
// after the kernel context has gone.
Diffuser *init_like_reference(c_ctx *chem_cctx, ChemStandIn *chem, int nchem, const float *const *windows, int k,
                              const float *lambdas, int n_steps, std::string &err)
{
    c_ctx kernel_cctx;
    std::memset(&kernel_cctx, 0, sizeof(kernel_cctx));
    kernel_cctx.windowD = kernel_cctx.windowH = kernel_cctx.windowW = k;
    const size_t wbytes = (size_t)k * k * k * sizeof(float);
    for (int ig = 0; ig < N_GPU; ++ig) kernel_cctx.h_data[ig] = (float *)std::malloc(wbytes);
    for (int ic = N_GPU; ic < N_CHEM; ++ic) kernel_cctx.h_data[ic] = kernel_cctx.h_data[ic % N_GPU];
    const int fD = chem_cctx->FFTD, fH = chem_cctx->FFTH, fW = chem_cctx->FFTW;
    if (lambdas) {
        // this library's kernel preparation in place of prepKernel (no cuFFT)
        const vfd_status s = vfd::prepKernelSpectra(chem_cctx, lambdas, nullptr, nchem, n_steps, 0);
        if (s != VFD_OK) {
            err = std::string("prepKernelSpectra: ") + vfd_last_error(nullptr);
            for (int ig = 0; ig < N_GPU; ++ig) std::free(kernel_cctx.h_data[ig]);
            return nullptr;
        }
    }
    for (int ic = 0; ic < nchem && !lambdas; ++ic) {
        // computeKernel3D leaves chemical ic's window in the shared per-GPU buffer
        std::memcpy(kernel_cctx.h_data[ic], windows[ic], wbytes);
        if (ref_kernel_spectrum(kernel_cctx.h_data[ic], chem_cctx->KD, chem_cctx->KH, chem_cctx->KW, chem_cctx->KZ,
                                chem_cctx->KY, chem_cctx->KX, fD, fH, fW,
                                reinterpret_cast<float *>(chem_cctx->h_kernelspectrum[ic])) != 0) {
            err = std::string("reference spectrum: ") + ref_replay_error();
            for (int ig = 0; ig < N_GPU; ++ig) std::free(kernel_cctx.h_data[ig]);
            return nullptr;
        }
    }
    Diffuser *d = new Diffuser(nchem, chem_cctx, &kernel_cctx, chem);
    for (int ig = 0; ig < N_GPU; ++ig) std::free(kernel_cctx.h_data[ig]);
    std::memset(&kernel_cctx, 0xA5, sizeof(kernel_cctx));  // any later read of it is garbage
    return d;
}

}  // namespace

// nx, ny, nz: data grid; windows[ic]: k^3 floats centred at k/2; fft3: FFTW,
// FFTH, FFTD; p_in[ic]: initial pChem.  decay == NULL: `calls` x
// diffuseChemGPU(epi), out[ic] <- tChem[ic] (h_obuffs).  Otherwise `calls` x
// diffuseAndUpdateChemGPU(epi, decay) with dChem[ic] <- d_in[ic] before each
// call, out[ic] <- pChem[ic], totals[ic] <- total[ic].  lambdas != NULL: the
// spectra come from vfd::prepKernelSpectra (stencil to the power n_steps,
// this library's FFT) instead of the reference's padKernel3D + cuFFT of
// windows[ic].  Returns the shim's status (or -1 when the harness itself
// failed); err receives the message.
extern "C" int shim_harness_run(int nx, int ny, int nz, int nchem, const float *const *windows, int k,
                                const int *fft3, const float *baselines, const float *const *p_in,
                                float *const *out, int epi, int calls, const float *decay,
                                const float *const *d_in, float *totals, const float *lambdas, int n_steps,
                                char *err, int errlen)
{
    if (nchem < 1 || nchem > N_CHEM || k < 1 || (k & 1) == 0) return -1;
    const size_t V = (size_t)nx * ny * nz;
    std::string msg;
    int rc = 0;
    c_ctx *chem_cctx = new c_ctx();
    std::memset(chem_cctx, 0, sizeof(*chem_cctx));
    ChemStandIn chem;
    float pb[N_CHEM] = {};
    chem.pbaseline = pb;
    chem_cctx->DW = nx;
    chem_cctx->DH = ny;
    chem_cctx->DD = nz;
    chem_cctx->KW = chem_cctx->KH = chem_cctx->KD = k;
    // DiffusionHelper.cpp:449-455 (the isEven flags are 0 for odd windows)
    chem_cctx->KZ = chem_cctx->KY = chem_cctx->KX = k / 2;
    chem_cctx->FFTW = fft3[0];
    chem_cctx->FFTH = fft3[1];
    chem_cctx->FFTD = fft3[2];
    const size_t nspec = (size_t)fft3[2] * fft3[1] * (fft3[0] / 2 + 1);
    for (int ic = 0; ic < N_CHEM; ++ic) {
        chem_cctx->gpu_id[ic] = ic % N_GPU;
        chem_cctx->dev_id[ic] = 0;
    }
    for (int ic = 0; ic < nchem; ++ic) {
        pb[ic] = baselines[ic];
        chem.pChem[ic] = (float *)std::malloc(V * sizeof(float));
        chem.dChem[ic] = (float *)std::malloc(V * sizeof(float));
        chem.tChem[ic] = (float *)std::malloc(V * sizeof(float));
        std::memcpy(chem.pChem[ic], p_in[ic], V * sizeof(float));
        std::memset(chem.tChem[ic], 0, V * sizeof(float));
        chem_cctx->h_ibuffs[ic] = chem.pChem[ic];
        chem_cctx->h_obuffs[ic] = chem.tChem[ic];
        chem_cctx->h_kernelspectrum[ic] = (fComplex *)std::malloc(nspec * sizeof(fComplex));
    }
    Diffuser *d = init_like_reference(chem_cctx, &chem, nchem, windows, k, lambdas, n_steps, msg);
    if (!d) {
        rc = -1;
    } else {
        for (int c = 0; c < calls && d->lastStatus() == VFD_OK; ++c) {
            if (!decay) {
                d->diffuseChemGPU(epi);
            } else {
                for (int ic = 0; ic < nchem; ++ic) std::memcpy(chem.dChem[ic], d_in[ic], V * sizeof(float));
                d->diffuseAndUpdateChemGPU(epi, decay);
            }
        }
        rc = d->lastStatus();
        msg = d->lastError();
        for (int ic = 0; ic < nchem && rc == VFD_OK; ++ic) {
            std::memcpy(out[ic], decay ? chem.pChem[ic] : chem.tChem[ic], V * sizeof(float));
            if (totals) totals[ic] = chem.total[ic];
        }
        delete d;
    }
    for (int ic = 0; ic < nchem; ++ic) {
        std::free(chem.pChem[ic]);
        std::free(chem.dChem[ic]);
        std::free(chem.tChem[ic]);
        std::free(chem_cctx->h_kernelspectrum[ic]);
    }
    delete chem_cctx;
    if (err && errlen > 0) {
        std::strncpy(err, msg.c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
    return rc;
}
