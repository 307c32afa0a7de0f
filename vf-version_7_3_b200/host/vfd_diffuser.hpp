// vfd_diffuser.hpp -- drop-in for the reference's Diffuser class
// (src/Diffusion/Diffuser.h:24-70, Diffuser.cpp:27-470) on top of the C ABI
// in include/vfd.h.
//
// The reference constructs `new Diffuser(nBaseChem, chem_cctx, &kernel_cctx,
// WHWorldChem)` (woundHealingWorld.cpp:1046-1050) and calls
// `diffuseChemGPU(bmcx - 1)` once per tick (woundHealingWorld.cpp:2403-2407).
// DiffuserShim keeps that surface.  It is a template over the reference's
// context and chemical types so that it compiles against them unchanged; it
// reads these members (the names the reference already uses):
//   c_ctx:      DW DH DD (data dims), KW KH KD, KX KY KZ (window dims and
//               centre, chem context), h_ibuffs[ic] / h_obuffs[ic] (host
//               buffers in / out), h_data[ic] (kernel context: the extracted
//               window on the host after prepKernel), dev_id[ic]
//   WHChemical: pbaseline[ic] (baseline per patch, woundHealingWorld.cpp:969)
//
// Per call, for every chemical: h_ibuffs[ic] -> device, the reference's FFT
// convolution with its own window and the padDataConstantVF3D boundary rule
// (epiBoundary = rightWallIndex, baseline = pbaseline[ic]) -> h_obuffs[ic].
// As in the reference there is no decay here: WHChemical::update applies
// cytokineDecay afterwards (WHChemical.cpp:420-450).
//
// Differences that are intended: one device (the reference splits chemicals
// over two GPUs by ic % 2, DiffusionHelper.cpp:386-392); FFT plans, buffers
// and kernel spectra live for the lifetime of the object (the reference
// re-creates plans every tick, Diffuser.cpp:266-275, and allocates its
// padded buffers inside every fftDiffuse3D call, Diffusion.cu:1686-1687);
// failures are reported through lastStatus()/lastError() instead of exit().
#pragma once

#include <algorithm>
#include <string>
#include <vector>

#include "vfd.h"

namespace vfd {

template <class CCtx, class Chem>
class DiffuserShim {
  public:
    DiffuserShim() : nBaseChem_(8), chem_(nullptr), kern_(nullptr), whChem_(nullptr) {}
    DiffuserShim(int nBaseChem, CCtx *cc, CCtx *kc, Chem *WHWorldChem)
        : nBaseChem_(nBaseChem), chem_(cc), kern_(kc), whChem_(WHWorldChem)
    {
    }
    virtual ~DiffuserShim()
    {
        if (world_) vfd_world_destroy(world_);
    }
    DiffuserShim(const DiffuserShim &) = delete;
    DiffuserShim &operator=(const DiffuserShim &) = delete;

    // Diffuser::diffuseChemGPU(int rightWallIndex), Diffuser.cpp:221-470.
    void diffuseChemGPU(int rightWallIndex)
    {
        status_ = VFD_OK;
        if (!chem_ || !kern_ || !whChem_) {
            fail(VFD_ERR_INVALID_ARG, "Diffuser constructed without contexts");
            return;
        }
        if (!world_ || rightWallIndex != epi_) {
            if (world_) vfd_world_destroy(world_);
            world_ = nullptr;
            if (!build(rightWallIndex)) return;
        }
        std::vector<const float *> in(nBaseChem_);
        std::vector<float *> out(nBaseChem_);
        for (int ic = 0; ic < nBaseChem_; ++ic) {
            in[ic] = chem_->h_ibuffs[ic];
            out[ic] = chem_->h_obuffs[ic];
        }
        vfd_status s = vfd_diffuse_host(world_, in.data(), out.data(), 1);
        if (s != VFD_OK) fail(s, vfd_last_error(world_));
        ++iter_;
    }

    vfd_status lastStatus() const { return status_; }
    const std::string &lastError() const { return err_; }
    int iterations() const { return iter_; }

  private:
    bool build(int epi)
    {
        const int nx = chem_->DW, ny = chem_->DH, nz = chem_->DD;
        const int kw = chem_->KW, kh = chem_->KH, kd = chem_->KD;
        const int cx = chem_->KX, cy = chem_->KY, cz = chem_->KZ;
        std::vector<vfd_field_params> p(nBaseChem_);
        for (int ic = 0; ic < nBaseChem_; ++ic) {
            vfd_field_params &f = p[ic];
            for (int a = 0; a < 3; ++a) f.sigma[a] = 1.0;  // replaced by the window below
            f.radius[0] = std::max(cx, kw - 1 - cx);
            f.radius[1] = std::max(cy, kh - 1 - cy);
            f.radius[2] = std::max(cz, kd - 1 - cz);
            for (int a = 0; a < 3; ++a) f.radius[a] = std::max(f.radius[a], 1);
            f.decay_rate = 0.0;
            f.baseline = whChem_->pbaseline[ic];
        }
        vfd_world_desc d;
        d.nx = nx;
        d.ny = ny;
        d.nz = nz;
        d.n_fields = nBaseChem_;
        d.fields = p.data();
        d.pad_mode = VFD_PAD_CONSTANT_VF;
        d.epi_boundary = epi;
        d.fft[0] = d.fft[1] = d.fft[2] = 0;
        d.method = VFD_METHOD_FFT3D;
        vfd_status s = vfd_world_create(&d, chem_->dev_id[0], &world_);
        if (s != VFD_OK) {
            fail(s, vfd_last_error(nullptr));
            world_ = nullptr;
            return false;
        }
        for (int ic = 0; ic < nBaseChem_; ++ic) {
            s = vfd_set_window(world_, ic, kern_->h_data[ic], kw, kh, kd, cx, cy, cz);
            if (s != VFD_OK) {
                fail(s, vfd_last_error(world_));
                vfd_world_destroy(world_);
                world_ = nullptr;
                return false;
            }
        }
        epi_ = epi;
        return true;
    }

    void fail(vfd_status s, const char *msg)
    {
        status_ = s;
        err_ = msg ? msg : "";
    }

    int nBaseChem_;
    CCtx *chem_;
    CCtx *kern_;
    Chem *whChem_;
    vfd_world *world_ = nullptr;
    int epi_ = -1;
    int iter_ = 0;
    vfd_status status_ = VFD_OK;
    std::string err_;
};

}  // namespace vfd
