// vfd_diffuser.hpp -- drop-in for the reference's Diffuser class
// (src/Diffusion/Diffuser.h:24-70, Diffuser.cpp:27-470) on top of the C ABI
// in include/vfd.h.
//
// The reference constructs `new Diffuser(nBaseChem, chem_cctx, &kernel_cctx,
// WHWorldChem)` (woundHealingWorld.cpp:1046-1050) and calls
// `diffuseChemGPU(bmcx - 1)` once per tick (woundHealingWorld.cpp:2403-2407).
// DiffuserShim keeps that surface.  It is a template over the reference's
// context and chemical types so that it compiles against them unchanged.
//
// Everything the shim needs from the contexts is captured in the
// constructor.  The kernel context is never read: in the reference it is a
// local of WHWorld::initializeChemGPU (woundHealingWorld.cpp:1010) whose
// buffers are freed right after construction (deallocConvCtxBuffers,
// :1038) and whose h_data holds one window per GPU, overwritten chemical by
// chemical (DiffusionHelper.cpp:218-247).  The kernel of chemical ic lives
// on only as chem_cctx->h_kernelspectrum[ic], one buffer per chemical
// (DiffusionHelper.cpp:556-592), filled by computeKernelSpectrum3D
// (Diffusion.cu:1540-1610): the unscaled R2C spectrum of the wrapped window
// on the FFTD x FFTH x (FFTW/2+1) grid.  The reference sizes that grid to at
// least n + window - 1 per axis (DiffusionHelper.cpp:410-437), so its
// circular convolution is the linear one, and any grid that also avoids
// wrap-around gives the same result.  The constructor therefore recovers
// each chemical's window from its spectrum (vfd_spectrum_window, this
// library's inverse transform) and runs on the cheapest 7-smooth grid of
// at least n + half-width points per axis (4.3x fewer points than the
// power-of-two grid at 512x256x384).  With the environment variable
// VFD_SHIM_REFERENCE_GRID=1 it keeps the reference's grid and uses the
// spectra as they are (vfd_set_spectrum).
//
// Members read, all at construction (the names the reference already uses):
//   c_ctx:      DW DH DD (data dims), FFTW FFTH FFTD (FFT grid), KW KH KD,
//               KX KY KZ (window dims and centre), h_kernelspectrum[ic],
//               dev_id[ic]
//   WHChemical: pbaseline[ic] (baseline per patch, woundHealingWorld.cpp:970-975)
// and per call: c_ctx h_ibuffs[ic] / h_obuffs[ic] (host buffers in / out,
// DiffusionHelper.cpp:529-531), and for diffuseAndUpdateChemGPU the
// WHChemical members pChem[ic], dChem[ic] and total[ic].
//
// Chemicals are split over devices by dev_id[ic] like the reference
// (ic % N_GPU, DiffusionHelper.cpp:386-392): one world per distinct device,
// each driven from its own host thread during a call.
//
// Differences that are intended: FFT plans, buffers and kernel spectra live
// for the lifetime of the object (the reference re-creates plans every tick,
// Diffuser.cpp:266-275, and allocates its padded buffers inside every
// fftDiffuse3D call, Diffusion.cu:1686-1687); failures are reported through
// lastStatus()/lastError() instead of exit().
#pragma once

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "vfd.h"

namespace vfd {

template <class CCtx, class Chem>
class DiffuserShim {
  public:
    DiffuserShim() : nBaseChem_(8), chem_(nullptr), whChem_(nullptr) {}
    DiffuserShim(int nBaseChem, CCtx *cc, CCtx *kc, Chem *WHWorldChem)
        : nBaseChem_(nBaseChem), chem_(cc), whChem_(WHWorldChem)
    {
        (void)kc;  // see the header comment: dead after construction in the reference
        build();
    }
    virtual ~DiffuserShim()
    {
        for (auto &g : groups_)
            if (g.world) vfd_world_destroy(g.world);
    }
    DiffuserShim(const DiffuserShim &) = delete;
    DiffuserShim &operator=(const DiffuserShim &) = delete;

    // Diffuser::diffuseChemGPU(int rightWallIndex), Diffuser.cpp:221-470:
    // h_ibuffs[ic] -> device, one FFT convolution with the chemical's stored
    // spectrum and the padDataConstantVF3D rule (epiBoundary = rightWallIndex,
    // baseline pbaseline[ic]) -> h_obuffs[ic].  No decay: WHChemical::update
    // applies cytokineDecay afterwards, as in the reference.
    void diffuseChemGPU(int rightWallIndex) { run<false>(rightWallIndex, nullptr); }

    // diffuseChemGPU followed by WHChemical::updateChemGPU
    // (WHChemical.cpp:420-450) with the update done on the device:
    // pChem[ic] = dChem[ic] + t * cytokineDecay[ic], dChem[ic] = 0 and
    // total[ic] = sum(pChem[ic]) (FP64, stored as float like the reference),
    // without the host sweep over tChem.  h_obuffs (tChem) is not written.
    // The attractant gradients of WHChemical::update need the ECM fragment
    // counts and stay with the caller (vfd_update_gradients computes them on
    // the device from device arrays).
    void diffuseAndUpdateChemGPU(int rightWallIndex, const float *cytokineDecay)
    {
        if (!cytokineDecay) {
            fail(VFD_ERR_INVALID_ARG, "cytokineDecay is NULL");
            return;
        }
        run<true>(rightWallIndex, cytokineDecay);
    }

    vfd_status lastStatus() const { return status_; }
    const std::string &lastError() const { return err_; }
    int iterations() const { return iter_; }

  private:
    struct Group {
        int device = 0;
        std::vector<int> chems;  // chemical indices of this device, in order
        vfd_world *world = nullptr;
        vfd_status status = VFD_OK;
        std::string err;
    };

    void build()
    {
        status_ = VFD_OK;
        if (!chem_ || !whChem_ || nBaseChem_ < 1) {
            fail(VFD_ERR_INVALID_ARG, "Diffuser constructed without contexts");
            return;
        }
        for (int ic = 0; ic < nBaseChem_; ++ic) {
            const int dev = chem_->dev_id[ic];
            auto it = std::find_if(groups_.begin(), groups_.end(), [&](const Group &g) { return g.device == dev; });
            if (it == groups_.end()) {
                groups_.emplace_back();
                groups_.back().device = dev;
                it = groups_.end() - 1;
            }
            it->chems.push_back(ic);
        }
        const int nx = chem_->DW, ny = chem_->DH, nz = chem_->DD;
        // window half-widths around the centre (padKernel3D wraps the centre to index 0)
        const int rx = std::max(1, std::max((int)chem_->KX, (int)chem_->KW - 1 - (int)chem_->KX));
        const int ry = std::max(1, std::max((int)chem_->KY, (int)chem_->KH - 1 - (int)chem_->KY));
        const int rz = std::max(1, std::max((int)chem_->KZ, (int)chem_->KD - 1 - (int)chem_->KZ));
        for (auto &g : groups_) {
            std::vector<vfd_field_params> p(g.chems.size());
            for (size_t k = 0; k < g.chems.size(); ++k) {
                vfd_field_params &f = p[k];
                for (int a = 0; a < 3; ++a) f.sigma[a] = 1.0;  // unused: the stored spectrum replaces it
                f.radius[0] = rx;
                f.radius[1] = ry;
                f.radius[2] = rz;
                f.decay_rate = 0.0;
                f.baseline = whChem_->pbaseline ? whChem_->pbaseline[g.chems[k]] : 0.0f;
            }
            const char *keep = std::getenv("VFD_SHIM_REFERENCE_GRID");
            const bool ref_grid = keep && keep[0] == '1';
            vfd_world_desc d;
            d.nx = nx;
            d.ny = ny;
            d.nz = nz;
            d.n_fields = (int)g.chems.size();
            d.fields = p.data();
            d.pad_mode = VFD_PAD_CONSTANT_VF;
            d.epi_boundary = nx;  // replaced by rightWallIndex on every call
            d.fft[0] = ref_grid ? chem_->FFTW : 0;
            d.fft[1] = ref_grid ? chem_->FFTH : 0;
            d.fft[2] = ref_grid ? chem_->FFTD : 0;
            d.method = VFD_METHOD_FFT3D;
            vfd_status s = vfd_world_create(&d, g.device, &g.world);
            if (s != VFD_OK) {
                g.world = nullptr;
                fail(s, vfd_last_error(nullptr));
                return;
            }
            const int kw = chem_->KW, kh = chem_->KH, kd = chem_->KD;
            std::vector<float> win(ref_grid ? 0 : (size_t)kw * kh * kd);
            for (size_t k = 0; k < g.chems.size(); ++k) {
                const int ic = g.chems[k];
                const float *spec = reinterpret_cast<const float *>(chem_->h_kernelspectrum[ic]);
                if (ref_grid) {
                    s = vfd_set_spectrum(g.world, (int)k, spec, chem_->FFTW, chem_->FFTH, chem_->FFTD);
                } else {
                    s = vfd_spectrum_window(spec, chem_->FFTW, chem_->FFTH, chem_->FFTD, kw, kh, kd, chem_->KX,
                                            chem_->KY, chem_->KZ, win.data(), g.device);
                    if (s == VFD_OK)
                        s = vfd_set_window(g.world, (int)k, win.data(), kw, kh, kd, chem_->KX, chem_->KY, chem_->KZ);
                }
                if (s != VFD_OK) {
                    fail(s, vfd_last_error(ref_grid ? g.world : nullptr));
                    if (std::string(err_).empty()) fail(s, vfd_last_error(g.world));
                    return;
                }
            }
        }
        built_ = true;
    }

    // One call on every device group, each from its own host thread.
    // UPD: the device-side update (reads the WHChemical members pChem, dChem
    // and total, so only instantiated when diffuseAndUpdateChemGPU is used).
    template <bool UPD>
    void run(int epi, const float *decay)
    {
        if (!built_) {
            if (status_ == VFD_OK) fail(VFD_ERR_INVALID_ARG, "Diffuser constructed without contexts");
            return;
        }
        status_ = VFD_OK;
        err_.clear();
        auto one = [&](Group &g) {
            const size_t n = g.chems.size();
            std::vector<float> base(n);
            for (size_t k = 0; k < n; ++k) base[k] = whChem_->pbaseline ? whChem_->pbaseline[g.chems[k]] : 0.0f;
            g.status = vfd_set_boundary(g.world, epi, base.data());
            if constexpr (!UPD) {
                if (g.status == VFD_OK) {
                    std::vector<const float *> in(n);
                    std::vector<float *> out(n);
                    for (size_t k = 0; k < n; ++k) {
                        in[k] = chem_->h_ibuffs[g.chems[k]];
                        out[k] = chem_->h_obuffs[g.chems[k]];
                    }
                    g.status = vfd_diffuse_host(g.world, in.data(), out.data(), 1);
                }
            } else if (g.status == VFD_OK) {
                std::vector<float *> p(n), dd(n);
                std::vector<float> dec(n);
                for (size_t k = 0; k < n; ++k) {
                    p[k] = whChem_->pChem[g.chems[k]];
                    dd[k] = whChem_->dChem[g.chems[k]];
                    dec[k] = decay[g.chems[k]];
                }
                g.status = vfd_diffuse_update_host(g.world, p.data(), dd.data(), dec.data(), 1);
                if (g.status == VFD_OK) {
                    std::vector<vfd_mass> m(n);
                    g.status = vfd_read_mass(g.world, m.data(), nullptr);
                    if (g.status == VFD_OK)
                        for (size_t k = 0; k < n; ++k) whChem_->total[g.chems[k]] = (float)m[k].total;
                }
            }
            g.err = g.status == VFD_OK ? std::string() : std::string(vfd_last_error(g.world));
        };
        if (groups_.size() == 1) {
            one(groups_[0]);
        } else {
            std::vector<std::thread> th;
            for (auto &g : groups_) th.emplace_back(one, std::ref(g));
            for (auto &t : th) t.join();
        }
        for (auto &g : groups_)
            if (g.status != VFD_OK) {
                fail(g.status, g.err.c_str());
                break;
            }
        ++iter_;
    }

    void fail(vfd_status s, const char *msg)
    {
        status_ = s;
        err_ = msg ? msg : "";
    }

    int nBaseChem_;
    CCtx *chem_;
    Chem *whChem_;
    std::vector<Group> groups_;
    bool built_ = false;
    int iter_ = 0;
    vfd_status status_ = VFD_OK;
    std::string err_;
};

// cuFFT-free replacement for the reference's kernel preparation
// (diffusion_helper::prepKernel -> computeKernel3DBatch / computeKernel3D /
// computeKernelSpectrum3D, DiffusionHelper.cpp:695-720, Diffusion.cu:988-1619):
// for every chemical ic, the window of the 7-point stencil (centre
// 1 - 6 lambda - gamma_dt, arms lambda) raised to nSteps, of the chemical
// context's window size (KW x KH x KD, centre KX, KY, KZ), computed on the
// device (vfd_stencil_window), and its spectrum on the chemical FFT grid
// (vfd_window_spectrum) written to chem->h_kernelspectrum[ic].  The
// reference's human-VF setting: nSteps = niter * (kernelRadius - 1) = 894
// (DiffusionHelper.cpp:48-100), gamma_dt = gamma[ic] * dt (0 there).  Call it
// where WHWorld::initializeChemGPU calls prepKernel; the Diffuser is then
// constructed as before.  Needs a cubic window (KW = KH = KD, centred).
template <class CCtx>
vfd_status prepKernelSpectra(CCtx *chem, const float *lambda, const float *gamma_dt, int nChem, int nSteps,
                             int device)
{
    if (!chem || !lambda || nChem < 1 || nSteps < 0) return VFD_ERR_INVALID_ARG;
    const int k = chem->KW;
    if (k < 1 || chem->KH != k || chem->KD != k || chem->KX != k / 2 || chem->KY != k / 2 || chem->KZ != k / 2)
        return VFD_ERR_NOT_SUPPORTED;
    const int R = k / 2;
    std::vector<float> win((size_t)k * k * k);
    for (int ic = 0; ic < nChem; ++ic) {
        vfd_status s = vfd_stencil_window(lambda[ic], gamma_dt ? gamma_dt[ic] : 0.0, nSteps, R, win.data(), device);
        if (s != VFD_OK) return s;
        s = vfd_window_spectrum(win.data(), k, k, k, R, R, R, chem->FFTW, chem->FFTH, chem->FFTD,
                                reinterpret_cast<float *>(chem->h_kernelspectrum[ic]), device);
        if (s != VFD_OK) return s;
    }
    return VFD_OK;
}

}  // namespace vfd
