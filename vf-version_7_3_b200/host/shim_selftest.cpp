// shim_selftest.cpp -- builds DiffuserShim against stand-in context types that
// carry the reference's member names (c_ctx / WHChemical), so tests can drive
// the drop-in exactly the way WHWorld drives the reference's Diffuser.
#include <cstring>

#include "vfd_diffuser.hpp"

namespace {
constexpr int kMaxChem = 8;  // N_CHEM of the reference (convolutionFFT_common.h:295)

struct TestCtx {
    int DW, DH, DD;
    int KW, KH, KD;
    int KX, KY, KZ;
    float *h_ibuffs[kMaxChem];
    float *h_obuffs[kMaxChem];
    float *h_data[kMaxChem];
    int dev_id[kMaxChem];
};

struct TestChem {
    float *pbaseline;
};
}  // namespace

extern "C" int vfd_shim_selftest(int nx, int ny, int nz, int nchem, float *const *in, float *const *out,
                                 float *const *windows, int kw, int kh, int kd, float *baselines, int epi,
                                 int calls, char *err, int errlen)
{
    if (nchem < 1 || nchem > kMaxChem) return VFD_ERR_INVALID_ARG;
    TestCtx chem, kern;
    std::memset(&chem, 0, sizeof(chem));
    std::memset(&kern, 0, sizeof(kern));
    chem.DW = nx;
    chem.DH = ny;
    chem.DD = nz;
    chem.KW = kw;
    chem.KH = kh;
    chem.KD = kd;
    chem.KX = kw / 2;
    chem.KY = kh / 2;
    chem.KZ = kd / 2;
    for (int ic = 0; ic < nchem; ++ic) {
        chem.h_ibuffs[ic] = in[ic];
        chem.h_obuffs[ic] = out[ic];
        kern.h_data[ic] = windows[ic];
        chem.dev_id[ic] = 0;
    }
    TestChem wc{baselines};
    vfd::DiffuserShim<TestCtx, TestChem> d(nchem, &chem, &kern, &wc);
    for (int c = 0; c < calls; ++c) {
        d.diffuseChemGPU(epi);
        if (d.lastStatus() != VFD_OK) break;
    }
    if (err && errlen > 0) {
        std::strncpy(err, d.lastError().c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
    return d.lastStatus();
}
