// vfd_tma.cu -- host side of the TMA staging (vfd_tma.h).
#include <cudaTypedefs.h>

#include <mutex>

#include "vfd_tma.h"

namespace vfd {

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static void lookup_encode()
{
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
}

bool tma_available()
{
    std::call_once(g_encode_once, lookup_encode);
    return g_encode != nullptr;
}

bool tma_encode_3d(CUtensorMap *m, const float *base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1,
                   uint64_t s2, uint32_t b0, uint32_t b1, uint32_t b2)
{
    if (!tma_available() || !m || !base) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (s1 & 15) != 0 || (s2 & 15) != 0) return false;
    if ((b0 * 4) % 16 != 0 || b0 < 1 || b1 < 1 || b2 < 1 || b0 > 256 || b1 > 256 || b2 > 256) return false;
    if (d0 < 1 || d1 < 1 || d2 < 1 || d0 >= (1ull << 32) || d1 >= (1ull << 32) || d2 >= (1ull << 32)) return false;
    if (s1 >= (1ull << 40) || s2 >= (1ull << 40)) return false;
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {s1, s2};
    const cuuint32_t box[3] = {b0, b1, b2};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace vfd
