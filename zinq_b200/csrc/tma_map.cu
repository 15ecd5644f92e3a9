// tma_map.cu -- host-side encoding of the TMA tensor maps (tma.cuh).
//
// cuTensorMapEncodeTiled is a driver API call; the runtime hands out its entry point, so the
// library keeps linking only the static CUDA runtime.
#include <cudaTypedefs.h>

#include <mutex>

#include "tma.cuh"

namespace zqd {

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

int encode_map_3d(CUtensorMap* map, void* base, const uint64_t dims[3], uint64_t stride1, uint64_t stride2,
                  const uint32_t box[3], int l2promo, bool swizzle128) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return (int)cudaErrorNotSupported;
    // the rules cuTensorMapEncodeTiled checks, checked here too so that a bad shape is a host error
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (stride1 & 15) || (stride2 & 15) || (box[0] * 8u) % 16u ||
        box[0] > 256 || box[1] > 256 || box[2] > 256 || (swizzle128 && box[0] * 8u != 128u))
        return (int)cudaErrorInvalidValue;
    const cuuint64_t gdim[3] = {dims[0], dims[1], dims[2]};
    const cuuint64_t gstr[2] = {stride1, stride2};
    const cuuint32_t bdim[3] = {box[0], box[1], box[2]};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapL2promotion promo = l2promo >= 256   ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
                                         : l2promo >= 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B
                                         : l2promo >= 64  ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
                                                          : CU_TENSOR_MAP_L2_PROMOTION_NONE;
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, base, gdim, gstr, bdim, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE,
                          swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE, promo,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

} // namespace zqd
