// ib_tma.cu -- host-side tensor-map encoding for the TMA-fed kernels.
//
// cuTensorMapEncodeTiled is a driver API function; it is looked up once through the runtime
// (cudaGetDriverEntryPoint), so the library links only the CUDA runtime.
#include "ib_internal.cuh"
#include "ib_tma.cuh"

#include <cudaTypedefs.h>
#include <mutex>

namespace ib {

static PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

int encode_tmap_f64(CUtensorMap *map, void *base, int rank, const uint64_t *dims, const uint64_t *strides_bytes,
                    const uint32_t *box)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encoder();
    if (!fn) return IB_ERROR_NOIMPLEMENT;
    if (rank < 1 || rank > 5 || ((uintptr_t)base & 15) != 0) return IB_ERROR_NOIMPLEMENT;
    cuuint64_t gd[5], gs[4];
    cuuint32_t bx[5], es[5];
    for (int i = 0; i < rank; i++) {
        gd[i] = dims[i];
        bx[i] = box[i];
        es[i] = 1;
        if (box[i] == 0 || box[i] > 256 || box[i] > dims[i]) return IB_ERROR_NOIMPLEMENT;
    }
    if ((box[0] * 8) % 16 != 0) return IB_ERROR_NOIMPLEMENT;
    for (int i = 0; i + 1 < rank; i++) {
        gs[i] = strides_bytes[i];
        if (gs[i] % 16 != 0) return IB_ERROR_NOIMPLEMENT;
    }
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, base, gd, gs, bx, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? IB_SUCCESSFUL : IB_ERROR_NOIMPLEMENT;
}

}  // namespace ib
