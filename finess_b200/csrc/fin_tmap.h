// Host-side TMA tensor maps of the FP64 state buffers (one per buffer and
// box shape), shared by the single-problem solver and the batch.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>

namespace fin {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// Map of one state buffer (5 planes of mx x my FP64 values, plane pitch
// `plane` elements) as a 3D tensor (j, i, component): row pitch my*8 bytes,
// component pitch plane*8 bytes (both multiples of 16 when my is even; odd
// my gets no map), box box_j x box_i x 5.
inline bool make_state_map(CUtensorMap* m, double* base, int mx, int my, size_t plane, int box_j, int box_i)
{
    EncodeTiledFn fn = encode_tiled();
    if (!fn || (my & 1)) return false;
    const cuuint64_t dims[3] = {cuuint64_t(my), cuuint64_t(mx), cuuint64_t(5)};
    const cuuint64_t strides[2] = {cuuint64_t(my) * 8, cuuint64_t(plane) * 8};
    const cuuint32_t box[3] = {cuuint32_t(box_j), cuuint32_t(box_i), cuuint32_t(5)};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

}  // namespace fin
