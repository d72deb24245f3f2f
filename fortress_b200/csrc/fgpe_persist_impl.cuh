// fgpe_persist_impl.cuh -- definitions of the persistent-kernel launchers,
// included by one translation unit per (precision, spin) so that the four
// instantiations compile in parallel.
#pragma once
#include "fgpe_persist.h"

namespace fgpe {

template <typename T, int MS, int V> constexpr auto persist_kernel() {
    constexpr PersistShape s = kPersistShapes[V];
    return k_persist<T, MS, s.th, s.rn, s.txb, s.pv>;
}

template <typename T, int MS, int V> cudaError_t persist_prepare_v(size_t smem, int* blocks) {
    constexpr auto k = persist_kernel<T, MS, V>();
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k, kPersistShapes[V].th, smem);
}

template <typename T, int MS> cudaError_t persist_prepare(int variant, size_t smem, int* blocks_per_sm) {
    *blocks_per_sm = 0;
    switch (variant) {
        case 0: return persist_prepare_v<T, MS, 0>(smem, blocks_per_sm);
        case 1: return persist_prepare_v<T, MS, 1>(smem, blocks_per_sm);
        case 2: return persist_prepare_v<T, MS, 2>(smem, blocks_per_sm);
        case 3: return persist_prepare_v<T, MS, 3>(smem, blocks_per_sm);
        case 4: return persist_prepare_v<T, MS, 4>(smem, blocks_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T, int MS>
cudaError_t persist_launch(int variant, const PersistArgs& a, int grid, size_t smem, cudaStream_t st) {
    switch (variant) {
#define PL(V) \
        case V: persist_kernel<T, MS, V>()<<<grid, kPersistShapes[V].th, smem, st>>>(a); break;
        PL(0) PL(1) PL(2) PL(3) PL(4)
#undef PL
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

#define FGPE_PERSIST_INSTANTIATE(T, MS)                                                  \
    template cudaError_t persist_prepare<T, MS>(int, size_t, int*);                      \
    template cudaError_t persist_launch<T, MS>(int, const PersistArgs&, int, size_t, cudaStream_t);

}  // namespace fgpe
