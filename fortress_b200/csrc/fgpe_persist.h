// fgpe_persist.h -- host side of the persistent batch kernel: its variants
// (launch shapes and y radix plans the autotuner chooses among) and the
// per-(precision, spin) launchers, compiled in fgpe_persist_<t><spin>.cu.
#pragma once
#include <cuda_runtime.h>

#include "fgpe_persist.cuh"

namespace fgpe {

struct PersistShape {
    int th;    // threads per block
    int rn;    // values per row tile (R rows of N, R a power of two)
    int txb;   // bytes of x per column tile row
    int pv;    // radix plan of the y lines (cplan)
};
constexpr int kPersistVariants = 5;
constexpr PersistShape kPersistShapes[kPersistVariants] = {
    {256, 512, 32, 0},    // base shape
    {256, 512, 32, 1},    // radix 4*4 in place of 8*2 on the y lines (128, 384)
    {256, 1024, 32, 0},   // twice the rows per row tile
    {128, 256, 16, 0},    // small blocks: more of them per SM
    {256, 1024, 32, 3},   // tall row tiles, radix-16 y lines (128, 256, 384)
};

// Set the variant's shared-memory limit and report its resident blocks per SM
// for smem bytes of dynamic shared memory (0 blocks: the shape does not fit).
template <typename T, int MS> cudaError_t persist_prepare(int variant, size_t smem, int* blocks_per_sm);
template <typename T, int MS>
cudaError_t persist_launch(int variant, const PersistArgs& a, int grid, size_t smem, cudaStream_t st);

#define FGPE_PERSIST_EXTERN(T, MS)                                                                  \
    extern template cudaError_t persist_prepare<T, MS>(int, size_t, int*);                          \
    extern template cudaError_t persist_launch<T, MS>(int, const PersistArgs&, int, size_t, cudaStream_t);
FGPE_PERSIST_EXTERN(float, 3)
FGPE_PERSIST_EXTERN(float, 5)
FGPE_PERSIST_EXTERN(double, 3)
FGPE_PERSIST_EXTERN(double, 5)
#undef FGPE_PERSIST_EXTERN

}  // namespace fgpe
