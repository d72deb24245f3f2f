// Persistent batch kernel, double complex, spin 2 (fgpe_persist.cuh).
#include "fgpe_persist_impl.cuh"

namespace fgpe {
FGPE_PERSIST_INSTANTIATE(double, 5)
}  // namespace fgpe
