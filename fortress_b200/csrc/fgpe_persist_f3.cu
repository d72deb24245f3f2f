// Persistent batch kernel, float complex, spin 1 (fgpe_persist.cuh).
#include "fgpe_persist_impl.cuh"

namespace fgpe {
FGPE_PERSIST_INSTANTIATE(float, 3)
}  // namespace fgpe
