// Persistent batch kernel, float complex, spin 2 (fgpe_persist.cuh).
#include "fgpe_persist_impl.cuh"

namespace fgpe {
FGPE_PERSIST_INSTANTIATE(float, 5)
}  // namespace fgpe
