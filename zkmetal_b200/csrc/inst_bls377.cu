// Explicit instantiation of the Bls377 device pipeline (kernels and launches).
#include "engine_impl.cuh"

namespace zkmsm {
ZKMSM_ENGINE_TEMPLATES(, Bls377)
}  // namespace zkmsm
