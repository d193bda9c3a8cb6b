// Explicit instantiation of the Bls381 device pipeline (kernels and launches).
#include "engine_impl.cuh"

namespace zkmsm {
ZKMSM_ENGINE_TEMPLATES(, Bls381)
}  // namespace zkmsm
