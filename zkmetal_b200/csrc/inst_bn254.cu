// Explicit instantiation of the Bn254 device pipeline (kernels and launches).
#include "engine_impl.cuh"

namespace zkmsm {
ZKMSM_ENGINE_TEMPLATES(, Bn254)
}  // namespace zkmsm
