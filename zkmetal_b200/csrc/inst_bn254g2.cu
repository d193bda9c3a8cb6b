// Explicit instantiation of the Bn254G2 device pipeline (kernels and launches).
#include "engine_impl.cuh"

namespace zkmsm {
ZKMSM_ENGINE_TEMPLATES(, Bn254G2)
}  // namespace zkmsm
