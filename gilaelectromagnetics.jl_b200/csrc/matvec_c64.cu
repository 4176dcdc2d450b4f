// matvec_c64.cu -- the matvec passes instantiated for float2.
#include "matvec_impl.cuh"

namespace gila {
GILA_INST(float2)
}  // namespace gila
