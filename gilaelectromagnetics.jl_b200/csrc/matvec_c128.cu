// matvec_c128.cu -- the matvec passes instantiated for double2.
#include "matvec_impl.cuh"

namespace gila {
GILA_INST(double2)
}  // namespace gila
