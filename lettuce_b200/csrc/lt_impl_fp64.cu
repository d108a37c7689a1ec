// Kernel instantiation for the fp64 link storage (double, 3 stored rows).
#include "lt_impl.cuh"

namespace lt {
const Backend* backend_fp64()
{
    static const BackendImpl<double, 3> impl;
    return &impl;
}
} // namespace lt
