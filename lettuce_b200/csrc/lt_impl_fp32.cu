// Kernel instantiation for the fp32 link storage (float, 3 stored rows).
#include "lt_impl.cuh"

namespace lt {
const Backend* backend_fp32()
{
    static const BackendImpl<float, 3> impl;
    return &impl;
}
} // namespace lt
