// Kernel instantiation for the fp32_12 link storage (float, 2 stored rows).
#include "lt_impl.cuh"

namespace lt {
const Backend* backend_fp32_12()
{
    static const BackendImpl<float, 2> impl;
    return &impl;
}
} // namespace lt
