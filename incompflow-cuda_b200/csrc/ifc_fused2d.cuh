// ifc_fused2d.cuh -- fused, temporally blocked 2D kernels (assembly + several
// red-black sweeps per pass through HBM).
#pragma once

#include "ifc_kernels.cuh"

namespace ifc {

template <typename T>
bool fused2d_supported(const Geo<T> &)
{
    return false;
}

}  // namespace ifc
