// ifc_fused2d_impl.cuh -- host-side launch sequences of the fused 2D kernels.
#pragma once

namespace ifc {

template <typename T>
void Engine<T>::enq_fused_mom()
{
}

template <typename T>
void Engine<T>::enq_fused_pcorr()
{
}

}  // namespace ifc
