// batch_f32.cu — binary32 instantiations of the persistent batch kernel.
#include "batch_kernels.cuh"

namespace plis {
BatchLaunch batch_pick_f32(uint32_t S, bool learned, bool small) {
  return learned ? batch_pick_impl<float, true>(S, small) : batch_pick_impl<float, false>(S, small);
}
}  // namespace plis
