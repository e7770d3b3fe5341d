// batch_f64.cu — binary64 instantiations of the persistent batch kernel.
#include "batch_kernels.cuh"

namespace plis {
BatchLaunch batch_pick_f64(uint32_t S, bool learned, bool small) {
  return learned ? batch_pick_impl<double, true>(S, small) : batch_pick_impl<double, false>(S, small);
}
}  // namespace plis
