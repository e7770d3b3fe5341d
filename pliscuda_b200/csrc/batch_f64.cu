// batch_f64.cu — binary64 instantiations of the persistent batch kernel.
#include "batch_kernels.cuh"

namespace plis {
BatchLaunch batch_pick_f64(uint32_t S) { return batch_pick_impl<double>(S); }
}  // namespace plis
