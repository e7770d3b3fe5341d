// batch_f32.cu — binary32 instantiations of the persistent batch kernel.
#include "batch_kernels.cuh"

namespace plis {
BatchLaunch batch_pick_f32(uint32_t S) { return batch_pick_impl<float>(S); }
}  // namespace plis
