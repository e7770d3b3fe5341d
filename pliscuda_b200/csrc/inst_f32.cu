// inst_f32.cu — binary32 instantiations of the step kernels.
#include "engine_kernels.cuh"

namespace plis {
Launchers pick_f32(uint32_t S) { return pick_impl<float>(S); }
}  // namespace plis
