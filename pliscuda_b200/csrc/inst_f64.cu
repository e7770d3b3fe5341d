// inst_f64.cu — binary64 instantiations of the step kernels.
#include "engine_kernels.cuh"

namespace plis {
Launchers pick_f64(uint32_t S) { return pick_impl<double>(S); }
}  // namespace plis
