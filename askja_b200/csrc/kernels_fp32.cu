// FP32 kernel table: links and momenta stored and updated in FP32 (complex),
// FP32 accumulation in the force and exponential, reunitarisation after each
// link update; every reduction still accumulates in FP64.
#include "kernels.cuh"

namespace askja {

const KernelSet kernels_fp32 = detail::make_set<float>();

}  // namespace askja
