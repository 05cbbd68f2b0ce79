// batch_mixed.cu -- batch kernels of the mixed precision mode (see batch_launch.cuh).
#include "batch_launch.cuh"

namespace ifdm {

const BatchKernels &batch_kernels_mixed() { return BatchTable<float, double>::table(); }

}  // namespace ifdm
