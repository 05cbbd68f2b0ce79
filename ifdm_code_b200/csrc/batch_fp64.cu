// batch_fp64.cu -- batch kernels of the FP64 precision mode (see batch_launch.cuh).
#include "batch_launch.cuh"

namespace ifdm {

const BatchKernels &batch_kernels_fp64() { return BatchTable<double, double>::table(); }

}  // namespace ifdm
