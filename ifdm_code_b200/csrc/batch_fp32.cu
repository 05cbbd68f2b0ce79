// batch_fp32.cu -- batch kernels of the FP32 precision mode (see batch_launch.cuh).
#include "batch_launch.cuh"

namespace ifdm {

const BatchKernels &batch_kernels_fp32() { return BatchTable<float, float>::table(); }

}  // namespace ifdm
