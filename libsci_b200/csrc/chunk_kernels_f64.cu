// chunk_kernels_f64.cu -- the generic (double) chunk interpreter, compiled ahead of time.
#include "chunk_kernel.cuh"

namespace sci_cuda {

    const void *generic_chunk_kernel_f64(int mode) {
        switch (mode) {
        case kEvaluate: return reinterpret_cast<const void *>(&chunk_stream<double, Dynamic, kEvaluate>);
        case kReduce: return reinterpret_cast<const void *>(&chunk_stream<double, Dynamic, kReduce>);
        default: return reinterpret_cast<const void *>(&chunk_stream<double, Dynamic, kDot>);
        }
    }

} // namespace sci_cuda
