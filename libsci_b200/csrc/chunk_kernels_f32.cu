// chunk_kernels_f32.cu -- the generic (float) chunk interpreter, compiled ahead of time.
#include "chunk_kernel.cuh"

namespace sci_cuda {

    const void *generic_chunk_kernel_f32(int mode) {
        switch (mode) {
        case kEvaluate: return reinterpret_cast<const void *>(&chunk_stream<float, Dynamic, kEvaluate>);
        case kReduce: return reinterpret_cast<const void *>(&chunk_stream<float, Dynamic, kReduce>);
        default: return reinterpret_cast<const void *>(&chunk_stream<float, Dynamic, kDot>);
        }
    }

} // namespace sci_cuda
