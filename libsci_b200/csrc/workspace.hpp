// workspace.hpp -- device scratch of the product and LU paths, grown on demand and reused.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace sci_cuda {

    struct Workspace {
        void *memory{nullptr};
        size_t bytes{0};

        // At least `need` bytes of device memory; the old contents are not kept.
        cudaError_t reserve(size_t need) {
            if (need <= bytes) return cudaSuccess;
            if (memory) cudaFree(memory);
            memory = nullptr;
            bytes = 0;
            cudaError_t code = cudaMalloc(&memory, need);
            if (code == cudaSuccess) bytes = need;
            return code;
        }

        void release() {
            if (memory) cudaFree(memory);
            memory = nullptr;
            bytes = 0;
        }
    };

} // namespace sci_cuda
