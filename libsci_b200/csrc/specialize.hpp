// specialize.hpp -- NVRTC specialisation of the chunk kernel, keyed by Chunk::signature().
//
// Stands where the reference's background Slang compiler stands (include/core/drivers/vulkan/
// compiler.hpp, src/core/drivers/vulkan/compiler.cpp:35-222): a chunk seen again is compiled
// into its own instance of the same kernel source (chunk_kernel.cuh) with the bytecode baked in;
// until that instance is ready the generic interpreter runs it.
#pragma once

#include "context.hpp"

#include <memory>

namespace sci_cuda {

    struct Specialized {
        const void *function;  // a cudaKernel_t, launched like a kernel symbol
    };

    class Specializer {
    public:
        virtual ~Specializer() = default;
        // The specialised kernel for this chunk and mode, or null while there is none (yet).
        virtual const Specialized *find(Context &ctx, const sci_chunk &chunk, int mode) = 0;
        // Waits until every queued compile has finished.
        virtual void wait() = 0;
    };

    std::unique_ptr<Specializer> make_specializer(Context &ctx);

} // namespace sci_cuda
