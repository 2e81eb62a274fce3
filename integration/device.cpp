// integration/device.cpp -- libsci's Device (include/core/drivers/device.hpp:27-89) with the CUDA
// target of the B200 backend, compiled against the reference's own headers, unchanged (the CUDA
// target is Target value 2, `cuda_target` in sci_cuda_device.hpp: the value the backend's one-line
// change to target.hpp names Target::cuda).
//
// This file stands where src/core/drivers/device.cpp stands. What it does per target:
//  - Target::processor: every entry point runs libsci's CPU path (processor::Dispatch), as the
//    reference does for a CPU device;
//  - Target::cuda (cuda_target): the device opens a libsci_cuda.so context on GPU `index`; memory is CUDA managed
//    memory (so Memory::host stays a usable host pointer, memory.hpp:16-27) and execute / reduce /
//    product run the backend's sm_100a kernels. There is no CPU fallback: a device that cannot open
//    throws, and a failing call throws std::runtime_error with the backend's message;
//  - Target::graphics: a request for "the GPU". This build has no Vulkan driver; where a CUDA GPU
//    exists it serves the request (target() stays Target::graphics, so code written for the
//    graphics target runs unchanged), otherwise the device falls back to the CPU with the
//    reference's message (device.cpp:186-199).
#include "sci_cuda_device.hpp"

#include "core/alignment.hpp"
#include "core/drivers/device.hpp"
#include "core/drivers/processor/dispatch.hpp"

#include <cstdio>
#include <limits>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

namespace sci::core::drivers {

    /// What a GPU Device owns: its libsci_cuda.so context.
    struct Graphics {
        sci_cuda_context *cuda{nullptr};
    };

    namespace {

        // Device -> context, for the free functions of sci_cuda_device.hpp (Device keeps its
        // Graphics private and the reference's header stays unchanged).
        std::mutex registry_guard;
        std::map<const Device *, sci_cuda_context *> registry;

        // core::Chunk -> sci_chunk: the same public fields (chunk.hpp:178-194).
        sci_chunk mirror(const Chunk &chunk) {
            sci_chunk out{};
            out.precision = static_cast<uint8_t>(chunk.precision);
            out.length = chunk.length;
            out.arguments = chunk.arguments;
            out.literals = chunk.literals;
            out.temporaries = chunk.temporaries;
            out.result = chunk.result;
            for (uint8 i = 0; i < chunk.length; ++i) {
                const Instruction &step = chunk.instructions[i];
                out.instructions[i].code = static_cast<uint8_t>(step.code);
                out.instructions[i].target = step.target;
                for (int s = 0; s < 3; ++s) out.instructions[i].sources[s] = step.sources[s];
            }
            for (uint8 i = 0; i < chunk.arguments; ++i) out.inputs[i] = chunk.inputs[i];
            for (uint8 i = 0; i < chunk.literals; ++i) out.constants[i] = chunk.constants[i];
            return out;
        }

        // For the noexcept entry points: report on stderr, as the reference reports (device.cpp:196).
        void report(sci_cuda_context *context, const int status, const char *what) noexcept {
            if (status == SCI_CUDA_OK) return;
            char message[512] = {0};
            sci_cuda_last_error(context, message, sizeof message);
            std::fprintf(stderr, "[sci] CUDA %s failed: %s\n", what, message);
        }

    } // namespace

    sci_cuda_context *cuda_context(const Device *device) noexcept {
        if (device == nullptr) return nullptr;
        std::lock_guard<std::mutex> lock(registry_guard);
        const auto found = registry.find(device);
        return found == registry.end() ? nullptr : found->second;
    }

    void cuda_must(sci_cuda_context *context, const int status, const char *what) {
        if (status == SCI_CUDA_OK) return;
        char message[512] = {0};
        if (context != nullptr) sci_cuda_last_error(context, message, sizeof message);
        throw std::runtime_error(std::string("[sci] CUDA ") + what + " failed (status " + std::to_string(status) +
                                 "): " + message);
    }

    Device::Device(const Target target, const uint32 index) : type(target), ordinal(index) {
        if (type == Target::processor) return;
        sci_cuda_context *context = nullptr;
        const int status = sci_cuda_open(ordinal, &context);
        if (status == SCI_CUDA_OK) {
            graphics = std::make_unique<Graphics>();
            graphics->cuda = context;
            std::lock_guard<std::mutex> lock(registry_guard);
            registry[this] = context;
            return;
        }
        if (type == cuda_target)
            throw std::runtime_error("[sci] no usable sm_100 CUDA device at index " + std::to_string(ordinal));
        std::fprintf(stderr, "[sci] no usable GPU at index %u; running on the CPU\n", static_cast<unsigned>(ordinal));
        type = Target::processor;
    }

    Device::~Device() {
        if (!graphics) return;
        {
            std::lock_guard<std::mutex> lock(registry_guard);
            registry.erase(this);
        }
        sci_cuda_close(graphics->cuda);
    }

    const char *Device::name() const noexcept { return graphics ? sci_cuda_name(graphics->cuda) : "cpu"; }

    void Device::synchronize() noexcept {
        if (graphics) report(graphics->cuda, sci_cuda_synchronize(graphics->cuda), "synchronize");
    }

    void Device::allocate(const size bytes, Memory &memory) {
        memory.bytes = bytes;
        memory.target = type;
        if (graphics) {
            cuda_must(graphics->cuda, sci_cuda_allocate(graphics->cuda, bytes, SCI_CUDA_MEMORY_MANAGED, &memory.host),
                      "allocate");
        } else {
            memory.allocation = core::memory::Allocation(bytes, alignment::line);
            memory.host = memory.allocation.data();
        }
        ASSERT(memory.host != nullptr);
    }

    void Device::dispose(Memory &memory) noexcept {
        // the free waits for work queued before it, as vulkan::Stream::retire (stream.cpp:117-130)
        if (graphics && memory.target == type && memory.host != nullptr)
            report(graphics->cuda, sci_cuda_dispose(graphics->cuda, memory.host), "dispose");
        memory = {};
    }

    void Device::execute(const Chunk &chunk, void *output, const size count) {
        if (count == 0) return;
        if (graphics) {
            const sci_chunk mirrored = mirror(chunk);
            cuda_must(graphics->cuda, sci_cuda_execute(graphics->cuda, &mirrored, output, count), "execute");
            return;
        }
        processor::Dispatch::global().execute(chunk, output, count);
    }

    double Device::reduce(const Chunk &chunk, const Fold fold, const size count) {
        if (count == 0) return fold == Fold::sum ? 0.0 : std::numeric_limits<double>::quiet_NaN();
        if (graphics) {
            const sci_chunk mirrored = mirror(chunk);
            double result = 0.0;
            cuda_must(graphics->cuda,
                      sci_cuda_reduce(graphics->cuda, &mirrored, static_cast<uint32_t>(fold), count, &result), "reduce");
            return result;
        }
        return processor::Dispatch::global().reduce(chunk, fold, count);
    }

    void Device::product(const Precision precision, const void *left, const void *right, void *output, const size rows,
                         const size columns, const size depth) {
        if (rows == 0 || columns == 0) return;
        if (graphics) {
            // Float products keep FP32 accuracy, as the reference's float multiply does
            // (dispatch.cpp:171-224): hi + mid + lo bf16 terms, six tensor-core products, FP32
            // accumulation. Double products run in plain FP64.
            cuda_must(graphics->cuda,
                      sci_cuda_product(graphics->cuda, static_cast<uint32_t>(precision), SCI_PRODUCT_SPLIT3_BF16, left,
                                       right, output, rows, columns, depth),
                      "product");
            return;
        }
        processor::Dispatch::product(precision, left, right, output, rows, columns, depth);
    }

}
