// noalloc.cu -- a chunk reduction that allocates nothing.
//
// Who needs it: code that runs where it may not create device memory of its own. A framework that
// owns the whole GPU heap through its own pool (so a stray cudaMalloc either fails against the
// pool's cap or fragments it), a plugin loaded into such a host, or a latency-critical thread on
// which an allocation would implicitly synchronize the device. sci_cuda_reduce needs a context,
// and opening one allocates a stream, pinned host words and the reduction's scratch. This entry
// point needs none of that: the caller passes the chunk (its inputs already in device memory), a
// device pointer for the result and a stream, and the single-pass fold keeps its per-block
// partials, its completion ticket and its error word in one fixed array compiled into this
// library (`noalloc_scratch`, below). The kernel is the same generic interpreter sci_cuda_reduce
// runs; only where its scratch lives differs.
//
// Limits and sharing:
//  - the array holds partials for at most kNoAllocBlocks (4096) blocks, 49,664 bytes in all
//    (sizeof(noalloc_scratch)); a request for a wider launch is rejected with
//    SCI_CUDA_ERROR_INVALID and a message;
//  - a block whose bounded wait on its copies runs out sets the error word; the last block then
//    writes a quiet NaN as the result instead of a fold of what the blocks saw, so a timeout can
//    never pass for a value (the call itself returned long before, with SCI_CUDA_OK);
//  - every GPU that loads this library holds one copy of the array until the process exits;
//  - every call on a device shares that device's copy, and it keeps whatever the last call left:
//    the ticket and the error word are cleared on the stream before each launch, the partials are
//    always written before they are read. Two calls whose kernels overlap on the GPU (different
//    streams, no ordering between them) race on the array and may return wrong results;
//  - the first call on a device looks up the array's device address (cudaGetSymbolAddress with
//    that device current) and keeps it; make that first call before capturing the stream into a
//    graph.
#include "context.hpp"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

// The scratch of every call on a device: a sci_cuda::ReduceState (block partials, NaN flags,
// ticket; 49,156 bytes, padded to 49,408) and, 256-byte aligned after it, the kernel's error word
// in a 256-byte slot: 49,664 bytes in all, partials for 4096 blocks.
// On the host this name is only a stand-in for the device variable, never a device address:
// passing it to a kernel would fault, or where the GPU can reach host memory, silently use the
// wrong memory. Host code gets the device address from cudaGetSymbolAddress (below).
static __device__ __align__(256) unsigned char noalloc_scratch[(sizeof(sci_cuda::ReduceState) + 255) / 256 * 256 + 256];

namespace sci_cuda {

    namespace {

        constexpr unsigned kNoAllocBlocks = kMaxBlocks;
        constexpr unsigned long long kStatusOffset = (sizeof(ReduceState) + 255) / 256 * 256;
        constexpr unsigned long long kNoAllocBytes = kStatusOffset + 256;
        constexpr int kMaxDevices = 64;
        static_assert(sizeof(noalloc_scratch) == kNoAllocBytes, "scratch layout");
        static_assert(kNoAllocBytes == 49664, "the documented size of the fixed scratch");

        struct DeviceSetup {
            bool ready{false};
            unsigned char *scratch{nullptr};
            int sms{0};
            int shared_limit{0};
        };

        std::mutex setup_guard;
        DeviceSetup setups[kMaxDevices];

        int say(char *message, size_t length, int code, const char *text, unsigned long long a = 0,
                unsigned long long b = 0) {
            if (message && length) std::snprintf(message, length, text, a, b);
            return code;
        }

        bool on_device(const void *pointer, int device) {
            cudaPointerAttributes attributes{};
            if (cudaPointerGetAttributes(&attributes, pointer) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
            if (attributes.type == cudaMemoryTypeManaged) return true;
            return attributes.type == cudaMemoryTypeDevice && attributes.device == device;
        }

        int check_chunk(const sci_chunk &chunk, char *message, size_t length) {
            if (chunk.precision > SCI_PRECISION_WIDE) return say(message, length, SCI_CUDA_ERROR_INVALID, "unknown precision");
            if (chunk.length > SCI_CHUNK_CAPACITY || chunk.arguments > SCI_CHUNK_CAPACITY ||
                chunk.literals > SCI_CHUNK_CAPACITY || chunk.temporaries > SCI_CHUNK_CAPACITY)
                return say(message, length, SCI_CUDA_ERROR_INVALID, "chunk counts exceed the capacity of 64");
            auto in_range = [&](unsigned char id, bool allow_none) {
                if (id == SCI_SLOT_NONE) return allow_none;
                const int kind = id & SCI_SLOT_TYPES, slot = id & 63;
                if (kind == SCI_SLOT_INPUT) return slot < chunk.arguments;
                if (kind == SCI_SLOT_LITERAL) return slot < chunk.literals;
                if (kind == SCI_SLOT_TEMPORARY) return slot < chunk.temporaries;
                return false;
            };
            for (int i = 0; i < chunk.length; ++i) {
                const sci_instruction &ins = chunk.instructions[i];
                if (ins.code >= SCI_CODE_COUNT)
                    return say(message, length, SCI_CUDA_ERROR_INVALID, "instruction %llu: unknown code", i);
                const int arity = ins.code < SCI_CODE_ADD ? 1 : (ins.code < SCI_CODE_FUSE ? 2 : 3);
                for (int s = 0; s < 3; ++s) {
                    if (!in_range(ins.sources[s], s >= arity))
                        return say(message, length, SCI_CUDA_ERROR_INVALID, "instruction %llu: a source is out of range", i);
                }
                if (ins.target != SCI_SLOT_OUTPUT &&
                    ((ins.target & SCI_SLOT_TYPES) != SCI_SLOT_TEMPORARY || (ins.target & 63) >= chunk.temporaries))
                    return say(message, length, SCI_CUDA_ERROR_INVALID, "instruction %llu: target out of range", i);
            }
            if (!in_range(chunk.result, false) && !(chunk.result == SCI_SLOT_OUTPUT && chunk.length > 0))
                return say(message, length, SCI_CUDA_ERROR_INVALID, "the chunk's result is out of range");
            return SCI_CUDA_OK;
        }

        template <typename T>
        int reduce(const sci_chunk &chunk, unsigned fold, unsigned long long count, double *result, cudaStream_t stream,
                   unsigned blocks, const DeviceSetup &setup, int device, char *message, size_t length) {
            Launch<T> L;
            std::memset(&L, 0, sizeof(L));
            const bool contract = fold == SCI_FOLD_SUM && chunk.length > 0 &&
                                  chunk.instructions[chunk.length - 1].code == SCI_CODE_MULTIPLY &&
                                  chunk.instructions[chunk.length - 1].target == chunk.result;
            const int mode = contract ? kDot : kReduce;
            L.length = contract ? chunk.length - 1 : chunk.length;
            for (int i = 0; i < chunk.length; ++i) {
                const sci_instruction &ins = chunk.instructions[i];
                L.steps[i] = Step{ins.code, ins.target, ins.sources[0], ins.sources[1], ins.sources[2]};
            }
            if (contract) {
                L.dot_left = chunk.instructions[chunk.length - 1].sources[0];
                L.dot_right = chunk.instructions[chunk.length - 1].sources[1];
            }
            L.value = chunk.result;
            L.arguments = chunk.arguments;
            L.temporaries = chunk.temporaries;
            L.fold = fold;
            for (int i = 0; i < chunk.length; ++i) {
                const int code = chunk.instructions[i].code;
                if (code == SCI_CODE_MINIMUM || code == SCI_CODE_MAXIMUM) L.tailed = 1;
            }
            bool aligned = true;
            for (int i = 0; i < chunk.literals; ++i) L.constants[i] = static_cast<T>(chunk.constants[i]);
            for (int i = 0; i < chunk.arguments; ++i) {
                if (!chunk.inputs[i] || !on_device(chunk.inputs[i], device))
                    return say(message, length, SCI_CUDA_ERROR_INVALID, "input %llu is not memory of the current device", i);
                L.inputs[i] = static_cast<const T *>(chunk.inputs[i]);
                aligned = aligned && reinterpret_cast<unsigned long long>(chunk.inputs[i]) % 16 == 0;
            }
            L.count = count;
            L.tail_start = count - count % (64 / sizeof(T));
            L.state = reinterpret_cast<ReduceState *>(setup.scratch);
            L.status = reinterpret_cast<int *>(setup.scratch + kStatusOffset);
            L.destination = result;

            // Block size and TMA ring depth chosen exactly as sci_cuda_reduce chooses them for the
            // generic interpreter (chunk_shape), so both entry points fold in the same order.
            const size_t budget = setup.shared_limit < 200 * 1024 ? size_t(setup.shared_limit) : size_t(200 * 1024);
            const ChunkShape shape = chunk_shape(L.steps, L.length, L.arguments, L.temporaries, sizeof(T), aligned, false,
                                                 budget);
            if (shape.threads < 32) return say(message, length, SCI_CUDA_ERROR_UNSUPPORTED, "chunk too wide for shared memory");
            const int threads = shape.threads;
            const size_t smem = shape.smem;
            L.stages = shape.stages;
            const void *kernel = generic_chunk_kernel(sizeof(T) == 8, mode);
            // Static shared memory (mbarriers, fold scratch) counts against the 48 KB a launch gets
            // without the opt-in, so the limit is raised from the same threshold sci_cuda_reduce uses.
            if (smem > kChunkSharedOptIn &&
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
                return say(message, length, SCI_CUDA_ERROR_LAUNCH, "cannot raise the kernel's shared memory limit");
            int per_sm = 1;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
                per_sm = 1;
            const unsigned long long tile = 1ull * Lanes<T>::count * threads;
            unsigned long long grid = (count + tile - 1) / tile;
            const unsigned long long wide = 1ull * per_sm * setup.sms;
            if (grid > wide) grid = wide;
            if (grid > (blocks ? blocks : kNoAllocBlocks)) grid = blocks ? blocks : kNoAllocBlocks;
            if (grid < 1) grid = 1;

            // The ticket and the error word must start at zero; the partials are written before read.
            if (cudaMemsetAsync(&L.state->ticket, 0, sizeof(unsigned), stream) != cudaSuccess ||
                cudaMemsetAsync(L.status, 0, sizeof(int), stream) != cudaSuccess)
                return say(message, length, SCI_CUDA_ERROR_LAUNCH, "cannot clear the scratch");
            void *args[] = {&L};
            if (cudaLaunchKernel(kernel, dim3(static_cast<unsigned>(grid)), dim3(threads), args, smem, stream) != cudaSuccess) {
                cudaGetLastError();
                return say(message, length, SCI_CUDA_ERROR_LAUNCH, "the reduction kernel did not launch");
            }
            return SCI_CUDA_OK;
        }

    } // namespace

} // namespace sci_cuda

using namespace sci_cuda;

extern "C" int sci_cuda_reduce_noalloc(const sci_chunk *chunk, uint32_t fold, uint64_t count, double *device_result,
                                       void *stream, uint32_t blocks, char *message, size_t message_length) {
    if (message && message_length) message[0] = '\0';
    if (!chunk || !device_result) return say(message, message_length, SCI_CUDA_ERROR_INVALID, "null chunk or result");
    if (fold > SCI_FOLD_MAXIMUM) return say(message, message_length, SCI_CUDA_ERROR_INVALID, "unknown fold %llu", fold);
    if (blocks > kNoAllocBlocks)
        return say(message, message_length, SCI_CUDA_ERROR_INVALID,
                   "blocks = %llu exceeds the %llu block partials the fixed scratch holds", blocks, kNoAllocBlocks);
    if (int code = check_chunk(*chunk, message, message_length)) return code;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return say(message, message_length, SCI_CUDA_ERROR_DEVICE, "no current CUDA device");
    if (!on_device(device_result, device))
        return say(message, message_length, SCI_CUDA_ERROR_INVALID, "the result is not memory of the current device");
    const cudaStream_t queue = static_cast<cudaStream_t>(stream);

    DeviceSetup setup;
    {
        std::lock_guard<std::mutex> lock(setup_guard);
        DeviceSetup &slot = setups[device];
        if (!slot.ready) {
            void *address = nullptr;
            const cudaError_t found = cudaGetSymbolAddress(&address, noalloc_scratch);
            if (found != cudaSuccess || address == nullptr) {
                cudaGetLastError();
                return say(message, message_length, SCI_CUDA_ERROR_LAUNCH,
                           "cudaGetSymbolAddress failed for the fixed scratch (error %llu)", found);
            }
            int sms = 0, shared = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            cudaDeviceGetAttribute(&shared, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
            slot.scratch = static_cast<unsigned char *>(address);
            slot.sms = sms > 0 ? sms : 1;
            slot.shared_limit = shared > 0 ? shared : 48 * 1024;
            slot.ready = true;
        }
        setup = slot;
    }

    if (count == 0) {
        // An empty sum is 0 and an empty extreme NaN (src/core/drivers/processor/dispatch.cpp:109-111):
        // all-zero bytes are +0.0, all-one bytes a NaN.
        if (cudaMemsetAsync(device_result, fold == SCI_FOLD_SUM ? 0x00 : 0xFF, sizeof(double), queue) != cudaSuccess)
            return say(message, message_length, SCI_CUDA_ERROR_LAUNCH, "cannot write the empty result");
        return SCI_CUDA_OK;
    }
    if (chunk->precision == SCI_PRECISION_WIDE)
        return reduce<double>(*chunk, fold, count, device_result, queue, blocks, setup, device, message, message_length);
    return reduce<float>(*chunk, fold, count, device_result, queue, blocks, setup, device, message, message_length);
}
