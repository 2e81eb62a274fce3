// device.cu -- the C ABI: contexts, memory, chunk execution and reductions on one B200.
//
// The CUDA counterpart of the reference's GPU branch of sci::core::drivers::Device
// (src/core/drivers/device.cpp:186-352). Differences by design:
//  - no CPU fallback: a chunk the device cannot run is an error (the reference silently falls back,
//    device.cpp:258-262,313-315);
//  - no slicing of launches into 2^30-work dispatches (device.cpp:97-100): CUDA has no watchdog
//    here, and counts are 64-bit throughout (the reference caps n below 2^31, device.cpp:149);
//  - the reduction folds on the device in a single pass instead of on the host from per-group
//    partials (device.cpp:277-311), so it never leaves the stream until the caller asks.
#include "context.hpp"
#include "specialize.hpp"
#include "workspace.hpp"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <limits>

using namespace sci_cuda;

namespace sci_cuda {

    int Context::drain(bool status_queued) {
        int code = status_queued ? SCI_CUDA_OK
                                 : check(cudaMemcpyAsync(host_status, status, sizeof(int), cudaMemcpyDeviceToHost, stream),
                                         "reading the device status");
        if (code) return code;
        code = check(cudaStreamSynchronize(stream), "synchronizing the stream");
        if (code) return code;
        // Frees whose work is done.
        for (auto it = retired.begin(); it != retired.end();) {
            if (cudaEventQuery(it->done) == cudaSuccess) {
                cudaEventDestroy(it->done);
                cudaFree(it->memory);
                it = retired.erase(it);
            } else {
                ++it;
            }
        }
        if (*host_status != 0) {
            const int seen = *host_status;
            *host_status = 0;
            cudaMemsetAsync(status, 0, sizeof(int), stream);
            // A reduction that gave up left its ticket behind; start the next one clean.
            cudaMemsetAsync(&state->ticket, 0, sizeof(unsigned), stream);
            cudaStreamSynchronize(stream);
            if (seen & kStatusTimeout) {
                return fail(SCI_CUDA_ERROR_TIMEOUT, "a kernel's bounded wait on its copies ran out");
            }
            return fail(SCI_CUDA_ERROR_LAUNCH, "device status %d", seen);
        }
        return SCI_CUDA_OK;
    }

    int validate(Context &ctx, const sci_chunk *chunk, const bool reducing) {
        if (!chunk) return ctx.fail(SCI_CUDA_ERROR_INVALID, "null chunk");
        if (chunk->precision > SCI_PRECISION_WIDE) return ctx.fail(SCI_CUDA_ERROR_INVALID, "unknown precision %d", chunk->precision);
        if (chunk->length > SCI_CHUNK_CAPACITY || chunk->arguments > SCI_CHUNK_CAPACITY ||
            chunk->literals > SCI_CHUNK_CAPACITY || chunk->temporaries > SCI_CHUNK_CAPACITY)
            return ctx.fail(SCI_CUDA_ERROR_INVALID, "chunk counts exceed the capacity of %d", SCI_CHUNK_CAPACITY);
        auto in_range = [&](uint8_t id, bool allow_none) {
            if (id == SCI_SLOT_NONE) return allow_none;
            const int kind = id & SCI_SLOT_TYPES, slot = id & 63;
            if (kind == SCI_SLOT_INPUT) return slot < chunk->arguments;
            if (kind == SCI_SLOT_LITERAL) return slot < chunk->literals;
            if (kind == SCI_SLOT_TEMPORARY) return slot < chunk->temporaries;
            return false;  // the output slot is never a source
        };
        bool writes_output = false;
        for (int i = 0; i < chunk->length; ++i) {
            const sci_instruction &ins = chunk->instructions[i];
            if (ins.code >= SCI_CODE_COUNT) return ctx.fail(SCI_CUDA_ERROR_INVALID, "instruction %d: unknown code %d", i, ins.code);
            const int arity = ins.code < SCI_CODE_ADD ? 1 : (ins.code < SCI_CODE_FUSE ? 2 : 3);
            for (int s = 0; s < 3; ++s) {
                if (!in_range(ins.sources[s], s >= arity))
                    return ctx.fail(SCI_CUDA_ERROR_INVALID, "instruction %d: source %d (0x%02x) out of range", i, s, ins.sources[s]);
            }
            if (ins.target == SCI_SLOT_OUTPUT) {
                writes_output = true;
            } else if ((ins.target & SCI_SLOT_TYPES) != SCI_SLOT_TEMPORARY || (ins.target & 63) >= chunk->temporaries) {
                return ctx.fail(SCI_CUDA_ERROR_INVALID, "instruction %d: target 0x%02x out of range", i, ins.target);
            }
        }
        if (reducing) {
            if (!in_range(chunk->result, false) && chunk->result != SCI_SLOT_OUTPUT)
                return ctx.fail(SCI_CUDA_ERROR_INVALID, "result 0x%02x out of range", chunk->result);
            if (chunk->result == SCI_SLOT_OUTPUT && chunk->length == 0)
                return ctx.fail(SCI_CUDA_ERROR_INVALID, "result is the output of an empty chunk");
        } else if (!writes_output) {
            return ctx.fail(SCI_CUDA_ERROR_INVALID, "the chunk writes no output");
        }
        return SCI_CUDA_OK;
    }

    // Whether a pointer is memory this context's GPU reads directly (the reference's
    // Allocator::locate, src/core/drivers/vulkan/allocator.cpp:81-89).
    bool reachable(Context &ctx, const void *pointer) {
        cudaPointerAttributes attributes{};
        if (cudaPointerGetAttributes(&attributes, pointer) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (attributes.type == cudaMemoryTypeManaged) return true;
        return attributes.type == cudaMemoryTypeDevice && attributes.device == ctx.device;
    }

    template <typename T>
    static int prepare(Context &ctx, const sci_chunk &chunk, int mode, uint32_t fold, uint64_t count, void *output,
                       double *result, Launch<T> &L) {
        std::memset(&L, 0, sizeof(L));
        const bool contract = mode != kEvaluate && fold == SCI_FOLD_SUM && chunk.length > 0 &&
                              chunk.instructions[chunk.length - 1].code == SCI_CODE_MULTIPLY &&
                              chunk.instructions[chunk.length - 1].target == chunk.result;
        L.length = contract ? chunk.length - 1 : chunk.length;
        for (int i = 0; i < chunk.length; ++i) {
            const sci_instruction &ins = chunk.instructions[i];
            L.steps[i] = Step{ins.code, ins.target, ins.sources[0], ins.sources[1], ins.sources[2]};
        }
        if (contract) {
            L.dot_left = chunk.instructions[chunk.length - 1].sources[0];
            L.dot_right = chunk.instructions[chunk.length - 1].sources[1];
        }
        L.arguments = chunk.arguments;
        L.temporaries = chunk.temporaries;
        L.fold = fold;
        for (int i = 0; i < chunk.length; ++i) {
            const int code = chunk.instructions[i].code;
            if (code == SCI_CODE_MINIMUM || code == SCI_CODE_MAXIMUM) L.tailed = 1;
        }
        for (int i = 0; i < chunk.literals; ++i) L.constants[i] = static_cast<T>(chunk.constants[i]);
        for (int i = 0; i < chunk.arguments; ++i) {
            if (!chunk.inputs[i] || !reachable(ctx, chunk.inputs[i]))
                return ctx.fail(SCI_CUDA_ERROR_INVALID, "input %d (%p) is not memory of this device", i, chunk.inputs[i]);
            L.inputs[i] = static_cast<const T *>(chunk.inputs[i]);
        }
        if (mode == kEvaluate) {
            if (!output || !reachable(ctx, output))
                return ctx.fail(SCI_CUDA_ERROR_INVALID, "output (%p) is not memory of this device", output);
        }
        L.output = static_cast<T *>(output);
        L.count = count;
        // Loop tails of the reference's AVX-512 table take the one-lane forms (elementwise.hpp:136-196).
        const uint64_t width = 64 / sizeof(T);
        L.tail_start = count - count % width;
        L.state = ctx.state;
        L.value = chunk.result;
        L.destination = result;
        L.status = ctx.status;
        return SCI_CUDA_OK;
    }

    template <typename T>
    static bool aligned(const Launch<T> &L, int mode) {
        for (unsigned i = 0; i < L.arguments; ++i) {
            if (reinterpret_cast<uintptr_t>(L.inputs[i]) % 16) return false;
        }
        if (mode == kEvaluate && reinterpret_cast<uintptr_t>(L.output) % 16) return false;
        return true;
    }


    // Picks the block size, ring depth and grid for a launch, and launches it.
    template <typename T>
    static int launch(Context &ctx, Launch<T> &L, int mode, double *device_result, const sci_chunk &chunk) {
        L.destination = device_result ? device_result : ctx.result;

        // A specialised kernel when one is ready for this signature (or compiled now in
        // synchronous mode); the generic interpreter otherwise.
        const Specialized *special = ctx.specializer ? ctx.specializer->find(ctx, chunk, mode) : nullptr;
        const void *kernel = special ? special->function : generic_chunk_kernel(sizeof(T) == 8, mode);
        const size_t budget = std::min<size_t>(ctx.shared_limit, 200 * 1024);
        const ChunkShape shape = chunk_shape(L.steps, L.length, L.arguments, L.temporaries, sizeof(T), aligned(L, mode),
                                             special != nullptr, budget);
        if (shape.threads < 32) return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "chunk too wide for shared memory");
        const int threads = shape.threads;
        const size_t smem = shape.smem;
        L.stages = shape.stages;

        const uint64_t tile = uint64_t(Lanes<T>::count) * threads;
        const uint64_t tiles = (L.count + tile - 1) / tile;
        void *args[] = {&L};
        if (special) {
            // An NVRTC module: a driver-API function.
            CUfunction function = reinterpret_cast<CUfunction>(const_cast<void *>(special->function));
            // the module is this context's own: its limit is raised past the largest use only
            ctx.allow_smem(special->function, smem, [&] {
                Driver::get().function_attribute(function, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, static_cast<int>(smem));
            });
            const auto key = std::make_tuple(special->function, threads, smem);
            auto found = ctx.occupancy.find(key);
            int per_sm = 1;
            if (found != ctx.occupancy.end()) {
                per_sm = found->second;
            } else {
                if (Driver::get().occupancy(&per_sm, function, threads, smem) != CUDA_SUCCESS || per_sm < 1)
                    per_sm = 1;
                ctx.occupancy[key] = per_sm;
            }
            const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>({tiles, uint64_t(per_sm) * ctx.sms, kMaxBlocks}));
            const CUresult code = Driver::get().launch(function, static_cast<unsigned>(grid), 1, 1, threads, 1, 1,
                                                 static_cast<unsigned>(smem), ctx.stream, args, nullptr);
            if (code != CUDA_SUCCESS) return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "launching a specialised chunk kernel: %d", int(code));
            return SCI_CUDA_OK;
        }
        // Set on every launch: other contexts, and the entry point without allocations, set the same
        // kernel's limit too (it is the process's, not this context's).
        if (smem > kChunkSharedOptIn) {
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        }
        const int per_sm = ctx.blocks_per_sm(kernel, threads, smem);
        const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>({tiles, uint64_t(per_sm) * ctx.sms, kMaxBlocks}));
        return ctx.check(cudaLaunchKernel(kernel, dim3(static_cast<unsigned>(grid)), dim3(threads), args, smem, ctx.stream),
                         "launching the chunk kernel");
    }

    template <typename T>
    static int run(Context &ctx, const sci_chunk &chunk, int mode, uint32_t fold, uint64_t count, void *output,
                   double *device_result) {
        Launch<T> L;
        if (int code = prepare<T>(ctx, chunk, mode, fold, count, output, device_result, L)) return code;
        const bool contract = mode != kEvaluate && L.length + 1 == chunk.length && fold == SCI_FOLD_SUM &&
                              chunk.length > 0 && chunk.instructions[chunk.length - 1].code == SCI_CODE_MULTIPLY &&
                              chunk.instructions[chunk.length - 1].target == chunk.result;
        return launch<T>(ctx, L, contract ? kDot : mode, device_result, chunk);
    }

    static int dispatch(Context &ctx, const sci_chunk &chunk, int mode, uint32_t fold, uint64_t count, void *output,
                        double *device_result) {
        if (chunk.precision == SCI_PRECISION_WIDE) return run<double>(ctx, chunk, mode, fold, count, output, device_result);
        return run<float>(ctx, chunk, mode, fold, count, output, device_result);
    }

} // namespace sci_cuda

extern "C" {

int sci_cuda_open(uint32_t ordinal, sci_cuda_context **context) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    *context = nullptr;
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || int(ordinal) >= devices) {
        cudaGetLastError();
        return SCI_CUDA_ERROR_DEVICE;
    }
    cudaDeviceProp props{};
    if (cudaGetDeviceProperties(&props, int(ordinal)) != cudaSuccess || props.major != 10) return SCI_CUDA_ERROR_DEVICE;
    auto ctx = std::make_unique<sci_cuda_context>();
    ctx->device = int(ordinal);
    ctx->sms = props.multiProcessorCount;
    ctx->shared_limit = props.sharedMemPerBlockOptin;
    ctx->name = props.name;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return SCI_CUDA_ERROR_DEVICE;
    // The context's stream at the highest priority: the LU look-ahead queues its bulk updates on a
    // lower-priority side stream, so blocks that free up go to the critical path first.
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, greatest) != cudaSuccess) return SCI_CUDA_ERROR_DEVICE;
    // the reduction's result with the status word after it (device and pinned host): a blocking
    // reduction reads both with one copy
    if (cudaMalloc(&ctx->state, sizeof(ReduceState)) != cudaSuccess || cudaMalloc(&ctx->result, kResultBytes) != cudaSuccess ||
        cudaMallocHost(&ctx->host_result, kResultBytes) != cudaSuccess) {
        return SCI_CUDA_ERROR_MEMORY;
    }
    ctx->status = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(ctx->result) + sizeof(double));
    ctx->host_status = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(ctx->host_result) + sizeof(double));
    cudaMemsetAsync(ctx->state, 0, sizeof(ReduceState), ctx->stream);
    cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream);
    *ctx->host_status = 0;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return SCI_CUDA_ERROR_DEVICE;
    if (const char *setting = std::getenv("SCI_CUDA_JIT")) {
        ctx->jit_mode = std::strcmp(setting, "0") == 0 ? 0 : (std::strcmp(setting, "sync") == 0 ? 2 : 1);
        ctx->jit_trace = std::strcmp(setting, "trace") == 0;
    }
    ctx->specializer = make_specializer(*ctx);
    ctx->workspace = std::make_unique<Workspace>();
    ctx->solver = std::make_unique<Workspace>();
    ctx->tape = std::make_unique<Workspace>();
    *context = ctx.release();
    return SCI_CUDA_OK;
}

int sci_cuda_close(sci_cuda_context *context) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    {
        std::lock_guard<std::recursive_mutex> lock(context->guard);
        cudaSetDevice(context->device);
        cudaStreamSynchronize(context->stream);
        context->specializer.reset();
        if (context->workspace) context->workspace->release();
        if (context->solver) context->solver->release();
        if (context->tape) context->tape->release();
        for (auto &r : context->retired) {
            cudaEventDestroy(r.done);
            cudaFree(r.memory);
        }
        context->retired.clear();
        cudaFree(context->state);
        cudaFree(context->result);  // and the status word
        cudaFree(context->sweep_flags);
        if (context->side) cudaStreamDestroy(context->side);
        if (context->side_done) cudaEventDestroy(context->side_done);
        if (context->main_ready) cudaEventDestroy(context->main_ready);
        if (context->side_space) context->side_space->release();
        if (context->upload_lane) {
            cudaStreamSynchronize(context->upload_lane);
            cudaStreamSynchronize(context->download_lane);
            cudaStreamDestroy(context->upload_lane);
            cudaStreamDestroy(context->download_lane);
            cudaEventDestroy(context->uploaded);
            cudaEventDestroy(context->downloaded);
            cudaEventDestroy(context->main_point);
        }
        cudaFreeHost(context->host_result);  // and host_status
        cudaFreeHost(context->pinned);
        cudaStreamDestroy(context->stream);
    }
    delete context;
    return SCI_CUDA_OK;
}

const char *sci_cuda_name(const sci_cuda_context *context) { return context ? context->name.c_str() : "none"; }

int sci_cuda_jit_wait(sci_cuda_context *context) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    if (context->specializer) context->specializer->wait();
    return SCI_CUDA_OK;
}

int sci_cuda_synchronize(sci_cuda_context *context) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    if (context->upload_lane) {
        if (int code = context->check(cudaStreamSynchronize(context->upload_lane), "synchronizing the upload lane")) return code;
        if (int code = context->check(cudaStreamSynchronize(context->download_lane), "synchronizing the download lane"))
            return code;
    }
    return context->drain();
}

int sci_cuda_last_error(const sci_cuda_context *context, char *buffer, size_t length) {
    if (!context || !buffer || length == 0) return SCI_CUDA_ERROR_INVALID;
    std::snprintf(buffer, length, "%s", context->error.c_str());
    return SCI_CUDA_OK;
}

void *sci_cuda_stream(sci_cuda_context *context) { return context ? static_cast<void *>(context->stream) : nullptr; }

int sci_cuda_allocate(sci_cuda_context *context, uint64_t bytes, uint32_t kind, void **memory) {
    if (!context || !memory || kind > SCI_CUDA_MEMORY_MANAGED) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    *memory = nullptr;
    if (bytes == 0) bytes = 256;
    cudaError_t code;
    if (kind == SCI_CUDA_MEMORY_MANAGED) {
        code = cudaMallocManaged(memory, bytes, cudaMemAttachGlobal);
        if (code == cudaSuccess) {
            cudaMemLocation location{};
            location.type = cudaMemLocationTypeDevice;
            location.id = context->device;
            cudaMemAdvise(*memory, bytes, cudaMemAdviseSetPreferredLocation, location);
        }
    } else {
        code = cudaMalloc(memory, bytes);
    }
    if (code != cudaSuccess) {
        // Like the reference's allocator (allocator.cpp:56-65): release what is pending, retry once.
        cudaGetLastError();
        context->drain();
        code = kind == SCI_CUDA_MEMORY_MANAGED ? cudaMallocManaged(memory, bytes, cudaMemAttachGlobal) : cudaMalloc(memory, bytes);
    }
    return context->check(code, "allocating device memory");
}

int sci_cuda_dispose(sci_cuda_context *context, void *memory) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    if (!memory) return SCI_CUDA_OK;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    Retired r{nullptr, memory, false};
    if (cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming) != cudaSuccess) return context->fail(SCI_CUDA_ERROR_LAUNCH, "event");
    cudaEventRecord(r.done, context->stream);
    context->retired.push_back(r);
    return SCI_CUDA_OK;
}

int sci_cuda_upload(sci_cuda_context *context, void *device, const void *host, uint64_t bytes) {
    if (!context || (!device && bytes) || (!host && bytes)) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    return context->check(cudaMemcpyAsync(device, host, bytes, cudaMemcpyHostToDevice, context->stream), "upload");
}

int sci_cuda_download(sci_cuda_context *context, void *host, const void *device, uint64_t bytes) {
    if (!context || (!device && bytes) || (!host && bytes)) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    return context->check(cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, context->stream), "download");
}

// ---- copy lanes: host <-> device copies that overlap the main stream's work -------------------
// Two more streams per context, made on first use. An upload on the lane starts at once (it does
// not wait for queued kernels) and everything queued on the main stream after it waits for it; a
// download on the lane waits for everything queued on the main stream before it and delays nothing
// queued after it. PCIe carries both directions at once, so a caller that splits its arrays into
// pieces overlaps the upload of one piece, the kernels of the previous and the download of the one
// before that. The caller keeps a buffer out of a lane copy while earlier queued work still uses it,
// or calls sci_cuda_join, a barrier between the lanes and the main stream in both directions.
namespace {
    int open_lanes(Context &ctx) {
        if (ctx.upload_lane) return SCI_CUDA_OK;
        if (int code = ctx.check(cudaStreamCreateWithFlags(&ctx.upload_lane, cudaStreamNonBlocking), "upload lane")) return code;
        if (int code = ctx.check(cudaStreamCreateWithFlags(&ctx.download_lane, cudaStreamNonBlocking), "download lane"))
            return code;
        for (cudaEvent_t *event : {&ctx.uploaded, &ctx.downloaded, &ctx.main_point})
            if (int code = ctx.check(cudaEventCreateWithFlags(event, cudaEventDisableTiming), "lane event")) return code;
        return SCI_CUDA_OK;
    }
} // namespace

int sci_cuda_upload_lane(sci_cuda_context *context, void *device, const void *host, uint64_t bytes) {
    if (!context || (!device && bytes) || (!host && bytes)) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    if (int code = open_lanes(*context)) return code;
    if (int code = context->check(cudaMemcpyAsync(device, host, bytes, cudaMemcpyHostToDevice, context->upload_lane),
                                  "lane upload"))
        return code;
    if (int code = context->check(cudaEventRecord(context->uploaded, context->upload_lane), "lane upload event")) return code;
    return context->check(cudaStreamWaitEvent(context->stream, context->uploaded, 0), "main stream waits for the upload");
}

int sci_cuda_download_lane(sci_cuda_context *context, void *host, const void *device, uint64_t bytes) {
    if (!context || (!device && bytes) || (!host && bytes)) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    if (int code = open_lanes(*context)) return code;
    if (int code = context->check(cudaEventRecord(context->main_point, context->stream), "main stream point")) return code;
    if (int code = context->check(cudaStreamWaitEvent(context->download_lane, context->main_point, 0), "download lane waits"))
        return code;
    if (int code = context->check(cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, context->download_lane),
                                  "lane download"))
        return code;
    return context->check(cudaEventRecord(context->downloaded, context->download_lane), "lane download event");
}

int sci_cuda_join(sci_cuda_context *context) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (!context->upload_lane) return SCI_CUDA_OK;
    cudaSetDevice(context->device);
    if (int code = context->check(cudaStreamWaitEvent(context->stream, context->uploaded, 0), "join uploads")) return code;
    if (int code = context->check(cudaStreamWaitEvent(context->stream, context->downloaded, 0), "join downloads")) return code;
    // and the other way: lane copies queued after the join wait for the main stream's work before it
    if (int code = context->check(cudaEventRecord(context->main_point, context->stream), "join point")) return code;
    if (int code = context->check(cudaStreamWaitEvent(context->upload_lane, context->main_point, 0), "join upload lane"))
        return code;
    return context->check(cudaStreamWaitEvent(context->download_lane, context->main_point, 0), "join download lane");
}

int sci_cuda_execute(sci_cuda_context *context, const sci_chunk *chunk, void *output, uint64_t count) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (int code = validate(*context, chunk, false)) return code;
    if (count == 0) return SCI_CUDA_OK;
    cudaSetDevice(context->device);
    return dispatch(*context, *chunk, kEvaluate, 0, count, output, nullptr);
}

int sci_cuda_reduce_async(sci_cuda_context *context, const sci_chunk *chunk, uint32_t fold, uint64_t count,
                          double *device_result) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (int code = validate(*context, chunk, true)) return code;
    if (fold > SCI_FOLD_MAXIMUM) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown fold %u", fold);
    if (!device_result) return context->fail(SCI_CUDA_ERROR_INVALID, "null result");
    cudaSetDevice(context->device);
    if (count == 0) {
        const double empty = fold == SCI_FOLD_SUM ? 0.0 : std::numeric_limits<double>::quiet_NaN();
        *context->host_result = empty;
        return context->check(cudaMemcpyAsync(device_result, context->host_result, sizeof(double), cudaMemcpyHostToDevice,
                                              context->stream),
                              "writing an empty reduction");
    }
    return dispatch(*context, *chunk, kReduce, fold, count, nullptr, device_result);
}

int sci_cuda_reduce(sci_cuda_context *context, const sci_chunk *chunk, uint32_t fold, uint64_t count, double *result) {
    if (!context || !result) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (int code = validate(*context, chunk, true)) return code;
    if (fold > SCI_FOLD_MAXIMUM) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown fold %u", fold);
    if (count == 0) {
        // dispatch.cpp:109-111
        *result = fold == SCI_FOLD_SUM ? 0.0 : std::numeric_limits<double>::quiet_NaN();
        return SCI_CUDA_OK;
    }
    cudaSetDevice(context->device);
    if (int code = dispatch(*context, *chunk, kReduce, fold, count, nullptr, context->result)) return code;
    // the result and the status word in one copy
    if (int code = context->check(cudaMemcpyAsync(context->host_result, context->result, kResultBytes,
                                                  cudaMemcpyDeviceToHost, context->stream),
                                  "reading the reduction"))
        return code;
    if (int code = context->drain(true)) return code;
    *result = *context->host_result;
    return SCI_CUDA_OK;
}

} // extern "C"
