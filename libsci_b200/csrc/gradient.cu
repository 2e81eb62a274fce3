// gradient.cu -- sci::gradient: reverse-mode derivatives on sm_100a (no counterpart in the
// reference, which has no differentiation). Entry points:
//  - sci_cuda_gradient: dL/d(arguments) of L = seed * sum(chunk), by the adjoint kernels of
//    gradient_kernel.cuh (recomputing, or the temporary-storing comparison form);
//  - sci_cuda_product_gradient: the adjoints of linear::product (two products);
//  - sci_cuda_solve_gradient: the adjoints of linear::solve (one transposed solve that reuses the
//    forward solve's LU factors, and one outer product).
#include "context.hpp"
#include "gradient_kernel.cuh"
#include "specialize.hpp"
#include "workspace.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <iterator>

namespace sci_cuda {

    namespace {

        template <typename T, int FORM> const void *generic_gradient_kernel() {
            return reinterpret_cast<const void *>(&gradient_stream<T, Dynamic, FORM>);
        }
        const void *generic_gradient_kernel(bool wide, int form) {
            if (wide) {
                return form == kGradRecompute ? generic_gradient_kernel<double, kGradRecompute>()
                                              : (form == kGradRecord ? generic_gradient_kernel<double, kGradRecord>()
                                                                     : generic_gradient_kernel<double, kGradReplay>());
            }
            return form == kGradRecompute ? generic_gradient_kernel<float, kGradRecompute>()
                                          : (form == kGradRecord ? generic_gradient_kernel<float, kGradRecord>()
                                                                 : generic_gradient_kernel<float, kGradReplay>());
        }

        // The chunk in value form, packed into a sci_chunk so that the specialiser keys and bakes it
        // like any chunk: instruction s is node s (its target names itself), a temporary id in a
        // source names a node, `temporaries` counts the nodes and `result` names the summed value.
        // A source reading a temporary resolves to the slot's last writer before it (chunk.hpp
        // reuses a temporary once its value is consumed); instructions the result does not depend on
        // are dropped.
        int value_form(Context &ctx, const sci_chunk &chunk, sci_chunk &out) {
            constexpr int kNode = 0x100;
            int writer[SCI_CHUNK_CAPACITY];
            std::fill(std::begin(writer), std::end(writer), -1);
            int output_writer = -1;
            int refs[SCI_CHUNK_CAPACITY][3];
            auto resolve = [&](uint8_t id) -> int {
                if (id == SCI_SLOT_NONE) return SCI_SLOT_NONE;
                const int kind = id & SCI_SLOT_TYPES;
                if (kind == SCI_SLOT_TEMPORARY) return writer[id & 63] < 0 ? -1 : kNode + writer[id & 63];
                if (kind == SCI_SLOT_OUTPUT) return output_writer < 0 ? -1 : kNode + output_writer;
                return id;
            };
            for (int s = 0; s < chunk.length; ++s) {
                const sci_instruction &ins = chunk.instructions[s];
                const int arity = ins.code < SCI_CODE_ADD ? 1 : (ins.code < SCI_CODE_FUSE ? 2 : 3);
                for (int k = 0; k < 3; ++k) {
                    refs[s][k] = k < arity ? resolve(ins.sources[k]) : SCI_SLOT_NONE;
                    if (refs[s][k] < 0)
                        return ctx.fail(SCI_CUDA_ERROR_INVALID, "instruction %d reads 0x%02x before anything writes it", s,
                                        ins.sources[k]);
                }
                if (ins.target == SCI_SLOT_OUTPUT) output_writer = s;
                else writer[ins.target & 63] = s;
            }
            const int result = resolve(chunk.result);
            if (result < 0) return ctx.fail(SCI_CUDA_ERROR_INVALID, "the result 0x%02x is never written", chunk.result);
            bool keep[SCI_CHUNK_CAPACITY] = {};
            if (result >= kNode) keep[result - kNode] = true;
            for (int s = chunk.length - 1; s >= 0; --s) {
                if (!keep[s]) continue;
                for (int k = 0; k < 3; ++k)
                    if (refs[s][k] >= kNode) keep[refs[s][k] - kNode] = true;
            }
            int index[SCI_CHUNK_CAPACITY];
            int nodes = 0;
            for (int s = 0; s < chunk.length; ++s) index[s] = keep[s] ? nodes++ : -1;
            auto encode = [&](int ref) -> uint8_t {
                return static_cast<uint8_t>(ref >= kNode ? (SCI_SLOT_TEMPORARY | index[ref - kNode]) : ref);
            };
            out = chunk;
            std::memset(out.instructions, 0, sizeof(out.instructions));
            for (int s = 0; s < chunk.length; ++s) {
                if (!keep[s]) continue;
                sci_instruction &node = out.instructions[index[s]];
                node.code = chunk.instructions[s].code;
                node.target = static_cast<uint8_t>(SCI_SLOT_TEMPORARY | index[s]);
                for (int k = 0; k < 3; ++k) node.sources[k] = encode(refs[s][k]);
            }
            out.length = static_cast<uint8_t>(nodes);
            out.temporaries = static_cast<uint8_t>(nodes);
            out.result = encode(result);
            return SCI_CUDA_OK;
        }

        // Queues one gradient form over `count` elements. `value` (device) receives the sum in the
        // forward forms, or is null.
        template <typename T>
        int launch_gradient(Context &ctx, const sci_chunk &program, int form, uint64_t count, double seed,
                            void *const *gradients, T *tape, double *value) {
            GradientLaunch<T> L;
            std::memset(&L, 0, sizeof(L));
            for (int s = 0; s < program.length; ++s) {
                const sci_instruction &ins = program.instructions[s];
                L.steps[s] = Step{ins.code, ins.target, ins.sources[0], ins.sources[1], ins.sources[2]};
                if (ins.code == SCI_CODE_MINIMUM || ins.code == SCI_CODE_MAXIMUM) L.tailed = 1;
            }
            L.length = program.length;
            L.result = program.result;
            L.arguments = program.arguments;
            constexpr uint64_t width = 16 / sizeof(T);
            bool vector = count % width == 0;
            for (int i = 0; i < program.literals; ++i) L.constants[i] = static_cast<T>(program.constants[i]);
            for (int a = 0; a < program.arguments; ++a) {
                if (!program.inputs[a] || !reachable(ctx, program.inputs[a]))
                    return ctx.fail(SCI_CUDA_ERROR_INVALID, "input %d (%p) is not memory of this device", a, program.inputs[a]);
                L.inputs[a] = static_cast<const T *>(program.inputs[a]);
                vector = vector && reinterpret_cast<uintptr_t>(L.inputs[a]) % 16 == 0;
                if (gradients && gradients[a]) {
                    if (!reachable(ctx, gradients[a]))
                        return ctx.fail(SCI_CUDA_ERROR_INVALID, "gradient %d (%p) is not memory of this device", a, gradients[a]);
                    L.gradients[a] = static_cast<T *>(gradients[a]);
                    vector = vector && reinterpret_cast<uintptr_t>(L.gradients[a]) % 16 == 0;
                }
            }
            L.tape = tape;
            vector = vector && reinterpret_cast<uintptr_t>(tape) % 16 == 0;
            L.vector = vector ? 1u : 0u;
            L.seed = seed;
            L.count = count;
            L.tail_start = count - count % (64 / sizeof(T));  // the reference's loop tails (see device.cu)
            L.state = ctx.state;
            L.destination = value;

            const Specialized *special = ctx.specializer ? ctx.specializer->find(ctx, program, form) : nullptr;
            const int per_thread = special && program.length <= 16 ? static_cast<int>(width) : 1;
            const int threads = 256;
            const uint64_t groups = (count + per_thread - 1) / per_thread;
            const uint64_t wanted = (groups + threads - 1) / threads;
            void *args[] = {&L};
            if (special) {
                CUfunction function = reinterpret_cast<CUfunction>(const_cast<void *>(special->function));
                const auto key = std::make_tuple(special->function, threads, size_t(0));
                auto found = ctx.occupancy.find(key);
                int per_sm = 1;
                if (found != ctx.occupancy.end()) {
                    per_sm = found->second;
                } else {
                    if (Driver::get().occupancy(&per_sm, function, threads, 0) != CUDA_SUCCESS || per_sm < 1) per_sm = 1;
                    ctx.occupancy[key] = per_sm;
                }
                const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>({wanted, uint64_t(per_sm) * ctx.sms, kMaxBlocks}));
                const CUresult code = Driver::get().launch(function, static_cast<unsigned>(grid), 1, 1, threads, 1, 1, 0,
                                                           ctx.stream, args, nullptr);
                if (code != CUDA_SUCCESS)
                    return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "launching a specialised gradient kernel: %d", int(code));
                return SCI_CUDA_OK;
            }
            const void *kernel = generic_gradient_kernel(sizeof(T) == 8, form);
            const int per_sm = ctx.blocks_per_sm(kernel, threads, 0);
            const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>({wanted, uint64_t(per_sm) * ctx.sms, kMaxBlocks}));
            return ctx.check(cudaLaunchKernel(kernel, dim3(static_cast<unsigned>(grid)), dim3(threads), args, 0, ctx.stream),
                             "launching the gradient kernel");
        }

        template <typename T>
        int gradient(Context &ctx, const sci_chunk &program, uint64_t count, double seed, void *const *gradients,
                     double *value, uint32_t form) {
            if (form == SCI_GRADIENT_RECOMPUTE)
                return launch_gradient<T>(ctx, program, kGradRecompute, count, seed, gradients, nullptr, value);
            const size_t need = size_t(std::max<int>(program.length, 1)) * count * sizeof(T);
            if (int code = ctx.check(ctx.tape->reserve(need), "reserving the gradient tape")) return code;
            T *tape = static_cast<T *>(ctx.tape->memory);
            if (int code = launch_gradient<T>(ctx, program, kGradRecord, count, seed, gradients, tape, value)) return code;
            return launch_gradient<T>(ctx, program, kGradReplay, count, seed, gradients, tape, nullptr);
        }

    } // namespace

} // namespace sci_cuda

using namespace sci_cuda;

extern "C" int sci_cuda_gradient(sci_cuda_context *context, const sci_chunk *chunk, uint64_t count, double seed,
                                 void *const *gradients, double *value, uint32_t form) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (int code = validate(*context, chunk, true)) return code;
    if (form > SCI_GRADIENT_STORED) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown gradient form %u", form);
    if (count == 0) {
        if (value) *value = 0.0;  // an empty sum (dispatch.cpp:109-111)
        return SCI_CUDA_OK;
    }
    cudaSetDevice(context->device);
    sci_chunk program;
    if (int code = value_form(*context, *chunk, program)) return code;
    double *device_value = value ? context->result : nullptr;
    const int code = chunk->precision == SCI_PRECISION_WIDE
                             ? gradient<double>(*context, program, count, seed, gradients, device_value, form)
                             : gradient<float>(*context, program, count, seed, gradients, device_value, form);
    if (code || !value) return code;  // without a value the call is only queued
    if (int c = context->check(cudaMemcpyAsync(context->host_result, context->result, sizeof(double),
                                               cudaMemcpyDeviceToHost, context->stream),
                               "reading the sum"))
        return c;
    if (int c = context->drain()) return c;
    *value = *context->host_result;
    return SCI_CUDA_OK;
}
