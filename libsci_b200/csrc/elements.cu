// elements.cu -- chunks over integer arrays on the device.
//
// libsci records bytecode only for float and double (core::native, traits.hpp:26); an array of any
// other element type evaluates its expression tree on the host, one element at a time, with the
// scalar semantics of array::calculate<code, element> (calculate.hpp:17-93), in assign()
// (expression.hpp:178-184) and reduce() (expression.hpp:203-220). Here the same expression, recorded
// into the same bytecode, runs on the GPU for the eight integer types:
//   - copy, negate, absolute, add, subtract, multiply, fuse: two's-complement arithmetic in the
//     element's width (calculate.hpp:20-24,81-85,95), wrapping where C++ leaves signed overflow
//     undefined;
//   - divide truncates toward zero (calculate.hpp:86-87); a zero divisor gives 0 and MIN / -1 gives
//     MIN here, where C++ leaves both undefined;
//   - minimum, maximum: beta < alpha ? beta : alpha and beta > alpha ? beta : alpha (:88-91);
//   - the 27 real functions take the element to double, evaluate in double exactly as written in
//     calculate.hpp:25-80 (csc = 1.0 / sin(x), acsc = asin(1.0 / x), ...) and convert back by
//     truncation; a NaN gives 0 and values beyond the element's range saturate, where C++ leaves the
//     conversion undefined;
//   - sum wraps in the element's width, minimum and maximum are exact, and an empty reduction is
//     element{} = 0 (expression.hpp:205).
// Integer sums, minima and maxima do not depend on the order of the fold, so every result is
// bit-identical to the host loop's, whatever the launch shape.
//
// Kernel: a persistent grid-stride interpreter. A thread owns 16 contiguous bytes of every input
// per tile (16 int8 ... 2 int64), read and written as one 128-bit access when the arrays are
// 16-byte aligned; temporaries live in a shared-memory slot file (16 bytes per thread per
// temporary), the output slot in registers. Each instruction is a warp-uniform switch. Reductions
// fold lanes in a 64-bit carrier, then the warp (shuffles) and the block, and one atomic per block
// lands in the context's 8-byte result word. HBM-bound for the arithmetic codes; the real
// functions are bound by the FP64 pipe.
#include "context.hpp"

#include <cuda_runtime.h>

#include <cstring>
#include <limits>
#include <type_traits>

using namespace sci_cuda;

namespace sci_cuda {
    namespace {

        struct ElementStep {
            unsigned char code, target, a, b, c;
        };

        template <typename T> struct ElementLaunch {
            ElementStep steps[kCapacity];
            unsigned length;
            unsigned result;       // value id reduced (reduce launches)
            unsigned reduce;       // 0 evaluate, 1 reduce
            unsigned fold;         // SCI_FOLD_*
            unsigned vectors;      // inputs and output are 16-byte aligned
            T constants[kCapacity];
            const T *inputs[kCapacity];
            T *output;
            unsigned long long count;
            unsigned long long *accumulator;
        };

        // Arithmetic word: the element's width promoted to at least 32 bits, unsigned, so every
        // wrap is defined.
        template <typename T> using Word = std::conditional_t<sizeof(T) <= 4, unsigned, unsigned long long>;
        // Fold carrier: the element widened to 64 bits with its signedness, so order is preserved.
        template <typename T> using Carrier = std::conditional_t<std::is_signed<T>::value, long long, unsigned long long>;

        template <typename T> __device__ __forceinline__ T quotient(T a, T b) {
            if (b == T(0)) return T(0);
            if constexpr (std::is_signed<T>::value) {
                if (b == T(-1)) return T(Word<T>(0) - Word<T>(a));  // MIN / -1 wraps to MIN
            }
            return T(a / b);
        }

        template <typename T> __device__ __forceinline__ T from_real(double x) {
            constexpr T lo = std::numeric_limits<T>::min(), hi = std::numeric_limits<T>::max();
            if (x != x) return T(0);
            if (x <= static_cast<double>(lo)) return lo;
            if (x >= static_cast<double>(hi)) return hi;
            return static_cast<T>(x);  // truncation toward zero
        }

        // Out of line: called once per lane, so the lane loop does not repeat the whole table.
        __device__ __noinline__ double real(int code, double x) {
            switch (code) {
            case SCI_CODE_ROOT: return sqrt(x);
            case SCI_CODE_EXPONENTIAL: return exp(x);
            case SCI_CODE_LOGARITHM: return log(x);
            case SCI_CODE_SIN: return sin(x);
            case SCI_CODE_COS: return cos(x);
            case SCI_CODE_TAN: return tan(x);
            case SCI_CODE_ASIN: return asin(x);
            case SCI_CODE_ACOS: return acos(x);
            case SCI_CODE_ATAN: return atan(x);
            case SCI_CODE_CSC: return 1.0 / sin(x);
            case SCI_CODE_SEC: return 1.0 / cos(x);
            case SCI_CODE_COT: return 1.0 / tan(x);
            case SCI_CODE_ACSC: return asin(1.0 / x);
            case SCI_CODE_ASEC: return acos(1.0 / x);
            case SCI_CODE_ACOT: return atan(1.0 / x);
            case SCI_CODE_SINH: return sinh(x);
            case SCI_CODE_COSH: return cosh(x);
            case SCI_CODE_TANH: return tanh(x);
            case SCI_CODE_ASINH: return asinh(x);
            case SCI_CODE_ACOSH: return acosh(x);
            case SCI_CODE_ATANH: return atanh(x);
            case SCI_CODE_CSCH: return 1.0 / sinh(x);
            case SCI_CODE_SECH: return 1.0 / cosh(x);
            case SCI_CODE_COTH: return 1.0 / tanh(x);
            case SCI_CODE_ACSCH: return asinh(1.0 / x);
            case SCI_CODE_ASECH: return acosh(1.0 / x);
            default: return atanh(1.0 / x);  // SCI_CODE_ACOTH
            }
        }

        template <typename T> struct ElementLanes {
            static constexpr int count = 16 / sizeof(T);
        };

        // One instruction over a thread's lanes; the switch is warp-uniform and sits outside the
        // lane loop.
        template <typename T> __device__ __forceinline__ void integer_lanes(int code, const T *a, const T *b, const T *c, T *r) {
            constexpr int K = ElementLanes<T>::count;
            using W = Word<T>;
            switch (code) {
            case SCI_CODE_COPY:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = a[e];
                break;
            case SCI_CODE_NEGATE:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = T(W(0) - W(a[e]));
                break;
            case SCI_CODE_ABSOLUTE:
#pragma unroll
                for (int e = 0; e < K; ++e) {
                    if constexpr (std::is_signed<T>::value) r[e] = a[e] < T(0) ? T(W(0) - W(a[e])) : a[e];
                    else r[e] = a[e];
                }
                break;
            case SCI_CODE_ADD:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = T(W(a[e]) + W(b[e]));
                break;
            case SCI_CODE_SUBTRACT:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = T(W(a[e]) - W(b[e]));
                break;
            case SCI_CODE_MULTIPLY:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = T(W(a[e]) * W(b[e]));
                break;
            case SCI_CODE_DIVIDE:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = quotient(a[e], b[e]);
                break;
            case SCI_CODE_MINIMUM:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = b[e] < a[e] ? b[e] : a[e];
                break;
            case SCI_CODE_MAXIMUM:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = b[e] > a[e] ? b[e] : a[e];
                break;
            case SCI_CODE_FUSE:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = T(W(a[e]) * W(b[e]) + W(c[e]));
                break;
            default:
#pragma unroll
                for (int e = 0; e < K; ++e) r[e] = from_real<T>(real(code, static_cast<double>(a[e])));
                break;
            }
        }

        template <typename T>
        __device__ __forceinline__ void element_fetch(const ElementLaunch<T> &L, unsigned id, unsigned long long first,
                                                      bool full, const T *slots, const T *out, T *v) {
            constexpr int K = ElementLanes<T>::count;
            const unsigned kind = id & kTypes, slot = id & 63;
            if (kind == kInput) {
                const T *src = L.inputs[slot] + first;
                if (full && L.vectors) {
                    const uint4 word = *reinterpret_cast<const uint4 *>(src);
                    memcpy(v, &word, 16);
                } else {
#pragma unroll
                    for (int e = 0; e < K; ++e) v[e] = first + e < L.count ? src[e] : T(0);
                }
            } else if (kind == kLiteral) {
#pragma unroll
                for (int e = 0; e < K; ++e) v[e] = L.constants[slot];
            } else if (id == kOutput) {
#pragma unroll
                for (int e = 0; e < K; ++e) v[e] = out[e];
            } else if (id != kNone) {
                const uint4 word = *reinterpret_cast<const uint4 *>(slots + (slot * blockDim.x + threadIdx.x) * K);
                memcpy(v, &word, 16);
            } else {
#pragma unroll
                for (int e = 0; e < K; ++e) v[e] = T(0);
            }
        }

        template <typename T> __device__ __forceinline__ Carrier<T> fold_two(unsigned fold, Carrier<T> x, Carrier<T> y) {
            if (fold == SCI_FOLD_SUM) return Carrier<T>(static_cast<unsigned long long>(x) + static_cast<unsigned long long>(y));
            if (fold == SCI_FOLD_MINIMUM) return y < x ? y : x;
            return y > x ? y : x;
        }

        template <typename T> __device__ __forceinline__ Carrier<T> fold_identity(unsigned fold) {
            if (fold == SCI_FOLD_SUM) return Carrier<T>(0);
            if (fold == SCI_FOLD_MINIMUM) return std::numeric_limits<Carrier<T>>::max();
            return std::numeric_limits<Carrier<T>>::min();
        }

        template <typename T> __global__ void element_seed(unsigned long long *accumulator, unsigned fold) {
            *accumulator = static_cast<unsigned long long>(fold_identity<T>(fold));
        }

        template <typename T> __global__ void __launch_bounds__(256) element_stream(const __grid_constant__ ElementLaunch<T> L) {
            constexpr int K = ElementLanes<T>::count;
            extern __shared__ uint4 element_slots[];
            T *slots = reinterpret_cast<T *>(element_slots);
            const unsigned long long tile = 1ull * K * blockDim.x;
            Carrier<T> total = fold_identity<T>(L.fold);
            for (unsigned long long base = 1ull * blockIdx.x * tile; base < L.count; base += 1ull * gridDim.x * tile) {
                const unsigned long long first = base + 1ull * threadIdx.x * K;
                const bool full = first + K <= L.count;
                T out[K];
#pragma unroll
                for (int e = 0; e < K; ++e) out[e] = T(0);
                for (unsigned i = 0; i < L.length; ++i) {
                    const ElementStep st = L.steps[i];
                    T a[K], b[K], c[K], r[K];
                    element_fetch(L, st.a, first, full, slots, out, a);
                    element_fetch(L, st.b, first, full, slots, out, b);
                    element_fetch(L, st.c, first, full, slots, out, c);
                    integer_lanes<T>(st.code, a, b, c, r);
                    if (st.target == kOutput) {
#pragma unroll
                        for (int e = 0; e < K; ++e) out[e] = r[e];
                    } else {
                        uint4 word;
                        memcpy(&word, r, 16);
                        *reinterpret_cast<uint4 *>(slots + ((st.target & 63) * blockDim.x + threadIdx.x) * K) = word;
                    }
                }
                if (L.reduce) {
                    T v[K];
                    element_fetch(L, L.result, first, full, slots, out, v);
#pragma unroll
                    for (int e = 0; e < K; ++e)
                        if (first + e < L.count) total = fold_two<T>(L.fold, total, static_cast<Carrier<T>>(v[e]));
                } else if (first < L.count) {
                    T *dst = L.output + first;
                    if (full && L.vectors) {
                        uint4 word;
                        memcpy(&word, out, 16);
                        *reinterpret_cast<uint4 *>(dst) = word;
                    } else {
#pragma unroll
                        for (int e = 0; e < K; ++e)
                            if (first + e < L.count) dst[e] = out[e];
                    }
                }
            }
            if (!L.reduce) return;
            // warp, then block, then one atomic per block
#pragma unroll
            for (int offset = 16; offset > 0; offset >>= 1)
                total = fold_two<T>(L.fold, total, __shfl_xor_sync(0xffffffffu, total, offset));
            __shared__ Carrier<T> warps[32];
            const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, count = (blockDim.x + 31) >> 5;
            if (lane == 0) warps[warp] = total;
            __syncthreads();
            if (warp == 0) {
                total = lane < count ? warps[lane] : fold_identity<T>(L.fold);
#pragma unroll
                for (int offset = 16; offset > 0; offset >>= 1)
                    total = fold_two<T>(L.fold, total, __shfl_xor_sync(0xffffffffu, total, offset));
                if (lane == 0) {
                    if (L.fold == SCI_FOLD_SUM) {
                        atomicAdd(L.accumulator, static_cast<unsigned long long>(total));
                    } else if constexpr (std::is_signed<T>::value) {
                        long long *word = reinterpret_cast<long long *>(L.accumulator);
                        if (L.fold == SCI_FOLD_MINIMUM) atomicMin(word, static_cast<long long>(total));
                        else atomicMax(word, static_cast<long long>(total));
                    } else {
                        if (L.fold == SCI_FOLD_MINIMUM) atomicMin(L.accumulator, static_cast<unsigned long long>(total));
                        else atomicMax(L.accumulator, static_cast<unsigned long long>(total));
                    }
                }
            }
        }

        bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

        // Fills the launch, picks the block size from the slot file's size and runs one pass.
        template <typename T>
        int run_elements(Context &ctx, const sci_chunk &chunk, bool reducing, uint32_t fold, uint64_t count, void *output,
                         void *result) {
            ElementLaunch<T> L{};
            L.length = chunk.length;
            L.result = chunk.result;
            L.reduce = reducing ? 1 : 0;
            L.fold = fold;
            bool vectors = reducing || aligned16(output);
            for (int i = 0; i < chunk.length; ++i) {
                const sci_instruction &ins = chunk.instructions[i];
                L.steps[i] = ElementStep{ins.code, ins.target, ins.sources[0], ins.sources[1], ins.sources[2]};
            }
            for (int i = 0; i < chunk.literals; ++i) L.constants[i] = static_cast<T>(chunk.constants[i]);
            for (int i = 0; i < chunk.arguments; ++i) {
                L.inputs[i] = static_cast<const T *>(chunk.inputs[i]);
                vectors = vectors && aligned16(chunk.inputs[i]);
            }
            L.vectors = vectors ? 1 : 0;
            L.output = static_cast<T *>(output);
            L.count = count;
            L.accumulator = reinterpret_cast<unsigned long long *>(ctx.result);

            const void *kernel = reinterpret_cast<const void *>(&element_stream<T>);
            int threads = 256;
            size_t smem = static_cast<size_t>(chunk.temporaries) * 16 * threads;
            if (smem > 48 * 1024) {
                threads = 128;
                smem = static_cast<size_t>(chunk.temporaries) * 16 * threads;
            }
            if (smem > 48 * 1024) {
                if (smem > ctx.shared_limit) return ctx.fail(SCI_CUDA_ERROR_INVALID, "%u temporaries exceed shared memory", chunk.temporaries);
                if (int code = ctx.check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                              static_cast<int>(smem)),
                                         "element slot file"))
                    return code;
            }
            const unsigned long long tile = 1ull * ElementLanes<T>::count * threads;
            const unsigned long long tiles = (count + tile - 1) / tile;
            const unsigned long long most = 1ull * ctx.sms * ctx.blocks_per_sm(kernel, threads, smem);
            const unsigned grid = static_cast<unsigned>(tiles < most ? tiles : most);
            if (reducing) element_seed<T><<<1, 1, 0, ctx.stream>>>(L.accumulator, fold);
            element_stream<T><<<grid, threads, smem, ctx.stream>>>(L);
            if (int code = ctx.check(cudaGetLastError(), "launching an element chunk")) return code;
            if (!reducing) return SCI_CUDA_OK;
            if (int code = ctx.check(cudaMemcpyAsync(ctx.host_result, ctx.result, sizeof(double), cudaMemcpyDeviceToHost,
                                                     ctx.stream),
                                     "reading the element reduction"))
                return code;
            if (int code = ctx.drain()) return code;
            unsigned long long word;
            std::memcpy(&word, ctx.host_result, sizeof(word));
            const T value = static_cast<T>(word);  // low bits: the sum wraps in the element's width
            std::memcpy(result, &value, sizeof(T));
            return SCI_CUDA_OK;
        }

        template <typename F> int by_element(uint32_t element, F &&f) {
            switch (element) {
            case SCI_ELEMENT_INT8: return f(int8_t{});
            case SCI_ELEMENT_INT16: return f(int16_t{});
            case SCI_ELEMENT_INT32: return f(int32_t{});
            case SCI_ELEMENT_INT64: return f(int64_t{});
            case SCI_ELEMENT_UINT8: return f(uint8_t{});
            case SCI_ELEMENT_UINT16: return f(uint16_t{});
            case SCI_ELEMENT_UINT32: return f(uint32_t{});
            case SCI_ELEMENT_UINT64: return f(uint64_t{});
            default: return SCI_CUDA_ERROR_INVALID;
            }
        }

        size_t element_size(uint32_t element) {
            switch (element) {
            case SCI_ELEMENT_FLOAT32: return 4;
            case SCI_ELEMENT_FLOAT64: return 8;
            case SCI_ELEMENT_INT8: case SCI_ELEMENT_UINT8: return 1;
            case SCI_ELEMENT_INT16: case SCI_ELEMENT_UINT16: return 2;
            case SCI_ELEMENT_INT32: case SCI_ELEMENT_UINT32: return 4;
            case SCI_ELEMENT_INT64: case SCI_ELEMENT_UINT64: return 8;
            default: return 0;
            }
        }

    } // namespace
} // namespace sci_cuda

extern "C" {

uint64_t sci_cuda_element_size(uint32_t element) { return element_size(element); }

int sci_cuda_execute_elements(sci_cuda_context *context, uint32_t element, const sci_chunk *chunk, void *output,
                              uint64_t count) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (element_size(element) == 0) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown element type %u", element);
    if (element <= SCI_ELEMENT_FLOAT64) {
        if (!chunk) return context->fail(SCI_CUDA_ERROR_INVALID, "null chunk");
        sci_chunk native = *chunk;
        native.precision = static_cast<uint8_t>(element);
        return sci_cuda_execute(context, &native, output, count);
    }
    if (int code = validate(*context, chunk, false)) return code;
    if (count == 0) return SCI_CUDA_OK;
    for (int i = 0; i < chunk->arguments; ++i)
        if (!chunk->inputs[i] || !reachable(*context, chunk->inputs[i]))
            return context->fail(SCI_CUDA_ERROR_INVALID, "input %d is not memory of this device", i);
    if (!output || !reachable(*context, output)) return context->fail(SCI_CUDA_ERROR_INVALID, "the output is not memory of this device");
    cudaSetDevice(context->device);
    return by_element(element, [&](auto tag) { return run_elements<decltype(tag)>(*context, *chunk, false, 0, count, output, nullptr); });
}

int sci_cuda_reduce_elements(sci_cuda_context *context, uint32_t element, const sci_chunk *chunk, uint32_t fold,
                             uint64_t count, void *result) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (element_size(element) == 0) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown element type %u", element);
    if (!result) return context->fail(SCI_CUDA_ERROR_INVALID, "null result");
    if (fold > SCI_FOLD_MAXIMUM) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown fold %u", fold);
    if (element <= SCI_ELEMENT_FLOAT64) {
        if (!chunk) return context->fail(SCI_CUDA_ERROR_INVALID, "null chunk");
        sci_chunk native = *chunk;
        native.precision = static_cast<uint8_t>(element);
        double folded = 0.0;
        if (int code = sci_cuda_reduce(context, &native, fold, count, &folded)) return code;
        if (element == SCI_ELEMENT_FLOAT32) {
            const float narrow = static_cast<float>(folded);  // static_cast<element> (expression.hpp:198)
            std::memcpy(result, &narrow, sizeof(narrow));
        } else {
            std::memcpy(result, &folded, sizeof(folded));
        }
        return SCI_CUDA_OK;
    }
    if (int code = validate(*context, chunk, true)) return code;
    if (count == 0) {
        std::memset(result, 0, element_size(element));  // element{} (expression.hpp:205)
        return SCI_CUDA_OK;
    }
    for (int i = 0; i < chunk->arguments; ++i)
        if (!chunk->inputs[i] || !reachable(*context, chunk->inputs[i]))
            return context->fail(SCI_CUDA_ERROR_INVALID, "input %d is not memory of this device", i);
    cudaSetDevice(context->device);
    return by_element(element, [&](auto tag) { return run_elements<decltype(tag)>(*context, *chunk, true, fold, count, nullptr, result); });
}

} // extern "C"
