// broadcast.cu -- elementwise operations over operands of different shapes, and the elementwise
// functions libsci lists as next on its roadmap (README.md:149-152: broadcasting, "so (3, 1) and
// (1, 4) arrays combine into (3, 4)"; power, floor, ceil, round, clip and where).
//
// libsci has none of these yet, so the rules are numpy's, which its operations are named after
// (include/operations/reduce.hpp:8-9):
//   - shapes: every operand has the output's rank (the caller prepends 1s), and each of its extents
//     equals the output's or is 1 (a broadcast axis, read with stride 0);
//   - add / subtract / multiply / divide: one IEEE operation, rounded once;
//   - minimum / maximum: numpy.minimum / maximum, a NaN in either operand gives NaN, and of two
//     equal values (+0 and -0) the second;
//   - floor, ceil: exact; round: numpy.round, halves to even;
//   - power: C pow; a float is raised in double and rounded once (within 1 ulp of powf);
//   - clip(x, lo, hi) = minimum(maximum(x, lo), hi), as numpy.clip;
//   - where(condition, x, y) = condition != 0 ? x : y (NaN counts as true, as in numpy).
//
// Kernels: the host merges adjacent axes that every operand reads alike (both broadcast or both
// full), so most calls reduce to one or two axes (a same-shape or scalar operation to one). When
// the last merged axis is long, blocks walk (row, piece of the last axis) pairs: the row's offsets
// are computed once per piece and the piece is read and written contiguously (stride 0 or 1 per
// operand) -- in 16-byte vectors, two per thread, with the code a template argument, when the axis
// is a whole number of vectors and the arrays are 16-byte aligned; element by element otherwise.
// Short last axes map each thread's flat index to every operand's offset. HBM bound: bytes = the output written + each operand read once
// (a broadcast operand mostly from L2).
#include "context.hpp"

#include <cuda_runtime.h>

#include <cmath>

using namespace sci_cuda;

namespace sci_cuda {
    namespace {

        constexpr int kMaxAxes = 8;
        constexpr unsigned kPiece = 1024;
        constexpr int kVectorsPerThread = 2;  // 16-byte vectors per thread per piece (vector form)

        template <typename T> struct ApplyLaunch {
            int code;
            int rank;                                       // merged axes
            unsigned long long extent[kMaxAxes];            // merged output extents
            unsigned long long stride[3][kMaxAxes];         // element strides (0 on broadcast axes)
            const T *input[3];
            T *output;
            unsigned long long count;
        };

        // numpy's minimum / maximum: the first operand if it is NaN or strictly smaller (larger),
        // else the second (so a NaN second operand, and the second of two equal values, win).
        template <typename T> __device__ __forceinline__ T nan_minimum(T a, T b) { return (a < b || a != a) ? a : b; }
        template <typename T> __device__ __forceinline__ T nan_maximum(T a, T b) { return (a > b || a != a) ? a : b; }

        __device__ __forceinline__ float quotient(float a, float b) { return __fdiv_rn(a, b); }
        __device__ __forceinline__ double quotient(double a, double b) { return __ddiv_rn(a, b); }
        __device__ __forceinline__ float raise(float a, float b) {
            return __double2float_rn(pow(static_cast<double>(a), static_cast<double>(b)));
        }
        __device__ __forceinline__ double raise(double a, double b) { return pow(a, b); }

        template <typename T> __device__ __forceinline__ T apply_shaped(int code, T a, T b, T c) {
            switch (code) {  // with a constant code (the vector kernel) the switch folds away
            case SCI_CODE_COPY: return a;
            case SCI_CODE_ADD: return add(a, b);
            case SCI_CODE_SUBTRACT: return sub(a, b);
            case SCI_CODE_MULTIPLY: return mul(a, b);
            case SCI_CODE_DIVIDE: return quotient(a, b);
            case SCI_CODE_MINIMUM: return nan_minimum(a, b);
            case SCI_CODE_MAXIMUM: return nan_maximum(a, b);
            case SCI_EXTRA_FLOOR: return floor(a);
            case SCI_EXTRA_CEIL: return ceil(a);
            case SCI_EXTRA_ROUND: return rint(a);
            case SCI_EXTRA_POWER: return raise(a, b);
            case SCI_EXTRA_CLIP: return nan_minimum(nan_maximum(a, b), c);
            default: return a != T(0) ? b : c;  // SCI_EXTRA_WHERE
            }
        }

        template <typename T> __device__ __forceinline__ T operand(const ApplyLaunch<T> &L, int k, unsigned long long offset) {
            return L.input[k] ? L.input[k][offset] : T(0);
        }

        // Flat: one element per thread per step, offsets from the flat index.
        template <typename T> __global__ void __launch_bounds__(256) apply_flat(const __grid_constant__ ApplyLaunch<T> L) {
            const unsigned long long step = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < L.count; i += step) {
                unsigned long long rest = i, offset[3] = {0, 0, 0};
                for (int axis = L.rank - 1; axis >= 0; --axis) {
                    const unsigned long long coordinate = rest % L.extent[axis];
                    rest /= L.extent[axis];
#pragma unroll
                    for (int k = 0; k < 3; ++k) offset[k] += coordinate * L.stride[k][axis];
                }
                L.output[i] = apply_shaped<T>(L.code, operand(L, 0, offset[0]), operand(L, 1, offset[1]), operand(L, 2, offset[2]));
            }
        }

        // Rows: (row, piece of the last axis) per block step; the last axis is read with stride 0
        // or 1 per operand.
        template <typename T> __global__ void __launch_bounds__(256) apply_rows(const __grid_constant__ ApplyLaunch<T> L) {
            const int last = L.rank - 1;
            const unsigned long long columns = L.extent[last];
            const unsigned long long chunks = (columns + kPiece - 1) / kPiece;
            const unsigned long long rows = L.count / columns, pieces = rows * chunks;
            for (unsigned long long piece = blockIdx.x; piece < pieces; piece += gridDim.x) {
                const unsigned long long row = piece / chunks, c0 = (piece - row * chunks) * kPiece;
                unsigned long long rest = row, base[3] = {0, 0, 0};
                for (int axis = last - 1; axis >= 0; --axis) {
                    const unsigned long long coordinate = rest % L.extent[axis];
                    rest /= L.extent[axis];
#pragma unroll
                    for (int k = 0; k < 3; ++k) base[k] += coordinate * L.stride[k][axis];
                }
                T *out = L.output + row * columns;
                for (unsigned long long c = c0 + threadIdx.x; c < c0 + kPiece && c < columns; c += blockDim.x) {
                    out[c] = apply_shaped<T>(L.code, operand(L, 0, base[0] + c * L.stride[0][last]),
                                             operand(L, 1, base[1] + c * L.stride[1][last]),
                                             operand(L, 2, base[2] + c * L.stride[2][last]));
                }
            }
        }

        // Vectors: the last axis in 16-byte vectors, two per thread per piece. Taken when the last
        // axis is a whole number of vectors and every array is 16-byte aligned, so each row of the
        // output and of every operand read along the last axis starts on a vector; an operand
        // broadcast along the last axis is one value per row. The code is a template argument.
        template <typename T, int CODE>
        __global__ void __launch_bounds__(256) apply_vectors(const __grid_constant__ ApplyLaunch<T> L) {
            constexpr int V = 16 / sizeof(T), U = kVectorsPerThread;
            const int last = L.rank - 1;
            const unsigned long long columns = L.extent[last];
            const unsigned long long span = 1ull * blockDim.x * V * U;
            const unsigned long long chunks = (columns + span - 1) / span;
            const unsigned long long pieces = (L.count / columns) * chunks;
            for (unsigned long long piece = blockIdx.x; piece < pieces; piece += gridDim.x) {
                const unsigned long long row = piece / chunks, c0 = (piece - row * chunks) * span;
                unsigned long long rest = row, base[3] = {0, 0, 0};
                for (int axis = last - 1; axis >= 0; --axis) {
                    const unsigned long long coordinate = rest % L.extent[axis];
                    rest /= L.extent[axis];
#pragma unroll
                    for (int k = 0; k < 3; ++k) base[k] += coordinate * L.stride[k][axis];
                }
                T v[3][U][V];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const bool along = L.stride[k][last] != 0;
                    const T single = (L.input[k] && !along) ? L.input[k][base[k]] : T(0);
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const unsigned long long c = c0 + (1ull * u * blockDim.x + threadIdx.x) * V;
                        if (along && c < columns) {
                            load16(L.input[k] + base[k] + c, v[k][u]);
                        } else {
#pragma unroll
                            for (int e = 0; e < V; ++e) v[k][u][e] = single;
                        }
                    }
                }
                T *out = L.output + row * columns;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const unsigned long long c = c0 + (1ull * u * blockDim.x + threadIdx.x) * V;
                    if (c >= columns) continue;
                    T r[V];
#pragma unroll
                    for (int e = 0; e < V; ++e) r[e] = apply_shaped<T>(CODE, v[0][u][e], v[1][u][e], v[2][u][e]);
                    store16(out + c, r);
                }
            }
        }

        template <typename T, int CODE> void launch_vectors(Context &ctx, const ApplyLaunch<T> &L) {
            constexpr int V = 16 / sizeof(T);
            const unsigned long long columns = L.extent[L.rank - 1], span = 256ull * V * kVectorsPerThread;
            const unsigned long long pieces = (L.count / columns) * ((columns + span - 1) / span);
            // one wave: as many blocks as stay resident
            const unsigned long long most =
                    1ull * ctx.sms * ctx.blocks_per_sm(reinterpret_cast<const void *>(&apply_vectors<T, CODE>), 256, 0);
            apply_vectors<T, CODE><<<static_cast<unsigned>(pieces < most ? pieces : most), 256, 0, ctx.stream>>>(L);
        }

        template <typename T> bool launch_vector_code(Context &ctx, const ApplyLaunch<T> &L) {
            switch (L.code) {
            case SCI_CODE_COPY: launch_vectors<T, SCI_CODE_COPY>(ctx, L); return true;
            case SCI_CODE_ADD: launch_vectors<T, SCI_CODE_ADD>(ctx, L); return true;
            case SCI_CODE_SUBTRACT: launch_vectors<T, SCI_CODE_SUBTRACT>(ctx, L); return true;
            case SCI_CODE_MULTIPLY: launch_vectors<T, SCI_CODE_MULTIPLY>(ctx, L); return true;
            case SCI_CODE_DIVIDE: launch_vectors<T, SCI_CODE_DIVIDE>(ctx, L); return true;
            case SCI_CODE_MINIMUM: launch_vectors<T, SCI_CODE_MINIMUM>(ctx, L); return true;
            case SCI_CODE_MAXIMUM: launch_vectors<T, SCI_CODE_MAXIMUM>(ctx, L); return true;
            case SCI_EXTRA_FLOOR: launch_vectors<T, SCI_EXTRA_FLOOR>(ctx, L); return true;
            case SCI_EXTRA_CEIL: launch_vectors<T, SCI_EXTRA_CEIL>(ctx, L); return true;
            case SCI_EXTRA_ROUND: launch_vectors<T, SCI_EXTRA_ROUND>(ctx, L); return true;
            case SCI_EXTRA_POWER: launch_vectors<T, SCI_EXTRA_POWER>(ctx, L); return true;
            case SCI_EXTRA_CLIP: launch_vectors<T, SCI_EXTRA_CLIP>(ctx, L); return true;
            case SCI_EXTRA_WHERE: launch_vectors<T, SCI_EXTRA_WHERE>(ctx, L); return true;
            default: return false;
            }
        }

        bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

        int arity(uint32_t code) {
            switch (code) {
            case SCI_CODE_COPY: case SCI_EXTRA_FLOOR: case SCI_EXTRA_CEIL: case SCI_EXTRA_ROUND: return 1;
            case SCI_CODE_ADD: case SCI_CODE_SUBTRACT: case SCI_CODE_MULTIPLY: case SCI_CODE_DIVIDE:
            case SCI_CODE_MINIMUM: case SCI_CODE_MAXIMUM: case SCI_EXTRA_POWER: return 2;
            case SCI_EXTRA_CLIP: case SCI_EXTRA_WHERE: return 3;
            default: return 0;
            }
        }

        template <typename T>
        int launch_apply(Context &ctx, uint32_t code, int rank, const unsigned long long *extent,
                         const unsigned long long (*stride)[kMaxAxes], const void *const *inputs, int operands, void *output,
                         unsigned long long count) {
            ApplyLaunch<T> L{};
            L.code = static_cast<int>(code);
            L.rank = rank;
            for (int a = 0; a < rank; ++a) L.extent[a] = extent[a];
            for (int k = 0; k < operands; ++k) {
                L.input[k] = static_cast<const T *>(inputs[k]);
                for (int a = 0; a < rank; ++a) L.stride[k][a] = stride[k][a];
            }
            L.output = static_cast<T *>(output);
            L.count = count;
            const unsigned long long columns = extent[rank - 1];
            bool vectors = columns % (16 / sizeof(T)) == 0 && aligned16(output);
            for (int k = 0; k < operands; ++k) vectors = vectors && aligned16(inputs[k]);
            if (vectors && columns >= 64 && launch_vector_code<T>(ctx, L)) {
                return ctx.check(cudaGetLastError(), "launching a broadcast operation");
            }
            if (columns >= 256) {
                const unsigned long long pieces = (count / columns) * ((columns + kPiece - 1) / kPiece);
                const unsigned long long most = 8ull * ctx.sms;
                apply_rows<T><<<static_cast<unsigned>(pieces < most ? pieces : most), 256, 0, ctx.stream>>>(L);
            } else {
                const unsigned long long wanted = (count + 255) / 256, most = 8ull * ctx.sms;
                apply_flat<T><<<static_cast<unsigned>(wanted < most ? wanted : most), 256, 0, ctx.stream>>>(L);
            }
            return ctx.check(cudaGetLastError(), "launching a broadcast operation");
        }

    } // namespace
} // namespace sci_cuda

extern "C" int sci_cuda_broadcast(sci_cuda_context *context, uint32_t precision, uint32_t code, uint32_t rank,
                                  const uint64_t *shape, uint32_t operands, const void *const *inputs,
                                  const uint64_t *input_shapes, void *output) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u", precision);
    if (arity(code) == 0) return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: unknown code %u", code);
    if (static_cast<int>(operands) != arity(code))
        return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: code %u takes %d operands, not %u", code, arity(code), operands);
    if (rank < 1 || rank > static_cast<uint32_t>(kMaxAxes) || !shape || !inputs || !input_shapes)
        return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: rank %u (1 to %d, with shapes)", rank, kMaxAxes);
    unsigned long long count = 1;
    for (uint32_t a = 0; a < rank; ++a) {
        if (shape[a] != 0 && count > ~0ull / shape[a]) return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: shape overflows");
        count *= shape[a];
    }
    for (uint32_t k = 0; k < operands; ++k)
        for (uint32_t a = 0; a < rank; ++a) {
            const uint64_t e = input_shapes[k * rank + a];
            if (e != shape[a] && e != 1)
                return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: operand %u axis %u has %llu, not 1 or %llu", k, a,
                                     static_cast<unsigned long long>(e), static_cast<unsigned long long>(shape[a]));
        }
    if (count == 0) return SCI_CUDA_OK;
    if (!output || !reachable(*context, output)) return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: the output is not memory of this device");
    for (uint32_t k = 0; k < operands; ++k) {
        if (!inputs[k] || !reachable(*context, inputs[k]))
            return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: operand %u is not memory of this device", k);
        if (inputs[k] == output) {
            // in place only when the operand is read exactly where it is written
            for (uint32_t a = 0; a < rank; ++a)
                if (input_shapes[k * rank + a] != shape[a])
                    return context->fail(SCI_CUDA_ERROR_INVALID, "broadcast: a broadcast operand cannot be the output");
        }
    }
    // Merge adjacent axes that every operand reads alike; drop axes of extent 1.
    unsigned long long extent[kMaxAxes], stride[3][kMaxAxes] = {};
    bool full[3][kMaxAxes];
    int merged = 0;
    for (uint32_t a = 0; a < rank; ++a) {
        if (shape[a] == 1) continue;
        bool same = merged > 0;
        for (uint32_t k = 0; k < operands && same; ++k) same = full[k][merged - 1] == (input_shapes[k * rank + a] != 1);
        if (same) {
            extent[merged - 1] *= shape[a];
        } else {
            extent[merged] = shape[a];
            for (uint32_t k = 0; k < operands; ++k) full[k][merged] = input_shapes[k * rank + a] != 1;
            ++merged;
        }
    }
    if (merged == 0) {
        extent[0] = 1;
        for (uint32_t k = 0; k < operands; ++k) full[k][0] = true;
        merged = 1;
    }
    for (uint32_t k = 0; k < operands; ++k) {
        unsigned long long s = 1;
        for (int a = merged - 1; a >= 0; --a) {
            stride[k][a] = full[k][a] ? s : 0;
            if (full[k][a]) s *= extent[a];
        }
    }
    cudaSetDevice(context->device);
    if (precision == SCI_PRECISION_WIDE)
        return launch_apply<double>(*context, code, merged, extent, stride, inputs, static_cast<int>(operands), output, count);
    return launch_apply<float>(*context, code, merged, extent, stride, inputs, static_cast<int>(operands), output, count);
}
