// axis.cu -- reductions along one axis (libsci's roadmap, README.md:151: "sum(a, axis) and the
// rest"): sum, minimum, maximum and mean of a row-major array over one of its axes.
//
// The whole-array reductions set the rules (include/operations/reduce.hpp:16-42, dispatch.cpp:
// 106-165): values fold in double whatever the element type, a NaN anywhere in a fold gives NaN,
// the result is cast to the element type once, and mean is that sum divided by the count in the
// element type (sum / static_cast<element>(count), reduce.hpp:27). An empty axis gives 0 for sum
// and mean and NaN for minimum and maximum.
//
// The array is viewed as (outer, extent, inner): out[o][j] = fold over k of in[o][k][j].
//   - inner == 1 (the last axis): a warp per (row, piece of the row); lanes stride the piece
//     (coalesced) and fold with shuffles in a fixed order;
//   - inner > 1: a thread per (o, piece, j), j fastest, so a warp reads 32 consecutive elements
//     per k -- or, when inner is a whole number of 16-byte vectors, a thread per (o, piece, vector
//     of j) reading 512 bytes per warp per k (rows shorter than 64 take the scalar form, a thread
//     per row);
// Short outputs over long axes split the axis into pieces so the grid fills the GPU; pieces write
// double partials that one more pass folds in piece order. The order of every fold is fixed by the
// shape alone, so results are deterministic. HBM bound: the input is read once.
#include "context.hpp"
#include "workspace.hpp"

#include <cuda_runtime.h>

#include <limits>

using namespace sci_cuda;

namespace sci_cuda {
    namespace {

        __device__ __forceinline__ double fold_pair(unsigned fold, double a, double b) {
            if (fold == SCI_FOLD_SUM) return __dadd_rn(a, b);
            if (a != a) return a;
            if (b != b) return b;
            if (fold == SCI_FOLD_MINIMUM) return b < a ? b : a;
            return b > a ? b : a;
        }

        __device__ __forceinline__ double fold_start(unsigned fold) {
            if (fold == SCI_FOLD_SUM) return 0.0;
            return fold == SCI_FOLD_MINIMUM ? __longlong_as_double(0x7ff0000000000000ll)    // +inf
                                            : __longlong_as_double(0xfff0000000000000ll);  // -inf
        }

        // fold 3 is mean: the sum, then divided by the count in the element type.
        template <typename T> __device__ __forceinline__ T finish(unsigned fold, double value, unsigned long long extent);
        template <> __device__ __forceinline__ float finish<float>(unsigned fold, double value, unsigned long long extent) {
            const float narrow = __double2float_rn(value);
            return fold == 3 ? __fdiv_rn(narrow, __ull2float_rn(extent)) : narrow;
        }
        template <> __device__ __forceinline__ double finish<double>(unsigned fold, double value, unsigned long long extent) {
            return fold == 3 ? __ddiv_rn(value, __ull2double_rn(extent)) : value;
        }

        struct AxisShape {
            unsigned long long outer, extent, inner, pieces, span;  // span: k per piece
            unsigned fold;    // SCI_FOLD_* or 3 (mean)
            unsigned folded;  // the fold applied to values (mean folds as a sum)
        };

        template <typename T>
        __global__ void __launch_bounds__(256) axis_rows(const T *in, AxisShape s, double *partial, T *out) {
            const unsigned lane = threadIdx.x & 31;
            const unsigned long long warps = 1ull * gridDim.x * (blockDim.x >> 5);
            const unsigned long long units = s.outer * s.pieces;
            for (unsigned long long unit = 1ull * blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); unit < units; unit += warps) {
                const unsigned long long row = unit / s.pieces, piece = unit - row * s.pieces;
                const unsigned long long k0 = piece * s.span, k1 = k0 + s.span < s.extent ? k0 + s.span : s.extent;
                const T *line = in + row * s.extent;
                double acc = fold_start(s.folded);
#pragma unroll 4
                for (unsigned long long k = k0 + lane; k < k1; k += 32) acc = fold_pair(s.folded, acc, static_cast<double>(line[k]));
#pragma unroll
                for (int offset = 16; offset > 0; offset >>= 1)
                    acc = fold_pair(s.folded, acc, __shfl_xor_sync(0xffffffffu, acc, offset));
                if (lane == 0) {
                    if (s.pieces == 1) out[row] = finish<T>(s.fold, acc, s.extent);
                    else partial[unit] = acc;
                }
            }
        }

        template <typename T>
        __global__ void __launch_bounds__(256) axis_columns(const T *in, AxisShape s, double *partial, T *out) {
            const unsigned long long threads = 1ull * gridDim.x * blockDim.x;
            const unsigned long long units = s.outer * s.pieces * s.inner;
            for (unsigned long long unit = 1ull * blockIdx.x * blockDim.x + threadIdx.x; unit < units; unit += threads) {
                const unsigned long long j = unit % s.inner, rest = unit / s.inner;
                const unsigned long long piece = rest % s.pieces, o = rest / s.pieces;
                const unsigned long long k0 = piece * s.span, k1 = k0 + s.span < s.extent ? k0 + s.span : s.extent;
                const T *column = in + o * s.extent * s.inner + j;
                double acc = fold_start(s.folded);
                // unrolled so eight loads are in flight ahead of the (ordered) fold
#pragma unroll 8
                for (unsigned long long k = k0; k < k1; ++k) acc = fold_pair(s.folded, acc, static_cast<double>(column[k * s.inner]));
                if (s.pieces == 1) out[o * s.inner + j] = finish<T>(s.fold, acc, s.extent);
                else partial[unit] = acc;
            }
        }

        // The column form over 16-byte vectors of adjacent columns (inner a whole number of vectors,
        // input 16-byte aligned): a thread per (o, piece, vector of j), each lane folding its own
        // column in the same order as the scalar form.
        template <typename T>
        __global__ void __launch_bounds__(256) axis_column_vectors(const T *in, AxisShape s, double *partial, T *out) {
            constexpr int V = 16 / sizeof(T);
            const unsigned long long threads = 1ull * gridDim.x * blockDim.x;
            const unsigned long long groups = s.inner / V;
            const unsigned long long units = s.outer * s.pieces * groups;
            for (unsigned long long unit = 1ull * blockIdx.x * blockDim.x + threadIdx.x; unit < units; unit += threads) {
                const unsigned long long g = unit % groups, rest = unit / groups;
                const unsigned long long piece = rest % s.pieces, o = rest / s.pieces;
                const unsigned long long k0 = piece * s.span, k1 = k0 + s.span < s.extent ? k0 + s.span : s.extent;
                const T *column = in + o * s.extent * s.inner + g * V;
                double acc[V];
#pragma unroll
                for (int e = 0; e < V; ++e) acc[e] = fold_start(s.folded);
#pragma unroll 4
                for (unsigned long long k = k0; k < k1; ++k) {
                    T v[V];
                    load16(column + k * s.inner, v);
#pragma unroll
                    for (int e = 0; e < V; ++e) acc[e] = fold_pair(s.folded, acc[e], static_cast<double>(v[e]));
                }
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    const unsigned long long j = g * V + e;
                    if (s.pieces == 1) out[o * s.inner + j] = finish<T>(s.fold, acc[e], s.extent);
                    else partial[(o * s.pieces + piece) * s.inner + j] = acc[e];
                }
            }
        }

        // Folds the pieces of every output in piece order: partial[(o * pieces + p) * inner + j].
        template <typename T>
        __global__ void __launch_bounds__(256) axis_pieces(const double *partial, AxisShape s, T *out) {
            const unsigned long long outputs = s.outer * s.inner, step = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < outputs; i += step) {
                const unsigned long long o = i / s.inner, j = i - o * s.inner;
                double acc = fold_start(s.folded);
                for (unsigned long long p = 0; p < s.pieces; ++p) acc = fold_pair(s.folded, acc, partial[(o * s.pieces + p) * s.inner + j]);
                out[i] = finish<T>(s.fold, acc, s.extent);
            }
        }

        template <typename T> int launch_axis(Context &ctx, const T *in, T *out, AxisShape s) {
            // Work units for four resident waves of threads, run by one persistent wave, so the last
            // units do not leave most of the GPU idle.
            const void *kernel = s.inner == 1 && s.extent >= 64 ? reinterpret_cast<const void *>(&axis_rows<T>)
                                                                : reinterpret_cast<const void *>(&axis_column_vectors<T>);
            const unsigned long long most = 1ull * ctx.sms * ctx.blocks_per_sm(kernel, 256, 0);  // blocks of 256
            const unsigned long long target = 4 * most * 256;                                     // threads' worth of units
            // short rows go a thread per row (the column form with inner = 1)
            const bool rows = s.inner == 1 && s.extent >= 64;
            constexpr unsigned long long V = 16 / sizeof(T);
            const bool vectors = !rows && s.inner % V == 0 && (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
            if (rows) {
                // a warp per (row, piece); pieces of at least 2048 values
                const unsigned long long want = (target / 32 + s.outer - 1) / s.outer;
                const unsigned long long cap = (s.extent + 2047) / 2048;
                s.pieces = want < cap ? want : cap;
            } else {
                // a thread per (o, piece, j or vector of j); pieces of at least 64 values
                const unsigned long long columns = s.outer * (vectors ? s.inner / V : s.inner);
                const unsigned long long want = (target + columns - 1) / columns;
                const unsigned long long cap = (s.extent + 63) / 64;
                s.pieces = want < cap ? want : cap;
            }
            if (s.pieces < 1) s.pieces = 1;
            s.span = (s.extent + s.pieces - 1) / s.pieces;
            s.pieces = (s.extent + s.span - 1) / s.span;
            double *partial = nullptr;
            if (s.pieces > 1) {
                if (int code = ctx.check(ctx.workspace->reserve(s.outer * s.pieces * s.inner * sizeof(double)),
                                         "reserving axis partials"))
                    return code;
                partial = static_cast<double *>(ctx.workspace->memory);
            }
            if (rows) {
                const unsigned long long blocks = (s.outer * s.pieces + 7) / 8;
                axis_rows<T><<<static_cast<unsigned>(blocks < most ? blocks : most), 256, 0, ctx.stream>>>(in, s, partial, out);
            } else if (vectors) {
                const unsigned long long blocks = (s.outer * s.pieces * (s.inner / V) + 255) / 256;
                axis_column_vectors<T><<<static_cast<unsigned>(blocks < most ? blocks : most), 256, 0, ctx.stream>>>(in, s, partial,
                                                                                                                   out);
            } else {
                const unsigned long long blocks = (s.outer * s.pieces * s.inner + 255) / 256;
                axis_columns<T><<<static_cast<unsigned>(blocks < most ? blocks : most), 256, 0, ctx.stream>>>(in, s, partial, out);
            }
            if (int code = ctx.check(cudaGetLastError(), "launching an axis reduction")) return code;
            if (s.pieces > 1) {
                const unsigned long long blocks = (s.outer * s.inner + 255) / 256;
                axis_pieces<T><<<static_cast<unsigned>(blocks < most ? blocks : most), 256, 0, ctx.stream>>>(partial, s, out);
                if (int code = ctx.check(cudaGetLastError(), "launching the axis piece fold")) return code;
            }
            return SCI_CUDA_OK;
        }

    } // namespace
} // namespace sci_cuda

extern "C" int sci_cuda_reduce_axis(sci_cuda_context *context, uint32_t precision, uint32_t fold, const void *input,
                                    uint32_t rank, const uint64_t *shape, uint32_t axis, void *output) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u", precision);
    if (fold > SCI_AXIS_MEAN) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown axis fold %u", fold);
    if (rank < 1 || rank > 8 || !shape || axis >= rank)
        return context->fail(SCI_CUDA_ERROR_INVALID, "reduce_axis: axis %u of rank %u (1 to 8, with its shape)", axis, rank);
    AxisShape s{1, shape[axis], 1, 1, 0, fold, fold == SCI_AXIS_MEAN ? static_cast<unsigned>(SCI_FOLD_SUM) : fold};
    unsigned long long total = 1;
    for (uint32_t a = 0; a < rank; ++a) {
        if (shape[a] != 0 && total > ~0ull / shape[a]) return context->fail(SCI_CUDA_ERROR_INVALID, "reduce_axis: shape overflows");
        total *= shape[a];
        if (a < axis) s.outer *= shape[a];
        if (a > axis) s.inner *= shape[a];
    }
    const unsigned long long outputs = s.outer * s.inner;
    if (outputs == 0) return SCI_CUDA_OK;
    if (!output || !reachable(*context, output)) return context->fail(SCI_CUDA_ERROR_INVALID, "reduce_axis: the output is not memory of this device");
    if (s.extent == 0) {
        // an empty axis: 0 for sum and mean, NaN for minimum and maximum
        const double empty = (fold == SCI_FOLD_SUM || fold == SCI_AXIS_MEAN) ? 0.0 : std::numeric_limits<double>::quiet_NaN();
        return sci_cuda_fill(context, precision, output, outputs, empty);
    }
    if (!input || !reachable(*context, input)) return context->fail(SCI_CUDA_ERROR_INVALID, "reduce_axis: the input is not memory of this device");
    if (input == output) return context->fail(SCI_CUDA_ERROR_INVALID, "reduce_axis: the output must not be the input");
    cudaSetDevice(context->device);
    if (precision == SCI_PRECISION_WIDE)
        return launch_axis<double>(*context, static_cast<const double *>(input), static_cast<double *>(output), s);
    return launch_axis<float>(*context, static_cast<const float *>(input), static_cast<float *>(output), s);
}
