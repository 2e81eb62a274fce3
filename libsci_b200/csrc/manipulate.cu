// manipulate.cu -- transpose on the device (include/operations/manipulations.hpp:33-62): the
// dimensions in reverse order, output[j_{r-1}, ..., j_0] = input[j_0, ..., j_{r-1}], for row-major
// arrays of rank 1 to 8. The reference copies element by element on the host.
//
// Rank 2 goes through 64 x 64 tiles in shared memory (pitch 65), so both the reads and the writes
// are coalesced; other ranks map each output element to its input element. A copy either way: the
// values are the input's bits. Bound by HBM: 2 x element size bytes per element.
#include "context.hpp"

#include <cuda_runtime.h>

using namespace sci_cuda;

namespace sci_cuda {
    namespace {

        constexpr int kMaxRank = 8;

        struct Dims {
            unsigned long long extent[kMaxRank];  // the input's extents
            unsigned long long input_stride[kMaxRank];
            int rank;
        };

        // 64 x 64 tiles, 256 threads (32 x 8): each thread loads its 16 elements of the tile before
        // storing any (16 loads in flight per thread), then writes 16 of the transposed tile.
        constexpr int kTile = 64;
        template <typename T>
        __global__ void __launch_bounds__(256) transpose_tiles(const T *in, T *out, unsigned long long rows,
                                                               unsigned long long columns) {
            __shared__ T tile[kTile][kTile + 1];
            const unsigned long long tiles_x = (columns + kTile - 1) / kTile, tiles = tiles_x * ((rows + kTile - 1) / kTile);
            for (unsigned long long t = blockIdx.x; t < tiles; t += gridDim.x) {
                const unsigned long long r0 = (t / tiles_x) * kTile, c0 = (t % tiles_x) * kTile;
                T staged[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int k = threadIdx.y + 8 * (q / 2), x = threadIdx.x + 32 * (q % 2);
                    const unsigned long long r = r0 + k, c = c0 + x;
                    staged[q] = (r < rows && c < columns) ? in[r * columns + c] : T(0);
                }
#pragma unroll
                for (int q = 0; q < 16; ++q) tile[threadIdx.y + 8 * (q / 2)][threadIdx.x + 32 * (q % 2)] = staged[q];
                __syncthreads();
                // out is columns x rows: out[c][r] = in[r][c]
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int k = threadIdx.y + 8 * (q / 2), x = threadIdx.x + 32 * (q % 2);
                    const unsigned long long c = c0 + k, r = r0 + x;
                    if (c < columns && r < rows) out[c * rows + r] = tile[x][k];
                }
                __syncthreads();
            }
        }

        template <typename T> __global__ void transpose_any(const T *in, T *out, unsigned long long count, Dims d) {
            const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
                // output coordinates, last axis fastest; output axis a is input axis rank - 1 - a
                unsigned long long rest = i, source = 0;
                for (int a = d.rank - 1; a >= 0; --a) {
                    const int axis = d.rank - 1 - a;  // the input axis of output axis a
                    const unsigned long long extent = d.extent[axis];
                    const unsigned long long coordinate = rest % extent;
                    rest /= extent;
                    source += coordinate * d.input_stride[axis];
                }
                out[i] = in[source];
            }
        }

        template <typename T>
        int launch(Context &ctx, const T *in, T *out, const Dims &d, unsigned long long count) {
            if (d.rank == 2) {
                const unsigned long long tiles = ((d.extent[0] + kTile - 1) / kTile) * ((d.extent[1] + kTile - 1) / kTile);
                const unsigned grid = static_cast<unsigned>(tiles < 8ull * ctx.sms ? tiles : 8ull * ctx.sms);
                transpose_tiles<T><<<grid, dim3(32, 8), 0, ctx.stream>>>(in, out, d.extent[0], d.extent[1]);
            } else {
                const unsigned long long wanted = (count + 255) / 256;
                const unsigned grid = static_cast<unsigned>(wanted < 8ull * ctx.sms ? wanted : 8ull * ctx.sms);
                transpose_any<T><<<grid, 256, 0, ctx.stream>>>(in, out, count, d);
            }
            return ctx.check(cudaGetLastError(), "launching transpose");
        }

    } // namespace
} // namespace sci_cuda

extern "C" int sci_cuda_transpose(sci_cuda_context *context, uint32_t precision, const void *input, uint32_t rank,
                                  const uint64_t *shape, void *output) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u", precision);
    if (rank < 1 || rank > static_cast<uint32_t>(kMaxRank) || !shape)
        return context->fail(SCI_CUDA_ERROR_INVALID, "transpose: rank %u (1 to %d, with its shape)", rank, kMaxRank);
    Dims d{};
    d.rank = static_cast<int>(rank);
    unsigned long long count = 1;
    for (int a = d.rank - 1; a >= 0; --a) {
        d.extent[a] = shape[a];
        d.input_stride[a] = count;
        if (shape[a] != 0 && count > ~0ull / shape[a]) return context->fail(SCI_CUDA_ERROR_INVALID, "transpose: shape overflows");
        count *= shape[a];
    }
    if (count == 0) return SCI_CUDA_OK;
    if (!input || !output || !reachable(*context, input) || !reachable(*context, output))
        return context->fail(SCI_CUDA_ERROR_INVALID, "transpose: input and output must be memory of this device");
    if (input == output) return context->fail(SCI_CUDA_ERROR_INVALID, "transpose: the output must not be the input");
    cudaSetDevice(context->device);
    if (rank == 1) {
        return context->check(cudaMemcpyAsync(output, input, count * (precision == SCI_PRECISION_WIDE ? 8 : 4),
                                              cudaMemcpyDeviceToDevice, context->stream),
                              "transpose of rank 1");
    }
    if (precision == SCI_PRECISION_WIDE)
        return launch<double>(*context, static_cast<const double *>(input), static_cast<double *>(output), d, count);
    return launch<float>(*context, static_cast<const float *>(input), static_cast<float *>(output), d, count);
}
