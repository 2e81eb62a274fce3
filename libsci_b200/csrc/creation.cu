// creation.cu -- arrays made on the device: full (zeros, ones), linspace, range, eye and grid,
// the element values of libsci's include/operations/creation.hpp computed where the array lives,
// so a CUDA array never fills through a host pointer.
//
// Each kernel is a grid-stride loop over the output, bound by HBM writes (4 or 8 bytes per element
// written, nothing read but grid's two small vectors). Values follow the reference's arithmetic
// step by step, with every operation rounded on its own (no contraction):
//   full      out[i] = value                                         (creation.hpp:34-58)
//   linspace  step = double(stop - start) / (double(count) - 1),
//             out[i] = element(double(start) + double(i) * step); count 1 gives start itself
//                                                                     (creation.hpp:66-84)
//   range     out[i] = start + element(i) * step, in the element type (creation.hpp:157-168)
//   eye       out[r * columns + c] = r == c                           (creation.hpp:91-106)
//   grid      xx[i][j] = x[j], yy[i][j] = y[i]                        (creation.hpp:120-140)
// eye and grid go row by row (a block per row piece), the others element by element.
#include "context.hpp"

#include <cuda_runtime.h>

#include <cmath>

using namespace sci_cuda;

namespace sci_cuda {
    namespace {

        unsigned blocks_for(unsigned long long count, int sms) {
            const unsigned long long wanted = (count + 255) / 256;
            const unsigned long long most = 8ull * static_cast<unsigned long long>(sms);
            return static_cast<unsigned>(wanted < 1 ? 1 : (wanted < most ? wanted : most));
        }

        __device__ __forceinline__ float to_element(double v, float) { return __double2float_rn(v); }
        __device__ __forceinline__ double to_element(double v, double) { return v; }
        __device__ __forceinline__ float from_index(unsigned long long i, float) { return __ull2float_rn(i); }
        __device__ __forceinline__ double from_index(unsigned long long i, double) { return __ull2double_rn(i); }

        template <typename T> __global__ void fill_kernel(T *out, unsigned long long count, T value) {
            const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) out[i] = value;
        }

        template <typename T>
        __global__ void linspace_kernel(T *out, unsigned long long count, double start, double step) {
            const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
                out[i] = to_element(__dadd_rn(start, __dmul_rn(static_cast<double>(i), step)), T());
        }

        template <typename T> __global__ void range_kernel(T *out, unsigned long long count, T start, T step) {
            const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
                out[i] = add(start, mul(from_index(i, T()), step));
        }

        // eye and grid walk (row, chunk of kSpan columns) pieces, one piece per block at a time: one
        // division per piece instead of one per element, and each row written front to back.
        constexpr unsigned kSpan = 1024;

        template <typename T> __global__ void eye_kernel(T *out, unsigned long long rows, unsigned long long columns) {
            const unsigned long long chunks = (columns + kSpan - 1) / kSpan, pieces = rows * chunks;
            for (unsigned long long piece = blockIdx.x; piece < pieces; piece += gridDim.x) {
                const unsigned long long row = piece / chunks, c0 = (piece - row * chunks) * kSpan;
                T *line = out + row * columns;
                for (unsigned long long c = c0 + threadIdx.x; c < c0 + kSpan && c < columns; c += blockDim.x)
                    line[c] = c == row ? T(1) : T(0);
            }
        }

        template <typename T>
        __global__ void grid_kernel(const T *x, unsigned long long nx, const T *y, unsigned long long ny, T *xx, T *yy) {
            const unsigned long long chunks = (nx + kSpan - 1) / kSpan, pieces = ny * chunks;
            for (unsigned long long piece = blockIdx.x; piece < pieces; piece += gridDim.x) {
                const unsigned long long row = piece / chunks, c0 = (piece - row * chunks) * kSpan;
                const T yv = y[row];
                for (unsigned long long c = c0 + threadIdx.x; c < c0 + kSpan && c < nx; c += blockDim.x) {
                    xx[row * nx + c] = x[c];
                    yy[row * nx + c] = yv;
                }
            }
        }

        // Common checks: a context, a known precision, and device memory of this context where
        // anything is written or read.
        int prologue(sci_cuda_context *context, uint32_t precision) {
            if (!context) return SCI_CUDA_ERROR_INVALID;
            if (precision > SCI_PRECISION_WIDE) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u", precision);
            cudaSetDevice(context->device);
            return SCI_CUDA_OK;
        }

        int memory(sci_cuda_context *context, const void *pointer, const char *what) {
            if (!pointer || !reachable(*context, pointer))
                return context->fail(SCI_CUDA_ERROR_INVALID, "%s (%p) is not memory of this device", what, pointer);
            return SCI_CUDA_OK;
        }

    } // namespace
} // namespace sci_cuda

extern "C" {

int sci_cuda_fill(sci_cuda_context *context, uint32_t precision, void *output, uint64_t count, double value) {
    if (int code = prologue(context, precision)) return code;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (count == 0) return SCI_CUDA_OK;
    if (int code = memory(context, output, "output")) return code;
    const unsigned grid = blocks_for(count, context->sms);
    if (precision == SCI_PRECISION_WIDE)
        fill_kernel<double><<<grid, 256, 0, context->stream>>>(static_cast<double *>(output), count, value);
    else
        fill_kernel<float><<<grid, 256, 0, context->stream>>>(static_cast<float *>(output), count, static_cast<float>(value));
    return context->check(cudaGetLastError(), "launching fill");
}

int sci_cuda_linspace(sci_cuda_context *context, uint32_t precision, void *output, uint64_t count, double start,
                      double stop) {
    if (int code = prologue(context, precision)) return code;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (count == 0) return SCI_CUDA_OK;
    if (count == 1) return sci_cuda_fill(context, precision, output, 1, start);  // start itself (creation.hpp:76-79)
    if (int code = memory(context, output, "output")) return code;
    const unsigned grid = blocks_for(count, context->sms);
    if (precision == SCI_PRECISION_WIDE) {
        const double step = (stop - start) / (static_cast<double>(count) - 1.0);
        linspace_kernel<double><<<grid, 256, 0, context->stream>>>(static_cast<double *>(output), count, start, step);
    } else {
        // start and stop are elements; their difference is taken in the element type
        const float first = static_cast<float>(start), last = static_cast<float>(stop);
        volatile float span = last - first;
        const double step = static_cast<double>(span) / (static_cast<double>(count) - 1.0);
        linspace_kernel<float><<<grid, 256, 0, context->stream>>>(static_cast<float *>(output), count, first, step);
    }
    return context->check(cudaGetLastError(), "launching linspace");
}

uint64_t sci_cuda_range_count(uint32_t precision, double start, double stop, double step) {
    // the arguments are elements, widened to double for the count (creation.hpp:159-161)
    if (precision != SCI_PRECISION_WIDE) {
        start = static_cast<float>(start);
        stop = static_cast<float>(stop);
        step = static_cast<float>(step);
    }
    volatile double difference = stop - start;
    const double span = std::ceil(difference / step);
    return span > 0 ? static_cast<uint64_t>(span) : 0;
}

int sci_cuda_range(sci_cuda_context *context, uint32_t precision, void *output, uint64_t count, double start,
                   double step) {
    if (int code = prologue(context, precision)) return code;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (count == 0) return SCI_CUDA_OK;
    if (int code = memory(context, output, "output")) return code;
    const unsigned grid = blocks_for(count, context->sms);
    if (precision == SCI_PRECISION_WIDE)
        range_kernel<double><<<grid, 256, 0, context->stream>>>(static_cast<double *>(output), count, start, step);
    else
        range_kernel<float><<<grid, 256, 0, context->stream>>>(static_cast<float *>(output), count, static_cast<float>(start),
                                                              static_cast<float>(step));
    return context->check(cudaGetLastError(), "launching range");
}

int sci_cuda_eye(sci_cuda_context *context, uint32_t precision, void *output, uint64_t rows, uint64_t columns) {
    if (int code = prologue(context, precision)) return code;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (rows == 0 || columns == 0) return SCI_CUDA_OK;
    if (rows > UINT64_MAX / columns) return context->fail(SCI_CUDA_ERROR_INVALID, "eye: %llu x %llu overflows",
                                                          static_cast<unsigned long long>(rows),
                                                          static_cast<unsigned long long>(columns));
    if (int code = memory(context, output, "output")) return code;
    const unsigned grid = blocks_for(rows * ((columns + kSpan - 1) / kSpan) * 256, context->sms);
    if (precision == SCI_PRECISION_WIDE)
        eye_kernel<double><<<grid, 256, 0, context->stream>>>(static_cast<double *>(output), rows, columns);
    else
        eye_kernel<float><<<grid, 256, 0, context->stream>>>(static_cast<float *>(output), rows, columns);
    return context->check(cudaGetLastError(), "launching eye");
}

int sci_cuda_grid(sci_cuda_context *context, uint32_t precision, const void *x, uint64_t nx, const void *y, uint64_t ny,
                  void *xx, void *yy) {
    if (int code = prologue(context, precision)) return code;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (nx == 0 || ny == 0) return SCI_CUDA_OK;
    if (nx > UINT64_MAX / ny) return context->fail(SCI_CUDA_ERROR_INVALID, "grid: %llu x %llu overflows",
                                                   static_cast<unsigned long long>(ny), static_cast<unsigned long long>(nx));
    if (int code = memory(context, x, "x")) return code;
    if (int code = memory(context, y, "y")) return code;
    if (int code = memory(context, xx, "xx")) return code;
    if (int code = memory(context, yy, "yy")) return code;
    const unsigned grid = blocks_for(ny * ((nx + kSpan - 1) / kSpan) * 256, context->sms);
    if (precision == SCI_PRECISION_WIDE)
        grid_kernel<double><<<grid, 256, 0, context->stream>>>(static_cast<const double *>(x), nx, static_cast<const double *>(y),
                                                              ny, static_cast<double *>(xx), static_cast<double *>(yy));
    else
        grid_kernel<float><<<grid, 256, 0, context->stream>>>(static_cast<const float *>(x), nx, static_cast<const float *>(y),
                                                             ny, static_cast<float *>(xx), static_cast<float *>(yy));
    return context->check(cudaGetLastError(), "launching grid");
}

} // extern "C"
