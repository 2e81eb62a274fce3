// context.hpp -- the per-device state behind a sci_cuda_context (host side, C++).
//
// Stands in for the reference's Graphics bundle (src/core/drivers/device.cpp:111-184): one CUDA
// stream plays vulkan::Stream (in-order queue, src/core/drivers/vulkan/stream.cpp:56-130), a
// mutex plays Graphics::guard, and the scratch of the single-pass reductions is allocated once
// when the context opens.
#pragma once

#include "../../include/sci_cuda.h"
#include "chunk_kernel.cuh"

#include <cuda.h>  // driver-API types only; the functions are resolved at run time (Driver)
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace sci_cuda {

    // The few driver-API calls the NVRTC path needs, resolved through the runtime
    // (cudaGetDriverEntryPoint), so the library links no libcuda and loads on machines without a
    // driver (the CPU build and test host); `ready` is false there.
    struct Driver {
        bool ready{false};
        CUresult (*module_load)(CUmodule *, const void *){nullptr};
        CUresult (*module_function)(CUfunction *, CUmodule, const char *){nullptr};
        CUresult (*module_unload)(CUmodule){nullptr};
        CUresult (*function_attribute)(CUfunction, CUfunction_attribute, int){nullptr};
        CUresult (*occupancy)(int *, CUfunction, int, size_t){nullptr};
        CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                           void **, void **){nullptr};

        static const Driver &get() {
            static const Driver table = [] {
                Driver d;
                auto resolve = [](const char *name, void **out) {
                    cudaDriverEntryPointQueryResult found{};
                    return cudaGetDriverEntryPoint(name, out, cudaEnableDefault, &found) == cudaSuccess &&
                           found == cudaDriverEntryPointSuccess && *out != nullptr;
                };
                d.ready = resolve("cuModuleLoadData", reinterpret_cast<void **>(&d.module_load)) &&
                          resolve("cuModuleGetFunction", reinterpret_cast<void **>(&d.module_function)) &&
                          resolve("cuModuleUnload", reinterpret_cast<void **>(&d.module_unload)) &&
                          resolve("cuFuncSetAttribute", reinterpret_cast<void **>(&d.function_attribute)) &&
                          resolve("cuOccupancyMaxActiveBlocksPerMultiprocessor", reinterpret_cast<void **>(&d.occupancy)) &&
                          resolve("cuLaunchKernel", reinterpret_cast<void **>(&d.launch));
                if (!d.ready) cudaGetLastError();
                return d;
            }();
            return table;
        }
    };

    class Specializer;  // NVRTC specialisation of the chunk kernel (specialize.cu)
    struct Workspace;   // scratch of the product / LU paths, grown on demand

    struct Retired {
        cudaEvent_t done;
        void *memory;
        bool managed;
    };

    struct Context {
        int device{0};
        int sms{0};
        size_t shared_limit{0};     // opt-in dynamic shared memory per block
        cudaStream_t stream{nullptr};
        std::recursive_mutex guard;
        std::string error;
        std::string name;

        ReduceState *state{nullptr};   // reduction scratch (device)
        double *result{nullptr};       // reduction result (device), with the status word 8 bytes on
        int *status{nullptr};          // device-side error word (in result's allocation)
        double *host_result{nullptr};  // pinned, with host_status 8 bytes on: one copy reads both
        int *host_status{nullptr};     // pinned (in host_result's allocation)
        double *pinned{nullptr};       // pinned doubles for small read-backs (grown on demand)
        size_t pinned_count{0};

        std::vector<Retired> retired;  // frees deferred until queued work is done
        std::map<std::tuple<const void *, int, size_t>, int> occupancy;  // (kernel, threads, smem) -> blocks/SM
        std::map<const void *, size_t> smem_raised;  // NVRTC function -> the dynamic shared memory it is allowed
        std::unique_ptr<Specializer> specializer;
        std::unique_ptr<Workspace> workspace;  // product / trailing-update operands
        std::unique_ptr<Workspace> solver;     // LU copies, pivots, residuals
        std::unique_ptr<Workspace> tape;       // the stored-form gradient's forward values
        cudaStream_t side{nullptr};             // the LU look-ahead's bulk updates (lower priority)
        cudaEvent_t side_done{nullptr};         // the side stream's queued work has finished
        cudaEvent_t main_ready{nullptr};        // the main stream reached the point the side waits for
        std::unique_ptr<Workspace> side_space;  // the side stream's product operands
        cudaStream_t upload_lane{nullptr};    // host-to-device copies that overlap the main stream
        cudaStream_t download_lane{nullptr};  // device-to-host copies that overlap the main stream
        cudaEvent_t uploaded{nullptr};        // the upload lane's last queued copy
        cudaEvent_t downloaded{nullptr};      // the download lane's last queued copy
        cudaEvent_t main_point{nullptr};      // where the main stream was when a download was queued
        unsigned *sweep_flags{nullptr};  // progress marks of the persistent substitution sweeps
        size_t sweep_capacity{0};        // flags allocated
        unsigned sweep_epoch{0};         // the value that marks a flag as set by the current sweep
        int jit_mode{1};  // 0 off, 1 background, 2 synchronous (SCI_CUDA_JIT)
        bool jit_trace{false};

        int fail(int code, const char *format, ...) {
            char buffer[512];
            va_list args;
            va_start(args, format);
            std::vsnprintf(buffer, sizeof(buffer), format, args);
            va_end(args);
            error = buffer;
            return code;
        }

        // Maps a CUDA error to a status, keeping the message.
        int check(cudaError_t code, const char *what) {
            if (code == cudaSuccess) return SCI_CUDA_OK;
            return fail(code == cudaErrorMemoryAllocation ? SCI_CUDA_ERROR_MEMORY : SCI_CUDA_ERROR_LAUNCH, "%s: %s",
                        what, cudaGetErrorString(code));
        }

        // Blocks per SM for a kernel at a block size and dynamic shared memory, cached.
        int blocks_per_sm(const void *kernel, int threads, size_t smem) {
            auto key = std::make_tuple(kernel, threads, smem);
            auto found = occupancy.find(key);
            if (found != occupancy.end()) return found->second;
            int blocks = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem) != cudaSuccess) blocks = 1;
            occupancy[key] = blocks > 0 ? blocks : 1;
            return occupancy[key];
        }

        // Reads and clears the device error word; waits for the stream. status_queued: a copy of the
        // status word into host_status is already queued on the stream.
        int drain(bool status_queued = false);

        // Lets `kernel` use `smem` bytes of dynamic shared memory, raising its limit only past the
        // largest one set so far: for kernels no other context or entry point sets (this context's
        // NVRTC modules).
        template <typename Raise> void allow_smem(const void *kernel, size_t smem, Raise raise) {
            auto found = smem_raised.find(kernel);
            if (found != smem_raised.end() && found->second >= smem) return;
            raise();
            smem_raised[kernel] = smem;
        }
    };

    // Block size, TMA ring depth and dynamic shared memory of a chunk launch: the widest tile whose
    // temporaries (none for a specialised kernel, which keeps them in registers) and staged inputs
    // fit in `budget` bytes. A chunk with transcendental codes is bound by instruction issue, not
    // by HBM: a two-stage ring already covers its load latency, and the shared memory it frees buys
    // more resident warps to hide its arithmetic latency; arithmetic-only chunks keep the deepest
    // ring. threads = 0 when even a 32-thread tile does not fit.
    struct ChunkShape {
        int threads{0};
        unsigned stages{0};
        size_t smem{0};
    };
    inline ChunkShape chunk_shape(const Step *steps, unsigned length, unsigned arguments, unsigned temporaries,
                                  size_t element, bool staged_ok, bool specialised, size_t budget) {
        bool heavy = false;
        for (unsigned s = 0; s < length; ++s) heavy = heavy || (steps[s].code >= kExponential && steps[s].code < kAdd);
        const size_t ring = heavy ? 2u : static_cast<size_t>(kMaxStages);
        ChunkShape shape;
        for (int threads = 256; threads >= 32; threads /= 2) {
            const size_t tile_bytes = size_t(32 / element) * threads * element;
            const size_t temps = specialised ? 0 : size_t(temporaries) * tile_bytes;
            if (temps > budget) continue;
            unsigned stages = 0;
            if (staged_ok && arguments > 0) {
                const size_t fit = (budget - temps) / (size_t(arguments) * tile_bytes);
                stages = static_cast<unsigned>(fit < ring ? fit : ring);
            }
            if (stages == 0 && staged_ok && arguments > 0 && threads > 32) continue;  // try a smaller tile
            shape.threads = threads;
            shape.stages = stages;
            shape.smem = temps + size_t(stages) * arguments * tile_bytes;
            break;
        }
        return shape;
    }

    // Without the opt-in, static plus dynamic shared memory must stay within 48 KB; the chunk
    // kernel's static part (mbarriers, fold scratch) is under 4 KB.
    constexpr size_t kChunkSharedOptIn = 44 * 1024;

    // The context's reduction result (a double) and status word (an int after it), one allocation.
    constexpr size_t kResultBytes = 16;

    // The generic interpreter's kernels, compiled ahead of time (chunk_kernels_f32.cu / _f64.cu).
    const void *generic_chunk_kernel(bool wide, int mode);
    const void *generic_chunk_kernel_f32(int mode);
    const void *generic_chunk_kernel_f64(int mode);
    inline const void *generic_chunk_kernel(bool wide, int mode) {
        return wide ? generic_chunk_kernel_f64(mode) : generic_chunk_kernel_f32(mode);
    }

    // Row-major GEMMs on submatrices (product.cu): C (pitch ldc) = A (pitch lda) * B (pitch ldb),
    // or C -= A * B with `subtract`. tensor_gemm splits each operand into `terms` (1-3) bf16 parts
    // and multiplies on the tensor cores; simt_gemm is the plain FP32 / FP64 form. Both queue on
    // ctx.stream. `whole_gpu`: the product has the GPU to itself, so products of 256 rows or more
    // run on the persistent CTA-pair kernel (a static split of the tiles over every SM); the LU's
    // updates, which share the GPU with the panels, keep the one-tile-per-CTA kernel. `chained`: the
    // first launch follows the kernel before it on the stream directly, so the conversions and the
    // product are launched with programmatic stream serialization (each waits for the one before).
    int tensor_gemm(Context &ctx, int terms, const float *a, unsigned long long lda, const float *b,
                    unsigned long long ldb, float *c, unsigned long long ldc, unsigned long long m, unsigned long long n,
                    unsigned long long k, bool subtract, bool whole_gpu = false, bool chained = false);
    template <typename T>
    int simt_gemm(Context &ctx, const T *a, unsigned long long lda, const T *b, unsigned long long ldb, T *c,
                  unsigned long long ldc, unsigned long long m, unsigned long long n, unsigned long long k, bool subtract);
    // The same with transposed operands read in place: a_t means A is stored k x m (pitch lda), b_t
    // that B is stored n x k (pitch ldb).
    int tensor_gemm_t(Context &ctx, int terms, const float *a, unsigned long long lda, bool a_t, const float *b,
                      unsigned long long ldb, bool b_t, float *c, unsigned long long ldc, unsigned long long m,
                      unsigned long long n, unsigned long long k, bool subtract, bool whole_gpu = false,
                      bool chained = false);
    template <typename T>
    int simt_gemm_t(Context &ctx, const T *a, unsigned long long lda, bool a_t, const T *b, unsigned long long ldb, bool b_t,
                    T *c, unsigned long long ldc, unsigned long long m, unsigned long long n, unsigned long long k,
                    bool subtract);

    // Validates a chunk before anything is launched: counts, codes, and every value id in range.
    int validate(Context &ctx, const sci_chunk *chunk, bool reducing);

    // Whether a pointer is memory this context's GPU reads directly (device memory of its GPU, or
    // managed memory).
    bool reachable(Context &ctx, const void *pointer);

} // namespace sci_cuda

struct sci_cuda_context : sci_cuda::Context {};
