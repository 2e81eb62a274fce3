// specialize.cu -- NVRTC specialisation of the chunk kernel (see specialize.hpp).
//
// The reference compiles a chunk it sees into a Slang shader of its own on a background thread and
// keeps running the interpreter until the shader is ready (src/core/drivers/vulkan/compiler.cpp:
// 35-92 generate, :94-151 compile, :169-182 find, :184-222 loop; cache keyed by Chunk::signature(),
// capped at 1024 kernels, compiler.cpp:27). Here the "generated code" is not new source: it is the
// same hand-written kernel (chunk_kernel.cuh, embedded in this library at build time) instantiated
// with the chunk's bytecode as a compile-time constant, so the instruction loop unrolls and the
// temporaries become registers. SCI_CUDA_JIT=0 turns it off, =sync compiles before the first
// launch, =trace reports every compile on stderr.
#include "specialize.hpp"
#include "batch_kernel.cuh"
#include "gradient_kernel.cuh"

#include <cuda.h>
#include <nvrtc.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

// Generated at build time from sci_math.cuh, chunk_kernel.cuh, gradient_kernel.cuh and
// batch_kernel.cuh (libsci_b200/build.py).
extern const char *const sci_embedded_math;
extern const char *const sci_embedded_kernel;
extern const char *const sci_embedded_gradient;
extern const char *const sci_embedded_batch;

namespace sci_cuda {

    namespace {

        constexpr size_t kCacheLimit = 1024;

        struct Job {
            std::string key;
            sci_chunk chunk;
            int mode;
        };

        struct Entry {
            enum State { kQueued, kReady, kFailed } state{kQueued};
            CUmodule module{nullptr};
            Specialized special{nullptr};
        };

        std::string key_of(const sci_chunk &chunk, int mode) {
            // Chunk::signature() (chunk.hpp:209-226) plus the launch mode.
            std::string key;
            key.reserve(8 + 5 * chunk.length);
            key += static_cast<char>(mode);
            key += static_cast<char>(chunk.precision);
            key += static_cast<char>(chunk.arguments);
            key += static_cast<char>(chunk.literals);
            key += static_cast<char>(chunk.temporaries);
            key += static_cast<char>(chunk.result);
            for (int i = 0; i < chunk.length; ++i) {
                const sci_instruction &ins = chunk.instructions[i];
                key += static_cast<char>(ins.code);
                key += static_cast<char>(ins.target);
                key += static_cast<char>(ins.sources[0]);
                key += static_cast<char>(ins.sources[1]);
                key += static_cast<char>(ins.sources[2]);
            }
            return key;
        }

        // The instantiation of chunk_stream<T, Baked<SciBaked>, MODE> for one chunk, or of
        // gradient_stream<T, Baked<SciBaked>, MODE> for a chunk in value form (the gradient modes).
        std::string program_of(const sci_chunk &chunk, int mode, std::string &name) {
            const bool gradient = mode == kGradRecompute || mode == kGradRecord || mode == kGradReplay;
            const bool contract = mode == kDot;
            const int length = contract ? chunk.length - 1 : chunk.length;
            int dot_left = kNone, dot_right = kNone;
            if (contract) {
                dot_left = chunk.instructions[chunk.length - 1].sources[0];
                dot_right = chunk.instructions[chunk.length - 1].sources[1];
            }
            const bool batch = mode == kBatchMode;
            std::string src = gradient ? "#include \"gradient_kernel.cuh\"\nstruct SciBaked {\n"
                              : batch  ? "#include \"batch_kernel.cuh\"\nstruct SciBaked {\n"
                                       : "#include \"chunk_kernel.cuh\"\nstruct SciBaked {\n";
            char line[256];
            std::snprintf(line, sizeof(line),
                          "  static constexpr int length = %d, arguments = %d, temporaries = %d, result = %d,"
                          " dot_left = %d, dot_right = %d;\n",
                          length, chunk.arguments, chunk.temporaries, chunk.result, dot_left, dot_right);
            src += line;
            src += "  static constexpr sci_cuda::Step steps[] = {";
            const int stored = length > 0 ? length : 0;
            for (int i = 0; i < stored; ++i) {
                const sci_instruction &ins = chunk.instructions[i];
                std::snprintf(line, sizeof(line), "%s{%d, %d, %d, %d, %d}", i ? ", " : "", ins.code, ins.target,
                              ins.sources[0], ins.sources[1], ins.sources[2]);
                src += line;
            }
            if (stored == 0) src += "{0, 255, 255, 255, 255}";
            src += "};\n};\n";
            const char *type = chunk.precision == SCI_PRECISION_WIDE ? "double" : "float";
            if (batch) {
                name = std::string("&sci_cuda::batch_stream<") + type + ", sci_cuda::Baked<SciBaked>>";
            } else {
                name = std::string(gradient ? "&sci_cuda::gradient_stream<" : "&sci_cuda::chunk_stream<") + type +
                       ", sci_cuda::Baked<SciBaked>, " + std::to_string(mode) + ">";
            }
            return src;
        }

        class Nvrtc final : public Specializer {
        public:
            explicit Nvrtc(Context &ctx) : device(ctx.device), mode(ctx.jit_mode), trace(ctx.jit_trace) {
                if (mode == 1) worker = std::thread([this] { loop(); });
            }

            ~Nvrtc() override {
                {
                    std::lock_guard<std::mutex> lock(guard);
                    stop = true;
                }
                wake.notify_all();
                if (worker.joinable()) worker.join();
                for (auto &item : table) {
                    if (item.second.module) Driver::get().module_unload(item.second.module);
                }
            }

            const Specialized *find(Context &ctx, const sci_chunk &chunk, int launch_mode) override {
                if (mode == 0) return nullptr;
                const std::string key = key_of(chunk, launch_mode);
                std::unique_lock<std::mutex> lock(guard);
                auto found = table.find(key);
                if (found != table.end()) {
                    return found->second.state == Entry::kReady ? &found->second.special : nullptr;
                }
                if (table.size() >= kCacheLimit) return nullptr;
                table.emplace(key, Entry{});
                Job job{key, chunk, launch_mode};
                if (mode == 2) {
                    lock.unlock();
                    Entry built = compile(job);
                    lock.lock();
                    auto &slot = table[key];
                    slot = built;
                    if (built.state != Entry::kReady) {
                        ctx.error = "NVRTC specialisation failed; the interpreter runs this chunk";
                        return nullptr;
                    }
                    return &slot.special;
                }
                queue.push_back(job);
                ++pending;
                wake.notify_one();
                return nullptr;
            }

            void wait() override {
                std::unique_lock<std::mutex> lock(guard);
                idle.wait(lock, [this] { return pending == 0; });
            }

        private:
            void loop() {
                cudaSetDevice(device);
                cudaFree(nullptr);  // makes the primary context current on this thread
                std::unique_lock<std::mutex> lock(guard);
                for (;;) {
                    wake.wait(lock, [this] { return stop || !queue.empty(); });
                    if (stop) break;
                    Job job = queue.front();
                    queue.pop_front();
                    lock.unlock();
                    Entry built = compile(job);
                    lock.lock();
                    table[job.key] = built;
                    --pending;
                    idle.notify_all();
                }
            }

            Entry compile(const Job &job) {
                const auto started = std::chrono::steady_clock::now();
                Entry entry;
                entry.state = Entry::kFailed;
                std::string name;
                const std::string source = program_of(job.chunk, job.mode, name);
                const char *headers[] = {sci_embedded_math, sci_embedded_kernel, sci_embedded_gradient, sci_embedded_batch};
                const char *names[] = {"sci_math.cuh", "chunk_kernel.cuh", "gradient_kernel.cuh", "batch_kernel.cuh"};
                nvrtcProgram program;
                if (nvrtcCreateProgram(&program, source.c_str(), "sci_specialized.cu", 4, headers, names) != NVRTC_SUCCESS)
                    return entry;
                nvrtcAddNameExpression(program, name.c_str());
                // --fmad=false: the chunk codes are exact sequences of rounded operations, so no
                // multiply and add may be contracted behind their back; the packed two-lane forms
                // need it most, since ptxas would otherwise fuse a packed multiply into a following
                // packed add.
                const char *options[] = {"-default-device", "-arch=sm_100a", "-std=c++17", "-lineinfo",
                                         "--extra-device-vectorization", "--fmad=false"};
                const nvrtcResult built = nvrtcCompileProgram(program, 6, options);
                if (built != NVRTC_SUCCESS) {
                    if (trace) {
                        size_t size = 0;
                        nvrtcGetProgramLogSize(program, &size);
                        std::string log(size, '\0');
                        nvrtcGetProgramLog(program, log.data());
                        std::fprintf(stderr, "[sci_cuda] NVRTC failed: %s\n", log.c_str());
                    }
                    nvrtcDestroyProgram(&program);
                    return entry;
                }
                const char *lowered = nullptr;
                nvrtcGetLoweredName(program, name.c_str(), &lowered);
                const std::string symbol = lowered ? lowered : "";
                size_t size = 0;
                nvrtcGetCUBINSize(program, &size);
                std::vector<char> cubin(size);
                nvrtcGetCUBIN(program, cubin.data());
                nvrtcDestroyProgram(&program);
                cudaSetDevice(device);
                cudaFree(nullptr);
                CUmodule module = nullptr;
                CUfunction function = nullptr;
                if (Driver::get().module_load(&module, cubin.data()) != CUDA_SUCCESS) return entry;
                if (Driver::get().module_function(&function, module, symbol.c_str()) != CUDA_SUCCESS) {
                    Driver::get().module_unload(module);
                    return entry;
                }
                entry.state = Entry::kReady;
                entry.module = module;
                entry.special.function = reinterpret_cast<const void *>(function);
                if (trace) {
                    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - started).count();
                    std::fprintf(stderr, "[sci_cuda] specialised %s (%d instructions) in %.0f ms\n", symbol.c_str(),
                                 job.chunk.length, ms);
                }
                return entry;
            }

            int device;
            int mode;
            bool trace;
            std::mutex guard;
            std::condition_variable wake, idle;
            std::deque<Job> queue;
            std::unordered_map<std::string, Entry> table;
            int pending{0};
            bool stop{false};
            std::thread worker;
        };

    } // namespace

    std::unique_ptr<Specializer> make_specializer(Context &ctx) {
        if (!Driver::get().ready) return nullptr;
        return std::make_unique<Nvrtc>(ctx);
    }

} // namespace sci_cuda
