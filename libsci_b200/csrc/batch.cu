// batch.cu -- many instances of one chunk in one persistent, graph-captured launch (new; the
// reference's analogue is its Vulkan command-buffer batching, src/core/drivers/vulkan/stream.cpp:
// 71-106). See batch_kernel.cuh for the kernel.
//
// sci_cuda_batch_create does the one-time work: it checks every item, compiles the chunk into its
// NVRTC instance of batch_stream (synchronously: the batch is built once and replayed), tunes the
// unit span of each item-size bucket (< 4096, < 65536, larger elements), lays out the item and unit
// tables in device memory and captures "clear the queue, launch" into a CUDA graph.
// sci_cuda_batch_launch replays that graph on the context's stream.
//
// The autotuner times every candidate span on the bucket's own items (one warm-up and three timed
// launches, CUDA events, median) and keeps the fastest. Results are cached per device name,
// precision, chunk signature and bucket, in memory and in a text file (SCI_CUDA_TUNE_CACHE, default
// $HOME/.cache/sci_cuda/batch_tune.txt) that later processes read; SCI_CUDA_TUNE=0 skips tuning.
#include "batch_kernel.cuh"
#include "context.hpp"
#include "solve_batch_kernel.cuh"
#include "specialize.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <sys/stat.h>
#include <vector>

using namespace sci_cuda;

struct sci_cuda_batch {
    sci_cuda_context *context{nullptr};
    bool wide{false};
    unsigned spans[3]{};
    int specialized{0};
    void *memory{nullptr};
    cudaGraph_t graph{nullptr};
    cudaGraphExec_t exec{nullptr};
};

namespace {

    constexpr int kBuckets = 3;
    constexpr unsigned long long kBucketLimit[kBuckets - 1] = {4096, 65536};
    constexpr unsigned kCandidates[] = {256, 1024, 4096, 16384, 65536};
    constexpr unsigned kDefaultSpan[kBuckets] = {1024, 4096, 16384};

    int bucket_of(unsigned long long count) { return count < kBucketLimit[0] ? 0 : (count < kBucketLimit[1] ? 1 : 2); }

    // ---- the tuning cache ------------------------------------------------------------------------
    std::mutex cache_guard;
    std::map<std::string, unsigned> cache;
    bool cache_loaded = false;

    std::string cache_path() {
        if (const char *path = std::getenv("SCI_CUDA_TUNE_CACHE")) return path;
        const char *home = std::getenv("HOME");
        return std::string(home ? home : "/tmp") + "/.cache/sci_cuda/batch_tune.txt";
    }

    void load_cache() {
        if (cache_loaded) return;
        cache_loaded = true;
        std::ifstream in(cache_path());
        std::string key;
        unsigned span;
        while (in >> key >> span) cache[key] = span;
    }

    void store_cache(const std::string &key, unsigned span) {
        cache[key] = span;
        const std::string path = cache_path();
        const size_t slash = path.find_last_of('/');
        if (slash != std::string::npos) {
            std::string dir = path.substr(0, slash);
            for (size_t at = 1; at <= dir.size(); ++at) {
                if (at == dir.size() || dir[at] == '/') mkdir(dir.substr(0, at).c_str(), 0755);
            }
        }
        std::ofstream out(path, std::ios::app);
        out << key << ' ' << span << '\n';
    }

    std::string tune_key(const Context &ctx, const sci_chunk &chunk, int bucket) {
        std::string key;
        for (char ch : ctx.name) key += (ch == ' ' ? '_' : ch);
        char part[16];
        std::snprintf(part, sizeof(part), "|%d|%d|", chunk.precision, bucket);
        key += part;
        auto hex = [&](unsigned v) {
            std::snprintf(part, sizeof(part), "%02x", v & 0xff);
            key += part;
        };
        hex(chunk.arguments), hex(chunk.literals), hex(chunk.temporaries), hex(chunk.result);
        for (int i = 0; i < chunk.length; ++i) {
            const sci_instruction &ins = chunk.instructions[i];
            hex(ins.code), hex(ins.target), hex(ins.sources[0]), hex(ins.sources[1]), hex(ins.sources[2]);
        }
        return key;
    }

    // ---- device tables ----------------------------------------------------------------------------
    template <typename T> struct Tables {
        const T **inputs;
        T **outputs;
        unsigned long long *counts;
        unsigned *first_unit, *unit_count;
        BatchUnit *units;
        double *partials;
        unsigned *magnitudes, *tickets;
        unsigned long long *queue;
    };

    struct Layout {
        size_t bytes{0};
        size_t take(size_t count, size_t size) {
            const size_t at = bytes;
            bytes += (count * size + 255) / 256 * 256;
            return at;
        }
    };

    // Units of the items in `order` whose bucket is selected, `spans[bucket]` elements each;
    // first_unit / unit_count of the other items are zero.
    void cut(const std::vector<unsigned long long> &counts, const std::vector<unsigned> &order, const unsigned *spans,
             const bool *selected, std::vector<BatchUnit> &units, std::vector<unsigned> &first, std::vector<unsigned> &number) {
        units.clear();
        std::fill(first.begin(), first.end(), 0u);
        std::fill(number.begin(), number.end(), 0u);
        for (unsigned item : order) {
            const int b = bucket_of(counts[item]);
            if (!selected[b]) continue;
            first[item] = static_cast<unsigned>(units.size());
            const unsigned long long span = spans[b];
            if (counts[item] == 0) units.push_back(BatchUnit{0, item, 0});
            for (unsigned long long start = 0; start < counts[item]; start += span)
                units.push_back(BatchUnit{start, item, static_cast<unsigned>(std::min(span, counts[item] - start))});
            number[item] = static_cast<unsigned>(units.size()) - first[item];
        }
    }

    template <typename T>
    int create(sci_cuda_batch &batch, Context &ctx, const sci_chunk &chunk, uint32_t fold, const sci_batch_items &items) {
        const unsigned n = items.items;
        const unsigned A = chunk.arguments;
        const bool reduce = items.results != nullptr;
        std::vector<unsigned long long> counts(items.counts, items.counts + n);
        std::vector<const T *> inputs(size_t(n) * A);
        std::vector<T *> outputs(n, nullptr);
        bool stores = false;
        for (int i = 0; i < chunk.length; ++i) stores = stores || chunk.instructions[i].target == SCI_SLOT_OUTPUT;
        for (unsigned item = 0; item < n; ++item) {
            for (unsigned a = 0; a < A; ++a) {
                const void *p = items.inputs[size_t(item) * A + a];
                if (counts[item] && (!p || !reachable(ctx, p)))
                    return ctx.fail(SCI_CUDA_ERROR_INVALID, "item %u input %u (%p) is not memory of this device", item, a, p);
                inputs[size_t(item) * A + a] = static_cast<const T *>(p);
            }
            if (stores && items.outputs) {
                void *p = items.outputs[item];
                if (counts[item] && (!p || !reachable(ctx, p)))
                    return ctx.fail(SCI_CUDA_ERROR_INVALID, "item %u output (%p) is not memory of this device", item, p);
                outputs[item] = static_cast<T *>(p);
            }
        }
        if (reduce && !reachable(ctx, items.results)) return ctx.fail(SCI_CUDA_ERROR_INVALID, "results are not memory of this device");

        // the kernel: the chunk's NVRTC instance, compiled now, or the interpreter
        const Specialized *special = nullptr;
        if (ctx.specializer) {
            special = ctx.specializer->find(ctx, chunk, kBatchMode);
            if (!special) {
                ctx.specializer->wait();
                special = ctx.specializer->find(ctx, chunk, kBatchMode);
            }
        }
        batch.specialized = special ? 1 : 0;
        const void *generic = reinterpret_cast<const void *>(&batch_stream<T, Dynamic>);
        int per_sm = 1;
        if (special) {
            CUfunction function = reinterpret_cast<CUfunction>(const_cast<void *>(special->function));
            if (Driver::get().occupancy(&per_sm, function, 256, 0) != CUDA_SUCCESS || per_sm < 1) per_sm = 1;
        } else {
            per_sm = ctx.blocks_per_sm(generic, 256, 0);
        }
        const unsigned grid = static_cast<unsigned>(per_sm * ctx.sms);

        // tables, sized for the smallest span any bucket can take
        unsigned long long most = 0;
        for (unsigned long long c : counts) most += std::max<unsigned long long>(1, (c + kCandidates[0] - 1) / kCandidates[0]);
        Layout layout;
        const size_t o_inputs = layout.take(size_t(n) * std::max(1u, A), sizeof(void *));
        const size_t o_outputs = layout.take(n, sizeof(void *));
        const size_t o_counts = layout.take(n, 8);
        const size_t o_first = layout.take(n, 4), o_number = layout.take(n, 4);
        const size_t o_units = layout.take(most, sizeof(BatchUnit));
        const size_t o_partials = layout.take(most, 8), o_magnitudes = layout.take(most, 4);
        const size_t o_tickets = layout.take(n, 4), o_queue = layout.take(1, 8);
        if (int code = ctx.check(cudaMalloc(&batch.memory, layout.bytes), "allocating the batch tables")) return code;
        auto *base = static_cast<unsigned char *>(batch.memory);
        Tables<T> t{reinterpret_cast<const T **>(base + o_inputs), reinterpret_cast<T **>(base + o_outputs),
                    reinterpret_cast<unsigned long long *>(base + o_counts), reinterpret_cast<unsigned *>(base + o_first),
                    reinterpret_cast<unsigned *>(base + o_number), reinterpret_cast<BatchUnit *>(base + o_units),
                    reinterpret_cast<double *>(base + o_partials), reinterpret_cast<unsigned *>(base + o_magnitudes),
                    reinterpret_cast<unsigned *>(base + o_tickets), reinterpret_cast<unsigned long long *>(base + o_queue)};
        cudaStream_t stream = ctx.stream;
        cudaMemcpyAsync(t.inputs, inputs.data(), inputs.size() * sizeof(void *), cudaMemcpyHostToDevice, stream);
        cudaMemcpyAsync(t.outputs, outputs.data(), n * sizeof(void *), cudaMemcpyHostToDevice, stream);
        cudaMemcpyAsync(t.counts, counts.data(), n * 8, cudaMemcpyHostToDevice, stream);
        cudaMemsetAsync(t.tickets, 0, n * 4, stream);

        BatchLaunch<T> L;
        std::memset(&L, 0, sizeof(L));
        for (int s = 0; s < chunk.length; ++s) {
            const sci_instruction &ins = chunk.instructions[s];
            L.steps[s] = Step{ins.code, ins.target, ins.sources[0], ins.sources[1], ins.sources[2]};
            if (ins.code == SCI_CODE_MINIMUM || ins.code == SCI_CODE_MAXIMUM) L.tailed = 1;
        }
        L.length = chunk.length;
        L.arguments = A;
        L.temporaries = chunk.temporaries;
        L.result = chunk.result;
        L.fold = fold;
        L.reduce = reduce ? 1u : 0u;
        for (int i = 0; i < chunk.literals; ++i) L.constants[i] = static_cast<T>(chunk.constants[i]);
        L.inputs = t.inputs;
        L.outputs = stores && items.outputs ? t.outputs : nullptr;
        L.counts = t.counts;
        L.first_unit = t.first_unit;
        L.unit_count = t.unit_count;
        L.units = t.units;
        L.partials = t.partials;
        L.magnitudes = t.magnitudes;
        L.tickets = t.tickets;
        L.queue = t.queue;
        L.results = static_cast<double *>(items.results);

        auto launch = [&]() -> int {
            cudaMemsetAsync(t.queue, 0, 8, stream);
            void *args[] = {&L};
            if (special) {
                CUfunction function = reinterpret_cast<CUfunction>(const_cast<void *>(special->function));
                if (Driver::get().launch(function, grid, 1, 1, 256, 1, 1, 0, stream, args, nullptr) != CUDA_SUCCESS)
                    return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "launching the specialised batch kernel");
                return SCI_CUDA_OK;
            }
            return ctx.check(cudaLaunchKernel(generic, dim3(grid), dim3(256), args, 0, stream), "launching the batch kernel");
        };

        // items largest first, so the long units start early and the short ones fill the end
        std::vector<unsigned> order(n);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](unsigned x, unsigned y) { return counts[x] > counts[y]; });
        std::vector<BatchUnit> units;
        std::vector<unsigned> first(n), number(n);
        auto upload_units = [&]() {
            cudaMemcpyAsync(t.units, units.data(), units.size() * sizeof(BatchUnit), cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(t.first_unit, first.data(), n * 4, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(t.unit_count, number.data(), n * 4, cudaMemcpyHostToDevice, stream);
            L.unit_total = units.size();
            // the host vectors are reused at once: wait for the copies
            return ctx.check(cudaStreamSynchronize(stream), "uploading the batch units");
        };

        // tune the span of every bucket that has items
        std::copy(kDefaultSpan, kDefaultSpan + kBuckets, batch.spans);
        const char *tune = std::getenv("SCI_CUDA_TUNE");
        const bool tuning = !(tune && tune[0] == '0');
        bool present[kBuckets] = {};
        unsigned long long largest[kBuckets] = {};
        for (unsigned long long c : counts) {
            present[bucket_of(c)] = true;
            largest[bucket_of(c)] = std::max(largest[bucket_of(c)], c);
        }
        {
            std::lock_guard<std::mutex> lock(cache_guard);
            load_cache();
        }
        for (int b = 0; b < kBuckets && tuning; ++b) {
            if (!present[b]) continue;
            const std::string key = tune_key(ctx, chunk, b);
            {
                std::lock_guard<std::mutex> lock(cache_guard);
                auto hit = cache.find(key);
                if (hit != cache.end()) {
                    batch.spans[b] = hit->second;
                    continue;
                }
            }
            bool selected[kBuckets] = {};
            selected[b] = true;
            float best = -1.0f;
            for (unsigned span : kCandidates) {
                if (span > kCandidates[0] && span / 2 >= largest[b]) break;  // longer than every item
                unsigned spans[kBuckets];
                std::copy(batch.spans, batch.spans + kBuckets, spans);
                spans[b] = span;
                cut(counts, order, spans, selected, units, first, number);
                if (int code = upload_units()) return code;
                cudaEvent_t start, stop;
                cudaEventCreate(&start);
                cudaEventCreate(&stop);
                std::vector<float> times;
                for (int rep = 0; rep < 4; ++rep) {
                    cudaEventRecord(start, stream);
                    if (int code = launch()) return code;
                    cudaEventRecord(stop, stream);
                    if (int code = ctx.check(cudaEventSynchronize(stop), "timing a batch span")) return code;
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, start, stop);
                    if (rep > 0) times.push_back(ms);
                }
                cudaEventDestroy(start);
                cudaEventDestroy(stop);
                std::sort(times.begin(), times.end());
                if (best < 0.0f || times[1] < best) {
                    best = times[1];
                    batch.spans[b] = span;
                }
            }
            std::lock_guard<std::mutex> lock(cache_guard);
            store_cache(key, batch.spans[b]);
        }

        bool all[kBuckets] = {true, true, true};
        cut(counts, order, batch.spans, all, units, first, number);
        if (int code = upload_units()) return code;

        // capture "clear the queue, launch" into a graph
        if (int code = ctx.check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capturing the batch")) return code;
        const int launched = launch();
        cudaGraph_t graph = nullptr;
        const cudaError_t ended = cudaStreamEndCapture(stream, &graph);
        if (launched) {
            if (graph) cudaGraphDestroy(graph);
            return launched;
        }
        if (int code = ctx.check(ended, "ending the batch capture")) return code;
        batch.graph = graph;
        return ctx.check(cudaGraphInstantiate(&batch.exec, graph, 0), "instantiating the batch graph");
    }

} // namespace

extern "C" int sci_cuda_batch_create(sci_cuda_context *context, const sci_chunk *chunk, uint32_t fold,
                                     const sci_batch_items *items, sci_cuda_batch **batch) {
    if (!context || !batch) return SCI_CUDA_ERROR_INVALID;
    *batch = nullptr;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (!items || (items->items && (!items->counts || (chunk && chunk->arguments && !items->inputs))))
        return context->fail(SCI_CUDA_ERROR_INVALID, "null batch tables");
    if (int code = validate(*context, chunk, items->results != nullptr)) return code;
    if (fold > SCI_FOLD_MAXIMUM) return context->fail(SCI_CUDA_ERROR_INVALID, "unknown fold %u", fold);
    unsigned long long units = 0;
    for (uint32_t i = 0; i < items->items; ++i) units += items->counts[i] / kCandidates[0] + 1;
    if (units >= (1ull << 32)) return context->fail(SCI_CUDA_ERROR_UNSUPPORTED, "batch of %llu units", units);
    cudaSetDevice(context->device);
    auto *made = new sci_cuda_batch;
    made->context = context;
    made->wide = chunk->precision == SCI_PRECISION_WIDE;
    const int code = made->wide ? create<double>(*made, *context, *chunk, fold, *items)
                                : create<float>(*made, *context, *chunk, fold, *items);
    if (code) {
        sci_cuda_batch_destroy(made);
        return code;
    }
    *batch = made;
    return SCI_CUDA_OK;
}

extern "C" int sci_cuda_batch_launch(sci_cuda_batch *batch) {
    if (!batch || !batch->exec) return SCI_CUDA_ERROR_INVALID;
    sci_cuda_context *context = batch->context;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    return context->check(cudaGraphLaunch(batch->exec, context->stream), "launching the batch graph");
}

extern "C" int sci_cuda_batch_spans(const sci_cuda_batch *batch, uint32_t *spans, int32_t *specialized) {
    if (!batch) return SCI_CUDA_ERROR_INVALID;
    if (spans)
        for (int b = 0; b < kBuckets; ++b) spans[b] = batch->spans[b];
    if (specialized) *specialized = batch->specialized;
    return SCI_CUDA_OK;
}

extern "C" int sci_cuda_batch_destroy(sci_cuda_batch *batch) {
    if (!batch) return SCI_CUDA_OK;
    sci_cuda_context *context = batch->context;
    {
        std::lock_guard<std::recursive_mutex> lock(context->guard);
        cudaSetDevice(context->device);
        cudaStreamSynchronize(context->stream);
        if (batch->exec) cudaGraphExecDestroy(batch->exec);
        if (batch->graph) cudaGraphDestroy(batch->graph);
        if (batch->memory) cudaFree(batch->memory);
    }
    delete batch;
    return SCI_CUDA_OK;
}

// ---- batched small solves ---------------------------------------------------------------------
// Thousands of independent systems (n <= 256, one right-hand side, double operands), FP32 LU and
// FP64 refinement inside one CTA per system (solve_batch_kernel.cuh). Systems are grouped into four
// buckets by order (<= 32, <= 64, <= 128, <= 256); each bucket is one launch whose block size the
// autotuner picks among the variants that fit it (timed on the bucket's own systems, cached like
// the chunk batches' spans). The four launches are captured into one CUDA graph on parallel
// branches, so small buckets fill the gaps of the large one.

struct sci_cuda_solve_batch {
    sci_cuda_context *context{nullptr};
    void *memory{nullptr};
    unsigned threads[4]{};
    cudaStream_t branches[4]{};
    cudaEvent_t fork{nullptr}, joins[4]{};
    cudaGraph_t graph{nullptr};
    cudaGraphExec_t exec{nullptr};
};

namespace {

    struct Variant {
        int threads, rc;
        const void *kernel;
    };
    const Variant kVariants[] = {
            {32, 0, reinterpret_cast<const void *>(&small_solve<32, 0>)},
            {64, 0, reinterpret_cast<const void *>(&small_solve<64, 0>)},
            {128, 0, reinterpret_cast<const void *>(&small_solve<128, 0>)},
            {256, 0, reinterpret_cast<const void *>(&small_solve<256, 0>)},
            {256, kSmallRegisters, reinterpret_cast<const void *>(&small_solve<256, kSmallRegisters>)},
            {512, kSmallRegisters, reinterpret_cast<const void *>(&small_solve<512, kSmallRegisters>)},
    };

    int solve_bucket(unsigned n) { return n <= 32 ? 0 : (n <= 64 ? 1 : (n <= 128 ? 2 : 3)); }

    // The variants that may run a bucket whose largest order is `most`.
    std::vector<const Variant *> candidates(int bucket, unsigned most) {
        std::vector<const Variant *> out;
        for (const Variant &v : kVariants) {
            const bool registers = v.rc > 0;
            if (bucket < 3 && registers) continue;
            if (bucket == 3 && most > kSmallShared && !registers) continue;  // only the register form fits
            if (registers && static_cast<unsigned>(v.threads) < most) continue;
            if (bucket == 0 && v.threads > 128) continue;
            if (bucket >= 2 && v.threads < 64) continue;
            out.push_back(&v);
        }
        return out;
    }

} // namespace

extern "C" int sci_cuda_solve_batch_create(sci_cuda_context *context, const sci_solve_items *items,
                                           sci_cuda_solve_batch **batch) {
    if (!context || !batch) return SCI_CUDA_ERROR_INVALID;
    *batch = nullptr;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    Context &ctx = *context;
    if (!items || (items->systems && (!items->orders || !items->matrices || !items->rights || !items->solutions)))
        return ctx.fail(SCI_CUDA_ERROR_INVALID, "null system tables");
    cudaSetDevice(ctx.device);
    const unsigned count = items->systems;
    std::vector<SmallSystem> systems(count);
    std::vector<unsigned> lists[4];
    unsigned most[4] = {};
    for (unsigned s = 0; s < count; ++s) {
        const unsigned n = items->orders[s];
        if (n == 0 || n > static_cast<unsigned>(kSmallMax))
            return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "system %u: order %u outside 1..%d", s, n, kSmallMax);
        const void *a = items->matrices[s], *b = items->rights[s];
        void *x = items->solutions[s];
        if (!a || !b || !x || !reachable(ctx, a) || !reachable(ctx, b) || !reachable(ctx, x))
            return ctx.fail(SCI_CUDA_ERROR_INVALID, "system %u: an operand is not memory of this device", s);
        systems[s] = SmallSystem{static_cast<const double *>(a), static_cast<const double *>(b), static_cast<double *>(x), n, 0};
        const int b_ = solve_bucket(n);
        lists[b_].push_back(s);
        most[b_] = std::max(most[b_], n);
    }
    if ((items->errors && !reachable(ctx, items->errors)) || (items->iterations && !reachable(ctx, items->iterations)))
        return ctx.fail(SCI_CUDA_ERROR_INVALID, "errors / iterations are not memory of this device");
    for (auto &list : lists)
        std::stable_sort(list.begin(), list.end(), [&](unsigned x, unsigned y) { return systems[x].n > systems[y].n; });

    auto *made = new sci_cuda_solve_batch;
    made->context = context;
    const size_t table = (count * sizeof(SmallSystem) + 255) / 256 * 256;
    if (int code = ctx.check(cudaMalloc(&made->memory, table + 4ull * count + 256), "allocating the system tables")) {
        delete made;
        return code;
    }
    auto fail = [&](int code) {
        sci_cuda_solve_batch_destroy(made);
        return code;
    };
    auto *device_systems = static_cast<SmallSystem *>(made->memory);
    auto *device_order = reinterpret_cast<unsigned *>(static_cast<unsigned char *>(made->memory) + table);
    unsigned offsets[4] = {};
    std::vector<unsigned> flat;
    for (int b = 0; b < 4; ++b) {
        offsets[b] = static_cast<unsigned>(flat.size());
        flat.insert(flat.end(), lists[b].begin(), lists[b].end());
    }
    cudaMemcpyAsync(device_systems, systems.data(), count * sizeof(SmallSystem), cudaMemcpyHostToDevice, ctx.stream);
    cudaMemcpyAsync(device_order, flat.data(), flat.size() * 4, cudaMemcpyHostToDevice, ctx.stream);
    if (int code = ctx.check(cudaStreamSynchronize(ctx.stream), "uploading the system tables")) return fail(code);

    double *errors = items->errors;
    int *iterations = items->iterations;
    auto launch = [&](int b, const Variant &v, cudaStream_t stream) -> int {
        const unsigned long long smem = small_shared_bytes(most[b], v.rc);
        if (smem > ctx.shared_limit) return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "bucket %d needs %llu bytes of shared memory", b, smem);
        cudaFuncSetAttribute(v.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        const unsigned *order = device_order + offsets[b];
        void *args[] = {&device_systems, &order, &errors, &iterations};
        return ctx.check(cudaLaunchKernel(v.kernel, dim3(static_cast<unsigned>(lists[b].size())), dim3(v.threads), args, smem, stream),
                         "launching a batch of small solves");
    };

    // tune each bucket's block size
    const char *tune = std::getenv("SCI_CUDA_TUNE");
    const bool tuning = !(tune && tune[0] == '0');
    {
        std::lock_guard<std::mutex> guard(cache_guard);
        load_cache();
    }
    const Variant *chosen[4] = {};
    for (int b = 0; b < 4; ++b) {
        if (lists[b].empty()) continue;
        const auto options = candidates(b, most[b]);
        if (options.empty()) return fail(ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "no variant for bucket %d", b));
        chosen[b] = options.back();
        std::string key;
        for (char ch : ctx.name) key += (ch == ' ' ? '_' : ch);
        key += "|solve|" + std::to_string(b);
        if (!tuning) continue;
        {
            std::lock_guard<std::mutex> guard(cache_guard);
            auto hit = cache.find(key);
            if (hit != cache.end()) {
                for (const Variant *v : options)
                    if (static_cast<unsigned>(v->threads) == hit->second) chosen[b] = v;
                continue;
            }
        }
        float best = -1.0f;
        for (const Variant *v : options) {
            cudaEvent_t start, stop;
            cudaEventCreate(&start);
            cudaEventCreate(&stop);
            std::vector<float> times;
            for (int rep = 0; rep < 4; ++rep) {
                cudaEventRecord(start, ctx.stream);
                if (int code = launch(b, *v, ctx.stream)) return fail(code);
                cudaEventRecord(stop, ctx.stream);
                if (int code = ctx.check(cudaEventSynchronize(stop), "timing a solve variant")) return fail(code);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, start, stop);
                if (rep > 0) times.push_back(ms);
            }
            cudaEventDestroy(start);
            cudaEventDestroy(stop);
            std::sort(times.begin(), times.end());
            if (best < 0.0f || times[1] < best) {
                best = times[1];
                chosen[b] = v;
            }
        }
        std::lock_guard<std::mutex> guard(cache_guard);
        store_cache(key, static_cast<unsigned>(chosen[b]->threads));
    }
    for (int b = 0; b < 4; ++b) made->threads[b] = chosen[b] ? static_cast<unsigned>(chosen[b]->threads) : 0u;

    // capture: fork to one branch per bucket, join back
    cudaEventCreateWithFlags(&made->fork, cudaEventDisableTiming);
    for (int b = 0; b < 4; ++b) {
        cudaStreamCreateWithFlags(&made->branches[b], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&made->joins[b], cudaEventDisableTiming);
    }
    if (int code = ctx.check(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal), "capturing the solves"))
        return fail(code);
    int launched = SCI_CUDA_OK;
    cudaEventRecord(made->fork, ctx.stream);
    for (int b = 3; b >= 0 && !launched; --b) {
        if (!chosen[b]) continue;
        cudaStreamWaitEvent(made->branches[b], made->fork, 0);
        launched = launch(b, *chosen[b], made->branches[b]);
        cudaEventRecord(made->joins[b], made->branches[b]);
        cudaStreamWaitEvent(ctx.stream, made->joins[b], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ended = cudaStreamEndCapture(ctx.stream, &graph);
    if (launched) {
        if (graph) cudaGraphDestroy(graph);
        return fail(launched);
    }
    if (int code = ctx.check(ended, "ending the solve capture")) return fail(code);
    made->graph = graph;
    if (int code = ctx.check(cudaGraphInstantiate(&made->exec, graph, 0), "instantiating the solve graph")) return fail(code);
    *batch = made;
    return SCI_CUDA_OK;
}

extern "C" int sci_cuda_solve_batch_launch(sci_cuda_solve_batch *batch) {
    if (!batch || !batch->exec) return SCI_CUDA_ERROR_INVALID;
    sci_cuda_context *context = batch->context;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    cudaSetDevice(context->device);
    return context->check(cudaGraphLaunch(batch->exec, context->stream), "launching the solve graph");
}

extern "C" int sci_cuda_solve_batch_shapes(const sci_cuda_solve_batch *batch, uint32_t *threads) {
    if (!batch || !threads) return SCI_CUDA_ERROR_INVALID;
    for (int b = 0; b < 4; ++b) threads[b] = batch->threads[b];
    return SCI_CUDA_OK;
}

extern "C" int sci_cuda_solve_batch_destroy(sci_cuda_solve_batch *batch) {
    if (!batch) return SCI_CUDA_OK;
    sci_cuda_context *context = batch->context;
    {
        std::lock_guard<std::recursive_mutex> lock(context->guard);
        cudaSetDevice(context->device);
        cudaStreamSynchronize(context->stream);
        if (batch->exec) cudaGraphExecDestroy(batch->exec);
        if (batch->graph) cudaGraphDestroy(batch->graph);
        for (int b = 0; b < 4; ++b) {
            if (batch->branches[b]) cudaStreamDestroy(batch->branches[b]);
            if (batch->joins[b]) cudaEventDestroy(batch->joins[b]);
        }
        if (batch->fork) cudaEventDestroy(batch->fork);
        if (batch->memory) cudaFree(batch->memory);
    }
    delete batch;
    return SCI_CUDA_OK;
}
