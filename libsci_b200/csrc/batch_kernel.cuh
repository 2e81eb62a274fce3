// batch_kernel.cuh -- many instances of one chunk in one persistent launch.
//
// The reference records one dispatch per array operation and submits them in batches through a
// Vulkan command buffer (src/core/drivers/vulkan/stream.cpp:71-106: up to 128 dispatches or 2^30
// work per batch). Here thousands of uneven instances of one chunk run in a single launch: the
// host cuts every item (an instance: its own inputs, output and element count) into units of
// `span` elements (the span is tuned per item-size bucket), and each warp of a persistent grid
// takes units off a device work queue (an atomic counter). A lane runs the chunk over 32 bytes of
// each input per step (8 floats or 4 doubles, two 16-byte vectors when the item is aligned),
// stores the chunk's output and folds its reduced value. A unit's fold goes to a partial slot; the
// warp that finishes an item's last unit (an atomic ticket per item) folds that item's partials in
// unit order, so every item's result is deterministic, and puts the ticket back to zero. The queue
// counter is the only state a launch needs cleared first (a memset ahead of the kernel in the same
// CUDA graph).
//
// Per element the arithmetic is the chunk interpreter's (apply<code>, loop tails of the reference's
// AVX-512 table from each item's own count - count % (64 / sizeof(T))), so stored outputs are
// bit-identical to sci_cuda_execute on each item.
#pragma once

#include "chunk_kernel.cuh"

namespace sci_cuda {

    constexpr int kBatchMode = 16;  // specialisation mode of batch_stream

    // `length` elements of item `item` from element `start` on.
    struct BatchUnit {
        unsigned long long start;
        unsigned item;
        unsigned length;
    };

    template <typename T> struct BatchLaunch {
        Step steps[kCapacity];
        unsigned length, arguments, temporaries, result;
        unsigned fold;    // SCI_FOLD_*, when reducing
        unsigned reduce;  // fold the chunk's result into results[item]
        unsigned tailed;  // minimum / maximum present
        T constants[kCapacity];
        const T *const *inputs;            // items x arguments
        T *const *outputs;                 // items, or null: nothing stored
        const unsigned long long *counts;  // items
        const unsigned *first_unit;        // items: an item's units are consecutive
        const unsigned *unit_count;        // items
        const BatchUnit *units;
        unsigned long long unit_total;
        double *partials;     // one per unit
        unsigned *magnitudes; // one per unit (NaN tracking of minimum / maximum)
        unsigned *tickets;    // one per item, zero between launches
        unsigned long long *queue;  // the next unit; zero at launch
        double *results;      // items
    };

    // Folds a lane's `live` values into its running state, as fold_tile does for a full tile.
    template <typename T>
    __device__ __forceinline__ void fold_lanes(Fold &f, unsigned op, const T *value, int live) {
        constexpr int N = Lanes<T>::count;
        if (op == 0) {
            T lanes[N];
#pragma unroll
            for (int e = 0; e < N; ++e) lanes[e] = e < live ? value[e] : T(0);
#pragma unroll
            for (int width = N / 2; width > 0; width /= 2) {
#pragma unroll
                for (int e = 0; e < width; ++e) lanes[e] = add(lanes[e], lanes[e + width]);
            }
            f.total += static_cast<double>(lanes[0]);
        } else {
            T best = op == 1 ? from_bits(Limits<T>::infinity) : -from_bits(Limits<T>::infinity);
            unsigned magnitude = 0;
#pragma unroll
            for (int e = 0; e < N; ++e) {
                if (e < live) {
                    magnitude = max(magnitude, magnitude_bits(value[e]));
                    best = op == 1 ? fmin(best, value[e]) : fmax(best, value[e]);
                }
            }
            f.magnitude = max(f.magnitude, magnitude);
            f.total = combine(op, f.total, static_cast<double>(best));
        }
    }

    // One lane's step: elements [base, base + live) of one item. `value` receives the reduced value.
    template <typename T, class Program>
    __device__ __forceinline__ void batch_lanes(const BatchLaunch<T> &L, const T *const *ptrs, T *out,
                                                unsigned long long base, int live, bool vec, const bool *tail, T *value) {
        constexpr int N = Lanes<T>::count, W = Lanes<T>::width;
        if constexpr (!Program::baked) {
            // The interpreter: one element at a time, temporaries in a per-thread array.
            for (int e = 0; e < N; ++e) {
                value[e] = T(0);
                if (e >= live) continue;
                const unsigned long long i = base + e;
                T slot[kCapacity];
                T last = T(0);
                auto fetch = [&](unsigned id) -> T {
                    const unsigned kind = id & kTypes, index = id & 63;
                    if (kind == kInput) return ptrs[index][i];
                    if (kind == kLiteral) return L.constants[index];
                    if (id == kNone) return T(0);
                    if (id == kOutput) return last;
                    return slot[index];
                };
                for (unsigned s = 0; s < L.length; ++s) {
                    const Step st = L.steps[s];
                    const T r = apply_one<T>(st.code, fetch(st.a), fetch(st.b), fetch(st.c), tail[e]);
                    if (st.target == kOutput) {
                        last = r;
                        if (out) out[i] = r;
                    } else {
                        slot[st.target & 63] = r;
                    }
                }
                if (L.reduce) value[e] = fetch(L.result);
            }
        } else {
            using C = typename Program::chunk;
            constexpr int A = C::arguments > 0 ? C::arguments : 1;
            constexpr int R = C::temporaries > 0 ? C::temporaries : 1;
            T in[A][N];
#pragma unroll
            for (int a = 0; a < C::arguments; ++a) {
                const T *src = ptrs[a] + base;
                if (vec) {
                    load16(src, in[a]);
                    load16(src + W, in[a] + W);
                } else {
#pragma unroll
                    for (int e = 0; e < N; ++e) in[a][e] = e < live ? src[e] : T(0);
                }
            }
            T regs[R][N];
            T last[N];
#pragma unroll
            for (int e = 0; e < N; ++e) last[e] = T(0);
            auto get = [&](auto id_c, T *v) {
                constexpr int id = decltype(id_c)::value;
#pragma unroll
                for (int e = 0; e < N; ++e) {
                    if constexpr ((id & kTypes) == kInput) v[e] = in[id & 63][e];
                    else if constexpr ((id & kTypes) == kLiteral) v[e] = L.constants[id & 63];
                    else if constexpr (id == kNone) v[e] = T(0);
                    else if constexpr (id == kOutput) v[e] = last[e];
                    else v[e] = regs[id & 63][e];
                }
            };
            static_for<C::length>([&](auto step_c) {
                constexpr Step st = C::steps[decltype(step_c)::value];
                T a[N], b[N], c[N];
                get(Int<st.a>{}, a);
                get(Int<st.b>{}, b);
                get(Int<st.c>{}, c);
                apply_lanes<st.code, true>(a, b, c, last, tail);
                if constexpr (st.target == kOutput) {
                    if (out) {
                        T *dst = out + base;
                        if (vec) {
                            store16(dst, last);
                            store16(dst + W, last + W);
                        } else {
#pragma unroll
                            for (int e = 0; e < N; ++e)
                                if (e < live) dst[e] = last[e];
                        }
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < N; ++e) regs[st.target & 63][e] = last[e];
                }
            });
            if (L.reduce) get(Int<C::result>{}, value);
        }
    }

    template <typename T, class Program>
    __global__ void __launch_bounds__(256) batch_stream(const __grid_constant__ BatchLaunch<T> L) {
        constexpr int N = Lanes<T>::count;
        const unsigned lane = threadIdx.x & 31;
        const unsigned op = L.fold;
        const double empty = op == 0 ? 0.0 : (op == 1 ? __longlong_as_double(0x7ff0000000000000ll)
                                                      : __longlong_as_double((long long)0xfff0000000000000ull));
        unsigned arguments;
        if constexpr (Program::baked) arguments = Program::chunk::arguments;
        else arguments = L.arguments;
        for (;;) {
            unsigned long long u = 0;
            if (lane == 0) u = atomicAdd(L.queue, 1ull);
            u = __shfl_sync(0xffffffffu, u, 0);
            if (u >= L.unit_total) break;
            const BatchUnit unit = L.units[u];
            const unsigned item = unit.item;
            const unsigned long long count = L.counts[item];
            const unsigned long long tail_start = count - count % (64 / sizeof(T));
            const T *const *ptrs = L.inputs + 1ull * item * arguments;
            T *out = L.outputs ? L.outputs[item] : nullptr;
            // units start at multiples of 256 elements, so an item whose pointers are 16-byte
            // aligned takes vector accesses throughout
            bool aligned = reinterpret_cast<unsigned long long>(out) % 16 == 0;
            for (unsigned a = 0; a < arguments; ++a) aligned = aligned && reinterpret_cast<unsigned long long>(ptrs[a]) % 16 == 0;
            Fold f{empty, 0u};
            for (unsigned off = lane * N; off < unit.length; off += 32u * N) {
                const unsigned long long base = unit.start + off;
                const int live = unit.length - off < static_cast<unsigned>(N) ? static_cast<int>(unit.length - off) : N;
                bool tail[N];
#pragma unroll
                for (int e = 0; e < N; ++e) tail[e] = L.tailed != 0 && base + e >= tail_start;
                T value[N];
                batch_lanes<T, Program>(L, ptrs, out, base, live, aligned && live == N, tail, value);
                if (L.reduce) fold_lanes<T>(f, op, value, live);
            }
            if (!L.reduce) continue;
#pragma unroll
            for (int offset = 16; offset > 0; offset >>= 1) {
                f.total = combine(op, f.total, __shfl_xor_sync(0xffffffffu, f.total, offset));
                f.magnitude = max(f.magnitude, __shfl_xor_sync(0xffffffffu, f.magnitude, offset));
            }
            unsigned last = 0;
            if (lane == 0) {
                L.partials[u] = f.total;
                L.magnitudes[u] = f.magnitude;
                __threadfence();
                last = atomicAdd(&L.tickets[item], 1u) == L.unit_count[item] - 1 ? 1u : 0u;
            }
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                // this warp finished the item: fold its partials in unit order
                __threadfence();
                const unsigned first = L.first_unit[item], units = L.unit_count[item];
                double total = empty;
                unsigned magnitude = 0;
                for (unsigned k = lane; k < units; k += 32) {
                    total = combine(op, total, __ldcg(&L.partials[first + k]));
                    magnitude = max(magnitude, __ldcg(&L.magnitudes[first + k]));
                }
#pragma unroll
                for (int offset = 16; offset > 0; offset >>= 1) {
                    total = combine(op, total, __shfl_xor_sync(0xffffffffu, total, offset));
                    magnitude = max(magnitude, __shfl_xor_sync(0xffffffffu, magnitude, offset));
                }
                if (lane == 0) {
                    // an empty sum is 0 and an empty extreme NaN (dispatch.cpp:109-111)
                    const bool nan = magnitude > nan_floor<T>() || (count == 0 && op != 0);
                    L.results[item] = nan ? __longlong_as_double(0x7ff8000000000000ll) : total;
                    L.tickets[item] = 0;
                }
            }
        }
    }

} // namespace sci_cuda
