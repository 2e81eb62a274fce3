// chunk_kernel.cuh -- the persistent, TMA-fed chunk interpreter for sm_100a.
//
// One kernel source serves two programs:
//  - Dynamic: the generic interpreter. Each instruction is read from the launch's constant bank and
//    dispatched with a warp-uniform switch; temporaries live in a shared-memory slot file (one
//    column per thread, so no synchronisation is needed).
//  - Baked<...>: the same kernel with the bytecode fixed at compile time (an NVRTC
//    specialisation keyed by the chunk's signature, chunk.hpp:209-226). The instruction loop
//    unrolls, every code folds to straight-line math and temporaries become registers.
// Both stream their inputs the same way: a persistent grid (a few CTAs per SM) walks tiles of
// 32 bytes x blockDim per input (8 floats or 4 doubles per thread); one elected thread issues a
// 1-D TMA bulk copy (cp.async.bulk) per input per tile into a ring of shared-memory stages that
// an mbarrier guards, so several tiles per input are in flight while the block computes. Results
// leave with 128-bit stores. Reductions fold each thread's lanes in the element type, carry the
// running total in double, then fold a warp (shuffle), the block, and finally the grid in a
// single pass: every block writes one double partial and the last block to arrive (an atomic
// ticket) folds them in block order, so the result is deterministic for a given launch shape and
// a*b is never stored for sum(a*b).
//
// Behavioural reference: the Vulkan interpreter and its entry points
// (shaders/interpreter.slang:163-248, shaders/common/entries.slang:17-80), the CPU sweep
// (src/core/drivers/processor/dispatch.cpp:42-165) and the NaN rules of core::Accumulator
// (include/core/bytecode/accumulator.hpp:28-34).
#pragma once

#include "sci_math.cuh"

namespace sci_cuda {

    constexpr int kCapacity = 64;
    constexpr int kMaxStages = 4;
    constexpr int kMaxBlocks = 4096;           // bound on the persistent grid (partials of a reduction)
    constexpr unsigned kWaitLimit = 1u << 22;  // bounded spin on an mbarrier phase

    // A thread carries 32 bytes of each input through the chunk per tile: two 16-byte vectors.
    template <typename T> struct Lanes {
        static constexpr int count = 32 / sizeof(T);   // elements per thread per tile
        static constexpr int width = 16 / sizeof(T);   // elements per 16-byte vector
        static constexpr int vectors = count / width;  // 16-byte vectors per thread per tile
    };

    enum Mode : int { kEvaluate = 0, kReduce = 1, kDot = 2 };
    enum Slot : int { kInput = 0x00, kLiteral = 0x40, kTemporary = 0x80, kOutput = 0xC0, kNone = 0xFF, kTypes = 0xC0 };
    enum Status : int { kStatusTimeout = 1 };

    struct Step {
        unsigned char code, target, a, b, c;
    };

    // Scratch of the single-pass global fold: one partial (and NaN flag) per block, and the ticket
    // the last block takes. The ticket returns to zero at the end of every launch.
    struct ReduceState {
        double partial[kMaxBlocks];
        int poisoned[kMaxBlocks];
        unsigned int ticket;
    };

    // Everything one launch needs, passed by value as a __grid_constant__ parameter (about
    // 1.5 KB), so the launch is self-contained and can be captured into a CUDA graph.
    template <typename T> struct Launch {
        Step steps[kCapacity];
        unsigned int length;       // instructions to run (the contracted multiply is skipped)
        unsigned int value;        // value id that is reduced
        unsigned int arguments;
        unsigned int temporaries;
        unsigned int fold;         // 0 sum, 1 minimum, 2 maximum
        unsigned int dot_left, dot_right;
        unsigned int stages;       // TMA ring depth, 0 when the inputs are read directly
        unsigned int tailed;       // the chunk has a minimum or maximum (loop-tail forms matter)
        T constants[kCapacity];
        const T *inputs[kCapacity];
        T *output;
        unsigned long long count;
        unsigned long long tail_start;  // elements from here on take the one-lane Scalar forms
        ReduceState *state;
        double *destination;       // where the folded value is written (device memory)
        int *status;
    };

    // ---- the two programs --------------------------------------------------------------------------
    struct Dynamic {
        static constexpr bool baked = false;
    };

    // Bytecode fixed at compile time. `Chunk` provides static constexpr members length, result,
    // arguments, temporaries, dot_left, dot_right and a constexpr array steps[].
    template <class Chunk> struct Baked {
        static constexpr bool baked = true;
        using chunk = Chunk;
        __host__ __device__ static constexpr bool tailed() {
            for (int i = 0; i < Chunk::length; ++i) {
                if (Chunk::steps[i].code == kMinimum || Chunk::steps[i].code == kMaximum) return true;
            }
            return false;
        }
    };

    template <int... I> struct Sequence {};
    template <int N, int... I> struct MakeSequence : MakeSequence<N - 1, N - 1, I...> {};
    template <int... I> struct MakeSequence<0, I...> {
        using type = Sequence<I...>;
    };
    template <int N> struct Int {
        static constexpr int value = N;
    };
    template <typename F, int... I> __device__ __forceinline__ void for_each(F &&f, Sequence<I...>) {
        (f(Int<I>{}), ...);
    }
    template <int N, typename F> __device__ __forceinline__ void static_for(F &&f) {
        for_each(f, typename MakeSequence<N>::type{});
    }

    // ---- applying one code to a thread's lanes -------------------------------------------------
    // With `fast`, a code that has a fast form runs it on every lane (two lanes per instruction where
    // it has a paired form), and a thread with any lane outside the fast form's inputs recomputes all
    // its lanes with the full form: one branch per thread, taken only for such inputs, and the same
    // values either way.
    //
    // Float tanh has a second fast form for |x| <= 1 (tanh_float_near: a polynomial instead of the
    // exponential and the quotient), taken when every lane of every active thread of the warp is in
    // that range (one vote, so a warp never runs both forms); its results are the same bits.
    template <int code, bool fast = false, typename T>
    __device__ __forceinline__ void apply_lanes(const T *a, const T *b, const T *c, T *r, const bool *tail) {
        if constexpr (fast && code == kTanh && sizeof(T) == 4) {
            bool near = true;
#pragma unroll
            for (int e = 0; e < Lanes<T>::count; ++e) near = near && fabsf(a[e]) <= 1.0f;  // false for NaN
            if (__all_sync(__activemask(), near)) {
                bool rare = false;
#pragma unroll
                for (int e = 0; e < Lanes<T>::count; ++e) r[e] = tanh_float_near(a[e], rare);
                if (rare) {
#pragma unroll
                    for (int e = 0; e < Lanes<T>::count; ++e) r[e] = apply<code>(a[e], b[e], c[e], tail[e]);
                }
                return;
            }
        }
        if constexpr (fast && has_fast<code, T>()) {
            bool rare = false;
            if constexpr (has_pair<code, T>()) {
#pragma unroll
                for (int e = 0; e < Lanes<T>::count; e += 2) apply_pair<code>(a[e], a[e + 1], rare, r[e], r[e + 1]);
            } else {
#pragma unroll
                for (int e = 0; e < Lanes<T>::count; ++e) r[e] = apply_fast<code>(a[e], rare);
            }
            if (rare) {
#pragma unroll
                for (int e = 0; e < Lanes<T>::count; ++e) r[e] = apply<code>(a[e], b[e], c[e], tail[e]);
            }
        } else {
#pragma unroll
            for (int e = 0; e < Lanes<T>::count; ++e) r[e] = apply<code>(a[e], b[e], c[e], tail[e]);
        }
    }

    template <typename T>
    __device__ __forceinline__ void apply_dynamic(int code, const T *a, const T *b, const T *c, T *r, const bool *tail) {
        switch (code) {
#define SCI_CASE(N) \
    case N: apply_lanes<N>(a, b, c, r, tail); break;
            SCI_CASE(0) SCI_CASE(1) SCI_CASE(2) SCI_CASE(3) SCI_CASE(4) SCI_CASE(5) SCI_CASE(6) SCI_CASE(7)
            SCI_CASE(8) SCI_CASE(9) SCI_CASE(10) SCI_CASE(11) SCI_CASE(12) SCI_CASE(13) SCI_CASE(14) SCI_CASE(15)
            SCI_CASE(16) SCI_CASE(17) SCI_CASE(18) SCI_CASE(19) SCI_CASE(20) SCI_CASE(21) SCI_CASE(22) SCI_CASE(23)
            SCI_CASE(24) SCI_CASE(25) SCI_CASE(26) SCI_CASE(27) SCI_CASE(28) SCI_CASE(29) SCI_CASE(30) SCI_CASE(31)
            SCI_CASE(32) SCI_CASE(33) SCI_CASE(34) SCI_CASE(35) SCI_CASE(36)
#undef SCI_CASE
        default:
#pragma unroll
            for (int e = 0; e < Lanes<T>::count; ++e) r[e] = T(0);
        }
    }

    // One code on one element, dispatched at run time.
    template <typename T> __device__ __forceinline__ T apply_one(int code, T a, T b, T c, bool tail) {
        switch (code) {
#define SCI_CASE(N) \
    case N: return apply<N>(a, b, c, tail);
            SCI_CASE(0) SCI_CASE(1) SCI_CASE(2) SCI_CASE(3) SCI_CASE(4) SCI_CASE(5) SCI_CASE(6) SCI_CASE(7)
            SCI_CASE(8) SCI_CASE(9) SCI_CASE(10) SCI_CASE(11) SCI_CASE(12) SCI_CASE(13) SCI_CASE(14) SCI_CASE(15)
            SCI_CASE(16) SCI_CASE(17) SCI_CASE(18) SCI_CASE(19) SCI_CASE(20) SCI_CASE(21) SCI_CASE(22) SCI_CASE(23)
            SCI_CASE(24) SCI_CASE(25) SCI_CASE(26) SCI_CASE(27) SCI_CASE(28) SCI_CASE(29) SCI_CASE(30) SCI_CASE(31)
            SCI_CASE(32) SCI_CASE(33) SCI_CASE(34) SCI_CASE(35) SCI_CASE(36)
#undef SCI_CASE
        default:
            return T(0);
        }
    }

    // ---- mbarrier and bulk-copy primitives (PTX ISA 8.x, sm_90+) -------------------------------
    __device__ __forceinline__ unsigned smem_address(const void *p) {
        return static_cast<unsigned>(__cvta_generic_to_shared(p));
    }
    __device__ __forceinline__ void barrier_init(unsigned long long *bar, unsigned count) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_address(bar)), "r"(count) : "memory");
    }
    __device__ __forceinline__ void barrier_expect(unsigned long long *bar, unsigned bytes) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_address(bar)), "r"(bytes)
                     : "memory");
    }
    __device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
        asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_address(dst)),
                "l"(src), "r"(bytes), "r"(smem_address(bar))
                : "memory");
    }
    __device__ __forceinline__ bool barrier_try(unsigned long long *bar, unsigned parity) {
        unsigned done;
        asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(smem_address(bar)), "r"(parity)
                : "memory");
        return done != 0;
    }
    // Waits for a phase with a bounded number of attempts; false when the bound ran out.
    __device__ __forceinline__ bool barrier_wait(unsigned long long *bar, unsigned parity) {
        for (unsigned attempt = 0; attempt < kWaitLimit; ++attempt) {
            if (barrier_try(bar, parity)) return true;
        }
        return false;
    }

    // ---- 16-byte vector access ------------------------------------------------------------------
    template <typename T> __device__ __forceinline__ void load16(const T *p, T *v) {
        if constexpr (sizeof(T) == 4) {
            const float4 q = *reinterpret_cast<const float4 *>(p);
            v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
        } else {
            const double2 q = *reinterpret_cast<const double2 *>(p);
            v[0] = q.x, v[1] = q.y;
        }
    }
    template <typename T> __device__ __forceinline__ void store16(T *p, const T *v) {
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
        }
    }

    // ---- the per-block working state -------------------------------------------------------------
    // Lane e of thread t sits at in-tile position (e / W) * (W * threads) + W * t + e % W, with W the
    // elements of a 16-byte vector, so every 128-bit shared or global access is contiguous across a
    // warp. The positions are fixed per thread; only the tile's base moves.
    template <typename T, class Program> struct Work {
        static constexpr int N = Lanes<T>::count, W = Lanes<T>::width, V = Lanes<T>::vectors;
        const Launch<T> &L;
        const T *stage;     // this tile's staged inputs (A x tile elements), or null for direct reads
        T *slots;           // the dynamic program's temporaries (temporaries x tile), shared memory
        unsigned long long base;
        unsigned tile;      // elements in a full tile (N x threads)
        unsigned live;      // elements of this tile that exist
        unsigned first;     // position of this thread's first vector
        bool tailed;        // whether loop-tail forms can matter for this chunk
        bool tail[N];

        __device__ __forceinline__ Work(const Launch<T> &launch, T *slot_file, unsigned threads, unsigned t)
            : L(launch), stage(nullptr), slots(slot_file), base(0), tile(N * threads), live(N * threads),
              first(W * t), tailed(false) {
            if constexpr (Program::baked) tailed = Program::tailed();
            else tailed = launch.tailed != 0;
#pragma unroll
            for (int e = 0; e < N; ++e) tail[e] = false;
        }

        __device__ __forceinline__ unsigned position(int e) const { return (e / W) * (tile / V) + first + e % W; }

        __device__ __forceinline__ void at(unsigned long long tile_base, unsigned tile_live, const T *staged) {
            base = tile_base;
            live = tile_live;
            stage = staged;
            if (tailed) {
#pragma unroll
                for (int e = 0; e < N; ++e) tail[e] = base + position(e) >= L.tail_start;
            }
        }

        // Values of one input for this thread's lanes.
        __device__ __forceinline__ void input(unsigned a, T *v) const {
            if (stage) {
#pragma unroll
                for (int j = 0; j < V; ++j) load16(stage + a * tile + position(j * W), v + j * W);
            } else {
                const T *src = L.inputs[a] + base;
#pragma unroll
                for (int e = 0; e < N; ++e) v[e] = position(e) < live ? src[position(e)] : src[0];
            }
        }

        // Dynamic fetch of a value id into this thread's lanes.
        __device__ __forceinline__ void fetch(unsigned id, T *v) const {
            const unsigned kind = id & kTypes, slot = id & 63;
            if (kind == kInput) {
                input(slot, v);
            } else if (kind == kLiteral) {
                const T c = L.constants[slot];
#pragma unroll
                for (int e = 0; e < N; ++e) v[e] = c;
            } else if (id != kNone) {
#pragma unroll
                for (int j = 0; j < V; ++j) load16(slots + slot * tile + position(j * W), v + j * W);
            } else {
#pragma unroll
                for (int e = 0; e < N; ++e) v[e] = T(0);
            }
        }

        __device__ __forceinline__ void store_temp(unsigned slot, const T *v) const {
#pragma unroll
            for (int j = 0; j < V; ++j) store16(slots + slot * tile + position(j * W), v + j * W);
        }

        __device__ __forceinline__ void write_output(const T *v) const {
            T *dst = L.output + base;
            // 128-bit stores only on the staged path, whose operands the host checked to be 16-byte
            // aligned; the direct path serves unaligned outputs and stores element by element.
            if (stage != nullptr && live == tile) {
#pragma unroll
                for (int j = 0; j < V; ++j) store16(dst + position(j * W), v + j * W);
            } else {
#pragma unroll
                for (int e = 0; e < N; ++e)
                    if (position(e) < live) dst[position(e)] = v[e];
            }
        }
    };

    // Runs the chunk over this thread's lanes of one tile. On return `value` holds the lanes of
    // the reduced value (kReduce) or the two operands of the contracted multiply (kDot).
    template <typename T, class Program, int MODE>
    __device__ __forceinline__ void run_tile(const Work<T, Program> &w, T *value, T *second) {
        constexpr int N = Lanes<T>::count;
        if constexpr (!Program::baked) {
            const Launch<T> &L = w.L;
            T last[N];
#pragma unroll
            for (int e = 0; e < N; ++e) last[e] = T(0);
            for (unsigned s = 0; s < L.length; ++s) {
                const Step st = L.steps[s];
                T a[N], b[N], c[N];
                w.fetch(st.a, a);
                if (st.code >= kAdd) w.fetch(st.b, b);
                else {
#pragma unroll
                    for (int e = 0; e < N; ++e) b[e] = T(0);
                }
                if (st.code == kFuse) w.fetch(st.c, c);
                else {
#pragma unroll
                    for (int e = 0; e < N; ++e) c[e] = T(0);
                }
                apply_dynamic<T>(st.code, a, b, c, last, w.tail);
                if (st.target == kOutput) {
                    if constexpr (MODE == kEvaluate) w.write_output(last);
                } else {
                    w.store_temp(st.target & 63, last);
                }
            }
            if constexpr (MODE == kReduce) {
                if (L.value == kOutput) {
#pragma unroll
                    for (int e = 0; e < N; ++e) value[e] = last[e];
                } else {
                    w.fetch(L.value, value);
                }
            } else if constexpr (MODE == kDot) {
                w.fetch(L.dot_left, value);
                w.fetch(L.dot_right, second);
            }
        } else {
            using C = typename Program::chunk;
            constexpr int R = C::temporaries > 0 ? C::temporaries : 1;
            T regs[R][N];
            T last[N];
            auto get = [&](auto id_c, T *v) {
                constexpr int id = decltype(id_c)::value;
                if constexpr ((id & kTypes) == kInput) {
                    w.input(id & 63, v);
                } else if constexpr ((id & kTypes) == kLiteral) {
                    const T c = w.L.constants[id & 63];
#pragma unroll
                    for (int e = 0; e < N; ++e) v[e] = c;
                } else if constexpr (id == kNone) {
#pragma unroll
                    for (int e = 0; e < N; ++e) v[e] = T(0);
                } else if constexpr (id == kOutput) {
#pragma unroll
                    for (int e = 0; e < N; ++e) v[e] = last[e];
                } else {
#pragma unroll
                    for (int e = 0; e < N; ++e) v[e] = regs[id & 63][e];
                }
            };
            static_for<C::length>([&](auto step_c) {
                constexpr Step st = C::steps[decltype(step_c)::value];
                T a[N], b[N], c[N];
                get(Int<st.a>{}, a);
                get(Int<st.b>{}, b);
                get(Int<st.c>{}, c);
                apply_lanes<st.code, true>(a, b, c, last, w.tail);
                if constexpr (st.target == kOutput) {
                    if constexpr (MODE == kEvaluate) w.write_output(last);
                } else {
#pragma unroll
                    for (int e = 0; e < N; ++e) regs[st.target & 63][e] = last[e];
                }
            });
            if constexpr (MODE == kReduce) {
                get(Int<C::result>{}, value);
            } else if constexpr (MODE == kDot) {
                get(Int<C::dot_left>{}, value);
                get(Int<C::dot_right>{}, second);
            }
        }
    }

    // Per-thread fold state: a double total plus a NaN flag. Minimum and maximum skip NaN and the
    // flag restores numpy's propagation, as entries.slang:55-78 and accumulator.hpp:28-34 do; a sum
    // lets NaN (and inf - inf) propagate arithmetically.
    struct Fold {
        double total;
        unsigned magnitude;  // largest |bits| seen by a minimum / maximum: above +inf's bits is NaN
    };

    __device__ __forceinline__ double combine(unsigned fold, double a, double b) {
        return fold == 0 ? a + b : (fold == 1 ? fmin(a, b) : fmax(a, b));
    }

    __device__ __forceinline__ float nan_min(float a, float b) {
        float r;
        asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
        return r;
    }
    __device__ __forceinline__ float nan_max(float a, float b) {
        float r;
        asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
        return r;
    }
    __device__ __forceinline__ unsigned magnitude_bits(float v) { return __float_as_uint(v) & 0x7fffffffu; }
    __device__ __forceinline__ unsigned magnitude_bits(double v) {
        // A double is NaN iff its high word without sign exceeds 0x7ff00000, or equals it with a
        // nonzero low word; folding the low word in as one bit keeps that order.
        const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v)) & 0x7fffffffffffffffull;
        return static_cast<unsigned>(b >> 32) | (static_cast<unsigned>(b) != 0u ? 1u : 0u);
    }
    template <typename T> __device__ __forceinline__ unsigned nan_floor() {
        return sizeof(T) == 4 ? 0x7f800000u : 0x7ff00000u;
    }

    // Folds one tile of this thread's lanes. A full tile folds its lanes in the element type first
    // (the reference folds whole 1024-element blocks that way, dispatch.cpp:121-150), then adds the
    // lane total to the double running total.
    template <typename T, int MODE, class W>
    __device__ __forceinline__ void fold_tile(Fold &f, unsigned fold, const T *value, const T *second, const W &w,
                                              bool full) {
        constexpr int N = Lanes<T>::count;
        if (MODE == kDot || fold == 0) {
            T lanes[N];
#pragma unroll
            for (int e = 0; e < N; ++e) {
                T v;
                if constexpr (MODE == kDot) v = fma_(value[e], second[e], T(0));
                else v = value[e];
                lanes[e] = (full || w.position(e) < w.live) ? v : T(0);
            }
            // pairwise within the thread, in the element type
#pragma unroll
            for (int width = N / 2; width > 0; width /= 2) {
#pragma unroll
                for (int e = 0; e < width; ++e) lanes[e] = add(lanes[e], lanes[e + width]);
            }
            f.total += static_cast<double>(lanes[0]);
        } else if constexpr (sizeof(T) == 4) {
            // NaN-propagating minimum / maximum: one instruction per lane, and a NaN among the
            // lanes shows in the result (the fold's value no longer matters then)
            T best = fold == 1 ? from_bits(Limits<T>::infinity) : -from_bits(Limits<T>::infinity);
            if (fold == 1) {
#pragma unroll
                for (int e = 0; e < N; ++e)
                    if (full || w.position(e) < w.live) best = nan_min(best, value[e]);
            } else {
#pragma unroll
                for (int e = 0; e < N; ++e)
                    if (full || w.position(e) < w.live) best = nan_max(best, value[e]);
            }
            if (is_nan(best)) f.magnitude = ~0u;
            else f.total = combine(fold, f.total, static_cast<double>(best));
        } else {
            T best = fold == 1 ? from_bits(Limits<T>::infinity) : -from_bits(Limits<T>::infinity);
            unsigned magnitude = 0;
#pragma unroll
            for (int e = 0; e < N; ++e) {
                if (full || w.position(e) < w.live) {
                    const T v = value[e];
                    magnitude = max(magnitude, magnitude_bits(v));
                    best = fold == 1 ? fmin(best, v) : fmax(best, v);
                }
            }
            f.magnitude = max(f.magnitude, magnitude);
            f.total = combine(fold, f.total, static_cast<double>(best));
        }
    }

    template <class Program, typename T> __device__ __forceinline__ unsigned arguments_of(const Launch<T> &L) {
        if constexpr (Program::baked) return Program::chunk::arguments;
        else return L.arguments;
    }

    // The grid-wide end of a single-pass fold: each thread's state folds across its warp (shuffle)
    // and block, every block writes one partial, and the last block to take a ticket folds the
    // partials in block order and writes the value to `destination`. Every thread of the block
    // calls it.
    template <typename T>
    // `status`, when given, is the launch's error word: if a block gave up on its copies (its
    // partial then covers only the tiles before it stopped), the result is a quiet NaN instead of a
    // partial fold, so a caller that never reads the word still cannot take the value for a result.
    __device__ __forceinline__ void finish_fold(Fold fold, unsigned op, ReduceState *state, double *destination,
                                                const int *status = nullptr) {
        __shared__ double block_total[32];
        __shared__ unsigned block_magnitude[32];
        __shared__ bool last_block;
        const unsigned threads = blockDim.x, t = threadIdx.x;
        // warp
#pragma unroll
        for (int offset = 16; offset > 0; offset >>= 1) {
            const double other = __shfl_xor_sync(0xffffffffu, fold.total, offset);
            fold.total = combine(op, fold.total, other);
            fold.magnitude = max(fold.magnitude, __shfl_xor_sync(0xffffffffu, fold.magnitude, offset));
        }
        const unsigned warp = t / 32, warps = (threads + 31) / 32;
        if ((t & 31) == 0) {
            block_total[warp] = fold.total;
            block_magnitude[warp] = fold.magnitude;
        }
        __syncthreads();
        if (t == 0) {
            double total = block_total[0];
            unsigned magnitude = block_magnitude[0];
            for (unsigned i = 1; i < warps; ++i) {
                total = combine(op, total, block_total[i]);
                magnitude = max(magnitude, block_magnitude[i]);
            }
            state->partial[blockIdx.x] = total;
            state->poisoned[blockIdx.x] = magnitude > nan_floor<T>() ? 1 : 0;
            __threadfence();
            const unsigned ticket = atomicAdd(&state->ticket, 1u);
            last_block = ticket == gridDim.x - 1;
        }
        __syncthreads();
        if (last_block && t < 32) {
            __threadfence();
            // Fold the block partials in block order: lane l takes blocks l, l+32, ... then the
            // lanes combine in a fixed tree, so the result depends only on the launch shape.
            double total = op == 0 ? 0.0 : (op == 1 ? __longlong_as_double(0x7ff0000000000000ll)
                                                    : __longlong_as_double((long long)0xfff0000000000000ull));
            int poisoned = 0;
            for (unsigned b = t; b < gridDim.x; b += 32) {
                total = combine(op, total, __ldcg(&state->partial[b]));
                poisoned |= __ldcg(&state->poisoned[b]);
            }
#pragma unroll
            for (int offset = 16; offset > 0; offset >>= 1) {
                total = combine(op, total, __shfl_xor_sync(0xffffffffu, total, offset));
                poisoned |= __shfl_xor_sync(0xffffffffu, poisoned, offset);
            }
            if (t == 0) {
                // every block's atomicOr on the word came before its ticket (fenced), so it is seen here
                const bool gave_up = status != nullptr && (__ldcg(status) & kStatusTimeout) != 0;
                *destination = poisoned || gave_up ? __longlong_as_double(0x7ff8000000000000ll) : total;
                state->ticket = 0;
            }
        }
    }

    // ---- the kernel -----------------------------------------------------------------------------------
    template <typename T, class Program, int MODE>
    __global__ void __launch_bounds__(256) chunk_stream(const __grid_constant__ Launch<T> L) {
        extern __shared__ __align__(128) unsigned char shared[];
        __shared__ unsigned long long bars[kMaxStages];
        constexpr int N = Lanes<T>::count;

        const unsigned threads = blockDim.x, t = threadIdx.x;
        const unsigned tile = N * threads;
        const unsigned A = arguments_of<Program>(L);
        const unsigned S = L.stages;
        T *ring = reinterpret_cast<T *>(shared);
        T *slots = ring + static_cast<unsigned long long>(S) * A * tile;
        const unsigned long long full = L.count / tile;
        const unsigned long long grid = gridDim.x;
        const unsigned op = MODE == kDot ? 0u : L.fold;

        Fold fold{op == 0 ? 0.0 : (op == 1 ? __longlong_as_double(0x7ff0000000000000ll)
                                           : __longlong_as_double((long long)0xfff0000000000000ull)),
                  0u};

        Work<T, Program> w(L, slots, threads, t);

        // Full tiles through the TMA ring.
        if (S > 0) {
            if (t == 0) {
                for (unsigned s = 0; s < S; ++s) barrier_init(&bars[s], 1);
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            __syncthreads();
            const unsigned bytes = tile * sizeof(T);
            auto issue = [&](unsigned s, unsigned long long k) {
                barrier_expect(&bars[s], A * bytes);
                T *dst = ring + static_cast<unsigned long long>(s) * A * tile;
                for (unsigned a = 0; a < A; ++a) bulk_load(dst + a * tile, L.inputs[a] + k * tile, bytes, &bars[s]);
            };
            if (t == 0) {
                for (unsigned s = 0; s < S; ++s) {
                    const unsigned long long k = blockIdx.x + s * grid;
                    if (k < full) issue(s, k);
                }
            }
            unsigned long long n = 0;
            unsigned s = 0, parity = 0;  // ring slot and phase of tile n, advanced without a division
            bool failed = false;
            for (unsigned long long k = blockIdx.x; k < full; k += grid, ++n) {
                const bool ok = barrier_wait(&bars[s], parity);
                w.at(k * tile, tile, ring + static_cast<unsigned long long>(s) * A * tile);
                T value[N], second[N];
                run_tile<T, Program, MODE>(w, value, second);
                if constexpr (MODE != kEvaluate) fold_tile<T, MODE>(fold, op, value, second, w, true);
                // One barrier per tile: the whole block is done with slot s, so it may be refilled,
                // and a wait that gave up anywhere in the block (its thread computed on whatever
                // the slot held, inside the tile's bounds) ends the loop for all threads.
                if (__syncthreads_or(!ok)) {
                    failed = true;
                    break;
                }
                if (t == 0) {
                    const unsigned long long next = k + S * grid;
                    if (next < full) issue(s, next);
                }
                if (++s == S) {
                    s = 0;
                    parity ^= 1u;
                }
            }
            if (failed) {
                if (t == 0) atomicOr(L.status, kStatusTimeout);
                // Let copies already in flight land before the block's shared memory goes away.
                for (unsigned long long m = n; m < n + S; ++m) {
                    const unsigned long long k = blockIdx.x + m * grid;
                    if (k >= full) break;
                    barrier_wait(&bars[m % S], static_cast<unsigned>((m / S) & 1));
                }
            }
        } else {
            // Direct reads: inputs that are not 16-byte aligned, or too wide to stage.
            for (unsigned long long k = blockIdx.x; k < full; k += grid) {
                w.at(k * tile, tile, nullptr);
                T value[N], second[N];
                run_tile<T, Program, MODE>(w, value, second);
                if constexpr (MODE != kEvaluate) fold_tile<T, MODE>(fold, op, value, second, w, true);
            }
        }

        // The ragged last tile, read directly by the block whose turn it is.
        const unsigned long long rest = L.count - full * tile;
        if (rest > 0 && blockIdx.x == full % grid) {
            w.at(full * tile, static_cast<unsigned>(rest), nullptr);
            T value[N], second[N];
            run_tile<T, Program, MODE>(w, value, second);
            if constexpr (MODE != kEvaluate) fold_tile<T, MODE>(fold, op, value, second, w, false);
        }

        if constexpr (MODE != kEvaluate) finish_fold<T>(fold, op, L.state, L.destination, L.status);
    }

} // namespace sci_cuda
