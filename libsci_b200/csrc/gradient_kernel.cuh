// gradient_kernel.cuh -- sci::gradient on sm_100a: reverse-mode derivatives of a summed chunk.
//
// L = seed * sum_i f(x_i), f the chunk's reduced value over the elements of its arguments. The
// chunk arrives in value form: node s is the s-th instruction's result, and an operand names an
// argument (kInput | a), a literal (kLiteral | l) or an earlier node (kTemporary | s) -- the
// temporaries' slot reuse is resolved on the host, so the reverse walk can name every forward value.
// One kernel source, three forms:
//  - kGradRecompute: per element, run the nodes forward (their values stay in registers), fold the
//    value into the sum, then walk the nodes in reverse accumulating adjoints in double and write
//    dL/d(argument). It reads the arguments once and writes the gradients once.
//  - kGradRecord + kGradReplay: the temporary-storing comparison form. The first pass runs forward,
//    folds the sum and stores every node's value on a tape in device memory; the second reads the
//    tape and the arguments back for the reverse walk.
// Forward values are bit-identical to the chunk interpreter's (the same apply<code> per node, with the
// loop-tail forms of minimum and maximum from the same element on), so the derivatives are those of
// the function the reference computes. Partial derivatives are evaluated in double from the node's
// operands and value (d e^x = e^x uses the value; d sin x = cos x uses this library's own cos).
// Conventions where calculus leaves a choice: d|x| at 0 is 0; minimum / maximum pass the adjoint to
// the operand their forward form returned (to both when that form returned l + r for a NaN); a
// node whose adjoint is exactly zero passes nothing back, so 0 * inf never manufactures a NaN.
#pragma once

#include "chunk_kernel.cuh"

namespace sci_cuda {

    // Specialisation modes of the gradient forms (distinct from the chunk kernel's kEvaluate/...).
    enum GradientMode : int { kGradRecompute = 8, kGradRecord = 9, kGradReplay = 10 };

    template <typename T> struct GradientLaunch {
        Step steps[kCapacity];  // value form (targets unused)
        unsigned length;        // nodes
        unsigned result;        // operand id of the summed value
        unsigned arguments;
        unsigned tailed;        // minimum / maximum present: loop-tail forms matter
        unsigned vector;        // inputs, gradients and tape rows are 16-byte aligned and count is a
                                // multiple of the vector width
        T constants[kCapacity];
        const T *inputs[kCapacity];
        T *gradients[kCapacity];  // per argument; null: not wanted
        T *tape;                  // tape[node * count + i]
        double seed;
        unsigned long long count;
        unsigned long long tail_start;
        ReduceState *state;
        double *destination;  // the sum, or null
    };

    // d(node)/d(operands) in double. a, b, c are the operands, v the node's value; `tail` selects the
    // loop-tail forms of minimum and maximum, as the forward pass did.
    template <int code, typename T>
    __device__ __forceinline__ void partials(T a, T b, T c, T v, bool tail, double &da, double &db, double &dc) {
        const double x = static_cast<double>(a), y = static_cast<double>(b), out = static_cast<double>(v);
        da = 0.0;
        db = 0.0;
        dc = 0.0;
        (void)c;
        if constexpr (code == kCopy) da = 1.0;
        else if constexpr (code == kNegate) da = -1.0;
        else if constexpr (code == kAbsolute) da = x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : (x == 0.0 ? 0.0 : x));
        else if constexpr (code == kRoot) da = 0.5 / out;
        else if constexpr (code == kExponential) da = out;
        else if constexpr (code == kLogarithm) da = 1.0 / x;
        else if constexpr (code == kSin) da = static_cast<double>(circular<true>(a));
        else if constexpr (code == kCos) da = -static_cast<double>(circular<false>(a));
        else if constexpr (code == kTan) da = fma(out, out, 1.0);
        else if constexpr (code == kAsin) da = 1.0 / sqrt((1.0 - x) * (1.0 + x));
        else if constexpr (code == kAcos) da = -1.0 / sqrt((1.0 - x) * (1.0 + x));
        else if constexpr (code == kAtan) da = 1.0 / fma(x, x, 1.0);
        else if constexpr (code == kCsc) da = -out * out * static_cast<double>(circular<true>(a));
        else if constexpr (code == kSec) da = out * out * static_cast<double>(circular<false>(a));
        else if constexpr (code == kCot) da = -fma(out, out, 1.0);
        else if constexpr (code == kAcsc) da = -1.0 / (fabs(x) * sqrt((x - 1.0) * (x + 1.0)));
        else if constexpr (code == kAsec) da = 1.0 / (fabs(x) * sqrt((x - 1.0) * (x + 1.0)));
        else if constexpr (code == kAcot) da = -1.0 / fma(x, x, 1.0);
        else if constexpr (code == kSinh) da = cosh(x);
        else if constexpr (code == kCosh) da = sinh(x);
        else if constexpr (code == kTanh) {
            const double h = cosh(x);
            da = 1.0 / (h * h);
        } else if constexpr (code == kAsinh) da = 1.0 / sqrt(fma(x, x, 1.0));
        else if constexpr (code == kAcosh) da = 1.0 / sqrt((x - 1.0) * (x + 1.0));
        else if constexpr (code == kAtanh) da = 1.0 / ((1.0 - x) * (1.0 + x));
        else if constexpr (code == kCsch) {
            const double s = sinh(x);
            da = -cosh(x) / (s * s);
        } else if constexpr (code == kSech) {
            const double h = cosh(x);
            da = -sinh(x) / (h * h);
        } else if constexpr (code == kCoth) {
            const double s = sinh(x);
            da = -1.0 / (s * s);
        } else if constexpr (code == kAcsch) da = -1.0 / (fabs(x) * sqrt(fma(x, x, 1.0)));
        else if constexpr (code == kAsech) da = -1.0 / (fabs(x) * sqrt((1.0 - x) * (1.0 + x)));
        else if constexpr (code == kAcoth) da = 1.0 / ((1.0 - x) * (1.0 + x));
        else if constexpr (code == kAdd) {
            da = 1.0;
            db = 1.0;
        } else if constexpr (code == kSubtract) {
            da = 1.0;
            db = -1.0;
        } else if constexpr (code == kMultiply) {
            da = y;
            db = x;
        } else if constexpr (code == kDivide) {
            da = 1.0 / y;
            db = -(x / y) / y;
        } else if constexpr (code == kMinimum || code == kMaximum) {
            constexpr bool low = code == kMinimum;
            if (tail) {  // smin / smax: NaN -> l + r, else the strictly better right operand
                if (is_nan(a) || is_nan(b)) {
                    da = 1.0;
                    db = 1.0;
                } else if (low ? (b < a) : (b > a)) {
                    db = 1.0;
                } else {
                    da = 1.0;
                }
            } else {  // vmin / vmax: a NaN left operand, else the strictly better left operand
                if (is_nan(a) || (low ? (a < b) : (a > b))) da = 1.0;
                else db = 1.0;
            }
        } else {  // kFuse: a * b + c
            da = y;
            db = x;
            dc = 1.0;
        }
    }

    template <typename T>
    __device__ __forceinline__ void partials_dynamic(int code, T a, T b, T c, T v, bool tail, double &da, double &db,
                                                     double &dc) {
        switch (code) {
#define SCI_CASE(N) \
    case N: partials<N>(a, b, c, v, tail, da, db, dc); break;
            SCI_CASE(0) SCI_CASE(1) SCI_CASE(2) SCI_CASE(3) SCI_CASE(4) SCI_CASE(5) SCI_CASE(6) SCI_CASE(7)
            SCI_CASE(8) SCI_CASE(9) SCI_CASE(10) SCI_CASE(11) SCI_CASE(12) SCI_CASE(13) SCI_CASE(14) SCI_CASE(15)
            SCI_CASE(16) SCI_CASE(17) SCI_CASE(18) SCI_CASE(19) SCI_CASE(20) SCI_CASE(21) SCI_CASE(22) SCI_CASE(23)
            SCI_CASE(24) SCI_CASE(25) SCI_CASE(26) SCI_CASE(27) SCI_CASE(28) SCI_CASE(29) SCI_CASE(30) SCI_CASE(31)
            SCI_CASE(32) SCI_CASE(33) SCI_CASE(34) SCI_CASE(35) SCI_CASE(36)
#undef SCI_CASE
        default:
            da = db = dc = 0.0;
        }
    }

    // An adjoint contribution: nothing when the adjoint is exactly zero.
    __device__ __forceinline__ double pass(double adjoint, double partial) { return adjoint == 0.0 ? 0.0 : adjoint * partial; }

    // Elements per thread per step: one 16-byte vector for baked programs of up to 16 nodes (their
    // values and adjoints stay in registers), else one.
    template <typename T, class Program> struct GradientWidth {
        static constexpr int value = 1;
    };
    template <typename T, class C> struct GradientWidth<T, Baked<C>> {
        static constexpr int value = C::length <= 16 ? static_cast<int>(16 / sizeof(T)) : 1;
    };

    template <typename T, class Program, int FORM>
    __global__ void __launch_bounds__(256) gradient_stream(const __grid_constant__ GradientLaunch<T> L) {
        constexpr int E = GradientWidth<T, Program>::value;
        constexpr bool forward = FORM != kGradReplay, backward = FORM != kGradRecord;
        const unsigned long long count = L.count;
        const unsigned long long groups = (count + E - 1) / E;
        const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
        Fold fold{0.0, 0u};

        for (unsigned long long g = 1ull * blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += stride) {
            const unsigned long long i0 = g * E;
            const int live = count - i0 < static_cast<unsigned long long>(E) ? static_cast<int>(count - i0) : E;
            const bool whole = live == E && L.vector != 0 && E > 1;
            bool tail[E];
#pragma unroll
            for (int e = 0; e < E; ++e) tail[e] = L.tailed != 0 && i0 + e >= L.tail_start;

            if constexpr (!Program::baked) {
                // The interpreter: one element, values and adjoints in per-thread arrays.
                const unsigned long long i = i0;
                T value[kCapacity];
                auto operand = [&](unsigned id) -> T {
                    const unsigned kind = id & kTypes, slot = id & 63;
                    if (kind == kInput) return L.inputs[slot][i];
                    if (kind == kLiteral) return L.constants[slot];
                    if (id == kNone) return T(0);
                    return value[slot];
                };
                for (unsigned s = 0; s < L.length; ++s) {
                    const Step st = L.steps[s];
                    if constexpr (forward) {
                        value[s] = apply_one<T>(st.code, operand(st.a), operand(st.b), operand(st.c), tail[0]);
                        if constexpr (FORM == kGradRecord) L.tape[s * count + i] = value[s];
                    } else {
                        value[s] = L.tape[s * count + i];
                    }
                }
                if constexpr (forward) fold.total += static_cast<double>(operand(L.result));
                if constexpr (backward) {
                    double adjoint[kCapacity], argument[kCapacity];
                    for (unsigned s = 0; s < L.length; ++s) adjoint[s] = 0.0;
                    for (unsigned a = 0; a < L.arguments; ++a) argument[a] = 0.0;
                    auto give = [&](unsigned id, double d) {
                        const unsigned kind = id & kTypes, slot = id & 63;
                        if (kind == kInput) argument[slot] += d;
                        else if (kind == kTemporary) adjoint[slot] += d;
                    };
                    give(L.result, L.seed);
                    for (int s = static_cast<int>(L.length) - 1; s >= 0; --s) {
                        const Step st = L.steps[s];
                        const double adj = adjoint[s];
                        double da, db, dc;
                        partials_dynamic<T>(st.code, operand(st.a), operand(st.b), operand(st.c), value[s], tail[0], da, db,
                                            dc);
                        give(st.a, pass(adj, da));
                        if (st.code >= kAdd) give(st.b, pass(adj, db));
                        if (st.code == kFuse) give(st.c, pass(adj, dc));
                    }
                    for (unsigned a = 0; a < L.arguments; ++a)
                        if (L.gradients[a]) L.gradients[a][i] = static_cast<T>(argument[a]);
                }
            } else {
                using C = typename Program::chunk;
                constexpr int NODES = C::length > 0 ? C::length : 1;
                constexpr int A = C::arguments > 0 ? C::arguments : 1;
                T in[A][E];
                T value[NODES][E];
                // arguments: every one the chunk names (the forward pass and the partials read them)
#pragma unroll
                for (int a = 0; a < C::arguments; ++a) {
                    const T *src = L.inputs[a] + i0;
                    if (whole) {
                        if constexpr (E > 1) load16(src, in[a]);
                    } else {
#pragma unroll
                        for (int e = 0; e < E; ++e) in[a][e] = e < live ? src[e] : T(0);
                    }
                }
                auto operand = [&](auto id_c, int e) -> T {
                    constexpr int id = decltype(id_c)::value;
                    if constexpr ((id & kTypes) == kInput) return in[id & 63][e];
                    else if constexpr ((id & kTypes) == kLiteral) return L.constants[id & 63];
                    else if constexpr (id == kNone) return T(0);
                    else return value[id & 63][e];
                };
                if constexpr (forward) {
                    static_for<C::length>([&](auto s_c) {
                        constexpr int s = decltype(s_c)::value;
                        constexpr Step st = C::steps[s];
                        if constexpr (has_fast<st.code, T>()) {
                            // the fast form on every lane, the full form again for all lanes when
                            // any lane falls outside it (same values either way)
                            bool rare = false;
#pragma unroll
                            for (int e = 0; e < E; ++e) value[s][e] = apply_fast<st.code>(operand(Int<st.a>{}, e), rare);
                            if (rare) {
#pragma unroll
                                for (int e = 0; e < E; ++e)
                                    value[s][e] = apply<st.code>(operand(Int<st.a>{}, e), operand(Int<st.b>{}, e),
                                                                 operand(Int<st.c>{}, e), tail[e]);
                            }
                        } else {
#pragma unroll
                            for (int e = 0; e < E; ++e)
                                value[s][e] = apply<st.code>(operand(Int<st.a>{}, e), operand(Int<st.b>{}, e),
                                                             operand(Int<st.c>{}, e), tail[e]);
                        }
                        if constexpr (FORM == kGradRecord) {
                            T *row = L.tape + s * count + i0;
                            if (whole) {
                                if constexpr (E > 1) store16(row, value[s]);
                            } else {
#pragma unroll
                                for (int e = 0; e < E; ++e)
                                    if (e < live) row[e] = value[s][e];
                            }
                        }
                    });
#pragma unroll
                    for (int e = 0; e < E; ++e)
                        if (e < live) fold.total += static_cast<double>(operand(Int<C::result>{}, e));
                } else {
                    static_for<C::length>([&](auto s_c) {
                        constexpr int s = decltype(s_c)::value;
                        const T *row = L.tape + s * count + i0;
                        if (whole) {
                            if constexpr (E > 1) load16(row, value[s]);
                        } else {
#pragma unroll
                            for (int e = 0; e < E; ++e) value[s][e] = e < live ? row[e] : T(0);
                        }
                    });
                }
                if constexpr (backward) {
                    double adjoint[NODES][E], argument[A][E];
#pragma unroll
                    for (int s = 0; s < NODES; ++s)
#pragma unroll
                        for (int e = 0; e < E; ++e) adjoint[s][e] = 0.0;
#pragma unroll
                    for (int a = 0; a < A; ++a)
#pragma unroll
                        for (int e = 0; e < E; ++e) argument[a][e] = 0.0;
                    auto give = [&](auto id_c, int e, double d) {
                        constexpr int id = decltype(id_c)::value;
                        if constexpr ((id & kTypes) == kInput) argument[id & 63][e] += d;
                        else if constexpr ((id & kTypes) == kTemporary && id != kNone) adjoint[id & 63][e] += d;
                    };
#pragma unroll
                    for (int e = 0; e < E; ++e) give(Int<C::result>{}, e, L.seed);
                    static_for<C::length>([&](auto k_c) {
                        constexpr int s = C::length - 1 - decltype(k_c)::value;
                        constexpr Step st = C::steps[s];
#pragma unroll
                        for (int e = 0; e < E; ++e) {
                            double da, db, dc;
                            partials<st.code>(operand(Int<st.a>{}, e), operand(Int<st.b>{}, e), operand(Int<st.c>{}, e),
                                              value[s][e], tail[e], da, db, dc);
                            const double adj = adjoint[s][e];
                            give(Int<st.a>{}, e, pass(adj, da));
                            if constexpr (st.code >= kAdd) give(Int<st.b>{}, e, pass(adj, db));
                            if constexpr (st.code == kFuse) give(Int<st.c>{}, e, pass(adj, dc));
                        }
                    });
#pragma unroll
                    for (int a = 0; a < C::arguments; ++a) {
                        T *dst = L.gradients[a];
                        if (dst == nullptr) continue;
                        T out[E];
#pragma unroll
                        for (int e = 0; e < E; ++e) out[e] = static_cast<T>(argument[a][e]);
                        if (whole) {
                            if constexpr (E > 1) store16(dst + i0, out);
                        } else {
#pragma unroll
                            for (int e = 0; e < E; ++e)
                                if (e < live) dst[i0 + e] = out[e];
                        }
                    }
                }
            }
        }
        if constexpr (forward) {
            if (L.destination != nullptr) finish_fold<T>(fold, 0u, L.state, L.destination);
        }
    }

} // namespace sci_cuda
