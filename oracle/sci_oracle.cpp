// sci_oracle.cpp -- CPU restatement of libsci's chunk arithmetic, reductions and LU.
//
// TEST INFRASTRUCTURE ONLY. The tests, __graft_entry__.smoke() and the CPU leg of bench.py load
// this library as the checker for the CUDA backend; the backend never links, loads or calls it.
//
// What it restates (all paths are inside the libsci reference tree):
//  - the per-element semantics of every chunk code as the AVX-512 kernel table computes them
//    (src/core/drivers/processor/kernels/avx512.cpp:17-153 through
//    include/core/drivers/processor/kernels/generic/operation.hpp:21-111), including the one-lane
//    Scalar pack used for loop tails (generic/scalar.hpp:16-205, generic/elementwise.hpp:127-196);
//  - the vector exp / log / sin / cos (generic/exponential.hpp:24-61, logarithm.hpp:90-126,
//    trigonometry.hpp:162-207) with their coefficients (polynomial.hpp:17-61) and constants
//    (constants.hpp:16-120), operation for operation, so results match the reference bit for bit;
//  - the nine functions the reference hands to the C library per lane (library.hpp:22-35), by
//    calling the same C library (glibc) functions;
//  - reductions folded in double with numpy NaN rules (accumulator.hpp:17-48,
//    dispatch.cpp:106-165), as the FP64 oracle the GPU reductions are held to;
//  - linear::factor / substitute (include/linear/decompose.hpp:29-72, solve.hpp:25-52);
//  - the element values of the creation functions full / linspace / range / eye / grid
//    (include/operations/creation.hpp:34-168);
//  - integer-element expressions, element by element: array::calculate<code, element>
//    (include/array/calculate.hpp:17-93) as assign() and reduce() run it for non-native element
//    types (include/array/expression.hpp:178-184,203-220), with the cases C++ leaves undefined
//    (signed overflow, a zero divisor, MIN / -1, a real result that is NaN or out of range) given
//    the definitions the CUDA backend documents: wrap, 0, MIN, 0 / saturate.
// Parity is pinned against the reference itself: tests compare this file's outputs with
// oracle/_ref/libsci_ref.so (the reference's own CPU path) and with tests/golden fixtures.
//
// Built with -ffp-contract=off: every multiply and add rounds on its own, and only the explicit
// fma() calls fuse, as in the reference kernels.
#include "../include/sci_cuda.h"

#include <algorithm>
#include <bit>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

    template <typename T> struct Bits;
    template <> struct Bits<float> { using type = uint32_t; };
    template <> struct Bits<double> { using type = uint64_t; };
    template <typename T> using bits_t = typename Bits<T>::type;

    template <typename T> bits_t<T> raw(T value) { return std::bit_cast<bits_t<T>>(value); }
    template <typename T> T cast(bits_t<T> value) { return std::bit_cast<T>(value); }

    inline float fused(float a, float b, float c) { return std::fmaf(a, b, c); }
    inline double fused(double a, double b, double c) { return std::fma(a, b, c); }

    // Constants of the vector functions (constants.hpp:16-120).
    template <typename T> struct Limits;
    template <> struct Limits<float> {
        static constexpr int mantissa = 23, width = 32;
        static constexpr uint32_t fraction = 0x007fffffu, one = 0x3f800000u;
        static constexpr float round = 12582912.0f, magnitude = 8388608.0f, exponent = 8388735.0f;
        static constexpr float binary = 1.44269504088896340736f;
        static constexpr float natural = 355.0f / 512.0f, remainder = -2.12194440e-4f;
        static constexpr float lower = -104.0f, upper = 89.0f, normal = 126.0f;
        static constexpr float tiny = 1.17549435e-38f, lift = 33554432.0f, shift = 25.0f;
        static constexpr float root = 1.41421356237309504880f;
        static constexpr float quadrant = 0.636619772367581343f;
        static constexpr float quarter[4] = {1.5703125f, 4.837512969970703125e-4f, 7.549790126404332e-08f,
                                             -1.7151245100058819e-15f};
        static constexpr float reach = 1048576.0f;
        static constexpr int exp_degree = 7, log_degree = 4, sin_degree = 5, cos_degree = 6;
    };
    template <> struct Limits<double> {
        static constexpr int mantissa = 52, width = 64;
        static constexpr uint64_t fraction = 0x000fffffffffffffull, one = 0x3ff0000000000000ull;
        static constexpr double round = 6755399441055744.0, magnitude = 4503599627370496.0,
                                exponent = 4503599627371519.0;
        static constexpr double binary = 1.44269504088896340736;
        static constexpr double natural =
                std::bit_cast<double>(std::bit_cast<uint64_t>(0.693147180559945309417232121458176568) &
                                      0xFFFFFFFFFFE00000ULL);
        static constexpr double remainder = 1.90821492927058770002e-10;
        static constexpr double lower = -746.0, upper = 710.0, normal = 1022.0;
        static constexpr double tiny = 2.2250738585072014e-308, lift = 18014398509481984.0, shift = 54.0;
        static constexpr double root = 1.41421356237309504880;
        static constexpr double quadrant = 6.36619772367581382433e-01;
        static constexpr double quarter[4] = {1.57079632673412561417e+00, 6.07710050630396597660e-11,
                                              2.02226624871116645580e-21, 8.47842766036889956997e-32};
        static constexpr double reach = 1048576.0;
        static constexpr int exp_degree = 13, log_degree = 10, sin_degree = 9, cos_degree = 10;
    };

    // Polynomial coefficients, computed in double and rounded to T (polynomial.hpp:17-51).
    template <typename T> struct Coefficients {
        static constexpr int E = Limits<T>::exp_degree + 1, L = Limits<T>::log_degree,
                             S = Limits<T>::sin_degree + 1, C = Limits<T>::cos_degree + 1;
        T exp[E], log[L], sin[S], cos[C];
        Coefficients() {
            double factor = 1.0;
            for (int k = 0; k < E; ++k) {
                if (k > 0) factor /= static_cast<double>(k);
                exp[k] = static_cast<T>(factor);
            }
            for (int k = 0; k < L; ++k) log[k] = static_cast<T>(2.0 / static_cast<double>(2 * k + 3));
            auto alternating = [](T *out, int count, int offset) {
                for (int k = 0; k < count; ++k) {
                    double f = 1.0;
                    for (int step = 2; step <= 2 * k + offset; ++step) f *= static_cast<double>(step);
                    out[k] = static_cast<T>((k % 2 == 0 ? 1.0 : -1.0) / f);
                }
            };
            alternating(sin, S, 1);
            alternating(cos, C, 0);
        }
        // sum c[k] x^(k - from), Horner from the top (polynomial.hpp:271-277).
        static T horner(const T *c, int count, int from, T x) {
            T result = c[count - 1];
            for (int k = count - 1; k-- > from;) result = fused(result, x, c[k]);
            return result;
        }
    };

    template <typename T> const Coefficients<T> &coefficients() {
        static const Coefficients<T> table;
        return table;
    }

    // Elementwise minimum / maximum. The vector body is the AVX-512 form
    // blend(unordered(l), min(l, r), l) (avx512.cpp:43-49): MINPS returns its second operand
    // unless l < r. Loop tails take the Scalar form (scalar.hpp:115-127).
    template <typename T> T vector_minimum(T l, T r) { return std::isnan(l) ? l : (l < r ? l : r); }
    template <typename T> T vector_maximum(T l, T r) { return std::isnan(l) ? l : (l > r ? l : r); }
    template <typename T> T scalar_minimum(T l, T r) {
        if (std::isnan(l) || std::isnan(r)) return l + r;
        return r < l ? r : l;
    }
    template <typename T> T scalar_maximum(T l, T r) {
        if (std::isnan(l) || std::isnan(r)) return l + r;
        return r > l ? r : l;
    }

    // e^x (exponential.hpp:24-61). The reference splits the final scale in two when any lane of
    // the pack has |k| > normal; for lanes with |k| <= normal both forms round the same exact
    // product once, so deciding per element gives the pack's bits.
    template <typename T> T exponential(T x) {
        using L = Limits<T>;
        const T clamped = vector_maximum(vector_minimum(x, L::upper), L::lower);
        const T k = fused(clamped, L::binary, L::round) - L::round;
        const T negative = -k;
        T reduced = fused(negative, L::natural, clamped);
        reduced = fused(negative, L::remainder, reduced);
        const auto &c = coefficients<T>();
        const T significand = fused(reduced, Coefficients<T>::horner(c.exp, Coefficients<T>::E, 1, reduced), T(1));
        auto scale = [](T e) { return cast<T>(raw<T>(e + L::exponent) << L::mantissa); };
        if (!(std::fabs(k) > L::normal)) return significand * scale(k);
        const T half = fused(k, T(0.5), L::round) - L::round;
        const T rest = k - half;
        return (significand * scale(half)) * scale(rest);
    }

    // ln x (logarithm.hpp:90-126).
    template <typename T> T logarithm(T x) {
        using L = Limits<T>;
        using U = bits_t<T>;
        const bool small = x < L::tiny;
        const T scaled = small ? x * L::lift : x;
        const U pattern = raw<T>(scaled);
        T exponent = cast<T>((pattern >> L::mantissa) | raw<T>(L::magnitude)) - L::exponent;
        T mantissa = cast<T>((pattern & static_cast<U>(L::fraction)) | static_cast<U>(L::one));
        const bool large = mantissa > L::root;
        mantissa = large ? mantissa * T(0.5) : mantissa;
        exponent = large ? exponent + T(1) : exponent;
        exponent = small ? exponent - L::shift : exponent;
        const T fraction = mantissa - T(1);
        const T ratio = fraction / (fraction + T(2));
        const T square = ratio * ratio;
        const auto &c = coefficients<T>();
        const T tail = square * Coefficients<T>::horner(c.log, Coefficients<T>::L, 0, square);
        const T half = (fraction * fraction) * T(0.5);
        const T inner = fused(ratio, half + tail, exponent * L::remainder);
        T result = exponent * L::natural - ((half - inner) - fraction);
        const T infinity = std::numeric_limits<T>::infinity();
        if (x == infinity) result = x;
        if (x == T(0)) result = -infinity;
        if (x < T(0)) result = std::numeric_limits<T>::quiet_NaN();
        if (std::isnan(x)) result = x;
        return result;
    }

    // sin (phase false) and cos (phase true) (trigonometry.hpp:162-207).
    template <typename T, bool phase> T circular(T x) {
        using L = Limits<T>;
        using U = bits_t<T>;
        const T shifted = fused(x, L::quadrant, L::round);
        const T quarters = shifted - L::round;
        const T negative = -quarters;
        T reduced = fused(negative, L::quarter[0], x);
        reduced = fused(negative, L::quarter[1], reduced);
        reduced = fused(negative, L::quarter[2], reduced);
        reduced = fused(negative, L::quarter[3], reduced);
        const T square = reduced * reduced;
        const auto &c = coefficients<T>();
        const T sine = fused(reduced * square, Coefficients<T>::horner(c.sin, Coefficients<T>::S, 1, square), reduced);
        const T cosine = fused(square, Coefficients<T>::horner(c.cos, Coefficients<T>::C, 1, square), T(1));
        U quadrant = raw<T>(shifted);
        if (phase) quadrant ^= quadrant << 1;
        const U flip = (quadrant & U(2)) << (L::width - 2);
        const bool swap = (raw<T>(shifted) & U(1)) != 0;
        T result = phase ? (swap ? sine : cosine) : (swap ? cosine : sine);
        result = cast<T>(raw<T>(result) ^ flip);
        if (!(x <= L::reach && x >= -L::reach)) {
            if constexpr (sizeof(T) == 4) {
                result = phase ? ::cosf(x) : ::sinf(x);
            } else {
                result = phase ? ::cos(x) : ::sin(x);
            }
        }
        return result;
    }

    template <typename T> T library(int code, T x) {
        if constexpr (sizeof(T) == 4) {
            switch (code) {
            case SCI_CODE_ASIN: return ::asinf(x);
            case SCI_CODE_ACOS: return ::acosf(x);
            case SCI_CODE_ATAN: return ::atanf(x);
            case SCI_CODE_SINH: return ::sinhf(x);
            case SCI_CODE_COSH: return ::coshf(x);
            case SCI_CODE_TANH: return ::tanhf(x);
            case SCI_CODE_ASINH: return ::asinhf(x);
            case SCI_CODE_ACOSH: return ::acoshf(x);
            default: return ::atanhf(x);
            }
        } else {
            switch (code) {
            case SCI_CODE_ASIN: return ::asin(x);
            case SCI_CODE_ACOS: return ::acos(x);
            case SCI_CODE_ATAN: return ::atan(x);
            case SCI_CODE_SINH: return ::sinh(x);
            case SCI_CODE_COSH: return ::cosh(x);
            case SCI_CODE_TANH: return ::tanh(x);
            case SCI_CODE_ASINH: return ::asinh(x);
            case SCI_CODE_ACOSH: return ::acosh(x);
            default: return ::atanh(x);
            }
        }
    }

    // One code applied to one element (operation.hpp:25-110). `tail` selects the Scalar pack's
    // minimum / maximum, which loop tails use (elementwise.hpp:136-138,163-165).
    template <typename T> T apply(int code, T a, T b, T c, bool tail) {
        using U = bits_t<T>;
        const U sign = U(1) << (sizeof(T) * 8 - 1);
        const T one = T(1);
        switch (code) {
        case SCI_CODE_COPY: return a;
        case SCI_CODE_NEGATE: return cast<T>(raw<T>(a) ^ sign);
        case SCI_CODE_ABSOLUTE: return cast<T>(raw<T>(a) & ~sign);
        case SCI_CODE_ROOT: return std::sqrt(a);
        case SCI_CODE_EXPONENTIAL: return exponential(a);
        case SCI_CODE_LOGARITHM: return logarithm(a);
        case SCI_CODE_SIN: return circular<T, false>(a);
        case SCI_CODE_COS: return circular<T, true>(a);
        case SCI_CODE_TAN: return circular<T, false>(a) / circular<T, true>(a);
        case SCI_CODE_ASIN:
        case SCI_CODE_ACOS:
        case SCI_CODE_ATAN:
        case SCI_CODE_SINH:
        case SCI_CODE_COSH:
        case SCI_CODE_TANH:
        case SCI_CODE_ASINH:
        case SCI_CODE_ACOSH:
        case SCI_CODE_ATANH: return library(code, a);
        case SCI_CODE_CSC: return one / circular<T, false>(a);
        case SCI_CODE_SEC: return one / circular<T, true>(a);
        case SCI_CODE_COT: return one / (circular<T, false>(a) / circular<T, true>(a));
        case SCI_CODE_ACSC: return library(SCI_CODE_ASIN, one / a);
        case SCI_CODE_ASEC: return library(SCI_CODE_ACOS, one / a);
        case SCI_CODE_ACOT: return library(SCI_CODE_ATAN, one / a);
        case SCI_CODE_CSCH: return one / library(SCI_CODE_SINH, a);
        case SCI_CODE_SECH: return one / library(SCI_CODE_COSH, a);
        case SCI_CODE_COTH: return one / library(SCI_CODE_TANH, a);
        case SCI_CODE_ACSCH: return library(SCI_CODE_ASINH, one / a);
        case SCI_CODE_ASECH: return library(SCI_CODE_ACOSH, one / a);
        case SCI_CODE_ACOTH: return library(SCI_CODE_ATANH, one / a);
        case SCI_CODE_ADD: return a + b;
        case SCI_CODE_SUBTRACT: return a - b;
        case SCI_CODE_MULTIPLY: return a * b;
        case SCI_CODE_DIVIDE: return a / b;
        case SCI_CODE_MINIMUM: return tail ? scalar_minimum(a, b) : vector_minimum(a, b);
        case SCI_CODE_MAXIMUM: return tail ? scalar_maximum(a, b) : vector_maximum(a, b);
        case SCI_CODE_FUSE: return fused(a, b, c);
        default: return std::numeric_limits<T>::quiet_NaN();
        }
    }

    bool valid(const sci_chunk &chunk) {
        if (chunk.length > SCI_CHUNK_CAPACITY || chunk.arguments > SCI_CHUNK_CAPACITY ||
            chunk.literals > SCI_CHUNK_CAPACITY || chunk.temporaries > SCI_CHUNK_CAPACITY)
            return false;
        for (int index = 0; index < chunk.length; ++index) {
            if (chunk.instructions[index].code >= SCI_CODE_COUNT) return false;
        }
        return true;
    }

    // Evaluates the first `steps` instructions for element `index`; returns the value of `want`
    // (a value id), or of the last instruction when `want` is the output slot.
    template <typename T>
    T element(const sci_chunk &chunk, const T *constants, uint64_t index, bool tail, int steps, uint8_t want,
              T *out_slot, T *operands) {
        T temporaries[SCI_CHUNK_CAPACITY];
        T last = T(0);
        auto fetch = [&](uint8_t id) -> T {
            if (id == SCI_SLOT_NONE) return T(0);
            const int kind = id & SCI_SLOT_TYPES, slot = id & 63;
            if (kind == SCI_SLOT_INPUT) return static_cast<const T *>(chunk.inputs[slot])[index];
            if (kind == SCI_SLOT_LITERAL) return constants[slot];
            if (kind == SCI_SLOT_TEMPORARY) return temporaries[slot];
            return last;
        };
        for (int step = 0; step < steps; ++step) {
            const sci_instruction &ins = chunk.instructions[step];
            const T value = apply<T>(ins.code, fetch(ins.sources[0]), fetch(ins.sources[1]), fetch(ins.sources[2]), tail);
            last = value;
            if (ins.target == SCI_SLOT_OUTPUT) {
                if (out_slot) *out_slot = value;
            } else if ((ins.target & SCI_SLOT_TYPES) == SCI_SLOT_TEMPORARY) {
                temporaries[ins.target & 63] = value;
            }
        }
        if (operands) {
            // The contracted dot reads the skipped multiply's operands.
            const sci_instruction &ins = chunk.instructions[steps];
            operands[0] = fetch(ins.sources[0]);
            operands[1] = fetch(ins.sources[1]);
            return T(0);
        }
        return want == SCI_SLOT_OUTPUT ? last : fetch(want);
    }

    template <typename F> void parallel(uint64_t count, F &&work) {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const uint64_t parts = count < (uint64_t{1} << 16) ? 1 : std::min<uint64_t>(hw, 64);
        if (parts == 1) {
            work(uint64_t{0}, count, 0u);
            return;
        }
        std::vector<std::thread> threads;
        for (uint64_t part = 0; part < parts; ++part) {
            threads.emplace_back([&, part] { work(count * part / parts, count * (part + 1) / parts, unsigned(part)); });
        }
        for (auto &thread : threads) thread.join();
    }

    template <typename T> void constants_of(const sci_chunk &chunk, T *out) {
        for (int index = 0; index < chunk.literals; ++index) out[index] = static_cast<T>(chunk.constants[index]);
    }

    template <typename T> int execute(const sci_chunk &chunk, T *output, uint64_t count, uint64_t tail_width) {
        T constants[SCI_CHUNK_CAPACITY];
        constants_of(chunk, constants);
        const uint64_t tail_start = count - count % tail_width;
        parallel(count, [&](uint64_t first, uint64_t last, unsigned) {
            for (uint64_t index = first; index < last; ++index) {
                T value;
                element<T>(chunk, constants, index, index >= tail_start, chunk.length, SCI_SLOT_OUTPUT, &value, nullptr);
                output[index] = value;
            }
        });
        return 0;
    }

    // The FP64 fold the GPU reductions are held to: every element's chunk value (in T, exactly as
    // the executor computes it) folded in double; NaN anywhere gives NaN (accumulator.hpp:28-34);
    // empty sums are 0, empty extremes NaN (dispatch.cpp:109-111). A sum that ends in a multiply is
    // contracted: the product is never rounded to T (chunk.hpp:201-204, reductions.hpp:223-257),
    // so the oracle sums the exact double product of the two operands.
    template <typename T> double reduce(const sci_chunk &chunk, int fold, uint64_t count, uint64_t tail_width) {
        if (count == 0) return fold == SCI_FOLD_SUM ? 0.0 : std::numeric_limits<double>::quiet_NaN();
        T constants[SCI_CHUNK_CAPACITY];
        constants_of(chunk, constants);
        const bool contract = fold == SCI_FOLD_SUM && chunk.length > 0 &&
                              chunk.instructions[chunk.length - 1].code == SCI_CODE_MULTIPLY &&
                              chunk.instructions[chunk.length - 1].target == chunk.result;
        const int steps = contract ? chunk.length - 1 : chunk.length;
        const uint64_t tail_start = count - count % tail_width;
        std::vector<double> partial(64, fold == SCI_FOLD_SUM ? 0.0
                                        : fold == SCI_FOLD_MINIMUM ? std::numeric_limits<double>::infinity()
                                                                   : -std::numeric_limits<double>::infinity());
        std::vector<int> poisoned(64, 0);
        parallel(count, [&](uint64_t first, uint64_t last, unsigned part) {
            double total = partial[part];
            int nan = 0;
            for (uint64_t index = first; index < last; ++index) {
                double value;
                if (contract) {
                    T operands[2];
                    element<T>(chunk, constants, index, index >= tail_start, steps, chunk.result, nullptr, operands);
                    value = static_cast<double>(operands[0]) * static_cast<double>(operands[1]);
                } else {
                    value = static_cast<double>(
                            element<T>(chunk, constants, index, index >= tail_start, steps, chunk.result, nullptr, nullptr));
                }
                if (std::isnan(value)) {
                    nan = 1;
                    continue;
                }
                if (fold == SCI_FOLD_SUM) total += value;
                else if (fold == SCI_FOLD_MINIMUM) total = std::min(total, value);
                else total = std::max(total, value);
            }
            partial[part] = total;
            poisoned[part] = nan;
        });
        double total = fold == SCI_FOLD_SUM ? 0.0
                       : fold == SCI_FOLD_MINIMUM ? std::numeric_limits<double>::infinity()
                                                  : -std::numeric_limits<double>::infinity();
        for (int part = 0; part < 64; ++part) {
            if (poisoned[part]) return std::numeric_limits<double>::quiet_NaN();
            if (fold == SCI_FOLD_SUM) total += partial[part];
            else if (fold == SCI_FOLD_MINIMUM) total = std::min(total, partial[part]);
            else total = std::max(total, partial[part]);
        }
        return total;
    }

    // In-place LU with partial pivoting (decompose.hpp:29-72): pivot is the first row with a
    // strictly larger |a| (decompose.hpp:35-38); a zero pivot is skipped (decompose.hpp:44-45).
    template <typename T> void factor(T *a, uint64_t *rows, uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) rows[i] = i;
        for (uint64_t step = 0; step < n; ++step) {
            uint64_t pivot = step;
            for (uint64_t row = step + 1; row < n; ++row) {
                if (std::fabs(a[row * n + step]) > std::fabs(a[pivot * n + step])) pivot = row;
            }
            if (pivot != step) {
                for (uint64_t column = 0; column < n; ++column) std::swap(a[step * n + column], a[pivot * n + column]);
                std::swap(rows[step], rows[pivot]);
            }
            const T diagonal = a[step * n + step];
            if (diagonal == T(0)) continue;
            const T *top = a + step * n;
            for (uint64_t row = step + 1; row < n; ++row) {
                T *target = a + row * n;
                const T scale = target[step] /= diagonal;
                for (uint64_t column = step + 1; column < n; ++column) target[column] -= scale * top[column];
            }
        }
    }

    // Forward then back substitution on `width` right-hand sides (solve.hpp:25-52).
    template <typename T>
    void substitute(const T *lu, const uint64_t *rows, const T *right, T *x, uint64_t n, uint64_t width) {
        for (uint64_t row = 0; row < n; ++row) {
            for (uint64_t column = 0; column < width; ++column) x[row * width + column] = right[rows[row] * width + column];
            for (uint64_t inner = 0; inner < row; ++inner) {
                const T scale = lu[row * n + inner];
                for (uint64_t column = 0; column < width; ++column)
                    x[row * width + column] -= scale * x[inner * width + column];
            }
        }
        for (uint64_t row = n; row-- > 0;) {
            for (uint64_t inner = row + 1; inner < n; ++inner) {
                const T scale = lu[row * n + inner];
                for (uint64_t column = 0; column < width; ++column)
                    x[row * width + column] -= scale * x[inner * width + column];
            }
            const T diagonal = lu[row * n + row];
            for (uint64_t column = 0; column < width; ++column) x[row * width + column] /= diagonal;
        }
    }

} // namespace

// ---- creation (include/operations/creation.hpp) -----------------------------------------------
namespace {
    template <typename T> void fill_values(T *out, uint64_t count, T value) {  // creation.hpp:34-58
        for (uint64_t i = 0; i < count; ++i) out[i] = value;
    }
    template <typename T> void linspace_values(T *out, uint64_t count, T start, T stop) {  // creation.hpp:66-84
        if (count == 0) return;
        if (count == 1) {
            out[0] = start;
            return;
        }
        const double step = static_cast<double>(stop - start) / (static_cast<double>(count) - 1.0);
        for (uint64_t i = 0; i < count; ++i) out[i] = static_cast<T>(static_cast<double>(start) + static_cast<double>(i) * step);
    }
    template <typename T> uint64_t range_count(T start, T stop, T step) {  // creation.hpp:159-161
        const double span = std::ceil((static_cast<double>(stop) - static_cast<double>(start)) / static_cast<double>(step));
        return span > 0 ? static_cast<uint64_t>(span) : 0;
    }
    template <typename T> void range_values(T *out, uint64_t count, T start, T step) {  // creation.hpp:163-165
        for (uint64_t i = 0; i < count; ++i) out[i] = static_cast<T>(start + static_cast<T>(i) * step);
    }
    template <typename T> void eye_values(T *out, uint64_t rows, uint64_t columns) {  // creation.hpp:91-106
        for (uint64_t i = 0; i < rows * columns; ++i) out[i] = T(0);
        for (uint64_t i = 0; i < (rows < columns ? rows : columns); ++i) out[i * columns + i] = T(1);
    }
    // ---- integer elements (calculate.hpp:17-93, expression.hpp:178-184,203-220) ----------------
    template <typename T> using IntWord = std::conditional_t<sizeof(T) <= 4, uint32_t, uint64_t>;

    template <typename T> T int_from_real(double x) {
        constexpr T lo = std::numeric_limits<T>::min(), hi = std::numeric_limits<T>::max();
        if (std::isnan(x)) return T(0);
        if (x <= static_cast<double>(lo)) return lo;
        if (x >= static_cast<double>(hi)) return hi;
        return static_cast<T>(x);
    }

    double int_real(int code, double x) {  // calculate.hpp:25-80, in double
        switch (code) {
        case SCI_CODE_ROOT: return std::sqrt(x);
        case SCI_CODE_EXPONENTIAL: return std::exp(x);
        case SCI_CODE_LOGARITHM: return std::log(x);
        case SCI_CODE_SIN: return std::sin(x);
        case SCI_CODE_COS: return std::cos(x);
        case SCI_CODE_TAN: return std::tan(x);
        case SCI_CODE_ASIN: return std::asin(x);
        case SCI_CODE_ACOS: return std::acos(x);
        case SCI_CODE_ATAN: return std::atan(x);
        case SCI_CODE_CSC: return 1.0 / std::sin(x);
        case SCI_CODE_SEC: return 1.0 / std::cos(x);
        case SCI_CODE_COT: return 1.0 / std::tan(x);
        case SCI_CODE_ACSC: return std::asin(1.0 / x);
        case SCI_CODE_ASEC: return std::acos(1.0 / x);
        case SCI_CODE_ACOT: return std::atan(1.0 / x);
        case SCI_CODE_SINH: return std::sinh(x);
        case SCI_CODE_COSH: return std::cosh(x);
        case SCI_CODE_TANH: return std::tanh(x);
        case SCI_CODE_ASINH: return std::asinh(x);
        case SCI_CODE_ACOSH: return std::acosh(x);
        case SCI_CODE_ATANH: return std::atanh(x);
        case SCI_CODE_CSCH: return 1.0 / std::sinh(x);
        case SCI_CODE_SECH: return 1.0 / std::cosh(x);
        case SCI_CODE_COTH: return 1.0 / std::tanh(x);
        case SCI_CODE_ACSCH: return std::asinh(1.0 / x);
        case SCI_CODE_ASECH: return std::acosh(1.0 / x);
        default: return std::atanh(1.0 / x);
        }
    }

    template <typename T> T int_apply(int code, T a, T b, T c) {
        using W = IntWord<T>;
        switch (code) {
        case SCI_CODE_COPY: return a;
        case SCI_CODE_NEGATE: return T(W(0) - W(a));
        case SCI_CODE_ABSOLUTE:
            if constexpr (std::is_signed_v<T>) return a < T(0) ? T(W(0) - W(a)) : a;
            else return a;
        case SCI_CODE_ADD: return T(W(a) + W(b));
        case SCI_CODE_SUBTRACT: return T(W(a) - W(b));
        case SCI_CODE_MULTIPLY: return T(W(a) * W(b));
        case SCI_CODE_DIVIDE:
            if (b == T(0)) return T(0);
            if constexpr (std::is_signed_v<T>) {
                if (b == T(-1)) return T(W(0) - W(a));
            }
            return T(a / b);
        case SCI_CODE_MINIMUM: return b < a ? b : a;
        case SCI_CODE_MAXIMUM: return b > a ? b : a;
        case SCI_CODE_FUSE: return T(W(a) * W(b) + W(c));
        default: return int_from_real<T>(int_real(code, static_cast<double>(a)));
        }
    }

    // One element through the chunk: value ids as in instruction.hpp:12-25.
    template <typename T> T int_element(const sci_chunk &chunk, uint64_t i, T *temporaries, T &out, unsigned wanted) {
        auto value = [&](unsigned id) -> T {
            const unsigned kind = id & SCI_SLOT_TYPES, slot = id & 63;
            if (id == SCI_SLOT_NONE) return T(0);
            if (kind == SCI_SLOT_INPUT) return static_cast<const T *>(chunk.inputs[slot])[i];
            if (kind == SCI_SLOT_LITERAL) return static_cast<T>(chunk.constants[slot]);
            if (kind == SCI_SLOT_TEMPORARY) return temporaries[slot];
            return out;
        };
        for (int k = 0; k < chunk.length; ++k) {
            const sci_instruction &ins = chunk.instructions[k];
            const T r = int_apply<T>(ins.code, value(ins.sources[0]), value(ins.sources[1]), value(ins.sources[2]));
            if (ins.target == SCI_SLOT_OUTPUT) out = r;
            else temporaries[ins.target & 63] = r;
        }
        return value(wanted);
    }

    template <typename T> void int_execute(const sci_chunk &chunk, T *output, uint64_t count) {
        T temporaries[SCI_CHUNK_CAPACITY] = {};
        for (uint64_t i = 0; i < count; ++i) {
            T out{};
            output[i] = int_element<T>(chunk, i, temporaries, out, SCI_SLOT_OUTPUT);
        }
    }

    template <typename T> T int_reduce(const sci_chunk &chunk, int fold, uint64_t count) {
        if (count == 0) return T{};
        T temporaries[SCI_CHUNK_CAPACITY] = {};
        T out{};
        T result = int_element<T>(chunk, 0, temporaries, out, chunk.result);
        for (uint64_t i = 1; i < count; ++i) {
            const T v = int_element<T>(chunk, i, temporaries, out, chunk.result);
            if (fold == SCI_FOLD_SUM) result = T(IntWord<T>(result) + IntWord<T>(v));
            else if (fold == SCI_FOLD_MINIMUM) result = v < result ? v : result;
            else result = v > result ? v : result;
        }
        return result;
    }

    template <typename F> int by_int_element(uint32_t element, F &&f) {
        switch (element) {
        case SCI_ELEMENT_INT8: return f(int8_t{});
        case SCI_ELEMENT_INT16: return f(int16_t{});
        case SCI_ELEMENT_INT32: return f(int32_t{});
        case SCI_ELEMENT_INT64: return f(int64_t{});
        case SCI_ELEMENT_UINT8: return f(uint8_t{});
        case SCI_ELEMENT_UINT16: return f(uint16_t{});
        case SCI_ELEMENT_UINT32: return f(uint32_t{});
        case SCI_ELEMENT_UINT64: return f(uint64_t{});
        default: return SCI_CUDA_ERROR_INVALID;
        }
    }

    template <typename T> void grid_values(const T *x, uint64_t nx, const T *y, uint64_t ny, T *xx, T *yy) {  // :120-140
        for (uint64_t i = 0; i < ny; ++i)
            for (uint64_t j = 0; j < nx; ++j) {
                xx[i * nx + j] = x[j];
                yy[i * nx + j] = y[i];
            }
    }
} // namespace

extern "C" {

// The pack width whose loop tails take the Scalar forms: 16 floats / 8 doubles for AVX-512.
uint64_t sci_oracle_tail_width(uint32_t precision) { return precision == SCI_PRECISION_WIDE ? 8 : 16; }

int sci_oracle_execute(const sci_chunk *chunk, void *output, uint64_t count) {
    if (!chunk || !valid(*chunk)) return SCI_CUDA_ERROR_INVALID;
    if (count == 0) return 0;
    if (chunk->precision == SCI_PRECISION_WIDE)
        return execute<double>(*chunk, static_cast<double *>(output), count, sci_oracle_tail_width(1));
    return execute<float>(*chunk, static_cast<float *>(output), count, sci_oracle_tail_width(0));
}

int sci_oracle_reduce(const sci_chunk *chunk, uint32_t fold, uint64_t count, double *result) {
    if (!chunk || !valid(*chunk) || fold > SCI_FOLD_MAXIMUM || !result) return SCI_CUDA_ERROR_INVALID;
    *result = chunk->precision == SCI_PRECISION_WIDE ? reduce<double>(*chunk, int(fold), count, sci_oracle_tail_width(1))
                                                     : reduce<float>(*chunk, int(fold), count, sci_oracle_tail_width(0));
    return 0;
}

// One element through one code, for ulp sweeps: apply(code, a, b, c) in float or double.
float sci_oracle_apply_f32(uint32_t code, float a, float b, float c, int tail) { return apply<float>(int(code), a, b, c, tail != 0); }
double sci_oracle_apply_f64(uint32_t code, double a, double b, double c, int tail) { return apply<double>(int(code), a, b, c, tail != 0); }

void sci_oracle_factor_f32(float *a, uint64_t *rows, uint64_t n) { factor(a, rows, n); }
void sci_oracle_factor_f64(double *a, uint64_t *rows, uint64_t n) { factor(a, rows, n); }
void sci_oracle_substitute_f64(const double *lu, const uint64_t *rows, const double *right, double *x, uint64_t n,
                               uint64_t width) {
    substitute(lu, rows, right, x, n, width);
}

// Row-major product of float inputs accumulated in double: the FP64 reference the GPU product
// modes report their error against (rows [first, last) only, to keep large cases cheap).
void sci_oracle_product_rows(const float *a, const float *b, double *c, uint64_t m, uint64_t n, uint64_t k,
                             uint64_t first, uint64_t last) {
    (void)m;
    parallel(last - first, [&](uint64_t lo, uint64_t hi, unsigned) {
        std::vector<double> row(n);
        for (uint64_t r = first + lo; r < first + hi; ++r) {
            std::fill(row.begin(), row.end(), 0.0);
            for (uint64_t inner = 0; inner < k; ++inner) {
                const double scale = a[r * k + inner];
                const float *brow = b + inner * n;
                for (uint64_t col = 0; col < n; ++col) row[col] += scale * static_cast<double>(brow[col]);
            }
            std::copy(row.begin(), row.end(), c + (r - first) * n);
        }
    });
}


void sci_oracle_fill(uint32_t precision, void *out, uint64_t count, double value) {
    if (precision == SCI_PRECISION_WIDE) fill_values(static_cast<double *>(out), count, value);
    else fill_values(static_cast<float *>(out), count, static_cast<float>(value));
}
void sci_oracle_linspace(uint32_t precision, void *out, uint64_t count, double start, double stop) {
    if (precision == SCI_PRECISION_WIDE) linspace_values(static_cast<double *>(out), count, start, stop);
    else linspace_values(static_cast<float *>(out), count, static_cast<float>(start), static_cast<float>(stop));
}
uint64_t sci_oracle_range_count(uint32_t precision, double start, double stop, double step) {
    if (precision == SCI_PRECISION_WIDE) return range_count(start, stop, step);
    return range_count(static_cast<float>(start), static_cast<float>(stop), static_cast<float>(step));
}
void sci_oracle_range(uint32_t precision, void *out, uint64_t count, double start, double step) {
    if (precision == SCI_PRECISION_WIDE) range_values(static_cast<double *>(out), count, start, step);
    else range_values(static_cast<float *>(out), count, static_cast<float>(start), static_cast<float>(step));
}
void sci_oracle_eye(uint32_t precision, void *out, uint64_t rows, uint64_t columns) {
    if (precision == SCI_PRECISION_WIDE) eye_values(static_cast<double *>(out), rows, columns);
    else eye_values(static_cast<float *>(out), rows, columns);
}
void sci_oracle_grid(uint32_t precision, const void *x, uint64_t nx, const void *y, uint64_t ny, void *xx, void *yy) {
    if (precision == SCI_PRECISION_WIDE)
        grid_values(static_cast<const double *>(x), nx, static_cast<const double *>(y), ny, static_cast<double *>(xx),
                    static_cast<double *>(yy));
    else
        grid_values(static_cast<const float *>(x), nx, static_cast<const float *>(y), ny, static_cast<float *>(xx),
                    static_cast<float *>(yy));
}

// Integer-element expressions (calculate.hpp, expression.hpp:178-184,203-220); element is a
// SCI_ELEMENT_INT* / UINT* code. reduce writes one element to `result`.
int sci_oracle_execute_elements(uint32_t element, const sci_chunk *chunk, void *output, uint64_t count) {
    if (!chunk || !valid(*chunk)) return SCI_CUDA_ERROR_INVALID;
    return by_int_element(element, [&](auto tag) {
        using T = decltype(tag);
        int_execute<T>(*chunk, static_cast<T *>(output), count);
        return 0;
    });
}

int sci_oracle_reduce_elements(uint32_t element, const sci_chunk *chunk, uint32_t fold, uint64_t count, void *result) {
    if (!chunk || !valid(*chunk) || fold > SCI_FOLD_MAXIMUM || !result) return SCI_CUDA_ERROR_INVALID;
    return by_int_element(element, [&](auto tag) {
        using T = decltype(tag);
        const T value = int_reduce<T>(*chunk, int(fold), count);
        std::memcpy(result, &value, sizeof(T));
        return 0;
    });
}

} // extern "C"
