// sci_math.cuh -- per-element arithmetic of libsci's chunk codes on sm_100a.
//
// Every operation rounds exactly as the reference's AVX-512 kernel table does
// (src/core/drivers/processor/kernels/avx512.cpp:17-153 via
// include/core/drivers/processor/kernels/generic/operation.hpp:21-111):
//  - add / subtract / multiply / divide / root are single IEEE operations; they are written with
//    the _rn intrinsics so the compiler cannot contract a multiply into a following add. Only a
//    chunk `fuse` becomes an fma (chunk.hpp:119-126,253-261).
//  - exp / log / sin / cos repeat the reference's operation sequence (exponential.hpp:24-61,
//    logarithm.hpp:90-126, trigonometry.hpp:162-207) with its coefficients, rounded from double
//    exactly as polynomial.hpp:17-51 computes them, and its constants (constants.hpp:16-120).
//  - the nine functions the reference sends to the C library per lane (library.hpp:22-35) and
//    sin / cos beyond the Cody-Waite reach (trigonometry.hpp:189-205) are evaluated in double
//    with CUDA's double-precision functions and rounded once to float: the nearest float to the
//    true value except for rare double-rounding cases, within 2 ulp of glibc's float result.
//  - minimum / maximum follow the AVX-512 blend form in the vector body and the one-lane Scalar
//    form (scalar.hpp:115-127) in the loop tail, which the caller selects per element.
// The file is included by the ahead-of-time build and by NVRTC specialisations alike, so it
// depends on nothing but the CUDA device headers.
#pragma once


namespace sci_cuda {

    enum Code : int {
        kCopy, kNegate, kAbsolute, kRoot, kExponential, kLogarithm,
        kSin, kCos, kTan, kAsin, kAcos, kAtan, kCsc, kSec, kCot, kAcsc, kAsec, kAcot,
        kSinh, kCosh, kTanh, kAsinh, kAcosh, kAtanh, kCsch, kSech, kCoth, kAcsch, kAsech, kAcoth,
        kAdd, kSubtract, kMultiply, kDivide, kMinimum, kMaximum, kFuse, kCodeCount
    };

    // ---- IEEE building blocks, never contracted ------------------------------------------------
    __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    __device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    __device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
    __device__ __forceinline__ float root(float a) { return __fsqrt_rn(a); }
    __device__ __forceinline__ double root(double a) { return __dsqrt_rn(a); }

    __device__ __forceinline__ unsigned int bits(float v) { return __float_as_uint(v); }
    __device__ __forceinline__ unsigned long long bits(double v) { return (unsigned long long)__double_as_longlong(v); }
    __device__ __forceinline__ float from_bits(unsigned int v) { return __uint_as_float(v); }
    __device__ __forceinline__ double from_bits(unsigned long long v) { return __longlong_as_double((long long)v); }

    __device__ __forceinline__ bool is_nan(float v) { return v != v; }
    __device__ __forceinline__ bool is_nan(double v) { return v != v; }

    // ---- constants (constants.hpp:16-120) ---------------------------------------------------------
    template <typename T> struct Limits;
    template <> struct Limits<float> {
        using U = unsigned int;
        static constexpr int mantissa = 23, width = 32;
        static constexpr U fraction = 0x007fffffu, one = 0x3f800000u, sign = 0x80000000u;
        static constexpr U infinity = 0x7f800000u, quiet = 0x7fc00000u;
        static constexpr float round = 12582912.0f, magnitude = 8388608.0f, exponent = 8388735.0f;
        static constexpr float binary = 1.44269504088896340736f;
        static constexpr float natural = 355.0f / 512.0f, remainder = -2.12194440e-4f;
        static constexpr float lower = -104.0f, upper = 89.0f, normal = 126.0f;
        static constexpr float tiny = 1.17549435e-38f, lift = 33554432.0f, shift = 25.0f;
        static constexpr float root2 = 1.41421356237309504880f;
        static constexpr float quadrant = 0.636619772367581343f;
        static constexpr float q0 = 1.5703125f, q1 = 4.837512969970703125e-4f, q2 = 7.549790126404332e-08f,
                               q3 = -1.7151245100058819e-15f;
        static constexpr float reach = 1048576.0f;
        static constexpr int exp_terms = 8, log_terms = 4, sin_terms = 6, cos_terms = 7;
    };
    template <> struct Limits<double> {
        using U = unsigned long long;
        static constexpr int mantissa = 52, width = 64;
        static constexpr U fraction = 0x000fffffffffffffull, one = 0x3ff0000000000000ull, sign = 0x8000000000000000ull;
        static constexpr U infinity = 0x7ff0000000000000ull, quiet = 0x7ff8000000000000ull;
        static constexpr double round = 6755399441055744.0, magnitude = 4503599627370496.0,
                                exponent = 4503599627371519.0;
        static constexpr double binary = 1.44269504088896340736;
        // ln 2 with its low 21 bits cleared, and the rest (constants.hpp:366-369)
        static constexpr double natural = 0x1.62e42fee00000p-1;
        static constexpr double remainder = 1.90821492927058770002e-10;
        static constexpr double lower = -746.0, upper = 710.0, normal = 1022.0;
        static constexpr double tiny = 2.2250738585072014e-308, lift = 18014398509481984.0, shift = 54.0;
        static constexpr double root2 = 1.41421356237309504880;
        static constexpr double quadrant = 6.36619772367581382433e-01;
        static constexpr double q0 = 1.57079632673412561417e+00, q1 = 6.07710050630396597660e-11,
                                q2 = 2.02226624871116645580e-21, q3 = 8.47842766036889956997e-32;
        static constexpr double reach = 1048576.0;
        static constexpr int exp_terms = 14, log_terms = 10, sin_terms = 10, cos_terms = 11;
    };

    // Polynomial coefficients, computed in double and rounded to T as polynomial.hpp:17-51 does:
    // 1/k! (factorials), 2/(2k+3) (reciprocals), (-1)^k/(2k+offset)! (alternating).
    template <typename T, int N> struct Poly {
        T c[N];
    };
    template <typename T, int N> __host__ __device__ constexpr Poly<T, N> factorials() {
        Poly<T, N> p{};
        double f = 1.0;
        for (int k = 0; k < N; ++k) {
            if (k > 0) f /= static_cast<double>(k);
            p.c[k] = static_cast<T>(f);
        }
        return p;
    }
    template <typename T, int N> __host__ __device__ constexpr Poly<T, N> reciprocals() {
        Poly<T, N> p{};
        for (int k = 0; k < N; ++k) p.c[k] = static_cast<T>(2.0 / static_cast<double>(2 * k + 3));
        return p;
    }
    template <typename T, int N, int offset> __host__ __device__ constexpr Poly<T, N> alternating() {
        Poly<T, N> p{};
        for (int k = 0; k < N; ++k) {
            double f = 1.0;
            for (int s = 2; s <= 2 * k + offset; ++s) f *= static_cast<double>(s);
            p.c[k] = static_cast<T>((k % 2 == 0 ? 1.0 : -1.0) / f);
        }
        return p;
    }
    // sum c[k] x^(k - from), Horner from the top coefficient (polynomial.hpp:271-277).
    template <int from, typename T, int N> __device__ __forceinline__ T horner(const Poly<T, N> &p, T x) {
        T r = p.c[N - 1];
#pragma unroll
        for (int k = N - 2; k >= from; --k) r = fma_(r, x, p.c[k]);
        return r;
    }

    // ---- minimum / maximum (avx512.cpp:43-49 body, scalar.hpp:115-127 tail) -----------------------
    template <typename T> __device__ __forceinline__ T vmin(T l, T r) { return is_nan(l) ? l : (l < r ? l : r); }
    template <typename T> __device__ __forceinline__ T vmax(T l, T r) { return is_nan(l) ? l : (l > r ? l : r); }
    template <typename T> __device__ __forceinline__ T smin(T l, T r) {
        return (is_nan(l) || is_nan(r)) ? add(l, r) : (r < l ? r : l);
    }
    template <typename T> __device__ __forceinline__ T smax(T l, T r) {
        return (is_nan(l) || is_nan(r)) ? add(l, r) : (r > l ? r : l);
    }

    // ---- e^x (exponential.hpp:24-61) --------------------------------------------------------------
    // The reference splits the final scale in two when any lane of its pack has |k| > normal; for
    // the other lanes both forms round the same exact product once, so the split is decided per
    // element here.
    template <typename T> __device__ __forceinline__ T exponential(T x) {
        using L = Limits<T>;
        constexpr Poly<T, L::exp_terms> series = factorials<T, L::exp_terms>();
        const T clamped = vmax(vmin(x, L::upper), L::lower);
        const T k = sub(fma_(clamped, L::binary, L::round), L::round);
        const T negative = -k;
        T reduced = fma_(negative, L::natural, clamped);
        reduced = fma_(negative, L::remainder, reduced);
        const T significand = fma_(reduced, horner<1>(series, reduced), T(1));
        auto scale = [](T e) { return from_bits(bits(add(e, L::exponent)) << L::mantissa); };
        if (!(fabs(k) > L::normal)) return mul(significand, scale(k));
        const T half = sub(fma_(k, T(0.5), L::round), L::round);
        const T rest = sub(k, half);
        return mul(mul(significand, scale(half)), scale(rest));
    }

    // ---- ln x (logarithm.hpp:90-126) --------------------------------------------------------------
    template <typename T> __device__ __forceinline__ T logarithm(T x) {
        using L = Limits<T>;
        using U = typename L::U;
        constexpr Poly<T, L::log_terms> series = reciprocals<T, L::log_terms>();
        const bool small = x < L::tiny;
        const T scaled = small ? mul(x, L::lift) : x;
        const U pattern = bits(scaled);
        T exponent = sub(from_bits((pattern >> L::mantissa) | bits(L::magnitude)), L::exponent);
        T mantissa = from_bits((pattern & L::fraction) | L::one);
        const bool large = mantissa > L::root2;
        mantissa = large ? mul(mantissa, T(0.5)) : mantissa;
        exponent = large ? add(exponent, T(1)) : exponent;
        exponent = small ? sub(exponent, L::shift) : exponent;
        const T fraction = sub(mantissa, T(1));
        const T ratio = div(fraction, add(fraction, T(2)));
        const T square = mul(ratio, ratio);
        const T tail = mul(square, horner<0>(series, square));
        const T half = mul(mul(fraction, fraction), T(0.5));
        const T inner = fma_(ratio, add(half, tail), mul(exponent, L::remainder));
        T result = sub(mul(exponent, L::natural), sub(sub(half, inner), fraction));
        const T infinity = from_bits(L::infinity);
        if (x == infinity) result = x;
        if (x == T(0)) result = -infinity;
        if (x < T(0)) result = from_bits(L::quiet);
        if (is_nan(x)) result = x;
        return result;
    }

    // ---- sin / cos (trigonometry.hpp:162-207) -----------------------------------------------------
    __device__ __forceinline__ float far_circular(float x, bool phase) {
        const double d = static_cast<double>(x);
        return static_cast<float>(phase ? cos(d) : sin(d));
    }
    __device__ __forceinline__ double far_circular(double x, bool phase) { return phase ? cos(x) : sin(x); }

    template <bool phase, typename T> __device__ __forceinline__ T circular(T x) {
        using L = Limits<T>;
        using U = typename L::U;
        constexpr Poly<T, L::sin_terms> odd = alternating<T, L::sin_terms, 1>();
        constexpr Poly<T, L::cos_terms> even = alternating<T, L::cos_terms, 0>();
        const T shifted = fma_(x, L::quadrant, L::round);
        const T quarters = sub(shifted, L::round);
        const T negative = -quarters;
        T reduced = fma_(negative, L::q0, x);
        reduced = fma_(negative, L::q1, reduced);
        reduced = fma_(negative, L::q2, reduced);
        reduced = fma_(negative, L::q3, reduced);
        const T square = mul(reduced, reduced);
        const T sine = fma_(mul(reduced, square), horner<1>(odd, square), reduced);
        const T cosine = fma_(square, horner<1>(even, square), T(1));
        U quadrant = bits(shifted);
        if (phase) quadrant ^= quadrant << 1;
        const U flip = (quadrant & U(2)) << (L::width - 2);
        const bool swap = (bits(shifted) & U(1)) != 0;
        T result = phase ? (swap ? sine : cosine) : (swap ? cosine : sine);
        result = from_bits(bits(result) ^ flip);
        if (!(x <= L::reach && x >= -L::reach)) result = far_circular(x, phase);
        return result;
    }

    // ---- the C-library functions (library.hpp:22-35), in double, rounded once -------------------
    template <int code> __device__ __forceinline__ double library_d(double x) {
        if constexpr (code == kAsin) return asin(x);
        else if constexpr (code == kAcos) return acos(x);
        else if constexpr (code == kAtan) return atan(x);
        else if constexpr (code == kSinh) return sinh(x);
        else if constexpr (code == kCosh) return cosh(x);
        else if constexpr (code == kTanh) return tanh(x);
        else if constexpr (code == kAsinh) return asinh(x);
        else if constexpr (code == kAcosh) return acosh(x);
        else return atanh(x);
    }
    // tanh of a float, in double and rounded once. With 2|x| = k ln 2 + r, |r| <= ln 2 / 2:
    //   e^{2|x|} - 1 = 2^k (1 + q) - 1 and e^{2|x|} + 1 = 2^k (1 + q) + 1, q = e^r - 1,
    // q from its Taylor series through r^12/12! (truncation below 2^-51 relative), and the quotient
    // of the two by Newton-Raphson refinement of an approximate reciprocal, then one correction of
    // the quotient with its residual. Relative error about 2^-50, so the float rounding is the
    // correctly rounded one except when the true value lies within ~2^-50 of a rounding midpoint.
    // k = 0 keeps q itself as the numerator, so small |x| loses nothing to cancellation.
    // |x| < 2^-12 rounds to x (tanh x = x (1 - x^2/3 + ...), and x^2/3 < 2^-25.5); |x| > 9.03
    // rounds to 1 (1 - tanh x < 2 e^{-18.06} < 2^-25).
    __device__ __forceinline__ float tanh_float(float x) {
        const float a = fabsf(x);
        if (!(a >= 0x1p-12f)) return a < 0x1p-12f ? x : __fadd_rn(x, x);  // tiny, or NaN
        if (a > 9.03125f) return copysignf(1.0f, x);
        const double d = 2.0 * static_cast<double>(a);
        const double k = __dadd_rn(__dadd_rn(__dmul_rn(d, 0x1.71547652b82fep+0), 0x1.8p52), -0x1.8p52);
        double r = __fma_rn(-k, 0x1.62e42fefa3800p-1, d);
        r = __fma_rn(-k, 0x1.ef35793c76730p-45, r);
        // 1/2!, 1/3!, ..., 1/12!
        double p = 1.0 / 479001600.0;
        p = __fma_rn(p, r, 1.0 / 39916800.0);
        p = __fma_rn(p, r, 1.0 / 3628800.0);
        p = __fma_rn(p, r, 1.0 / 362880.0);
        p = __fma_rn(p, r, 1.0 / 40320.0);
        p = __fma_rn(p, r, 1.0 / 5040.0);
        p = __fma_rn(p, r, 1.0 / 720.0);
        p = __fma_rn(p, r, 1.0 / 120.0);
        p = __fma_rn(p, r, 1.0 / 24.0);
        p = __fma_rn(p, r, 1.0 / 6.0);
        p = __fma_rn(p, r, 0.5);
        const double q = __fma_rn(__dmul_rn(r, r), p, r);
        const double s = __longlong_as_double(static_cast<long long>(static_cast<int>(k) + 1023) << 52);
        const double num = __fma_rn(s, q, __dsub_rn(s, 1.0));
        const double den = __fma_rn(s, q, __dadd_rn(s, 1.0));
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(den));
        double e = __fma_rn(-den, y, 1.0);
        y = __fma_rn(y, e, y);
        e = __fma_rn(-den, y, 1.0);
        y = __fma_rn(y, e, y);
        double t = __dmul_rn(num, y);
        t = __fma_rn(__fma_rn(-den, t, num), y, t);
        return copysignf(static_cast<float>(t), x);
    }

    template <int code, typename T> __device__ __forceinline__ T library(T x) {
        if constexpr (code == kTanh && sizeof(T) == 4) return tanh_float(x);
        else return static_cast<T>(library_d<code>(static_cast<double>(x)));
    }

    // ---- one code on one element (operation.hpp:25-110) ------------------------------------------
    template <int code, typename T> __device__ __forceinline__ T apply(T a, T b, T c, bool tail) {
        using L = Limits<T>;
        const T one = T(1);
        if constexpr (code == kCopy) return a;
        else if constexpr (code == kNegate) return from_bits(bits(a) ^ L::sign);
        else if constexpr (code == kAbsolute) return from_bits(bits(a) & ~L::sign);
        else if constexpr (code == kRoot) return root(a);
        else if constexpr (code == kExponential) return exponential(a);
        else if constexpr (code == kLogarithm) return logarithm(a);
        else if constexpr (code == kSin) return circular<false>(a);
        else if constexpr (code == kCos) return circular<true>(a);
        else if constexpr (code == kTan) return div(circular<false>(a), circular<true>(a));
        else if constexpr (code == kAsin || code == kAcos || code == kAtan || code == kSinh || code == kCosh ||
                           code == kTanh || code == kAsinh || code == kAcosh || code == kAtanh)
            return library<code>(a);
        else if constexpr (code == kCsc) return div(one, circular<false>(a));
        else if constexpr (code == kSec) return div(one, circular<true>(a));
        else if constexpr (code == kCot) return div(one, div(circular<false>(a), circular<true>(a)));
        else if constexpr (code == kAcsc) return library<kAsin>(div(one, a));
        else if constexpr (code == kAsec) return library<kAcos>(div(one, a));
        else if constexpr (code == kAcot) return library<kAtan>(div(one, a));
        else if constexpr (code == kCsch) return div(one, library<kSinh>(a));
        else if constexpr (code == kSech) return div(one, library<kCosh>(a));
        else if constexpr (code == kCoth) return div(one, library<kTanh>(a));
        else if constexpr (code == kAcsch) return library<kAsinh>(div(one, a));
        else if constexpr (code == kAsech) return library<kAcosh>(div(one, a));
        else if constexpr (code == kAcoth) return library<kAtanh>(div(one, a));
        else if constexpr (code == kAdd) return add(a, b);
        else if constexpr (code == kSubtract) return sub(a, b);
        else if constexpr (code == kMultiply) return mul(a, b);
        else if constexpr (code == kDivide) return div(a, b);
        else if constexpr (code == kMinimum) return tail ? smin(a, b) : vmin(a, b);
        else if constexpr (code == kMaximum) return tail ? smax(a, b) : vmax(a, b);
        else return fma_(a, b, c);
    }

    // ---- fast forms --------------------------------------------------------------------------------
    // The same operations as the forms above, in the same order, for the inputs that take none of
    // their special branches; an element outside that set raises `rare`, and the caller recomputes
    // the whole group with the forms above. Each returns exactly what its full form returns whenever
    // it leaves `rare` alone.

    // a / d for |a| <= 1/2 and d in [1.5, 2.5] (the logarithm's ratio), by the division method of
    // Markstein (IBM J. Res. Dev. 34(1), 1990): a reciprocal estimate, one Newton-Raphson step with
    // a fused multiply-add, then one correction of the quotient q + (a - d q) y. On this range no
    // step can overflow or underflow, and the result is the correctly rounded quotient (checked
    // against IEEE division for every operand pair the logarithm can form).
    __device__ __forceinline__ float ratio_quotient(float a, float d) {
        float y;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
        const float e = __fmaf_rn(-d, y, 1.0f);
        y = __fmaf_rn(y, e, y);
        const float q = __fmul_rn(a, y);
        const float r = __fmaf_rn(-d, q, a);
        return __fmaf_rn(r, y, q);
    }
    __device__ __forceinline__ double ratio_quotient(double a, double d) { return div(a, d); }

    // e^x for |x| below (normal + 1/2) ln 2: no clamp applies and |k| <= normal, so the single scale.
    template <typename T> __device__ __forceinline__ T exponential_fast(T x, bool &rare) {
        using L = Limits<T>;
        constexpr Poly<T, L::exp_terms> series = factorials<T, L::exp_terms>();
        constexpr T reach = sizeof(T) == 4 ? T(87) : T(708);
        rare |= !(fabs(x) <= reach);
        const T k = sub(fma_(x, L::binary, L::round), L::round);
        const T negative = -k;
        T reduced = fma_(negative, L::natural, x);
        reduced = fma_(negative, L::remainder, reduced);
        const T significand = fma_(reduced, horner<1>(series, reduced), T(1));
        return mul(significand, from_bits(bits(add(k, L::exponent)) << L::mantissa));
    }

    // ln x for positive, normal, finite x: no scaling of subnormals and none of the special results.
    template <typename T> __device__ __forceinline__ T logarithm_fast(T x, bool &rare) {
        using L = Limits<T>;
        using U = typename L::U;
        constexpr Poly<T, L::log_terms> series = reciprocals<T, L::log_terms>();
        const U pattern = bits(x);
        rare |= pattern - bits(L::tiny) >= L::infinity - bits(L::tiny);
        T exponent = sub(from_bits((pattern >> L::mantissa) | bits(L::magnitude)), L::exponent);
        T mantissa = from_bits((pattern & L::fraction) | L::one);
        const bool large = mantissa > L::root2;
        mantissa = large ? mul(mantissa, T(0.5)) : mantissa;
        exponent = large ? add(exponent, T(1)) : exponent;
        const T fraction = sub(mantissa, T(1));
        const T ratio = ratio_quotient(fraction, add(fraction, T(2)));
        const T square = mul(ratio, ratio);
        const T tail = mul(square, horner<0>(series, square));
        const T half = mul(mul(fraction, fraction), T(0.5));
        const T inner = fma_(ratio, add(half, tail), mul(exponent, L::remainder));
        return sub(mul(exponent, L::natural), sub(sub(half, inner), fraction));
    }

    // sin / cos for |x| <= reach (no far reduction).
    template <bool phase, typename T> __device__ __forceinline__ T circular_fast(T x, bool &rare) {
        using L = Limits<T>;
        using U = typename L::U;
        constexpr Poly<T, L::sin_terms> odd = alternating<T, L::sin_terms, 1>();
        constexpr Poly<T, L::cos_terms> even = alternating<T, L::cos_terms, 0>();
        rare |= !(fabs(x) <= L::reach);
        const T shifted = fma_(x, L::quadrant, L::round);
        const T quarters = sub(shifted, L::round);
        const T negative = -quarters;
        T reduced = fma_(negative, L::q0, x);
        reduced = fma_(negative, L::q1, reduced);
        reduced = fma_(negative, L::q2, reduced);
        reduced = fma_(negative, L::q3, reduced);
        const T square = mul(reduced, reduced);
        const T sine = fma_(mul(reduced, square), horner<1>(odd, square), reduced);
        const T cosine = fma_(square, horner<1>(even, square), T(1));
        U quadrant = bits(shifted);
        if (phase) quadrant ^= quadrant << 1;
        const U flip = (quadrant & U(2)) << (L::width - 2);
        const bool swap = (bits(shifted) & U(1)) != 0;
        const T result = phase ? (swap ? sine : cosine) : (swap ? cosine : sine);
        return from_bits(bits(result) ^ flip);
    }

    // tanh of a float without branches: the double-precision evaluation of tanh_float runs on
    // min(|x|, 9.03125) (so no infinity or NaN enters it), and the tiny, saturated and NaN results
    // are selected at the end. Three changes cut its FP64 work: 2|x| is assembled as a double from
    // the float's fields with integer operations (exact for every normal float; the others are
    // selected away), k is rounded from one fused multiply-add and 2^k is formed from the bits of
    // that sum, and the reciprocal takes one Newton-Raphson step, since the final correction of the
    // quotient squares its error. Its float results equal tanh_float's for every float input.
    __device__ __forceinline__ float tanh_float_fast(float x) {
        const float a = fabsf(x);
        const unsigned field = __float_as_uint(fminf(a, 9.03125f));
        // sign 0; exponent e - 127 + 1023 + 1 (the factor 2); the 23 fraction bits at the top of 52
        const double d = __hiloint2double(static_cast<int>((field >> 3) + (897u << 20)), static_cast<int>(field << 29));
        const double sum = __fma_rn(d, 0x1.71547652b82fep+0, 0x1.8p52);
        const double k = __dadd_rn(sum, -0x1.8p52);
        double r = __fma_rn(-k, 0x1.62e42fefa3800p-1, d);
        r = __fma_rn(-k, 0x1.ef35793c76730p-45, r);
        double p = 1.0 / 479001600.0;
        p = __fma_rn(p, r, 1.0 / 39916800.0);
        p = __fma_rn(p, r, 1.0 / 3628800.0);
        p = __fma_rn(p, r, 1.0 / 362880.0);
        p = __fma_rn(p, r, 1.0 / 40320.0);
        p = __fma_rn(p, r, 1.0 / 5040.0);
        p = __fma_rn(p, r, 1.0 / 720.0);
        p = __fma_rn(p, r, 1.0 / 120.0);
        p = __fma_rn(p, r, 1.0 / 24.0);
        p = __fma_rn(p, r, 1.0 / 6.0);
        p = __fma_rn(p, r, 0.5);
        const double q = __fma_rn(__dmul_rn(r, r), p, r);
        // k is a small non-negative integer held in the low bits of `sum`
        const unsigned kbits = static_cast<unsigned>(__double2loint(sum));
        const double s = __hiloint2double(static_cast<int>((kbits + 1023u) << 20), 0);
        const double num = __fma_rn(s, q, __dsub_rn(s, 1.0));
        const double den = __fma_rn(s, q, __dadd_rn(s, 1.0));
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(den));
        y = __fma_rn(y, __fma_rn(-den, y, 1.0), y);
        double t = __dmul_rn(num, y);
        t = __fma_rn(__fma_rn(-den, t, num), y, t);
        float result = copysignf(static_cast<float>(t), x);
        result = a > 9.03125f ? copysignf(1.0f, x) : result;
        result = a < 0x1p-12f ? x : result;
        return a == a ? result : __fadd_rn(x, x);
    }

    // tanh of a float with |x| <= 1, in double: tanh x = x + x^3 g(x^2), where g is the degree-11
    // polynomial interpolating g(u) = (tanh(sqrt u) / sqrt u - 1) / u at the 12 Chebyshev nodes of
    // [0, 1] (coefficients computed in 60-digit arithmetic by libsci_b200/coefficients.py and
    // rounded to double; their relative error against g is below 2^-41.7 on [0, 1]). u = x^2 is
    // exact in double, and the result t is within 2^-43 relative of tanh x. Its float rounding is
    // therefore the correctly rounded value -- the one tanh_float returns, whose own error is about
    // 2^-50 -- unless tanh x lies within 2^-41 relative of a float rounding midpoint: the 29 bits of
    // t below the float's last place then lie within 2^12 of 100...0, and `rare` is set so that the
    // caller recomputes with tanh_float. No infinity or NaN reaches it (|x| <= 1).
    __device__ __forceinline__ float tanh_float_near(float x, bool &rare) {
        const double a = static_cast<double>(x);
        const double u = __dmul_rn(a, a);
        double g = 0x1.fcc078193c27dp-20;
        g = __fma_rn(g, u, -0x1.0d3ce4aaa45fcp-16);
        g = __fma_rn(g, u, 0x1.2347b46ddb8b5p-14);
        g = __fma_rn(g, u, -0x1.c5bfee363a8b2p-13);
        g = __fma_rn(g, u, 0x1.2e76669b584c5p-11);
        g = __fma_rn(g, u, -0x1.7c4648492ca7bp-10);
        g = __fma_rn(g, u, 0x1.d6a56a6f2f6f3p-9);
        g = __fma_rn(g, u, -0x1.226c3a99b757dp-7);
        g = __fma_rn(g, u, 0x1.664f2ec3a9f0dp-6);
        g = __fma_rn(g, u, -0x1.ba1ba10bdf714p-5);
        g = __fma_rn(g, u, 0x1.1111111028c6fp-3);
        g = __fma_rn(g, u, -0x1.5555555554ee4p-2);
        const double t = __fma_rn(__dmul_rn(a, u), g, a);
        const unsigned below = static_cast<unsigned>(__double2loint(t)) & 0x1fffffffu;
        rare = rare || below - 0x0ffff000u <= 0x2000u;
        // t has x's sign except at x = -0, where the sum gives +0: the sign is taken from x
        return copysignf(static_cast<float>(t), x);
    }

    // ---- two floats per instruction ----------------------------------------------------------------
    // sm_100 adds packed two-lane FP32 arithmetic (add / sub / mul / fma .rn .f32x2): each lane is
    // rounded exactly as the one-lane instruction rounds it, and one instruction issues for both. The
    // paired fast forms below run the fast forms' floating-point steps on two elements at once
    // (integer, compare and select steps stay per lane) and return the same bits. Where a fast form
    // multiplies by a negated value, the pair form multiplies by the negated constant instead: the
    // exact products are equal, so the rounded results are.
    struct Pair {
        unsigned long long v;
    };
    __device__ __forceinline__ Pair pair(float lo, float hi) {
        Pair p;
        asm("mov.b64 %0, {%1, %2};" : "=l"(p.v) : "f"(lo), "f"(hi));
        return p;
    }
    __device__ __forceinline__ Pair pair(float both) { return pair(both, both); }
    __device__ __forceinline__ void unpair(Pair p, float &lo, float &hi) {
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(p.v));
    }
    __device__ __forceinline__ Pair add(Pair a, Pair b) {
        Pair d;
        asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
        return d;
    }
    __device__ __forceinline__ Pair sub(Pair a, Pair b) {
        Pair d;
        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
        return d;
    }
    __device__ __forceinline__ Pair mul(Pair a, Pair b) {
        Pair d;
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
        return d;
    }
    __device__ __forceinline__ Pair fma_(Pair a, Pair b, Pair c) {
        Pair d;
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
        return d;
    }
    template <int from, int N> __device__ __forceinline__ Pair horner(const Poly<float, N> &p, Pair x) {
        Pair r = pair(p.c[N - 1]);
#pragma unroll
        for (int k = N - 2; k >= from; --k) r = fma_(r, x, pair(p.c[k]));
        return r;
    }

    // exponential_fast on two elements.
    __device__ __forceinline__ void exponential_pair(float x0, float x1, bool &rare, float &r0, float &r1) {
        using L = Limits<float>;
        constexpr Poly<float, L::exp_terms> series = factorials<float, L::exp_terms>();
        rare |= !(fabsf(x0) <= 87.0f) | !(fabsf(x1) <= 87.0f);
        const Pair x = pair(x0, x1);
        const Pair k = sub(fma_(x, pair(L::binary), pair(L::round)), pair(L::round));
        Pair reduced = fma_(k, pair(-L::natural), x);
        reduced = fma_(k, pair(-L::remainder), reduced);
        const Pair significand = fma_(reduced, horner<1>(series, reduced), pair(1.0f));
        float e0, e1, s0, s1;
        unpair(add(k, pair(L::exponent)), e0, e1);
        // the last multiply per lane, so no packed product reaches an add of the caller's
        unpair(significand, s0, s1);
        r0 = mul(s0, from_bits(bits(e0) << L::mantissa));
        r1 = mul(s1, from_bits(bits(e1) << L::mantissa));
    }

    // logarithm_fast on two elements. The two selects of the `large` adjustment become a multiply by
    // 1/2 or 1 and an add of 1 or 0 (exact either way; the exponent is never -0).
    __device__ __forceinline__ void logarithm_pair(float x0, float x1, bool &rare, float &r0, float &r1) {
        using L = Limits<float>;
        constexpr Poly<float, L::log_terms> series = reciprocals<float, L::log_terms>();
        const unsigned p0 = bits(x0), p1 = bits(x1);
        rare |= (p0 - bits(L::tiny) >= L::infinity - bits(L::tiny)) | (p1 - bits(L::tiny) >= L::infinity - bits(L::tiny));
        const Pair field = pair(from_bits((p0 >> L::mantissa) | bits(L::magnitude)),
                                from_bits((p1 >> L::mantissa) | bits(L::magnitude)));
        const float m0 = from_bits((p0 & L::fraction) | L::one), m1 = from_bits((p1 & L::fraction) | L::one);
        const bool g0 = m0 > L::root2, g1 = m1 > L::root2;
        const Pair mantissa = mul(pair(m0, m1), pair(g0 ? 0.5f : 1.0f, g1 ? 0.5f : 1.0f));
        const Pair exponent = add(sub(field, pair(L::exponent)), pair(g0 ? 1.0f : 0.0f, g1 ? 1.0f : 0.0f));
        const Pair fraction = sub(mantissa, pair(1.0f));
        // ratio_quotient(fraction, fraction + 2) with the negated divisor formed directly
        const Pair divisor = add(fraction, pair(2.0f));
        const Pair negated = sub(pair(-2.0f), fraction);
        float d0, d1, y0, y1;
        unpair(divisor, d0, d1);
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(d0));
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y1) : "f"(d1));
        Pair y = pair(y0, y1);
        y = fma_(y, fma_(negated, y, pair(1.0f)), y);
        const Pair q = mul(fraction, y);
        const Pair ratio = fma_(fma_(negated, q, fraction), y, q);
        const Pair square = mul(ratio, ratio);
        // One-lane multiplies for the tail: a packed multiply feeding the packed add below can be
        // fused into one packed fma by the code generator (seen on sm_100a despite .rn), which
        // changes the rounding; the other products that feed adds here are exact (mantissa x 1/2,
        // fraction^2 x 1/2, exponent x 355/512), so fusing them changes nothing.
        float s0, s1, h0, h1;
        unpair(square, s0, s1);
        unpair(horner<0>(series, square), h0, h1);
        const Pair tail = pair(mul(s0, h0), mul(s1, h1));
        const Pair half = mul(mul(fraction, fraction), pair(0.5f));
        const Pair inner = fma_(ratio, add(half, tail), mul(exponent, pair(L::remainder)));
        unpair(sub(mul(exponent, pair(L::natural)), sub(sub(half, inner), fraction)), r0, r1);
    }

    // circular_fast<phase> on two elements.
    template <bool phase>
    __device__ __forceinline__ void circular_pair(float x0, float x1, bool &rare, float &r0, float &r1) {
        using L = Limits<float>;
        constexpr Poly<float, L::sin_terms> odd = alternating<float, L::sin_terms, 1>();
        constexpr Poly<float, L::cos_terms> even = alternating<float, L::cos_terms, 0>();
        rare |= !(fabsf(x0) <= L::reach) | !(fabsf(x1) <= L::reach);
        const Pair x = pair(x0, x1);
        const Pair shifted = fma_(x, pair(L::quadrant), pair(L::round));
        const Pair quarters = sub(shifted, pair(L::round));
        Pair reduced = fma_(quarters, pair(-L::q0), x);
        reduced = fma_(quarters, pair(-L::q1), reduced);
        reduced = fma_(quarters, pair(-L::q2), reduced);
        reduced = fma_(quarters, pair(-L::q3), reduced);
        const Pair square = mul(reduced, reduced);
        const Pair sine = fma_(mul(reduced, square), horner<1>(odd, square), reduced);
        const Pair cosine = fma_(square, horner<1>(even, square), pair(1.0f));
        float s[2], c[2], h[2], out[2];
        unpair(sine, s[0], s[1]);
        unpair(cosine, c[0], c[1]);
        unpair(shifted, h[0], h[1]);
        // Per lane, q = the low bits of `shifted`: bit 0 swaps sine and cosine, and the sign flips
        // with bit 1 of q for the sine, with bit 1 of q ^ (q << 1) = bit 1 of q + 1 for the cosine
        // (the forms above); shifted left by 30 either lands on the sign bit.
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const unsigned q = bits(h[i]);
            const unsigned sign = ((phase ? q + 1u : q) << 30) & 0x80000000u;
            const float result = ((q & 1u) != 0) != phase ? c[i] : s[i];
            out[i] = from_bits(bits(result) ^ sign);
        }
        r0 = out[0];
        r1 = out[1];
    }

    template <int code, typename T> __device__ __forceinline__ constexpr bool has_pair() {
        return sizeof(T) == 4 && (code == kExponential || code == kLogarithm || code == kSin || code == kCos ||
                                  code == kTan || code == kCsc || code == kSec || code == kCot);
    }

    // The paired fast form of a code (has_pair<code, float>()).
    template <int code> __device__ __forceinline__ void apply_pair(float a0, float a1, bool &rare, float &r0, float &r1) {
        if constexpr (code == kExponential) {
            exponential_pair(a0, a1, rare, r0, r1);
        } else if constexpr (code == kLogarithm) {
            logarithm_pair(a0, a1, rare, r0, r1);
        } else if constexpr (code == kSin) {
            circular_pair<false>(a0, a1, rare, r0, r1);
        } else if constexpr (code == kCos) {
            circular_pair<true>(a0, a1, rare, r0, r1);
        } else {
            float s0, s1, c0, c1;
            if constexpr (code != kSec) circular_pair<false>(a0, a1, rare, s0, s1);
            if constexpr (code != kCsc) circular_pair<true>(a0, a1, rare, c0, c1);
            if constexpr (code == kTan) {
                r0 = div(s0, c0);
                r1 = div(s1, c1);
            } else if constexpr (code == kCsc) {
                r0 = div(1.0f, s0);
                r1 = div(1.0f, s1);
            } else if constexpr (code == kSec) {
                r0 = div(1.0f, c0);
                r1 = div(1.0f, c1);
            } else {
                r0 = div(1.0f, div(s0, c0));
                r1 = div(1.0f, div(s1, c1));
            }
        }
    }

    template <int code, typename T> __device__ __forceinline__ constexpr bool has_fast() {
        return code == kExponential || code == kLogarithm || code == kSin || code == kCos || code == kTan ||
               code == kCsc || code == kSec || code == kCot || ((code == kTanh || code == kCoth) && sizeof(T) == 4);
    }

    // The fast form of a unary code (has_fast<code, T>()).
    template <int code, typename T> __device__ __forceinline__ T apply_fast(T a, bool &rare) {
        const T one = T(1);
        if constexpr (code == kExponential) return exponential_fast(a, rare);
        else if constexpr (code == kLogarithm) return logarithm_fast(a, rare);
        else if constexpr (code == kSin) return circular_fast<false>(a, rare);
        else if constexpr (code == kCos) return circular_fast<true>(a, rare);
        else if constexpr (code == kTan) return div(circular_fast<false>(a, rare), circular_fast<true>(a, rare));
        else if constexpr (code == kCsc) return div(one, circular_fast<false>(a, rare));
        else if constexpr (code == kSec) return div(one, circular_fast<true>(a, rare));
        else if constexpr (code == kCot) return div(one, div(circular_fast<false>(a, rare), circular_fast<true>(a, rare)));
        else if constexpr (code == kTanh) return tanh_float_fast(a);
        else return div(one, tanh_float_fast(a));
    }

} // namespace sci_cuda