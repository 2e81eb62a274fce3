// integration/device_test.cpp -- libsci's public API (sci.hpp) on a Device(Target::cuda), checked
// against the same API on the host. Built against the reference's headers, unchanged, with
// integration/device.cpp as the Device and libsci_cuda.so as the backend.
//
// What is checked, after the pins of the reference's own tests:
//  - tests/core/drivers/test_device.cpp:14-26: an expression of arrays moved to the device, read
//    back with host(), equals the host's (here bit for bit), and so does sum();
//  - tests/operations/test_binary.cpp:29-50: every binary operation, scalars on either side, the
//    fused multiply-add and NaN in minimum / maximum, bit for bit against the host;
//  - tests/operations/test_unary.cpp: exp / log / sin / cos / sqrt / abs / negate bit for bit, the
//    C-library functions within 2 ulp;
//  - tests/operations/test_reduce.cpp: sum / mean / minimum / maximum of device expressions;
//  - tests/linear/test_product.cpp:8-33: the 37 x 53 x 29 product within 1e-3 of a double loop,
//    and a larger one within the FP32 bound of the host's product;
//  - tests/linear/test_solve.cpp:8-25 and test_decompose.cpp:21-36: solve and decompose through
//    sci::linear::cuda on device arrays;
//  - double arrays on the device (the reference's GPU refuses them, device.cpp:148);
//  - no CPU fallback: an expression over a host array assigned on the device throws.
// Exit status: 0 all passed, 1 a check failed, 77 no CUDA device here.
#include <sci.hpp>

#include "sci_cuda_device.hpp"

#include <bit>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

    int failures = 0;

    void expect(const bool ok, const char *what) {
        std::printf("%s %s\n", ok ? "ok" : "FAIL", what);
        if (!ok) ++failures;
    }

    template <typename T> bool same_bits(const T a, const T b) {
        if (std::isnan(a) && std::isnan(b)) return true;
        if constexpr (sizeof(T) == 4) return std::bit_cast<uint32_t>(a) == std::bit_cast<uint32_t>(b);
        else return std::bit_cast<uint64_t>(a) == std::bit_cast<uint64_t>(b);
    }

    // Distance in units in the last place between two floats of the same sign class.
    int64_t ulps(const float a, const float b) {
        if (std::isnan(a) || std::isnan(b)) return std::isnan(a) && std::isnan(b) ? 0 : INT64_MAX;
        auto ordered = [](const float v) {
            const int32_t i = std::bit_cast<int32_t>(v);
            return i < 0 ? -int64_t(i & 0x7fffffff) : int64_t(i);
        };
        const int64_t d = ordered(a) - ordered(b);
        return d < 0 ? -d : d;
    }

    template <typename T, sci::core::size R>
    bool bitwise(const sci::Array<T, R> &device_result, const sci::Array<T, R> &host_result) {
        const sci::Array<T, R> read = device_result.host();
        if (read.size() != host_result.size()) return false;
        for (sci::core::size i = 0; i < read.size(); ++i)
            if (!same_bits(read.data()[i], host_result.data()[i])) return false;
        return true;
    }

    template <typename T> sci::Array<T, 1> seeded(const std::size_t count, const unsigned seed, const double low,
                                                  const double high) {
        std::mt19937_64 engine(seed);
        std::uniform_real_distribution<double> uniform(low, high);
        sci::Array<T, 1> out(sci::Shape<1>{count});
        for (std::size_t i = 0; i < count; ++i) out.data()[i] = static_cast<T>(uniform(engine));
        return out;
    }

} // namespace

int main() {
    std::unique_ptr<sci::Device> opened;
    try {
        opened = std::make_unique<sci::Device>(sci::core::drivers::cuda_target);
    } catch (const std::runtime_error &error) {
        std::printf("skip: %s\n", error.what());
        return 77;
    }
    sci::Device &gpu = *opened;
    expect(gpu.target() == sci::core::drivers::cuda_target, "the device is the CUDA target");
    std::printf("device: %s\n", gpu.name());

    // test_device.cpp:14-26, bit for bit
    {
        constexpr std::size_t count = 200'000;
        const sci::Array<float, 1> first = sci::linspace(0.0f, 2.0f, count);
        const sci::Array<float, 1> second = sci::linspace(1.0f, 3.0f, count);
        const sci::Array<float, 1> expected = first * second + 1.0f;
        const auto moved = first.to(gpu);
        const auto other = second.to(gpu);
        const sci::Array<float, 1> computed = moved * other + 1.0f;
        expect(computed.device() == &gpu, "an expression of device arrays lives on the device");
        expect(bitwise(computed, expected), "device expression = host expression, bit for bit");
        const double on_device = sci::sum(moved), on_host = sci::sum(first);
        expect(std::abs(on_device - on_host) <= 1e-6 * std::abs(on_host), "sum on the device = sum on the host");
    }

    // test_binary.cpp:29-50
    {
        constexpr std::size_t count = 300'000;
        const sci::Array<float, 1> first = sci::linspace(-3.0f, 5.0f, count);
        const sci::Array<float, 1> second = sci::linspace(2.0f, 7.0f, count);
        const auto a = first.to(gpu);
        const auto b = second.to(gpu);
        expect(bitwise(sci::Array<float, 1>(sci::add(a, b)), sci::Array<float, 1>(sci::add(first, second))), "add");
        expect(bitwise(sci::Array<float, 1>(sci::subtract(a, b)), sci::Array<float, 1>(sci::subtract(first, second))),
               "subtract");
        expect(bitwise(sci::Array<float, 1>(sci::multiply(a, b)), sci::Array<float, 1>(sci::multiply(first, second))),
               "multiply");
        expect(bitwise(sci::Array<float, 1>(sci::divide(a, b)), sci::Array<float, 1>(sci::divide(first, second))),
               "divide");
        expect(bitwise(sci::Array<float, 1>(sci::minimum(a, b)), sci::Array<float, 1>(sci::minimum(first, second))),
               "minimum");
        expect(bitwise(sci::Array<float, 1>(sci::maximum(a, b)), sci::Array<float, 1>(sci::maximum(first, second))),
               "maximum");
        expect(bitwise(sci::Array<float, 1>(a + 2.0f), sci::Array<float, 1>(first + 2.0f)), "a scalar on the right");
        expect(bitwise(sci::Array<float, 1>(2.0f * a), sci::Array<float, 1>(2.0f * first)), "and on the left");
        const sci::Array<float, 1> fused = a * b + a;
        const sci::Array<float, 1> read = fused.host();
        bool rounds_once = true;
        for (std::size_t i = 0; i < count; ++i)
            rounds_once = rounds_once && same_bits(read.data()[i], std::fma(first.data()[i], second.data()[i], first.data()[i]));
        expect(rounds_once, "a multiply-add is fused into one rounding (std::fma)");
        const sci::Array<float, 1> nan = sci::Array<float, 1>(sci::Shape<1>{4}, std::nanf("")).to(gpu);
        const sci::Array<float, 1> one = sci::Array<float, 1>(sci::Shape<1>{4}, 1.0f).to(gpu);
        const sci::Array<float, 1> lowest = sci::minimum(nan, one);
        const sci::Array<float, 1> highest = sci::maximum(one, nan);
        const sci::Array<float, 1> low_read = lowest.host(), high_read = highest.host();
        bool nan_wins = true;
        for (std::size_t i = 0; i < 4; ++i) nan_wins = nan_wins && std::isnan(low_read[i]) && std::isnan(high_read[i]);
        expect(nan_wins, "NaN wins a minimum and a maximum");
    }

    // test_unary.cpp: the vector functions bit for bit, the C-library ones within 2 ulp
    {
        const sci::Array<float, 1> x = seeded<float>(1'000'003, 1, -20.0, 20.0);
        const sci::Array<float, 1> positive = seeded<float>(1'000'003, 2, 1e-3, 1e3);
        const sci::Array<float, 1> unit = seeded<float>(1'000'003, 3, -0.99, 0.99);
        const auto dx = x.to(gpu), dp = positive.to(gpu), du = unit.to(gpu);
        expect(bitwise(sci::Array<float, 1>(sci::exponential(dx)), sci::Array<float, 1>(sci::exponential(x))), "exponential");
        expect(bitwise(sci::Array<float, 1>(sci::logarithm(dp)), sci::Array<float, 1>(sci::logarithm(positive))), "logarithm");
        expect(bitwise(sci::Array<float, 1>(sci::sin(dx)), sci::Array<float, 1>(sci::sin(x))), "sin");
        expect(bitwise(sci::Array<float, 1>(sci::cos(dx)), sci::Array<float, 1>(sci::cos(x))), "cos");
        expect(bitwise(sci::Array<float, 1>(sci::root(dp)), sci::Array<float, 1>(sci::root(positive))), "root");
        expect(bitwise(sci::Array<float, 1>(sci::absolute(dx)), sci::Array<float, 1>(sci::absolute(x))), "absolute");
        expect(bitwise(sci::Array<float, 1>(-dx), sci::Array<float, 1>(-x)), "negate");
        auto within = [](const sci::Array<float, 1> &device_result, const sci::Array<float, 1> &host_result,
                         const int64_t bound) {
            const sci::Array<float, 1> read = device_result.host();
            for (std::size_t i = 0; i < read.size(); ++i)
                if (ulps(read.data()[i], host_result.data()[i]) > bound) return false;
            return true;
        };
        expect(within(sci::tanh(du), sci::tanh(unit), 2), "tanh within 2 ulp of the C library");
        expect(within(sci::asin(du), sci::asin(unit), 2), "asin within 2 ulp");
        expect(within(sci::atan(dx), sci::atan(x), 2), "atan within 2 ulp");
        expect(within(sci::sinh(du), sci::sinh(unit), 2), "sinh within 2 ulp");
    }

    // test_reduce.cpp
    {
        const sci::Array<float, 1> x = seeded<float>(4'000'037, 4, -1.0, 1.0);
        const sci::Array<float, 1> z = seeded<float>(4'000'037, 5, 0.5, 2.0);
        const auto dx = x.to(gpu), dz = z.to(gpu);
        double folded = 0.0;
        float low = x.data()[0], high = x.data()[0];
        for (std::size_t i = 0; i < x.size(); ++i) {
            const float v = std::fma(x.data()[i], z.data()[i], 0.5f);
            folded += v;
            (void)v;
        }
        for (std::size_t i = 0; i < x.size(); ++i) {
            low = std::min(low, x.data()[i]);
            high = std::max(high, x.data()[i]);
        }
        const double total = sci::sum(dx * dz + 0.5f);
        expect(std::abs(total - folded) <= 1e-6 * std::abs(folded), "sum of a fused expression");
        expect(sci::minimum(dx) == low && sci::maximum(dx) == high, "minimum and maximum exact");
        expect(std::abs(double(sci::mean(dz)) - double(sci::mean(z))) <= 1e-6, "mean");
        expect(std::abs(double(sci::dot(dx, dz)) - double(sci::dot(x, z))) <= 1e-4 * std::abs(double(sci::dot(x, z))) + 1e-3,
               "dot (contracted: the products are never stored)");
    }

    // test_product.cpp:8-33, then an FP32-accurate product against the host's
    {
        constexpr std::size_t rows = 37, inner = 53, columns = 29;
        sci::Array<float, 2> left(sci::Shape<2>{rows, inner});
        sci::Array<float, 2> right(sci::Shape<2>{inner, columns});
        for (std::size_t r = 0; r < rows; ++r)
            for (std::size_t c = 0; c < inner; ++c) left.data()[r * inner + c] = float((r * 7 + c * 3) % 11) - 5.0f;
        for (std::size_t r = 0; r < inner; ++r)
            for (std::size_t c = 0; c < columns; ++c) right.data()[r * columns + c] = float((r * 5 + c) % 13) * 0.25f;
        const sci::Array<float, 2> computed = sci::product(left.to(gpu), right.to(gpu));
        expect(computed.device() == &gpu, "the product lives on the device");
        const sci::Array<float, 2> read = computed.host();
        bool close = true;
        for (std::size_t r = 0; r < rows; ++r)
            for (std::size_t c = 0; c < columns; ++c) {
                double want = 0.0;
                for (std::size_t k = 0; k < inner; ++k)
                    want += double(left.data()[r * inner + k]) * double(right.data()[k * columns + c]);
                close = close && std::abs(read.data()[r * columns + c] - want) < 1e-3;
            }
        expect(close, "37 x 53 x 29 product within 1e-3 of a double loop");

        constexpr std::size_t m = 300, k = 700, n = 250;
        const sci::Array<float, 1> a_flat = seeded<float>(m * k, 6, -1.0, 1.0);
        const sci::Array<float, 1> b_flat = seeded<float>(k * n, 7, -1.0, 1.0);
        sci::Array<float, 2> a(sci::Shape<2>{m, k}), b(sci::Shape<2>{k, n});
        std::memcpy(a.data(), a_flat.data(), m * k * sizeof(float));
        std::memcpy(b.data(), b_flat.data(), k * n * sizeof(float));
        const sci::Array<float, 2> host_product = sci::product(a, b);
        const sci::Array<float, 2> device_product = sci::product(a.to(gpu), b.to(gpu)).host();
        bool fp32_accurate = true;
        for (std::size_t r = 0; r < m; ++r)
            for (std::size_t c = 0; c < n; ++c) {
                double scale = 0.0;
                for (std::size_t j = 0; j < k; ++j) scale += std::abs(double(a.data()[r * k + j]) * b.data()[j * n + c]);
                // both within k 2^-23 scale of the exact product
                fp32_accurate = fp32_accurate && std::abs(double(device_product.data()[r * n + c]) -
                                                          host_product.data()[r * n + c]) <= 2.0 * k * std::ldexp(scale, -23);
            }
        expect(fp32_accurate, "float product keeps FP32 accuracy (the default mode)");
    }

    // test_solve.cpp:8-25 and test_decompose.cpp:21-36 through sci::linear::cuda
    {
        const sci::Array<double, 2> matrix(sci::Shape<2>{3, 3}, {4, -2, 1, -2, 4, -2, 1, -2, 4});
        const sci::Array<double, 1> right(sci::Shape<1>{3}, {11, -16, 17});
        const auto dm = matrix.to(gpu);
        const sci::Array<double, 1> solution = sci::linear::cuda::solve(dm, right.to(gpu));
        expect(solution.device() == &gpu, "the solution lives where the matrix does");
        const sci::Array<double, 1> x = solution.host();
        bool solved = true;
        for (std::size_t r = 0; r < 3; ++r) {
            double total = 0.0;
            for (std::size_t c = 0; c < 3; ++c) total += matrix.data()[r * 3 + c] * x[c];
            solved = solved && std::abs(total - right[r]) < 1e-9;
        }
        expect(solved, "a vector is solved for");
        const sci::Array<double, 2> several(sci::Shape<2>{3, 2}, {11, 1, -16, 0, 17, 2});
        const sci::Array<double, 2> xs = sci::linear::cuda::solve(dm, several).host();
        bool every = true;
        for (std::size_t r = 0; r < 3; ++r)
            for (std::size_t c = 0; c < 2; ++c) {
                double total = 0.0;
                for (std::size_t j = 0; j < 3; ++j) total += matrix.data()[r * 3 + j] * xs.data()[j * 2 + c];
                every = every && std::abs(total - several.data()[r * 2 + c]) < 1e-9;
            }
        expect(every, "and every column of a matrix (right-hand side on the host, moved first)");

        const sci::Array<double, 2> pivoted(sci::Shape<2>{3, 3}, {0, 2, 1, 4, 1, 3, 2, 5, 7});
        const auto factors = sci::linear::cuda::decompose(pivoted.to(gpu));
        const auto reference = sci::linear::decompose(pivoted);
        expect(factors.permutation.device() == &gpu, "the factors live on the device");
        expect(bitwise(factors.permutation, reference.permutation), "the zero first pivot: P equals the host's");
        const auto lower = factors.lower.host(), upper = factors.upper.host();
        bool close = true;
        for (std::size_t i = 0; i < 9; ++i)
            close = close && std::abs(lower.data()[i] - reference.lower.data()[i]) < 1e-12 &&
                    std::abs(upper.data()[i] - reference.upper.data()[i]) < 1e-12;
        expect(close, "L and U equal the host's");

        constexpr std::size_t order = 512, width = 16;
        std::mt19937_64 engine(11);
        std::normal_distribution<double> normal;
        sci::Array<double, 2> big(sci::Shape<2>{order, order}), rhs(sci::Shape<2>{order, width});
        for (std::size_t i = 0; i < order * order; ++i) big.data()[i] = normal(engine) + (i % (order + 1) == 0 ? order : 0.0);
        for (std::size_t i = 0; i < order * width; ++i) rhs.data()[i] = normal(engine);
        sci_solve_report report{};
        const sci::Array<double, 2> refined = sci::linear::cuda::solve(big.to(gpu), rhs.to(gpu), SCI_REFINE_FP64, &report).host();
        const sci::Array<double, 2> plain = sci::linear::solve(big, rhs);
        double largest = 0.0, gap = 0.0;
        for (std::size_t i = 0; i < order * width; ++i) {
            largest = std::max(largest, std::abs(plain.data()[i]));
            gap = std::max(gap, std::abs(refined.data()[i] - plain.data()[i]));
        }
        expect(report.backward_error <= 1e-14 && report.iterations >= 1, "FP32 LU + FP64 refinement: backward error <= 1e-14");
        expect(gap <= 1e-10 * largest, "refined solution = the host's solve<double>");

        sci::Array<float, 2> square(sci::Shape<2>{256, 256});
        for (std::size_t i = 0; i < 256 * 256; ++i) square.data()[i] = static_cast<float>(normal(engine));
        sci::Array<float, 2> on_device = square.to(gpu);
        const std::vector<sci::core::size> rows = sci::linear::cuda::factor(on_device, SCI_FACTOR_PLAIN);
        sci::Array<float, 2> on_host = square.host();
        std::vector<sci::core::size> host_rows(256);
        sci::linear::factor(on_host.data(), host_rows.data(), 256);
        expect(rows == host_rows, "pivot sequence equals the host's factor<float>");
    }

    // double arrays run on the device too
    {
        const sci::Array<double, 1> x = seeded<double>(100'003, 8, -5.0, 5.0);
        const auto dx = x.to(gpu);
        expect(bitwise(sci::Array<double, 1>(dx * dx + 3.0), sci::Array<double, 1>(x * x + 3.0)), "double fma on the device");
        expect(bitwise(sci::Array<double, 1>(sci::exponential(dx)), sci::Array<double, 1>(sci::exponential(x))),
               "double exponential on the device");
    }

    // no CPU fallback: a host operand in a device expression is an error, not a silent CPU run
    {
        const sci::Array<float, 1> host_array = sci::linspace(0.0f, 1.0f, 1000);
        const auto device_array = host_array.to(gpu);
        bool threw = false;
        try {
            const sci::Array<float, 1> mixed = device_array * host_array;
            (void)mixed;
        } catch (const std::runtime_error &) {
            threw = true;
        }
        expect(threw, "a host operand on the CUDA device is refused");
    }

    std::printf("%s: %d failure(s)\n", failures ? "FAILED" : "PASSED", failures);
    return failures ? 1 : 0;
}
