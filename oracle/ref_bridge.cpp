// ref_bridge.cpp -- C entry points into the reference's own CPU path (test infrastructure only).
//
// This file is compiled together with the reference's unchanged CPU sources (see Makefile) into
// oracle/_ref/libsci_ref.so. Tests and the CPU arm of bench.py load it to obtain what libsci
// itself computes: the chunk executor (src/core/drivers/processor/dispatch.cpp:246-265), the
// matrix product (dispatch.cpp:267-301), LU and substitution (include/linear/decompose.hpp:29-72,
// include/linear/solve.hpp:25-52) and the expression recorder (include/array/node.hpp:75-88,
// include/core/bytecode/chunk.hpp:90-168). Nothing in the product links it.
#include <sci.hpp>

#include "core/drivers/processor/dispatch.hpp"
#include "core/drivers/processor/pool.hpp"

#include "../include/sci_cuda.h"

#include <cstring>
#include <vector>

using sci::core::Chunk;
using sci::core::Code;
using sci::core::Fold;
using sci::core::Instruction;
using sci::core::Precision;
using sci::core::drivers::processor::Dispatch;

namespace {

    // Rebuilds the reference's Chunk from its C mirror, field for field (chunk.hpp:228-246).
    Chunk rebuild(const sci_chunk &source) {
        Chunk chunk(source.precision == SCI_PRECISION_WIDE ? Precision::wide : Precision::single);
        chunk.length = source.length;
        chunk.arguments = source.arguments;
        chunk.literals = source.literals;
        chunk.temporaries = source.temporaries;
        chunk.result = source.result;
        for (int index = 0; index < source.length; ++index) {
            const sci_instruction &step = source.instructions[index];
            chunk.instructions[index] = Instruction{.code = static_cast<Code>(step.code),
                                                    .target = step.target,
                                                    .sources = {step.sources[0], step.sources[1], step.sources[2]}};
        }
        for (int index = 0; index < source.arguments; ++index) chunk.inputs[index] = source.inputs[index];
        for (int index = 0; index < source.literals; ++index) chunk.constants[index] = source.constants[index];
        return chunk;
    }

    // Copies a recorded Chunk back into the C mirror; inputs are replaced by which named array
    // (0, 1, 2 for the first, second, third operand array) each slot refers to.
    void export_chunk(const Chunk &chunk, const void *const *arrays, sci_chunk &out) {
        std::memset(&out, 0, sizeof(out));
        out.precision = chunk.precision == Precision::wide ? SCI_PRECISION_WIDE : SCI_PRECISION_SINGLE;
        out.length = chunk.length;
        out.arguments = chunk.arguments;
        out.literals = chunk.literals;
        out.temporaries = chunk.temporaries;
        out.result = chunk.result;
        for (int index = 0; index < chunk.length; ++index) {
            const Instruction &step = chunk.instructions[index];
            out.instructions[index] = sci_instruction{static_cast<uint8_t>(step.code), step.target,
                                                      {step.sources[0], step.sources[1], step.sources[2]}};
        }
        for (int index = 0; index < chunk.arguments; ++index) {
            std::uintptr_t which = 255;
            for (std::uintptr_t name = 0; name < 3; ++name) {
                if (chunk.inputs[index] == arrays[name]) which = name;
            }
            out.inputs[index] = reinterpret_cast<const void *>(which);
        }
        for (int index = 0; index < chunk.literals; ++index) out.constants[index] = chunk.constants[index];
    }

    template <typename item> void finish_output(Chunk &chunk, const item &expression) {
        chunk.output(sci::array::capture(expression).record(chunk));
    }

    template <typename item> void finish_reduce(Chunk &chunk, const item &expression) {
        chunk.reduce(sci::array::capture(expression).record(chunk));
    }

} // namespace

extern "C" {

// Dispatch::execute (dispatch.cpp:246-254).
int sci_ref_execute(const sci_chunk *chunk, void *output, const uint64_t count) {
    if (!chunk) return 1;
    const Chunk rebuilt = rebuild(*chunk);
    if (count == 0) return 0;
    Dispatch::global().execute(rebuilt, output, count);
    return 0;
}

// Dispatch::reduce (dispatch.cpp:256-265); empty input gives 0 for sum, NaN otherwise
// (dispatch.cpp:109-111).
double sci_ref_reduce(const sci_chunk *chunk, const uint32_t fold, const uint64_t count) {
    const Chunk rebuilt = rebuild(*chunk);
    return Dispatch::global().reduce(rebuilt, static_cast<Fold>(fold), count);
}

// Dispatch::product (dispatch.cpp:267-301): row-major output = left * right.
void sci_ref_product(const uint32_t precision, const void *left, const void *right, void *output,
                     const uint64_t rows, const uint64_t columns, const uint64_t depth) {
    Dispatch::product(precision == SCI_PRECISION_WIDE ? Precision::wide : Precision::single, left, right, output,
                      rows, columns, depth);
}

// linear::factor (decompose.hpp:29-72): in-place LU with partial pivoting; rows[i] is the
// original row now at position i.
void sci_ref_factor_f32(float *matrix, uint64_t *rows, const uint64_t order) {
    std::vector<sci::core::size> order_rows(order);
    sci::linear::factor(matrix, order_rows.data(), order);
    for (uint64_t index = 0; index < order; ++index) rows[index] = order_rows[index];
}

void sci_ref_factor_f64(double *matrix, uint64_t *rows, const uint64_t order) {
    std::vector<sci::core::size> order_rows(order);
    sci::linear::factor(matrix, order_rows.data(), order);
    for (uint64_t index = 0; index < order; ++index) rows[index] = order_rows[index];
}

// linear::solve (solve.hpp:60-76) on host arrays: factor a copy, then substitute.
void sci_ref_solve_f64(const double *matrix, const double *right, double *solution, const uint64_t order,
                       const uint64_t width) {
    std::vector<double> work(matrix, matrix + order * order);
    std::vector<sci::core::size> rows(order);
    sci::linear::factor(work.data(), rows.data(), order);
    sci::linear::substitute(work.data(), rows.data(), right, solution, order, width);
}

void sci_ref_solve_f32(const float *matrix, const float *right, float *solution, const uint64_t order,
                       const uint64_t width) {
    std::vector<float> work(matrix, matrix + order * order);
    std::vector<sci::core::size> rows(order);
    sci::linear::factor(work.data(), rows.data(), order);
    sci::linear::substitute(work.data(), rows.data(), right, solution, order, width);
}

// Threads the reference's pool runs on (pool.cpp:62-73): every host core unless SCI_THREADS.
uint64_t sci_ref_threads(void) { return sci::core::drivers::processor::Pool::global().width(); }

// Records one of the named expressions the workloads use through the reference's own
// expression templates (include/operations/*.hpp -> node.hpp:75-88 -> chunk.hpp:119-168), so the
// tests can check that a recorder produces the same bytecode. `wide` records it over double
// arrays. Returns 0, or 1 for an unknown name.
int sci_ref_record(const int which, const int wide, sci_chunk *out) {
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        sci::Array<T, 1> first(sci::Shape<1>{1});
        sci::Array<T, 1> second(sci::Shape<1>{1});
        sci::Array<T, 1> third(sci::Shape<1>{1});
        const void *arrays[3] = {first.data(), second.data(), third.data()};
        Chunk chunk(wide ? Precision::wide : Precision::single);
        const auto &a = first;
        const auto &b = second;
        const auto &c = third;
        switch (which) {
        case 0: finish_output(chunk, a * b + c * T(2)); break;                                        // t = a*b + c*2
        case 1: finish_output(chunk, sci::exponential(a) * T(0.5)); break;                            // e = exp(t)*0.5
        case 2: finish_reduce(chunk, sci::sin(a)); break;                                              // sum(sin(t))
        case 3: finish_output(chunk, sci::root(sci::absolute(a)) * sci::logarithm(b) + sci::tanh(c)); break;
        case 4: finish_output(chunk, sci::minimum(a, c)); break;
        case 5: finish_output(chunk, sci::maximum(a, c)); break;
        case 6: finish_reduce(chunk, sci::exponential(-a * a)); break;                                 // mean(exp(-x*x))
        case 7: finish_reduce(chunk, sci::sin(a) * sci::cos(c)); break;                                // max(sin(x)*cos(z))
        case 8: finish_reduce(chunk, a * c); break;                                                    // dot(x, z)
        case 9: finish_reduce(chunk, sci::exponential(-a * a) * sci::sin(b) + sci::logarithm(T(1) + c * c)); break;
        case 10: finish_output(chunk, a * b + c); break;                                               // t = a*b + c
        case 11: finish_reduce(chunk, sci::tanh(a)); break;                                            // sum(tanh(t))
        case 12: finish_output(chunk, a * b + a); break;                                               // fma pin
        case 13: finish_output(chunk, T(2) * a); break;                                                // scalar on the left
        case 14: finish_output(chunk, sci::cot(a) - sci::acoth(b) / sci::sech(c)); break;
        case 15: finish_output(chunk, a); break;                                                       // plain copy
        default: return 1;
        }
        export_chunk(chunk, arrays, *out);
        return chunk.valid() ? 0 : 2;
    };
    return wide ? run(double{}) : run(float{});
}

// The workload of the large fused chunks, run through the reference's public API
// (include/operations/*.hpp): three arrays x, y, z; stores sqrt(|x|)*log(y)+tanh(z), minimum(x,z),
// maximum(x,z); reduces mean(exp(-x*x)), maximum(sin(x)*cos(z)), dot(x,z). Arrays are owned here
// and created once; the step runs the six operations the way a libsci user writes them.
struct sci_ref_workload {
    sci::Array<float, 1> x, y, z, stored, lower, upper;
};

void *sci_ref_workload_create(const float *x, const float *y, const float *z, const uint64_t count) {
    auto *work = new sci_ref_workload{
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
    };
    std::memcpy(work->x.data(), x, count * sizeof(float));
    std::memcpy(work->y.data(), y, count * sizeof(float));
    std::memcpy(work->z.data(), z, count * sizeof(float));
    return work;
}

void sci_ref_workload_step(void *handle, double *reductions) {
    auto &work = *static_cast<sci_ref_workload *>(handle);
    const auto &x = work.x;
    const auto &y = work.y;
    const auto &z = work.z;
    work.stored = sci::root(sci::absolute(x)) * sci::logarithm(y) + sci::tanh(z);
    work.lower = sci::minimum(x, z);
    work.upper = sci::maximum(x, z);
    reductions[0] = sci::mean(sci::exponential(-x * x));
    reductions[1] = sci::maximum(sci::sin(x) * sci::cos(z));
    reductions[2] = sci::dot(x, z);
}

const float *sci_ref_workload_output(void *handle, const int which) {
    auto &work = *static_cast<sci_ref_workload *>(handle);
    return which == 0 ? work.stored.data() : which == 1 ? work.lower.data() : work.upper.data();
}

void sci_ref_workload_destroy(void *handle) { delete static_cast<sci_ref_workload *>(handle); }

// The plain fused expression, run through the reference's public API: a = linspace(0, 1, n),
// b, c given; each step stores t = a*b + c*2.0f and e = exponential(t)*0.5f and reduces
// s = sum(sin(t)), the way a libsci user writes them.
struct sci_ref_plain {
    sci::Array<float, 1> a, b, c, t, e;
};

void *sci_ref_plain_create(const float *b, const float *c, const uint64_t count) {
    auto *work = new sci_ref_plain{
            sci::linspace(0.0f, 1.0f, count),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
            sci::Array<float, 1>(sci::Shape<1>{count}, sci::array::Uninitialized{}),
    };
    std::memcpy(work->b.data(), b, count * sizeof(float));
    std::memcpy(work->c.data(), c, count * sizeof(float));
    return work;
}

double sci_ref_plain_step(void *handle) {
    auto &work = *static_cast<sci_ref_plain *>(handle);
    work.t = work.a * work.b + work.c * 2.0f;
    work.e = sci::exponential(work.t) * 0.5f;
    return sci::sum(sci::sin(work.t));
}

const float *sci_ref_plain_output(void *handle, const int which) {
    auto &work = *static_cast<sci_ref_plain *>(handle);
    return which == 0 ? work.t.data() : which == 1 ? work.e.data() : work.a.data();
}

void sci_ref_plain_destroy(void *handle) { delete static_cast<sci_ref_plain *>(handle); }

// ---- creation: the reference's own functions (include/operations/creation.hpp) -----------------
void sci_ref_full(uint32_t precision, void *out, uint64_t count, double value) {  // creation.hpp:52-58
    if (precision == SCI_PRECISION_WIDE) {
        const auto made = sci::operations::full<double>({count}, value);
        std::memcpy(out, made.data(), count * sizeof(double));
    } else {
        const auto made = sci::operations::full<float>({count}, static_cast<float>(value));
        std::memcpy(out, made.data(), count * sizeof(float));
    }
}

void sci_ref_linspace(uint32_t precision, void *out, uint64_t count, double start, double stop) {  // :66-84
    if (precision == SCI_PRECISION_WIDE) {
        const auto made = sci::operations::linspace<double>(start, stop, count);
        if (count) std::memcpy(out, made.data(), count * sizeof(double));
    } else {
        const auto made = sci::operations::linspace<float>(static_cast<float>(start), static_cast<float>(stop), count);
        if (count) std::memcpy(out, made.data(), count * sizeof(float));
    }
}

// range (creation.hpp:157-168): fills `out` (room for `capacity` values) and returns the count.
uint64_t sci_ref_range(uint32_t precision, void *out, uint64_t capacity, double start, double stop, double step) {
    if (precision == SCI_PRECISION_WIDE) {
        const auto made = sci::operations::range<double>(start, stop, step);
        const uint64_t count = made.shape()[0];
        if (count && count <= capacity) std::memcpy(out, made.data(), count * sizeof(double));
        return count;
    }
    const auto made = sci::operations::range<float>(static_cast<float>(start), static_cast<float>(stop), static_cast<float>(step));
    const uint64_t count = made.shape()[0];
    if (count && count <= capacity) std::memcpy(out, made.data(), count * sizeof(float));
    return count;
}

void sci_ref_eye(uint32_t precision, void *out, uint64_t rows, uint64_t columns) {  // creation.hpp:91-106
    if (precision == SCI_PRECISION_WIDE) {
        const auto made = sci::operations::eye<double>({rows, columns});
        std::memcpy(out, made.data(), rows * columns * sizeof(double));
    } else {
        const auto made = sci::operations::eye<float>({rows, columns});
        std::memcpy(out, made.data(), rows * columns * sizeof(float));
    }
}

// ---- integer elements: the reference's own host loop (expression.hpp:178-184,203-220) ----------
// Named expressions over three arrays of one integer element type, written the way a libsci user
// writes them; the reference evaluates them element by element through array::calculate
// (calculate.hpp:17-93). Evaluations (which < 10) fill `out` with `count` elements; reductions
// (which >= 10) write one element. Returns 1 for an unknown name or element type.
int sci_ref_elements(const int which, const uint32_t element, const void *a, const void *b, const void *c,
                     const uint64_t count, void *out) {
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        sci::Array<T, 1> x(sci::Shape<1>{count}, sci::array::Uninitialized{});
        sci::Array<T, 1> y(sci::Shape<1>{count}, sci::array::Uninitialized{});
        sci::Array<T, 1> z(sci::Shape<1>{count}, sci::array::Uninitialized{});
        sci::Array<T, 1> r(sci::Shape<1>{count}, sci::array::Uninitialized{});
        std::memcpy(x.data(), a, count * sizeof(T));
        std::memcpy(y.data(), b, count * sizeof(T));
        std::memcpy(z.data(), c, count * sizeof(T));
        T folded{};
        switch (which) {
        case 0: r = x * y + z; break;
        case 1: r = -x + y * T(3); break;
        case 2: r = sci::absolute(x) - sci::minimum(y, z); break;
        case 3: r = sci::maximum(x, z) / y; break;
        case 4: r = sci::root(sci::absolute(x)) + y; break;
        case 5: r = sci::atan(x) * y + sci::cos(z); break;
        case 6: r = sci::logarithm(sci::absolute(x) + T(1)) * T(2) - sci::tanh(y); break;
        case 10: folded = sci::sum(x * y); break;
        case 11: folded = sci::minimum(x - z); break;
        case 12: folded = sci::maximum(sci::absolute(y) + x); break;
        case 13: folded = sci::mean(x * y); break;
        default: return 1;
        }
        if (which >= 10) std::memcpy(out, &folded, sizeof(T));
        else std::memcpy(out, r.data(), count * sizeof(T));
        return 0;
    };
    switch (element) {
    case SCI_ELEMENT_INT8: return run(int8_t{});
    case SCI_ELEMENT_INT16: return run(int16_t{});
    case SCI_ELEMENT_INT32: return run(int32_t{});
    case SCI_ELEMENT_INT64: return run(int64_t{});
    case SCI_ELEMENT_UINT8: return run(uint8_t{});
    case SCI_ELEMENT_UINT16: return run(uint16_t{});
    case SCI_ELEMENT_UINT32: return run(uint32_t{});
    case SCI_ELEMENT_UINT64: return run(uint64_t{});
    default: return 1;
    }
}

} // extern "C"
