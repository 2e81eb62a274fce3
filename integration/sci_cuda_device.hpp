#pragma once

// The CUDA side of libsci's Device, for code built against libsci's headers with the B200 backend
// (integration/device.cpp). Two things the reference's Device interface (device.hpp:27-89) cannot
// say by itself:
//
//  - cuda_context(device): the libsci_cuda.so context behind a Device opened on a CUDA GPU (null
//    for a CPU device), so free functions can reach entry points Device has no method for;
//  - sci::linear::cuda::{factor, solve, decompose}: linear::factor / solve / decompose
//    (include/linear/decompose.hpp:29-103, solve.hpp:60-76) on arrays that live on a CUDA device,
//    where the reference always copies to the host and factors there (solve.hpp:68-75). Arrays on
//    the host, or on a device without CUDA, take the reference's own functions.

#include "array/array.hpp"
#include "core/drivers/device.hpp"
#include "linear/decompose.hpp"
#include "linear/factors.hpp"
#include "linear/solve.hpp"
#include "sci_cuda.h"

#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace sci::core::drivers {

    /// The CUDA target. libsci's Target (include/core/drivers/target.hpp:11) is
    /// `enum class Target : uint8 { processor, graphics }`; the backend's change to that line appends
    /// `cuda`, value 2. A build that keeps the reference's headers unchanged, like this one, names
    /// the same value here: Device(cuda_target) is Device(Target::cuda).
    inline constexpr Target cuda_target = static_cast<Target>(2);

    /// The libsci_cuda.so context of a Device opened on a CUDA GPU; null for a CPU device (or none).
    sci_cuda_context *cuda_context(const Device *device) noexcept;

    /// Throws std::runtime_error with the context's last message when `status` is not SCI_CUDA_OK.
    void cuda_must(sci_cuda_context *context, int status, const char *what);

}

namespace sci::linear::cuda {

    using array::Array;
    using array::Shape;

    template <typename element> constexpr uint32_t precision_of() {
        static_assert(std::is_same_v<element, float> || std::is_same_v<element, double>,
                      "the CUDA linear algebra takes float or double");
        return std::is_same_v<element, double> ? SCI_PRECISION_WIDE : SCI_PRECISION_SINGLE;
    }

    /// linear::factor on a CUDA array, in place: returns rows[] (the original row now at each
    /// position), with the reference's pivot rule (first strictly largest |a|, zero pivot skipped).
    /// `mode` SCI_FACTOR_TENSOR runs float trailing updates on the tensor cores; SCI_FACTOR_PLAIN
    /// keeps the element type throughout.
    template <typename element>
    std::vector<core::size> factor(Array<element, 2> &matrix, const uint32_t mode = SCI_FACTOR_TENSOR) {
        const core::size order = matrix.shape()[0];
        ASSERT(order == matrix.shape()[1]);
        sci_cuda_context *context = core::drivers::cuda_context(matrix.device());
        std::vector<core::size> rows(order);
        if (context == nullptr) {
            matrix.device() ? matrix.device()->synchronize() : void();
            linear::factor(matrix.data(), rows.data(), order);
            return rows;
        }
        std::vector<uint64_t> order_out(order);
        core::drivers::cuda_must(context, sci_cuda_factor(context, precision_of<element>(), mode, matrix.data(),
                                                          order_out.data(), order),
                                 "factor");
        for (core::size i = 0; i < order; ++i) rows[i] = static_cast<core::size>(order_out[i]);
        return rows;
    }

    /// linear::solve on CUDA arrays: the result has right's shape and lives where the matrix does.
    /// Double systems factor in FP32 and refine in FP64 to a normwise backward error <= 1e-14 unless
    /// `refine` is SCI_REFINE_NONE (the reference's behaviour: factor and substitute in the element
    /// type). `report`, when given, receives the backward error and the refinement steps.
    template <typename element, core::size rank>
        requires(rank == 1 || rank == 2)
    Array<element, rank> solve(const Array<element, 2> &matrix, const Array<element, rank> &right,
                               const uint32_t refine = std::is_same_v<element, double> ? SCI_REFINE_FP64 : SCI_REFINE_NONE,
                               sci_solve_report *report = nullptr) {
        core::drivers::Device *device = matrix.device();
        sci_cuda_context *context = core::drivers::cuda_context(device);
        if (context == nullptr) return linear::solve(matrix, right);
        const core::size order = right.shape()[0];
        const core::size width = rank == 1 ? 1 : right.shape()[rank - 1];
        ASSERT(matrix.shape()[0] == order && matrix.shape()[1] == order);
        // the right-hand side on the matrix's device (the caller's other device finishes first)
        const Array<element, rank> moved = right.device() == device ? Array<element, rank>() : right.to(*device);
        const Array<element, rank> &operand = right.device() == device ? right : moved;
        Array<element, rank> solution(*device, right.shape(), array::Uninitialized{});
        core::drivers::cuda_must(context, sci_cuda_solve(context, precision_of<element>(), refine, matrix.data(),
                                                         operand.data(), solution.data(), order, width, report),
                                 "solve");
        return solution;
    }

    /// linear::decompose on a CUDA array: P, L, U made on the device (the reference factors on the
    /// host and copies three dense matrices up, decompose.hpp:77-103).
    template <typename element>
    Factors<element> decompose(const Array<element, 2> &matrix, const uint32_t mode = SCI_FACTOR_PLAIN) {
        core::drivers::Device *device = matrix.device();
        sci_cuda_context *context = core::drivers::cuda_context(device);
        if (context == nullptr) return linear::decompose(matrix);
        const core::size order = matrix.shape()[0];
        ASSERT(order == matrix.shape()[1]);
        Factors<element> out{Array<element, 2>(*device, Shape<2>{order, order}, array::Uninitialized{}),
                             Array<element, 2>(*device, Shape<2>{order, order}, array::Uninitialized{}),
                             Array<element, 2>(*device, Shape<2>{order, order}, array::Uninitialized{})};
        core::drivers::cuda_must(context, sci_cuda_decompose(context, precision_of<element>(), mode, matrix.data(),
                                                             out.permutation.data(), out.lower.data(), out.upper.data(),
                                                             order),
                                 "decompose");
        return out;
    }

}
