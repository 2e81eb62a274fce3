// Oracle build stub (test infrastructure only): stands in for src/core/drivers/device.cpp with
// a CPU-only Device, the state the reference reaches when no Vulkan device opens
// (src/core/drivers/device.cpp:186-199): every entry point forwards to processor::Dispatch.
#include "core/drivers/device.hpp"
#include "core/alignment.hpp"
#include "core/drivers/processor/dispatch.hpp"

#include <limits>

namespace sci::core::drivers {

    struct Graphics {};

    Device::Device(const Target, const uint32 index) : type(Target::processor), ordinal(index) {}

    Device::~Device() = default;

    const char *Device::name() const noexcept { return "cpu"; }

    void Device::synchronize() noexcept {}

    void Device::allocate(const size bytes, Memory &memory) {
        memory.bytes = bytes;
        memory.target = type;
        memory.allocation = core::memory::Allocation(bytes, alignment::line);
        memory.host = memory.allocation.data();
    }

    void Device::dispose(Memory &memory) noexcept { memory = {}; }

    void Device::execute(const Chunk &chunk, void *output, const size count) {
        if (count == 0) return;
        processor::Dispatch::global().execute(chunk, output, count);
    }

    double Device::reduce(const Chunk &chunk, const Fold fold, const size count) {
        if (count == 0) return fold == Fold::sum ? 0.0 : std::numeric_limits<double>::quiet_NaN();
        return processor::Dispatch::global().reduce(chunk, fold, count);
    }

    void Device::product(const Precision precision, const void *left, const void *right, void *output,
                         const size rows, const size columns, const size depth) {
        if (rows == 0 || columns == 0) return;
        processor::Dispatch::product(precision, left, right, output, rows, columns, depth);
    }

}
