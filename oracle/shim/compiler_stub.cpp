// Oracle build stub (test infrastructure only): stands in for
// src/core/drivers/processor/compiler.cpp. compile() returns null, so every chunk runs on the
// kernel tables -- what the reference itself does with the AVX-512 table, whose width() is 0
// (src/core/drivers/processor/compiler.cpp:36-41).
#include "core/drivers/processor/compiler.hpp"

namespace sci::core::drivers::processor {

    Compiler::Compiler() { enabled = false; }

    Compiler &Compiler::global() {
        static Compiler compiler;
        return compiler;
    }

    size Compiler::width(const kernels::Table &, const Precision) noexcept { return 0; }

    Compiler::Function Compiler::compile(const Chunk &, const kernels::Table &, const size) { return nullptr; }

}
