// Oracle build shim (test infrastructure only).
//
// include/core/drivers/processor/compiler.hpp:11,59 hold a std::optional<asmjit::JitRuntime>.
// The oracle build replaces the CPU JIT with a stub whose compile() always returns null (the
// same as SCI_JIT=0, and what the reference does on an AVX-512 table anyway:
// src/core/drivers/processor/compiler.cpp:41-46), so only complete, empty types are needed.
#pragma once
namespace asmjit {
    class JitRuntime {};
    class CodeHolder {};
}
