"""The Python chunk recorder emits the bytecode libsci's own expression templates emit (CPU only).

Each named expression is recorded by the reference (oracle/_ref: include/array/node.hpp:75-88 ->
include/core/bytecode/chunk.hpp:90-168) and by libsci_b200.chunk, and the two chunks compared
field by field: counts, result, instructions, constants and which array each input slot holds.
"""
import ctypes

import numpy as np
import pytest

from libsci_b200 import chunk as C


def named(which, a, b, c):
    u = C.unary
    return {
        0: (a * b + c * 2.0, "o"), 1: (u("exponential", a) * 0.5, "o"), 2: (u("sin", a), "r"),
        3: (u("root", u("absolute", a)) * u("logarithm", b) + u("tanh", c), "o"),
        4: (C.binary("minimum", a, c), "o"), 5: (C.binary("maximum", a, c), "o"),
        6: (u("exponential", -a * a), "r"), 7: (u("sin", a) * u("cos", c), "r"), 8: (a * c, "r"),
        9: (u("exponential", -a * a) * u("sin", b) + u("logarithm", 1.0 + c * c), "r"),
        10: (a * b + c, "o"), 11: (u("tanh", a), "r"), 12: (a * b + a, "o"), 13: (2.0 * a, "o"),
        14: (u("cot", a) - u("acoth", b) / u("sech", c), "o"), 15: (a, "o"),
    }[which]


@pytest.mark.parametrize("wide", [0, 1])
@pytest.mark.parametrize("which", range(16))
def test_recorder_matches_the_reference(reference, which, wide):
    dtype = np.float64 if wide else np.float32
    a, b, c = (C.Reference(p, 1, dtype) for p in (1, 2, 3))
    expr, kind = named(which, a, b, c)
    mine = C.record_output(expr) if kind == "o" else C.record_reduce(expr)
    theirs = C.ChunkStruct()
    assert reference.sci_ref_record(which, wide, ctypes.byref(theirs)) == 0
    for field in ("precision", "length", "arguments", "literals", "temporaries", "result"):
        assert getattr(mine, field) == getattr(theirs, field), field
    for i in range(mine.length):
        assert bytes(mine.instructions[i]) == bytes(theirs.instructions[i]), i
    assert [mine.constants[i] for i in range(mine.literals)] == [theirs.constants[i] for i in range(theirs.literals)]
    assert [mine.inputs[i] - 1 for i in range(mine.arguments)] == [(theirs.inputs[i] or 0) for i in range(theirs.arguments)]


def test_recorder_rules():
    a, b, c = (C.Reference(p, 8, np.float32) for p in (1, 2, 3))
    # the second operand's product fuses first (chunk.hpp:123-126): c*2 + a*b -> fma(a, b, t(c*2))
    chunk = C.record_output(c * 2.0 + a * b)
    assert [n for n, _, _ in chunk.listing()] == ["multiply", "fuse"]
    # sum(x*y) is contracted; max(x*y) is not
    assert C.record_reduce(a * b).contracted(C.SUM)
    assert not C.record_reduce(a * b).contracted(C.MAXIMUM)
    # inputs and constants are deduplicated
    chunk = C.record_output(a * a + 2.0 * a + 2.0)
    assert chunk.arguments == 1 and chunk.literals == 1
    # an expression that outgrows 64 entries is flagged, as Chunk::valid() (chunk.hpp:172)
    e = a
    for k in range(70):
        e = e + float(k)
    assert not C.record_output(e).valid()


def test_operands_must_share_an_element_type():
    # node.hpp:32-33 rejects a node over arrays of different element types at compile time; the
    # recorder raises instead of recording one of them under the other's type
    a = C.Reference(16, 8, np.float32)
    b = C.Reference(32, 8, np.int32)
    with pytest.raises(TypeError):
        C.binary("add", a, b)
    assert C.binary("add", a, 2).dtype == np.float32  # a literal takes the array's type


def test_unsupported_and_integer_chunks_stay_off_the_float_kernels():
    # a float16 or bool array has no device chunk; an integer chunk is refused by the float entry
    # points (which would read its lanes at the float width) before anything launches
    with pytest.raises(TypeError):
        C.record_output(C.Reference(16, 8, np.float16) * 2)
    with pytest.raises(TypeError):
        C.record_reduce(C.Reference(16, 8, np.bool_) + 1)
    integer = C.record_output(C.Reference(16, 8, np.int8) * 2)
    assert integer.element == C.ELEMENT[np.dtype(np.int8)]
    with pytest.raises(TypeError):
        C.require_float(integer)
    C.require_float(C.record_output(C.Reference(16, 8, np.float64) * 2))
