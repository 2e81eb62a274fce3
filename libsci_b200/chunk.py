"""Chunk bytecode and the expression recorder, mirroring libsci's front end.

libsci never computes ``a * b + c`` eagerly: the expression tree records itself into a
fixed-capacity bytecode ``Chunk`` (include/core/bytecode/chunk.hpp:78-282) and the chunk runs
in one pass. This module restates that recorder so that host code in Python produces the very
bytecode the C++ templates produce:

- ``Chunk.input`` / ``Chunk.constant`` deduplicate by pointer / by the bits of the double
  (chunk.hpp:90-110);
- ``Chunk.emit`` tries the multiply-add contraction on the *second* operand first, then the
  first (chunk.hpp:119-126, 253-261), releases consumed temporaries and takes the lowest free
  temporary as the target (chunk.hpp:128-143);
- ``Chunk.output`` retargets the last instruction to the output slot or appends a copy
  (chunk.hpp:148-160); ``Chunk.reduce`` only records the result value (chunk.hpp:165-168);
- ``Chunk.contracted`` marks sum(... * ...) as a dot product (chunk.hpp:201-204).

Expression nodes record children left to right, then emit their code (include/array/node.hpp:75-88);
a scalar operand becomes a constant of the array's element type (include/array/expression.hpp:88-104,
include/array/literal.hpp:34-36). ``Chunk`` is also the ctypes mirror of ``sci_chunk`` in
include/sci_cuda.h, so a recorded chunk is passed to the C ABI as is.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

CAPACITY = 64

# value ids (instruction.hpp:12-25)
INPUT, LITERAL, TEMPORARY, OUTPUT, NONE, TYPES = 0x00, 0x40, 0x80, 0xC0, 0xFF, 0xC0

# codes, in core::Code order (code.hpp:18-61)
CODES = [
    "copy", "negate", "absolute",
    "root", "exponential", "logarithm",
    "sin", "cos", "tan", "asin", "acos", "atan", "csc", "sec", "cot", "acsc", "asec", "acot",
    "sinh", "cosh", "tanh", "asinh", "acosh", "atanh", "csch", "sech", "coth", "acsch", "asech", "acoth",
    "add", "subtract", "multiply", "divide", "minimum", "maximum", "fuse",
]
CODE = {name: index for index, name in enumerate(CODES)}
UNARY = CODES[: CODE["add"]]
BINARY = ["add", "subtract", "multiply", "divide", "minimum", "maximum"]

SUM, MINIMUM, MAXIMUM = 0, 1, 2  # fold.hpp:11
SINGLE, WIDE = 0, 1  # precision.hpp:12

# codes beyond core::Code for sci_cuda_broadcast (libsci's roadmap functions, README.md:149-152),
# and the mean fold of sci_cuda_reduce_axis
EXTRA = {"floor": 64, "ceil": 65, "round": 66, "power": 67, "clip": 68, "where": 69}
AXIS_MEAN = 3

# element types of sci_cuda_execute_elements / sci_cuda_reduce_elements (SCI_ELEMENT_*): float and
# double are libsci's native types (traits.hpp:26); the integer types run the same bytecode with
# array::calculate's scalar semantics (calculate.hpp:17-93).
ELEMENT = {np.dtype(t): code for code, t in enumerate(
    [np.float32, np.float64, np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64])}


class Instruction(ctypes.Structure):
    """core::Instruction (instruction.hpp:28-35)."""

    _fields_ = [("code", ctypes.c_uint8), ("target", ctypes.c_uint8), ("sources", ctypes.c_uint8 * 3)]


class ChunkStruct(ctypes.Structure):
    """sci_chunk: the public state of core::Chunk (chunk.hpp:228-246)."""

    _fields_ = [
        ("precision", ctypes.c_uint8),
        ("length", ctypes.c_uint8),
        ("arguments", ctypes.c_uint8),
        ("literals", ctypes.c_uint8),
        ("temporaries", ctypes.c_uint8),
        ("result", ctypes.c_uint8),
        ("instructions", Instruction * CAPACITY),
        ("inputs", ctypes.c_void_p * CAPACITY),
        ("constants", ctypes.c_double * CAPACITY),
    ]


class Chunk(ChunkStruct):
    """A chunk being recorded; the recording rules follow chunk.hpp line by line (see module doc)."""

    def __init__(self, precision: int = SINGLE, element: int | None = None):
        super().__init__()
        self.precision = precision
        # SCI_ELEMENT_* of the arrays the chunk reads (not part of the C struct): the float kernels
        # take only float / double chunks, the element kernels any
        self.element = precision if element is None else element
        self.result = NONE
        self._busy = 0
        self._overflow = False

    # -- recording (chunk.hpp:90-168) ------------------------------------------------------------
    def input(self, pointer: int) -> int:
        for index in range(self.arguments):
            if self.inputs[index] == pointer:
                return INPUT | index
        if self.arguments == CAPACITY:
            return self._fail()
        self.inputs[self.arguments] = pointer
        self.arguments += 1
        return INPUT | (self.arguments - 1)

    def constant(self, value: float) -> int:
        key = struct.pack("<d", float(value))
        for index in range(self.literals):
            if struct.pack("<d", self.constants[index]) == key:
                return LITERAL | index
        if self.literals == CAPACITY:
            return self._fail()
        self.constants[self.literals] = float(value)
        self.literals += 1
        return LITERAL | (self.literals - 1)

    def emit(self, code: int, first: int, second: int = NONE, third: int = NONE) -> int:
        if self._overflow:
            return NONE
        if code == CODE["add"]:
            merged = self._contract(second, first)
            if merged != NONE:
                return merged
            merged = self._contract(first, second)
            if merged != NONE:
                return merged
        if self.length == CAPACITY:
            return self._fail()
        for value in (first, second, third):
            self._release(value)
        if self._busy == (1 << 64) - 1:
            return self._fail()
        index = 0
        while self._busy >> index & 1:
            index += 1
        self._busy |= 1 << index
        self.temporaries = max(self.temporaries, index + 1)
        target = TEMPORARY | index
        ins = self.instructions[self.length]
        ins.code, ins.target = code, target
        ins.sources[0], ins.sources[1], ins.sources[2] = first, second, third
        self.length += 1
        return target

    def output(self, value: int) -> "Chunk":
        if self._overflow:
            return self
        last = self.instructions[self.length - 1] if self.length > 0 else None
        if last is not None and last.target == value and (value & TYPES) == TEMPORARY:
            last.target = OUTPUT
        elif self.length < CAPACITY:
            ins = self.instructions[self.length]
            ins.code, ins.target = CODE["copy"], OUTPUT
            ins.sources[0], ins.sources[1], ins.sources[2] = value, NONE, NONE
            self.length += 1
        else:
            self._fail()
        self.result = OUTPUT
        return self

    def reduce(self, value: int) -> "Chunk":
        self.result = value
        return self

    def valid(self) -> bool:
        return not self._overflow

    def contracted(self, fold: int) -> bool:
        if fold != SUM or self.length == 0:
            return False
        last = self.instructions[self.length - 1]
        return last.code == CODE["multiply"] and last.target == self.result

    def signature(self) -> bytes:
        """chunk.hpp:209-226: instructions and counts without addresses or constant values."""
        key = bytearray([self.precision, self.arguments, self.literals, self.temporaries, self.result])
        for index in range(self.length):
            ins = self.instructions[index]
            key += bytes([ins.code, ins.target, ins.sources[0], ins.sources[1], ins.sources[2]])
        return bytes(key)

    def listing(self) -> list[tuple[str, int, tuple[int, int, int]]]:
        return [
            (CODES[self.instructions[i].code], self.instructions[i].target, tuple(self.instructions[i].sources))
            for i in range(self.length)
        ]

    # -- private (chunk.hpp:253-276) -------------------------------------------------------------
    def _contract(self, product: int, addend: int) -> int:
        if self.length == 0 or (product & TYPES) != TEMPORARY:
            return NONE
        last = self.instructions[self.length - 1]
        if last.code != CODE["multiply"] or last.target != product:
            return NONE
        last.code = CODE["fuse"]
        last.sources[2] = addend
        self._release(addend)
        return product

    def _release(self, value: int) -> None:
        if (value & TYPES) == TEMPORARY:
            self._busy &= ~(1 << (value & ~TYPES & 0xFF))

    def _fail(self) -> int:
        self._overflow = True
        return NONE


# ---- expression nodes (include/array/node.hpp, reference.hpp, literal.hpp) ---------------------


class Expression:
    """A lazy elementwise expression over arrays of one element type."""

    dtype: np.dtype
    count: int

    def record(self, chunk: Chunk) -> int:  # pragma: no cover - abstract
        raise NotImplementedError

    def leaves(self):  # pragma: no cover - abstract
        raise NotImplementedError

    # operators (expression.hpp:109-152)
    def __add__(self, other):
        return binary("add", self, other)

    def __radd__(self, other):
        return binary("add", other, self)

    def __sub__(self, other):
        return binary("subtract", self, other)

    def __rsub__(self, other):
        return binary("subtract", other, self)

    def __mul__(self, other):
        return binary("multiply", self, other)

    def __rmul__(self, other):
        return binary("multiply", other, self)

    def __truediv__(self, other):
        return binary("divide", self, other)

    def __rtruediv__(self, other):
        return binary("divide", other, self)

    def __neg__(self):
        return unary("negate", self)


class Reference(Expression):
    """An array operand: records its first element's address as an input (reference.hpp:45)."""

    def __init__(self, pointer: int, count: int, dtype, device=None):
        self.pointer = int(pointer)
        self.count = int(count)
        self.dtype = np.dtype(dtype)
        self.device = device  # where the array lives; the first leaf's device runs it (node.hpp:66-70)

    def record(self, chunk: Chunk) -> int:
        return chunk.input(self.pointer)

    def leaves(self):
        return [self]


class Literal(Expression):
    """A scalar operand, converted to the array's element type first (expression.hpp:88-96)."""

    def __init__(self, value: float, dtype):
        self.dtype = np.dtype(dtype)
        self.value = float(self.dtype.type(value))
        self.count = -1

    def record(self, chunk: Chunk) -> int:
        return chunk.constant(self.value)

    def leaves(self):
        return []


class Node(Expression):
    def __init__(self, code: str, children):
        self.code = CODE[code]
        self.children = children
        arrays = [c for c in children if not isinstance(c, Literal)]
        self.dtype = arrays[0].dtype
        self.count = arrays[0].count
        # node.hpp:32-33: every operand has the node's element type (a compile-time error there)
        for other in arrays[1:]:
            if other.dtype != self.dtype:
                raise TypeError(f"operands must share an element type: {self.dtype} and {other.dtype}")

    def record(self, chunk: Chunk) -> int:
        slots = [child.record(chunk) for child in self.children]
        return chunk.emit(self.code, *slots)

    def leaves(self):
        out = []
        for child in self.children:
            out += child.leaves()
        return out


def _operand(item, dtype):
    if isinstance(item, Expression):
        return item
    if hasattr(item, "expression"):
        return item.expression()
    return Literal(item, dtype)


def binary(code: str, left, right) -> Node:
    anchor = left if isinstance(left, Expression) or hasattr(left, "expression") else right
    dtype = _operand(anchor, None).dtype
    return Node(code, [_operand(left, dtype), _operand(right, dtype)])


def unary(code: str, item) -> Node:
    return Node(code, [_operand(item, None)])


def _new_chunk(dtype) -> Chunk:
    dtype = np.dtype(dtype)
    if dtype not in ELEMENT:
        raise TypeError(f"no device chunks over {dtype} elements (float32, float64 and the integer types)")
    return Chunk(WIDE if dtype == np.float64 else SINGLE, ELEMENT[dtype])


def record_output(expression: Expression) -> Chunk:
    """assign(): chunk.output(item.record(chunk)) (expression.hpp:162-163)."""
    chunk = _new_chunk(expression.dtype)
    chunk.output(expression.record(chunk))
    return chunk


def record_reduce(expression: Expression) -> Chunk:
    """reduce(): chunk.reduce(item.record(chunk)) (expression.hpp:194-195)."""
    chunk = _new_chunk(expression.dtype)
    chunk.reduce(expression.record(chunk))
    return chunk


def require_float(chunk) -> None:
    """The float kernels (execute, reduce, gradients, batches) read float or double lanes: a chunk
    recorded over another element type would be read at the wrong width."""
    if getattr(chunk, "element", chunk.precision) not in (SINGLE, WIDE):
        raise TypeError("an integer-element chunk runs through execute_elements / reduce_elements")
