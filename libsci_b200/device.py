"""Python host layer over the C ABI: a CUDA ``Device`` and arrays that live on it.

Mirrors the parts of libsci's C++ front end that the chunk, product and solve paths use:

- ``Device`` is ``sci::Device`` with a CUDA target (include/core/drivers/device.hpp:27-89):
  ``execute`` / ``reduce`` / ``synchronize`` / ``name`` and memory.
- ``DeviceArray`` is a one-dimensional ``sci::Array`` placed on that device (include/array/array.hpp:
  ``to(device)`` / ``host()`` at :223-237). It records itself into chunks as an input
  (include/array/reference.hpp:45).
- ``evaluate`` is ``assign`` (include/array/expression.hpp:158-185) and ``sum`` / ``mean`` /
  ``minimum`` / ``maximum`` / ``dot`` are the reductions of include/operations/reduce.hpp:19-42 and
  include/linear/product.hpp:72-76, including ``mean`` as ``float(sum) / float(count)`` in the
  element type.

Every call goes through libsci_cuda.so; errors raise ``SciCudaError`` and nothing runs on the CPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import chunk as C
from .native import MEMORY_DEVICE, MEMORY_MANAGED, SciCudaError, check, lib


class Device:
    def __init__(self, ordinal: int = 0):
        handle = ctypes.c_void_p()
        status = lib.sci_cuda_open(ordinal, ctypes.byref(handle))
        if status != 0:
            raise SciCudaError(status, f"cannot open CUDA device {ordinal}")
        self.handle = handle

    # -- lifetime -------------------------------------------------------------------------------
    def close(self) -> None:
        if self.handle:
            check(lib.sci_cuda_close(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def name(self) -> str:
        return lib.sci_cuda_name(self.handle).decode()

    @property
    def stream(self) -> int:
        return lib.sci_cuda_stream(self.handle)

    def synchronize(self) -> None:
        check(lib.sci_cuda_synchronize(self.handle), self.handle)

    def jit_wait(self) -> None:
        """Waits for queued NVRTC specialisations (chunks run on the interpreter until then)."""
        check(lib.sci_cuda_jit_wait(self.handle), self.handle)

    # -- memory ---------------------------------------------------------------------------------
    def allocate(self, nbytes: int, managed: bool = False) -> int:
        pointer = ctypes.c_void_p()
        kind = MEMORY_MANAGED if managed else MEMORY_DEVICE
        check(lib.sci_cuda_allocate(self.handle, nbytes, kind, ctypes.byref(pointer)), self.handle)
        return pointer.value

    def dispose(self, pointer: int) -> None:
        check(lib.sci_cuda_dispose(self.handle, pointer), self.handle)

    def empty(self, count: int, dtype=np.float32) -> "DeviceArray":
        dtype = np.dtype(dtype)
        return DeviceArray(self, self.allocate(max(count, 1) * dtype.itemsize), count, dtype)

    def array(self, values, dtype=None) -> "DeviceArray":
        """Array.to(device): a device copy of host values (array.hpp:223-228)."""
        host = np.ascontiguousarray(values, dtype=dtype)
        out = self.empty(host.size, host.dtype)
        out.upload(host)
        return out

    # -- creation on the device (include/operations/creation.hpp) ---------------------------------
    @staticmethod
    def _precision(dtype) -> int:
        dtype = np.dtype(dtype)
        if dtype == np.float32:
            return C.SINGLE
        if dtype == np.float64:
            return C.WIDE
        raise TypeError(f"device arrays are float32 or float64, not {dtype}")

    def full(self, count: int, value: float, dtype=np.float32) -> "DeviceArray":
        """full (creation.hpp:52-58), filled on the device."""
        out = self.empty(count, dtype)
        check(lib.sci_cuda_fill(self.handle, self._precision(dtype), out.pointer, count, float(value)), self.handle)
        return out

    def zeros(self, count: int, dtype=np.float32) -> "DeviceArray":
        """zeros (creation.hpp:34-38)."""
        return self.full(count, 0.0, dtype)

    def ones(self, count: int, dtype=np.float32) -> "DeviceArray":
        """ones (creation.hpp:44-47)."""
        return self.full(count, 1.0, dtype)

    def linspace(self, start: float, stop: float, count: int, dtype=np.float32) -> "DeviceArray":
        """linspace (creation.hpp:66-84): count values from start to stop, both included."""
        out = self.empty(count, dtype)
        check(lib.sci_cuda_linspace(self.handle, self._precision(dtype), out.pointer, count, float(start), float(stop)),
              self.handle)
        return out

    def range(self, start: float, stop: float | None = None, step: float = 1.0, dtype=np.float32) -> "DeviceArray":
        """range (creation.hpp:157-176, numpy.arange): start, start + step, ... below stop;
        range(stop) counts from 0."""
        if stop is None:
            start, stop = 0.0, start
        precision = self._precision(dtype)
        count = int(lib.sci_cuda_range_count(precision, float(start), float(stop), float(step)))
        out = self.empty(count, dtype)
        check(lib.sci_cuda_range(self.handle, precision, out.pointer, count, float(start), float(step)), self.handle)
        return out

    def eye(self, rows: int, columns: int | None = None, dtype=np.float32) -> "DeviceArray":
        """eye (creation.hpp:91-117): a rows x columns row-major matrix, ones on the diagonal."""
        columns = rows if columns is None else columns
        out = self.empty(rows * columns, dtype)
        check(lib.sci_cuda_eye(self.handle, self._precision(dtype), out.pointer, rows, columns), self.handle)
        return out

    def grid(self, x: "DeviceArray", y: "DeviceArray"):
        """grid (creation.hpp:120-140, numpy.meshgrid): (xx, yy), each len(y) x len(x), row-major."""
        if x.dtype != y.dtype:
            raise TypeError("grid: x and y differ in type")
        xx, yy = self.empty(x.count * y.count, x.dtype), self.empty(x.count * y.count, x.dtype)
        check(lib.sci_cuda_grid(self.handle, self._precision(x.dtype), x.pointer, x.count, y.pointer, y.count,
                                xx.pointer, yy.pointer), self.handle)
        return xx, yy

    def transpose(self, array: "DeviceArray", shape) -> "DeviceArray":
        """transpose (manipulations.hpp:33-62): `array` read with `shape` (row-major), the result
        with the extents reversed."""
        shape = [int(v) for v in shape]
        if int(np.prod(shape)) != array.count:
            raise ValueError("transpose: the shape does not cover the array")
        out = self.empty(array.count, array.dtype)
        extents = (ctypes.c_uint64 * len(shape))(*shape)
        check(lib.sci_cuda_transpose(self.handle, self._precision(array.dtype), array.pointer, len(shape), extents,
                                     out.pointer), self.handle)
        return out

    def decompose(self, matrix: "DeviceArray", order: int, plain: bool = False):
        """decompose (decompose.hpp:77-103): (P, L, U) with A = P L U, each order x order, made on the
        device."""
        _require(matrix, order * order, matrix.dtype, "decompose")
        p, l, u = (self.empty(order * order, matrix.dtype) for _ in range(3))
        check(lib.sci_cuda_decompose(self.handle, self._precision(matrix.dtype), 1 if plain else 0,
                                     matrix.pointer, p.pointer, l.pointer, u.pointer, order), self.handle)
        return p, l, u

    # -- shapes: broadcasting, the roadmap's elementwise functions, axis reductions --------------
    def broadcast(self, code, operands, shape=()):
        """code(operands...) with numpy broadcasting (libsci's roadmap, README.md:149-152).

        `code` is a name ("add", "minimum", "power", "clip", "where", "copy", ...) and `operands`
        a list of (DeviceArray, shape) pairs of one element type; shapes align on the right as in
        numpy, and the result has their broadcast shape (with `shape` broadcast in too).
        Returns (DeviceArray, shape)."""
        number = C.EXTRA[code] if code in C.EXTRA else C.CODE[code]
        dtype = operands[0][0].dtype
        shapes = [tuple(int(e) for e in shape) for _, shape in operands]
        for (array, _), own in zip(operands, shapes):
            if array.dtype != dtype or array.count != int(np.prod(own, dtype=np.int64)):
                raise ValueError(f"operand of {array.count} {array.dtype} elements does not have shape {own}")
        shape = tuple(int(e) for e in np.broadcast_shapes(*shapes, tuple(shape)))
        rank = max(len(shape), 1)
        aligned = [(1,) * (rank - len(s)) + s for s in shapes]
        out = self.empty(int(np.prod(shape, dtype=np.int64)), dtype)
        inputs = (ctypes.c_void_p * len(operands))(*[array.pointer for array, _ in operands])
        extents = (ctypes.c_uint64 * (len(operands) * rank))(*[e for s in aligned for e in s])
        out_extents = (ctypes.c_uint64 * rank)(*(shape or (1,)))
        check(lib.sci_cuda_broadcast(self.handle, self._precision(dtype), number, rank, out_extents, len(operands),
                                     inputs, extents, out.pointer), self.handle)
        return out, shape

    def reduce_axis(self, array: "DeviceArray", shape, axis: int, fold: int):
        """sum / minimum / maximum / mean (C.AXIS_MEAN) of a row-major array along `axis`
        (negative counts from the end). Returns (DeviceArray, shape without that axis)."""
        shape = tuple(int(e) for e in shape)
        axis = axis + len(shape) if axis < 0 else axis
        if not 0 <= axis < len(shape):
            raise ValueError(f"axis {axis} of a rank-{len(shape)} array")
        kept = shape[:axis] + shape[axis + 1:]
        if array.count != int(np.prod(shape, dtype=np.int64)):
            raise ValueError(f"reduce_axis: {array.count} elements do not have shape {shape}")
        out = self.empty(int(np.prod(kept, dtype=np.int64)), array.dtype)
        extents = (ctypes.c_uint64 * len(shape))(*shape)
        check(lib.sci_cuda_reduce_axis(self.handle, self._precision(array.dtype), fold, array.pointer, len(shape), extents,
                                       axis, out.pointer), self.handle)
        return out, kept

    # -- chunks ---------------------------------------------------------------------------------
    def execute(self, chunk: C.Chunk, output: int, count: int) -> None:
        C.require_float(chunk)
        check(lib.sci_cuda_execute(self.handle, ctypes.byref(chunk), output, count), self.handle)

    def reduce_chunk(self, chunk: C.Chunk, fold: int, count: int) -> float:
        C.require_float(chunk)
        result = ctypes.c_double()
        check(lib.sci_cuda_reduce(self.handle, ctypes.byref(chunk), fold, count, ctypes.byref(result)), self.handle)
        return result.value

    def execute_elements(self, dtype, chunk: C.Chunk, output: int, count: int) -> None:
        """assign() for any element type (expression.hpp:158-185), integers included."""
        _same_element(chunk, dtype)
        check(lib.sci_cuda_execute_elements(self.handle, C.ELEMENT[np.dtype(dtype)], ctypes.byref(chunk), output, count),
              self.handle)

    def reduce_elements(self, dtype, chunk: C.Chunk, fold: int, count: int):
        """reduce() for any element type (expression.hpp:191-221): one element of `dtype`."""
        dtype = np.dtype(dtype)
        _same_element(chunk, dtype)
        result = np.zeros(1, dtype)
        check(lib.sci_cuda_reduce_elements(self.handle, C.ELEMENT[dtype], ctypes.byref(chunk), fold, count,
                                           result.ctypes.data), self.handle)
        return result[0]

    def reduce_async(self, chunk: C.Chunk, fold: int, count: int, device_result: int) -> None:
        C.require_float(chunk)
        check(lib.sci_cuda_reduce_async(self.handle, ctypes.byref(chunk), fold, count, device_result), self.handle)

    def product(self, left: "DeviceArray", right: "DeviceArray", rows: int, columns: int, depth: int,
                mode: int = 3, out: "DeviceArray | None" = None) -> "DeviceArray":
        """linear::product (include/linear/product.hpp:22-65): row-major out = left @ right.

        mode: 3 (the default) split3-bf16, six tensor-core products that keep FP32 accuracy like the
        reference's float product (dispatch.cpp:171-224); 0 bf16 tensor cores (about 8 bits per
        operand, an explicit opt-in); 1 split-bf16 (three products, about 16 bits); 2 plain FP32
        SIMT. Double operands always multiply in plain FP64."""
        dtype = left.dtype
        if out is None:
            out = self.empty(rows * columns, dtype)
        precision = self._precision(dtype)
        _require(left, rows * depth, dtype, "product left")
        _require(right, depth * columns, dtype, "product right")
        _require(out, rows * columns, dtype, "product output")
        check(lib.sci_cuda_product(self.handle, precision, mode, left.pointer, right.pointer, out.pointer, rows, columns,
                                   depth), self.handle)
        return out

    def factor(self, matrix: "DeviceArray", order: int, plain: bool = False) -> np.ndarray:
        """linear::factor (decompose.hpp:29-72) in place; returns rows[] (original row at each position)."""
        rows = np.zeros(order, np.uint64)
        precision = self._precision(matrix.dtype)
        _require(matrix, order * order, matrix.dtype, "factor")
        check(lib.sci_cuda_factor(self.handle, precision, 1 if plain else 0, matrix.pointer, rows.ctypes.data, order),
              self.handle)
        return rows

    def solve(self, matrix: "DeviceArray", right: "DeviceArray", order: int, width: int, refine: bool = False,
              out: "DeviceArray | None" = None):
        """linear::solve (solve.hpp:60-76). refine=True: FP32 LU plus FP64 refinement (double operands).
        Returns (solution, backward_error, iterations)."""
        from .native import SolveReport

        if out is None:
            out = self.empty(order * width, right.dtype)
        precision = self._precision(matrix.dtype)
        _require(matrix, order * order, matrix.dtype, "solve matrix")
        _require(right, order * width, matrix.dtype, "solve right-hand side")
        _require(out, order * width, matrix.dtype, "solve output")
        report = SolveReport()
        check(lib.sci_cuda_solve(self.handle, precision, 1 if refine else 0, matrix.pointer, right.pointer, out.pointer,
                                 order, width, ctypes.byref(report)), self.handle)
        return out, report.backward_error, report.iterations

    def evaluate(self, expression, out: "DeviceArray | None" = None) -> "DeviceArray":
        """assign(target, expression) (expression.hpp:158-185); allocates the target if needed."""
        expr = C._operand(expression, None)
        if out is None:
            out = self.empty(expr.count, expr.dtype)
        elif out.dtype != expr.dtype or out.count != expr.count:
            # assign's ASSERT(target.shape() == item.shape()) (expression.hpp:160), and the element
            # types match by construction there
            raise ValueError(f"target of {out.count} {out.dtype} elements for an expression of {expr.count} "
                             f"{expr.dtype} elements")
        chunk = C.record_output(expr)
        if not chunk.valid():
            raise SciCudaError(1, "expression outgrew the 64-entry chunk")
        if expr.dtype.kind in "iu":
            self.execute_elements(expr.dtype, chunk, out.pointer, expr.count)
        else:
            self.execute(chunk, out.pointer, expr.count)
        return out

    def reduce(self, expression, fold: int) -> float:
        expr = C._operand(expression, None)
        chunk = C.record_reduce(expr)
        if not chunk.valid():
            raise SciCudaError(1, "expression outgrew the 64-entry chunk")
        if expr.dtype.kind in "iu":
            return self.reduce_elements(expr.dtype, chunk, fold, expr.count)
        value = self.reduce_chunk(chunk, fold, expr.count)
        return float(expr.dtype.type(value))  # static_cast<element>(device->reduce(...)) (expression.hpp:198)


    def gradient(self, expression, wrt, seed: float = 1.0, stored: bool = False):
        """sci::gradient (new; the reference has none): for L = seed * sum(expression), returns
        (sum, [dL/dw for w in wrt]) with each gradient a DeviceArray shaped like w. stored=True runs
        the temporary-storing comparison form instead of the recomputing adjoint."""
        expr = C._operand(expression, None)
        chunk = C.record_reduce(expr)
        C.require_float(chunk)
        if not chunk.valid():
            raise SciCudaError(1, "expression outgrew the 64-entry chunk")
        wanted = {int(w.pointer): i for i, w in enumerate(wrt)}
        grads = [self.empty(w.count, w.dtype) for w in wrt]
        slots = (ctypes.c_void_p * max(1, chunk.arguments))()
        for a in range(chunk.arguments):
            pointer = int(chunk.inputs[a] or 0)
            if pointer in wanted:
                slots[a] = grads[wanted[pointer]].pointer
        for i, w in enumerate(wrt):
            if not any(int(chunk.inputs[a] or 0) == int(w.pointer) for a in range(chunk.arguments)):
                grads[i].upload(np.zeros(w.count, w.dtype))  # L does not depend on w
        value = ctypes.c_double()
        check(lib.sci_cuda_gradient(self.handle, ctypes.byref(chunk), expr.count, seed, slots, ctypes.byref(value),
                                    1 if stored else 0), self.handle)
        return value.value, grads


    def product_gradient(self, left: "DeviceArray", right: "DeviceArray", upstream: "DeviceArray", rows: int,
                         columns: int, depth: int, mode: int = 3):
        """Adjoints of product (new): (upstream @ right.T, left.T @ upstream) as DeviceArrays."""
        dtype = left.dtype
        precision = self._precision(dtype)
        _require(left, rows * depth, dtype, "product_gradient left")
        _require(right, depth * columns, dtype, "product_gradient right")
        _require(upstream, rows * columns, dtype, "product_gradient upstream")
        dl, dr = self.empty(rows * depth, dtype), self.empty(depth * columns, dtype)
        check(lib.sci_cuda_product_gradient(self.handle, precision, mode, left.pointer, right.pointer, upstream.pointer,
                                            dl.pointer, dr.pointer, rows, columns, depth), self.handle)
        return dl, dr

    def solve_gradient(self, matrix: "DeviceArray", right: "DeviceArray", upstream: "DeviceArray", order: int,
                       width: int, refine: bool = False):
        """Adjoints of solve (new): returns (X, dL/dmatrix, dL/dright, backward_error, iterations)."""
        from .native import SolveReport

        dtype = matrix.dtype
        precision = self._precision(dtype)
        _require(matrix, order * order, dtype, "solve_gradient matrix")
        _require(right, order * width, dtype, "solve_gradient right-hand side")
        _require(upstream, order * width, dtype, "solve_gradient upstream")
        x, dm, db = self.empty(order * width, dtype), self.empty(order * order, dtype), self.empty(order * width, dtype)
        report = SolveReport()
        check(lib.sci_cuda_solve_gradient(self.handle, precision, 1 if refine else 0, matrix.pointer, right.pointer,
                                          upstream.pointer, x.pointer, dm.pointer, db.pointer, order, width,
                                          ctypes.byref(report)), self.handle)
        return x, dm, db, report.backward_error, report.iterations


    def batch(self, chunk: C.Chunk, fold: int, inputs: np.ndarray, counts: np.ndarray, outputs=None,
              results: "DeviceArray | None" = None) -> "Batch":
        """Many instances of one chunk in one graph-captured launch (new; the reference batches
        dispatches into Vulkan command buffers). inputs: items x arguments device pointers; counts:
        items element counts; outputs: items device pointers or None; results: a float64
        DeviceArray of items values, or None."""
        C.require_float(chunk)
        return Batch(self, chunk, fold, inputs, counts, outputs, results)


    def solve_batch(self, orders, matrices, rights, solutions, errors: "DeviceArray | None" = None,
                    iterations: "DeviceArray | None" = None) -> "SolveBatch":
        """Many small solves (n <= 256, one right-hand side, double) in one graph replay: FP32 LU +
        FP64 refinement per system. matrices / rights / solutions: device pointers per system."""
        return SolveBatch(self, orders, matrices, rights, solutions, errors, iterations)


class SolveBatch:
    """A prepared batch of small solves (sci_cuda_solve_batch_*)."""

    def __init__(self, device: Device, orders, matrices, rights, solutions, errors, iterations):
        from .native import SolveItems

        self.device = device
        self._keep = [np.ascontiguousarray(orders, np.uint32)] + [np.ascontiguousarray(t, np.uint64)
                                                                  for t in (matrices, rights, solutions)]
        items = SolveItems(len(self._keep[0]), *[k.ctypes.data for k in self._keep],
                           None if errors is None else errors.pointer,
                           None if iterations is None else iterations.pointer)
        self.handle = ctypes.c_void_p()
        check(lib.sci_cuda_solve_batch_create(device.handle, ctypes.byref(items), ctypes.byref(self.handle)),
              device.handle)

    def launch(self) -> None:
        check(lib.sci_cuda_solve_batch_launch(self.handle), self.device.handle)

    def shapes(self):
        threads = (ctypes.c_uint32 * 4)()
        check(lib.sci_cuda_solve_batch_shapes(self.handle, threads), self.device.handle)
        return list(threads)

    def close(self) -> None:
        if self.handle:
            lib.sci_cuda_solve_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()


class Batch:
    """A prepared batch (sci_cuda_batch_*): launch() replays its CUDA graph on the device stream."""

    def __init__(self, device: Device, chunk: C.Chunk, fold: int, inputs, counts, outputs, results):
        from .native import BatchItems

        self.device = device
        self._inputs = np.ascontiguousarray(inputs, np.uint64)
        self._counts = np.ascontiguousarray(counts, np.uint64)
        self._outputs = None if outputs is None else np.ascontiguousarray(outputs, np.uint64)
        items = BatchItems(len(self._counts), self._inputs.ctypes.data,
                           None if self._outputs is None else self._outputs.ctypes.data, self._counts.ctypes.data,
                           None if results is None else results.pointer)
        self.handle = ctypes.c_void_p()
        check(lib.sci_cuda_batch_create(device.handle, ctypes.byref(chunk), fold, ctypes.byref(items),
                                        ctypes.byref(self.handle)), device.handle)

    def launch(self) -> None:
        check(lib.sci_cuda_batch_launch(self.handle), self.device.handle)

    def spans(self):
        spans = (ctypes.c_uint32 * 3)()
        specialized = ctypes.c_int32()
        check(lib.sci_cuda_batch_spans(self.handle, spans, ctypes.byref(specialized)), self.device.handle)
        return list(spans), bool(specialized.value)

    def close(self) -> None:
        if self.handle:
            lib.sci_cuda_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()


class DeviceArray:
    """A one-dimensional array in this device's memory."""

    def __init__(self, device: Device, pointer: int, count: int, dtype):
        self.device = device
        self.pointer = int(pointer)
        self.count = int(count)
        self.dtype = np.dtype(dtype)

    @property
    def nbytes(self) -> int:
        return self.count * self.dtype.itemsize

    def expression(self) -> C.Reference:
        return C.Reference(self.pointer, self.count, self.dtype, self.device)

    def offset(self, elements: int, count: int | None = None) -> "DeviceArray":
        """A view starting `elements` in (not owning memory)."""
        view = DeviceArray.__new__(DeviceArray)
        view.device, view.dtype = self.device, self.dtype
        view.pointer = self.pointer + elements * self.dtype.itemsize
        view.count = self.count - elements if count is None else count
        view._view = True
        return view

    def upload(self, host: np.ndarray) -> None:
        host = np.ascontiguousarray(host, dtype=self.dtype)
        check(lib.sci_cuda_upload(self.device.handle, self.pointer, host.ctypes.data, host.nbytes), self.device.handle)
        self.device.synchronize()

    def numpy(self) -> np.ndarray:
        """Array.host(): waits for queued work, then copies back (array.hpp:232-237)."""
        out = np.empty(self.count, self.dtype)
        check(lib.sci_cuda_download(self.device.handle, out.ctypes.data, self.pointer, out.nbytes), self.device.handle)
        self.device.synchronize()
        return out

    def free(self) -> None:
        if self.pointer and not getattr(self, "_view", False):
            self.device.dispose(self.pointer)
            self.pointer = 0

    # operators build expressions
    def __add__(self, other):
        return self.expression() + other

    def __radd__(self, other):
        return other + self.expression()

    def __sub__(self, other):
        return self.expression() - other

    def __rsub__(self, other):
        return other - self.expression()

    def __mul__(self, other):
        return self.expression() * other

    def __rmul__(self, other):
        return other * self.expression()

    def __truediv__(self, other):
        return self.expression() / other

    def __rtruediv__(self, other):
        return other / self.expression()

    def __neg__(self):
        return -self.expression()


# ---- numpy-named front end (include/operations/unary.hpp, binary.hpp, reduce.hpp) -------------
def _unary(code):
    def op(item):
        return C.unary(code, item)

    op.__name__ = code
    return op


for _code in C.UNARY:
    globals()[_code] = _unary(_code)
negate = _unary("negate")


def minimum(first, second=None):
    """Elementwise with two operands, a reduction with one (include/sci.hpp: numpy.minimum / min)."""
    if second is None:
        return _device_of(first).reduce(first, C.MINIMUM)
    return C.binary("minimum", first, second)


def maximum(first, second=None):
    if second is None:
        return _device_of(first).reduce(first, C.MAXIMUM)
    return C.binary("maximum", first, second)


def add(a, b):
    return C.binary("add", a, b)


def subtract(a, b):
    return C.binary("subtract", a, b)


def multiply(a, b):
    return C.binary("multiply", a, b)


def divide(a, b):
    return C.binary("divide", a, b)


def sum(item):  # noqa: A001 - numpy name
    return _device_of(item).reduce(item, C.SUM)


def mean(item):
    """reduce.hpp:24-28: sum / count in the element type (for integers: the wrapped sum divided by
    the count converted to the element type, truncating toward zero)."""
    expr = C._operand(item, None)
    if expr.count == 0:
        return expr.dtype.type(0) if expr.dtype.kind in "iu" else 0.0
    if expr.dtype.kind in "iu":
        return integer_mean(sum(item), expr.count, expr.dtype)
    total = expr.dtype.type(sum(item))
    return float(total / expr.dtype.type(expr.count))


def integer_mean(total, count: int, dtype):
    """reduce.hpp:27 for an integer element: sum / static_cast<element>(count), the sum already
    wrapped in the element's width, the count converted (wrapping) to the element type, and the
    division truncating toward zero (wrapping for MIN / -1)."""
    dtype = np.dtype(dtype)
    divisor = int(np.array(count, np.uint64).astype(dtype))
    if divisor == 0:
        raise ZeroDivisionError("the count converts to 0 in the element type")
    total = int(total)
    quotient = abs(total) // abs(divisor) * (1 if (total < 0) == (divisor < 0) else -1)
    return np.array(quotient).astype(dtype)[()]


def dot(first, second):
    """linear::dot: reduce(first * second, sum) (product.hpp:72-76), contracted on the device."""
    return _device_of(first).reduce(C.binary("multiply", first, second), C.SUM)


def _require(array: "DeviceArray", count: int, dtype, what: str) -> None:
    """The C ABI sees raw pointers: the host checks that each operand holds what the call reads or
    writes, in the call's element type, before anything launches."""
    if array.dtype != np.dtype(dtype):
        raise TypeError(f"{what}: {array.dtype} elements where {np.dtype(dtype)} is needed")
    if array.count < count:
        raise ValueError(f"{what}: {array.count} elements where the call uses {count}")


def _same_element(chunk, dtype) -> None:
    element = getattr(chunk, "element", None)
    if element is not None and element != C.ELEMENT[np.dtype(dtype)]:
        raise TypeError(f"the chunk was recorded over another element type than {np.dtype(dtype)}")


def _shaped(item, device=None, dtype=None):
    """(DeviceArray, shape) from a pair, a DeviceArray (one axis) or a scalar (shape ())."""
    if isinstance(item, tuple) and len(item) == 2 and isinstance(item[0], DeviceArray):
        return item
    if isinstance(item, DeviceArray):
        return item, (item.count,)
    return device.full(1, float(item), dtype), ()


def _broadcast(code, *items):
    anchor = next(i for i in items if isinstance(i, DeviceArray) or isinstance(i, tuple))
    array = anchor[0] if isinstance(anchor, tuple) else anchor
    operands = [_shaped(item, array.device, array.dtype) for item in items]
    return array.device.broadcast(code, operands)


def power(x, y):
    """numpy.power with broadcasting; returns (DeviceArray, shape)."""
    return _broadcast("power", x, y)


def floor(x):
    return _broadcast("floor", x)


def ceil(x):
    return _broadcast("ceil", x)


def round(x):  # noqa: A001 - numpy name
    """numpy.round: halves to even."""
    return _broadcast("round", x)


def clip(x, lower, upper):
    """numpy.clip: minimum(maximum(x, lower), upper); bounds may be arrays or scalars."""
    return _broadcast("clip", x, lower, upper)


def where(condition, x, y):
    """numpy.where(condition != 0, x, y) with broadcasting."""
    return _broadcast("where", condition, x, y)


def broadcast_to(x, shape):
    """numpy.broadcast_to, materialised (a copy): (DeviceArray, shape)."""
    array, own = _shaped(x)
    shape = tuple(int(e) for e in shape)
    if np.broadcast_shapes(tuple(own), shape) != shape:
        raise ValueError(f"cannot broadcast {tuple(own)} to {shape}")
    return array.device.broadcast("copy", [(array, own)], shape)


def sum_axis(x, axis):
    array, shape = _shaped(x)
    return array.device.reduce_axis(array, shape, axis, C.SUM)


def mean_axis(x, axis):
    array, shape = _shaped(x)
    return array.device.reduce_axis(array, shape, axis, C.AXIS_MEAN)


def minimum_axis(x, axis):
    array, shape = _shaped(x)
    return array.device.reduce_axis(array, shape, axis, C.MINIMUM)


def maximum_axis(x, axis):
    array, shape = _shaped(x)
    return array.device.reduce_axis(array, shape, axis, C.MAXIMUM)


def _device_of(item) -> Device:
    if isinstance(item, DeviceArray):
        return item.device
    expr = C._operand(item, None)
    for leaf in expr.leaves():
        if getattr(leaf, "device", None) is not None:
            return leaf.device
    raise SciCudaError(1, "expression has no operand on a device")


__all__ = ["Device", "DeviceArray", "minimum", "maximum", "add", "subtract", "multiply", "divide", "sum", "mean",
           "dot", "negate", "power", "floor", "ceil", "round", "clip", "where", "broadcast_to", "sum_axis",
           "mean_axis", "minimum_axis", "maximum_axis"] + list(C.UNARY)
