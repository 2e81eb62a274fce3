/* sci_cuda.h -- C ABI of the B200 (sm_100a) backend for libsci.
 *
 * The reference drives every compute device through sci::core::drivers::Device
 * (include/core/drivers/device.hpp:27-89 in libsci). This header is the boundary a new
 * `Target::cuda` branch of that class calls: plain pointers, sizes and status codes, no C++
 * or torch types. Each entry point names the reference interface it stands in for.
 *
 * Conventions
 *  - Every call returns SCI_CUDA_OK (0) or a nonzero status; sci_cuda_last_error() gives the
 *    message. Nothing falls back to the CPU: a chunk the device cannot run is an error.
 *  - Work is queued in order on one CUDA stream per context (the reference's vulkan::Stream,
 *    src/core/drivers/vulkan/stream.cpp:56-130); calls that return a host value wait for it.
 *  - One mutex per context serialises its users (Graphics::guard, src/core/drivers/device.cpp:127).
 */
#ifndef SCI_CUDA_H
#define SCI_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
enum {
    SCI_CUDA_OK = 0,
    SCI_CUDA_ERROR_INVALID = 1,     /* bad argument: null pointer, size, code, slot, ...      */
    SCI_CUDA_ERROR_MEMORY = 2,      /* device allocation failed                                */
    SCI_CUDA_ERROR_LAUNCH = 3,      /* a CUDA call or kernel launch failed                     */
    SCI_CUDA_ERROR_UNSUPPORTED = 4, /* valid request this build does not run                   */
    SCI_CUDA_ERROR_DEVICE = 5,      /* no usable sm_100 device at that ordinal                 */
    SCI_CUDA_ERROR_TIMEOUT = 6,     /* a bounded device-side wait ran out                      */
    SCI_CUDA_ERROR_COMPILE = 7      /* NVRTC specialisation failed (the interpreter still runs) */
};

/* ---- the chunk: mirrors sci::core::Chunk field for field --------------------------------- */
/* include/core/bytecode/chunk.hpp:78-246, instruction.hpp:12-35, code.hpp:18-61, fold.hpp:11 */
#define SCI_CHUNK_CAPACITY 64

enum { SCI_PRECISION_SINGLE = 0, SCI_PRECISION_WIDE = 1 }; /* precision.hpp:12 */

/* value ids: kind in the top two bits, index in the low six (instruction.hpp:12-25) */
enum {
    SCI_SLOT_INPUT = 0x00,
    SCI_SLOT_LITERAL = 0x40,
    SCI_SLOT_TEMPORARY = 0x80,
    SCI_SLOT_OUTPUT = 0xC0,
    SCI_SLOT_NONE = 0xFF,
    SCI_SLOT_TYPES = 0xC0
};

/* operation codes, in core::Code's order (code.hpp:18-61) */
enum {
    SCI_CODE_COPY, SCI_CODE_NEGATE, SCI_CODE_ABSOLUTE,
    SCI_CODE_ROOT, SCI_CODE_EXPONENTIAL, SCI_CODE_LOGARITHM,
    SCI_CODE_SIN, SCI_CODE_COS, SCI_CODE_TAN, SCI_CODE_ASIN, SCI_CODE_ACOS, SCI_CODE_ATAN,
    SCI_CODE_CSC, SCI_CODE_SEC, SCI_CODE_COT, SCI_CODE_ACSC, SCI_CODE_ASEC, SCI_CODE_ACOT,
    SCI_CODE_SINH, SCI_CODE_COSH, SCI_CODE_TANH, SCI_CODE_ASINH, SCI_CODE_ACOSH, SCI_CODE_ATANH,
    SCI_CODE_CSCH, SCI_CODE_SECH, SCI_CODE_COTH, SCI_CODE_ACSCH, SCI_CODE_ASECH, SCI_CODE_ACOTH,
    SCI_CODE_ADD, SCI_CODE_SUBTRACT, SCI_CODE_MULTIPLY, SCI_CODE_DIVIDE,
    SCI_CODE_MINIMUM, SCI_CODE_MAXIMUM, SCI_CODE_FUSE,
    SCI_CODE_COUNT
};

enum { SCI_FOLD_SUM = 0, SCI_FOLD_MINIMUM = 1, SCI_FOLD_MAXIMUM = 2 }; /* fold.hpp:11 */

typedef struct sci_instruction { /* core::Instruction, instruction.hpp:28-35 */
    uint8_t code;
    uint8_t target;
    uint8_t sources[3];
} sci_instruction;

typedef struct sci_chunk { /* core::Chunk's public state, chunk.hpp:228-246 */
    uint8_t precision;
    uint8_t length;
    uint8_t arguments;
    uint8_t literals;
    uint8_t temporaries;
    uint8_t result;
    sci_instruction instructions[SCI_CHUNK_CAPACITY];
    const void *inputs[SCI_CHUNK_CAPACITY];
    double constants[SCI_CHUNK_CAPACITY];
} sci_chunk;


/* ---- context ----------------------------------------------------------------------------- */
typedef struct sci_cuda_context sci_cuda_context;

/* Device::Device(Target, index) (device.hpp:32, device.cpp:186-199). Opens device `ordinal`;
 * fails with SCI_CUDA_ERROR_DEVICE when it is not an sm_100 part (no CPU fallback). */
int sci_cuda_open(uint32_t ordinal, sci_cuda_context **context);
/* Device::~Device(): waits for queued work, then frees everything the context owns. */
int sci_cuda_close(sci_cuda_context *context);
/* Device::name() (device.hpp:46). */
const char *sci_cuda_name(const sci_cuda_context *context);
/* Device::synchronize() (device.hpp:49, device.cpp:205-210): waits for queued work and reports
 * any error a kernel recorded on the device since the last wait. */
int sci_cuda_synchronize(sci_cuda_context *context);
/* The message of the last failed call on this context. */
int sci_cuda_last_error(const sci_cuda_context *context, char *buffer, size_t length);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own work with it. */
void *sci_cuda_stream(sci_cuda_context *context);

/* ---- memory ------------------------------------------------------------------------------ */
enum {
    SCI_CUDA_MEMORY_DEVICE = 0, /* HBM only; reach it with upload / download                   */
    SCI_CUDA_MEMORY_MANAGED = 1 /* also a valid host pointer, like the reference's Memory::host */
};
/* Device::allocate(bytes, Memory&) (device.hpp:55, device.cpp:212-224). 256-byte aligned. */
int sci_cuda_allocate(sci_cuda_context *context, uint64_t bytes, uint32_t kind, void **memory);
/* Device::dispose(Memory&) (device.hpp:58, device.cpp:226-233): the free is deferred until work
 * queued before it has finished, as vulkan::Stream::retire does (stream.cpp:117-130). */
int sci_cuda_dispose(sci_cuda_context *context, void *memory);
/* Array::to(device) / Array::host() transfers (array.hpp:223-237), queued on the stream. */
int sci_cuda_upload(sci_cuda_context *context, void *device, const void *host, uint64_t bytes);
int sci_cuda_download(sci_cuda_context *context, void *host, const void *device, uint64_t bytes);
/* Copy lanes (new; the reference copies through the host pointer): the same copies on two more
 * streams, so that uploads, kernels and downloads of different pieces overlap. An upload on the
 * lane starts without waiting for queued work, and work queued after it waits for it; a download
 * on the lane waits for the work queued before it and delays nothing queued after it. Host memory
 * should be pinned for the copies to overlap. sci_cuda_join is a barrier between the lanes and the
 * main stream: work queued after it waits for every lane copy queued before it, and lane copies
 * queued after it wait for the main stream's work queued before it. sci_cuda_synchronize waits for
 * the lanes too. */
int sci_cuda_upload_lane(sci_cuda_context *context, void *device, const void *host, uint64_t bytes);
int sci_cuda_download_lane(sci_cuda_context *context, void *host, const void *device, uint64_t bytes);
int sci_cuda_join(sci_cuda_context *context);

/* ---- chunks ------------------------------------------------------------------------------ */
/* Device::execute(chunk, output, count) (device.hpp:63, device.cpp:235-263): output[i] =
 * chunk(inputs[i]) for i < count, queued. Inputs and output must be device or managed memory of
 * this context's GPU. Arithmetic is bit-identical to the reference's AVX-512 kernel table;
 * the C-library functions are within 2 ulp of it. */
int sci_cuda_execute(sci_cuda_context *context, const sci_chunk *chunk, void *output, uint64_t count);
/* Device::reduce(chunk, fold, count) (device.hpp:69, device.cpp:265-316): the sum, minimum or
 * maximum of the chunk's result over count elements, folded in double in a single pass; NaN
 * anywhere gives NaN; an empty sum is 0 and an empty extreme NaN. sum(a*b) is contracted
 * (chunk.hpp:201-204): a*b is never rounded or stored. Waits for the result. */
int sci_cuda_reduce(sci_cuda_context *context, const sci_chunk *chunk, uint32_t fold, uint64_t count,
                    double *result);
/* The same reduction, queued: the double result is written to device memory `device_result`. */
int sci_cuda_reduce_async(sci_cuda_context *context, const sci_chunk *chunk, uint32_t fold, uint64_t count,
                          double *device_result);

/* ---- shapes: broadcasting, the roadmap's elementwise functions, axis reductions ------------- */
/* libsci lists these as next (README.md:149-152) and has no implementation yet; the rules are
 * numpy's, which its operations are named after (reduce.hpp:8-9). */
enum { /* codes beyond core::Code, for sci_cuda_broadcast only */
    SCI_EXTRA_FLOOR = 64, SCI_EXTRA_CEIL = 65, SCI_EXTRA_ROUND = 66, /* round: halves to even (numpy.round) */
    SCI_EXTRA_POWER = 67,                                            /* C pow; float raised in double */
    SCI_EXTRA_CLIP = 68,                                             /* minimum(maximum(x, lo), hi) */
    SCI_EXTRA_WHERE = 69                                             /* condition != 0 ? x : y */
};
/* output = code(operands...) over the output `shape` (rank 1 to 8). Every operand has `rank`
 * extents in input_shapes[k * rank + axis], each equal to the output's or 1 (broadcast: the caller
 * prepends 1s, as numpy aligns shapes on the right). Codes: SCI_CODE_COPY (broadcast_to), ADD,
 * SUBTRACT, MULTIPLY, DIVIDE, MINIMUM, MAXIMUM (NaN propagates, numpy.minimum / maximum) and the
 * SCI_EXTRA codes; 1, 2 or 3 operands by code. Queued. */
int sci_cuda_broadcast(sci_cuda_context *context, uint32_t precision, uint32_t code, uint32_t rank,
                       const uint64_t *shape, uint32_t operands, const void *const *inputs,
                       const uint64_t *input_shapes, void *output);
enum { SCI_AXIS_MEAN = 3 }; /* beside SCI_FOLD_SUM / MINIMUM / MAXIMUM */
/* sum(a, axis) and the rest: folds `input` (row-major, `shape`, rank 1 to 8) over `axis` into
 * `output` (the shape without that axis). Folds in double, NaN propagates, one cast to the element
 * type; mean = sum / count in the element type (reduce.hpp:24-28); an empty axis gives 0 for sum
 * and mean, NaN for minimum and maximum. Queued. */
int sci_cuda_reduce_axis(sci_cuda_context *context, uint32_t precision, uint32_t fold, const void *input,
                         uint32_t rank, const uint64_t *shape, uint32_t axis, void *output);

/* ---- chunks over other element types ------------------------------------------------------- */
/* The reference records chunks for float and double only (core::native, traits.hpp:26); any other
 * element type evaluates its expression tree on the host, element by element, with the scalar
 * semantics of array::calculate (calculate.hpp:17-93) in assign() (expression.hpp:178-184) and
 * reduce() (expression.hpp:203-220). These entry points run the same expression, recorded into the
 * same bytecode (the chunk's precision field is ignored), on the device. FLOAT32 / FLOAT64 go to
 * sci_cuda_execute / sci_cuda_reduce. Integer arithmetic wraps in the element's width; a zero
 * divisor gives 0; a real function's NaN converts to 0 and out-of-range values saturate (the cases
 * C++ leaves undefined). */
enum {
    SCI_ELEMENT_FLOAT32 = 0, SCI_ELEMENT_FLOAT64 = 1, /* = SCI_PRECISION_SINGLE / _WIDE */
    SCI_ELEMENT_INT8 = 2, SCI_ELEMENT_INT16 = 3, SCI_ELEMENT_INT32 = 4, SCI_ELEMENT_INT64 = 5,
    SCI_ELEMENT_UINT8 = 6, SCI_ELEMENT_UINT16 = 7, SCI_ELEMENT_UINT32 = 8, SCI_ELEMENT_UINT64 = 9
};
/* Bytes per element, 0 for an unknown type. */
uint64_t sci_cuda_element_size(uint32_t element);
/* assign(target, expression) for an array of `element` (expression.hpp:158-185), queued. */
int sci_cuda_execute_elements(sci_cuda_context *context, uint32_t element, const sci_chunk *chunk, void *output,
                              uint64_t count);
/* reduce(expression, fold) (expression.hpp:191-221): writes one element (its own size) to the host
 * pointer `result`; an empty reduction is element{} = 0 for every fold (expression.hpp:205). Waits. */
int sci_cuda_reduce_elements(sci_cuda_context *context, uint32_t element, const sci_chunk *chunk, uint32_t fold,
                             uint64_t count, void *result);
/* ---- matrix product ------------------------------------------------------------------------ */
enum {
    SCI_PRODUCT_BF16 = 0,       /* bf16 operands on tcgen05 tensor cores, FP32 accumulation           */
    SCI_PRODUCT_SPLIT_BF16 = 1, /* hi+lo bf16 split, three tensor-core products, ~16-bit operands      */
    SCI_PRODUCT_FP32 = 2,       /* plain FP32 SIMT: the comparison form (double always runs plain FP64) */
    SCI_PRODUCT_SPLIT3_BF16 = 3 /* hi+mid+lo bf16 split, six tensor-core products, ~FP32-accurate      */
};
/* Device::product(precision, left, right, output, rows, columns, depth) (device.hpp:79-80,
 * device.cpp:318-352; linear::product, include/linear/product.hpp:22-65): row-major
 * output (rows x columns) = left (rows x depth) * right (depth x columns), queued. `mode` chooses
 * how single-precision products run; depth 0 writes zeros (dispatch.cpp:270-273). The bf16 modes
 * use a workspace of the context that grows to 2 bytes x (rows + columns) x depth x terms. */
int sci_cuda_product(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *left, const void *right,
                     void *output, uint64_t rows, uint64_t columns, uint64_t depth);

/* ---- LU and solve -------------------------------------------------------------------------- */
enum {
    SCI_FACTOR_TENSOR = 0, /* float: trailing updates on the tensor cores (split-bf16, FP32 accumulation) */
    SCI_FACTOR_PLAIN = 1   /* float: trailing updates in plain FP32 SIMT (double always plain FP64)     */
};
enum { SCI_REFINE_NONE = 0, SCI_REFINE_FP64 = 1 };

typedef struct sci_solve_report {
    double backward_error; /* max over columns of |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf), in FP64 */
    int iterations;        /* refinement iterations (0 without refinement) */
} sci_solve_report;

/* linear::factor (include/linear/decompose.hpp:29-72): in-place LU with partial pivoting of the
 * order x order row-major device matrix; on return the strict lower triangle holds L (unit
 * diagonal implied), the rest U, and host array rows[i] is the original row now at position i.
 * The pivot is the first row with the strictly largest |a|; a zero pivot is skipped. Waits.
 * order <= 8192. */
int sci_cuda_factor(sci_cuda_context *context, uint32_t precision, uint32_t mode, void *matrix, uint64_t *rows,
                    uint64_t order);
/* linear::solve (include/linear/solve.hpp:60-76): solution (order x width) with matrix * solution =
 * right, all device memory, row-major. refine = SCI_REFINE_NONE factors and substitutes in the
 * element type (the reference's behaviour); SCI_REFINE_FP64 (double operands) factors in FP32
 * and iterates r = b - A x in FP64 until the normwise backward error is <= min(sqrt(n) 2^-53, 1e-14)
 * (LAPACK DSGESV's test) or stalls.
 * `report` (may be null) receives the backward error and iteration count. Waits. order <= 8192. */
int sci_cuda_solve(sci_cuda_context *context, uint32_t precision, uint32_t refine, const void *matrix, const void *right,
                   void *solution, uint64_t order, uint64_t width, sci_solve_report *report);

/* ---- gradients ------------------------------------------------------------------------------- */
/* No counterpart in the reference (sci::gradient is new; the reference has no differentiation).
 * For L = seed * sum over count elements of the chunk's reduced value (the sum
 * sci_cuda_reduce(SCI_FOLD_SUM) computes), writes dL/d(argument a) elementwise to gradients[a]
 * (device memory, count elements of the chunk's element type; a null entry, or a null array, skips
 * it) and, when `value` is not null, the sum itself to *value (double). The derivatives are those of
 * the function the device computes: forward values are bit-identical to sci_cuda_execute's, partial
 * derivatives are evaluated in double and adjoints accumulate in double before one rounding.
 * Conventions: d|x| at 0 is 0; minimum / maximum pass the adjoint to the operand they returned;
 * a zero adjoint passes nothing back. Waits for the sum when `value` is not null; without it the
 * call is only queued (errors a kernel records surface at the next sci_cuda_synchronize). `form`: */
enum {
    SCI_GRADIENT_RECOMPUTE = 0, /* one pass: forward values recomputed in registers, reverse walk, no tape */
    SCI_GRADIENT_STORED = 1     /* the plain comparison form: a forward pass stores every value of the chunk
                                   on a device tape (nodes x count elements, kept by the context), and a
                                   backward pass reads it */
};
int sci_cuda_gradient(sci_cuda_context *context, const sci_chunk *chunk, uint64_t count, double seed,
                      void *const *gradients, double *value, uint32_t form);
/* No counterpart in the reference. The adjoints of sci_cuda_product (linear::product): for
 * C = left * right (rows x depth times depth x columns) and upstream = dL/dC (rows x columns),
 * left_gradient = upstream * right^T (rows x depth) and right_gradient = left^T * upstream
 * (depth x columns), two products in `mode` with the transposed operands read in place. Either
 * gradient may be null. Queued. */
int sci_cuda_product_gradient(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *left,
                              const void *right, const void *upstream, void *left_gradient, void *right_gradient,
                              uint64_t rows, uint64_t columns, uint64_t depth);
/* No counterpart in the reference. The adjoints of sci_cuda_solve (linear::solve): for
 * X = matrix^-1 right and upstream = dL/dX (order x width), right_gradient = lambda = matrix^-T upstream
 * and matrix_gradient = -lambda X^T (order x order). One factorisation serves both solves: the
 * transposed solve runs the substitutions through U^T and L^T of the same factors, then P^T. X is
 * written to `solution` when it is not null; either gradient may be null. `refine` as for
 * sci_cuda_solve, applied to both solves; `report` receives the larger of the two backward errors and
 * the iterations of both. Waits. order <= 8192. */
int sci_cuda_solve_gradient(sci_cuda_context *context, uint32_t precision, uint32_t refine, const void *matrix,
                            const void *right, const void *upstream, void *solution, void *matrix_gradient,
                            void *right_gradient, uint64_t order, uint64_t width, sci_solve_report *report);

/* ---- batches ---------------------------------------------------------------------------------- */
/* Many instances ("items") of one chunk in one persistent launch, replayed from a CUDA graph. No
 * counterpart in the reference's API; it stands where the reference batches its dispatches into a
 * Vulkan command buffer (src/core/drivers/vulkan/stream.cpp:71-106). Every item supplies its own
 * inputs, output and element count; the chunk's own inputs[] are ignored. Tables are host arrays,
 * read once at creation; the pointers in them are device memory of the context's GPU. */
typedef struct sci_batch_items {
    uint32_t items;
    const void *const *inputs; /* items x chunk->arguments pointers, one row per item             */
    void *const *outputs;      /* items pointers receiving the chunk's stored output, or null      */
    const uint64_t *counts;    /* items element counts (0 allowed)                                  */
    void *results;             /* device memory, items doubles: each item's reduced value (the fold
                                  of the chunk's result), or null when the batch only stores       */
} sci_batch_items;
typedef struct sci_cuda_batch sci_cuda_batch;
/* Prepares a batch: checks every item, compiles the chunk's batch kernel (NVRTC, synchronously),
 * tunes the unit span of each item-size bucket (< 4096, < 65536, larger; cached per device, chunk
 * signature and bucket in SCI_CUDA_TUNE_CACHE, default $HOME/.cache/sci_cuda/batch_tune.txt;
 * SCI_CUDA_TUNE=0 skips tuning), uploads the item tables and captures the launch into a CUDA graph.
 * The tuning launches run the batch, so outputs and results are written. A chunk may both store
 * an output and reduce a result. Stored outputs are bit-identical to sci_cuda_execute on each item;
 * results are folded in double like sci_cuda_reduce (in a fixed, per-item order). Waits. */
int sci_cuda_batch_create(sci_cuda_context *context, const sci_chunk *chunk, uint32_t fold,
                          const sci_batch_items *items, sci_cuda_batch **batch);
/* Replays the batch's graph on the context's stream (queued). */
int sci_cuda_batch_launch(sci_cuda_batch *batch);
/* The unit span chosen for each of the three buckets and whether the kernel is the NVRTC instance. */
int sci_cuda_batch_spans(const sci_cuda_batch *batch, uint32_t *spans, int32_t *specialized);
/* Waits for the context's queued work, then frees the batch. */
int sci_cuda_batch_destroy(sci_cuda_batch *batch);

/* Thousands of small independent solves (linear::solve, include/linear/solve.hpp:60-76, one
 * right-hand side each, double operands, order 1..256) in one graph replay: FP32 LU with the
 * reference's pivoting rules and FP64 refinement, one CTA per system (no counterpart in the
 * reference's API). Tables are host arrays read once at creation; the pointers in them, and
 * `errors` / `iterations` (systems entries each, may be null), are device memory. */
typedef struct sci_solve_items {
    uint32_t systems;
    const uint32_t *orders;        /* order of each system                                  */
    const void *const *matrices;   /* n x n row-major doubles per system                    */
    const void *const *rights;     /* n doubles per system                                  */
    void *const *solutions;        /* n doubles per system, written                         */
    double *errors;                /* normwise backward error per system, or null          */
    int32_t *iterations;           /* refinement iterations per system, or null            */
} sci_solve_items;
typedef struct sci_cuda_solve_batch sci_cuda_solve_batch;
/* Checks every system, tunes the block size of each order bucket (<= 32, <= 64, <= 128, <= 256;
 * cached like the chunk batches), and captures one launch per bucket into a CUDA graph. The tuning
 * launches solve the systems. Waits. */
int sci_cuda_solve_batch_create(sci_cuda_context *context, const sci_solve_items *items, sci_cuda_solve_batch **batch);
/* Replays the graph on the context's stream (queued). */
int sci_cuda_solve_batch_launch(sci_cuda_solve_batch *batch);
/* Threads per CTA chosen for each bucket (0: the bucket is empty). */
int sci_cuda_solve_batch_shapes(const sci_cuda_solve_batch *batch, uint32_t *threads);
/* Waits for the context's queued work, then frees the batch. */
int sci_cuda_solve_batch_destroy(sci_cuda_solve_batch *batch);

/* No counterpart in the reference. The same reduction for callers that may not allocate device
 * memory (a host framework that owns the GPU heap through its own pool, a plugin inside one, a
 * latency-critical thread where an allocation would synchronize the device). It needs no context:
 * it runs on the calling thread's current device and on `stream` (a cudaStream_t; 0 is the legacy
 * default stream), reads the chunk's inputs from device memory and writes the double result to
 * `device_result`, both on that device. Its scratch is one fixed 49,664-byte array compiled into
 * the library, holding partials for at most 4096 blocks: `blocks` = 0 picks the launch width,
 * a larger value than 4096 is rejected with SCI_CUDA_ERROR_INVALID. It calls no cudaMalloc or
 * cudaFree. Every call on a device shares that array: calls whose kernels may overlap on the GPU
 * race and must be ordered by the caller (one stream, or events). The first call on a device
 * looks up the array's device address; make it before capturing the stream into a graph. The
 * call returns before the kernel runs, so a device-side failure cannot come back as a status: if
 * a block's bounded wait on its input copies runs out, `device_result` receives a quiet NaN
 * rather than a partial value. On failure a message is written to `message` (may be null). */
int sci_cuda_reduce_noalloc(const sci_chunk *chunk, uint32_t fold, uint64_t count, double *device_result,
                            void *stream, uint32_t blocks, char *message, size_t message_length);
/* ---- arrays made on the device (include/operations/creation.hpp) ----------------------------
 * The element values of libsci's creation functions, computed where the array lives, on the
 * context's stream (asynchronous). `output` (and grid's operands) must be device memory of the
 * context; `precision` is SCI_PRECISION_SINGLE (float) or SCI_PRECISION_WIDE (double). */
/* zeros / ones / full (creation.hpp:34-58): output[0, count) := value, cast to the element type. */
int sci_cuda_fill(sci_cuda_context *context, uint32_t precision, void *output, uint64_t count, double value);
/* linspace (creation.hpp:66-84): count values from start to stop, both included; start and stop
 * are elements (their difference is taken in the element type, the rest in double). */
int sci_cuda_linspace(sci_cuda_context *context, uint32_t precision, void *output, uint64_t count, double start,
                      double stop);
/* range (creation.hpp:157-168): the count of start, start + step, ... below stop (host only). */
uint64_t sci_cuda_range_count(uint32_t precision, double start, double stop, double step);
/* range: output[i] = start + element(i) * step in the element type, for that count. */
int sci_cuda_range(sci_cuda_context *context, uint32_t precision, void *output, uint64_t count, double start,
                   double step);
/* eye (creation.hpp:91-106): a rows x columns row-major matrix with ones on the main diagonal. */
int sci_cuda_eye(sci_cuda_context *context, uint32_t precision, void *output, uint64_t rows, uint64_t columns);
/* grid (creation.hpp:120-140, numpy.meshgrid): xx[i][j] = x[j], yy[i][j] = y[i], both ny x nx. */
int sci_cuda_grid(sci_cuda_context *context, uint32_t precision, const void *x, uint64_t nx, const void *y, uint64_t ny,
                  void *xx, void *yy);
/* decompose (include/linear/decompose.hpp:77-103, scipy.linalg.lu): A = P L U with the
 * factorisation (mode as sci_cuda_factor: SCI_FACTOR_PLAIN follows the reference's pivot order
 * step for step) and the split into dense factors on the device. matrix (unchanged) and the three
 * order x order outputs are device memory of the context; permutation[rows[c]][c] = 1. Waits. */
int sci_cuda_decompose(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *matrix,
                       void *permutation, void *lower, void *upper, uint64_t order);
/* transpose (include/operations/manipulations.hpp:33-62, numpy.transpose): output (extents in
 * reverse order) [j_{r-1}, ..., j_0] = input[j_0, ..., j_{r-1}], row-major, rank 1 to 8; output
 * must not be the input. */
int sci_cuda_transpose(sci_cuda_context *context, uint32_t precision, const void *input, uint32_t rank,
                       const uint64_t *shape, void *output);
/* Waits until every queued NVRTC specialisation has been compiled and loaded
 * (vulkan::Compiler::loop, src/core/drivers/vulkan/compiler.cpp:184-222, compiles in the
 * background the same way; a chunk runs on the interpreter until its kernel is ready).
 * SCI_CUDA_JIT=0 disables specialisation, =sync compiles on first use, =trace logs compiles. */
int sci_cuda_jit_wait(sci_cuda_context *context);

#ifdef __cplusplus
}
#endif

#endif /* SCI_CUDA_H */
