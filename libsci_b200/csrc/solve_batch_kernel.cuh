// solve_batch_kernel.cuh -- thousands of small independent solves, one CTA per system.
//
// Each system (n <= 256, one right-hand side, double operands) is factored in FP32 and refined in
// FP64 inside one CTA, with nothing but its matrix, right-hand side and solution in global memory:
//  - the FP32 copy of A lives in shared memory: columns [0, sc) of every row, sc = min(n, S), pitch
//    sc + 1; for n > S (the register variants, S = 192) thread r also holds columns [S, n) of row r
//    in registers (RC of them), so a 256 x 256 system fits one SM;
//  - LU with partial pivoting column by column, the reference's rules (include/linear/
//    decompose.hpp:29-72: the first row with the strictly largest |a|; a zero pivot skips the
//    column's elimination; l = a / pivot, a -= l * pivot_row with two roundings);
//  - refinement: x = 0, r = b; repeat { d = U^-1 L^-1 P r in FP32; x += d; r = b - A x in FP64 }
//    until the normwise backward error |r|_inf / (|A|_inf |x|_inf + |b|_inf) is at most 1e-15 or
//    stops halving (at most 30 corrections): the rule of sci_cuda_solve's refinement.
#pragma once

#include "sci_math.cuh"

namespace sci_cuda {

    struct SmallSystem {
        const double *a;  // n x n, row-major
        const double *b;  // n
        double *x;        // n
        unsigned n;
        unsigned pad;
    };

    constexpr int kSmallMax = 256;       // largest order
    constexpr int kSmallShared = 192;    // columns kept in shared memory by the register variant (a multiple of 32)
    constexpr int kSmallRegisters = kSmallMax - kSmallShared;

    // Shared memory of one launch for systems up to order `most`.
    inline unsigned long long small_shared_bytes(unsigned most, int rc) {
        const unsigned sc = rc > 0 ? (most < kSmallShared ? most : kSmallShared) : most;
        unsigned long long bytes = (4ull * most * (sc + 1) + 15) / 16 * 16;  // the FP32 matrix
        bytes += 2ull * 4 * (rc > 0 ? rc : 1);                              // pivot-row and swap buffers
        bytes = (bytes + 15) / 16 * 16;
        bytes += 8ull * most * 2;   // x, r (double)
        bytes += 4ull * most * 2;   // d (float), row order
        return bytes;
    }

    template <int T>
    __device__ __forceinline__ void block_argmax(float &m, int &row, float *vals, int *rows, int *winner) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int offset = 16; offset > 0; offset >>= 1) {
            const float om = __shfl_xor_sync(0xffffffffu, m, offset);
            const int orow = __shfl_xor_sync(0xffffffffu, row, offset);
            if (om > m || (om == m && orow < row)) {
                m = om;
                row = orow;
            }
        }
        if (T == 32) {
            if (lane == 0) *winner = row;
            __syncthreads();
            return;
        }
        if (lane == 0) {
            vals[warp] = m;
            rows[warp] = row;
        }
        __syncthreads();
        if (warp == 0) {
            m = lane < T / 32 ? vals[lane] : -1.0f;
            row = lane < T / 32 ? rows[lane] : 0x7fffffff;
#pragma unroll
            for (int offset = 16; offset > 0; offset >>= 1) {
                const float om = __shfl_xor_sync(0xffffffffu, m, offset);
                const int orow = __shfl_xor_sync(0xffffffffu, row, offset);
                if (om > m || (om == m && orow < row)) {
                    m = om;
                    row = orow;
                }
            }
            if (lane == 0) *winner = row;
        }
        __syncthreads();
    }

    template <int T>
    __device__ __forceinline__ double block_max(double v, double *scratch) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int offset = 16; offset > 0; offset >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, v, offset);
            v = (o > v || o != o) ? o : v;
        }
        __syncthreads();
        if (lane == 0) scratch[warp] = v;
        __syncthreads();
        double out = scratch[0];
        for (int w = 1; w < T / 32; ++w) out = (scratch[w] > out || scratch[w] != scratch[w]) ? scratch[w] : out;
        return out;
    }

    // Register column k of this thread's row, for a column index known only at run time.
    template <int RC> __device__ __forceinline__ float pick(const float *v, int k) {
        float out = 0.0f;
#pragma unroll
        for (int i = 0; i < RC; ++i)
            if (i == k) out = v[i];
        return out;
    }
    template <int RC> __device__ __forceinline__ void place(float *v, int k, float value) {
#pragma unroll
        for (int i = 0; i < RC; ++i)
            if (i == k) v[i] = value;
    }

    // A diagonal block of the blocked sweeps held in registers (columns sc + O .. sc + O + 31): its
    // rows belong to one warp, thread r holding row r's columns, so the block's triangle is solved
    // with shuffles and the rows beyond it read their own registers. Ends with a barrier.
    template <int O, int V>
    __device__ __forceinline__ void forward_block(const float (&v)[V], float *d, int b0, int bw, int n, int tid, int lane,
                                                  int warp) {
        if (warp == b0 / 32) {
            float di = lane < bw ? d[b0 + lane] : 0.0f;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < bw) {
                    const float y = __shfl_sync(0xffffffffu, di, j);
                    if (lane > j && lane < bw) di = sub(di, mul(v[O + j], y));
                }
            }
            if (lane < bw) d[b0 + lane] = di;
        }
        __syncthreads();
        if (tid >= b0 + bw && tid < n) {
            float acc = d[tid];
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j < bw) acc = sub(acc, mul(v[O + j], d[b0 + j]));
            d[tid] = acc;
        }
    }
    template <int O, int V>
    __device__ __forceinline__ void backward_block(const float (&v)[V], float *d, int b0, int bw, int n, int tid, int lane,
                                                   int warp) {
        if (warp == b0 / 32) {
            float di = lane < bw ? d[b0 + lane] : 0.0f;
#pragma unroll
            for (int j = 31; j >= 0; --j) {
                if (j < bw) {
                    const float own = lane == j ? div(di, v[O + j]) : di;
                    const float z = __shfl_sync(0xffffffffu, own, j);
                    if (lane == j) di = z;
                    else if (lane < j) di = sub(di, mul(v[O + j], z));
                }
            }
            if (lane < bw) d[b0 + lane] = di;
        }
        __syncthreads();
        if (tid < b0) {
            float acc = d[tid];
#pragma unroll
            for (int j = 31; j >= 0; --j)
                if (j < bw) acc = sub(acc, mul(v[O + j], d[b0 + j]));
            d[tid] = acc;
        }
    }

    template <int T, int RC>
    __global__ void __launch_bounds__(T) small_solve(const SmallSystem *systems, const unsigned *order, double *errors,
                                                     int *iterations) {
        constexpr int V = RC > 0 ? RC : 1;
        __shared__ float warp_vals[32];
        __shared__ int warp_rows[32];
        __shared__ int winner;
        __shared__ double reduce_scratch[32];
        extern __shared__ __align__(16) unsigned char small_shared[];

        const unsigned id = order[blockIdx.x];
        const SmallSystem sys = systems[id];
        const int n = static_cast<int>(sys.n);
        const int tid = threadIdx.x;
        const int sc = RC > 0 ? (n < kSmallShared ? n : kSmallShared) : n;  // shared-memory columns
        const int P = sc + 1;
        float *A = reinterpret_cast<float *>(small_shared);
        unsigned char *cursor = small_shared + (4ull * n * P + 15) / 16 * 16;
        float *pivot_reg = reinterpret_cast<float *>(cursor);
        float *swap_reg = pivot_reg + V;
        cursor += ((2 * 4 * V) + 15) / 16 * 16;
        double *x = reinterpret_cast<double *>(cursor);
        double *r = x + n;
        float *d = reinterpret_cast<float *>(r + n);
        int *rows = reinterpret_cast<int *>(d + n);
        // thread tid holds the register columns of row tid (only systems wider than the shared columns have any)
        const bool owner = RC > 0 && n > kSmallShared && tid < n;

        // load A in FP32 (and |A|_inf, |b|_inf in FP64)
        float v[V];
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = 0.0f;
        // one warp per row, each lane's loads of the row issued before its stores; the row's |a| sum
        // (for |A|_inf) comes from the same loads
        double row_sum = 0.0, b_max = 0.0;
        for (int row = tid >> 5; row < n; row += T / 32) {
            constexpr int G = kSmallMax / 32;
            double values[G];
#pragma unroll
            for (int u = 0; u < G; ++u) {
                const int col = (tid & 31) + 32 * u;
                values[u] = col < n ? sys.a[row * n + col] : 0.0;
            }
            double sum = 0.0;
#pragma unroll
            for (int u = 0; u < G; ++u) {
                const int col = (tid & 31) + 32 * u;
                if (col < sc) A[row * P + col] = static_cast<float>(values[u]);
                sum += fabs(values[u]);
            }
#pragma unroll
            for (int offset = 16; offset > 0; offset >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, offset);
            row_sum = (sum > row_sum || sum != sum) ? sum : row_sum;
        }
        if (RC > 0 && owner) {
#pragma unroll
            for (int k = 0; k < V; ++k)
                if (sc + k < n) v[k] = static_cast<float>(sys.a[tid * n + sc + k]);
        }
        for (int row = tid; row < n; row += T) {
            const double bv = fabs(sys.b[row]);
            b_max = (bv > b_max || bv != bv) ? bv : b_max;
        }
        const double a_norm = block_max<T>(row_sum, reduce_scratch);
        const double b_norm = block_max<T>(b_max, reduce_scratch);
        for (int i = tid; i < n; i += T) rows[i] = i;
        __syncthreads();

        // LU with partial pivoting
        for (int j = 0; j < n; ++j) {
            float best = -1.0f;
            int brow = 0x7fffffff;
            if (j < sc) {
                for (int row = j + tid; row < n; row += T) {
                    const float value = A[row * P + j];
                    const float m = fabsf(value);
                    // a NaN only stands at the pivot position, where every comparison fails
                    const float mag = m == m ? m : (row == j ? INFINITY : -1.0f);
                    if (mag > best || (mag == best && row < brow)) {
                        best = mag;
                        brow = row;
                    }
                }
            } else if (owner && tid >= j) {
                const float m = fabsf(pick<V>(v, j - sc));
                best = m == m ? m : (tid == j ? INFINITY : -1.0f);
                brow = tid;
            }
            block_argmax<T>(best, brow, warp_vals, warp_rows, &winner);
            int p = winner;
            if (p >= n || p < j) p = j;
            if (p != j) {
                for (int c = tid; c < sc; c += T) {
                    const float t0 = A[j * P + c];
                    A[j * P + c] = A[p * P + c];
                    A[p * P + c] = t0;
                }
                if (RC > 0 && n > sc) {
                    if (tid == p) {
#pragma unroll
                        for (int k = 0; k < V; ++k) swap_reg[k] = v[k];
                    }
                    if (tid == j) {
#pragma unroll
                        for (int k = 0; k < V; ++k) pivot_reg[k] = v[k];
                    }
                    __syncthreads();
                    if (tid == j) {
#pragma unroll
                        for (int k = 0; k < V; ++k) v[k] = swap_reg[k];
                    }
                    if (tid == p) {
#pragma unroll
                        for (int k = 0; k < V; ++k) v[k] = pivot_reg[k];
                    }
                }
                if (tid == 0) {
                    const int t0 = rows[j];
                    rows[j] = rows[p];
                    rows[p] = t0;
                }
            }
            __syncthreads();
            if (RC > 0 && n > sc) {
                if (tid == j) {
#pragma unroll
                    for (int k = 0; k < V; ++k) pivot_reg[k] = v[k];
                }
                __syncthreads();
            }
            const float diagonal = j < sc ? A[j * P + j] : pivot_reg[j - sc];
            if (diagonal != 0.0f) {
                // multipliers
                if (j < sc) {
                    for (int row = j + 1 + tid; row < n; row += T) A[row * P + j] = div(A[row * P + j], diagonal);
                } else if (owner && tid > j) {
                    place<V>(v, j - sc, div(pick<V>(v, j - sc), diagonal));
                }
                __syncthreads();
                // rank-1 update of the shared columns: lane l keeps the pivot row's columns
                // j + 1 + l + 32 u in registers for the whole step, and a warp walks its rows with every
                // load of a row issued before the row's stores (no chain through shared memory)
                if (j + 1 < sc) {
                    constexpr int G = kSmallMax / 32;
                    const int lane = tid & 31, cols = sc - j - 1;
                    float pivot[G];
#pragma unroll
                    for (int u = 0; u < G; ++u) pivot[u] = lane + 32 * u < cols ? A[j * P + j + 1 + lane + 32 * u] : 0.0f;
                    for (int row = j + 1 + tid / 32; row < n; row += T / 32) {
                        float *target = A + row * P + j + 1;
                        const float l = A[row * P + j];
                        float old[G];
#pragma unroll
                        for (int u = 0; u < G; ++u)
                            if (lane + 32 * u < cols) old[u] = target[lane + 32 * u];
#pragma unroll
                        for (int u = 0; u < G; ++u)
                            if (lane + 32 * u < cols) target[lane + 32 * u] = sub(old[u], mul(l, pivot[u]));
                    }
                }
                // and of this thread's register columns, in halves of 32 that hold live columns
                if (RC > 0 && owner && tid > j) {
                    const float l = j < sc ? A[tid * P + j] : pick<V>(v, j - sc);
#pragma unroll
                    for (int h = 0; h < V / 32; ++h) {
                        if (n > sc + 32 * h && j < sc + 32 * h + 31) {
#pragma unroll
                            for (int k = 32 * h; k < 32 * h + 32; ++k)
                                if (sc + k > j && sc + k < n) v[k] = sub(v[k], mul(l, pivot_reg[k]));
                        }
                    }
                }
            }
            __syncthreads();
        }

        // refinement
        for (int i = tid; i < n; i += T) {
            x[i] = 0.0;
            r[i] = sys.b[i];
        }
        __syncthreads();
        double berr = INFINITY, previous = INFINITY;
        int count = 0;
        const int lane = tid & 31, warp = tid >> 5;
        while (count < 30) {
            // d = P r in FP32
            for (int i = tid; i < n; i += T) d[i] = static_cast<float>(r[rows[i]]);
            __syncthreads();
            if (T >= n) {
                // Blocked sweeps: every 32-row block belongs to one warp (thread r holds row r), which
                // solves the block's triangle with shuffles; one barrier later the threads of the rows
                // beyond it apply the block. Each row sees its updates in the same order as the
                // column-by-column sweep below, so the result is the same to the bit.
                for (int b0 = 0; b0 < n; b0 += 32) {
                    const int bw = n - b0 < 32 ? n - b0 : 32;
                    if (b0 >= sc) {
                        if constexpr (RC > 0) {
                            if (b0 - sc == 0) forward_block<0>(v, d, b0, bw, n, tid, lane, warp);
                            else forward_block<32>(v, d, b0, bw, n, tid, lane, warp);
                        }
                    } else {
                        if (warp == b0 / 32) {
                            float di = lane < bw ? d[b0 + lane] : 0.0f;
                            for (int j = 0; j < bw; ++j) {
                                const float y = __shfl_sync(0xffffffffu, di, j);
                                if (lane > j && lane < bw) di = sub(di, mul(A[(b0 + lane) * P + b0 + j], y));
                            }
                            if (lane < bw) d[b0 + lane] = di;
                        }
                        __syncthreads();
                        if (tid >= b0 + bw && tid < n) {
                            float acc = d[tid];
                            for (int j = 0; j < bw; ++j) acc = sub(acc, mul(A[tid * P + b0 + j], d[b0 + j]));
                            d[tid] = acc;
                        }
                    }
                    __syncthreads();
                }
                for (int b0 = (n - 1) / 32 * 32; b0 >= 0; b0 -= 32) {
                    const int bw = n - b0 < 32 ? n - b0 : 32;
                    if (b0 >= sc) {
                        if constexpr (RC > 0) {
                            if (b0 - sc == 0) backward_block<0>(v, d, b0, bw, n, tid, lane, warp);
                            else backward_block<32>(v, d, b0, bw, n, tid, lane, warp);
                        }
                    } else {
                        if (warp == b0 / 32) {
                            float di = lane < bw ? d[b0 + lane] : 0.0f;
                            for (int j = bw - 1; j >= 0; --j) {
                                const float own = lane == j ? div(di, A[(b0 + j) * P + b0 + j]) : di;
                                const float z = __shfl_sync(0xffffffffu, own, j);
                                if (lane == j) di = z;
                                else if (lane < j) di = sub(di, mul(A[(b0 + lane) * P + b0 + j], z));
                            }
                            if (lane < bw) d[b0 + lane] = di;
                        }
                        __syncthreads();
                        if (tid < b0) {
                            float acc = d[tid];
                            for (int j = bw - 1; j >= 0; --j) {
                                const int col = b0 + j;
                                const float u = col < sc ? A[tid * P + col] : pick<V>(v, col - sc);
                                acc = sub(acc, mul(u, d[col]));
                            }
                            d[tid] = acc;
                        }
                    }
                    __syncthreads();
                }
            } else {
            // forward: unit lower, column by column
            for (int j = 0; j < n; ++j) {
                const float y = d[j];
                if (RC > 0) {
                    if (tid > j && tid < n) {
                        const float l = j < sc ? A[tid * P + j] : pick<V>(v, j - sc);
                        d[tid] = sub(d[tid], mul(l, y));
                    }
                } else {
                    for (int row = j + 1 + tid; row < n; row += T) d[row] = sub(d[row], mul(A[row * P + j], y));
                }
                __syncthreads();
            }
            // backward: upper
            for (int j = n - 1; j >= 0; --j) {
                float diagonal;
                if (RC > 0 && j >= sc) {  // U[j][j] is in thread j's registers
                    if (tid == j) pivot_reg[0] = pick<V>(v, j - sc);
                    __syncthreads();
                    diagonal = pivot_reg[0];
                } else {
                    diagonal = A[j * P + j];
                }
                const float z = div(d[j], diagonal);
                __syncthreads();
                if (tid == 0) d[j] = z;
                if (RC > 0) {
                    if (tid < j) {
                        const float ur = j < sc ? A[tid * P + j] : pick<V>(v, j - sc);
                        d[tid] = sub(d[tid], mul(ur, z));
                    }
                } else {
                    for (int row = tid; row < j; row += T) d[row] = sub(d[row], mul(A[row * P + j], z));
                }
                __syncthreads();
            }
            }
            // x += d; r = b - A x in FP64, one warp per row
            for (int i = tid; i < n; i += T) x[i] += static_cast<double>(d[i]);
            __syncthreads();
            double r_max = 0.0, x_max = 0.0;
            for (int row = warp; row < n; row += T / 32) {
                // every load of the row is issued before the first multiply
                constexpr int G = kSmallMax / 32;
                double values[G];
#pragma unroll
                for (int u = 0; u < G; ++u) values[u] = lane + 32 * u < n ? sys.a[row * n + lane + 32 * u] : 0.0;
                double s = 0.0;
#pragma unroll
                for (int u = 0; u < G; ++u)
                    if (lane + 32 * u < n) s = fma(values[u], x[lane + 32 * u], s);
#pragma unroll
                for (int offset = 16; offset > 0; offset >>= 1) s += __shfl_xor_sync(0xffffffffu, s, offset);
                const double residual = sys.b[row] - s;
                if (lane == 0) r[row] = residual;
                const double ar = fabs(residual);
                r_max = (ar > r_max || ar != ar) ? ar : r_max;
            }
            for (int i = tid; i < n; i += T) {
                const double ax = fabs(x[i]);
                x_max = (ax > x_max || ax != ax) ? ax : x_max;
            }
            r_max = block_max<T>(r_max, reduce_scratch);
            x_max = block_max<T>(x_max, reduce_scratch);
            __syncthreads();
            berr = r_max / (a_norm * x_max + b_norm);
            ++count;
            if (!(berr > 1e-15) || !(berr < 0.5 * previous)) break;
            previous = berr;
        }
        for (int i = tid; i < n; i += T) sys.x[i] = x[i];
        if (tid == 0) {
            if (errors) errors[id] = berr;
            if (iterations) iterations[id] = count;
        }
    }

} // namespace sci_cuda
