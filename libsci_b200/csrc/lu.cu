// lu.cu -- linear::factor / linear::solve on sm_100a, with FP64 iterative refinement.
//
// The reference factors in place, unblocked and right-looking, one row swap and one rank-1 update
// per column, on the host (include/linear/decompose.hpp:29-72), then substitutes forward through
// the unit lower triangle and back through the upper one (include/linear/solve.hpp:25-52). Pivoting
// is partial: the first row with the strictly largest |a| (decompose.hpp:35-38); a zero pivot is
// skipped (decompose.hpp:44-45). This file keeps those rules and blocks the work for the GPU:
//
//  for each outer block of 256 columns:
//    for each narrow panel of W columns (W = 32 float, 16 double) inside it:
//      1. panel_factor: one thread-block cluster (1 to 16 CTAs of 512 threads, by the rows left),
//         one panel row per thread held in registers (so up to 8192 rows). Per column: a warp
//         argmax, one CTA barrier, each CTA's candidate pushed into every CTA's inbox (st.async on
//         an mbarrier), every warp picks the pivot from its inbox and eliminates its own rows.
//      2. move_solve: the panel's net row movement applied to the block's other columns, and the
//         panel's U rows over the block's columns right of it.
//      3. rank_update: the rows below the panel, inside the block.
//    after the block: its row movements applied to the other columns (move_rows_all), its U rows
//    for the columns beyond it (block_rows_strip, once the block's pivots are final), then the
//    trailing update of everything right of and below it (GEMM, K = 256): on the tensor cores for
//    float (three-term bf16 split, six products, about FP32 accuracy, FP32 accumulation), or plain
//    FP32 / FP64 SIMT.
//
// solve with refinement (SCI_REFINE_FP64): the matrix is factored in FP32, then
//    x = 0, r = b;  repeat: solve LU d = P r in FP32; x += d;  r = b - A x in FP64
// until the normwise backward error |r|_inf / (|A|_inf |x|_inf + |b|_inf) of every column is at
// most sqrt(n) eps (eps = 2^-53, as LAPACK's DSGESV; at most 1e-14) or stops improving. Only the
// residual and the update run in FP64.
#include "context.hpp"
#include "workspace.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <vector>

namespace sci_cuda {

    namespace {

        constexpr unsigned long long kPanelRows = 8192;  // the panel cluster holds every row in registers
        constexpr unsigned long long kOuter = 256;
        // per-panel row movements of two outer blocks (by block parity: the side stream still applies
        // one block's while the next block's panels write theirs)
        constexpr int kMovements = 2 * static_cast<int>(kOuter / 16);
        constexpr int kSolveBlock = 128;

        template <typename T> struct PanelWidth {
            static constexpr int value = sizeof(T) == 4 ? 32 : 16;
        };

        // ---- cluster primitives ------------------------------------------------------------------
        __device__ __forceinline__ unsigned cluster_rank() {
            unsigned r;
            asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
            return r;
        }
        __device__ __forceinline__ void cluster_sync() {
            asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
        }
        // 16 bytes into another CTA's shared memory (a shared::cluster address from mapa), counted
        // as complete_tx bytes on that CTA's mbarrier `bar` (also a mapped address).
        __device__ __forceinline__ void send16(unsigned address, unsigned x, unsigned y, unsigned z, unsigned w, unsigned bar) {
            asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                                 address),
                         "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
                         : "memory");
        }
        __device__ __forceinline__ unsigned remote(const void *local, unsigned rank) {
            const unsigned address = static_cast<unsigned>(__cvta_generic_to_shared(local));
            unsigned mapped;
            asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(mapped) : "r"(address), "r"(rank));
            return mapped;
        }

        // The panel's net row movement: after its exchanges, row rows[i] holds what row src[i] held.
        // Only rows the panel touched appear (at most twice its width).
        struct Movement {
            long long count;
            long long rows[64];
            long long src[64];
        };

        // ---- pivot search keys ---------------------------------------------------------------------
        // A candidate's |value| as an unsigned key that orders like the value (non-negative floats
        // order like their bits), plus one so that a candidate of magnitude 0 still beats "no
        // candidate" (key 0). Rows are offsets from the panel's first row; kNoRow marks none. The
        // pivot is the largest key and, among equal keys, the lowest row: the reference's "first
        // strictly larger" scan (decompose.hpp:35-38).
        constexpr unsigned kNoRow = 0xFFFFFFFFu;
        template <typename T> struct MagnitudeKey;
        template <> struct MagnitudeKey<float> {
            using type = unsigned;
        };
        template <> struct MagnitudeKey<double> {
            using type = unsigned long long;
        };
        __device__ __forceinline__ unsigned magnitude_key(float m) { return __float_as_uint(m) + 1u; }
        __device__ __forceinline__ unsigned long long magnitude_key(double m) {
            return static_cast<unsigned long long>(__double_as_longlong(m)) + 1ull;
        }
        // Every lane of the warp ends with the warp's best (key, row): warp reductions of the key,
        // then of the row among the lanes that hold the best key.
        __device__ __forceinline__ void best_of_warp(unsigned &key, unsigned &rel) {
            const unsigned top = __reduce_max_sync(0xffffffffu, key);
            rel = __reduce_min_sync(0xffffffffu, key == top ? rel : kNoRow);
            key = top;
        }
        __device__ __forceinline__ void best_of_warp(unsigned long long &key, unsigned &rel) {
            const unsigned hi = static_cast<unsigned>(key >> 32), lo = static_cast<unsigned>(key);
            const unsigned top_hi = __reduce_max_sync(0xffffffffu, hi);
            const unsigned top_lo = __reduce_max_sync(0xffffffffu, hi == top_hi ? lo : 0u);
            const bool tie = hi == top_hi && lo == top_lo;
            rel = __reduce_min_sync(0xffffffffu, tie ? rel : kNoRow);
            key = (static_cast<unsigned long long>(top_hi) << 32) | top_lo;
        }
        template <int N> struct Span {
            static constexpr int value = N;
        };

        // The panel runs on one thread-block cluster of CL CTAs of 512 threads covering ROWS rows from
        // the panel's first: CTA c holds rows [ROWS c / CL, ROWS (c + 1) / CL), ROWS / (512 CL) rows
        // per thread. The full panel (ROWS = 8192) takes 8 CTAs, the portable size, or 16 where the
        // GPU can co-schedule them; a panel with fewer rows below its diagonal takes the smallest
        // cluster of 1, 2, 4 or 8 CTAs that holds them at one row per thread, so its per-column
        // exchange involves fewer CTAs (one CTA exchanges nothing across SMs).
        constexpr int kPanelBlock = 512;
        template <int CL, int ROWS = static_cast<int>(kPanelRows)> struct PanelShape {
            static constexpr int rows = ROWS / CL;  // rows per CTA
            static constexpr int per_thread = rows / kPanelBlock;
            static_assert(per_thread >= 1 && rows % kPanelBlock == 0, "whole rows per thread");
        };
        // Dynamic shared memory of panel_factor: the staged multipliers, W x (rows per CTA + 1).
        template <typename T, int CL, int ROWS = static_cast<int>(kPanelRows)> constexpr size_t panel_shared_bytes() {
            return sizeof(T) * PanelWidth<T>::value * (PanelShape<CL, ROWS>::rows + 1);
        }

        // Programmatic dependent launch along the factorisation's critical path: a kernel launched
        // with programmatic stream serialization (launch_chained) may start while the kernel before
        // it on the stream is still running; chain_wait() returns once that kernel has finished and
        // its writes are visible, and chain_release() lets the kernel after this one start. Both are
        // no-ops in a kernel launched the ordinary way.
        __device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
        __device__ __forceinline__ void chain_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

        // v[k] -= l * p[k] for k in [0, Q), each product and difference rounded on its own as in
        // the reference's column step (decompose.hpp:50-55); p is 16-byte aligned in shared memory.
        // Split in two: eliminate_head takes columns 0 and 1 (1 is the next column, whose pivot
        // search can then start), eliminate_tail columns [2, Q). Float rows go two columns per
        // instruction (mul / sub .rn.f32x2 round each lane exactly as the one-lane instructions
        // do). Column 0 is computed too: the caller overwrites it.
        __device__ __forceinline__ void eliminate_head(float *v, float l, const float *p) {
            const float2 q = *reinterpret_cast<const float2 *>(p);
            const Pair d = sub(pair(v[0], v[1]), mul(pair(l), pair(q.x, q.y)));
            unpair(d, v[0], v[1]);
        }
        template <int Q> __device__ __forceinline__ void eliminate_tail(float *v, float l, const float *p) {
            const Pair lp = pair(l);
            {
                const float2 q = *reinterpret_cast<const float2 *>(p + 2);
                const Pair d = sub(pair(v[2], v[3]), mul(lp, pair(q.x, q.y)));
                unpair(d, v[2], v[3]);
            }
#pragma unroll
            for (int k0 = 4; k0 < Q; k0 += 4) {
                const float4 q = *reinterpret_cast<const float4 *>(p + k0);
                const Pair d0 = sub(pair(v[k0], v[k0 + 1]), mul(lp, pair(q.x, q.y)));
                const Pair d1 = sub(pair(v[k0 + 2], v[k0 + 3]), mul(lp, pair(q.z, q.w)));
                unpair(d0, v[k0], v[k0 + 1]);
                unpair(d1, v[k0 + 2], v[k0 + 3]);
            }
        }
        __device__ __forceinline__ void eliminate_head(double *v, double l, const double *p) {
            v[0] = sub(v[0], mul(l, p[0]));
            v[1] = sub(v[1], mul(l, p[1]));
        }
        template <int Q> __device__ __forceinline__ void eliminate_tail(double *v, double l, const double *p) {
#pragma unroll
            for (int k0 = 2; k0 < Q; k0 += 2) {
                const double2 q = *reinterpret_cast<const double2 *>(p + k0);
                v[k0] = sub(v[k0], mul(l, q.x));
                v[k0 + 1] = sub(v[k0 + 1], mul(l, q.y));
            }
        }

        // W values (128 bytes) from a 16-byte aligned address.
        __device__ __forceinline__ void load_row(const float *p, float *v) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 x = reinterpret_cast<const float4 *>(p)[q];
                v[4 * q] = x.x;
                v[4 * q + 1] = x.y;
                v[4 * q + 2] = x.z;
                v[4 * q + 3] = x.w;
            }
        }
        __device__ __forceinline__ void load_row(const double *p, double *v) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double2 x = reinterpret_cast<const double2 *>(p)[q];
                v[2 * q] = x.x;
                v[2 * q + 1] = x.y;
            }
        }

        // Factors columns [j0, j0 + width) of rows [j0, n) in place; piv[j0 + j] = the row swapped into
        // position j0 + j, and *moved = the net movement of the panel's exchanges. One cluster of 8
        // CTAs of 512 threads, 1024 rows per CTA: thread t of CTA c holds rows j0 + 1024 c + t and
        // j0 + 1024 c + 512 + t, their panel values in registers, shifted left one column per step so
        // the current column is always v[i][0] (the column loop stays rolled: unrolled, every column
        // ran cold out of the instruction cache).
        //
        // Each finished value belongs to the row's original position (`origin`). A multiplier of L
        // whose row is still at its origin is staged in shared memory and written out coalesced at
        // the end; one of a row the exchanges moved, and each pivot row of U, goes to global memory
        // at once. A final permutation moves the at most 2 W displaced rows to their positions.
        //
        // Per column: each warp's best row is published in shared memory; after one CTA barrier,
        // warp 0 pushes the CTA's candidate with its values into every CTA's inbox (st.async,
        // counted on the receiver's mbarrier; CTA 0 also pushes the row at the pivot position);
        // then every warp of every CTA waits for its own inbox to fill (a bounded wait), picks the
        // pivot from it and eliminates, so the column takes one CTA barrier. A row's next column is
        // eliminated first and the warp's search for the next pivot issued at once, so the search's
        // latency overlaps the rest of the elimination. Inboxes and the published candidates
        // alternate by column parity; a CTA sends into an inbox again only after the barrier of the
        // column in between, which its warps reach only after reading every message of the earlier
        // column, and warp 0 reads a parity's candidates before the barrier after which the warps
        // publish into it again.
        template <typename T, int CL, int ROWS>
        __global__ void __launch_bounds__(kPanelBlock, 1)
                panel_factor(T *a, unsigned long long n, unsigned long long j0, int width, long long *piv, Movement *moved,
                             int *status) {
            constexpr int kClusterCtas = CL, kCtaRows = PanelShape<CL, ROWS>::rows;
            constexpr int W = PanelWidth<T>::value, R = PanelShape<CL, ROWS>::per_thread, TH = kPanelBlock, WARPS = TH / 32;
            constexpr int P = kCtaRows + 1;  // pitch of the staged multipliers
            extern __shared__ __align__(16) unsigned char panel_shared[];
            T *stage = reinterpret_cast<T *>(panel_shared);  // stage[k * P + local row]
            __shared__ unsigned home[kCtaRows];          // bit k: stage holds column k of the row
            using Key = typename MagnitudeKey<T>::type;
            __shared__ Key warp_key[2][WARPS];
            __shared__ unsigned warp_rel[2][WARPS];
            __shared__ unsigned long long warp_origin[2][WARPS];
            __shared__ __align__(16) T warp_values[2][WARPS][W];
            // The inbox, by column parity: slot q < CL holds CTA q's candidate (its values, then a
            // 16-byte head: key, then origin and row), slot CL the row at the pivot position (from
            // CTA 0). Rows are below 2^32 (n <= kPanelRows), so origin and row take 32 bits each.
            // Senders write it with st.async; inbox_bar[parity] counts the bytes.
            __shared__ __align__(16) T inbox[2][kClusterCtas + 1][W];
            __shared__ __align__(16) unsigned long long inbox_head[2][kClusterCtas + 1][2];
            __shared__ __align__(8) unsigned long long inbox_bar[2];
            __shared__ bool stalled;
            __shared__ __align__(16) T jbuf[2][W];  // CTA 0: the row at the pivot position
            __shared__ unsigned long long jbuf_origin[2];
            __shared__ long long exchanges[W];  // CTA 0: piv[j0 + j]
            // CTA 0: U's rows of the panel (row j from column j0 + j on, at u_rows[j][0, width - j)) and
            // the positions they are stored at until the final permutation, written out at the end
            __shared__ __align__(16) T u_rows[W][W];
            __shared__ unsigned long long u_origin[W];

            chain_wait();
            chain_release();
            const unsigned c = cluster_rank(), t = threadIdx.x, lane = t % 32, warp = t / 32;
            const unsigned long long first = j0 + 1ull * c * kCtaRows;  // this CTA's first row
            unsigned long long r[R], origin[R];
            bool valid[R];
            unsigned mask[R];
            T v[R][W];  // at step j: v[i][p] = column j0 + j + p of row i
            const bool vector = width == W && (n * sizeof(T)) % 16 == 0;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                r[i] = first + 1ull * i * TH + t;
                valid[i] = r[i] < n;
                origin[i] = r[i];
                mask[i] = 0;
                if (valid[i] && vector) {
                    load_row(a + r[i] * n + j0, v[i]);
                } else {
#pragma unroll
                    for (int k = 0; k < W; ++k) v[i][k] = (valid[i] && k < width) ? a[r[i] * n + j0 + k] : T(0);
                }
            }

            // The warp's candidate for the column whose values sit at v[i][O], among rows `from` on: the
            // best key and row, published by lane 0 at `parity`; returns the row (kNoRow: none). A NaN
            // only stands at the pivot position itself, where the reference's comparisons against it
            // all fail (decompose.hpp:35-38).
            auto search = [&](auto offset, const int parity, const unsigned long long from) -> unsigned {
                constexpr int O = decltype(offset)::value;
                Key key = 0;
                unsigned rel = kNoRow;
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    if (valid[i] && r[i] >= from) {
                        const T m = fabs(v[i][O]);
                        const bool candidate = m == m || r[i] == from;
                        const Key k = candidate ? magnitude_key(m == m ? m : T(INFINITY)) : Key(0);
                        const unsigned at = static_cast<unsigned>(r[i] - j0);
                        if (k > key || (k == key && k != 0 && at < rel)) {
                            key = k;
                            rel = at;
                        }
                    }
                }
                best_of_warp(key, rel);
                if (lane == 0) {
                    warp_key[parity][warp] = key;
                    warp_rel[parity][warp] = rel;
                }
                return rel;
            };
            // The winning lane's values from v[i][O] on (Q of them, zero past the row's W) and origin at
            // `parity`; in CTA 0 the thread holding row `from` (the next pivot position) stages it too.
            auto stage_candidate = [&](auto offset, auto span, const int parity, const unsigned rel,
                                       const unsigned long long from) {
                constexpr int O = decltype(offset)::value, Q = decltype(span)::value;
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    if (rel != kNoRow && r[i] - j0 == rel) {
#pragma unroll
                        for (int k = 0; k < Q; ++k) warp_values[parity][warp][k] = k + O < W ? v[i][k + O] : T(0);
                        warp_origin[parity][warp] = origin[i];
                    }
                }
                if (c == 0 && t == static_cast<unsigned>(from - j0)) {  // row `from` is row 0 of that thread
#pragma unroll
                    for (int k = 0; k < Q; ++k) jbuf[parity][k] = k + O < W ? v[0][k + O] : T(0);
                    jbuf_origin[parity] = origin[0];
                }
            };

            // One column step, specialised on Q >= width - j: after j shifts only v[i][0, width - j)
            // is live (the rest is zero), so publication, elimination and the shift stop at Q. The
            // column's candidates were published (parity j & 1) by the step before, or before the loop.
            auto column = [&](auto span, const int j) {
                constexpr int Q = decltype(span)::value;
                const int par = j & 1;
                const unsigned long long row_j = j0 + j;
                __syncthreads();  // every warp's candidate (and CTA 0's pivot-position row) is staged
                // 1. warp 0: the CTA's candidate; lane q sends it to CTA q (and lane q of CTA 0's warp 1
                //    the pivot-position row), 16 bytes per store, the message's words read from shared
                //    memory before the first store. A slot of parity par is rewritten two columns later, after every
                //    reader has taken its pivot from it (each CTA's next message follows its own
                //    barrier of the column in between, which its warps reach only after reading).
                constexpr unsigned kValueBytes = Q * sizeof(T), kMessage = kValueBytes + 16;
                static_assert(kValueBytes % 16 == 0, "16-byte stores");
                // One message: the values, then a 16-byte head (key; origin and row, 32 bits each).
                auto send = [&](const T *values, unsigned slot, unsigned long long k, unsigned long long o, unsigned rw) {
                    const unsigned bar = remote(&inbox_bar[par], lane);
                    uint4 words[kValueBytes / 16];
#pragma unroll
                    for (unsigned m = 0; m < kValueBytes / 16; ++m) words[m] = reinterpret_cast<const uint4 *>(values)[m];
                    const unsigned base = remote(&inbox[par][slot][0], lane);
                    const unsigned head = remote(&inbox_head[par][slot][0], lane);
#pragma unroll
                    for (unsigned m = 0; m < kValueBytes / 16; ++m)
                        send16(base + 16 * m, words[m].x, words[m].y, words[m].z, words[m].w, bar);
                    send16(head, static_cast<unsigned>(k), static_cast<unsigned>(k >> 32), static_cast<unsigned>(o), rw, bar);
                };
                if (warp == 0) {
                    Key k2 = lane < WARPS ? warp_key[par][lane] : Key(0);
                    unsigned r2 = lane < WARPS ? warp_rel[par][lane] : kNoRow;
                    best_of_warp(k2, r2);
                    const unsigned source = r2 == kNoRow ? 0u : ((r2 - c * kCtaRows) % TH) / 32;
                    if (lane < static_cast<unsigned>(kClusterCtas))
                        send(warp_values[par][source], c, static_cast<unsigned long long>(k2), warp_origin[par][source], r2);
                    if (lane == 0) barrier_expect(&inbox_bar[par], (kClusterCtas + 1) * kMessage);
                } else if (warp == 1 && c == 0 && lane < static_cast<unsigned>(kClusterCtas)) {
                    // CTA 0's pivot-position row, from another warp (another scheduler) at the same time
                    send(jbuf[par], kClusterCtas, 0ull, jbuf_origin[par], 0u);
                }
                // 2. every warp waits for its CTA's inbox to fill (a bounded wait: one that runs out
                //    flags the status, and no later column waits) and takes the pivot from it
                if (!stalled && !barrier_wait(&inbox_bar[par], static_cast<unsigned>(j >> 1) & 1u) && lane == 0) {
                    stalled = true;
                    atomicOr(status, kStatusTimeout);
                }
                __syncwarp();
                Key k3 = 0;
                unsigned r3 = kNoRow;
                unsigned long long org = 0;
                if (lane < kClusterCtas) {
                    k3 = static_cast<Key>(inbox_head[par][lane][0]);
                    const unsigned long long where = inbox_head[par][lane][1];
                    org = where & 0xFFFFFFFFull;
                    r3 = static_cast<unsigned>(where >> 32);
                }
                best_of_warp(k3, r3);
                // the winner's CTA owns its row; no candidate cannot happen (row_j is one)
                const unsigned q = r3 == kNoRow ? 0u : r3 / kCtaRows;
                org = __shfl_sync(0xffffffffu, org, q);
                const unsigned long long prow = r3 == kNoRow ? row_j : j0 + r3;
                const T *const pivot_row = inbox[par][q];
                if (c == 0 && t == 0) exchanges[j] = static_cast<long long>(prow);
                constexpr int E = 16 / sizeof(T);  // pivot-row values per 16-byte load
                const T diagonal = pivot_row[0];
                T l[R];
                bool below[R];
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    if (r[i] == prow && prow != row_j) {
                        // this row moves to the pivot's old place: it takes the displaced row's values
#pragma unroll
                        for (int k = 0; k < Q; k += E) load16(&inbox[par][kClusterCtas][k], &v[i][k]);
                        origin[i] = inbox_head[par][kClusterCtas][1] & 0xFFFFFFFFull;
                    }
                    if (r[i] == row_j) {
                        // the pivot row is final: U's row j0 + j from column j0 + j on, kept for the end
                        // (16-byte shared stores here instead of Q scalar global stores in the
                        // column's critical warp)
#pragma unroll
                        for (int k = 0; k < Q; k += E)
                            *reinterpret_cast<uint4 *>(&u_rows[j][k]) = *reinterpret_cast<const uint4 *>(pivot_row + k);
                        origin[i] = org;
                        u_origin[j] = org;
                    }
                    // 3. eliminate below the pivot: l = a / pivot; a[k] -= l * pivot_row[k]; a zero
                    //    pivot leaves the column as it is (decompose.hpp:44-45). The next column
                    //    (v[i][1]) first.
                    below[i] = valid[i] && r[i] > row_j;
                    l[i] = v[i][0];
                    if (below[i] && diagonal != T(0)) {
                        l[i] = div(v[i][0], diagonal);
                        eliminate_head(v[i], l[i], pivot_row);
                    }
                }
                // 4. the next column's search, while the rest of the elimination runs
                const bool more = j + 1 < width;
                const unsigned next_rel = more ? search(Span<1>{}, par ^ 1, row_j + 1) : kNoRow;
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    if (below[i] && diagonal != T(0)) eliminate_tail<Q>(v[i], l[i], pivot_row);
                    if (below[i]) {
                        v[i][0] = l[i];
                        if (origin[i] == r[i]) {
                            stage[j * P + static_cast<int>(r[i] - first)] = l[i];
                            mask[i] |= 1u << j;
                        } else {
                            a[origin[i] * n + row_j] = l[i];
                        }
                    }
                }
                if (more) stage_candidate(Span<1>{}, span, par ^ 1, next_rel, row_j + 1);
#pragma unroll
                for (int i = 0; i < R; ++i) {
#pragma unroll
                    for (int k = 0; k + 1 < Q; ++k) v[i][k] = v[i][k + 1];
                    v[i][Q - 1] = T(0);
                }
            };
            if (t == 0) {
                barrier_init(&inbox_bar[0], 1);
                barrier_init(&inbox_bar[1], 1);
                stalled = false;
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            // column 0's candidates
            stage_candidate(Span<0>{}, Span<W>{}, 0, search(Span<0>{}, 0, j0), j0);
            cluster_sync();  // every CTA's inbox barriers exist before the first message
#pragma unroll 1
            for (int j = 0; j < width; ++j) {
                const int live = width - j;
                if (live > 3 * W / 4) column(Span<W>{}, j);
                else if (live > W / 2) column(Span<3 * W / 4>{}, j);
                else if (live > W / 4) column(Span<W / 2>{}, j);
                else column(Span<W / 4>{}, j);
            }
            // The staged multipliers, one row per warp store. Then every row's panel values sit at the
            // position the row started in; move the rows the exchanges displaced: all reads, a
            // cluster barrier, then all writes.
#pragma unroll
            for (int i = 0; i < R; ++i) home[r[i] - first] = mask[i];
            __syncthreads();
            for (int row = warp; row < kCtaRows; row += WARPS) {
                const unsigned long long g = first + row;
                if (g >= n) break;
                if (lane < static_cast<unsigned>(width) && (home[row] >> lane & 1u)) a[g * n + j0 + lane] = stage[lane * P + row];
            }
            if (c == 0) {
                // U's rows, at the positions the pivot rows started in (moved with them below)
                for (int j = warp; j < width; j += WARPS)
                    if (lane < static_cast<unsigned>(width - j)) a[u_origin[j] * n + j0 + j + lane] = u_rows[j][lane];
            }
            __threadfence();
            cluster_sync();
#pragma unroll
            for (int i = 0; i < R; ++i) {
                if (valid[i] && origin[i] != r[i]) {
#pragma unroll
                    for (int k = 0; k < W; ++k) v[i][k] = k < width ? a[origin[i] * n + j0 + k] : T(0);
                }
            }
            cluster_sync();  // also: no CTA leaves while another may still read its shared memory
#pragma unroll
            for (int i = 0; i < R; ++i) {
                if (valid[i] && origin[i] != r[i]) {
#pragma unroll
                    for (int k = 0; k < W; ++k)
                        if (k < width) a[r[i] * n + j0 + k] = v[i][k];
                }
            }
            if (c == 0 && warp == 0) {
                // The net movement of rows: the exchanges applied in order to a table of the rows they
                // touch (at most 2W), one warp, each lane holding two table entries.
                __syncwarp();
                long long row_a = lane < static_cast<unsigned>(width) ? static_cast<long long>(j0 + lane) : -1;
                long long row_b = -1;
                long long src_a = row_a, src_b = -1;
                int count = width;
                if (lane < static_cast<unsigned>(width)) piv[j0 + lane] = exchanges[lane];
                for (int j = 0; j < width; ++j) {
                    const long long p = exchanges[j];
                    // where p sits in the table: entry index, or -1
                    const unsigned in_a = __ballot_sync(0xffffffffu, row_a == p);
                    const unsigned in_b = __ballot_sync(0xffffffffu, row_b == p);
                    int at = in_a ? __ffs(in_a) - 1 : (in_b ? 32 + __ffs(in_b) - 1 : -1);
                    if (at < 0) {
                        at = count++;
                        if (at < 32) {
                            if (lane == static_cast<unsigned>(at)) row_a = src_a = p;
                        } else if (lane == static_cast<unsigned>(at - 32)) {
                            row_b = src_b = p;
                        }
                    }
                    // exchange the contents of entries j and at
                    const long long from_j = __shfl_sync(0xffffffffu, src_a, j);
                    const long long from_at = at < 32 ? __shfl_sync(0xffffffffu, src_a, at & 31)
                                                      : __shfl_sync(0xffffffffu, src_b, at & 31);
                    if (lane == static_cast<unsigned>(j)) src_a = from_at;
                    if (at < 32) {
                        if (lane == static_cast<unsigned>(at)) src_a = from_j;
                    } else if (lane == static_cast<unsigned>(at - 32)) {
                        src_b = from_j;
                    }
                }
                // keep the entries that moved, in order
                const bool keep_a = static_cast<int>(lane) < count && row_a != src_a;
                const bool keep_b = static_cast<int>(lane) + 32 < count && row_b != src_b;
                const unsigned mask_a = __ballot_sync(0xffffffffu, keep_a), mask_b = __ballot_sync(0xffffffffu, keep_b);
                const unsigned below = (1u << lane) - 1u;
                if (keep_a) {
                    const int slot = __popc(mask_a & below);
                    moved->rows[slot] = row_a;
                    moved->src[slot] = src_a;
                }
                if (keep_b) {
                    const int slot = __popc(mask_a) + __popc(mask_b & below);
                    moved->rows[slot] = row_b;
                    moved->src[slot] = src_b;
                }
                if (lane == 0) moved->count = __popc(mask_a) + __popc(mask_b);
            }
        }

        // Launches panel_factor<T, CL, ROWS> as one cluster of CL CTAs (chained: see chain_wait).
        template <typename T, int CL, int ROWS = static_cast<int>(kPanelRows)>
        cudaError_t launch_panel(cudaStream_t stream, T *a, unsigned long long n, unsigned long long j0, int w, long long *piv,
                                 Movement *moved, int *status, bool chained = false) {
            cudaLaunchConfig_t config{};
            config.gridDim = dim3(CL);
            config.blockDim = dim3(kPanelBlock);
            config.dynamicSmemBytes = panel_shared_bytes<T, CL, ROWS>();
            config.stream = stream;
            cudaLaunchAttribute attribute[2];
            attribute[0].id = cudaLaunchAttributeClusterDimension;
            attribute[0].val.clusterDim.x = CL;
            attribute[0].val.clusterDim.y = 1;
            attribute[0].val.clusterDim.z = 1;
            attribute[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attribute[1].val.programmaticStreamSerializationAllowed = 1;
            config.attrs = attribute;
            config.numAttrs = chained ? 2 : 1;
            return cudaLaunchKernelEx(&config, panel_factor<T, CL, ROWS>, a, n, j0, w, piv, moved, status);
        }

        // Raises the dynamic shared-memory limit of the short panels (one row per thread) once.
        template <typename T> void prepare_short_panels() {
            static const bool done = [] {
                cudaFuncSetAttribute(reinterpret_cast<const void *>(&panel_factor<T, 1, 512>),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(panel_shared_bytes<T, 1, 512>()));
                cudaFuncSetAttribute(reinterpret_cast<const void *>(&panel_factor<T, 2, 1024>),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(panel_shared_bytes<T, 2, 1024>()));
                cudaFuncSetAttribute(reinterpret_cast<const void *>(&panel_factor<T, 4, 2048>),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(panel_shared_bytes<T, 4, 2048>()));
                cudaFuncSetAttribute(reinterpret_cast<const void *>(&panel_factor<T, 8, 4096>),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(panel_shared_bytes<T, 8, 4096>()));
                return true;
            }();
            (void)done;
        }

        // The panel at columns [j0, j0 + w): the smallest cluster that holds its n - j0 rows at one
        // row per thread, or the full panel's cluster (`cluster` CTAs, 8192 rows).
        template <typename T>
        cudaError_t launch_panel_for(int cluster, cudaStream_t stream, T *a, unsigned long long n, unsigned long long j0, int w,
                                     long long *piv, Movement *moved, int *status, bool chained) {
            const unsigned long long rows = n - j0;
            prepare_short_panels<T>();
            if (rows <= 512) return launch_panel<T, 1, 512>(stream, a, n, j0, w, piv, moved, status, chained);
            if (rows <= 1024) return launch_panel<T, 2, 1024>(stream, a, n, j0, w, piv, moved, status, chained);
            if (rows <= 2048) return launch_panel<T, 4, 2048>(stream, a, n, j0, w, piv, moved, status, chained);
            if (rows <= 4096 && cluster == 16) return launch_panel<T, 8, 4096>(stream, a, n, j0, w, piv, moved, status, chained);
            return cluster == 16 ? launch_panel<T, 16>(stream, a, n, j0, w, piv, moved, status, chained)
                                 : launch_panel<T, 8>(stream, a, n, j0, w, piv, moved, status, chained);
        }

        // Launches `kernel` on `stream` with programmatic stream serialization, for kernels that
        // call chain_wait() before reading what the kernel before them wrote.
        template <typename... Params, typename... Args>
        cudaError_t launch_chained_shared(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                          Args... args) {
            cudaLaunchConfig_t config{};
            config.gridDim = grid;
            config.blockDim = block;
            config.dynamicSmemBytes = smem;
            config.stream = stream;
            cudaLaunchAttribute attribute[1];
            attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attribute[0].val.programmaticStreamSerializationAllowed = 1;
            config.attrs = attribute;
            config.numAttrs = 1;
            return cudaLaunchKernelEx(&config, kernel, static_cast<Params>(args)...);
        }
        template <typename... Params, typename... Args>
        cudaError_t launch_chained(void (*kernel)(Params...), dim3 grid, dim3 block, cudaStream_t stream, Args... args) {
            cudaLaunchConfig_t config{};
            config.gridDim = grid;
            config.blockDim = block;
            config.dynamicSmemBytes = 0;
            config.stream = stream;
            cudaLaunchAttribute attribute[1];
            attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attribute[0].val.programmaticStreamSerializationAllowed = 1;
            config.attrs = attribute;
            config.numAttrs = 1;
            return cudaLaunchKernelEx(&config, kernel, static_cast<Params>(args)...);
        }

        // The panel's cluster size for this process: 16 CTAs (half the rows per SM, a non-portable
        // cluster size) when the GPU can schedule such a cluster, else 8; SCI_CUDA_PANEL_CLUSTER=8 or
        // 16 asks for one. 0 when neither can run. Decided once per element type.
        template <typename T> int panel_cluster() {
            static const int chosen = [] {
                const int smem8 = static_cast<int>(panel_shared_bytes<T, 8>()), smem16 = static_cast<int>(panel_shared_bytes<T, 16>());
                const void *full8 = reinterpret_cast<const void *>(&panel_factor<T, 8, static_cast<int>(kPanelRows)>);
                const void *full16 = reinterpret_cast<const void *>(&panel_factor<T, 16, static_cast<int>(kPanelRows)>);
                cudaFuncSetAttribute(full8, cudaFuncAttributeMaxDynamicSharedMemorySize, smem8);
                cudaFuncSetAttribute(full16, cudaFuncAttributeMaxDynamicSharedMemorySize, smem16);
                cudaFuncSetAttribute(full16, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
                auto schedulable = [](const void *kernel, int cl, int smem) {
                    cudaLaunchConfig_t config{};
                    config.gridDim = dim3(cl);
                    config.blockDim = dim3(kPanelBlock);
                    config.dynamicSmemBytes = smem;
                    cudaLaunchAttribute attribute[1];
                    attribute[0].id = cudaLaunchAttributeClusterDimension;
                    attribute[0].val.clusterDim.x = cl;
                    attribute[0].val.clusterDim.y = 1;
                    attribute[0].val.clusterDim.z = 1;
                    config.attrs = attribute;
                    config.numAttrs = 1;
                    int clusters = 0;
                    if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &config) != cudaSuccess) {
                        cudaGetLastError();
                        return false;
                    }
                    return clusters >= 1;
                };
                const bool can16 = schedulable(full16, 16, smem16);
                const bool can8 = schedulable(full8, 8, smem8);
                const char *asked = std::getenv("SCI_CUDA_PANEL_CLUSTER");
                if (asked && std::atoi(asked) == 8 && can8) return 8;
                if (can16) return 16;
                return can8 ? 8 : 0;
            }();
            return chosen;
        }

        // The panels' net row movements for `count` movements in turn (a block's panels, in their
        // order) over the columns [c0, c1). One CTA of 256 threads per 32 columns: lane l takes column
        // l of the CTA's 32 and warp g the movement's entries g, g + 8, ..., so a row's 32 columns are
        // one coalesced 128-byte access; per movement all reads, a barrier, all writes, a barrier
        // (each movement sees the one before it).
        template <typename T>
        __global__ void __launch_bounds__(256) move_rows_all(T *a, unsigned long long n, const Movement *moved, int count,
                                                            unsigned long long c0, unsigned long long c1) {
            const int lane = static_cast<int>(threadIdx.x % 32), g = static_cast<int>(threadIdx.x / 32);
            const unsigned long long col = c0 + blockIdx.x * 32ull + lane;
            const bool active = col < c1;
            for (int p = 0; p < count; ++p) {
                const int rows = static_cast<int>(moved[p].count);
                T values[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int e = g + 8 * u;
                    if (active && e < rows) values[u] = a[static_cast<unsigned long long>(moved[p].src[e]) * n + col];
                }
                __syncthreads();
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int e = g + 8 * u;
                    if (active && e < rows) a[static_cast<unsigned long long>(moved[p].rows[e]) * n + col] = values[u];
                }
                __syncthreads();
            }
        }

        // order[i] = i: the row order before the first exchange.
        __global__ void identity_rows(unsigned *order, unsigned long long n) {
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < n; i += 256ull * gridDim.x)
                order[i] = static_cast<unsigned>(i);
        }

        // x[i][:] = (U) b[rows[i]][:], optionally narrowing double to float: P b for the substitution.
        template <typename S, typename D>
        __global__ void gather_rows(const S *b, D *x, const unsigned *rows, unsigned long long n, unsigned long long width) {
            const unsigned long long total = n * width;
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < total; i += 256ull * gridDim.x) {
                const unsigned long long row = i / width, column = i % width;
                x[i] = static_cast<D>(b[static_cast<unsigned long long>(rows[row]) * width + column]);
            }
        }

        // C (m x n, pitch ldc) -= A (m x k, pitch lda) * B (k x n, pitch ldb) for small k: 64 x BN tiles,
        // K in slices of 32 through shared memory, 4 x (BN / 16) outputs per thread.
        template <typename T, int BN>
        __global__ void __launch_bounds__(256) rank_update(const T *__restrict__ a, unsigned long long lda,
                                                           const T *__restrict__ b, unsigned long long ldb, T *c,
                                                           unsigned long long ldc, unsigned long long m, unsigned long long n,
                                                           unsigned long long k) {
            constexpr int BM = 64, BK = 32, TN = BN / 16, LA = BM * BK / 256, LB = BK * BN / 256;
            __shared__ T as[BK][BM + 1];
            __shared__ T bs[BK][BN + 1];
            chain_wait();
            chain_release();
            const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
            const unsigned long long m0 = blockIdx.y * 1ull * BM, n0 = blockIdx.x * 1ull * BN;
            T acc[4][TN];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
            // Each K slice is loaded into registers (all of a thread's loads in flight together) while
            // the previous one is multiplied out of shared memory.
            T ra[LA], rb[LB];
            auto fetch = [&](unsigned long long k0) {
#pragma unroll
                for (int u = 0; u < LA; ++u) {
                    const int i = threadIdx.x + u * 256, row = i / BK, q = i % BK;
                    const unsigned long long gr = m0 + row, gk = k0 + q;
                    ra[u] = (gr < m && gk < k) ? a[gr * lda + gk] : T(0);
                }
#pragma unroll
                for (int u = 0; u < LB; ++u) {
                    const int i = threadIdx.x + u * 256, q = i / BN, col = i % BN;
                    const unsigned long long gk = k0 + q, gc = n0 + col;
                    rb[u] = (gk < k && gc < n) ? b[gk * ldb + gc] : T(0);
                }
            };
            fetch(0);
            // the thread's outputs as they are, loaded with the first slice (one wait for both)
            T old[4][TN];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const unsigned long long row = m0 + ty * 4 + i;
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    const unsigned long long col = n0 + tx * TN + j;
                    old[i][j] = (row < m && col < n) ? c[row * ldc + col] : T(0);
                }
            }
            for (unsigned long long k0 = 0; k0 < k; k0 += BK) {
#pragma unroll
                for (int u = 0; u < LA; ++u) {
                    const int i = threadIdx.x + u * 256;
                    as[i % BK][i / BK] = ra[u];
                }
#pragma unroll
                for (int u = 0; u < LB; ++u) {
                    const int i = threadIdx.x + u * 256;
                    bs[i / BN][i % BN] = rb[u];
                }
                __syncthreads();
                if (k0 + BK < k) fetch(k0 + BK);
#pragma unroll 8
                for (int q = 0; q < BK; ++q) {
                    T av[4], bv[TN];
#pragma unroll
                    for (int i = 0; i < 4; ++i) av[i] = as[q][ty * 4 + i];
#pragma unroll
                    for (int j = 0; j < TN; ++j) bv[j] = bs[q][tx * TN + j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) acc[i][j] = fma_(av[i], bv[j], acc[i][j]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const unsigned long long row = m0 + ty * 4 + i;
                if (row >= m) continue;
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    const unsigned long long col = n0 + tx * TN + j;
                    if (col < n) c[row * ldc + col] = sub(old[i][j], acc[i][j]);
                }
            }
        }

        template <typename T>
        int update(Context &ctx, const T *a, unsigned long long lda, const T *b, unsigned long long ldb, T *c,
                   unsigned long long ldc, unsigned long long m, unsigned long long n, unsigned long long k,
                   bool chained = false) {
            if (m == 0 || n == 0 || k == 0) return SCI_CUDA_OK;
            if ((m + 63) / 64 > 65535) return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "update: too many rows");
            const bool narrow = n <= 16;
            const dim3 grid(static_cast<unsigned>(narrow ? (n + 15) / 16 : (n + 63) / 64), static_cast<unsigned>((m + 63) / 64));
            if (chained) {
                const cudaError_t launched = narrow ? launch_chained(rank_update<T, 16>, grid, dim3(256), ctx.stream, a, lda, b,
                                                                     ldb, c, ldc, m, n, k)
                                                    : launch_chained(rank_update<T, 64>, grid, dim3(256), ctx.stream, a, lda, b,
                                                                     ldb, c, ldc, m, n, k);
                return ctx.check(launched, "launching a rank update");
            }
            if (narrow) {
                rank_update<T, 16><<<grid, 256, 0, ctx.stream>>>(a, lda, b, ldb, c, ldc, m, n, k);
            } else {
                rank_update<T, 64><<<grid, 256, 0, ctx.stream>>>(a, lda, b, ldb, c, ldc, m, n, k);
            }
            return ctx.check(cudaGetLastError(), "launching a rank update");
        }

        // Rows [J0, J0 + ob) of columns [c0, c1) := L11^-1 times themselves, L11 the block's unit lower
        // triangle (ob <= kOuter): the U rows of a block over other columns. The same steps, rounded
        // the same way, as a chain of move_solve's solve (a panel's W rows in order) and rank_update
        // (the rows below the panel minus the sum, in order, of the panel's products), in one launch:
        // one CTA of 256 threads per strip of CS columns holds the strip's block rows in shared
        // memory: CS = 16 for the bulk of the columns (each CTA reads the whole triangle), CS = 4 for
        // the next block's columns on the critical path (more CTAs, a quarter of the update per
        // panel). Per panel: warp w < CS / 4 solves columns [4 w, 4 w + 4) with eight lanes per
        // column, lane l % 8 holding rows l % 8, + 8, ... of the panel (the owner of row k hands its
        // value to the column's lanes, which subtract its product from their later rows); then each
        // thread takes (row below, four columns) items with the row's W multipliers in registers.
        constexpr int kStripColumns = 16, kStripColumnsNarrow = 4, kStripRows = 256;
        template <typename T, int CS> constexpr size_t strip_shared_bytes() {
            return sizeof(T) * kStripRows * ((CS + 16 / sizeof(T)) + (PanelWidth<T>::value + 16 / sizeof(T)));
        }
        template <typename T> __device__ __forceinline__ void load4(const T *p, T *v) {
            if constexpr (sizeof(T) == 4) {
                load16(p, v);
            } else {
                load16(p, v);
                load16(p + 2, v + 2);
            }
        }
        template <typename T, int CS>
        __global__ void __launch_bounds__(256) block_rows_strip(T *a, unsigned long long n, unsigned long long J0, int ob,
                                                               unsigned long long c0, unsigned long long c1) {
            constexpr int W = PanelWidth<T>::value, RW = kStripRows;
            constexpr int XP = CS + 16 / sizeof(T), LP = W + 16 / sizeof(T);  // 16-byte aligned rows
            constexpr int PER = W / 8;  // panel rows per lane in the solve
            extern __shared__ __align__(16) unsigned char strip_shared[];
            T *const x = reinterpret_cast<T *>(strip_shared);  // x[row * XP + column]: the strip's block rows
            T *const l = x + RW * XP;                           // l[row * LP + q] = L[p0 + row][p0 + q]
            chain_wait();
            chain_release();
            const int t = threadIdx.x, lane = t % 32, warp = t / 32;
            const unsigned long long s0 = c0 + blockIdx.x * 1ull * CS;
            // the strip's block rows; rows past ob are zero (a padded panel multiplies them by zero).
            // Every global load of a thread is issued before its first shared store.
            {
                T staged[RW * CS / 256];
#pragma unroll
                for (int u = 0; u < RW * CS / 256; ++u) {
                    const int i = t + u * 256, row = i / CS, col = i % CS;
                    staged[u] = (row < ob && s0 + col < c1) ? a[(J0 + row) * n + s0 + col] : T(0);
                }
#pragma unroll
                for (int u = 0; u < RW * CS / 256; ++u) {
                    const int i = t + u * 256;
                    x[(i / CS) * XP + i % CS] = staged[u];
                }
            }
            // a panel's multipliers L[p0 + row][p0 + q] (rows below ob and columns past the panel
            // zero), loaded into registers one panel ahead so their latency overlaps the panel before
            T staged[RW * W / 256];
            auto load_panel = [&](int p0) {
                const int w = min(W, ob - p0), rest = ob - p0;
#pragma unroll
                for (int u = 0; u < RW * W / 256; ++u) {
                    const int i = t + u * 256, row = i / W, q = i % W;
                    staged[u] = (row < rest && q < w) ? a[(J0 + p0 + row) * n + J0 + p0 + q] : T(0);
                }
            };
            load_panel(0);
            for (int p0 = 0; p0 < ob; p0 += W) {
                const int w = min(W, ob - p0), rest = ob - p0;
                __syncthreads();  // x in place; the previous panel's multipliers no longer read
#pragma unroll
                for (int u = 0; u < RW * W / 256; ++u) {
                    const int i = t + u * 256;
                    l[(i / W) * LP + i % W] = staged[u];
                }
                __syncthreads();
                if (p0 + W < ob) load_panel(p0 + W);
                // the panel's rows: v[r] -= L[r][k] v[k] for k = 0, 1, ... (move_solve's order per row)
                if (warp < CS / 4) {
                    const int col = 4 * warp + lane / 8, l8 = lane % 8;
                    T v[PER];
#pragma unroll
                    for (int u = 0; u < PER; ++u) v[u] = x[(p0 + l8 + 8 * u) * XP + col];
#pragma unroll
                    for (int k = 0; k < W - 1; ++k) {
                        const T vk = __shfl_sync(0xffffffffu, v[k / 8], (lane & ~7u) | (k % 8));
#pragma unroll
                        for (int u = 0; u < PER; ++u) {
                            const int r = l8 + 8 * u;
                            if (r > k) v[u] = sub(v[u], mul(l[r * LP + k], vk));
                        }
                    }
#pragma unroll
                    for (int u = 0; u < PER; ++u)
                        if (l8 + 8 * u < w) x[(p0 + l8 + 8 * u) * XP + col] = v[u];
                }
                __syncthreads();
                // the rows below: x[r] -= sum over q of L[r][q] x[p0 + q] (rank_update's order)
                for (int i = t; i < (rest - w) * (CS / 4); i += 256) {
                    const int row = w + i / (CS / 4), c4 = 4 * (i % (CS / 4));
                    T m[W];
#pragma unroll
                    for (int q = 0; q < W; q += 16 / static_cast<int>(sizeof(T))) load16(l + row * LP + q, m + q);
                    T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
                    for (int q = 0; q < W; ++q) {
                        T xv[4];
                        load4(x + (p0 + q) * XP + c4, xv);
#pragma unroll
                        for (int e = 0; e < 4; ++e) acc[e] = fma_(m[q], xv[e], acc[e]);
                    }
                    T *const target = x + (p0 + row) * XP + c4;
#pragma unroll
                    for (int e = 0; e < 4; ++e) target[e] = sub(target[e], acc[e]);
                }
            }
            __syncthreads();
            for (int i = t; i < ob * CS; i += 256) {
                const int row = i / CS, col = i % CS;
                if (s0 + col < c1) a[(J0 + row) * n + s0 + col] = x[row * XP + col];
            }
        }

        // A panel's row movement over columns [c0, c1) but its own [j0, j0 + w), and, for the block's
        // columns right of the panel ([right, block_end)), the panel's U rows := L^-1 times themselves
        // (L the unit lower triangle of the panel's top w x w block), in one launch. One thread per
        // column does the column's moves and then its solve (row i minus L[i][k] times row k for
        // k = 0, 1, ..., i - 1, each product and difference rounded, as the reference's column steps
        // subtract them); no other thread touches the column. Block 0's first warp also moves the row order.
        template <typename T>
        __global__ void __launch_bounds__(128) move_solve(T *a, unsigned long long n, const Movement *moved, unsigned long long c0,
                                                         unsigned long long c1, unsigned long long j0, int w,
                                                         unsigned long long right, unsigned long long block_end,
                                                         unsigned *order) {
            constexpr int W = PanelWidth<T>::value;
            constexpr int threads = 128, L = W * W / threads;
            __shared__ T lower[W][W];
            chain_wait();
            chain_release();
            if (order != nullptr && blockIdx.x == 0 && threadIdx.x < 32) {
                const int count = static_cast<int>(moved->count), i0 = static_cast<int>(threadIdx.x), i1 = i0 + 32;
                const unsigned v0 = i0 < count ? order[moved->src[i0]] : 0u, v1 = i1 < count ? order[moved->src[i1]] : 0u;
                __syncwarp();
                if (i0 < count) order[moved->rows[i0]] = v0;
                if (i1 < count) order[moved->rows[i1]] = v1;
            }
            // the panel's top triangle (its own columns, which this kernel does not move)
            T staged[L];
#pragma unroll
            for (int u = 0; u < L; ++u) {
                const int i = threadIdx.x + u * threads, row = i / W, k = i % W;
                staged[u] = (row < w && k < w) ? a[(j0 + row) * n + j0 + k] : T(0);
            }
#pragma unroll
            for (int u = 0; u < L; ++u) {
                const int i = threadIdx.x + u * threads;
                lower[i / W][i % W] = staged[u];
            }
            __syncthreads();
            const unsigned long long col = c0 + blockIdx.x * 1ull * threads + threadIdx.x;
            if (col >= c1 || (col >= j0 && col < j0 + w)) return;
            {
                const int count = static_cast<int>(moved->count);
                T values[64];
#pragma unroll
                for (int i = 0; i < 64; ++i)
                    if (i < count) values[i] = a[static_cast<unsigned long long>(moved->src[i]) * n + col];
#pragma unroll
                for (int i = 0; i < 64; ++i)
                    if (i < count) a[static_cast<unsigned long long>(moved->rows[i]) * n + col] = values[i];
            }
            if (col < right || col >= block_end) return;
            T x[W];
#pragma unroll
            for (int i = 0; i < W; ++i) x[i] = i < w ? a[(j0 + i) * n + col] : T(0);
#pragma unroll
            for (int i = 1; i < W; ++i) {
#pragma unroll
                for (int k = 0; k < i; ++k) x[i] = sub(x[i], mul(lower[i][k], x[k]));
            }
#pragma unroll
            for (int i = 0; i < W; ++i)
                if (i < w) a[(j0 + i) * n + col] = x[i];
        }

        // ---- substitution (solve.hpp:25-52), blocked ----------------------------------------------------
        // One diagonal block of `size` rows: lower (unit) or upper (divide by the diagonal) solve of
        // `width` right-hand-side columns in place. Warp w solves column (blockIdx.y * 32 + w); lane l
        // holds rows l, l + 32, ... of the block.
        template <typename T, bool upper>
        __global__ void __launch_bounds__(1024) solve_block(const T *lu, unsigned long long n, unsigned long long s, int size, T *x,
                                    unsigned long long width) {
            extern __shared__ __align__(16) unsigned char solve_shared[];
            T(*tri)[kSolveBlock + 1] = reinterpret_cast<T(*)[kSolveBlock + 1]>(solve_shared);
            {
                constexpr int L = kSolveBlock * kSolveBlock / 1024;
                T staged[L];
#pragma unroll
                for (int u = 0; u < L; ++u) {
                    const int i = threadIdx.x + u * 1024, row = i / kSolveBlock, k = i % kSolveBlock;
                    staged[u] = (row < size && k < size) ? lu[(s + row) * n + s + k] : T(0);
                }
#pragma unroll
                for (int u = 0; u < L; ++u) {
                    const int i = threadIdx.x + u * 1024;
                    tri[i / kSolveBlock][i % kSolveBlock] = staged[u];
                }
            }
            __syncthreads();
            const unsigned lane = threadIdx.x % 32, warp = threadIdx.x / 32;
            const unsigned long long column = blockIdx.y * 32ull + warp;
            if (column >= width) return;
            constexpr int R = kSolveBlock / 32;
            T b[R];
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int row = lane + 32 * q;
                b[q] = row < size ? x[(s + row) * width + column] : T(0);
            }
            for (int step = 0; step < size; ++step) {
                const int i = upper ? size - 1 - step : step;
                const int owner = i % 32, slot = i / 32;
                T value = T(0);
#pragma unroll
                for (int q = 0; q < R; ++q)
                    if (q == slot) value = b[q];
                if (upper) value = div(value, tri[i][i]);
                value = __shfl_sync(0xffffffffu, value, owner);
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    const int row = lane + 32 * q;
                    if (row == i) b[q] = value;
                    else if (upper ? row < i : (row > i && row < size)) b[q] = sub(b[q], mul(tri[row][i], value));
                }
            }
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int row = lane + 32 * q;
                if (row < size) x[(s + row) * width + column] = b[q];
            }
        }

        // Inverses of the diagonal blocks of L (unit lower) and U, kSolveBlock x kSolveBlock each, zero
        // padded past the matrix: inv[2 b] is L's block b (blockIdx.y 0), inv[2 b + 1] U's (blockIdx.y
        // 1). The block is staged in shared memory; warp w builds columns w, w + 32, ... of the inverse
        // by substitution against the identity (solve.hpp:25-52 applied to e_c), lane l holding rows
        // l, l + 32, ...: once entry k is final it is broadcast by a shuffle and every row it reaches
        // takes its term, so the chain from one entry to the next is a shuffle and one multiply-add
        // (the earlier form, a thread per column summing each entry's terms on its own, took 116 us
        // for the 64 blocks of n = 8192). An entry of L's inverse takes its terms in the order of k,
        // as the row-by-row substitution adds them; one of U's takes them from the diagonal outwards
        // (k descending) and is then divided by the diagonal.
        constexpr int kInvertPitch = kSolveBlock + 1;
        template <typename T> constexpr size_t invert_shared_bytes() { return sizeof(T) * kSolveBlock * kInvertPitch; }
        constexpr int kInvertThreads = 1024;
        template <typename T>
        __global__ void __launch_bounds__(kInvertThreads) invert_blocks(const T *lu, unsigned long long n, T *inv) {
            constexpr int B = kSolveBlock, PD = kInvertPitch, R = B / 32;
            extern __shared__ __align__(16) unsigned char invert_shared[];
            T *const ds = reinterpret_cast<T *>(invert_shared);  // ds[i * PD + k] = d[i][k]
            const unsigned long long s = blockIdx.x * 1ull * B;
            const int size = static_cast<int>(n - s < B ? n - s : B);
            const bool upper = blockIdx.y != 0;
            T *const out = inv + (2ull * blockIdx.x + (upper ? 1ull : 0ull)) * B * B;
            const T *d = lu + s * n + s;
            for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
                const int i = e / B, k = e % B;
                ds[i * PD + k] = (i < size && k < size) ? d[i * n + k] : T(0);
            }
            __syncthreads();
            const int lane = static_cast<int>(threadIdx.x % 32);
            for (int c = static_cast<int>(threadIdx.x / 32); c < B; c += kInvertThreads / 32) {
                T x[R];  // x[r]: row 32 r + lane of column c
#pragma unroll
                for (int r = 0; r < R; ++r) x[r] = (c < size && 32 * r + lane == c) ? T(1) : T(0);
                if (c < size && !upper) {
                    // x_i = [i == c] - sum over k = c .. i - 1 of L_ik x_k
#pragma unroll
                    for (int q = 0; q < R; ++q) {
                        if (32 * q + 31 < c) continue;
                        for (int kk = 0; kk < 32; ++kk) {
                            const int k = 32 * q + kk;
                            if (k < c || k >= size) continue;
                            const T xk = __shfl_sync(0xffffffffu, x[q], kk);
#pragma unroll
                            for (int r = q; r < R; ++r) {
                                const int i = 32 * r + lane;
                                if (i > k && i < size) x[r] = fma_(-ds[i * PD + k], xk, x[r]);
                            }
                        }
                    }
                } else if (c < size) {
                    // x_i = ([i == c] - sum over k = c down to i + 1 of U_ik x_k) / U_ii
#pragma unroll
                    for (int q = R - 1; q >= 0; --q) {
                        if (32 * q > c) continue;
                        for (int kk = 31; kk >= 0; --kk) {
                            const int k = 32 * q + kk;
                            if (k > c) continue;
                            if (lane == kk) x[q] = div(x[q], ds[k * PD + k]);
                            const T xk = __shfl_sync(0xffffffffu, x[q], kk);
#pragma unroll
                            for (int r = 0; r <= q; ++r) {
                                const int i = 32 * r + lane;
                                if (i < k) x[r] = fma_(-ds[i * PD + k], xk, x[r]);
                            }
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) out[(32ull * r + lane) * B + c] = x[r];
            }
        }

        // The coupling blocks of the sweeps, 128 x 128 each, rows and columns past the matrix zero:
        // couple[2 i] = inv(L_ii) L_i,i-1 (block rows i >= 1), couple[2 i + 1] = inv(U_ii) U_i,i+1
        // (i <= blocks - 2), and two block rows apart couple[2 blocks + 2 i] = inv(L_ii) L_i,i-2,
        // couple[2 blocks + 2 i + 1] = inv(U_ii) U_i,i+2. One CTA per block (blockIdx.y: bit 0 upper,
        // bit 1 two rows apart), 256 threads of 8 x 8 outputs, k in slices of 16 staged in shared
        // memory.
        __global__ void __launch_bounds__(256) couple_blocks(const float *lu, const float *inv, unsigned long long n,
                                                             float *couple) {
            constexpr int B = kSolveBlock, K = 16;
            __shared__ float left[B][K + 1];  // inv[:, k0 : k0 + 16]
            __shared__ float right[K][B];     // the tile's rows k0 .. k0 + 15
            const unsigned long long blocks = (n + B - 1) / B, i = blockIdx.x;
            const bool upper = (blockIdx.y & 1) != 0;
            const unsigned long long distance = 1 + (blockIdx.y >> 1);
            if (upper ? i + distance >= blocks : i < distance) return;
            const unsigned long long s = i * B, sj = upper ? s + distance * B : s - distance * B;
            const float *inverse = inv + (2 * i + (upper ? 1 : 0)) * B * B;
            float *target = couple + ((distance - 1) * 2 * blocks + 2 * i + (upper ? 1 : 0)) * B * B;
            const int t = threadIdx.x, r0 = (t / 16) * 8, c0 = (t % 16) * 8;
            float acc[8][8] = {};
            for (int k0 = 0; k0 < B; k0 += K) {
                for (int q = t; q < B * K; q += 256) {
                    const int row = q / K, k = q % K;
                    left[row][k] = inverse[row * B + k0 + k];
                }
                for (int q = t; q < K * B; q += 256) {
                    const int k = q / B, c = q % B;
                    const unsigned long long gr = s + k0 + k, gc = sj + c;
                    right[k][c] = (gr < n && gc < n) ? lu[gr * n + gc] : 0.0f;
                }
                __syncthreads();
                for (int k = 0; k < K; ++k) {
                    float a[8], b[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) a[u] = left[r0 + u][k];
#pragma unroll
                    for (int u = 0; u < 8; ++u) b[u] = right[k][c0 + u];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
#pragma unroll
                        for (int v = 0; v < 8; ++v) acc[u][v] = fma_(a[u], b[v], acc[u][v]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) target[(r0 + u) * B + c0 + v] = acc[u][v];
        }

        // y[s + r][col] := sum_k inv[r][k] x[s + k][col] for the `size` rows of one diagonal block, out
        // of place: 16 rows (blockIdx.x) by 32 columns (blockIdx.y) per CTA of 512 threads, warp w
        // computing row 16 blockIdx.x + w with lane = column. inv is zero padded to kSolveBlock
        // square and triangular: lower blocks sum over k <= r, upper ones over k >= r.
        constexpr int kApplyRows = 16;
        template <typename T> constexpr size_t apply_shared_bytes() {
            return sizeof(T) * (kApplyRows * kSolveBlock + kSolveBlock * 32);
        }
        // transposed: apply inv^T instead (the blocks of U^T and L^T in the transposed solve).
        template <typename T, bool upper, bool transposed = false>
        __global__ void __launch_bounds__(kApplyRows * 32) apply_inverse(const T *inv, unsigned long long s, int size,
                                                                         const T *x, T *y, unsigned long long width) {
            constexpr int B = kSolveBlock, threads = kApplyRows * 32;
            extern __shared__ __align__(16) unsigned char apply_shared[];
            T *ms = reinterpret_cast<T *>(apply_shared);  // [kApplyRows][B]: this CTA's rows of inv
            T *xs = ms + kApplyRows * B;                  // [B][32]: the block of x
            const int r0 = blockIdx.x * kApplyRows;
            const unsigned long long c0 = blockIdx.y * 32ull;
            constexpr int LM = kApplyRows * B / threads, LX = B * 32 / threads;
            T rm[LM], rx[LX];  // every global load of the thread is issued before the first shared store
#pragma unroll
            for (int u = 0; u < LM; ++u) {
                const int i = threadIdx.x + u * threads, row = i / B, k = i % B;
                rm[u] = transposed ? inv[k * B + r0 + row] : inv[(r0 + row) * B + k];
            }
#pragma unroll
            for (int u = 0; u < LX; ++u) {
                const int i = threadIdx.x + u * threads, k = i / 32, col = i % 32;
                rx[u] = (k < size && c0 + col < width) ? x[(s + k) * width + c0 + col] : T(0);
            }
#pragma unroll
            for (int u = 0; u < LM; ++u) ms[threadIdx.x + u * threads] = rm[u];
#pragma unroll
            for (int u = 0; u < LX; ++u) xs[threadIdx.x + u * threads] = rx[u];
            __syncthreads();
            const int lane = threadIdx.x % 32, row = threadIdx.x / 32, r = r0 + row;
            if (r >= size) return;
            const int k0 = upper ? r : 0, k1 = upper ? size : r + 1;
            T acc = T(0);
            for (int k = k0; k < k1; ++k) acc = fma_(ms[row * B + k], xs[k * 32 + lane], acc);
            if (c0 + lane < width) y[(s + r) * width + c0 + lane] = acc;
        }

        // C (m x w, pitch ldc) -= A (m x k, pitch lda) * B (k x w, pitch ldb) for w <= 32 and
        // k <= kSolveBlock: the substitution's update of the rows beyond a diagonal block. 32 rows per
        // CTA; A's rows and all of B staged in shared memory; thread = (row, 4 columns).
        constexpr int kSkinnyRows = 32;
        template <typename T> constexpr size_t skinny_shared_bytes() {
            return sizeof(T) * (kSkinnyRows * (kSolveBlock + 1) + kSolveBlock * 32);
        }
        // transposed: A is stored k x m (pitch lda) and read in place.
        template <typename T, bool transposed = false>
        __global__ void __launch_bounds__(256) skinny_update(const T *a, unsigned long long lda, const T *b,
                                                             unsigned long long ldb, T *c, unsigned long long ldc,
                                                             unsigned long long m, int w, int k) {
            constexpr int B = kSolveBlock, P = kSolveBlock + 1;
            extern __shared__ __align__(16) unsigned char skinny_shared[];
            T *as = reinterpret_cast<T *>(skinny_shared);  // [kSkinnyRows][P]
            T *bs = as + kSkinnyRows * P;                  // [B][32]
            const unsigned long long m0 = blockIdx.x * 1ull * kSkinnyRows;
            constexpr int LA = kSkinnyRows * B / 256, LB = B * 32 / 256;
            T ra[LA], rb[LB];  // every global load of the thread is issued before the first shared store
#pragma unroll
            for (int u = 0; u < LA; ++u) {
                const int i = threadIdx.x + u * 256;
                const int row = transposed ? i % kSkinnyRows : i / B, q = transposed ? i / kSkinnyRows : i % B;
                ra[u] = (m0 + row < m && q < k) ? (transposed ? a[q * lda + m0 + row] : a[(m0 + row) * lda + q]) : T(0);
            }
#pragma unroll
            for (int u = 0; u < LB; ++u) {
                const int i = threadIdx.x + u * 256, q = i / 32, col = i % 32;
                rb[u] = (q < k && col < w) ? b[q * ldb + col] : T(0);
            }
#pragma unroll
            for (int u = 0; u < LA; ++u) {
                const int i = threadIdx.x + u * 256;
                const int row = transposed ? i % kSkinnyRows : i / B, q = transposed ? i / kSkinnyRows : i % B;
                as[row * P + q] = ra[u];
            }
#pragma unroll
            for (int u = 0; u < LB; ++u) bs[threadIdx.x + u * 256] = rb[u];
            __syncthreads();
            const int row = threadIdx.x / 8, c4 = (threadIdx.x % 8) * 4;
            if (c4 >= w) return;
            T acc[4] = {T(0), T(0), T(0), T(0)};
            for (int q = 0; q < k; ++q) {
                const T av = as[row * P + q];
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[j] = fma_(av, bs[q * 32 + c4 + j], acc[j]);
            }
            const unsigned long long gr = m0 + row;
            if (gr >= m) return;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (c4 + j < w) c[gr * ldc + c4 + j] = sub(c[gr * ldc + c4 + j], acc[j]);
        }

        // *target = max(*target, v) for v >= 0 or a NaN with the sign bit clear: such doubles order
        // like their bit patterns (a NaN above +inf, so it propagates).
        __device__ __forceinline__ void max_nonnegative(double *target, double v) {
            atomicMax(reinterpret_cast<unsigned long long *>(target), static_cast<unsigned long long>(__double_as_longlong(v)));
        }

        // r = b - A x in FP64, the refinement's residual. One CTA of 512 threads per 64 rows
        // (blockIdx.x) and 16 columns of x (blockIdx.y); A and x stream through shared memory in
        // slices of 64 columns (cp.async, four slices in flight: 160 KB), so A is read once, from HBM,
        // with enough bytes in flight per SM to keep it busy. Warp w of a slice takes its columns
        // [4 w, 4 w + 4); lane (g = lane % 16, h = lane / 16) accumulates rows g, g + 16, g + 32,
        // g + 48 against columns [8 h, 8 h + 8) of x: 32 FP64 FMAs per six 16-byte shared loads.
        // A's slice rows are stored with their 16-byte chunks XOR-swizzled by row % 8, so the
        // sixteen rows a load instruction reads fall on distinct banks. At the end the sixteen
        // warps' partial sums are added in warp order: the result is deterministic.
        constexpr int kResidualRows = 64, kResidualSlice = 64, kResidualColumns = 16, kResidualStages = 4;
        constexpr int kResidualThreads = 512;
        constexpr size_t kResidualShared =
                sizeof(double) * kResidualStages * (kResidualRows * kResidualSlice + kResidualSlice * kResidualColumns);
        static_assert(sizeof(double) * 16 * kResidualRows * kResidualColumns <= kResidualShared, "partials fit");

        // cp.async of `bytes` (16, 8 or 0: the rest of the 16 / 8 bytes zero-filled)
        __device__ __forceinline__ void residual_copy16(void *shared, const void *global, unsigned bytes) {
            const unsigned address = static_cast<unsigned>(__cvta_generic_to_shared(shared));
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(address), "l"(global), "r"(bytes) : "memory");
        }
        __device__ __forceinline__ void residual_copy8(void *shared, const void *global, unsigned bytes) {
            const unsigned address = static_cast<unsigned>(__cvta_generic_to_shared(shared));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(address), "l"(global), "r"(bytes) : "memory");
        }

        __global__ void __launch_bounds__(kResidualThreads, 1)
                residual_tiles(const double *__restrict__ a, const double *__restrict__ x, const double *__restrict__ b,
                               double *__restrict__ r, unsigned long long n, unsigned long long width, double *r_max) {
            constexpr int RW = kResidualRows, K = kResidualSlice, C = kResidualColumns, S = kResidualStages;
            constexpr int CH = K / 2;  // 16-byte chunks per slice row
            extern __shared__ __align__(16) double residual_shared[];
            double *const as = residual_shared;             // S slices of A: [row][chunk ^ (row % 8)]
            double *const xs = residual_shared + S * RW * K;  // S slices of x: [k][c]
            const unsigned long long r0 = blockIdx.x * 1ull * RW, c0 = blockIdx.y * 1ull * C;
            const int t = threadIdx.x, lane = t % 32, warp = t / 32, g = lane % 16, h = lane / 16;
            // 16-byte copies of A when every row starts on a 16-byte boundary
            const bool chunks = n % 2 == 0 && (reinterpret_cast<unsigned long long>(a) & 15) == 0;
            const unsigned long long slices = (n + K - 1) / K;
            auto issue = [&](int stage, unsigned long long k0) {
                double *const at = as + stage * RW * K;
#pragma unroll
                for (int u = 0; u < RW * CH / kResidualThreads; ++u) {
                    const int q = t + u * kResidualThreads, row = q / CH, c = q % CH;
                    const unsigned long long gr = r0 + row, gk = k0 + 2ull * c;
                    double *const dst = at + row * K + 2 * (c ^ (row & 7));
                    if (chunks) {
                        const unsigned bytes = gr < n && gk < n ? (gk + 1 < n ? 16u : 8u) : 0u;
                        residual_copy16(dst, bytes ? a + gr * n + gk : a, bytes);
                    } else {
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const bool inside = gr < n && gk + e < n;
                            residual_copy8(dst + e, inside ? a + gr * n + gk + e : a, inside ? 8u : 0u);
                        }
                    }
                }
                double *const xt = xs + stage * K * C;
#pragma unroll
                for (int u = 0; u < K * C / kResidualThreads; ++u) {
                    const int q = t + u * kResidualThreads, k = q / C, c = q % C;
                    const bool inside = k0 + k < n && c0 + c < width;
                    residual_copy8(xt + q, inside ? x + (k0 + k) * width + c0 + c : x, inside ? 8u : 0u);
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
#pragma unroll
            for (int s = 0; s < S - 1; ++s) {
                if (s < static_cast<long long>(slices)) issue(s, s * 1ull * K);
                else asm volatile("cp.async.commit_group;" ::: "memory");
            }
            double acc[4][8];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[p][j] = 0.0;
            for (unsigned long long it = 0; it < slices; ++it) {
                asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");
                __syncthreads();  // slice `it` is in place; slice it - 1's stage is free again
                const unsigned long long next = it + S - 1;
                if (next < slices) issue(static_cast<int>(next % S), next * K);
                else asm volatile("cp.async.commit_group;" ::: "memory");
                const int stage = static_cast<int>(it % S);
                const double *const at = as + stage * RW * K;
                const double *const xt = xs + stage * K * C;
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const int c = 2 * warp + half;  // this warp's chunk: columns 2 c, 2 c + 1 of the slice
                    double2 av[4];
#pragma unroll
                    for (int p = 0; p < 4; ++p) {
                        const int row = g + 16 * p;
                        av[p] = *reinterpret_cast<const double2 *>(at + row * K + 2 * (c ^ (row & 7)));
                    }
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        double xv[8];
                        const double2 *const xp = reinterpret_cast<const double2 *>(xt + (2 * c + e) * C + 8 * h);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const double2 pair = xp[j];
                            xv[2 * j] = pair.x;
                            xv[2 * j + 1] = pair.y;
                        }
#pragma unroll
                        for (int p = 0; p < 4; ++p) {
                            const double av_e = e == 0 ? av[p].x : av[p].y;
#pragma unroll
                            for (int j = 0; j < 8; ++j) acc[p][j] = fma(av_e, xv[j], acc[p][j]);
                        }
                    }
                }
            }
            // the warps' partial sums, then r = b - (warp 0 + warp 1 + ... + warp 15)
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncthreads();
            double *const partial = residual_shared;  // [warp][row][column]
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int j = 0; j < 8; ++j) partial[(warp * RW + g + 16 * p) * C + 8 * h + j] = acc[p][j];
            __syncthreads();
            double largest = 0.0;  // this thread's largest |r|: its outputs share column t % C
#pragma unroll
            for (int u = 0; u < RW * C / kResidualThreads; ++u) {
                const int q = t + u * kResidualThreads, row = q / C, c = q % C;
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < kResidualThreads / 32; ++w) sum += partial[w * RW * C + q];
                const unsigned long long gr = r0 + row, gc = c0 + c;
                if (gr < n && gc < width) {
                    const double value = b[gr * width + gc] - sum;
                    r[gr * width + gc] = value;
                    const double m = fabs(value);
                    largest = (m > largest || m != m) ? m : largest;
                }
            }
            // each column's largest |r| over the CTA, max-ed into r_max[column] (zeroed before)
            const double other = __shfl_xor_sync(0xffffffffu, largest, 16);  // lane ^ 16: the same column
            largest = (other > largest || other != other) ? other : largest;
            __syncthreads();  // the partial sums are read
            double *const fold = residual_shared;  // fold[warp][column]
            if (lane < C) fold[warp * C + lane] = largest;
            __syncthreads();
            if (t < C && c0 + t < width) {
                double m = 0.0;
                for (int w = 0; w < kResidualThreads / 32; ++w) m = (fold[w * C + t] > m || fold[w * C + t] != fold[w * C + t]) ? fold[w * C + t] : m;
                max_nonnegative(&r_max[c0 + t], m);
            }
        }

        // ---- FP64 helpers of the refinement -----------------------------------------------------------
        __global__ void narrow(const double *in, float *out, unsigned long long count) {
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < count; i += 256ull * gridDim.x)
                out[i] = static_cast<float>(in[i]);
        }
        __global__ void widen_add(const float *d, double *x, unsigned long long count) {
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < count; i += 256ull * gridDim.x)
                x[i] += static_cast<double>(d[i]);
        }
        // The refinement's update x += d (n x width, width <= 256 and a divisor of 256 * gridDim.x's
        // stride, so each thread stays in one column) and each column's largest |x|, max-ed into
        // x_max[column] (zeroed before).
        __global__ void __launch_bounds__(256) widen_add_max(const float *d, double *x, unsigned long long count,
                                                            unsigned width, double *x_max) {
            __shared__ double best[256];
            double mine = 0.0;
            const unsigned long long stride = 256ull * gridDim.x;
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < count; i += stride) {
                const double v = x[i] + static_cast<double>(d[i]);
                x[i] = v;
                const double m = fabs(v);
                mine = (m > mine || m != m) ? m : mine;
            }
            best[threadIdx.x] = mine;
            __syncthreads();
            // thread t's elements all lie in column (blockIdx.x * 256 + t) % width: fold the threads
            // of one column, then one atomic per column and CTA
            if (threadIdx.x < width) {
                const unsigned c = static_cast<unsigned>((blockIdx.x * 256ull + threadIdx.x) % width);
                double m = 0.0;
                for (unsigned t = threadIdx.x; t < 256; t += width) m = (best[t] > m || best[t] != best[t]) ? best[t] : m;
                max_nonnegative(&x_max[c], m);
            }
        }
        // out = (float) a for the n x n matrix but its first `skip` columns (skip even), and |a|_inf (the
        // largest row sum of |a|, every column) max-ed into *a_norm (zeroed before): one warp per row,
        // the row read once for both, two elements per 16-byte load when `paired` (n even, a 16-byte
        // and out 8-byte aligned: every row then starts on those boundaries; narrow_paired).
        __global__ void __launch_bounds__(256) narrow_sums(const double *a, float *out, unsigned long long n, double *a_norm,
                                                           unsigned long long skip, bool paired) {
            const unsigned long long row = blockIdx.x * 8ull + threadIdx.x / 32;
            if (row >= n) return;
            const unsigned lane = threadIdx.x % 32;
            const double *src = a + row * n;
            float *dst = out + row * n;
            double s = 0.0;
            if (paired) {
                const double2 *src2 = reinterpret_cast<const double2 *>(src);
                float2 *dst2 = reinterpret_cast<float2 *>(dst);
                const unsigned long long pairs = n / 2, from = skip / 2;
#pragma unroll 4
                for (unsigned long long k = lane; k < pairs; k += 32) {
                    const double2 v = src2[k];
                    if (k >= from) dst2[k] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
                    s += fabs(v.x);
                    s += fabs(v.y);
                }
            } else {
#pragma unroll 4
                for (unsigned long long k = lane; k < n; k += 32) {
                    const double v = src[k];
                    if (k >= skip) dst[k] = static_cast<float>(v);
                    s += fabs(v);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) max_nonnegative(a_norm, s);
        }
        // Whether narrow_sums may read a in 16-byte pairs and write out in 8-byte pairs.
        inline bool narrow_paired(const double *a, const float *out, unsigned long long n) {
            return n % 2 == 0 && reinterpret_cast<uintptr_t>(a) % 16 == 0 && reinterpret_cast<uintptr_t>(out) % 8 == 0;
        }
        // out = (float) a over the columns [0, columns) of every row: one warp per row.
        __global__ void __launch_bounds__(256) narrow_columns(const double *a, float *out, unsigned long long n,
                                                              unsigned long long columns) {
            const unsigned long long row = blockIdx.x * 8ull + threadIdx.x / 32;
            if (row >= n) return;
            for (unsigned long long k = threadIdx.x % 32; k < columns; k += 32)
                out[row * n + k] = static_cast<float>(a[row * n + k]);
        }
        // |rows of a|_1, the infinity norm's terms: one warp per row.
        template <typename T> __global__ void row_sums(const T *a, unsigned long long n, double *out) {
            const unsigned long long row = blockIdx.x * 8ull + threadIdx.x / 32;
            if (row >= n) return;
            double s = 0.0;
            for (unsigned long long k = threadIdx.x % 32; k < n; k += 32) s += fabs(static_cast<double>(a[row * n + k]));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (threadIdx.x % 32 == 0) out[row] = s;
        }
        // Per column of an n x width matrix: the largest |entry| (NaN propagates).
        __global__ void column_max(const double *m, unsigned long long n, unsigned long long width, double *out) {
            const unsigned long long column = blockIdx.x;
            double best = 0.0;
            for (unsigned long long i = threadIdx.x; i < n; i += blockDim.x) {
                const double v = fabs(m[i * width + column]);
                best = (v > best || v != v) ? v : best;
            }
            __shared__ double shared[256];
            shared[threadIdx.x] = best;
            __syncthreads();
            for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
                if (threadIdx.x < s) {
                    const double o = shared[threadIdx.x + s];
                    shared[threadIdx.x] = (o > shared[threadIdx.x] || o != o) ? o : shared[threadIdx.x];
                }
                __syncthreads();
            }
            if (threadIdx.x == 0) out[column] = shared[0];
        }

        unsigned blocks_for(unsigned long long count, int sms) {
            return static_cast<unsigned>(std::max<unsigned long long>(1, std::min<unsigned long long>((count + 255) / 256, sms * 32ull)));
        }

        // In-place blocked LU of an n x n row-major matrix on the context's stream; pivots to piv
        // (device, LAPACK style: at step k row k was exchanged with row piv[k]).
        // Work queued on the context's side stream (and with its side workspace) while in scope.
        struct OnSide {
            Context &ctx;
            cudaStream_t stream;
            std::unique_ptr<Workspace> space;
            explicit OnSide(Context &c) : ctx(c), stream(c.stream) {
                ctx.stream = ctx.side;
                ctx.workspace.swap(ctx.side_space);
            }
            ~OnSide() {
                ctx.workspace.swap(ctx.side_space);
                ctx.stream = stream;
            }
        };

        // The factorisation's look-ahead (a second stream for the columns beyond the next block):
        // orders above 2 kOuter, unless SCI_CUDA_LOOKAHEAD=0.
        bool look_ahead(unsigned long long n) {
            static const bool enabled = [] {
                const char *setting = std::getenv("SCI_CUDA_LOOKAHEAD");
                return !(setting && std::strcmp(setting, "0") == 0);
            }();
            return enabled && n > 2 * kOuter;
        }

        int side_stream(Context &ctx) {
            if (ctx.side) return SCI_CUDA_OK;
            int least = 0, greatest = 0;
            cudaDeviceGetStreamPriorityRange(&least, &greatest);
            if (int code = ctx.check(cudaStreamCreateWithPriority(&ctx.side, cudaStreamNonBlocking, least), "side stream"))
                return code;
            if (int code = ctx.check(cudaEventCreateWithFlags(&ctx.side_done, cudaEventDisableTiming), "side event"))
                return code;
            if (int code = ctx.check(cudaEventCreateWithFlags(&ctx.main_ready, cudaEventDisableTiming), "main event"))
                return code;
            if (!ctx.side_space) ctx.side_space = std::make_unique<Workspace>();
            return SCI_CUDA_OK;
        }

        // A (n x n, in place) := L\U with partial pivoting, right-looking in outer blocks of kOuter
        // columns and panels of W inside them. moved holds kMovements row movements: one per panel of
        // a block, in the half of the block's parity. With look-ahead (SCI_CUDA_LOOKAHEAD unset or
        // not 0), each block's panels move rows only inside the block's columns; the block's
        // movements reach every other column after the previous block's bulk update is done. Then
        // the main stream updates the next block's columns (its U rows and trailing update) and goes
        // on to its panels, while the side stream updates the columns beyond it. The two streams
        // touch disjoint columns (and movement halves), and the main stream waits for the side
        // before it moves rows outside a block.
        //
        // side_busy: the side stream (look_ahead(n) only) already holds work on the columns beyond the
        // first block, with side_done recorded after it; the main stream waits for it before its
        // first work there, as it waits for a block's side work.
        template <typename T>
        int factor_device(Context &ctx, T *a, unsigned long long n, long long *piv, Movement *moved, bool tensor,
                          bool split, unsigned *order = nullptr, bool side_busy = false) {
            constexpr int W = PanelWidth<T>::value;
            if (n > kPanelRows) return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "factor: order %llu above %llu", n, kPanelRows);
            const bool ahead = look_ahead(n);
            if (ahead) {
                if (int code = side_stream(ctx)) return code;
            }
            if (tensor && sizeof(T) == 4 && n > kOuter) {
                // the largest trailing updates reserve the product workspaces once (the main
                // stream's holds at most kOuter columns of U with look-ahead)
                const unsigned long long big = n - kOuter;
                const unsigned long long terms = split ? 3 : 1;
                const unsigned long long main_columns = ahead ? kOuter : big;
                if (int code = ctx.check(ctx.workspace->reserve(terms * ((big + main_columns) * kOuter * 2 + 2048) + 1024),
                                         "reserving the trailing-update workspace"))
                    return code;
                if (ahead) {
                    if (int code = ctx.check(ctx.side_space->reserve(terms * (2 * big * kOuter * 2 + 2048) + 1024),
                                             "reserving the side workspace"))
                        return code;
                }
            }
            const int cluster = panel_cluster<T>();
            if (cluster == 0) return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "the panel kernel's cluster cannot be scheduled");
            // a block's row movements over the columns [c0, c1) (move_rows_all: 32 columns per CTA)
            auto move_rows = [&](const Movement *block_moves, unsigned long long c0, unsigned long long c1, int panels) {
                if (c1 > c0)
                    move_rows_all<T><<<static_cast<unsigned>((c1 - c0 + 31) / 32), 256, 0, ctx.stream>>>(a, n, block_moves,
                                                                                                     panels, c0, c1);
            };
            // U rows of the block (columns [c0, c1)) = L11^-1 A12: one launch, a CTA per strip of columns
            // (narrow strips for the next block's columns, on the critical path)
            static const cudaError_t strip_sized = [] {
                const cudaError_t wide = cudaFuncSetAttribute(
                        reinterpret_cast<const void *>(&block_rows_strip<T, kStripColumns>),
                        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(strip_shared_bytes<T, kStripColumns>()));
                const cudaError_t thin = cudaFuncSetAttribute(
                        reinterpret_cast<const void *>(&block_rows_strip<T, kStripColumnsNarrow>),
                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                        static_cast<int>(strip_shared_bytes<T, kStripColumnsNarrow>()));
                return wide != cudaSuccess ? wide : thin;
            }();
            if (int code = ctx.check(strip_sized, "sizing the block rows' shared memory")) return code;
            // chained: the launch follows the kernel before it on the stream directly (narrow strips only)
            auto block_rows = [&](unsigned long long J0, unsigned long long block_end, unsigned long long c0,
                                  unsigned long long c1, bool narrow, bool chained = false) -> int {
                if (c1 <= c0) return SCI_CUDA_OK;
                const int ob = static_cast<int>(block_end - J0);
                if (narrow) {
                    constexpr int CS = kStripColumnsNarrow;
                    const dim3 grid(static_cast<unsigned>((c1 - c0 + CS - 1) / CS));
                    if (chained)
                        return ctx.check(launch_chained_shared(block_rows_strip<T, CS>, grid, dim3(256), strip_shared_bytes<T, CS>(),
                                                               ctx.stream, a, n, J0, ob, c0, c1),
                                         "launching the block's U rows");
                    block_rows_strip<T, CS><<<grid, 256, strip_shared_bytes<T, CS>(), ctx.stream>>>(a, n, J0, ob, c0, c1);
                } else {
                    constexpr int CS = kStripColumns;
                    block_rows_strip<T, CS><<<static_cast<unsigned>((c1 - c0 + CS - 1) / CS), 256, strip_shared_bytes<T, CS>(),
                                              ctx.stream>>>(a, n, J0, ob, c0, c1);
                }
                return ctx.check(cudaGetLastError(), "launching the block's U rows");
            };
            // trailing update of columns [c0, c1): A[t0:, c0:c1] -= L[t0:, J0:t0] U[J0:t0, c0:c1]
            // narrow: the next block's columns on the critical path, where the SIMT rank update
            // (no operand conversion) beats a small tensor-core product
            auto trailing = [&](unsigned long long J0, unsigned long long t0, unsigned long long c0,
                                unsigned long long c1, bool narrow) -> int {
                if (t0 >= n || c1 <= c0) return SCI_CUDA_OK;
                const unsigned long long ob = t0 - J0;
                // narrow (the next block's columns, on the main stream) in FP64 follows the block's U
                // rows directly: the SIMT rank update, chained; in float the tensor cores take it too
                if constexpr (sizeof(T) == 8) {
                    if (narrow)
                        return update<T>(ctx, a + t0 * n + J0, n, a + J0 * n + c0, n, a + t0 * n + c0, n, n - t0, c1 - c0, ob,
                                         true);
                } else {
                    if (narrow && !tensor)
                        return update<T>(ctx, a + t0 * n + J0, n, a + J0 * n + c0, n, a + t0 * n + c0, n, n - t0, c1 - c0, ob,
                                         true);
                    // the next block's columns follow the block's U rows directly on the main stream
                    if (tensor)
                        return tensor_gemm(ctx, split ? 3 : 1, a + t0 * n + J0, n, a + J0 * n + c0, n, a + t0 * n + c0, n,
                                           n - t0, c1 - c0, ob, true, false, narrow);
                }
                return simt_gemm<T>(ctx, a + t0 * n + J0, n, a + J0 * n + c0, n, a + t0 * n + c0, n, n - t0, c1 - c0, ob,
                                    true);
            };
            // order (optional): the row order, kept up to date by each panel's row moves
            if (order != nullptr) identity_rows<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx.stream>>>(order, n);
            bool side_pending = side_busy;
            if (side_busy && !ahead) {
                if (int code = ctx.check(cudaStreamWaitEvent(ctx.stream, ctx.side_done, 0), "waiting for the side"))
                    return code;
                side_pending = false;
            }
            for (unsigned long long J0 = 0; J0 < n; J0 += kOuter) {
                const unsigned long long ob = std::min<unsigned long long>(kOuter, n - J0), block_end = J0 + ob;
                Movement *const block_moves = moved + (J0 / kOuter % 2) * (kMovements / 2);
                int panels = 0;
                for (unsigned long long j0 = J0; j0 < block_end; j0 += W, ++panels) {
                    const int w = static_cast<int>(std::min<unsigned long long>(W, block_end - j0));
                    Movement *mine = block_moves + panels;
                    // Within a block, each kernel of the chain panel -> row moves -> U rows -> rank
                    // update -> next panel follows the one before it directly on the stream, so it is
                    // launched chained (programmatic dependent launch): its launch overlaps the end of
                    // its predecessor. The block's first panel follows other work and waits plainly.
                    const bool chained = j0 != J0;
                    const cudaError_t launched =
                            launch_panel_for<T>(cluster, ctx.stream, a, n, j0, w, piv, mine, ctx.status, chained);
                    if (int code = ctx.check(launched, "launching the panel factorisation")) return code;
                    // the panel's row movement: now inside the block (everywhere without look-ahead)
                    // Inside the outer block only: U rows of the panel (with the moves, one launch),
                    // then the rows below it. Columns beyond the block wait until the block's pivots
                    // are all known (a later pivot of this block may still bring a row up from below).
                    const unsigned long long m0 = ahead ? J0 : 0, m1 = ahead ? block_end : n;
                    const unsigned long long right = j0 + w;
                    if (int code = ctx.check(launch_chained(move_solve<T>, dim3(static_cast<unsigned>((m1 - m0 + 127) / 128)),
                                                            dim3(128), ctx.stream, a, n, mine, m0, m1, j0, w, right, block_end,
                                                            order),
                                             "launching the panel's row moves and U rows"))
                        return code;
                    if (right < block_end) {
                        if (int code = update<T>(ctx, a + right * n + j0, n, a + j0 * n + right, n, a + right * n + right, n,
                                                 n - right, block_end - right, w, true))
                            return code;
                    }
                    if (int code = ctx.check(cudaGetLastError(), "launching the panel updates")) return code;
                }
                if (!ahead) {
                    // without look-ahead every panel moved its rows everywhere; the rest of the matrix
                    if (block_end >= n) continue;
                    if (int code = block_rows(J0, block_end, block_end, n, false)) return code;
                    if (int code = trailing(J0, block_end, block_end, n, false)) return code;
                    continue;
                }
                // The block's movements reach the other columns once the side stream is done with
                // them. The main stream moves the next block's rows, takes its U rows and trailing
                // update and goes on to its panels; the side stream moves the rows of the columns
                // left of the block and beyond the next one and updates the latter. With the tensor
                // cores the side's work is short, and it starts only after the main stream's (so the
                // critical path's small kernels find the SMs free); the SIMT update is long and
                // bounds the factorisation, so there the side starts first.
                if (side_pending) {
                    if (int code = ctx.check(cudaStreamWaitEvent(ctx.stream, ctx.side_done, 0), "waiting for the side"))
                        return code;
                    side_pending = false;
                }
                const unsigned long long split_at = std::min<unsigned long long>(block_end + kOuter, n);
                move_rows(block_moves, block_end, split_at, panels);
                if (split_at >= n) move_rows(block_moves, 0, J0, panels);
                auto side_work = [&]() -> int {
                    if (int code = ctx.check(cudaEventRecord(ctx.main_ready, ctx.stream), "recording the main stream"))
                        return code;
                    OnSide side(ctx);
                    if (int code = ctx.check(cudaStreamWaitEvent(ctx.stream, ctx.main_ready, 0), "side waits")) return code;
                    move_rows(block_moves, 0, J0, panels);
                    move_rows(block_moves, split_at, n, panels);
                    if (int code = block_rows(J0, block_end, split_at, n, false)) return code;
                    if (int code = trailing(J0, block_end, split_at, n, false)) return code;
                    if (int code = ctx.check(cudaEventRecord(ctx.side_done, ctx.stream), "recording the side")) return code;
                    side_pending = true;
                    return SCI_CUDA_OK;
                };
                const bool side_late = tensor && sizeof(T) == 4;
                if (split_at < n && !side_late) {
                    if (int code = side_work()) return code;
                }
                if (block_end < n) {
                    // with the tensor cores the side's work comes after these, so they follow the row
                    // moves and each other directly on the main stream (chained)
                    if (int code = block_rows(J0, block_end, block_end, split_at, true, side_late)) return code;
                    if (int code = trailing(J0, block_end, block_end, split_at, true)) return code;
                }
                if (split_at < n && side_late) {
                    if (int code = side_work()) return code;
                }
            }
            if (side_pending) {
                if (int code = ctx.check(cudaStreamWaitEvent(ctx.stream, ctx.side_done, 0), "waiting for the side")) return code;
            }
            return SCI_CUDA_OK;
        }

        // The inverses of the diagonal blocks (2 per block row) followed by the coupling blocks of the
        // persistent sweeps (4 per block row, couple_blocks).
        unsigned long long inverse_elements(unsigned long long n) {
            return 6ull * ((n + kSolveBlock - 1) / kSolveBlock) * kSolveBlock * kSolveBlock;
        }

        template <typename T> int invert_diagonal(Context &ctx, const T *lu, unsigned long long n, T *inv) {
            const unsigned blocks = static_cast<unsigned>((n + kSolveBlock - 1) / kSolveBlock);
            static const cudaError_t sized = cudaFuncSetAttribute(reinterpret_cast<const void *>(&invert_blocks<T>),
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                  static_cast<int>(invert_shared_bytes<T>()));
            if (int code = ctx.check(sized, "sizing the inversion's shared memory")) return code;
            invert_blocks<T><<<dim3(blocks, 2), kInvertThreads, invert_shared_bytes<T>(), ctx.stream>>>(lu, n, inv);
            if constexpr (sizeof(T) == 4) {
                if (blocks > 1)
                    couple_blocks<<<dim3(blocks, 4), 256, 0, ctx.stream>>>(lu, inv, n, inv + 2ull * blocks * kSolveBlock * kSolveBlock);
            }
            return ctx.check(cudaGetLastError(), "inverting the diagonal blocks");
        }

        // x (n x width, in place: holds P b on entry) := U^-1 L^-1 x, a substitution in the
        // reference's order inside each diagonal block (the FP64 form).
        template <typename T>
        int substitute_device(Context &ctx, const T *lu, unsigned long long n, T *x, unsigned long long width) {
            const dim3 groups(1, static_cast<unsigned>((width + 31) / 32));
            const size_t smem = sizeof(T) * kSolveBlock * (kSolveBlock + 1);
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&solve_block<T, false>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&solve_block<T, true>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            for (unsigned long long s = 0; s < n; s += kSolveBlock) {
                const int size = static_cast<int>(std::min<unsigned long long>(kSolveBlock, n - s));
                solve_block<T, false><<<groups, 1024, smem, ctx.stream>>>(lu, n, s, size, x, width);
                const unsigned long long below = s + size;
                if (below < n) {
                    if (int code = update<T>(ctx, lu + below * n + s, n, x + s * width, width, x + below * width, width,
                                             n - below, width, size))
                        return code;
                }
            }
            const unsigned long long last = (n - 1) / kSolveBlock * kSolveBlock;
            for (long long s = static_cast<long long>(last); s >= 0; s -= kSolveBlock) {
                const unsigned long long us = static_cast<unsigned long long>(s);
                const int size = static_cast<int>(std::min<unsigned long long>(kSolveBlock, n - us));
                solve_block<T, true><<<groups, 1024, smem, ctx.stream>>>(lu, n, us, size, x, width);
                if (us > 0) {
                    if (int code = update<T>(ctx, lu + us, n, x + us * width, width, x, width, us, width, size))
                        return code;
                }
            }
            return ctx.check(cudaGetLastError(), "launching the substitution");
        }

        // ---- persistent substitution sweeps ---------------------------------------------------------
        // One cooperative launch solves a whole unit-lower (L) or upper (U) system in place of the
        // block-by-block launches. CTA (block row i, column group g) adds up the products of its
        // off-diagonal tiles with the other block rows' results in a fixed order, each as soon as
        // that row has published, except the last two block rows' before it along the chain; applies
        // its diagonal block's inverse to (right-hand side - sum); and only then takes those two rows,
        // whose results enter through the coupling blocks inv(D_ii) D_i,j (the one two rows back as
        // soon as it is published). So the chain from one block row to the next is one wait, one
        // 128 x 128 x C product, one reduction and the write, and the inverse's product, which needs
        // every earlier tile, runs while the row before is still being computed. Block rows
        // publish in chain order (written, fenced, then the group's progress mark released), so one
        // acquire of the mark shows every block row published so far.
        // Every CTA is resident (cooperative launch), and every wait is bounded: one that runs out
        // sets the timeout status and ends its CTA, so the CTAs after it end the same way.
        constexpr int kSweepThreads = 4 * kSolveBlock;  // 8 k-groups x 64 row pairs of the block's 128 rows
        constexpr int kSweepGroups = 8;                 // k-groups of 16 columns of a 128-column tile
        constexpr unsigned kSweepWaitLimit = 1u << 22;

        __device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
            return v;
        }
        // A polling read: relaxed, so it does not queue behind this thread's earlier loads; the read
        // that sees the release is followed by one acquire read of the same word (monotonic: it sees
        // that mark or a later one, each written by a release), which orders what follows. That took
        // 4.6-4.7 us per chain step at n = 8192 against 4.9-5.1 us with fence.acq_rel after the
        // relaxed read instead.
        __device__ __forceinline__ unsigned load_relaxed(const unsigned *p) {
            unsigned v;
            asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
            return v;
        }
        __device__ __forceinline__ void store_release(unsigned *p, unsigned v) {
            asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
        }

        // acc[0..C) += a * v[0..C), two columns per packed instruction
        template <int C> __device__ __forceinline__ void axpy(float a, const float *v, Pair *acc) {
            const Pair pa = pair(a);
            const Pair *pv = reinterpret_cast<const Pair *>(v);
#pragma unroll
            for (int c = 0; c < C / 2; ++c) acc[c] = fma_(pa, pv[c], acc[c]);
        }
        // acc0 += a0 * v and acc1 += a1 * v: each value of v loaded once for two rows
        template <int C> __device__ __forceinline__ void axpy2(float a0, float a1, const float *v, Pair *acc0, Pair *acc1) {
            const Pair p0 = pair(a0), p1 = pair(a1);
            const Pair *pv = reinterpret_cast<const Pair *>(v);
#pragma unroll
            for (int c = 0; c < C / 2; ++c) {
                const Pair x = pv[c];
                acc0[c] = fma_(p0, x, acc0[c]);
                acc1[c] = fma_(p1, x, acc1[c]);
            }
        }
        constexpr int kCouplePitch = kSolveBlock + 4;  // a staged coupling block's row pitch (16-byte rows)
        template <int C> constexpr size_t sweep_shared_bytes() {
            return sizeof(float) * (kSolveBlock * (C + 4) + kSweepGroups * kSolveBlock * (C + 1) + 2 * kSolveBlock * kCouplePitch);
        }

        // 16-byte asynchronous copy global -> shared through L2 only (no stale L1 line of another SM's
        // results can be read), zero-filled when `full` is false.
        __device__ __forceinline__ void copy16_async(void *shared, const void *global, bool full) {
            const unsigned address = static_cast<unsigned>(__cvta_generic_to_shared(shared));
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(address), "l"(global), "r"(full ? 16 : 0)
                         : "memory");
        }
        __device__ __forceinline__ void copies_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
        template <int pending> __device__ __forceinline__ void copies_wait() {
            asm volatile("cp.async.wait_group %0;" ::"n"(pending) : "memory");
        }

        template <bool upper, int C>
        __global__ void __launch_bounds__(kSweepThreads, 1)
        sweep(const float *__restrict__ lu, const float *__restrict__ inv, const float *__restrict__ couple, unsigned n,
              unsigned width, unsigned groups, const float *__restrict__ in, float *out, unsigned *flags, unsigned epoch,
              int *status) {
            static_assert(C == 8 || C == 16, "column groups of 8 or 16");
            constexpr int B = kSolveBlock;
            constexpr int P = C + 4;  // pitch of a staged block row: 16-byte aligned rows
            constexpr int Q = C + 1;  // pitch of a partial-sum row
            constexpr int V = B * C / kSweepThreads;  // block elements per thread in the row-major mapping
            constexpr int G = kSweepGroups, KG = B / G;  // k-groups and their width
            // staged[0]: a block of results (or the rhs) being applied; staged[1], the next block's
            // copy in flight, lives in the partial sums' space, which is free until the tiles are done
            extern __shared__ __align__(16) float space[];  // sweep_shared_bytes<C>()
            float *const staged0 = space, *const staged1 = space + B * P;
            float (*partial)[B * Q] = reinterpret_cast<float (*)[B * Q]>(space + B * P);
            // the two coupling blocks (two rows back, adjacent), copied in at the start: loaded into
            // registers after the tiles instead, their 128 KB held up the shared-memory reductions
            // that follow (3 us of a 4 us step)
            float *const couple_far = space + B * P + G * B * Q, *const couple_adjacent = couple_far + B * kCouplePitch;
            __shared__ bool stop;
            __shared__ int ready_shared;
            const unsigned blocks = (n + B - 1) / B;
            const unsigned i = upper ? blocks - 1 - blockIdx.x / groups : blockIdx.x / groups;
            const unsigned g = blockIdx.x % groups, s = i * B, size = min(static_cast<unsigned>(B), n - s), c0 = g * C;
            // thread = (k-group h, row pair): rows r0 and r1 = r0 + 64, the columns [16 h, 16 h + 16)
            // of each tile. A warp holds 32 row pairs of one k-group, so the staged reads below are
            // broadcasts, each value used for both rows (half the shared loads of one row a thread).
            const int t = threadIdx.x, h = t / (B / 2), r0 = t % (B / 2), r1 = r0 + B / 2;
            const unsigned tiles = upper ? blocks - 1 - i : i;
            const unsigned bulk = tiles > 2 ? tiles - 2 : 0;  // all tiles but the last two block rows'
            if (t == 0) stop = false;
            // this thread's 16 values of rows r0 and r1 of block (2 i + upper) of `base` (the inverses
            // and the coupling blocks share the layout)
            const unsigned long long block_base = (2ull * i + (upper ? 1 : 0)) * B * B;
            auto rows_of = [&](const float *base, float4 *dst) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    dst[u] = __ldg(reinterpret_cast<const float4 *>(base + block_base + r0 * B + KG * h) + u);
                    dst[4 + u] = __ldg(reinterpret_cast<const float4 *>(base + block_base + r1 * B + KG * h) + u);
                }
            };
            // loaded before any wait: this block's inverse rows and its right-hand side
            float4 m[8];
            rows_of(inv, m);
            float rhs[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const unsigned q = t + v * kSweepThreads, k = q / C, c = q % C;
                rhs[v] = (s + k < n && c0 + c < width) ? in[static_cast<unsigned long long>(s + k) * width + c0 + c] : 0.0f;
            }
            Pair acc[2][C / 2];  // rows r0, r1
#pragma unroll
            for (int c = 0; c < C / 2; ++c) acc[0][c] = acc[1][c] = pair(0.0f);
            // the coupling blocks into shared memory, one group of copies committed before any other
            // (the first wait for copies, at the latest the far block's, completes it)
            {
                const float *const far_block = couple + 2ull * blocks * B * B + block_base;
                const float *const adjacent_block = couple + block_base;
#pragma unroll 4
                for (int u = 0; u < B * B / 4 / kSweepThreads; ++u) {
                    const int q = t + u * kSweepThreads, row = q / (B / 4), c4 = 4 * (q % (B / 4));
                    if (tiles > 1) copy16_async(couple_far + row * kCouplePitch + c4, far_block + row * B + c4, true);
                    if (tiles > 0) copy16_async(couple_adjacent + row * kCouplePitch + c4, adjacent_block + row * B + c4, true);
                }
                copies_commit();
            }
            // this thread's 16 values of rows r0 and r1 of a staged coupling block
            auto staged_rows = [&](const float *block, float4 *dst) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    dst[u] = *reinterpret_cast<const float4 *>(block + r0 * kCouplePitch + KG * h + 4 * u);
                    dst[4 + u] = *reinterpret_cast<const float4 *>(block + r1 * kCouplePitch + KG * h + 4 * u);
                }
            };

            // Step k of this CTA applies the block row k places along the chain (row_of(k)), which is
            // also its place in publishing order.
            auto row_of = [&](unsigned step) { return upper ? blocks - 1 - step : step; };
            // `known` (uniform): the steps seen ready so far. Waits until `step` is; false if the wait
            // ran out. One read of the group's progress counter covers every earlier step too.
            unsigned known = 0;
            const unsigned base_mark = epoch << 16;
            auto ready = [&](unsigned step) -> bool {
                if (step < known) return true;
                if (t == 0) {
                    unsigned seen = 0;
                    for (unsigned spin = 0; spin < kSweepWaitLimit; ++spin) {
                        const unsigned mark = load_relaxed(flags + g);
                        if (mark > base_mark + step) {  // marks of earlier sweeps are below base_mark
                            seen = load_acquire(flags + g) - base_mark;  // the same mark or a later one
                            break;
                        }
                        __nanosleep(32);  // every waiting CTA polls the same word
                    }
                    if (seen == 0) {
                        atomicOr(status, kStatusTimeout);
                        stop = true;
                    }
                    ready_shared = static_cast<int>(seen);
                }
                __syncthreads();
                known = static_cast<unsigned>(ready_shared);
                return !stop;
            };
            // Starts copying block row row_of(step)'s results into `target` (row-major mapping: thread
            // = row t / (C / 4), columns 4 (t % (C / 4)) .. + 3; B C / 4 threads copy), or loads them
            // directly when rows are not 16-byte aligned (a width not a multiple of 4, or a caller's
            // unaligned buffer).
            auto fetch = [&](unsigned step, float *target) {
                const unsigned sj = row_of(step) * B;
                if (width % 4 == 0 && (reinterpret_cast<unsigned long long>(out) & 15) == 0) {
                    const unsigned k = t / (C / 4), c = 4 * (t % (C / 4));
                    if (t < B * C / 4) {
                        const bool inside = sj + k < n && c0 + c < width;
                        const float *source = out + (inside ? static_cast<unsigned long long>(sj + k) * width + c0 + c : 0ull);
                        copy16_async(target + k * P + c, source, inside);
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const unsigned q = t + v * kSweepThreads, k = q / C, c = q % C;
                        target[k * P + c] = (sj + k < n && c0 + c < width)
                                                ? __ldcg(out + static_cast<unsigned long long>(sj + k) * width + c0 + c)
                                                : 0.0f;
                    }
                }
                copies_commit();
            };
            // acc += this k-group's part of rows4 (rows r0: [0, 4), r1: [4, 8)) times the block in `source`
            auto accumulate = [&](const float4 *rows4, const float *source) {
                const float *base = source + KG * h * P;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    axpy2<C>(rows4[u].x, rows4[4 + u].x, base + (4 * u + 0) * P, acc[0], acc[1]);
                    axpy2<C>(rows4[u].y, rows4[4 + u].y, base + (4 * u + 1) * P, acc[0], acc[1]);
                    axpy2<C>(rows4[u].z, rows4[4 + u].z, base + (4 * u + 2) * P, acc[0], acc[1]);
                    axpy2<C>(rows4[u].w, rows4[4 + u].w, base + (4 * u + 3) * P, acc[0], acc[1]);
                }
            };
            // acc (zeroed) := the same
            auto multiply = [&](const float4 *rows4, const float *source) {
#pragma unroll
                for (int c = 0; c < C / 2; ++c) acc[0][c] = acc[1][c] = pair(0.0f);
                accumulate(rows4, source);
            };
            // the k-groups' acc into `partial` (callers have synchronised past its last reads)
            auto publish = [&]() {
#pragma unroll
                for (int row = 0; row < 2; ++row) {
                    float lanes[C];
#pragma unroll
                    for (int c = 0; c < C / 2; ++c) unpair(acc[row][c], lanes[2 * c], lanes[2 * c + 1]);
                    const int r = row == 0 ? r0 : r1;
#pragma unroll
                    for (int c = 0; c < C; ++c) partial[h][r * Q + c] = lanes[c];
                }
            };
            auto total = [&](unsigned q) {
                const unsigned k = q / C, c = q % C;
                float sum = partial[0][k * Q + c];
#pragma unroll
                for (int w = 1; w < G; ++w) sum += partial[w][k * Q + c];
                return sum;
            };

            // Every off-diagonal tile but the adjacent one, oldest results first, summed into acc;
            // the next block of results is copied in while the current one is applied.
            const float *row0 = lu + static_cast<unsigned long long>(r0 < size ? s + r0 : s) * n;
            const float *row1 = lu + static_cast<unsigned long long>(r1 < size ? s + r1 : s) * n;
            bool fetched = false;  // whether the current step's block is already on its way
            for (unsigned step = 0; step < bulk; ++step) {
                const unsigned sj = row_of(step) * B;
                float4 a[8];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const unsigned column = sj + KG * h + 4 * u;
                    a[u] = (r0 < size && column < n) ? __ldg(reinterpret_cast<const float4 *>(row0 + column))
                                                     : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    a[4 + u] = (r1 < size && column < n) ? __ldg(reinterpret_cast<const float4 *>(row1 + column))
                                                         : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                }
                // the next block is copied in now only if it is already known to be published (a
                // CTA that has caught up with the chain applies the block it has, then waits)
                if (!fetched) {
                    if (!ready(step)) return;
                    fetch(step, (step & 1) ? staged1 : staged0);
                }
                fetched = step + 1 < bulk && step + 1 < known;
                if (fetched) {
                    fetch(step + 1, (step & 1) ? staged0 : staged1);
                    copies_wait<1>();
                } else {
                    copies_wait<0>();
                }
                __syncthreads();  // the current block is in place for every thread
                accumulate(a, (step & 1) ? staged1 : staged0);
                __syncthreads();  // before the buffer is refilled
            }
            // pre = inverse (rhs - sum), kept in registers in the row-major mapping
            publish();
            __syncthreads();
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const unsigned q = t + v * kSweepThreads;
                staged0[(q / C) * P + q % C] = rhs[v] - total(q);
            }
            __syncthreads();
            multiply(m, staged0);
            publish();
            __syncthreads();
            float result[V];
#pragma unroll
            for (int v = 0; v < V; ++v) result[v] = total(t + v * kSweepThreads);
            // then the last two block rows: result = pre - inv(D_ii) (D_i,far x_far + D_i,adjacent x_adjacent),
            // the far one applied as soon as it is published, both summed before the one reduction.
#pragma unroll
            for (int c = 0; c < C / 2; ++c) acc[0][c] = acc[1][c] = pair(0.0f);
            if (tiles > 1) {
                __syncthreads();  // `partial` and staged0 are free again
                if (!ready(tiles - 2)) return;
                fetch(tiles - 2, staged0);
                copies_wait<0>();
                __syncthreads();
                float4 rows4[8];
                staged_rows(couple_far, rows4);
                accumulate(rows4, staged0);
            }
            if (tiles > 0) {
                __syncthreads();
                if (!ready(tiles - 1)) return;
                fetch(tiles - 1, staged0);
                copies_wait<0>();
                __syncthreads();
                float4 rows4[8];
                staged_rows(couple_adjacent, rows4);
                accumulate(rows4, staged0);
                publish();
                __syncthreads();
#pragma unroll
                for (int v = 0; v < V; ++v) result[v] = result[v] - total(t + v * kSweepThreads);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const unsigned q = t + v * kSweepThreads, k = q / C, c = q % C;
                if (s + k < n && c0 + c < width) out[static_cast<unsigned long long>(s + k) * width + c0 + c] = result[v];
            }
            // The block's writes reach thread 0 through the barrier, and its release (cumulative, after
            // a GPU-scope fence) publishes them. This CTA is blockIdx.x / groups places along the
            // chain and the row before it has published (its results were waited for above), so the
            // group's mark only grows.
            __syncthreads();
            if (t == 0) {
                __threadfence();
                store_release(flags + g, base_mark + blockIdx.x / groups + 1);
            }
        }

        // The progress marks of the sweeps (one per column group): zeroed when (re)allocated; each
        // sweep counts from a fresh epoch.
        int sweep_flags(Context &ctx, size_t count) {
            if (count > ctx.sweep_capacity) {
                if (ctx.sweep_flags) {
                    if (int code = ctx.check(cudaStreamSynchronize(ctx.stream), "retiring the sweep flags")) return code;
                    cudaFree(ctx.sweep_flags);
                    ctx.sweep_flags = nullptr;
                    ctx.sweep_capacity = 0;
                }
                if (int code = ctx.check(cudaMalloc(&ctx.sweep_flags, count * sizeof(unsigned)), "sweep flags")) return code;
                ctx.sweep_capacity = count;
                if (int code = ctx.check(cudaMemsetAsync(ctx.sweep_flags, 0, count * sizeof(unsigned), ctx.stream), "sweep flags"))
                    return code;
            }
            return SCI_CUDA_OK;
        }

        // Epochs take 16 bits (the marks are epoch << 16 | rows published): on wrapping, the marks of
        // earlier sweeps are cleared so none can look current.
        unsigned next_epoch(Context &ctx) {
            if (++ctx.sweep_epoch == 0x10000) {
                cudaMemsetAsync(ctx.sweep_flags, 0, ctx.sweep_capacity * sizeof(unsigned), ctx.stream);
                ctx.sweep_epoch = 1;
            }
            return ctx.sweep_epoch;
        }

        // x (n x width, the right-hand side on entry) := U^-1 L^-1 x by the two persistent sweeps, y
        // scratch; `done` stays false (and nothing is queued) when they do not apply: n not a multiple
        // of 4 (the tiles are read as 16-byte vectors), or more CTAs than can be resident at once.
        // The right-hand sides go in column groups of 8 when that many chains fit on the GPU at once
        // (each chain step is then half the work: 16 columns run as two chains side by side), else 16.
        int sweep_substitute(Context &ctx, const float *lu, const float *inv, unsigned long long n, float *x, float *y,
                             unsigned long long width, bool &done) {
            done = false;
            const unsigned long long blocks = (n + kSolveBlock - 1) / kSolveBlock;
            if (n % 4 != 0 || n > 0x7fffffffull || width > 0x7fffffffull) return SCI_CUDA_OK;
            if (blocks >= 0xffff) return SCI_CUDA_OK;  // the progress marks count block rows in 16 bits
            static int cooperative = -1;
            if (cooperative < 0) {
                int value = 0;
                cudaDeviceGetAttribute(&value, cudaDevAttrCooperativeLaunch, ctx.device);
                cooperative = value;
            }
            if (!cooperative) return SCI_CUDA_OK;
            const void *kernels[2][2] = {
                    {reinterpret_cast<const void *>(&sweep<false, 8>), reinterpret_cast<const void *>(&sweep<true, 8>)},
                    {reinterpret_cast<const void *>(&sweep<false, 16>), reinterpret_cast<const void *>(&sweep<true, 16>)}};
            const size_t shared[2] = {sweep_shared_bytes<8>(), sweep_shared_bytes<16>()};
            static const bool sized = [&] {
                bool ok = true;
                for (int f = 0; f < 2; ++f)
                    for (int u = 0; u < 2; ++u)
                        ok = ok && cudaFuncSetAttribute(kernels[f][u], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        static_cast<int>(shared[f])) == cudaSuccess;
                return ok;
            }();
            if (!sized) return SCI_CUDA_OK;  // the block-by-block path instead
            auto capacity = [&](const void *lower, const void *upper, size_t bytes) {
                return static_cast<unsigned long long>(std::min(ctx.blocks_per_sm(lower, kSweepThreads, bytes),
                                                                ctx.blocks_per_sm(upper, kSweepThreads, bytes))) *
                       ctx.sms;
            };
            int form = -1;
            unsigned long long groups = 0;
            for (int f = 0; f < 2 && form < 0; ++f) {
                const unsigned long long columns = f == 0 ? 8 : 16, g = (width + columns - 1) / columns;
                if (blocks * g <= capacity(kernels[f][0], kernels[f][1], shared[f])) {
                    form = f;
                    groups = g;
                }
            }
            if (form < 0) return SCI_CUDA_OK;
            if (int code = sweep_flags(ctx, groups)) return code;
            const float *couple = inv + 2ull * blocks * kSolveBlock * kSolveBlock;
            unsigned nn = static_cast<unsigned>(n), ww = static_cast<unsigned>(width), gg = static_cast<unsigned>(groups);
            for (int pass = 0; pass < 2; ++pass) {
                const bool upper = pass == 1;
                unsigned epoch = next_epoch(ctx);
                const float *source = upper ? y : x;
                float *target = upper ? x : y;
                void *args[] = {&lu, &inv, &couple, &nn, &ww, &gg, &source, &target, &ctx.sweep_flags, &epoch, &ctx.status};
                if (int code = ctx.check(cudaLaunchCooperativeKernel(kernels[form][pass], dim3(static_cast<unsigned>(blocks * groups)),
                                                                    dim3(kSweepThreads), args, shared[form], ctx.stream),
                                         "launching a substitution sweep"))
                    return code;
            }
            done = true;
            return SCI_CUDA_OK;
        }

        // C -= A B for the substitution (k <= kSolveBlock), 32 columns of B per launch of the skinny
        // kernel; transposed: A is stored k x m (pitch lda).
        template <typename T, bool transposed = false>
        int substitution_update(Context &ctx, const T *a, unsigned long long lda, const T *b, T *c, unsigned long long m,
                                unsigned long long width, int k) {
            if (m == 0) return SCI_CUDA_OK;
            for (unsigned long long c0 = 0; c0 < width; c0 += 32) {
                const int w = static_cast<int>(std::min<unsigned long long>(32, width - c0));
                skinny_update<T, transposed><<<static_cast<unsigned>((m + kSkinnyRows - 1) / kSkinnyRows), 256,
                                               skinny_shared_bytes<T>(), ctx.stream>>>(a, lda, b + c0, width, c + c0, width,
                                                                                       m, w, k);
            }
            return SCI_CUDA_OK;
        }

        // x (n x width; holds P b on entry) := U^-1 L^-1 x with the diagonal blocks' inverses (from
        // invert_diagonal): each block is one small product, spread over 8 CTAs, and the rows beyond
        // it are updated by the skinny kernel. y (n x width) is scratch: the forward sweep writes
        // L^-1 P b there and the backward sweep writes the solution back into x.
        template <typename T>
        int substitute_inverse(Context &ctx, const T *lu, const T *inv, unsigned long long n, T *x, T *y,
                               unsigned long long width) {
            if constexpr (sizeof(T) == 4) {
                bool done = false;
                if (int code = sweep_substitute(ctx, lu, inv, n, x, y, width, done)) return code;
                if (done) return SCI_CUDA_OK;
            }
            const unsigned column_groups = static_cast<unsigned>((width + 31) / 32);
            const int apply_smem = static_cast<int>(apply_shared_bytes<T>());
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&apply_inverse<T, false>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, apply_smem);
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&apply_inverse<T, true>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, apply_smem);
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&skinny_update<T, false>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(skinny_shared_bytes<T>()));
            constexpr unsigned long long block_elements = 1ull * kSolveBlock * kSolveBlock;
            for (unsigned long long s = 0; s < n; s += kSolveBlock) {
                const int size = static_cast<int>(std::min<unsigned long long>(kSolveBlock, n - s));
                const dim3 grid(static_cast<unsigned>((size + kApplyRows - 1) / kApplyRows), column_groups);
                apply_inverse<T, false><<<grid, kApplyRows * 32, apply_smem, ctx.stream>>>(
                        inv + 2 * (s / kSolveBlock) * block_elements, s, size, x, y, width);
                const unsigned long long below = s + size;
                if (int code = substitution_update<T>(ctx, lu + below * n + s, n, y + s * width, x + below * width, n - below,
                                                      width, size))
                    return code;
            }
            const unsigned long long last = (n - 1) / kSolveBlock * kSolveBlock;
            for (long long s = static_cast<long long>(last); s >= 0; s -= kSolveBlock) {
                const unsigned long long us = static_cast<unsigned long long>(s);
                const int size = static_cast<int>(std::min<unsigned long long>(kSolveBlock, n - us));
                const dim3 grid(static_cast<unsigned>((size + kApplyRows - 1) / kApplyRows), column_groups);
                apply_inverse<T, true><<<grid, kApplyRows * 32, apply_smem, ctx.stream>>>(
                        inv + (2 * (us / kSolveBlock) + 1) * block_elements, us, size, y, x, width);
                if (int code = substitution_update<T>(ctx, lu + us, n, x + us * width, y, us, width, size)) return code;
            }
            return ctx.check(cudaGetLastError(), "launching the substitution");
        }

        // x (n x width; holds the right-hand side on entry) := L^-T U^-T x, the transposed system's
        // substitutions with the same factors and inverses: forward through U^T (the transposed
        // inverses of U's diagonal blocks, the updates reading U's rows in place), then back through L^T.
        // P^T is left to the caller (A^T = U^T L^T P). y (n x width) is scratch.
        template <typename T>
        int substitute_inverse_transposed(Context &ctx, const T *lu, const T *inv, unsigned long long n, T *x, T *y,
                                          unsigned long long width) {
            const unsigned column_groups = static_cast<unsigned>((width + 31) / 32);
            const int apply_smem = static_cast<int>(apply_shared_bytes<T>());
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&apply_inverse<T, false, true>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, apply_smem);
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&apply_inverse<T, true, true>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, apply_smem);
            cudaFuncSetAttribute(reinterpret_cast<const void *>(&skinny_update<T, true>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(skinny_shared_bytes<T>()));
            constexpr unsigned long long block_elements = 1ull * kSolveBlock * kSolveBlock;
            for (unsigned long long s = 0; s < n; s += kSolveBlock) {
                const int size = static_cast<int>(std::min<unsigned long long>(kSolveBlock, n - s));
                const dim3 grid(static_cast<unsigned>((size + kApplyRows - 1) / kApplyRows), column_groups);
                // (U_ss^-1)^T is lower triangular
                apply_inverse<T, false, true><<<grid, kApplyRows * 32, apply_smem, ctx.stream>>>(
                        inv + (2 * (s / kSolveBlock) + 1) * block_elements, s, size, x, y, width);
                const unsigned long long below = s + size;
                // x[below] -= U[s, below]^T y[s]
                if (int code = substitution_update<T, true>(ctx, lu + s * n + below, n, y + s * width, x + below * width,
                                                            n - below, width, size))
                    return code;
            }
            const unsigned long long last = (n - 1) / kSolveBlock * kSolveBlock;
            for (long long s = static_cast<long long>(last); s >= 0; s -= kSolveBlock) {
                const unsigned long long us = static_cast<unsigned long long>(s);
                const int size = static_cast<int>(std::min<unsigned long long>(kSolveBlock, n - us));
                const dim3 grid(static_cast<unsigned>((size + kApplyRows - 1) / kApplyRows), column_groups);
                // (L_ss^-1)^T is upper triangular
                apply_inverse<T, true, true><<<grid, kApplyRows * 32, apply_smem, ctx.stream>>>(
                        inv + 2 * (us / kSolveBlock) * block_elements, us, size, y, x, width);
                // y[0, us) -= L[us, 0:us)^T x[us]
                if (int code = substitution_update<T, true>(ctx, lu + us * n, n, x + us * width, y, us, width, size))
                    return code;
            }
            return ctx.check(cudaGetLastError(), "launching the transposed substitution");
        }

        // x[rows[i]][:] (+)= z[i][:]: P^T z, added into a double accumulator or stored.
        template <typename S, typename D, bool accumulate>
        __global__ void scatter_rows(const S *z, D *x, const unsigned *rows, unsigned long long n, unsigned long long width) {
            const unsigned long long total = n * width;
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < total; i += 256ull * gridDim.x) {
                const unsigned long long row = i / width, column = i % width;
                D &out = x[static_cast<unsigned long long>(rows[row]) * width + column];
                if (accumulate) out += static_cast<D>(z[i]);
                else out = static_cast<D>(z[i]);
            }
        }

        // out (n x n) = in^T, 32 x 32 tiles through shared memory.
        // decompose's split of the packed factors (decompose.hpp:86-97): lower takes the strict lower
        // part and a unit diagonal, upper keeps the rest (in place: it holds the packed factors on
        // entry), and permutation[rows[c]][c] = 1.
        template <typename T>
        __global__ void split_factors(T *upper, T *lower, T *permutation, const unsigned *rows, unsigned long long n) {
            const unsigned long long count = n * n, stride = 1ull * gridDim.x * blockDim.x;
            for (unsigned long long i = 1ull * blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
                const unsigned long long r = i / n, c = i - r * n;
                const T v = upper[i];
                if (c < r) {
                    lower[i] = v;
                    upper[i] = T(0);
                } else {
                    lower[i] = c == r ? T(1) : T(0);
                }
                permutation[i] = rows[c] == r ? T(1) : T(0);
            }
        }

        template <typename T> __global__ void transpose_square(const T *in, T *out, unsigned long long n) {
            __shared__ T tile[32][33];
            const unsigned long long r0 = blockIdx.y * 32ull, c0 = blockIdx.x * 32ull;
            for (unsigned j = threadIdx.y; j < 32; j += 8) {
                const unsigned long long r = r0 + j, c = c0 + threadIdx.x;
                if (r < n && c < n) tile[j][threadIdx.x] = in[r * n + c];
            }
            __syncthreads();
            for (unsigned j = threadIdx.y; j < 32; j += 8) {
                const unsigned long long r = c0 + j, c = r0 + threadIdx.x;
                if (r < n && c < n) out[r * n + c] = tile[threadIdx.x][j];
            }
        }


        // x = (P b) in the element type D.
        template <typename S, typename D>
        void permute(Context &ctx, const S *b, D *x, const unsigned *rows, unsigned long long n, unsigned long long width) {
            gather_rows<S, D><<<blocks_for(n * width, ctx.sms), 256, 0, ctx.stream>>>(b, x, rows, n, width);
        }

        // Workspace carving helper.
        struct Carve {
            unsigned char *base;
            unsigned long long used{0};
            template <typename T> T *take(unsigned long long count) {
                T *p = reinterpret_cast<T *>(base + used);
                used += (count * sizeof(T) + 255) / 256 * 256;
                return p;
            }
        };

    } // namespace

} // namespace sci_cuda

using namespace sci_cuda;

extern "C" int sci_cuda_factor(sci_cuda_context *context, uint32_t precision, uint32_t mode, void *matrix, uint64_t *rows,
                               uint64_t order) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || mode > SCI_FACTOR_PLAIN)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or mode %u", precision, mode);
    if (order == 0) return SCI_CUDA_OK;
    if (!matrix || !rows) return context->fail(SCI_CUDA_ERROR_INVALID, "null matrix or rows");
    cudaSetDevice(context->device);
    if (int code = context->check(context->solver->reserve(order * 8 + kMovements * sizeof(Movement) + 1024), "pivot storage")) return code;
    Carve carve{static_cast<unsigned char *>(context->solver->memory)};
    long long *piv = carve.take<long long>(order);
    Movement *moved = carve.take<Movement>(kMovements);
    int code = precision == SCI_PRECISION_WIDE
                       ? factor_device<double>(*context, static_cast<double *>(matrix), order, piv, moved, false, false)
                       : factor_device<float>(*context, static_cast<float *>(matrix), order, piv, moved,
                                              mode != SCI_FACTOR_PLAIN, true);
    std::vector<long long> host(order);
    if (!code) code = context->check(cudaMemcpyAsync(host.data(), piv, order * sizeof(long long), cudaMemcpyDeviceToHost,
                                                     context->stream),
                                     "reading the pivots");
    if (!code) code = context->drain();
    if (code) return code;
    // rows[i] = the original row now at position i (decompose.hpp:30-42)
    for (uint64_t i = 0; i < order; ++i) rows[i] = i;
    for (uint64_t i = 0; i < order; ++i) std::swap(rows[i], rows[static_cast<uint64_t>(host[i])]);
    return SCI_CUDA_OK;
}

// decompose (decompose.hpp:77-103) with the factorisation and the split on the device.
extern "C" int sci_cuda_decompose(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *matrix,
                                  void *permutation, void *lower, void *upper, uint64_t order) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || mode > SCI_FACTOR_PLAIN)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or mode %u", precision, mode);
    if (order == 0) return SCI_CUDA_OK;
    if (order > kPanelRows) return context->fail(SCI_CUDA_ERROR_UNSUPPORTED, "decompose: order %llu above %llu",
                                                 static_cast<unsigned long long>(order), kPanelRows);
    for (const void *p : {static_cast<const void *>(matrix), static_cast<const void *>(permutation),
                          static_cast<const void *>(lower), static_cast<const void *>(upper)})
        if (!p || !reachable(*context, p)) return context->fail(SCI_CUDA_ERROR_INVALID, "decompose: %p is not device memory", p);
    cudaSetDevice(context->device);
    const size_t element = precision == SCI_PRECISION_WIDE ? 8 : 4;
    if (int code = context->check(context->solver->reserve(order * 12 + kMovements * sizeof(Movement) + 2048), "pivot storage"))
        return code;
    Carve carve{static_cast<unsigned char *>(context->solver->memory)};
    long long *piv = carve.take<long long>(order);
    Movement *moved = carve.take<Movement>(kMovements);
    unsigned *rows = carve.take<unsigned>(order);
    if (int code = context->check(cudaMemcpyAsync(upper, matrix, order * order * element, cudaMemcpyDeviceToDevice, context->stream),
                                  "copying the matrix"))
        return code;
    int code = precision == SCI_PRECISION_WIDE
                       ? factor_device<double>(*context, static_cast<double *>(upper), order, piv, moved, false, false, rows)
                       : factor_device<float>(*context, static_cast<float *>(upper), order, piv, moved,
                                              mode != SCI_FACTOR_PLAIN, true, rows);
    if (code) return code;
    const unsigned grid = static_cast<unsigned>(std::min<unsigned long long>((order * order + 255) / 256, 8ull * context->sms));
    if (precision == SCI_PRECISION_WIDE)
        split_factors<double><<<grid, 256, 0, context->stream>>>(static_cast<double *>(upper), static_cast<double *>(lower),
                                                                static_cast<double *>(permutation), rows, order);
    else
        split_factors<float><<<grid, 256, 0, context->stream>>>(static_cast<float *>(upper), static_cast<float *>(lower),
                                                               static_cast<float *>(permutation), rows, order);
    if (int c = context->check(cudaGetLastError(), "splitting the factors")) return c;
    return context->drain();
}

namespace {

    // Pinned host doubles for the refinement's small read-backs, at least `count` of them. Growing
    // waits for the stream first: a copy into the old buffer may still be queued.
    double *pinned_doubles(Context &ctx, size_t count) {
        if (count <= ctx.pinned_count) return ctx.pinned;
        cudaStreamSynchronize(ctx.stream);
        cudaFreeHost(ctx.pinned);
        ctx.pinned = nullptr;
        ctx.pinned_count = 0;
        void *memory = nullptr;
        if (cudaMallocHost(&memory, count * sizeof(double)) != cudaSuccess) return nullptr;
        ctx.pinned = static_cast<double *>(memory);
        ctx.pinned_count = count;
        return ctx.pinned;
    }

    // The normwise backward error max_j |b_j - A x_j|_inf / (|A|_inf |x_j|_inf + |b_j|_inf), in FP64.
    // r is scratch (n x width), norms (2 width: |r_j|_inf, then |x_j|_inf); `host` is pinned memory
    // for 2 width doubles; waits for the stream, then reads |A|_inf from *a_norm and |b_j|_inf from
    // b_norm[j] (host memory a copy queued earlier on the stream may fill). x_ready: norms[width + j]
    // already holds |x_j|_inf (the update computed it).
    int backward_error(Context &ctx, const double *a, const double *b, const double *x, double *r, double *norms,
                       unsigned long long n, unsigned long long width, const double *a_norm, const double *b_norm,
                       double *host, double &berr, bool x_ready = false) {
        static const cudaError_t sized = cudaFuncSetAttribute(
                reinterpret_cast<const void *>(&residual_tiles), cudaFuncAttributeMaxDynamicSharedMemorySize,
                static_cast<int>(kResidualShared));
        if (int code = ctx.check(sized, "sizing the residual's shared memory")) return code;
        cudaMemsetAsync(norms, 0, width * 8, ctx.stream);
        residual_tiles<<<dim3(static_cast<unsigned>((n + kResidualRows - 1) / kResidualRows),
                              static_cast<unsigned>((width + kResidualColumns - 1) / kResidualColumns)),
                         kResidualThreads, kResidualShared, ctx.stream>>>(a, x, b, r, n, width, norms);
        if (int code = ctx.check(cudaGetLastError(), "launching the residual")) return code;
        if (!x_ready) column_max<<<static_cast<unsigned>(width), 256, 0, ctx.stream>>>(x, n, width, norms + width);
        cudaMemcpyAsync(host, norms, 2 * width * 8, cudaMemcpyDeviceToHost, ctx.stream);
        if (int code = ctx.drain()) return code;
        berr = 0.0;
        for (unsigned long long j = 0; j < width; ++j) {
            const double e = host[j] / (*a_norm * host[width + j] + b_norm[j]);
            berr = (e > berr || e != e) ? e : berr;
        }
        return SCI_CUDA_OK;
    }

    // Queues |b_j|_inf (into norms[0, width)) and |A|_inf and their copies to host[0, width) and
    // host[width], without waiting: the next wait for the stream makes them readable. a_norm_device:
    // |A|_inf already computed on the device (narrow_sums takes it with the FP32 copy), else the row
    // sums are taken here (into sums) and their maximum into norms[2 width].
    void norms_enqueue(Context &ctx, const double *a, const double *b, double *sums, double *norms, unsigned long long n,
                       unsigned long long width, const double *a_norm_device, double *host) {
        column_max<<<static_cast<unsigned>(width), 256, 0, ctx.stream>>>(b, n, width, norms);
        if (a_norm_device == nullptr) {
            row_sums<double><<<static_cast<unsigned>((n + 7) / 8), 256, 0, ctx.stream>>>(a, n, sums);
            column_max<<<1, 256, 0, ctx.stream>>>(sums, n, 1, norms + 2 * width);
            a_norm_device = norms + 2 * width;
        }
        cudaMemcpyAsync(host, norms, width * 8, cudaMemcpyDeviceToHost, ctx.stream);
        cudaMemcpyAsync(host + width, a_norm_device, 8, cudaMemcpyDeviceToHost, ctx.stream);
    }

    // The refinement loop for a x = b (a n x n, b and x n x width, double): x = 0, r = b; repeat
    // { x += correct(r); r = b - a x in FP64 } until the normwise backward error
    // max_j |r_j|_inf / (|A|_inf |x_j|_inf + |b_j|_inf) is at most sqrt(n) eps (eps = 2^-53, the
    // stopping test of LAPACK's mixed-precision DSGESV) capped at 1e-14, or stops halving; at most
    // 30 corrections.
    // correct(r, x) adds the FP32 correction for residual r into x; with x_max_in_correct it also
    // max-es each column's |x| into norms[width + j], which the loop zeroes before each correction.
    // a_norm_device: |A|_inf already computed on the device (or null). host: pinned memory of
    // 3 width + 1 doubles whose first width + 1 the caller has already queued with norms_enqueue
    // (earlier on the stream, so nothing waits for them), or null: the loop queues them itself.
    template <class Correct>
    int refine_loop(Context &ctx, const double *a, const double *b, double *x, double *r, double *sums, double *norms,
                    unsigned long long n, unsigned long long width, Correct correct, double &berr, int &iterations,
                    const double *a_norm_device = nullptr, bool x_max_in_correct = false, double *host = nullptr) {
        if (host == nullptr) {
            host = pinned_doubles(ctx, 3 * width + 1);
            if (host == nullptr) return ctx.fail(SCI_CUDA_ERROR_MEMORY, "pinned host memory for the refinement");
            norms_enqueue(ctx, a, b, sums, norms, n, width, a_norm_device, host);
        }
        const double *b_norm = host, *a_norm = host + width;
        cudaMemsetAsync(x, 0, n * width * 8, ctx.stream);
        const double target = std::min(std::sqrt(static_cast<double>(n)) * 0x1p-53, 1e-14);
        constexpr int kMaxIterations = 30;
        double previous = INFINITY;
        berr = INFINITY;
        iterations = 0;
        const double *residual = b;  // the first correction solves for b itself
        while (iterations < kMaxIterations) {
            if (x_max_in_correct) cudaMemsetAsync(norms + width, 0, width * 8, ctx.stream);
            if (int code = correct(residual, x)) return code;
            ++iterations;
            if (int code = backward_error(ctx, a, b, x, r, norms, n, width, a_norm, b_norm, host + width + 1, berr,
                                          x_max_in_correct))
                return code;
            residual = r;
            if (!(berr > target) || !(berr < 0.5 * previous)) break;
            previous = berr;
        }
        return SCI_CUDA_OK;
    }

} // namespace

extern "C" int sci_cuda_solve(sci_cuda_context *context, uint32_t precision, uint32_t refine, const void *matrix,
                              const void *right, void *solution, uint64_t order, uint64_t width, sci_solve_report *report) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || refine > SCI_REFINE_FP64)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or refinement %u", precision, refine);
    if (refine == SCI_REFINE_FP64 && precision != SCI_PRECISION_WIDE)
        return context->fail(SCI_CUDA_ERROR_INVALID, "FP64 refinement needs double operands");
    if (report) std::memset(report, 0, sizeof(*report));
    if (order == 0 || width == 0) return SCI_CUDA_OK;
    if (!matrix || !right || !solution) return context->fail(SCI_CUDA_ERROR_INVALID, "null operand");
    if (order > kPanelRows) return context->fail(SCI_CUDA_ERROR_UNSUPPORTED, "solve: order %llu above %llu",
                                                 static_cast<unsigned long long>(order), kPanelRows);
    cudaSetDevice(context->device);
    const unsigned long long n = order, nw = order * width;
    const bool wide = precision == SCI_PRECISION_WIDE;
    const size_t element = (wide && refine == SCI_REFINE_NONE) ? 8 : 4;
    const unsigned long long need = n * n * element + n * 8 + kMovements * sizeof(Movement) + n * 4 + nw * 12 + n * 8 + width * 16 +
                                    inverse_elements(n) * 4 + nw * 4 + 8192;
    if (int code = context->check(context->solver->reserve(need), "reserving the solver workspace")) return code;
    Carve carve{static_cast<unsigned char *>(context->solver->memory)};
    long long *piv = carve.take<long long>(n);
    Movement *moved = carve.take<Movement>(kMovements);
    unsigned *rows = carve.take<unsigned>(n);

    if (refine == SCI_REFINE_NONE) {
        // linear::solve (solve.hpp:60-76): factor a copy, substitute, in the element type.
        int code;
        if (wide) {
            double *lu = carve.take<double>(n * n);
            cudaMemcpyAsync(lu, matrix, n * n * 8, cudaMemcpyDeviceToDevice, context->stream);
            code = factor_device<double>(*context, lu, n, piv, moved, false, false, rows);
            if (!code) permute<double, double>(*context, static_cast<const double *>(right), static_cast<double *>(solution),
                                               rows, n, width);
            if (!code) code = substitute_device<double>(*context, lu, n, static_cast<double *>(solution), width);
            if (!code && report) {
                double *r = carve.take<double>(nw);
                double *sums = carve.take<double>(n);
                double *norms = carve.take<double>(2 * width + 1);
                double berr = 0.0;
                double *host = pinned_doubles(*context, 3 * width + 1);
                if (host == nullptr) return context->fail(SCI_CUDA_ERROR_MEMORY, "pinned host memory for the report");
                norms_enqueue(*context, static_cast<const double *>(matrix), static_cast<const double *>(right), sums, norms,
                              n, width, nullptr, host);
                code = backward_error(*context, static_cast<const double *>(matrix), static_cast<const double *>(right),
                                      static_cast<const double *>(solution), r, norms, n, width, host + width, host,
                                      host + width + 1, berr);
                if (!code) report->backward_error = berr;
            }
        } else {
            float *lu = carve.take<float>(n * n);
            float *inv = carve.take<float>(inverse_elements(n));
            float *y = carve.take<float>(nw);
            cudaMemcpyAsync(lu, matrix, n * n * 4, cudaMemcpyDeviceToDevice, context->stream);
            code = factor_device<float>(*context, lu, n, piv, moved, true, true, rows);
            if (!code) code = invert_diagonal<float>(*context, lu, n, inv);
            if (!code) permute<float, float>(*context, static_cast<const float *>(right), static_cast<float *>(solution), rows,
                                             n, width);
            if (!code) code = substitute_inverse<float>(*context, lu, inv, n, static_cast<float *>(solution), y, width);
        }
        if (!code) code = context->drain();
        return code;
    }

    // FP32 factorisation, FP64 residual and update.
    const double *a = static_cast<const double *>(matrix);
    const double *b = static_cast<const double *>(right);
    double *x = static_cast<double *>(solution);
    float *lu = carve.take<float>(n * n);
    float *inv = carve.take<float>(inverse_elements(n));
    float *y = carve.take<float>(nw);
    double *r = carve.take<double>(nw);
    float *d = carve.take<float>(nw);
    double *sums = carve.take<double>(n);
    double *norms = carve.take<double>(2 * width + 1);
    double *a_norm = norms + 2 * width;
    const int sms = context->sms;

    double *host = pinned_doubles(*context, 3 * width + 1);
    if (host == nullptr) return context->fail(SCI_CUDA_ERROR_MEMORY, "pinned host memory for the refinement");
    // The FP32 copy of A and |A|_inf in one pass over A, then |b_j|_inf and |A|_inf on their way to
    // the host before the factorisation (the refinement's first wait for the stream finds them
    // there). With the look-ahead, the main stream converts only the first block's columns, which
    // are all that the first block's panels read, and starts factoring; the side stream converts
    // the rest and takes the norms meanwhile, and the factorisation waits for it before it first
    // touches the columns beyond the first block.
    const bool overlap = look_ahead(n);
    if (overlap) {
        if (int code = side_stream(*context)) return code;
    }
    const unsigned long long first = overlap ? kOuter : 0;
    cudaStream_t convert = overlap ? context->side : context->stream;
    if (overlap)
        narrow_columns<<<static_cast<unsigned>((n + 7) / 8), 256, 0, context->stream>>>(a, lu, n, first);
    cudaMemsetAsync(a_norm, 0, 8, convert);
    narrow_sums<<<static_cast<unsigned>((n + 7) / 8), 256, 0, convert>>>(a, lu, n, a_norm, first,
                                                                       narrow_paired(a, lu, n));
    {
        const cudaStream_t main = context->stream;
        context->stream = convert;
        norms_enqueue(*context, a, b, sums, norms, n, width, a_norm, host);
        context->stream = main;
    }
    if (overlap) {
        if (int code = context->check(cudaEventRecord(context->side_done, context->side), "recording the conversion"))
            return code;
    }
    if (int code = factor_device<float>(*context, lu, n, piv, moved, true, true, rows, overlap)) return code;
    if (int code = invert_diagonal<float>(*context, lu, n, inv)) return code;
    // the update also takes each column's |x|_inf when every thread of it stays in one column
    const bool fused_max = 256 % width == 0;
    auto correct = [&](const double *residual, double *xx) -> int {
        permute<double, float>(*context, residual, d, rows, n, width);
        if (int code = substitute_inverse<float>(*context, lu, inv, n, d, y, width)) return code;
        if (fused_max)
            widen_add_max<<<blocks_for(nw, sms), 256, 0, context->stream>>>(d, xx, nw, static_cast<unsigned>(width),
                                                                           norms + width);
        else
            widen_add<<<blocks_for(nw, sms), 256, 0, context->stream>>>(d, xx, nw);
        return SCI_CUDA_OK;
    };
    double berr = 0.0;
    int iterations = 0;
    if (int code = refine_loop(*context, a, b, x, r, sums, norms, n, width, correct, berr, iterations, a_norm, fused_max,
                               host))
        return code;
    if (report) {
        report->backward_error = berr;
        report->iterations = iterations;
    }
    return SCI_CUDA_OK;
}

namespace {

    // The plain form of the solve adjoint in the element type T: factor a copy of A, X = A^-1 B, then
    // lambda = A^-T G with the same factors (substitutions through U^T and L^T, then P^T), and
    // d A = -lambda X^T.
    template <typename T>
    int solve_gradient_plain(Context &ctx, Carve &carve, const T *a, const T *b, const T *g, T *x, T *dA, T *dB,
                             long long *piv, Movement *moved, unsigned *rows, unsigned long long n, unsigned long long width) {
        const unsigned long long nw = n * width;
        T *lu = carve.take<T>(n * n);
        T *inv = carve.take<T>(inverse_elements(n));
        T *y = carve.take<T>(nw);
        T *z = carve.take<T>(nw);
        T *lambda = dB ? dB : carve.take<T>(nw);
        cudaMemcpyAsync(lu, a, n * n * sizeof(T), cudaMemcpyDeviceToDevice, ctx.stream);
        if (int code = factor_device<T>(ctx, lu, n, piv, moved, sizeof(T) == 4, sizeof(T) == 4, rows)) return code;
        if (int code = invert_diagonal<T>(ctx, lu, n, inv)) return code;
        permute<T, T>(ctx, b, x, rows, n, width);
        if constexpr (sizeof(T) == 8) {
            if (int code = substitute_device<T>(ctx, lu, n, x, width)) return code;
        } else {
            if (int code = substitute_inverse<T>(ctx, lu, inv, n, x, y, width)) return code;
        }
        cudaMemcpyAsync(z, g, nw * sizeof(T), cudaMemcpyDeviceToDevice, ctx.stream);
        if (int code = substitute_inverse_transposed<T>(ctx, lu, inv, n, z, y, width)) return code;
        scatter_rows<T, T, false><<<blocks_for(nw, ctx.sms), 256, 0, ctx.stream>>>(z, lambda, rows, n, width);
        if (dA) {
            cudaMemsetAsync(dA, 0, n * n * sizeof(T), ctx.stream);
            if (int code = simt_gemm_t<T>(ctx, lambda, width, false, x, width, true, dA, n, n, n, width, true)) return code;
        }
        return ctx.check(cudaGetLastError(), "launching the solve adjoint");
    }

} // namespace

extern "C" int sci_cuda_solve_gradient(sci_cuda_context *context, uint32_t precision, uint32_t refine, const void *matrix,
                                       const void *right, const void *upstream, void *solution, void *matrix_gradient,
                                       void *right_gradient, uint64_t order, uint64_t width, sci_solve_report *report) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || refine > SCI_REFINE_FP64)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or refinement %u", precision, refine);
    if (refine == SCI_REFINE_FP64 && precision != SCI_PRECISION_WIDE)
        return context->fail(SCI_CUDA_ERROR_INVALID, "FP64 refinement needs double operands");
    if (report) std::memset(report, 0, sizeof(*report));
    if (order == 0 || width == 0) return SCI_CUDA_OK;
    if (!matrix || !right || !upstream) return context->fail(SCI_CUDA_ERROR_INVALID, "null operand");
    if (order > kPanelRows) return context->fail(SCI_CUDA_ERROR_UNSUPPORTED, "solve: order %llu above %llu",
                                                 static_cast<unsigned long long>(order), kPanelRows);
    cudaSetDevice(context->device);
    const unsigned long long n = order, nw = order * width;
    const size_t element = precision == SCI_PRECISION_WIDE ? 8 : 4;
    // everything either form carves, generously: matrices, inverses, right-hand-side blocks, norms
    const unsigned long long need = n * n * (8 + element) + inverse_elements(n) * element + nw * 8 * 10 + n * 32 +
                                    kMovements * sizeof(Movement) + width * 16 + 16384;
    if (int code = context->check(context->solver->reserve(need), "reserving the solver workspace")) return code;
    Carve carve{static_cast<unsigned char *>(context->solver->memory)};
    long long *piv = carve.take<long long>(n);
    Movement *moved = carve.take<Movement>(kMovements);
    unsigned *rows = carve.take<unsigned>(n);

    if (refine == SCI_REFINE_NONE) {
        int code;
        if (precision == SCI_PRECISION_WIDE) {
            double *x = solution ? static_cast<double *>(solution) : carve.take<double>(nw);
            code = solve_gradient_plain<double>(*context, carve, static_cast<const double *>(matrix),
                                                static_cast<const double *>(right), static_cast<const double *>(upstream), x,
                                                static_cast<double *>(matrix_gradient), static_cast<double *>(right_gradient),
                                                piv, moved, rows, n, width);
        } else {
            float *x = solution ? static_cast<float *>(solution) : carve.take<float>(nw);
            code = solve_gradient_plain<float>(*context, carve, static_cast<const float *>(matrix),
                                               static_cast<const float *>(right), static_cast<const float *>(upstream), x,
                                               static_cast<float *>(matrix_gradient), static_cast<float *>(right_gradient),
                                               piv, moved, rows, n, width);
        }
        if (!code) code = context->drain();
        return code;
    }

    // FP32 factorisation shared by both solves; FP64 residuals and updates.
    const double *a = static_cast<const double *>(matrix);
    const double *b = static_cast<const double *>(right);
    const double *g = static_cast<const double *>(upstream);
    double *x = solution ? static_cast<double *>(solution) : carve.take<double>(nw);
    double *lambda = right_gradient ? static_cast<double *>(right_gradient) : carve.take<double>(nw);
    float *lu = carve.take<float>(n * n);
    float *inv = carve.take<float>(inverse_elements(n));
    double *at = carve.take<double>(n * n);
    float *y = carve.take<float>(nw);
    float *d = carve.take<float>(nw);
    double *r = carve.take<double>(nw);
    double *sums = carve.take<double>(n);
    double *norms = carve.take<double>(2 * width + 1);
    const int sms = context->sms;

    narrow<<<blocks_for(n * n, sms), 256, 0, context->stream>>>(a, lu, n * n);
    if (int code = factor_device<float>(*context, lu, n, piv, moved, true, true, rows)) return code;
    if (int code = invert_diagonal<float>(*context, lu, n, inv)) return code;
    auto forward = [&](const double *residual, double *xx) -> int {
        permute<double, float>(*context, residual, d, rows, n, width);
        if (int code = substitute_inverse<float>(*context, lu, inv, n, d, y, width)) return code;
        widen_add<<<blocks_for(nw, sms), 256, 0, context->stream>>>(d, xx, nw);
        return SCI_CUDA_OK;
    };
    // A^T lambda = G: A^T = U^T L^T P, so lambda = P^T (L^-T U^-T G), with the same factors
    auto transposed = [&](const double *residual, double *xx) -> int {
        narrow<<<blocks_for(nw, sms), 256, 0, context->stream>>>(residual, d, nw);
        if (int code = substitute_inverse_transposed<float>(*context, lu, inv, n, d, y, width)) return code;
        scatter_rows<float, double, true><<<blocks_for(nw, sms), 256, 0, context->stream>>>(d, xx, rows, n, width);
        return SCI_CUDA_OK;
    };
    double berr_x = 0.0, berr_l = 0.0;
    int it_x = 0, it_l = 0;
    if (int code = refine_loop(*context, a, b, x, r, sums, norms, n, width, forward, berr_x, it_x)) return code;
    transpose_square<double><<<dim3(static_cast<unsigned>((n + 31) / 32), static_cast<unsigned>((n + 31) / 32)), dim3(32, 8), 0,
                               context->stream>>>(a, at, n);
    if (int code = refine_loop(*context, at, g, lambda, r, sums, norms, n, width, transposed, berr_l, it_l)) return code;
    if (matrix_gradient) {
        double *dA = static_cast<double *>(matrix_gradient);
        cudaMemsetAsync(dA, 0, n * n * 8, context->stream);
        if (int code = simt_gemm_t<double>(*context, lambda, width, false, x, width, true, dA, n, n, n, width, true)) return code;
    }
    if (int code = context->drain()) return code;
    if (report) {
        report->backward_error = std::max(berr_x, berr_l);
        report->iterations = it_x + it_l;
    }
    return SCI_CUDA_OK;
}
