// product.cu -- linear::product on sm_100a: C = A * B, row-major.
//
// The reference multiplies in the element type with a register-blocked CPU loop
// (src/core/drivers/processor/dispatch.cpp:171-224) or a 64x64-tile SIMT shader
// (shaders/product.slang:37-131) reached through Device::product (src/core/drivers/device.cpp:318-352).
// Here float products run in one of three forms:
//  - SCI_PRODUCT_BF16: A and B rounded to bf16 and multiplied on the 5th-generation tensor cores
//    (tcgen05.mma, kind::f16, FP32 accumulation in tensor memory), operands staged by 2-D TMA;
//  - SCI_PRODUCT_SPLIT_BF16: each operand split into hi + lo bf16 parts, three tensor-core
//    products hi*hi + hi*lo + lo*hi accumulated in the same TMEM tile (the lo*lo term, below
//    2^-16 relative, is dropped);
//  - SCI_PRODUCT_SPLIT3_BF16: hi + mid + lo parts and the six products down to 2^-24 relative,
//    about FP32 accuracy (the LU's trailing update uses it);
//  - SCI_PRODUCT_FP32: a plain FP32 SIMT kernel, the comparison form.
// Double products run a plain FP64 SIMT kernel.
//
// The tensor-core kernel: one CTA per 128 x 256 output tile (128 x 128 with three terms), six warps.
// Warp 4 issues TMA loads of 64-deep K slices of every term of A (128 x 64) and of B^T (N x 64) into
// a ring of shared-memory stages (128-byte swizzle); warp 5 issues tcgen05.mma (M=128, K=16) from one thread and
// commits each stage back to the producer; warps 0-3 read the FP32 accumulator out of tensor
// memory (tcgen05.ld, 32 lanes each) and store C. Every mbarrier wait is bounded: on timeout the
// kernel records an error word, stops issuing, frees its tensor memory and returns.
#include "context.hpp"
#include "workspace.hpp"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

namespace sci_cuda {

    namespace {

        constexpr int kBM = 128, kBK = 64;  // output tile and K slice (bf16: 64 x 2 = 128 bytes)
        constexpr int kUmmaK = 16;
                        constexpr unsigned kProductWait = 1u << 24;

        // ---- conversion: fp32 -> up to three bf16 terms, padded along K -------------------------------
        // a = t0 + t1 + t2 + (a remainder): t0 = bf16(a), t1 = bf16(a - t0), t2 = bf16(a - t0 - t1), each
        // difference exact in float. A is M x K row-major (pitch lda); its terms are M x Kp (Kp = K
        // rounded up to 64, zero-filled).
        struct Terms {
            __nv_bfloat16 *t[3];
        };
        // Eight K-consecutive values of one row split into the terms, one 16-byte store per term (`at`
        // is a multiple of 8: Kp is a multiple of 64 and every term buffer 1024-byte aligned).
        __device__ __forceinline__ void split_eight(const float (&v)[8], int terms, const Terms &out, unsigned long long at) {
            float rest[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) rest[e] = v[e];
            for (int q = 0; q < terms; ++q) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    h[e] = __float2bfloat16_rn(rest[e]);
                    rest[e] = rest[e] - __bfloat162float(h[e]);
                }
                *reinterpret_cast<uint4 *>(out.t[q] + at) = *reinterpret_cast<const uint4 *>(h);
            }
        }

        // A (rows x k, pitch lda) into K-major terms, rows x kp: eight values per thread step, read as
        // two 16-byte vectors where the row allows it.
        // Programmatic dependent launch: returns once the kernel before this one on the stream has
        // finished and its writes are visible, and lets the kernel after this one launch. Both are
        // no-ops in a kernel launched the ordinary way.
        __device__ __forceinline__ void follow_previous() {
            asm volatile("griddepcontrol.wait;" ::: "memory");
            asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
        }

        __global__ void split_rows(const float *__restrict__ a, unsigned long long lda, Terms out, int terms,
                                   unsigned long long rows, unsigned long long k, unsigned long long kp) {
            follow_previous();
            const unsigned long long per_row = kp / 8, total = rows * per_row;
            const bool vector = lda % 4 == 0 && reinterpret_cast<unsigned long long>(a) % 16 == 0;
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < total; i += 256ull * gridDim.x) {
                const unsigned long long r = i / per_row, c = (i - r * per_row) * 8;
                const float *src = a + r * lda + c;
                float v[8];
                if (vector && c + 8 <= k) {
                    const float4 lo = *reinterpret_cast<const float4 *>(src), hi = *reinterpret_cast<const float4 *>(src + 4);
                    v[0] = lo.x, v[1] = lo.y, v[2] = lo.z, v[3] = lo.w, v[4] = hi.x, v[5] = hi.y, v[6] = hi.z, v[7] = hi.w;
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) v[e] = c + e < k ? src[e] : 0.0f;
                }
                split_eight(v, terms, out, r * kp + c);
            }
        }

        // B is K x N row-major (pitch ldb); its terms are the transpose, N x Kp, so both operands are
        // K-major. 64 x 64 tiles through shared memory: read as 16-byte vectors along N, written as
        // 16-byte vectors (eight K values) along K, eight lanes covering one output row's 64 K values
        // so each warp's stores are whole 128-byte lines (one lane per row left every 32-byte sector
        // half written: 108 us for the 8192^2 bf16 term, 3.4 TB/s); the padded pitch keeps both
        // passes free of bank conflicts but for the 2-way ones of the reads.
        __global__ void __launch_bounds__(256) split_transpose(const float *__restrict__ b, unsigned long long ldb, Terms out,
                                                               int terms, unsigned long long k, unsigned long long n,
                                                               unsigned long long kp) {
            __shared__ float tile[64][65];
            follow_previous();
            const unsigned long long k0 = blockIdx.y * 64ull, n0 = blockIdx.x * 64ull;
            const bool vector = ldb % 4 == 0 && reinterpret_cast<unsigned long long>(b) % 16 == 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const unsigned idx = threadIdx.x + 256u * u, kr = idx / 16, nv = idx % 16;
                const unsigned long long kk = k0 + kr, nn = n0 + 4 * nv;
                float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (kk < k) {
                    const float *src = b + kk * ldb + nn;
                    if (vector && nn + 4 <= n) {
                        const float4 q = *reinterpret_cast<const float4 *>(src);
                        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
                    } else {
#pragma unroll
                        for (int e = 0; e < 4; ++e) v[e] = nn + e < n ? src[e] : 0.0f;
                    }
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) tile[kr][4 * nv + e] = v[e];
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                // eight lanes per output row: a warp writes four rows' 128 contiguous bytes each
                const unsigned idx = threadIdx.x + 256u * u, nr = idx / 8, kv = idx % 8;
                if (n0 + nr >= n) continue;
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) v[e] = tile[8 * kv + e][nr];
                split_eight(v, terms, out, (n0 + nr) * kp + k0 + 8 * kv);
            }
        }

        // ---- PTX helpers (tcgen05 / TMA / mbarrier), sm_100a ---------------------------------------
        __device__ __forceinline__ unsigned saddr(const void *p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

        __device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
        }
        __device__ __forceinline__ void mbar_expect(unsigned long long *bar, unsigned bytes) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
        }
        __device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
            unsigned done;
            asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(done)
                    : "r"(saddr(bar)), "r"(parity)
                    : "memory");
            return done != 0;
        }
        __device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
            for (unsigned i = 0; i < kProductWait; ++i) {
                if (mbar_try(bar, parity)) return true;
            }
            return false;
        }
        __device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, unsigned long long *bar) {
            asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                            saddr(dst)),
                    "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(saddr(bar))
                    : "memory");
        }
        __device__ __forceinline__ void tmem_alloc(unsigned *slot, unsigned columns) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(columns)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        __device__ __forceinline__ void tmem_free(unsigned base, unsigned columns) {
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(columns) : "memory");
        }
        // Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
        __device__ __forceinline__ unsigned long long smem_desc(const void *p) {
            const unsigned long long start = (saddr(p) >> 4) & 0x3FFFull;
            const unsigned long long lbo = 1ull, sbo = 1024ull >> 4;
            return start | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
        }
        // kind::f16 instruction descriptor (cute/arch/mma_sm100_desc.hpp InstrDescriptor layout):
        // D = F32 (bits 4-5), A = B = BF16 (bits 7-9, 10-12), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
        __device__ __forceinline__ void mma_bf16(unsigned tmem, unsigned long long a, unsigned long long b, unsigned instr,
                                                 unsigned accumulate) {
            asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(a), "l"(b), "r"(instr), "r"(accumulate)
                    : "memory");
        }
        __device__ __forceinline__ void mma_commit(unsigned long long *bar) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                         : "memory");
        }

        struct ProductArgs {
            float *c;
            unsigned long long m, n, kp, ldc;
            int subtract;  // C -= A B instead of C = A B
            int *status;
        };

        // The bf16 term products a tensor-core tile accumulates: (i, j) multiplies term i of A by term
        // j of B. One term: t0 t0. Two: + t0 t1 + t1 t0. Three: + t0 t2 + t1 t1 + t2 t0 (the dropped
        // products are below 2^-24 relative).
        template <int TERMS> struct Products {
            static constexpr int count = TERMS == 1 ? 1 : (TERMS == 2 ? 3 : 6);
        };
        // product p multiplies term product_a(p) of A by term product_b(p) of B:
        // (0,0) (0,1) (1,0) (0,2) (1,1) (2,0)
        __host__ __device__ constexpr int product_a(int p) { return (p == 2 || p == 4) ? 1 : (p == 5 ? 2 : 0); }
        __host__ __device__ constexpr int product_b(int p) { return (p == 1 || p == 4) ? 1 : (p == 3 ? 2 : 0); }
        template <int TERMS> struct Shape {
            static constexpr int BN = TERMS == 3 ? 128 : 256;  // N of the tile and of the MMA
            static constexpr int stages = TERMS == 1 ? 4 : 2;
            static constexpr unsigned a_bytes = kBM * kBK * 2, b_bytes = BN * kBK * 2;
            static constexpr unsigned stage = TERMS * (a_bytes + b_bytes);
            static constexpr unsigned instr =
                    (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(BN >> 3) << 17) | (unsigned(kBM >> 4) << 24);
        };

        struct Maps {
            CUtensorMap a[3], b[3];
        };

        // One 128 x BN tile of C per CTA.
        template <int TERMS>
        __global__ void __launch_bounds__(192, 1) tensor_product(const __grid_constant__ Maps maps, const ProductArgs args) {
            using Sh = Shape<TERMS>;
            using Pr = Products<TERMS>;
            constexpr int S = Sh::stages, BN = Sh::BN;
            extern __shared__ unsigned char raw[];
            __shared__ unsigned long long full[S], empty[S], done;
            __shared__ unsigned tmem_slot;
            follow_previous();
            __shared__ int abort_flag;
            unsigned char *ring = reinterpret_cast<unsigned char *>((reinterpret_cast<unsigned long long>(raw) + 1023) & ~1023ull);

            const unsigned warp = threadIdx.x / 32, lane = threadIdx.x % 32;
            const unsigned long long m0 = static_cast<unsigned long long>(blockIdx.y) * kBM;
            const unsigned long long n0 = static_cast<unsigned long long>(blockIdx.x) * BN;
            const int kblocks = static_cast<int>(args.kp / kBK);

            if (threadIdx.x == 0) {
                for (int s = 0; s < S; ++s) {
                    mbar_init(&full[s], 1);
                    mbar_init(&empty[s], 1);
                }
                mbar_init(&done, 1);
                abort_flag = 0;
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            if (warp == 0) tmem_alloc(&tmem_slot, BN);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned tmem = tmem_slot;

            if (warp == 4 && lane == 0) {
                // TMA producer: stage = [A term 0 .. TERMS-1][B term 0 .. TERMS-1]
                for (int kb = 0; kb < kblocks; ++kb) {
                    const int s = kb % S;
                    if (kb >= S && !mbar_wait(&empty[s], ((kb / S) - 1) & 1)) {
                        atomicExch(&abort_flag, 1);
                        break;
                    }
                    if (*static_cast<volatile int *>(&abort_flag)) break;
                    unsigned char *stage = ring + s * Sh::stage;
                    mbar_expect(&full[s], Sh::stage);
                    const int x = kb * kBK;
#pragma unroll
                    for (int q = 0; q < TERMS; ++q) {
                        tma_load_2d(stage + q * Sh::a_bytes, &maps.a[q], x, static_cast<int>(m0), &full[s]);
                        tma_load_2d(stage + TERMS * Sh::a_bytes + q * Sh::b_bytes, &maps.b[q], x, static_cast<int>(n0),
                                    &full[s]);
                    }
                }
            } else if (warp == 5 && lane == 0) {
                // MMA issuer
                bool ok = true;
                for (int kb = 0; kb < kblocks; ++kb) {
                    const int s = kb % S;
                    if (!mbar_wait(&full[s], (kb / S) & 1)) {
                        atomicExch(&abort_flag, 1);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    unsigned char *stage = ring + s * Sh::stage;
#pragma unroll
                    for (int kk = 0; kk < kBK / kUmmaK; ++kk) {
                        const unsigned long long step = (kk * kUmmaK * 2) >> 4;  // 32 bytes along K
#pragma unroll
                        for (int p = 0; p < Pr::count; ++p) {
                            const unsigned long long da = smem_desc(stage + product_a(p) * Sh::a_bytes) + step;
                            const unsigned long long db = smem_desc(stage + TERMS * Sh::a_bytes + product_b(p) * Sh::b_bytes) + step;
                            mma_bf16(tmem, da, db, Sh::instr, (kb | kk | p) != 0);
                        }
                    }
                    mma_commit(&empty[s]);  // frees the stage once these MMAs have read it
                }
                if (ok) mma_commit(&done);
                else asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(&done)) : "memory");
            } else if (warp < 4) {
                // Epilogue: TMEM lanes 32*warp .. 32*warp+31 hold rows m0 + 32*warp + lane.
                // tcgen05.ld is warp-collective: the whole warp takes the same branch.
                const bool waited = mbar_wait(&done, 0);
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const bool ok = __all_sync(0xffffffffu, waited && !*static_cast<volatile int *>(&abort_flag));
                if (ok) {
                    const unsigned long long row = m0 + warp * 32 + lane;
#pragma unroll 1
                    for (int chunk = 0; chunk < BN / 32; ++chunk) {
                        unsigned v[32];
                        const unsigned address = tmem + ((warp * 32u) << 16) + chunk * 32u;
                        asm volatile(
                                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                                  "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                                  "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                                  "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                                : "r"(address));
                        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                        const unsigned long long col = n0 + chunk * 32;
                        if (row < args.m) {
                            float *dst = args.c + row * args.ldc + col;
                            if (col + 32 <= args.n && (args.ldc % 4) == 0 &&
                                (reinterpret_cast<unsigned long long>(args.c) % 16) == 0) {
#pragma unroll
                                for (int j = 0; j < 32; j += 4) {
                                    float4 out = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                             __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
                                    if (args.subtract) {
                                        const float4 old = *reinterpret_cast<const float4 *>(dst + j);
                                        out = make_float4(old.x - out.x, old.y - out.y, old.z - out.z, old.w - out.w);
                                    }
                                    *reinterpret_cast<float4 *>(dst + j) = out;
                                }
                            } else {
                                for (int j = 0; j < 32; ++j)
                                    if (col + j < args.n)
                                        dst[j] = args.subtract ? dst[j] - __uint_as_float(v[j]) : __uint_as_float(v[j]);
                            }
                        }
                    }
                } else if (lane == 0 && warp == 0) {
                    atomicOr(args.status, kStatusTimeout);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (warp == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                tmem_free(tmem, BN);
            }
        }

        // ---- the persistent CTA-pair kernel -----------------------------------------------------------
        // Two CTAs of a cluster compute 256 x BN tiles of C together with tcgen05.mma.cta_group::2
        // (M = 256): each CTA stages 128 rows of A and BN / 2 rows of B^T per term and holds 128 rows of
        // the FP32 accumulators in its own tensor memory, so each byte of B a CTA stages feeds twice
        // the tensor work of the one-CTA kernel. The grid is persistent: pair p takes tiles p,
        // p + pairs, ... in a grouped order (kGroup tile rows at a time, so the rows of A and the
        // columns of B in use stay in L2). Tensor memory holds two accumulator buffers of 256 columns:
        // the epilogue drains one while the MMA issuer fills the other.
        //
        // Accuracy of the split modes. The tensor cores' FP32 accumulation loses accuracy in
        // proportion to the number of products accumulated into one accumulator (measured at
        // 8192^3: split3 with one accumulator over all of K was 5.4e-5 relative, twice the split
        // mode's error, where FP32 arithmetic gives 1.6e-6). So with two or three terms each
        // 256 x 128 tile is computed in K segments of kSegment k-blocks, and each buffer holds two
        // accumulators: the leading product t0 * t0 and, separately, the sum of the small products
        // (2^-8 of it and below). The epilogue adds the two in FP32 and adds the segment into C
        // (the first segment stores), so no accumulator takes more than kSegment * 4 leading
        // products.
        //
        // 192 threads per CTA: warps 0-3 epilogue (tensor-memory lanes 32 w .. 32 w + 31), warp 4
        // producer (both CTAs load their halves of each stage, and the bytes are counted on the
        // leader's `full` barrier), warp 5 MMA issuer (leader CTA, rank 0, only). Barriers: full[s]
        // (leader: both CTAs' bytes), empty[s] and acc_full[b] (both CTAs, arrived by the leader's
        // commit, multicast to the pair), acc_empty[b] (leader: one arrival per epilogue warp of both
        // CTAs). Work items are (tile, segment) pairs in the same order for every role. Every wait is
        // bounded: a role whose wait runs out records the timeout in the status word and stops; the
        // others' waits then run out too, and the pair meets at a cluster barrier before freeing its
        // tensor memory.
        constexpr unsigned kGroup = 8;
        constexpr int kSegment = 32;  // k-blocks (64 deep) per segment of the split modes
        template <int TERMS> struct PairShape {
            static constexpr int BN = TERMS == 1 ? 256 : 128;               // N of the tile and of the MMA
            static constexpr bool split = TERMS > 1;                        // two accumulators per buffer
            static constexpr int stages = TERMS == 1 ? 6 : (TERMS == 2 ? 4 : 3);
            static constexpr unsigned a_bytes = 128 * kBK * 2;              // this CTA's rows of A, one term
            static constexpr unsigned b_bytes = (BN / 2) * kBK * 2;         // this CTA's rows of B^T, one term
            static constexpr unsigned stage = TERMS * (a_bytes + b_bytes);  // one CTA's share of a stage
            static constexpr unsigned buffer = 256;                         // tensor-memory columns per buffer
            static constexpr unsigned instr =
                    (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(BN >> 3) << 17) | (unsigned(256 >> 4) << 24);
        };

        __device__ __forceinline__ unsigned pair_rank() {
            unsigned r;
            asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
            return r;
        }
        __device__ __forceinline__ unsigned pair_address(const void *local, unsigned rank) {
            unsigned mapped;
            asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(mapped) : "r"(saddr(local)), "r"(rank));
            return mapped;
        }
        __device__ __forceinline__ void pair_sync() {
            asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
        }
        __device__ __forceinline__ void pair_tma_load(void *dst, const CUtensorMap *map, int x, int y, unsigned leader_bar) {
            asm volatile(
                    "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                            saddr(dst)),
                    "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(leader_bar)
                    : "memory");
        }
        __device__ __forceinline__ void pair_mma(unsigned tmem, unsigned long long a, unsigned long long b, unsigned instr,
                                                 unsigned accumulate) {
            asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(a), "l"(b), "r"(instr), "r"(accumulate)
                    : "memory");
        }
        // Arrives on the barrier at this offset in both CTAs of the pair once the MMAs issued so far are done.
        __device__ __forceinline__ void pair_commit(unsigned long long *bar) {
            asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
                                 saddr(bar)),
                         "h"(static_cast<unsigned short>(0x3))
                         : "memory");
        }
        __device__ __forceinline__ void pair_arrive(unsigned address) {
            asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(address) : "memory");
        }
        // Tile t of the grouped order: kGroup tile rows at a time, down the rows of the group first.
        __device__ __forceinline__ void pair_tile(unsigned t, unsigned tiles_m, unsigned tiles_n, unsigned &tm, unsigned &tn) {
            const unsigned per_group = kGroup * tiles_n;
            const unsigned group = t / per_group, first = group * kGroup;
            const unsigned rows = tiles_m - first < kGroup ? tiles_m - first : kGroup;
            const unsigned local = t - group * per_group;
            tm = first + local % rows;
            tn = local / rows;
        }
        __device__ __forceinline__ void tmem_load32(unsigned address, unsigned (&v)[32]) {
            asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(address));
        }

        template <int TERMS>
        __global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 1)
                tensor_product_pair(const __grid_constant__ Maps maps, const ProductArgs args, unsigned tiles_m,
                                    unsigned tiles_n) {
            using Sh = PairShape<TERMS>;
            using Pr = Products<TERMS>;
            constexpr int S = Sh::stages, BN = Sh::BN;
            extern __shared__ unsigned char raw[];
            __shared__ unsigned long long full[S], empty[S], acc_full[2], acc_empty[2];
            __shared__ unsigned tmem_slot;
            unsigned char *ring = reinterpret_cast<unsigned char *>((reinterpret_cast<unsigned long long>(raw) + 1023) & ~1023ull);

            const unsigned warp = threadIdx.x / 32, lane = threadIdx.x % 32;
            const unsigned rank = pair_rank();
            const unsigned pair = blockIdx.x / 2, pairs = gridDim.x / 2;
            const unsigned tiles = tiles_m * tiles_n;
            const int kblocks = static_cast<int>(args.kp / kBK);
            const int per_segment = Sh::split ? kSegment : kblocks;
            const int segments = (kblocks + per_segment - 1) / per_segment;

            if (threadIdx.x == 0) {
                for (int s = 0; s < S; ++s) {
                    mbar_init(&full[s], 1);
                    mbar_init(&empty[s], 1);
                }
                for (int b = 0; b < 2; ++b) {
                    mbar_init(&acc_full[b], 1);
                    mbar_init(&acc_empty[b], 8);
                }
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            if (warp == 0) {
                asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_slot)),
                             "r"(2 * Sh::buffer)
                             : "memory");
                asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            pair_sync();  // both CTAs' barriers exist before either sees a remote arrival or a transfer
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned tmem = tmem_slot;

            if (warp == 4) {
                if (lane == 0) {
                    // producer: this CTA's 128 rows of A and BN / 2 rows of B^T per term, per stage
                    unsigned s = 0, phase = 0;
                    bool ok = true;
                    for (unsigned t = pair; t < tiles && ok; t += pairs) {
                        unsigned tm, tn;
                        pair_tile(t, tiles_m, tiles_n, tm, tn);
                        const int ya = static_cast<int>(tm * 256 + rank * 128), yb = static_cast<int>(tn * BN + rank * (BN / 2));
                        for (int kb = 0; kb < kblocks && ok; ++kb) {
                            if (!mbar_wait(&empty[s], phase ^ 1u)) {
                                ok = false;
                                break;
                            }
                            if (rank == 0) mbar_expect(&full[s], 2 * Sh::stage);
                            const unsigned bar = pair_address(&full[s], 0);
                            unsigned char *stage = ring + s * Sh::stage;
                            const int x = kb * kBK;
#pragma unroll
                            for (int q = 0; q < TERMS; ++q) {
                                pair_tma_load(stage + q * Sh::a_bytes, &maps.a[q], x, ya, bar);
                                pair_tma_load(stage + TERMS * Sh::a_bytes + q * Sh::b_bytes, &maps.b[q], x, yb, bar);
                            }
                            if (++s == S) {
                                s = 0;
                                phase ^= 1u;
                            }
                        }
                    }
                    if (!ok) atomicOr(args.status, kStatusTimeout);
                }
            } else if (warp == 5) {
                if (rank == 0 && lane == 0) {
                    // MMA issuer: 256 x BN x 16 steps into the accumulators of buffer b for work item i
                    unsigned s = 0, phase = 0, i = 0;
                    bool ok = true;
                    for (unsigned t = pair; t < tiles && ok; t += pairs) {
                        for (int segment = 0; segment < segments && ok; ++segment, ++i) {
                            const unsigned b = i & 1u;
                            if (!mbar_wait(&acc_empty[b], ((i >> 1) & 1u) ^ 1u)) {
                                ok = false;
                                break;
                            }
                            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                            const unsigned lead = tmem + b * Sh::buffer, rest = Sh::split ? lead + BN : lead;
                            const int k0 = segment * per_segment;
                            const int k1 = k0 + per_segment < kblocks ? k0 + per_segment : kblocks;
                            for (int kb = k0; kb < k1; ++kb) {
                                if (!mbar_wait(&full[s], phase)) {
                                    ok = false;
                                    break;
                                }
                                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                                unsigned char *stage = ring + s * Sh::stage;
#pragma unroll
                                for (int kk = 0; kk < kBK / kUmmaK; ++kk) {
                                    const unsigned long long step = (kk * kUmmaK * 2) >> 4;  // 32 bytes along K
                                    const bool first = kb == k0 && kk == 0;
#pragma unroll
                                    for (int p = 0; p < Pr::count; ++p) {
                                        const unsigned long long da = smem_desc(stage + product_a(p) * Sh::a_bytes) + step;
                                        const unsigned long long db =
                                                smem_desc(stage + TERMS * Sh::a_bytes + product_b(p) * Sh::b_bytes) + step;
                                        // the leading product into its own accumulator; the small ones together
                                        const bool into_rest = Sh::split && p > 0;
                                        const bool starts = first && (p == 0 || (into_rest && p == 1));
                                        pair_mma(into_rest ? rest : lead, da, db, Sh::instr, starts ? 0u : 1u);
                                    }
                                }
                                pair_commit(&empty[s]);  // both CTAs' stage s is free once these MMAs have read it
                                if (++s == S) {
                                    s = 0;
                                    phase ^= 1u;
                                }
                            }
                            if (!ok) break;
                            pair_commit(&acc_full[b]);  // the item's accumulators are complete in both CTAs
                        }
                    }
                    if (!ok) atomicOr(args.status, kStatusTimeout);
                }
            } else {
                // epilogue: tensor-memory lanes 32 warp .. 32 warp + 31 hold this CTA's rows
                // tm * 256 + 128 rank + 32 warp + lane; tcgen05.ld is warp-collective
                const unsigned empty0 = pair_address(&acc_empty[0], 0), empty1 = pair_address(&acc_empty[1], 0);
                const bool vector = (args.ldc % 4) == 0 && (reinterpret_cast<unsigned long long>(args.c) % 16) == 0;
                unsigned i = 0;
                bool ok = true;
                for (unsigned t = pair; t < tiles && ok; t += pairs) {
                    unsigned tm, tn;
                    pair_tile(t, tiles_m, tiles_n, tm, tn);
                    const unsigned long long row = 256ull * tm + 128 * rank + warp * 32 + lane;
                    const unsigned long long n0 = 1ull * tn * BN;
                    for (int segment = 0; segment < segments; ++segment, ++i) {
                        const unsigned b = i & 1u;
                        const bool waited = mbar_wait(&acc_full[b], (i >> 1) & 1u);
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        if (!__all_sync(0xffffffffu, waited)) {
                            if (lane == 0) atomicOr(args.status, kStatusTimeout);
                            ok = false;
                            break;
                        }
                        // the first segment of a product stores; later ones (and every segment of a
                        // subtracting update) combine with what C holds
                        const int how = args.subtract ? -1 : (segment == 0 ? 0 : 1);
#pragma unroll 1
                        for (int chunk = 0; chunk < BN / 32; ++chunk) {
                            unsigned v[32];
                            const unsigned address = tmem + ((warp * 32u) << 16) + b * Sh::buffer + chunk * 32u;
                            tmem_load32(address, v);
                            if constexpr (Sh::split) {
                                unsigned w[32];
                                tmem_load32(address + BN, w);
                                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                                for (int j = 0; j < 32; ++j)
                                    v[j] = __float_as_uint(__fadd_rn(__uint_as_float(v[j]), __uint_as_float(w[j])));
                            } else {
                                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                            }
                            const unsigned long long col = n0 + chunk * 32;
                            if (row < args.m && col < args.n) {
                                float *dst = args.c + row * args.ldc + col;
                                if (col + 32 <= args.n && vector) {
#pragma unroll
                                    for (int j = 0; j < 32; j += 4) {
                                        float4 out = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                                 __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
                                        if (how != 0) {
                                            const float4 old = *reinterpret_cast<const float4 *>(dst + j);
                                            out = how < 0 ? make_float4(old.x - out.x, old.y - out.y, old.z - out.z, old.w - out.w)
                                                          : make_float4(old.x + out.x, old.y + out.y, old.z + out.z, old.w + out.w);
                                        }
                                        *reinterpret_cast<float4 *>(dst + j) = out;
                                    }
                                } else {
                                    for (int j = 0; j < 32; ++j) {
                                        if (col + j >= args.n) break;
                                        const float x = __uint_as_float(v[j]);
                                        dst[j] = how == 0 ? x : (how < 0 ? dst[j] - x : dst[j] + x);
                                    }
                                }
                            }
                        }
                        // buffer b may be refilled once all eight epilogue warps have read it
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        __syncwarp();
                        if (lane == 0) pair_arrive(b ? empty1 : empty0);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            pair_sync();  // neither CTA leaves while the pair's MMAs may still read its shared memory
            if (warp == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * Sh::buffer)
                             : "memory");
            }
        }

        // ---- plain SIMT products (the comparison forms) ---------------------------------------------
        // 128 x 128 output tile per 256-thread block, 8 x 8 per thread, K slices of 8 through shared
        // memory. T = float accumulates in float, T = double in double (the reference's
        // multiply<type> accumulates in the element type, dispatch.cpp:171-224).
        // Element (r, q) of A is a[r * a_row + q * a_col] and element (q, j) of B is b[q * b_row + j * b_col],
        // so a transposed operand is read in place.
        template <typename T>
        __global__ void __launch_bounds__(256) simt_product(const T *__restrict__ a, unsigned long long a_row,
                                                            unsigned long long a_col, const T *__restrict__ b,
                                                            unsigned long long b_row, unsigned long long b_col,
                                                            T *__restrict__ c, unsigned long long ldc, unsigned long long m,
                                                            unsigned long long n, unsigned long long k, int subtract) {
            constexpr int BM = 128, BN = 128, BK = 8, TM = 8, TN = 8, LA = BM * BK / 256, LB = BK * BN / 256;
            __shared__ T as[BK][BM + 4];
            __shared__ T bs[BK][BN + 4];
            const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
            const unsigned long long m0 = static_cast<unsigned long long>(blockIdx.y) * BM;
            const unsigned long long n0 = static_cast<unsigned long long>(blockIdx.x) * BN;
            T acc[TM][TN];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
            // A tile: 128 rows x 8 columns, stored transposed; B tile: 8 rows x 128 columns. Each K
            // slice is loaded into registers (all of a thread's loads in flight together) while the
            // previous one is multiplied out of shared memory.
            T ra[LA], rb[LB];
            auto fetch = [&](unsigned long long k0) {
#pragma unroll
                for (int u = 0; u < LA; ++u) {
                    const int i = threadIdx.x + u * 256, r = i / BK, q = i % BK;
                    const unsigned long long gr = m0 + r, gk = k0 + q;
                    ra[u] = (gr < m && gk < k) ? a[gr * a_row + gk * a_col] : T(0);
                }
#pragma unroll
                for (int u = 0; u < LB; ++u) {
                    const int i = threadIdx.x + u * 256, q = i / BN, col = i % BN;
                    const unsigned long long gk = k0 + q, gc = n0 + col;
                    rb[u] = (gk < k && gc < n) ? b[gk * b_row + gc * b_col] : T(0);
                }
            };
            fetch(0);
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
#pragma unroll
                for (int q = 0; q < BK; ++q) {
                    T av[TM], bv[TN];
#pragma unroll
                    for (int i = 0; i < TM; ++i) av[i] = as[q][ty * TM + i];
#pragma unroll
                    for (int j = 0; j < TN; ++j) bv[j] = bs[q][tx * TN + j];
#pragma unroll
                    for (int i = 0; i < TM; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) acc[i][j] = fma_(av[i], bv[j], acc[i][j]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                const unsigned long long r = m0 + ty * TM + i;
                if (r >= m) continue;
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    const unsigned long long col = n0 + tx * TN + j;
                    if (col < n) c[r * ldc + col] = subtract ? c[r * ldc + col] - acc[i][j] : acc[i][j];
                }
            }
        }

        using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                         const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                         CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

        EncodeTiled encoder() {
            static EncodeTiled fn = [] {
                void *p = nullptr;
                cudaDriverEntryPointQueryResult found{};
                if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &found) != cudaSuccess ||
                    found != cudaDriverEntryPointSuccess) {
                    cudaGetLastError();
                    return static_cast<EncodeTiled>(nullptr);
                }
                return reinterpret_cast<EncodeTiled>(p);
            }();
            return fn;
        }

        // Whether products of 256 rows or more run on the CTA-pair kernel (the default); the
        // environment variable SCI_CUDA_PRODUCT_PAIR=0 keeps them on the one-CTA kernel.
        bool pair_kernel_enabled() {
            static const bool enabled = [] {
                const char *setting = std::getenv("SCI_CUDA_PRODUCT_PAIR");
                return !(setting && std::strcmp(setting, "0") == 0);
            }();
            return enabled;
        }

        // CTA pairs of the pair kernel that can be resident at once (persistent grid), at most one
        // per two SMs; cached per kernel.
        unsigned long long pair_slots(const void *kernel, size_t smem, int sms) {
            static std::mutex guard;
            static std::map<const void *, unsigned long long> known;
            std::lock_guard<std::mutex> lock(guard);
            auto found = known.find(kernel);
            if (found != known.end()) return found->second;
            cudaLaunchConfig_t config{};
            config.gridDim = dim3(static_cast<unsigned>(sms / 2 * 2));
            config.blockDim = dim3(192);
            config.dynamicSmemBytes = smem;
            cudaLaunchAttribute attribute[1];
            attribute[0].id = cudaLaunchAttributeClusterDimension;
            attribute[0].val.clusterDim.x = 2;
            attribute[0].val.clusterDim.y = 1;
            attribute[0].val.clusterDim.z = 1;
            config.attrs = attribute;
            config.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &config) != cudaSuccess || clusters < 1) {
                cudaGetLastError();
                clusters = sms / 2;
            }
            const unsigned long long slots = static_cast<unsigned long long>(std::min(clusters, sms / 2));
            known[kernel] = slots;
            return slots;
        }

        // A 2-D bf16 tensor map over a rows x kp K-major matrix, box rows_box x 64, 128-byte swizzle.
        bool make_map(CUtensorMap *map, const void *base, unsigned long long rows, unsigned long long kp, unsigned box_rows) {
            EncodeTiled encode = encoder();
            if (!encode) return false;
            const cuuint64_t dims[2] = {kp, rows};
            const cuuint64_t strides[1] = {kp * 2};
            const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), box_rows};
            const cuuint32_t elements[2] = {1, 1};
            return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, elements,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        }

    } // namespace

    // C (m x n, row pitch ldc) = or -= A (m x k, pitch lda) * B (k x n, pitch ldb) on the tensor cores, each
    // operand split into `terms` bf16 parts (1, 2 or 3). a_t: A is stored transposed (k x m, pitch lda);
    // b_t: B is stored transposed (n x k, pitch ldb). The conversion to K-major bf16 terms absorbs the
    // transposition, so the tensor-core kernel is the same either way.
    int tensor_gemm(Context &ctx, int terms, const float *a, unsigned long long lda, const float *b,
                    unsigned long long ldb, float *c, unsigned long long ldc, unsigned long long m, unsigned long long n,
                    unsigned long long k, bool subtract, bool whole_gpu, bool chained) {
        return tensor_gemm_t(ctx, terms, a, lda, false, b, ldb, false, c, ldc, m, n, k, subtract, whole_gpu, chained);
    }

    int tensor_gemm_t(Context &ctx, int terms, const float *a, unsigned long long lda, bool a_t, const float *b,
                      unsigned long long ldb, bool b_t, float *c, unsigned long long ldc, unsigned long long m,
                      unsigned long long n, unsigned long long k, bool subtract, bool whole_gpu, bool chained) {
        if (terms < 1 || terms > 3) return ctx.fail(SCI_CUDA_ERROR_INVALID, "bf16 terms %d", terms);
        const unsigned long long kp = (k + kBK - 1) / kBK * kBK;
        if (kp > (1ull << 31) || m > (1ull << 31) || n > (1ull << 31))
            return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "product dimensions beyond 2^31");
        const unsigned long long a_bytes = (m * kp * 2 + 1023) / 1024 * 1024, b_bytes = (n * kp * 2 + 1023) / 1024 * 1024;
        const unsigned long long need = terms * (a_bytes + b_bytes) + 1024;
        if (int code = ctx.check(ctx.workspace->reserve(need), "reserving the product workspace")) return code;
        auto *base = static_cast<unsigned char *>(ctx.workspace->memory);
        Terms at{}, bt{};
        for (int q = 0; q < terms; ++q) {
            at.t[q] = reinterpret_cast<__nv_bfloat16 *>(base + q * a_bytes);
            bt.t[q] = reinterpret_cast<__nv_bfloat16 *>(base + terms * a_bytes + q * b_bytes);
        }
        // chained: launched with programmatic stream serialization (the kernels start with
        // follow_previous), else the ordinary way
        auto launch = [&](const void *kernel, dim3 grid, dim3 block, void **params, size_t smem) -> cudaError_t {
            if (!chained) return cudaLaunchKernel(kernel, grid, block, params, smem, ctx.stream);
            cudaLaunchConfig_t config{};
            config.gridDim = grid;
            config.blockDim = block;
            config.dynamicSmemBytes = smem;
            config.stream = ctx.stream;
            cudaLaunchAttribute attribute[1];
            attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attribute[0].val.programmaticStreamSerializationAllowed = 1;
            config.attrs = attribute;
            config.numAttrs = 1;
            return cudaLaunchKernelExC(&config, kernel, params);
        };
        auto rows_of = [&](const float *x, unsigned long long ld, Terms out, unsigned long long rows) {
            const unsigned grid =
                    static_cast<unsigned>(std::min<unsigned long long>((rows * (kp / 8) + 255) / 256, ctx.sms * 16ull));
            int count = terms;
            unsigned long long kk = k, kpp = kp;
            void *params[] = {&x, &ld, &out, &count, &rows, &kk, &kpp};
            return launch(reinterpret_cast<const void *>(&split_rows), dim3(grid), dim3(256), params, 0);
        };
        auto columns_of = [&](const float *x, unsigned long long ld, Terms out, unsigned long long columns) {
            const dim3 tgrid(static_cast<unsigned>((columns + 63) / 64), static_cast<unsigned>(kp / 64));
            int count = terms;
            unsigned long long kk = k, kpp = kp;
            void *params[] = {&x, &ld, &out, &count, &kk, &columns, &kpp};
            return launch(reinterpret_cast<const void *>(&split_transpose), tgrid, dim3(256), params, 0);
        };
        if (int code = ctx.check(a_t ? columns_of(a, lda, at, m) : rows_of(a, lda, at, m), "launching the bf16 conversion"))
            return code;
        if (int code = ctx.check(b_t ? rows_of(b, ldb, bt, n) : columns_of(b, ldb, bt, n), "launching the bf16 conversion"))
            return code;

        ProductArgs args{c, m, n, kp, ldc, subtract ? 1 : 0, ctx.status};
        if (whole_gpu && m >= 256 && pair_kernel_enabled()) {
            // 256 x 256 (one term) or 256 x 128 tiles on CTA pairs, persistent
            Maps maps;
            std::memset(&maps, 0, sizeof(maps));
            for (int q = 0; q < terms; ++q) {
                const unsigned b_box = terms == 1 ? PairShape<1>::BN / 2 : PairShape<3>::BN / 2;
                if (!make_map(&maps.a[q], at.t[q], m, kp, 128) || !make_map(&maps.b[q], bt.t[q], n, kp, b_box))
                    return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "cuTensorMapEncodeTiled failed");
            }
            const void *kernel = terms == 1 ? reinterpret_cast<const void *>(&tensor_product_pair<1>)
                               : terms == 2 ? reinterpret_cast<const void *>(&tensor_product_pair<2>)
                                            : reinterpret_cast<const void *>(&tensor_product_pair<3>);
            const size_t smem = terms == 1 ? PairShape<1>::stages * PairShape<1>::stage + 1024
                              : terms == 2 ? PairShape<2>::stages * PairShape<2>::stage + 1024
                                           : PairShape<3>::stages * PairShape<3>::stage + 1024;
            if (int code = ctx.check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                                     "raising the pair kernel's shared memory"))
                return code;
            const unsigned bn = terms == 1 ? PairShape<1>::BN : PairShape<3>::BN;
            unsigned tiles_m = static_cast<unsigned>((m + 255) / 256), tiles_n = static_cast<unsigned>((n + bn - 1) / bn);
            const unsigned long long tiles = 1ull * tiles_m * tiles_n;
            const unsigned long long pairs = std::min<unsigned long long>(tiles, pair_slots(kernel, smem, ctx.sms));
            void *params[] = {&maps, &args, &tiles_m, &tiles_n};
            return ctx.check(cudaLaunchKernel(kernel, dim3(static_cast<unsigned>(2 * pairs)), dim3(192), params, smem, ctx.stream),
                             "launching the pair tensor product");
        }

        const unsigned bn = terms == 3 ? 128u : 256u;
        Maps maps;
        std::memset(&maps, 0, sizeof(maps));
        for (int q = 0; q < terms; ++q) {
            if (!make_map(&maps.a[q], at.t[q], m, kp, kBM) || !make_map(&maps.b[q], bt.t[q], n, kp, bn))
                return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "cuTensorMapEncodeTiled failed");
        }
        const void *kernel = terms == 1 ? reinterpret_cast<const void *>(&tensor_product<1>)
                           : terms == 2 ? reinterpret_cast<const void *>(&tensor_product<2>)
                                        : reinterpret_cast<const void *>(&tensor_product<3>);
        const size_t smem = terms == 1 ? Shape<1>::stages * Shape<1>::stage + 1024
                          : terms == 2 ? Shape<2>::stages * Shape<2>::stage + 1024
                                       : Shape<3>::stages * Shape<3>::stage + 1024;
        if (int code = ctx.check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                                 "raising the product kernel's shared memory"))
            return code;
        void *params[] = {&maps, &args};
        const dim3 pgrid(static_cast<unsigned>((n + bn - 1) / bn), static_cast<unsigned>((m + kBM - 1) / kBM));
        return ctx.check(launch(kernel, pgrid, dim3(192), params, smem), "launching the tensor product");
    }

    // C (pitch ldc) = or -= A (pitch lda) * B (pitch ldb) with the plain SIMT kernel; a_t / b_t as for
    // tensor_gemm_t.
    template <typename T>
    int simt_gemm_t(Context &ctx, const T *a, unsigned long long lda, bool a_t, const T *b, unsigned long long ldb, bool b_t,
                    T *c, unsigned long long ldc, unsigned long long m, unsigned long long n, unsigned long long k,
                    bool subtract) {
        const dim3 grid(static_cast<unsigned>((n + 127) / 128), static_cast<unsigned>((m + 127) / 128));
        if (grid.y > 65535) return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "too many rows for one launch");
        if (m == 0 || n == 0) return SCI_CUDA_OK;
        simt_product<T><<<grid, 256, 0, ctx.stream>>>(a, a_t ? 1ull : lda, a_t ? lda : 1ull, b, b_t ? 1ull : ldb,
                                                      b_t ? ldb : 1ull, c, ldc, m, n, k, subtract ? 1 : 0);
        return ctx.check(cudaGetLastError(), "launching the SIMT product");
    }
    template <typename T>
    int simt_gemm(Context &ctx, const T *a, unsigned long long lda, const T *b, unsigned long long ldb, T *c,
                  unsigned long long ldc, unsigned long long m, unsigned long long n, unsigned long long k, bool subtract) {
        return simt_gemm_t<T>(ctx, a, lda, false, b, ldb, false, c, ldc, m, n, k, subtract);
    }
    template int simt_gemm_t<float>(Context &, const float *, unsigned long long, bool, const float *, unsigned long long,
                                    bool, float *, unsigned long long, unsigned long long, unsigned long long,
                                    unsigned long long, bool);
    template int simt_gemm_t<double>(Context &, const double *, unsigned long long, bool, const double *,
                                     unsigned long long, bool, double *, unsigned long long, unsigned long long,
                                     unsigned long long, unsigned long long, bool);
    template int simt_gemm<float>(Context &, const float *, unsigned long long, const float *, unsigned long long, float *,
                                  unsigned long long, unsigned long long, unsigned long long, unsigned long long, bool);
    template int simt_gemm<double>(Context &, const double *, unsigned long long, const double *, unsigned long long,
                                   double *, unsigned long long, unsigned long long, unsigned long long, unsigned long long,
                                   bool);

} // namespace sci_cuda

using namespace sci_cuda;

extern "C" int sci_cuda_product(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *left,
                                const void *right, void *output, uint64_t rows, uint64_t columns, uint64_t depth) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || mode > SCI_PRODUCT_SPLIT3_BF16)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or mode %u", precision, mode);
    if (rows == 0 || columns == 0) return SCI_CUDA_OK;
    if (!left || !right || !output) return context->fail(SCI_CUDA_ERROR_INVALID, "null matrix");
    cudaSetDevice(context->device);
    const size_t element = precision == SCI_PRECISION_WIDE ? 8 : 4;
    if (depth == 0) {  // dispatch.cpp:270-273
        return context->check(cudaMemsetAsync(output, 0, rows * columns * element, context->stream), "zeroing the product");
    }
    if (precision == SCI_PRECISION_WIDE) {
        return simt_gemm<double>(*context, static_cast<const double *>(left), depth, static_cast<const double *>(right),
                                 columns, static_cast<double *>(output), columns, rows, columns, depth, false);
    }
    if (mode == SCI_PRODUCT_FP32) {
        return simt_gemm<float>(*context, static_cast<const float *>(left), depth, static_cast<const float *>(right),
                                columns, static_cast<float *>(output), columns, rows, columns, depth, false);
    }
    return tensor_gemm(*context, mode == SCI_PRODUCT_SPLIT3_BF16 ? 3 : (mode == SCI_PRODUCT_SPLIT_BF16 ? 2 : 1),
                       static_cast<const float *>(left), depth,
                       static_cast<const float *>(right), columns, static_cast<float *>(output), columns, rows, columns,
                       depth, false, true);
}

extern "C" int sci_cuda_product_gradient(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *left,
                                         const void *right, const void *upstream, void *left_gradient, void *right_gradient,
                                         uint64_t rows, uint64_t columns, uint64_t depth) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || mode > SCI_PRODUCT_SPLIT3_BF16)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or mode %u", precision, mode);
    if (!upstream || (left_gradient && !right) || (right_gradient && !left))
        return context->fail(SCI_CUDA_ERROR_INVALID, "null matrix");
    cudaSetDevice(context->device);
    const size_t element = precision == SCI_PRECISION_WIDE ? 8 : 4;
    // d left (rows x depth) = G (rows x columns) * right^T; d right (depth x columns) = left^T * G.
    // An empty inner dimension (columns for d left, rows for d right) gives zeros.
    auto one = [&](void *out, const void *a, uint64_t lda, bool a_t, const void *b, uint64_t ldb, bool b_t, uint64_t m,
                   uint64_t n, uint64_t k) -> int {
        if (!out || m == 0 || n == 0) return SCI_CUDA_OK;
        if (k == 0) return context->check(cudaMemsetAsync(out, 0, m * n * element, context->stream), "zeroing a gradient");
        if (precision == SCI_PRECISION_WIDE)
            return simt_gemm_t<double>(*context, static_cast<const double *>(a), lda, a_t, static_cast<const double *>(b), ldb,
                                       b_t, static_cast<double *>(out), n, m, n, k, false);
        if (mode == SCI_PRODUCT_FP32)
            return simt_gemm_t<float>(*context, static_cast<const float *>(a), lda, a_t, static_cast<const float *>(b), ldb,
                                      b_t, static_cast<float *>(out), n, m, n, k, false);
        return tensor_gemm_t(*context, mode == SCI_PRODUCT_SPLIT3_BF16 ? 3 : (mode == SCI_PRODUCT_SPLIT_BF16 ? 2 : 1),
                             static_cast<const float *>(a), lda, a_t, static_cast<const float *>(b), ldb, b_t,
                             static_cast<float *>(out), n, m, n, k, false, true);
    };
    if (int code = one(left_gradient, upstream, columns, false, right, columns, true, rows, depth, columns)) return code;
    return one(right_gradient, left, depth, true, upstream, columns, false, depth, columns, rows);
}
