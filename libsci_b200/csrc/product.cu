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
//  - SCI_PRODUCT_FP32: a plain FP32 SIMT kernel, the comparison form.
// Double products run a plain FP64 SIMT kernel.
//
// The tensor-core kernel: one CTA per 128 x 256 output tile, six warps. Warp 4 issues TMA loads of
// 64-deep K slices of A (128 x 64) and of B^T (256 x 64) into a ring of shared-memory stages
// (128-byte swizzle); warp 5 issues tcgen05.mma (M=128, N=256, K=16) from one thread and
// commits each stage back to the producer; warps 0-3 read the FP32 accumulator out of tensor
// memory (tcgen05.ld, 32 lanes each) and store C. Every mbarrier wait is bounded: on timeout the
// kernel records an error word, stops issuing, frees its tensor memory and returns.
#include "context.hpp"
#include "workspace.hpp"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

namespace sci_cuda {

    namespace {

        constexpr int kBM = 128, kBN = 256, kBK = 64;  // output tile and K slice (bf16: 64 x 2 = 128 bytes)
        constexpr int kUmmaK = 16;
        constexpr int kStagesPlain = 4, kStagesSplit = 2;
        constexpr unsigned kTmemColumns = 256;
        constexpr unsigned kProductWait = 1u << 24;

        // ---- conversion: fp32 -> bf16 (hi, and lo = bf16(a - hi)), padded along K ----------------
        // A is M x K row-major; its bf16 copies are M x Kp (Kp = K rounded up to 64, zero-filled).
        __global__ void split_rows(const float *__restrict__ a, __nv_bfloat16 *__restrict__ hi,
                                   __nv_bfloat16 *__restrict__ lo, unsigned long long rows, unsigned long long k,
                                   unsigned long long kp) {
            const unsigned long long total = rows * kp;
            for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < total; i += 256ull * gridDim.x) {
                const unsigned long long r = i / kp, c = i % kp;
                const float v = c < k ? a[r * k + c] : 0.0f;
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                hi[i] = h;
                if (lo) lo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
            }
        }

        // B is K x N row-major; its bf16 copies are the transpose, N x Kp, so both operands are
        // K-major. 32 x 32 tiles through shared memory keep both sides coalesced.
        __global__ void split_transpose(const float *__restrict__ b, __nv_bfloat16 *__restrict__ hi,
                                        __nv_bfloat16 *__restrict__ lo, unsigned long long k, unsigned long long n,
                                        unsigned long long kp) {
            __shared__ float tile[32][33];
            const unsigned long long k0 = blockIdx.y * 32ull, n0 = blockIdx.x * 32ull;
            const unsigned tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
            for (unsigned j = ty; j < 32; j += 8) {
                const unsigned long long kk = k0 + j, nn = n0 + tx;
                tile[j][tx] = (kk < k && nn < n) ? b[kk * n + nn] : 0.0f;
            }
            __syncthreads();
            for (unsigned j = ty; j < 32; j += 8) {
                const unsigned long long nn = n0 + j, kk = k0 + tx;
                if (nn < n && kk < kp) {
                    const float v = tile[tx][j];
                    const __nv_bfloat16 h = __float2bfloat16_rn(v);
                    hi[nn * kp + kk] = h;
                    if (lo) lo[nn * kp + kk] = __float2bfloat16_rn(v - __bfloat162float(h));
                }
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
        // kind::f16 instruction descriptor: D = F32, A = B = BF16, both K-major, M = 128, N = 256.
        constexpr unsigned kInstr = (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(kBN >> 3) << 17) | (unsigned(kBM >> 4) << 24);

        __device__ __forceinline__ void mma_bf16(unsigned tmem, unsigned long long a, unsigned long long b, unsigned accumulate) {
            asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(a), "l"(b), "r"(kInstr), "r"(accumulate)
                    : "memory");
        }
        __device__ __forceinline__ void mma_commit(unsigned long long *bar) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                         : "memory");
        }

        struct ProductArgs {
            float *c;
            unsigned long long m, n, kp;
            int *status;
        };

        // One 128 x 256 tile of C per CTA. `split` adds the hi*lo and lo*hi products.
        template <bool split>
        __global__ void __launch_bounds__(192, 1)
                tensor_product(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
                               const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo,
                               const ProductArgs args) {
            constexpr int S = split ? kStagesSplit : kStagesPlain;
            constexpr unsigned A_BYTES = kBM * kBK * 2, B_BYTES = kBN * kBK * 2;
            constexpr unsigned STAGE = split ? 2 * (A_BYTES + B_BYTES) : (A_BYTES + B_BYTES);
            extern __shared__ unsigned char raw[];
            __shared__ unsigned long long full[S], empty[S], done;
            __shared__ unsigned tmem_slot;
            __shared__ int abort_flag;
            unsigned char *ring = reinterpret_cast<unsigned char *>((reinterpret_cast<unsigned long long>(raw) + 1023) & ~1023ull);

            const unsigned warp = threadIdx.x / 32, lane = threadIdx.x % 32;
            const unsigned long long m0 = static_cast<unsigned long long>(blockIdx.y) * kBM;
            const unsigned long long n0 = static_cast<unsigned long long>(blockIdx.x) * kBN;
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
            if (warp == 0) tmem_alloc(&tmem_slot, kTmemColumns);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned tmem = tmem_slot;

            if (warp == 4 && lane == 0) {
                // TMA producer
                for (int kb = 0; kb < kblocks; ++kb) {
                    const int s = kb % S;
                    if (kb >= S && !mbar_wait(&empty[s], ((kb / S) - 1) & 1)) {
                        atomicExch(&abort_flag, 1);
                        break;
                    }
                    if (*static_cast<volatile int *>(&abort_flag)) break;
                    unsigned char *stage = ring + s * STAGE;
                    mbar_expect(&full[s], STAGE);
                    const int x = kb * kBK;
                    tma_load_2d(stage, &a_hi, x, static_cast<int>(m0), &full[s]);
                    tma_load_2d(stage + A_BYTES, &b_hi, x, static_cast<int>(n0), &full[s]);
                    if constexpr (split) {
                        tma_load_2d(stage + A_BYTES + B_BYTES, &a_lo, x, static_cast<int>(m0), &full[s]);
                        tma_load_2d(stage + 2 * A_BYTES + B_BYTES, &b_lo, x, static_cast<int>(n0), &full[s]);
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
                    unsigned char *stage = ring + s * STAGE;
                    const unsigned long long ah = smem_desc(stage), bh = smem_desc(stage + A_BYTES);
#pragma unroll
                    for (int kk = 0; kk < kBK / kUmmaK; ++kk) {
                        const unsigned long long step = (kk * kUmmaK * 2) >> 4;  // 32 bytes along K
                        mma_bf16(tmem, ah + step, bh + step, (kb | kk) != 0);
                        if constexpr (split) {
                            const unsigned long long al = smem_desc(stage + A_BYTES + B_BYTES);
                            const unsigned long long bl = smem_desc(stage + 2 * A_BYTES + B_BYTES);
                            mma_bf16(tmem, ah + step, bl + step, 1);
                            mma_bf16(tmem, al + step, bh + step, 1);
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
                    for (int chunk = 0; chunk < kBN / 32; ++chunk) {
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
                            float *dst = args.c + row * args.n + col;
                            if (col + 32 <= args.n && (args.n % 4) == 0 &&
                                (reinterpret_cast<unsigned long long>(args.c) % 16) == 0) {
#pragma unroll
                                for (int j = 0; j < 32; j += 4)
                                    *reinterpret_cast<float4 *>(dst + j) = make_float4(
                                            __uint_as_float(v[j]), __uint_as_float(v[j + 1]), __uint_as_float(v[j + 2]),
                                            __uint_as_float(v[j + 3]));
                            } else {
                                for (int j = 0; j < 32; ++j)
                                    if (col + j < args.n) dst[j] = __uint_as_float(v[j]);
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
                tmem_free(tmem, kTmemColumns);
            }
        }

        // ---- plain SIMT products (the comparison forms) ---------------------------------------------
        // 128 x 128 output tile per 256-thread block, 8 x 8 per thread, K slices of 8 through shared
        // memory. T = float accumulates in float, T = double in double (the reference's
        // multiply<type> accumulates in the element type, dispatch.cpp:171-224).
        template <typename T>
        __global__ void __launch_bounds__(256) simt_product(const T *__restrict__ a, const T *__restrict__ b, T *__restrict__ c,
                                                            unsigned long long m, unsigned long long n, unsigned long long k) {
            constexpr int BM = 128, BN = 128, BK = 8, TM = 8, TN = 8;
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
            for (unsigned long long k0 = 0; k0 < k; k0 += BK) {
                // A tile: 128 rows x 8 columns, stored transposed; B tile: 8 rows x 128 columns.
                for (int i = threadIdx.x; i < BM * BK; i += 256) {
                    const int r = i / BK, q = i % BK;
                    const unsigned long long gr = m0 + r, gk = k0 + q;
                    as[q][r] = (gr < m && gk < k) ? a[gr * k + gk] : T(0);
                }
                for (int i = threadIdx.x; i < BK * BN; i += 256) {
                    const int q = i / BN, col = i % BN;
                    const unsigned long long gk = k0 + q, gc = n0 + col;
                    bs[q][col] = (gk < k && gc < n) ? b[gk * n + gc] : T(0);
                }
                __syncthreads();
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
                    if (col < n) c[r * n + col] = acc[i][j];
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

        int tensor_path(Context &ctx, bool split, const float *a, const float *b, float *c, unsigned long long m,
                        unsigned long long n, unsigned long long k) {
            const unsigned long long kp = (k + kBK - 1) / kBK * kBK;
            if (kp > (1ull << 31) || m > (1ull << 31) || n > (1ull << 31))
                return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "product dimensions beyond 2^31");
            const unsigned long long a_bytes = m * kp * 2, b_bytes = n * kp * 2;
            const unsigned long long need = (split ? 2 : 1) * (a_bytes + b_bytes) + 1024;
            if (int code = ctx.check(ctx.workspace->reserve(need), "reserving the product workspace")) return code;
            auto *base = static_cast<unsigned char *>(ctx.workspace->memory);
            auto *a_hi = reinterpret_cast<__nv_bfloat16 *>(base);
            auto *b_hi = reinterpret_cast<__nv_bfloat16 *>(base + a_bytes);
            __nv_bfloat16 *a_lo = split ? reinterpret_cast<__nv_bfloat16 *>(base + a_bytes + b_bytes) : nullptr;
            __nv_bfloat16 *b_lo = split ? reinterpret_cast<__nv_bfloat16 *>(base + 2 * a_bytes + b_bytes) : nullptr;

            const unsigned grid = static_cast<unsigned>(std::min<unsigned long long>((m * kp + 255) / 256, ctx.sms * 16ull));
            split_rows<<<grid, 256, 0, ctx.stream>>>(a, a_hi, a_lo, m, k, kp);
            const dim3 tgrid(static_cast<unsigned>((n + 31) / 32), static_cast<unsigned>((kp + 31) / 32));
            split_transpose<<<tgrid, dim3(32, 8), 0, ctx.stream>>>(b, b_hi, b_lo, k, n, kp);
            if (int code = ctx.check(cudaGetLastError(), "launching the bf16 conversion")) return code;

            CUtensorMap maps[4];
            std::memset(maps, 0, sizeof(maps));
            if (!make_map(&maps[0], a_hi, m, kp, kBM) || !make_map(&maps[2], b_hi, n, kp, kBN))
                return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "cuTensorMapEncodeTiled failed");
            if (split && (!make_map(&maps[1], a_lo, m, kp, kBM) || !make_map(&maps[3], b_lo, n, kp, kBN)))
                return ctx.fail(SCI_CUDA_ERROR_LAUNCH, "cuTensorMapEncodeTiled failed");
            if (!split) {
                maps[1] = maps[0];
                maps[3] = maps[2];
            }
            const int stages = split ? kStagesSplit : kStagesPlain;
            const unsigned stage_bytes = (split ? 2u : 1u) * (kBM * kBK * 2 + kBN * kBK * 2);
            const size_t smem = static_cast<size_t>(stages) * stage_bytes + 1024;
            const void *kernel = split ? reinterpret_cast<const void *>(&tensor_product<true>)
                                       : reinterpret_cast<const void *>(&tensor_product<false>);
            if (int code = ctx.check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                                     "raising the product kernel's shared memory"))
                return code;
            ProductArgs args{c, m, n, kp, ctx.status};
            void *params[] = {&maps[0], &maps[1], &maps[2], &maps[3], &args};
            const dim3 pgrid(static_cast<unsigned>((n + kBN - 1) / kBN), static_cast<unsigned>((m + kBM - 1) / kBM));
            return ctx.check(cudaLaunchKernel(kernel, pgrid, dim3(192), params, smem, ctx.stream), "launching the tensor product");
        }

        template <typename T>
        int simt_path(Context &ctx, const T *a, const T *b, T *c, unsigned long long m, unsigned long long n,
                      unsigned long long k) {
            const dim3 grid(static_cast<unsigned>((n + 127) / 128), static_cast<unsigned>((m + 127) / 128));
            if (grid.y > 65535) return ctx.fail(SCI_CUDA_ERROR_UNSUPPORTED, "too many rows for one launch");
            simt_product<T><<<grid, 256, 0, ctx.stream>>>(a, b, c, m, n, k);
            return ctx.check(cudaGetLastError(), "launching the SIMT product");
        }

    } // namespace

} // namespace sci_cuda

using namespace sci_cuda;

extern "C" int sci_cuda_product(sci_cuda_context *context, uint32_t precision, uint32_t mode, const void *left,
                                const void *right, void *output, uint64_t rows, uint64_t columns, uint64_t depth) {
    if (!context) return SCI_CUDA_ERROR_INVALID;
    std::lock_guard<std::recursive_mutex> lock(context->guard);
    if (precision > SCI_PRECISION_WIDE || mode > SCI_PRODUCT_FP32)
        return context->fail(SCI_CUDA_ERROR_INVALID, "unknown precision %u or mode %u", precision, mode);
    if (rows == 0 || columns == 0) return SCI_CUDA_OK;
    if (!left || !right || !output) return context->fail(SCI_CUDA_ERROR_INVALID, "null matrix");
    cudaSetDevice(context->device);
    const size_t element = precision == SCI_PRECISION_WIDE ? 8 : 4;
    if (depth == 0) {  // dispatch.cpp:270-273
        return context->check(cudaMemsetAsync(output, 0, rows * columns * element, context->stream), "zeroing the product");
    }
    if (precision == SCI_PRECISION_WIDE) {
        return simt_path<double>(*context, static_cast<const double *>(left), static_cast<const double *>(right),
                                 static_cast<double *>(output), rows, columns, depth);
    }
    if (mode == SCI_PRODUCT_FP32) {
        return simt_path<float>(*context, static_cast<const float *>(left), static_cast<const float *>(right),
                                static_cast<float *>(output), rows, columns, depth);
    }
    return tensor_path(*context, mode == SCI_PRODUCT_SPLIT_BF16, static_cast<const float *>(left),
                       static_cast<const float *>(right), static_cast<float *>(output), rows, columns, depth);
}
