// BF16 GEMM on the 5th-generation tensor cores (tcgen05, FP32 accumulators in tensor memory, operands brought in by
// TMA) for the warm-start MLP's forward and backward passes: C[M][N] (f32) = sum_k A(m, k) B(n, k), each operand
// either K-major (stored [rows][K], K contiguous) or MN-major (stored [K][rows], the M or N index contiguous), with
// row strides for padded storage and an optional split of K into slices summed afterwards in slice order.
//
// Structure (one persistent CTA of 6 warps per SM, 128 x 256 output tiles, 64-wide K blocks):
//   warp 0, one thread -- producer: per K block, waits until its stage of a 4-stage shared-memory ring is free and
//                         issues the TMA tile loads of A (16 KB) and B (32 KB) into it (128-byte swizzle), counted on
//                         the stage's `full` mbarrier by transaction bytes;
//   warp 1             -- allocates 512 TMEM columns (two 128 x 256 FP32 accumulators); one thread issues, per K
//                         block, four tcgen05.mma (K = 16 each) and commits them to the stage's `empty` mbarrier (the
//                         stage is reusable once the MMAs have read it), and after a tile's last block commits to the
//                         accumulator's `full` mbarrier;
//   warps 2-5          -- epilogue: wait for an accumulator, read it with tcgen05.ld (each warp the 32 TMEM lanes of
//                         its quadrant), store FP32 rows, and release the accumulator; the other accumulator is
//                         meanwhile being filled with the next tile.
// Tiles are visited M-fastest, so the CTAs working at the same time share B tiles (the weights) in L2. Every
// mbarrier wait is bounded; a wait that gives up sets *err, the CTA stops issuing work, waits (bounded) for the TMA
// loads and MMAs it started, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "../../include/taral_pdhg.h"

namespace taral {
namespace tc {

using bf16 = __nv_bfloat16;
constexpr int TM = 128, TN = 256, TK = 64, kStages = 4;
constexpr int kBytesA = TM * TK * 2, kBytesB = TN * TK * 2, kStageBytes = kBytesA + kBytesB;
constexpr int kEpiFloats = 32 * 33;  // per epilogue warp: a 32 x 32 chunk of the accumulator, rows padded to 33
constexpr int kSmemBytes = kStages * kStageBytes + 4 * kEpiFloats * 4 + 1024;  // + alignment slack: 1 CTA per SM
constexpr uint32_t kTmemCols = 512;                        // two accumulators of 256 columns
constexpr int kThreads = 192;
constexpr int kSpinLimit = 1 << 24;

// Instruction descriptor of tcgen05.mma kind::f16: F32 accumulate (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 =
// 1), A MN-major (bit 15), B MN-major (bit 16), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc(bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u) |
           (uint32_t(TN >> 3) << 17) | (uint32_t(TM >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Shared-memory descriptor of a tile in the 128-byte swizzle (version 1, layout SWIZZLE_128B = 2). K-major: rows of
// 128 B (64 K elements), 8-row atoms 1024 B apart (stride byte offset), leading byte offset unused (1). MN-major:
// rows of 128 B along M / N (64 elements) for one k, 8-k atoms 1024 B apart (stride byte offset) and 64-element M /
// N atoms `mn_atom` bytes apart (leading byte offset). Offsets in 16-byte units.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr, uint32_t lbo_bytes) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo_bytes >> 4) & 0x3FFF) << 16) |
           (uint64_t(1024 >> 4) << 32) | (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

__device__ __forceinline__ bool wait_parity(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

struct GemmShape {
    int M, N, K, ldc;
    int m_tiles, n_tiles, slices, kb_per_slice, kb_total;
    int a_mn, b_mn;
};

// C (or, with slices > 1, the partial of slice s at ws + s * M * ldc) for every (m tile, n tile, K slice) work item.
__global__ void __launch_bounds__(kThreads, 1) k_umma_gemm(const __grid_constant__ CUtensorMap mapA,
                                                           const __grid_constant__ CUtensorMap mapB, GemmShape g,
                                                           float* __restrict__ C, int* err) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2], drain;
    __shared__ uint32_t tmem_sh;
    __shared__ int failed;
    const uint32_t s0 = smem_u32(smem_raw), pad = (1024u - (s0 & 1023u)) & 1023u;
    const uint32_t ring = s0 + pad;  // 1024-byte aligned: the swizzle pattern is a function of the address bits
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int items = g.m_tiles * g.n_tiles * g.slices;

    if (tid == 0) {
        failed = 0;
        for (int s = 0; s < kStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])));
        }
        for (int a = 0; a < 2; ++a) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&acc_full[a])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(smem_u32(&acc_empty[a])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&drain)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_sh;
    auto stopped = [&] { return *reinterpret_cast<volatile int*>(&failed) != 0; };  // set by another role's thread

    auto item_coords = [&](int item, int& m0, int& n0, int& kb0, int& kb1, int& slice) {
        const int mt = item % g.m_tiles, rest = item / g.m_tiles;
        slice = rest % g.slices;
        m0 = mt * TM, n0 = (rest / g.slices) * TN;
        kb0 = slice * g.kb_per_slice;
        kb1 = min(kb0 + g.kb_per_slice, g.kb_total);
    };

    if (warp == 0) {
        if (lane == 0) {  // producer
            uint32_t it = 0;
            for (int item = blockIdx.x; item < items && !stopped(); item += gridDim.x) {
                int m0, n0, kb0, kb1, slice;
                item_coords(item, m0, n0, kb0, kb1, slice);
                for (int kb = kb0; kb < kb1; ++kb, ++it) {
                    const uint32_t s = it % kStages, use = it / kStages;
                    if (use > 0 && !wait_parity(smem_u32(&empty[s]), (use - 1) & 1)) {
                        atomicOr(&failed, 1);
                        break;
                    }
                    const uint32_t fb = smem_u32(&full[s]), a = ring + s * kStageBytes, b = a + kBytesA;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                                 "r"(uint32_t(kStageBytes))
                                 : "memory");
                    const int k0 = kb * TK;
                    if (g.a_mn) {  // [K][M] storage: two boxes of 64 M x 64 K
                        tma_load(a, &mapA, m0, k0, fb);
                        tma_load(a + 8192, &mapA, m0 + 64, k0, fb);
                    } else {  // [M][K] storage: one box of 64 K x 128 M
                        tma_load(a, &mapA, k0, m0, fb);
                    }
                    if (g.b_mn) {  // [K][N]: four boxes of 64 N x 64 K
                        for (int j = 0; j < 4; ++j) tma_load(b + 8192 * j, &mapB, n0 + 64 * j, k0, fb);
                    } else {  // [N][K]: one box of 64 K x 256 N
                        tma_load(b, &mapB, k0, n0, fb);
                    }
                }
            }
            // drain: every stage this thread filled has been consumed or its loads have landed before exit
            const uint32_t issued = it;
            for (uint32_t q = issued > kStages ? issued - kStages : 0; q < issued; ++q)
                wait_parity(smem_u32(&full[q % kStages]), (q / kStages) & 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            const uint32_t id = idesc(g.a_mn != 0, g.b_mn != 0);
            const uint32_t lbo_a = g.a_mn ? 8192u : 16u, lbo_b = g.b_mn ? 8192u : 16u;
            const uint32_t kstep_a = g.a_mn ? 2048u : 32u, kstep_b = g.b_mn ? 2048u : 32u;  // 16 K elements
            uint32_t it = 0, tile = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < items && ok && !stopped(); item += gridDim.x, ++tile) {
                int m0, n0, kb0, kb1, slice;
                item_coords(item, m0, n0, kb0, kb1, slice);
                const uint32_t acc = tile & 1, use = tile >> 1;
                if (use > 0 && !wait_parity(smem_u32(&acc_empty[acc]), (use - 1) & 1)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t d = tmem + acc * 256;
                for (int kb = kb0; kb < kb1; ++kb, ++it) {
                    const uint32_t s = it % kStages;
                    if (!wait_parity(smem_u32(&full[s]), (it / kStages) & 1)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t a = ring + s * kStageBytes, b = a + kBytesA;
#pragma unroll
                    for (int ks = 0; ks < TK / 16; ++ks) {
                        const uint64_t ad = sw128_desc(a + ks * kstep_a, lbo_a), bd = sw128_desc(b + ks * kstep_b, lbo_b);
                        const uint32_t accumulate = (kb > kb0 || ks > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                            "l"(ad), "l"(bd), "r"(id), "r"(accumulate));
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&empty[s]))
                                 : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&acc_full[acc]))
                             : "memory");
            }
            if (!ok) atomicOr(&failed, 1);
            // every MMA this thread issued has completed before the tensor memory is freed
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&drain))
                         : "memory");
            if (!wait_parity(smem_u32(&drain), 0)) atomicOr(&failed, 1);
        }
    } else {  // epilogue, warps 2-5: TMEM lanes 32 (warp % 4) .. + 31
        const int q = warp & 3;
        uint32_t tile = 0;
        for (int item = blockIdx.x; item < items; item += gridDim.x, ++tile) {
            int m0, n0, kb0, kb1, slice;
            item_coords(item, m0, n0, kb0, kb1, slice);
            const uint32_t acc = tile & 1, use = tile >> 1;
            if (stopped() || !wait_parity(smem_u32(&acc_full[acc]), use & 1)) {
                atomicOr(&failed, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            // lane l holds row (m0 + 32 q + l) of each 32-column chunk; the chunk goes through this warp's tile in
            // shared memory so that each store instruction writes 32 consecutive floats of one row
            float* tile_sm = reinterpret_cast<float*>(smem_raw + pad + kStages * kStageBytes) + (warp - 2) * kEpiFloats;
            float* out = C + size_t(slice) * size_t(g.M) * g.ldc;
#pragma unroll 1
            for (int cb = 0; cb < TN / 32; ++cb) {
                uint32_t r[32];
                const uint32_t taddr = tmem + (uint32_t(q * 32) << 16) + acc * 256 + uint32_t(cb * 32);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int c0 = n0 + cb * 32, col = c0 + lane;
#pragma unroll
                for (int i = 0; i < 32; ++i) tile_sm[lane * 33 + i] = __uint_as_float(r[i]);  // banks (lane + i) % 32
                __syncwarp();
#pragma unroll 8
                for (int rr = 0; rr < 32; ++rr) {
                    const int row = m0 + q * 32 + rr;
                    if (row < g.M && col < g.N) out[size_t(row) * g.ldc + col] = tile_sm[rr * 33 + lane];
                }
                __syncwarp();
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[acc])) : "memory");
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 1) {
        __syncwarp();  // the warp converged for the .sync.aligned dealloc
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
    if (tid == 0 && failed) atomicExch(err, 1);
}

// Sum of the slice partials in slice order (deterministic): C[r][c] = sum_s ws[s][r][c].
__global__ void k_sum_slices(int M, int N, int ldc, int slices, const float* __restrict__ ws, float* __restrict__ C) {
    const size_t total = size_t(M) * N;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const size_t r = e / size_t(N), c = e % size_t(N), at = r * size_t(ldc) + c;
        float s = 0.f;
        for (int q = 0; q < slices; ++q) s += ws[size_t(q) * size_t(M) * ldc + at];
        C[at] = s;
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link-time dependency on the driver library).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// A bf16 matrix stored row-major [rows][ld] (cols <= ld used), read in boxes of 64 columns x box_rows rows with the
// 128-byte swizzle; out-of-range elements read as zero.
static bool make_map(CUtensorMap* m, const void* base, int rows, int cols, int ld, int box_rows) {
    const auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
    const cuuint64_t strides[1] = {cuuint64_t(ld) * 2};
    const cuuint32_t box[2] = {64u, cuuint32_t(box_rows)};
    const cuuint32_t estr[2] = {1u, 1u};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C[M][N] (row stride ldc) = sum_k A(m, k) B(n, k). a_mn = 0: A stored [M][lda] (K contiguous); 1: [K][lda] (M
// contiguous); likewise b_mn for B with N. lda, ldb multiples of 8 (16-byte rows), A and B 16-byte aligned.
// slices > 1: K split into that many slices whose partials go to ws (slices * M * ldc floats) and are summed in
// order into C. err: device int set to 1 when a completion wait gave up (the result is then undefined).
int gemm_umma(int M, int N, int K, const void* A, int lda, int a_mn, const void* B, int ldb, int b_mn, float* C,
              int ldc, int slices, float* ws, int* err, cudaStream_t stream) {
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C || !err || ldc < N) return TARAL_ERR_INPUT;
    if (lda % 8 || ldb % 8 || lda < (a_mn ? M : K) || ldb < (b_mn ? N : K)) return TARAL_ERR_INPUT;
    if (reinterpret_cast<uintptr_t>(A) % 16 || reinterpret_cast<uintptr_t>(B) % 16) return TARAL_ERR_INPUT;
    slices = slices < 1 ? 1 : slices;
    if (slices > 1 && !ws) return TARAL_ERR_INPUT;
    CUtensorMap ma, mb;
    const bool okA = a_mn ? make_map(&ma, A, K, M, lda, 64) : make_map(&ma, A, M, K, lda, TM);
    const bool okB = b_mn ? make_map(&mb, B, K, N, ldb, 64) : make_map(&mb, B, N, K, ldb, TN);
    if (!okA || !okB) return TARAL_ERR_CUDA;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return TARAL_ERR_CUDA;
    {  // the shared-memory opt-in is a per-device attribute of the kernel: set once on every device used
        static std::mutex mu;
        static bool configured[64] = {};
        std::lock_guard<std::mutex> lock(mu);
        if (!configured[dev]) {
            if (cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) !=
                cudaSuccess)
                return TARAL_ERR_CUDA;
            configured[dev] = true;
        }
    }
    GemmShape g;
    g.M = M, g.N = N, g.K = K, g.ldc = ldc, g.a_mn = a_mn, g.b_mn = b_mn;
    g.m_tiles = (M + TM - 1) / TM, g.n_tiles = (N + TN - 1) / TN;
    g.kb_total = (K + TK - 1) / TK;
    slices = slices > g.kb_total ? g.kb_total : slices;
    g.kb_per_slice = (g.kb_total + slices - 1) / slices;
    g.slices = (g.kb_total + g.kb_per_slice - 1) / g.kb_per_slice;  // every slice holds at least one K block
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int items = g.m_tiles * g.n_tiles * g.slices;
    k_umma_gemm<<<items < sms ? items : sms, kThreads, kSmemBytes, stream>>>(ma, mb, g, g.slices > 1 ? ws : C, err);
    if (g.slices > 1) k_sum_slices<<<sms * 4, 256, 0, stream>>>(M, N, ldc, g.slices, ws, C);
    return cudaGetLastError() == cudaSuccess ? TARAL_OK : TARAL_ERR_CUDA;
}

int gemm_tc(int M, int N, int K, const void* A, const void* Bt, float* C, int* err, cudaStream_t stream) {
    if (K % 8) return TARAL_ERR_INPUT;
    return gemm_umma(M, N, K, A, K, 0, Bt, K, 0, C, N, 1, nullptr, err, stream);
}

}  // namespace tc
}  // namespace taral

// C (M x N, f32) = A (M x K, bf16, row-major) * Bt (N x K, bf16, row-major)^T on the tcgen05 tensor cores.
// K must be a multiple of 8 and A, Bt 16-byte aligned. err: device int, set to 1 when an MMA completion wait gave
// up (the result is then undefined).
extern "C" int taral_gemm_bf16_tc(int M, int N, int K, const void* A, const void* Bt, float* C, int* err,
                                  void* stream) {
    return taral::tc::gemm_tc(M, N, K, A, Bt, C, err, static_cast<cudaStream_t>(stream));
}

// The general form: operand layouts, row strides and split-K (see gemm_umma).
extern "C" int taral_gemm_bf16_umma(int M, int N, int K, const void* A, int lda, int a_mn, const void* B, int ldb,
                                    int b_mn, float* C, int ldc, int slices, float* ws, int* err, void* stream) {
    return taral::tc::gemm_umma(M, N, K, A, lda, a_mn, B, ldb, b_mn, C, ldc, slices, ws, err,
                                static_cast<cudaStream_t>(stream));
}
