// BF16 GEMM on the 5th-generation tensor cores (tcgen05, accumulator in tensor memory) for the warm-start MLP's
// inference pass: C[M][N] (f32) = A[M][K] * Bt[N][K]^T, both operands K-major bf16 (A = activations, Bt = the
// layer's weights transposed). Checked against the mma.sync GEMM of mlp.cu by the tests.
//
// One CTA (4 warps) computes a 128 x 256 tile; per 64-wide K slice the CTA stages A (16 KB) and Bt (32 KB) in shared
// memory in the 128-byte-swizzled K-major layout the MMA reads through its shared-memory descriptors, one thread
// issues four tcgen05.mma (K = 16 each) into a 128-lane x 256-column FP32 accumulator in tensor memory and commits
// them to an mbarrier; every wait is bounded and a timeout sets *err. The epilogue reads the accumulator with
// tcgen05.ld (each warp its 32 lanes) and writes C.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/taral_pdhg.h"

namespace taral {
namespace tc {

using bf16 = __nv_bfloat16;
constexpr int TM = 128, TN = 256, TK = 64;
constexpr int kBytesA = TM * TK * 2, kBytesB = TN * TK * 2;
constexpr int kSmemBytes = 100 * 1024;  // more than A + B + alignment: at most 2 CTAs per SM, TMEM never oversubscribed
constexpr uint32_t kTmemCols = 256;
static_assert(kBytesA + kBytesB + 1023 <= kSmemBytes, "staging tiles plus alignment slack must fit");
constexpr int kSpinLimit = 1 << 22;

// Instruction descriptor of tcgen05.mma kind::f16: F32 accumulate (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 =
// 1), both K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(TN >> 3) << 17) | (uint32_t(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Shared-memory descriptor of a K-major tile with 128-byte rows in the 128-byte swizzle: start address >> 4
// (bits 0-13), leading byte offset 1 (unused for swizzled K-major, bits 16-29), stride byte offset between 8-row
// groups 1024 B >> 4 (bits 32-45), descriptor version 1 (bits 46-47), layout SWIZZLE_128B = 2 (bits 61-63).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) | (uint64_t(1) << 46) |
           (uint64_t(2) << 61);
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

__global__ void __launch_bounds__(128) k_gemm_tc(int M, int N, int K, const bf16* __restrict__ A,
                                                 const bf16* __restrict__ Bt, float* __restrict__ C, int* err) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_sh;
    __shared__ int failed;
    const uint32_t s0 = smem_u32(smem_raw), pad = (1024u - (s0 & 1023u)) & 1023u;
    uint8_t* sA = smem_raw + pad;  // 1024-byte aligned: the swizzle pattern is a function of the address bits
    uint8_t* sB = sA + kBytesA;
    const uint32_t aA = s0 + pad, aB = aA + kBytesA, aBar = smem_u32(&mbar);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        failed = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(aBar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_sh;

    uint32_t parity = 0;
    for (int k0 = 0; k0 < K; k0 += TK) {
        for (int c = tid; c < TM * 8; c += 128) {  // A: 128 rows x 8 chunks of 16 B, chunk j of row r at j ^ (r & 7)
            const int r = c >> 3, j = c & 7, gm = m0 + r, gk = k0 + j * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gm < M && gk + 8 <= K) v = *reinterpret_cast<const uint4*>(A + size_t(gm) * K + gk);
            *reinterpret_cast<uint4*>(sA + r * 128 + ((j ^ (r & 7)) << 4)) = v;
        }
        for (int c = tid; c < TN * 8; c += 128) {  // Bt: 256 rows x 8 chunks
            const int r = c >> 3, j = c & 7, gn = n0 + r, gk = k0 + j * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gn < N && gk + 8 <= K) v = *reinterpret_cast<const uint4*>(Bt + size_t(gn) * K + gk);
            *reinterpret_cast<uint4*>(sB + r * 128 + ((j ^ (r & 7)) << 4)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> the MMA's async proxy
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int ks = 0; ks < TK / 16; ++ks) {  // K = 16 per MMA: advance the start address by 32 bytes
                const uint64_t ad = sw128_desc(aA + ks * 32), bd = sw128_desc(aB + ks * 32);
                const uint32_t accumulate = (k0 > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(kIdesc), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(aBar)
                         : "memory");
        }
        if (!wait_parity(aBar, parity)) atomicOr(&failed, 1);  // the MMAs have read this slice
        asm volatile("tcgen05.fence::after_thread_sync;");
        __syncthreads();
        if (failed) {                  // CTA-uniform (read after the barrier)
            wait_parity(aBar, parity);  // one more bounded wait for MMAs still in flight before TMEM is freed
            break;
        }
        parity ^= 1u;
    }

    if (!failed) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int cb = 0; cb < TN / 32; ++cb) {
            uint32_t r[32];
            const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(cb * 32);
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
            if (row < M) {
                float* out = C + size_t(row) * N + n0 + cb * 32;
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (n0 + cb * 32 + i < N) out[i] = __uint_as_float(r[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    if (tid == 0 && failed) atomicExch(err, 1);
}

int gemm_tc(int M, int N, int K, const void* A, const void* Bt, float* C, int* err, cudaStream_t stream) {
    if (M <= 0 || N <= 0 || K <= 0 || K % 8 || !A || !Bt || !C || !err) return TARAL_ERR_INPUT;
    if (reinterpret_cast<uintptr_t>(A) % 16 || reinterpret_cast<uintptr_t>(Bt) % 16) return TARAL_ERR_INPUT;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess)
            return TARAL_ERR_CUDA;
        configured = true;
    }
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    k_gemm_tc<<<grid, 128, kSmemBytes, stream>>>(M, N, K, static_cast<const bf16*>(A), static_cast<const bf16*>(Bt),
                                                  C, err);
    return cudaGetLastError() == cudaSuccess ? TARAL_OK : TARAL_ERR_CUDA;
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
