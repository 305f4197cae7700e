// Learned warm start: a small MLP (in -> hidden x depth, GELU -> out) trained and evaluated on the GPU with this
// file's own BF16 tensor-core kernels (include/taral_pdhg.h, part 7). It maps a scenario's 256-dim price/capacity
// perturbation to an initial (x, y) for the PDHG solve. No counterpart in the reference.
//
// Layout: weights W_l bf16 [in_l][out_l] row-major (with FP32 master copies and Adam moments), biases FP32.
// Forward per layer: C = H_{l-1} W_l (GEMM, FP32 accumulate), Z = C + b, H = bf16(gelu(Z)) (last layer: Y = Z).
// Backward: dW = H_{l-1}^T dZ, db = sum_b dZ, dH_{l-1} = dZ W_l^T, dZ = dH * gelu'(Z); loss = mean (Y - T)^2.
//
// GEMMs: for every layer whose input width is a multiple of 8 (and whose dZ rows are 16-byte multiples: the output
// gradient of the last layer is stored with its row stride rounded up to 8) all three GEMMs run on the tcgen05 tensor
// cores through TMA (mlp_tc.cu, gemm_umma): the forward C = H Wt^T with Wt = W^T kept as a bf16 [out][in] copy
// refreshed whenever the weights change (both operands K-major), dW = H_prev^T dZ (both operands read MN-major) and
// dH_prev = dZ W^T (dZ K-major, Wt MN-major, K split into slices summed in order). Any other layer uses mma.sync
// m16n8k16 (bf16 x bf16 -> f32), 128 x 128 x 32 CTA tiles, 8 warps of 64 x 32, operands staged in shared memory and
// fed with ldmatrix; A may be stored transposed (TA: A = X^T) and B as [N][K] (TB: B = W^T); split-K writes per-slice
// partials that a second kernel adds in slice order (deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/taral_pdhg.h"

namespace taral {
namespace tc {
int gemm_tc(int M, int N, int K, const void* A, const void* Bt, float* C, int* err, cudaStream_t stream);
int gemm_umma(int M, int N, int K, const void* A, int lda, int a_mn, const void* B, int ldb, int b_mn, float* C,
              int ldc, int slices, float* ws, int* err, cudaStream_t stream);
}
namespace mlp {

using bf16 = __nv_bfloat16;

struct MlpError {
    std::string msg;
};
#define MK(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) throw MlpError{std::string(#call) + ": " + cudaGetErrorString(e_)};      \
    } while (0)

constexpr int BM = 128, BN = 128, BK = 32, PAD = 8;

__device__ __forceinline__ void ldsm_x4(const bf16* p, uint32_t (&r)[4]) {
    uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[z][M][N] = sum over k in slice z of op(A)[m][k] op(B)[k][n].
//   TA = false: A stored [M][K];  TA = true: A stored [K][M] (op(A) = stored^T).
//   TB = false: B stored [K][N];  TB = true: B stored [N][K].
// VEC: every dimension is a multiple of 8 and the pointers are 16-byte aligned (8-element vector loads).
template <bool TA, bool TB, bool VEC>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, int kslice, const bf16* __restrict__ A,
                                              const bf16* __restrict__ B, float* __restrict__ C) {
    __shared__ __align__(16) bf16 As[BM][BK + PAD];
    __shared__ __align__(16) bf16 Bs[BN][BK + PAD];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 2, wn = warp & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kb = blockIdx.z * kslice, ke = min(K, kb + kslice);
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
    const bf16 zero = __float2bfloat16(0.f);
    for (int k0 = kb; k0 < ke; k0 += BK) {
        // ---- A tile: As[m][k]
        for (int v = tid; v < BM * BK / 8; v += 256) {
            if (!TA) {
                const int r = v / (BK / 8), c8 = (v % (BK / 8)) * 8, gm = m0 + r, gk = k0 + c8;
                if (VEC && gm < M && gk + 8 <= ke) {
                    *reinterpret_cast<uint4*>(&As[r][c8]) = *reinterpret_cast<const uint4*>(A + size_t(gm) * K + gk);
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) As[r][c8 + e] = (gm < M && gk + e < ke) ? A[size_t(gm) * K + gk + e] : zero;
                }
            } else {
                const int kk = v / (BM / 8), m8 = (v % (BM / 8)) * 8, gk = k0 + kk, gm = m0 + m8;
                if (VEC && gk < ke && gm + 8 <= M) {
                    uint4 q = *reinterpret_cast<const uint4*>(A + size_t(gk) * M + gm);
                    const bf16* e8 = reinterpret_cast<const bf16*>(&q);
#pragma unroll
                    for (int e = 0; e < 8; ++e) As[m8 + e][kk] = e8[e];
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) As[m8 + e][kk] = (gk < ke && gm + e < M) ? A[size_t(gk) * M + gm + e] : zero;
                }
            }
        }
        // ---- B tile: Bs[n][k]
        for (int v = tid; v < BN * BK / 8; v += 256) {
            if (TB) {
                const int r = v / (BK / 8), c8 = (v % (BK / 8)) * 8, gn = n0 + r, gk = k0 + c8;
                if (VEC && gn < N && gk + 8 <= ke) {
                    *reinterpret_cast<uint4*>(&Bs[r][c8]) = *reinterpret_cast<const uint4*>(B + size_t(gn) * K + gk);
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) Bs[r][c8 + e] = (gn < N && gk + e < ke) ? B[size_t(gn) * K + gk + e] : zero;
                }
            } else {
                const int kk = v / (BN / 8), n8 = (v % (BN / 8)) * 8, gk = k0 + kk, gn = n0 + n8;
                if (VEC && gk < ke && gn + 8 <= N) {
                    uint4 q = *reinterpret_cast<const uint4*>(B + size_t(gk) * N + gn);
                    const bf16* e8 = reinterpret_cast<const bf16*>(&q);
#pragma unroll
                    for (int e = 0; e < 8; ++e) Bs[n8 + e][kk] = e8[e];
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) Bs[n8 + e][kk] = (gk < ke && gn + e < N) ? B[size_t(gk) * N + gn + e] : zero;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t a[4][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) ldsm_x4(&As[wm * 64 + mi * 16 + (lane & 15)][ks + (lane >> 4) * 8], a[mi]);
#pragma unroll
            for (int nj = 0; nj < 2; ++nj) {
                uint32_t r[4];
                ldsm_x4(&Bs[wn * 32 + nj * 16 + (lane & 7) + (lane >> 4) * 8][ks + ((lane >> 3) & 1) * 8], r);
                b[2 * nj][0] = r[0], b[2 * nj][1] = r[1], b[2 * nj + 1][0] = r[2], b[2 * nj + 1][1] = r[3];
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], a[mi], b[ni]);
        }
        __syncthreads();
    }
    float* Cz = C + size_t(blockIdx.z) * M * N;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int row = m0 + wm * 64 + mi * 16 + (lane >> 2), col = n0 + wn * 32 + ni * 8 + (lane & 3) * 2;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int rr = row + 8 * h;
                if (rr < M) {
                    if (col < N) Cz[size_t(rr) * N + col] = acc[mi][ni][2 * h];
                    if (col + 1 < N) Cz[size_t(rr) * N + col + 1] = acc[mi][ni][2 * h + 1];
                }
            }
        }
}

// C = sum over slices s of P[s] (fixed order).
__global__ void k_splitk_sum(size_t count, int slices, const float* __restrict__ P, float* __restrict__ C) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < slices; ++z) s += P[size_t(z) * count + i];
        C[i] = s;
    }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// Z = C + b; H = bf16(gelu(Z)) (act) or Y = Z (no act, H may be NULL).
__global__ void k_bias_act(int rows, int cols, const float* __restrict__ C, const float* __restrict__ b,
                           float* __restrict__ Z, bf16* __restrict__ H, int act) {
    const size_t n = size_t(rows) * cols;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float z = C[i] + b[i % cols];
        Z[i] = z;
        if (H) H[i] = __float2bfloat16(act ? gelu(z) : z);
    }
}

// R = Y - T (FP32), dY = bf16(2 R / (rows * cols)); per-row partial sums of R^2 into part[row].
__global__ void k_loss_grad(int rows, int cols, int ldy, const float* __restrict__ Y, const float* __restrict__ T,
                            float* __restrict__ R, bf16* __restrict__ dY, double* __restrict__ part) {
    const int row = blockIdx.x;
    const float scale = 2.f / (float(rows) * float(cols));
    double s = 0;
    for (int j = threadIdx.x; j < cols; j += blockDim.x) {
        const size_t i = size_t(row) * cols + j;
        const float r = Y[i] - T[i];
        R[i] = r * scale;
        dY[size_t(row) * ldy + j] = __float2bfloat16(r * scale);  // row stride ldy >= cols (padded for TMA)
        s += double(r) * double(r);
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sh[w];
        part[row] = t;
    }
}

// db[j] = sum over rows of G[r][j] (fixed order).
__global__ void k_colsum(int rows, int cols, const float* __restrict__ G, float* __restrict__ db) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cols; j += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int r = 0; r < rows; ++r) s += G[size_t(r) * cols + j];
        db[j] = s;
    }
}

// dZ = dH * gelu'(Z): FP32 copy (for db) and bf16 copy (GEMM operand).
__global__ void k_gelu_back(size_t n, const float* __restrict__ dH, const float* __restrict__ Z, float* __restrict__ dZf,
                            bf16* __restrict__ dZ) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float g = dH[i] * gelu_grad(Z[i]);
        dZf[i] = g;
        dZ[i] = __float2bfloat16(g);
    }
}

__global__ void k_to_bf16(size_t n, const float* __restrict__ src, bf16* __restrict__ dst) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] = __float2bfloat16(src[i]);
}

// Adam on FP32 masters; refreshes the bf16 copy.
__global__ void k_adam(size_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, bf16* __restrict__ wb, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi, v = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a, m2[i] = v;
        const float wi = w[i] - lr * (a / c1) / (sqrtf(v / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

// Wt[c][r] = W[r][c] for W rows x cols (bf16), through a 32 x 32 shared-memory tile.
__global__ void k_transpose(int rows, int cols, const bf16* __restrict__ W, bf16* __restrict__ Wt) {
    __shared__ bf16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int i = ty; i < 32; i += 8) {
        const int r = r0 + i, c = c0 + tx;
        if (r < rows && c < cols) t[i][tx] = W[size_t(r) * cols + c];
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        const int c = c0 + i, r = r0 + tx;
        if (r < rows && c < cols) Wt[size_t(c) * rows + r] = t[tx][i];
    }
}

// Gather dataset rows idx[0..rows) into contiguous batch buffers.
__global__ void k_gather_rows(int rows, int cols, const int* __restrict__ idx, const float* __restrict__ src,
                              float* __restrict__ dst, bf16* __restrict__ dstb) {
    const size_t n = size_t(rows) * cols;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const size_t r = i / cols, c = i % cols;
        const float v = src[size_t(idx[r]) * cols + c];
        if (dst) dst[i] = v;
        if (dstb) dstb[i] = __float2bfloat16(v);
    }
}

static int grid1(size_t n) { return int(std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16))); }

struct Layer {
    int in = 0, out = 0;
    float *W = nullptr, *b = nullptr, *gW = nullptr, *gb = nullptr, *mW = nullptr, *vW = nullptr, *mb = nullptr,
          *vb = nullptr;
    bf16* Wb = nullptr;
    bf16* Wt = nullptr;  // W^T [out][in] (the tcgen05 forward GEMM's K-major B operand); null: forward on mma.sync
    float* Z = nullptr;  // pre-activation [batch][out]
    bf16* H = nullptr;   // activation [batch][out] (GEMM operand of the next layer)
};

struct Mlp {
    int in_dim = 0, hidden = 0, depth = 0, out_dim = 0, max_batch = 0;
    std::vector<Layer> L;
    bf16* Xb = nullptr;  // input batch
    float *Xf = nullptr, *Tf = nullptr, *C = nullptr, *R = nullptr, *dHf = nullptr, *dZf = nullptr, *ws = nullptr;
    bf16 *dYb = nullptr, *dZb = nullptr;
    int ldy = 0;  // row stride of dYb: the output width, rounded up to 8 when the last layer's backward runs on tcgen05
    double* part = nullptr;
    int* d_idx = nullptr;
    int* d_err = nullptr;  // set by the tcgen05 GEMM when a completion wait gave up
    float *DX = nullptr, *DT = nullptr;  // dataset
    int dcount = 0;
    size_t ws_count = 0;
    int64_t steps = 0;
    cudaStream_t s = nullptr;
    std::vector<void*> allocs;
    std::string err;

    template <class U>
    U* alloc(size_t n) {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(U));
        if (e != cudaSuccess) throw MlpError{std::string("cudaMalloc: ") + cudaGetErrorString(e)};
        allocs.push_back(p);
        return static_cast<U*>(p);
    }
    ~Mlp() {
        if (s) cudaStreamSynchronize(s);
        for (void* p : allocs) cudaFree(p);
        if (s) cudaStreamDestroy(s);
    }

    void create(int in, int hid, int dep, int out, int mb) {
        in_dim = in, hidden = hid, depth = dep, out_dim = out, max_batch = mb;
        MK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        int prev = in;
        for (int l = 0; l <= depth; ++l) {
            Layer y;
            y.in = prev, y.out = l < depth ? hidden : out;
            size_t nw = size_t(y.in) * y.out;
            y.W = alloc<float>(nw), y.gW = alloc<float>(nw), y.mW = alloc<float>(nw), y.vW = alloc<float>(nw);
            y.Wb = alloc<bf16>(nw);
            if (y.in % 8 == 0) y.Wt = alloc<bf16>(nw);
            y.b = alloc<float>(y.out), y.gb = alloc<float>(y.out), y.mb = alloc<float>(y.out), y.vb = alloc<float>(y.out);
            y.Z = alloc<float>(size_t(mb) * y.out), y.H = alloc<bf16>(size_t(mb) * y.out);
            MK(cudaMemsetAsync(y.mW, 0, nw * sizeof(float), s));
            MK(cudaMemsetAsync(y.vW, 0, nw * sizeof(float), s));
            MK(cudaMemsetAsync(y.mb, 0, y.out * sizeof(float), s));
            MK(cudaMemsetAsync(y.vb, 0, y.out * sizeof(float), s));
            L.push_back(y);
            prev = y.out;
        }
        size_t widest = std::max<size_t>(size_t(out), size_t(hid));
        Xb = alloc<bf16>(size_t(mb) * in), Xf = alloc<float>(size_t(mb) * in), Tf = alloc<float>(size_t(mb) * out);
        ldy = L[depth].Wt ? (out + 7) / 8 * 8 : out;
        C = alloc<float>(size_t(mb) * widest), R = alloc<float>(size_t(mb) * out), dYb = alloc<bf16>(size_t(mb) * ldy);
        dHf = alloc<float>(size_t(mb) * widest), dZf = alloc<float>(size_t(mb) * hid), dZb = alloc<bf16>(size_t(mb) * hid);
        part = alloc<double>(mb), d_idx = alloc<int>(mb), d_err = alloc<int>(1);
        MK(cudaMemsetAsync(d_err, 0, sizeof(int), s));
        ws_count = size_t(64) * mb * hid;  // split-K partials of dH = dZ W^T (K = out)
        ws = alloc<float>(ws_count);
        MK(cudaStreamSynchronize(s));
    }

    int64_t param_count() const {
        int64_t n = 0;
        for (const Layer& y : L) n += int64_t(y.in) * y.out + y.out;
        return n;
    }

    // C[M][N] = op(A) op(B); split-K (slices > 1) through the workspace.
    template <bool TA, bool TB>
    void gemm(int M, int N, int K, const bf16* A, const bf16* B, float* out, int slices = 1) {
        bool vec = M % 8 == 0 && N % 8 == 0 && K % 8 == 0 && (reinterpret_cast<uintptr_t>(A) % 16 == 0) &&
                   (reinterpret_cast<uintptr_t>(B) % 16 == 0);
        int kslice = (K + slices - 1) / slices;
        kslice = (kslice + BK - 1) / BK * BK;
        slices = (K + kslice - 1) / kslice;
        float* dst = slices > 1 ? ws : out;
        if (slices > 1 && size_t(slices) * M * N > ws_count) throw MlpError{"split-K workspace too small"};
        dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, slices);
        if (vec) k_gemm<TA, TB, true><<<grid, 256, 0, s>>>(M, N, K, kslice, A, B, dst);
        else k_gemm<TA, TB, false><<<grid, 256, 0, s>>>(M, N, K, kslice, A, B, dst);
        if (slices > 1) k_splitk_sum<<<grid1(size_t(M) * N), 256, 0, s>>>(size_t(M) * N, slices, ws, out);
        MK(cudaGetLastError());
    }

    void refresh_transposes() {  // Wt = Wb^T for the layers whose forward GEMM runs on tcgen05
        for (Layer& y : L)
            if (y.Wt) {
                dim3 grid((y.out + 31) / 32, (y.in + 31) / 32);
                k_transpose<<<grid, 256, 0, s>>>(y.in, y.out, y.Wb, y.Wt);
            }
        MK(cudaGetLastError());
    }

    void check_tc() {  // after a stream synchronisation: did a tcgen05 GEMM give up waiting?
        int e = 0;
        MK(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
        MK(cudaStreamSynchronize(s));
        if (e) {
            MK(cudaMemsetAsync(d_err, 0, sizeof(int), s));
            throw MlpError{"tcgen05 GEMM: an MMA completion wait timed out"};
        }
    }

    void forward(int batch) {  // Xb -> L[l].Z, L[l].H ; output Z of the last layer is Y
        const bf16* in = Xb;
        for (int l = 0; l <= depth; ++l) {
            Layer& y = L[l];
            if (y.Wt) {
                if (taral::tc::gemm_tc(batch, y.out, y.in, in, y.Wt, C, d_err, s) != TARAL_OK)
                    throw MlpError{std::string("tcgen05 GEMM launch: ") + cudaGetErrorString(cudaGetLastError())};
            } else {
                gemm<false, false>(batch, y.out, y.in, in, y.Wb, C);
            }
            k_bias_act<<<grid1(size_t(batch) * y.out), 256, 0, s>>>(batch, y.out, C, y.b, y.Z, l < depth ? y.H : nullptr,
                                                                    l < depth ? 1 : 0);
            in = y.H;
        }
        MK(cudaGetLastError());
    }

    double backward(int batch) {  // needs forward(batch) and Tf; fills gW, gb; returns the loss
        Layer& top = L[depth];
        k_loss_grad<<<batch, 256, 0, s>>>(batch, top.out, ldy, top.Z, Tf, R, dYb, part);
        const bf16* dZ = dYb;
        const float* dZfl = R;
        int ldz = ldy;  // row stride of dZ
        for (int l = depth; l >= 0; --l) {
            Layer& y = L[l];
            const bf16* Hprev = l > 0 ? L[l - 1].H : Xb;
            // tcgen05 when the operands fit TMA (16-byte rows): dW = H_prev^T dZ reads both operands MN-major,
            // dH_prev = dZ W^T reads dZ K-major and W^T (kept as Wt [out][in]) MN-major; mma.sync otherwise
            const bool tc = y.Wt && ldz % 8 == 0;
            if (tc) {
                if (taral::tc::gemm_umma(y.in, y.out, batch, Hprev, y.in, 1, dZ, ldz, 1, y.gW, y.out, 1, nullptr, d_err, s) !=
                    TARAL_OK)
                    throw MlpError{std::string("tcgen05 GEMM launch: ") + cudaGetErrorString(cudaGetLastError())};
            } else {
                gemm<true, false>(y.in, y.out, batch, Hprev, dZ, y.gW);              // dW = H_prev^T dZ
            }
            k_colsum<<<grid1(y.out), 256, 0, s>>>(batch, y.out, dZfl, y.gb);     // db = sum_b dZ
            if (l > 0) {
                if (tc) {
                    const int tiles = ((batch + 127) / 128) * ((y.in + 255) / 256);
                    const size_t per_slice = size_t(batch) * y.in;
                    const int slices = int(std::max<size_t>(1, std::min<size_t>(std::max(1, 148 / tiles),
                                                                                ws_count / per_slice)));
                    if (taral::tc::gemm_umma(batch, y.in, y.out, dZ, ldz, 0, y.Wt, y.in, 1, dHf, y.in, slices, ws, d_err, s) !=
                        TARAL_OK)
                        throw MlpError{std::string("tcgen05 GEMM launch: ") + cudaGetErrorString(cudaGetLastError())};
                } else {
                    int slices = std::max(1, std::min(64, y.out / 2048));
                    gemm<false, true>(batch, y.in, y.out, dZ, y.Wb, dHf, slices);    // dH_prev = dZ W^T
                }
                Layer& p = L[l - 1];
                k_gelu_back<<<grid1(size_t(batch) * p.out), 256, 0, s>>>(size_t(batch) * p.out, dHf, p.Z, dZf, dZb);
                dZ = dZb, dZfl = dZf, ldz = p.out;
            }
        }
        std::vector<double> h(batch);
        MK(cudaMemcpyAsync(h.data(), part, batch * sizeof(double), cudaMemcpyDeviceToHost, s));
        MK(cudaStreamSynchronize(s));
        double t = 0;
        for (double v : h) t += v;
        return t / (double(batch) * top.out);
    }

    void adam(float lr) {
        ++steps;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        float c1 = 1.f - std::pow(b1, float(steps)), c2 = 1.f - std::pow(b2, float(steps));
        for (Layer& y : L) {
            size_t nw = size_t(y.in) * y.out;
            k_adam<<<grid1(nw), 256, 0, s>>>(nw, y.W, y.gW, y.mW, y.vW, y.Wb, lr, b1, b2, eps, c1, c2);
            k_adam<<<grid1(y.out), 256, 0, s>>>(y.out, y.b, y.gb, y.mb, y.vb, nullptr, lr, b1, b2, eps, c1, c2);
        }
        refresh_transposes();
    }

    void load_input(int batch, const float* x_host) {
        MK(cudaMemcpyAsync(Xf, x_host, size_t(batch) * in_dim * sizeof(float), cudaMemcpyHostToDevice, s));
        k_to_bf16<<<grid1(size_t(batch) * in_dim), 256, 0, s>>>(size_t(batch) * in_dim, Xf, Xb);
    }
};

}  // namespace mlp
}  // namespace taral

// ================================================================================================ C ABI
using taral::mlp::Mlp;
using taral::mlp::MlpError;

struct taral_mlp {
    Mlp m;
};

#define MLP_GUARD(h, ...)                                     \
    try {                                                     \
        __VA_ARGS__;                                          \
        return TARAL_OK;                                      \
    } catch (const MlpError& e) {                             \
        (h)->m.err = e.msg;                                   \
        return e.msg.find("cudaMalloc") != std::string::npos ? TARAL_ERR_ALLOC : TARAL_ERR_CUDA; \
    } catch (const std::bad_alloc&) {                         \
        return TARAL_ERR_ALLOC;                               \
    }

extern "C" int taral_mlp_create(int in_dim, int hidden, int depth, int out_dim, int max_batch, taral_mlp** out) {
    if (!out || in_dim <= 0 || hidden <= 0 || depth < 0 || out_dim <= 0 || max_batch <= 0) return TARAL_ERR_INPUT;
    *out = nullptr;
    int dev = 0;
    if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) return TARAL_ERR_NO_DEVICE;
    auto* h = new taral_mlp;
    try {
        h->m.create(in_dim, hidden, depth, out_dim, max_batch);
    } catch (const MlpError& e) {
        delete h;
        return e.msg.find("cudaMalloc") != std::string::npos ? TARAL_ERR_ALLOC : TARAL_ERR_CUDA;
    }
    *out = h;
    return TARAL_OK;
}

extern "C" int64_t taral_mlp_param_count(const taral_mlp* h) { return h ? h->m.param_count() : 0; }

// Parameter layout: for each layer W (in x out, row-major) then b (out).
extern "C" int taral_mlp_set_params(taral_mlp* h, const float* params) {
    if (!h || !params) return TARAL_ERR_INPUT;
    MLP_GUARD(h, {
        Mlp& m = h->m;
        const float* p = params;
        for (auto& y : m.L) {
            size_t nw = size_t(y.in) * y.out;
            MK(cudaMemcpyAsync(y.W, p, nw * sizeof(float), cudaMemcpyHostToDevice, m.s));
            taral::mlp::k_to_bf16<<<taral::mlp::grid1(nw), 256, 0, m.s>>>(nw, y.W, y.Wb);
            p += nw;
            MK(cudaMemcpyAsync(y.b, p, y.out * sizeof(float), cudaMemcpyHostToDevice, m.s));
            p += y.out;
        }
        m.refresh_transposes();
        MK(cudaStreamSynchronize(m.s));
    })
}

extern "C" int taral_mlp_get_params(taral_mlp* h, float* params) {
    if (!h || !params) return TARAL_ERR_INPUT;
    MLP_GUARD(h, {
        Mlp& m = h->m;
        float* p = params;
        for (auto& y : m.L) {
            size_t nw = size_t(y.in) * y.out;
            MK(cudaMemcpyAsync(p, y.W, nw * sizeof(float), cudaMemcpyDeviceToHost, m.s));
            p += nw;
            MK(cudaMemcpyAsync(p, y.b, y.out * sizeof(float), cudaMemcpyDeviceToHost, m.s));
            p += y.out;
        }
        MK(cudaStreamSynchronize(m.s));
    })
}

extern "C" int taral_mlp_forward(taral_mlp* h, int batch, const float* x, float* y) {
    if (!h || !x || !y || batch <= 0 || batch > h->m.max_batch) return TARAL_ERR_INPUT;
    MLP_GUARD(h, {
        Mlp& m = h->m;
        m.load_input(batch, x);
        m.forward(batch);
        MK(cudaMemcpyAsync(y, m.L[m.depth].Z, size_t(batch) * m.out_dim * sizeof(float), cudaMemcpyDeviceToHost, m.s));
        MK(cudaStreamSynchronize(m.s));
        m.check_tc();
    })
}

extern "C" int taral_mlp_gradients(taral_mlp* h, int batch, const float* x, const float* target, double* loss,
                                   float* grads) {
    if (!h || !x || !target || batch <= 0 || batch > h->m.max_batch) return TARAL_ERR_INPUT;
    MLP_GUARD(h, {
        Mlp& m = h->m;
        m.load_input(batch, x);
        MK(cudaMemcpyAsync(m.Tf, target, size_t(batch) * m.out_dim * sizeof(float), cudaMemcpyHostToDevice, m.s));
        m.forward(batch);
        double l = m.backward(batch);
        m.check_tc();
        if (loss) *loss = l;
        if (grads) {
            float* p = grads;
            for (auto& y : m.L) {
                size_t nw = size_t(y.in) * y.out;
                MK(cudaMemcpyAsync(p, y.gW, nw * sizeof(float), cudaMemcpyDeviceToHost, m.s));
                p += nw;
                MK(cudaMemcpyAsync(p, y.gb, y.out * sizeof(float), cudaMemcpyDeviceToHost, m.s));
                p += y.out;
            }
            MK(cudaStreamSynchronize(m.s));
        }
    })
}

extern "C" int taral_mlp_set_dataset(taral_mlp* h, int count, const float* x, const float* target) {
    if (!h || count <= 0 || !x || !target) return TARAL_ERR_INPUT;
    MLP_GUARD(h, {
        Mlp& m = h->m;
        if (m.DX) throw MlpError{"dataset already set"};
        m.DX = m.alloc<float>(size_t(count) * m.in_dim), m.DT = m.alloc<float>(size_t(count) * m.out_dim);
        MK(cudaMemcpyAsync(m.DX, x, size_t(count) * m.in_dim * sizeof(float), cudaMemcpyHostToDevice, m.s));
        MK(cudaMemcpyAsync(m.DT, target, size_t(count) * m.out_dim * sizeof(float), cudaMemcpyHostToDevice, m.s));
        MK(cudaStreamSynchronize(m.s));
        m.dcount = count;
    })
}

// Adam over the dataset: `epochs` passes of shuffled mini-batches (the last partial batch is dropped).
extern "C" int taral_mlp_train(taral_mlp* h, int epochs, int batch, float lr, uint64_t seed, double* last_loss) {
    if (!h || epochs <= 0 || batch <= 0 || batch > h->m.max_batch || !h->m.DX || h->m.dcount < batch)
        return TARAL_ERR_INPUT;
    MLP_GUARD(h, {
        Mlp& m = h->m;
        std::mt19937_64 rng(seed);
        std::vector<int> perm(m.dcount);
        double loss = 0;
        for (int e = 0; e < epochs; ++e) {
            for (int i = 0; i < m.dcount; ++i) perm[i] = i;
            std::shuffle(perm.begin(), perm.end(), rng);
            for (int b0 = 0; b0 + batch <= m.dcount; b0 += batch) {
                MK(cudaMemcpyAsync(m.d_idx, perm.data() + b0, batch * sizeof(int), cudaMemcpyHostToDevice, m.s));
                taral::mlp::k_gather_rows<<<taral::mlp::grid1(size_t(batch) * m.in_dim), 256, 0, m.s>>>(
                    batch, m.in_dim, m.d_idx, m.DX, m.Xf, m.Xb);
                taral::mlp::k_gather_rows<<<taral::mlp::grid1(size_t(batch) * m.out_dim), 256, 0, m.s>>>(
                    batch, m.out_dim, m.d_idx, m.DT, m.Tf, nullptr);
                m.forward(batch);
                loss = m.backward(batch);
                m.adam(lr);
            }
        }
        m.check_tc();
        if (last_loss) *last_loss = loss;
    })
}

extern "C" const char* taral_mlp_last_error(const taral_mlp* h) { return h ? h->m.err.c_str() : "NULL mlp"; }
extern "C" void taral_mlp_destroy(taral_mlp* h) { delete h; }

// Standalone GEMM on device buffers (test hook): C[M][N] (f32) = op(A) op(B), bf16 operands, per the TA/TB rules
// of k_gemm; slices > 1 uses split-K through a caller-provided workspace of slices * M * N floats.
extern "C" int taral_gemm_bf16(int M, int N, int K, int ta, int tb, const void* A, const void* B, float* C,
                               int slices, float* workspace, void* stream) {
    using namespace taral::mlp;
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C || slices < 1 || (slices > 1 && !workspace)) return TARAL_ERR_INPUT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bool vec = M % 8 == 0 && N % 8 == 0 && K % 8 == 0 && reinterpret_cast<uintptr_t>(A) % 16 == 0 &&
               reinterpret_cast<uintptr_t>(B) % 16 == 0;
    int kslice = (K + slices - 1) / slices;
    kslice = (kslice + BK - 1) / BK * BK;
    slices = (K + kslice - 1) / kslice;
    float* dst = slices > 1 ? workspace : C;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, slices);
    const bf16* a = static_cast<const bf16*>(A);
    const bf16* b = static_cast<const bf16*>(B);
#define LAUNCH(TA_, TB_)                                                                       \
    if (vec) k_gemm<TA_, TB_, true><<<grid, 256, 0, s>>>(M, N, K, kslice, a, b, dst);          \
    else k_gemm<TA_, TB_, false><<<grid, 256, 0, s>>>(M, N, K, kslice, a, b, dst);
    if (!ta && !tb) { LAUNCH(false, false) }
    else if (ta && !tb) { LAUNCH(true, false) }
    else if (!ta && tb) { LAUNCH(false, true) }
    else { LAUNCH(true, true) }
#undef LAUNCH
    if (slices > 1) k_splitk_sum<<<grid1(size_t(M) * N), 256, 0, s>>>(size_t(M) * N, slices, workspace, C);
    return cudaGetLastError() == cudaSuccess ? TARAL_OK : TARAL_ERR_CUDA;
}
