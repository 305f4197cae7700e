// Ruiz (10 passes, inf-norm) and Pock-Chambolle (alpha = 1) scaling on the device (gpu/pdhg.cu:92-130), applied to
// the unscaled A and A^T together. Every value is produced by the same FP64 operations on the same operands as the
// reference's host scaling (gpu/pdhg.cu:92-130), so the scaled matrices, Dr and Dc are bit-identical to it:
//   * row / column maxima: a max is independent of the visiting order (the comparison keeps the current value when
//     the new one is not larger, as std::max does, so a NaN entry is never taken);
//   * square roots and divisions are IEEE round-to-nearest in CUDA double precision, and v / (r_i * c_j) has no
//     multiply-add to contract;
//   * the Pock-Chambolle sums run sequentially, one thread per row, in the host's order: row i of A in entry order,
//     and column j as row j of A^T, whose entries ascend in i like the host's row-major pass.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace taral {

// r[i] = max |val| over row i (a warp per row, lanes strided).
static __global__ void k_row_absmax(int rows, const int* __restrict__ ptr, const double* __restrict__ val,
                                    double* __restrict__ r) {
    const int lane = threadIdx.x & 31, w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = w0; i < rows; i += nw) {
        double mx = 0;
        for (int k = ptr[i] + lane; k < ptr[i + 1]; k += 32) {
            const double a = fabs(val[k]);
            mx = mx < a ? a : mx;
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, mx, off);
            mx = mx < o ? o : mx;
        }
        if (lane == 0) r[i] = mx;
    }
}

// r[i] = sum |val| over row i, sequentially in entry order (one thread per row).
static __global__ void k_row_abssum(int rows, const int* __restrict__ ptr, const double* __restrict__ val,
                                    double* __restrict__ r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) s += fabs(val[k]);
        r[i] = s;
    }
}

// v = v > 0 ? sqrt(v) : 1;  D /= v.
static __global__ void k_fold(int k, double* __restrict__ v, double* __restrict__ D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const double s = v[i] > 0 ? sqrt(v[i]) : 1.0;
        v[i] = s;
        D[i] /= s;
    }
}

// val[k] /= r[i] * c[idx[k]] over the rows i of one matrix (a warp per row).
static __global__ void k_scale_entries(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                                       double* __restrict__ val, const double* __restrict__ r,
                                       const double* __restrict__ c) {
    const int lane = threadIdx.x & 31, w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = w0; i < rows; i += nw) {
        const double ri = r[i];
        for (int k = ptr[i] + lane; k < ptr[i + 1]; k += 32) val[k] /= ri * c[idx[k]];
    }
}

static __global__ void k_fill(int k, double v, double* __restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) d[i] = v;
}

template <class T>
__global__ void k_narrow(int64_t k, const double* __restrict__ src, T* __restrict__ dst) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < k; i += int64_t(gridDim.x) * blockDim.x)
        dst[i] = T(src[i]);
}

// The scaling passes on device buffers: A (m rows) and AT (n rows) with double values, Dr (m) and Dc (n) outputs,
// rs (m) and cs (n) scratch. Asynchronous on `st`.
inline void scale_on_device(int m, int n, const int* a_ptr, const int* a_idx, double* a_val, const int* t_ptr,
                            const int* t_idx, double* t_val, double* Dr, double* Dc, double* rs, double* cs,
                            cudaStream_t st) {
    auto grid = [](int64_t threads) { return int(std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, 148 * 8))); };
    const int gm = grid(m), gn = grid(n), wm = grid(int64_t(m) * 32), wn = grid(int64_t(n) * 32);
    k_fill<<<gm, 256, 0, st>>>(m, 1.0, Dr);
    k_fill<<<gn, 256, 0, st>>>(n, 1.0, Dc);
    for (int pass = 0; pass <= 10; ++pass) {
        if (pass < 10) {  // Ruiz: inf-norms of rows and columns
            k_row_absmax<<<wm, 256, 0, st>>>(m, a_ptr, a_val, rs);
            k_row_absmax<<<wn, 256, 0, st>>>(n, t_ptr, t_val, cs);
        } else {          // Pock-Chambolle: 1-norms
            k_row_abssum<<<gm, 256, 0, st>>>(m, a_ptr, a_val, rs);
            k_row_abssum<<<gn, 256, 0, st>>>(n, t_ptr, t_val, cs);
        }
        k_fold<<<gm, 256, 0, st>>>(m, rs, Dr);
        k_fold<<<gn, 256, 0, st>>>(n, cs, Dc);
        k_scale_entries<<<wm, 256, 0, st>>>(m, a_ptr, a_idx, a_val, rs, cs);
        k_scale_entries<<<wn, 256, 0, st>>>(n, t_ptr, t_idx, t_val, cs, rs);
    }
}

}  // namespace taral
