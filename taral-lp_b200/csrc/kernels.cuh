// Device kernels of the B200 PDHG engine (sm_100a).
//
// One SpMV skeleton serves every matrix-vector product of the method: y = A x for the power iteration and the
// exact products, the dual step (row phase over A) and the primal step (column phase over A^T). The matrix is
// cut at set-up into ROW BLOCKS of consecutive rows holding at most kTile nonzeros and kRowsMax rows (a row
// longer than kTile forms a block of its own). One CTA per block:
//   1. stage  -- the block's val/idx range is read with 16-byte vector loads (scalar at the ragged ends), each
//                nonzero's product with the gathered vector entry is written to shared memory;
//   2. reduce -- rows are summed from shared memory by groups of G lanes (G = power of two >= the block's mean
//                row length, 1..32) with a shuffle tree, in FP64;
//   3. epilogue -- one thread per row applies the fused step (prox, projection, running sums) with its operands
//                loaded before stage 1, so their latency overlaps the matrix stream.
// The summation order depends only on the matrix, so results are bit-reproducible run to run.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace taral {

constexpr int kThreads = 256;  // threads per CTA in every SpMV-shaped kernel
constexpr int kTile = 2048;    // nonzeros staged per row block
constexpr int kRowsMax = 256;  // rows per row block (one epilogue row per thread)
constexpr int kRedThreads = 256;

template <class T>
__device__ __forceinline__ T clampv(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ------------------------------------------------------------------------------------------ vector loads
template <class T> struct Quad;
template <> struct Quad<float> {
    __device__ __forceinline__ static void load(const float* p, float (&v)[4]) {
        float4 q = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
    }
};
template <> struct Quad<double> {
    __device__ __forceinline__ static void load(const double* p, double (&v)[4]) {
        double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
    }
};
__device__ __forceinline__ void load_idx4(const int* p, int (&v)[4]) {
    int4 q = __ldg(reinterpret_cast<const int4*>(p));
    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
}

// Product type staged in shared memory: float products for a float matrix, double otherwise.
template <class T, class X> struct ProdT { using type = double; };
template <> struct ProdT<float, float> { using type = float; };

// ------------------------------------------------------------------------------------------ epilogues
// y[r] = s
template <class Y>
struct EpiStore {
    Y* y;
    struct Ops {};
    __device__ __forceinline__ Ops load(int) const { return {}; }
    __device__ __forceinline__ void apply(int r, double s, const Ops&) const { y[r] = Y(s); }
};

// Dual step of one row (gpu/pdhg.cu:178-190 semantics, running sum of z in FP64):
//   v = z + sigma (2 s - Ax_old);  z = prox: v - sigma*rl if v/sigma < rl, v - sigma*ru if v/sigma > ru, else 0;
//   Ax_old = s;  zs += z.
template <class T>
struct EpiRow {
    T *Ax, *z;
    double* zs;
    const T *rl, *ru, *par;
    struct Ops { T z, ax, rl, ru, sig; double zs; };
    __device__ __forceinline__ Ops load(int r) const { return {z[r], Ax[r], rl[r], ru[r], par[1], zs[r]}; }
    __device__ __forceinline__ void apply(int r, double s, const Ops& o) const {
        T st = T(s), sig = o.sig;
        T v = o.z + sig * (T(2) * st - o.ax), q = v / sig;
        T zn = q < o.rl ? v - sig * o.rl : (q > o.ru ? v - sig * o.ru : T(0));
        Ax[r] = st, z[r] = zn, zs[r] = o.zs + double(zn);
    }
};

// Column step (gpu/pdhg.cu:192-206 semantics): ATz = s; with upd, the next primal step
//   x = clamp(x - tau (c + s), l, u);  xs += x  (FP64 sum).
template <class T>
struct EpiCol {
    T *ATz, *x;
    double* xs;
    const T *c, *l, *u, *par;
    int upd;
    struct Ops { T x, c, l, u, tau; double xs; };
    __device__ __forceinline__ Ops load(int r) const {
        if (!upd) return {T(0), T(0), T(0), T(0), T(0), 0.0};
        return {x[r], c[r], l[r], u[r], par[0], xs[r]};
    }
    __device__ __forceinline__ void apply(int r, double s, const Ops& o) const {
        T st = T(s);
        ATz[r] = st;
        if (upd) {
            T xn = clampv(o.x - o.tau * (o.c + st), o.l, o.u);
            x[r] = xn, xs[r] = o.xs + double(xn);
        }
    }
};

// ------------------------------------------------------------------------------------------ SpMV skeleton
// blk[b] = first row of block b (blk[nblk] = rows). VEC: the val/idx base pointers are 16-byte aligned.
template <class T, class X, class E, bool VEC>
__global__ void __launch_bounds__(kThreads) k_rowblock(const int* __restrict__ ptr, const int* __restrict__ idx,
                                                         const T* __restrict__ val, const X* __restrict__ xin,
                                                         const int* __restrict__ blk, const int* __restrict__ skip,
                                                         E epi) {
    using P = typename ProdT<T, X>::type;
    __shared__ P prod[kTile];
    __shared__ double rowsum[kRowsMax];
    __shared__ int rptr[kRowsMax + 1];
    if (skip && *skip) return;
    const int b = blockIdx.x, tid = threadIdx.x;
    const int r0 = blk[b], r1 = blk[b + 1], nrows = r1 - r0;
    const int p0 = ptr[r0], p1 = ptr[r1], len = p1 - p0;

    typename E::Ops ops{};
    const bool mine = tid < nrows;
    if (mine) ops = epi.load(r0 + tid);

    if (len > kTile) {  // one long row: strided partial sums, fixed-order block reduction
        double s = 0;
        if (VEC) {
            const int a0 = p0 & ~3;
            for (int q = a0 + 4 * tid; q < p1; q += 4 * kThreads) {
                if (q >= p0 && q + 4 <= p1) {
                    T v[4]; int c[4];
                    Quad<T>::load(val + q, v), load_idx4(idx + q, c);
#pragma unroll
                    for (int e = 0; e < 4; ++e) s += double(v[e]) * double(__ldg(xin + c[e]));
                } else {
                    for (int e = 0; e < 4; ++e)
                        if (q + e >= p0 && q + e < p1) s += double(__ldg(val + q + e)) * double(__ldg(xin + __ldg(idx + q + e)));
                }
            }
        } else {
            for (int k = p0 + tid; k < p1; k += kThreads) s += double(__ldg(val + k)) * double(__ldg(xin + __ldg(idx + k)));
        }
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if ((tid & 31) == 0) rowsum[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) {
            double t = 0;
            for (int w = 0; w < kThreads / 32; ++w) t += rowsum[w];
            epi.apply(r0, t, ops);
        }
        return;
    }

    // 1. stage products
    for (int t = tid; t <= nrows; t += kThreads) rptr[t] = ptr[r0 + t] - p0;
    if (VEC) {
        const int a0 = p0 & ~3;
        for (int q = a0 + 4 * tid; q < p1; q += 4 * kThreads) {
            if (q >= p0 && q + 4 <= p1) {
                T v[4]; int c[4];
                Quad<T>::load(val + q, v), load_idx4(idx + q, c);
                X g[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) g[e] = __ldg(xin + c[e]);
#pragma unroll
                for (int e = 0; e < 4; ++e) prod[q - p0 + e] = P(v[e]) * P(g[e]);
            } else {
                for (int e = 0; e < 4; ++e) {
                    int k = q + e;
                    if (k >= p0 && k < p1) prod[k - p0] = P(__ldg(val + k)) * P(__ldg(xin + __ldg(idx + k)));
                }
            }
        }
    } else {
        for (int k = p0 + tid; k < p1; k += kThreads) prod[k - p0] = P(__ldg(val + k)) * P(__ldg(xin + __ldg(idx + k)));
    }
    __syncthreads();

    // 2. reduce rows with G-lane groups
    int mean = nrows > 0 ? (len + nrows - 1) / nrows : 1;
    int G = 1;
    while (G < 32 && G < mean) G <<= 1;
    const int lane = tid & (G - 1), grp = tid / G, ngrp = kThreads / G;
    for (int base = 0; base < nrows; base += ngrp) {  // CTA-uniform trip count: every lane reaches the shuffles
        const int t = base + grp;
        double s = 0;
        if (t < nrows)
            for (int k = rptr[t] + lane; k < rptr[t + 1]; k += G) s += double(prod[k]);
        for (int off = G >> 1; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off, G);
        if (t < nrows && lane == 0) rowsum[t] = s;
    }
    __syncthreads();

    // 3. epilogue
    if (mine) epi.apply(r0 + tid, rowsum[tid], ops);
}

// First primal step of a block (gpu/pdhg.cu:208-214): x = clamp(x - tau (c + ATz), l, u), xs += x.
template <class T>
__global__ void k_xupd(int n, T* __restrict__ x, const T* __restrict__ ATz, const T* __restrict__ c,
                       const T* __restrict__ l, const T* __restrict__ u, const T* __restrict__ par,
                       double* __restrict__ xs) {
    const T tau = par[0];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        T xn = clampv(x[j] - tau * (c[j] + ATz[j]), l[j], u[j]);
        x[j] = xn, xs[j] += double(xn);
    }
}

// ------------------------------------------------------------------------------------------ reductions
// Sum K doubles over the CTA; the last CTA to finish (ticket) adds the per-CTA partials in CTA order.
// Deterministic for a fixed grid size; no CTA waits on another.
template <int K>
__device__ __forceinline__ void reduce_finish(double (&v)[K], double* part, unsigned* ticket, double* out) {
    __shared__ double sh[K][kRedThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = v[k];
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) sh[k][w] = s;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[threadIdx.x][i];
        part[blockIdx.x * K + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) {
        __threadfence();
        if (threadIdx.x < K) {
            double s = 0;
            for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(part + b * K + threadIdx.x);
            out[threadIdx.x] = s;
        }
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// Weight of row i in the per-row relative residual (gpu/pdhg.cu:138-144).
__device__ __forceinline__ double row_rel_weight(double lo, double up, double dr) {
    double b = 0;
    if (lo > -INFINITY) b = lo < 0 ? -lo : lo;
    if (up < INFINITY) { double a = up < 0 ? -up : up; b = a > b ? a : b; }
    return 1.0 / (1.0 + b / dr);
}

// Row part of the KKT evaluation (gpu/pdhg.cu:236-251): out = {PR2S, PR2O, PR2R, DROW, DZ2}.
template <class T, class V>
__global__ void __launch_bounds__(kRedThreads) k_eval_row(int m, double f, const V* __restrict__ Ax,
                                                          const V* __restrict__ z, const T* __restrict__ rl,
                                                          const T* __restrict__ ru, const T* __restrict__ Dr,
                                                          const T* __restrict__ zlast, double* part,
                                                          unsigned* ticket, double* out) {
    double v[5] = {0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double ax = double(Ax[i]) * f, zz = double(z[i]) * f, lo = rl[i], up = ru[i];
        double r = ax < lo ? lo - ax : (ax > up ? ax - up : 0), ro = r / double(Dr[i]);
        double rr = ro * row_rel_weight(lo, up, double(Dr[i]));
        v[0] += r * r, v[1] += ro * ro, v[2] += rr * rr;
        if (zz > 0 && up < INFINITY) v[3] -= zz * up;
        if (zz < 0 && lo > -INFINITY) v[3] -= zz * lo;
        double dz = zz - double(zlast[i]);
        v[4] += dz * dz;
    }
    reduce_finish<5>(v, part, ticket, out);
}

// Column part (gpu/pdhg.cu:253-271): out = {DR2S, DR2O, POBJ, DCOL, DX2}.
template <class T, class V>
__global__ void __launch_bounds__(kRedThreads) k_eval_col(int n, double f, const V* __restrict__ x,
                                                          const V* __restrict__ ATz, const T* __restrict__ c,
                                                          const T* __restrict__ l, const T* __restrict__ u,
                                                          const T* __restrict__ Dc, const T* __restrict__ xlast,
                                                          double* part, unsigned* ticket, double* out) {
    double v[5] = {0, 0, 0, 0, 0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double xx = double(x[j]) * f, cj = c[j], d = cj + double(ATz[j]) * f, lo = l[j], up = u[j], res = 0;
        v[2] += cj * xx;
        if (d > 0) {
            if (lo > -INFINITY) v[3] += d * lo;
            else res = d;
        } else if (d < 0) {
            if (up < INFINITY) v[3] += d * up;
            else res = -d;
        }
        double ro = res / double(Dc[j]), dx = xx - double(xlast[j]);
        v[0] += res * res, v[1] += ro * ro, v[4] += dx * dx;
    }
    reduce_finish<5>(v, part, ticket, out);
}

// Power iteration on A_s^T A_s with the stop test on the device (gpu/pdhg.cu:425-434). st = {est, prev, scale};
// *done is set once the estimate has converged (after step 10, |est - prev| <= 1e-7 est) or when ||v||^2 <= 0,
// and every later kernel of the queued steps returns at once.
template <class T>
__global__ void __launch_bounds__(kRedThreads) k_power_sumsq(int n, const T* __restrict__ v, double* part,
                                                             unsigned* ticket, double* out, const int* done) {
    if (*done) return;
    double a[1] = {0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) a[0] += double(v[j]) * double(v[j]);
    reduce_finish<1>(a, part, ticket, out);
}

__global__ void k_power_update(const double* out, double* st, int* done, int it) {  // one thread
    if (*done) return;
    double s = out[0], prev = st[0];
    if (s <= 0) { st[0] = 0, *done = 1; return; }
    double est = sqrt(sqrt(s));
    st[0] = est, st[1] = prev, st[2] = 1 / sqrt(s);
    if (it >= 10 && fabs(est - prev) <= 1e-7 * est) *done = 2;
}

template <class T>
__global__ void k_power_scale(int n, T* __restrict__ v, const double* __restrict__ st, const int* done) {
    if (*done) return;
    double f = st[2];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) v[j] = T(double(v[j]) * f);
}

template <class T>
__global__ void k_set_par(T* par, T tau, T sigma) { par[0] = tau, par[1] = sigma; }

// Default start (gpu/pdhg.cu:450-455): x = x_last = clamp(0, l, u), sum <- 0.
template <class T>
__global__ void k_start_x(int n, const T* __restrict__ l, const T* __restrict__ u, T* __restrict__ x,
                          T* __restrict__ xlast, double* __restrict__ xs) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        T lo = l[j], v = T(0) < lo ? lo : T(0), up = u[j];
        v = up < v ? up : v;
        x[j] = v, xlast[j] = v, xs[j] = 0;
    }
}

template <class T>
__global__ void k_zero_point(int m, T* __restrict__ z, T* __restrict__ zlast, double* __restrict__ zs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) z[i] = 0, zlast[i] = 0, zs[i] = 0;
}

// Restart (gpu/pdhg.cu:293-299): point <- average*f (avg) or current; last point <- point; sum <- 0.
template <class T>
__global__ void k_restart(int n, int avg, double f, T* __restrict__ x, double* __restrict__ xs,
                          T* __restrict__ xlast) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        T v = avg ? T(xs[j] * f) : x[j];
        x[j] = v, xlast[j] = v, xs[j] = 0;
    }
}

// Start: point and last point from a host-supplied FP64 vector (already on the device), sum <- 0.
template <class T>
__global__ void k_set_point(int n, const double* __restrict__ src, T* __restrict__ x, T* __restrict__ xlast,
                            double* __restrict__ xs) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        T v = T(src[j]);
        x[j] = v, xlast[j] = v, xs[j] = 0;
    }
}

// Download (gpu/pdhg.cu:301-304): dst = src * f in FP64.
template <class V>
__global__ void k_scale_out(int n, double f, const V* __restrict__ src, double* __restrict__ dst) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) dst[j] = double(src[j]) * f;
}

template <class T>
__global__ void k_cast(int n, const double* __restrict__ src, T* __restrict__ dst) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) dst[j] = T(src[j]);
}

}  // namespace taral
