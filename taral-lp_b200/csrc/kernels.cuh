// Device kernels of the B200 PDHG engine (sm_100a).
//
// One SpMV skeleton serves every matrix-vector product of the method: y = A x for the power iteration and the
// exact products, the dual step (row phase over A) and the primal step (column phase over A^T). The matrix is
// cut at set-up into ROW BLOCKS of consecutive rows holding at most kTile nonzeros and kRowsMax rows (a row
// longer than kTile forms a block of its own). One CTA per block:
//   1. stage  -- the block's val/idx range is read with 16-byte vector loads (scalar at the ragged ends), each
//                nonzero's product with the gathered vector entry is written to shared memory;
//   2. reduce -- rows are summed from shared memory in FP64: a row of at most kShort nonzeros by its own thread
//                in entry order, a longer row by a warp (lanes strided, shuffle tree); the autotuner's row-split
//                policies (block flags below) change this per block;
//   3. epilogue -- one thread per row applies the fused step (prox, projection, running sums) with its operands
//                copied asynchronously into shared memory before stage 1, so their latency overlaps the matrix
//                stream without holding registers across it.
// The summation order depends only on the matrix, so results are bit-reproducible run to run.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace taral {

constexpr int kThreads = 256;  // threads per CTA in every SpMV-shaped kernel
constexpr int kTile = 2044;    // nonzeros staged per row block: with the 16-byte alignment slack, 512 quads
constexpr int kRowsMax = 256;  // rows per row block (one epilogue row per thread)
constexpr int kRedThreads = 256;
// Resident CTAs per SM the row-block kernels are compiled for, by product type: 8 (32 registers) with float
// products; 5 (48 registers) with double products, whose staging registers would otherwise spill to local memory
// (measured on the bench LP's row phase in FP64: 55.7 us at 8 CTAs with spills, 40.2 us at 5 without).
template <class P> constexpr int kMinBlocks = 5;
template <> constexpr int kMinBlocks<float> = 8;

template <class T>
__device__ __forceinline__ T clampv(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ------------------------------------------------------------------------------------------ vector loads
template <class T> struct Quad;
// The matrix is streamed once per phase: its 16-byte loads bypass L1 (no_allocate) so that L1 keeps the gathered
// vector entries, which are reused across rows.
template <> struct Quad<float> {
    __device__ __forceinline__ static void load(const float* p, float (&v)[4]) {
        asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
                     : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(p));
    }
};
template <> struct Quad<double> {
    __device__ __forceinline__ static void load(const double* p, double (&v)[4]) {
        asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
        asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];" : "=d"(v[2]), "=d"(v[3]) : "l"(p + 2));
    }
};
__device__ __forceinline__ void load_idx4(const int* p, int (&v)[4]) {
    asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "l"(p));
}

// Gathered vector entries are reused across rows and blocks: keep them in L1 as long as possible.
__device__ __forceinline__ float gather(const float* p) {
    float v;
    asm volatile("ld.global.nc.L1::evict_last.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double gather(const double* p) {
    double v;
    asm volatile("ld.global.nc.L1::evict_last.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

// Programmatic dependent launch (sm_90+, opt-in with TARAL_PDL=1): a phase kernel waits for its predecessor grid to
// complete, with its memory visible, before touching anything the predecessor may write, and only then lets its own
// successor launch (pdl_acquire). Releasing the successor only after the wait keeps the chain ordered: when a kernel
// starts early, its predecessor has passed its own wait, so every kernel before that one has completed, and what the
// early part reads -- its constant matrix stream and the vectors only its own phase writes -- is final. Without the
// launch attribute (a plain launch) the wait returns at once and the release has no effect.
__device__ __forceinline__ void pdl_acquire() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Products rounded on their own (never fused into a following add), as the staged paths round them.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Product type staged in shared memory: float products for a float matrix, double otherwise.
template <class T, class X> struct ProdT { using type = double; };
template <> struct ProdT<float, float> { using type = float; };

// ------------------------------------------------------------------------------------------ async copies
// Global -> shared copies of one 4- or 8-byte element (cp.async): while in flight they hold no registers, so the
// row-block kernels fetch a row's epilogue operands before the matrix stream without keeping them in registers
// across it (at the 32 registers of 8 CTAs per SM, operands held in registers spill to local memory).
__device__ __forceinline__ void copy_async(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;"
                 :: "r"(unsigned(__cvta_generic_to_shared(dst))), "l"(src) : "memory");
}
__device__ __forceinline__ void copy_async(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;"
                 :: "r"(unsigned(__cvta_generic_to_shared(dst))), "l"(src) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ------------------------------------------------------------------------------------------ epilogues
// Two forms of the same step:
//   load(r, inst) -> Ops, apply(r, s, ops): the operands of row r in registers (the thread-per-row kernels);
//   stage(r, t, st), finish(r, inst, t, s, st): the operands copied asynchronously into slot t of a shared-memory
//     Stage before the matrix stream and consumed after the sums (the row-block kernels; t < kRowsMax).
// inst = the row's instance in a batch, 0 otherwise; step sizes par[2 inst] = tau, par[2 inst + 1] = sigma.
// y[r] = s
template <class Y>
struct EpiStore {
    Y* y;
    struct Ops {};
    struct Stage {};
    __device__ __forceinline__ Ops load(int, int) const { return {}; }
    __device__ __forceinline__ void apply(int r, double s, const Ops&) const { y[r] = Y(s); }
    __device__ __forceinline__ void stage(int, int, Stage&) const {}
    __device__ __forceinline__ void finish(int r, int, int, double s, Stage&) const { y[r] = Y(s); }
};

// Dual step of one row (gpu/pdhg.cu:178-190 semantics, running sum of z in FP64):
//   v = z + sigma (2 s - Ax_old);  z = prox: v - sigma*rl if v/sigma < rl, v - sigma*ru if v/sigma > ru, else 0;
//   Ax_old = s;  zs += z.
// The arithmetic is FP64 whatever T is: with a small sigma, v - sigma*rl cancels, and in float that
// cancellation stalls the method (the reference's --fp32 failure); only the stored values are rounded to T.
template <class T>
struct EpiRow {
    T *Ax, *z;
    double* zs;
    const T *rl, *ru;
    const double* par;
    struct Ops { double z, ax, rl, ru, sig, zs; };
    struct Stage { double zs[kRowsMax]; T z[kRowsMax], ax[kRowsMax], rl[kRowsMax], ru[kRowsMax]; };
    __device__ __forceinline__ void step(int r, double s, double z0, double ax, double lo, double hi, double sig,
                                         double zs0) const {
        const T st = T(s);
        const double v = z0 + sig * (2.0 * double(st) - ax), q = v / sig;
        const T zn = T(q < lo ? v - sig * lo : (q > hi ? v - sig * hi : 0.0));
        Ax[r] = st, z[r] = zn, zs[r] = zs0 + double(zn);
    }
    __device__ __forceinline__ Ops load(int r, int inst) const {
        return {double(z[r]), double(Ax[r]), double(rl[r]), double(ru[r]), par[2 * inst + 1], zs[r]};
    }
    __device__ __forceinline__ void apply(int r, double s, const Ops& o) const {
        step(r, s, o.z, o.ax, o.rl, o.ru, o.sig, o.zs);
    }
    __device__ __forceinline__ void stage(int r, int t, Stage& st) const {
        copy_async(&st.z[t], z + r), copy_async(&st.ax[t], Ax + r), copy_async(&st.rl[t], rl + r);
        copy_async(&st.ru[t], ru + r), copy_async(&st.zs[t], zs + r);
        copy_async_commit();
    }
    __device__ __forceinline__ void finish(int r, int inst, int t, double s, Stage& st) const {
        copy_async_wait();
        step(r, s, double(st.z[t]), double(st.ax[t]), double(st.rl[t]), double(st.ru[t]), par[2 * inst + 1],
             st.zs[t]);
    }
};

// Column step (gpu/pdhg.cu:192-206 semantics): ATz = s; with upd, the next primal step
//   x = clamp(x - tau (c + s), l, u);  xs += x  (FP64 arithmetic and sum, T storage).
template <class T>
struct EpiCol {
    T *ATz, *x;
    double* xs;
    const T *c, *l, *u;
    const double* par;
    int upd;
    struct Ops { double x, c, l, u, tau, xs; };
    struct Stage { double xs[kRowsMax]; T x[kRowsMax], c[kRowsMax], l[kRowsMax], u[kRowsMax]; };
    __device__ __forceinline__ void step(int r, double s, double x0, double c0, double lo, double hi, double tau,
                                         double xs0) const {
        const T st = T(s);
        ATz[r] = st;
        if (upd) {
            const T xn = T(clampv(x0 - tau * (c0 + double(st)), lo, hi));
            x[r] = xn, xs[r] = xs0 + double(xn);
        }
    }
    __device__ __forceinline__ Ops load(int r, int inst) const {
        if (!upd) return {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        return {double(x[r]), double(c[r]), double(l[r]), double(u[r]), par[2 * inst], xs[r]};
    }
    __device__ __forceinline__ void apply(int r, double s, const Ops& o) const {
        step(r, s, o.x, o.c, o.l, o.u, o.tau, o.xs);
    }
    __device__ __forceinline__ void stage(int r, int t, Stage& st) const {
        if (!upd) return;
        copy_async(&st.x[t], x + r), copy_async(&st.c[t], c + r), copy_async(&st.l[t], l + r);
        copy_async(&st.u[t], u + r), copy_async(&st.xs[t], xs + r);
        copy_async_commit();
    }
    __device__ __forceinline__ void finish(int r, int inst, int t, double s, Stage& st) const {
        if (!upd) {
            ATz[r] = T(s);
            return;
        }
        copy_async_wait();
        step(r, s, double(st.x[t]), double(st.c[t]), double(st.l[t]), double(st.u[t]), par[2 * inst], st.xs[t]);
    }
};

// ------------------------------------------------------------------------------------------ SpMV skeleton
// Row-block metadata, one int4 per block, built on the host (build_row_blocks): x = first row, y = number of rows,
// z = first nonzero, w = end of the nonzeros. VEC: the val/idx base pointers are 16-byte aligned.
constexpr int kShort = 48;                       // rows up to this length are summed by their own thread
// Block flags in the high bits of the metadata's row count (the row count itself is the low 16 bits):
// kUniformRows -- every row of the block, however long, is summed by its own thread in entry order (the warp path
//                 only pays off when a few long rows would otherwise hold up a warp of short ones). Set by the
//                 autotuner (Engine::tune, Batch::tune) on kUniformCandidate blocks when that is measurably faster.
// kUniformCandidate -- the block's rows have similar lengths (longest <= 2 x mean + 8) and some row exceeds kShort.
constexpr int kUniformRows = 1 << 16;
constexpr int kUniformCandidate = 1 << 17;
// kSegmented -- balanced reduction: each thread sums kSeg consecutive products and rows crossing threads are joined
//               by a segmented scan over the CTA (summation order fixed by the block's structure). Set by the
//               autotuner on FP32 matrices when it is measurably faster.
constexpr int kSegmented = 1 << 18;
constexpr int kSeg = 8;
// kMidGroups -- rows of kShort + 1 .. kMid nonzeros are summed by groups of kGroup lanes (four rows per warp, lanes
//               strided by kGroup, a three-level shuffle tree) instead of a whole warp each. Set by the autotuner.
constexpr int kMidGroups = 1 << 19;
constexpr int kMid = 128;
constexpr int kGroup = 8;
constexpr int kPolicies = 5;  // row-split policies the autotuners choose from (0 = the hybrid rule)
static_assert(kSeg * kThreads >= kTile, "kSeg products per thread must cover a block");
constexpr int kQuads = (kTile + 3 + 3) / 4 / kThreads;  // 16-byte quads per thread in the staging loop (2)
static_assert(kQuads * 4 * kThreads >= kTile + 3, "a block's quads must fit the staging loop");
__device__ __forceinline__ int pidx(int k) { return k + (k >> 5); }  // one pad slot per 32: no bank conflicts
// 16-byte shared-memory accesses of 4 / 8 consecutive products (16-byte aligned addresses)
__device__ __forceinline__ void store4(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double* p, const double (&v)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void load8(const float* p, float (&v)[8]) {
    const float4 a = reinterpret_cast<const float4*>(p)[0], b = reinterpret_cast<const float4*>(p)[1];
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
}
__device__ __forceinline__ void load8(const double* p, double (&v)[8]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double2 a = reinterpret_cast<const double2*>(p)[i];
        v[2 * i] = a.x, v[2 * i + 1] = a.y;
    }
}

template <class P>
struct RowSmem {
    alignas(16) P prod[kTile + kTile / 32];  // hybrid: product k at pidx(k - p0); segmented: at k - (p0 & ~3)
    double rowsum[kRowsMax];
    int rptr[kRowsMax + 1];
    short longrow[kRowsMax];
    short midrow[kRowsMax];
    int nlong, nmid;
    double segv[kThreads / 32];  // segmented scan: per-warp carry value and flag
    int segf[kThreads / 32];
};

// Balanced row sums (kSegmented blocks) of the staged products sm.prod[pidx(0 .. len)], rows delimited by
// sm.rptr[0 .. nrows]: thread t sums products [kSeg t, kSeg t + kSeg) in order. A row that starts and ends inside the
// thread is written at once; the partial of a row that continues past the thread (its tail) is carried by a
// segmented inclusive scan over the CTA (combine(a, b) = b started a row ? b : a + b), and the thread in which a
// continued row ends adds the carried partial to its own head part. Ends with a barrier.
template <class P>
__device__ __forceinline__ void segmented_sums(RowSmem<P>& sm, int nrows) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int begin = sm.rptr[0], len = sm.rptr[nrows];  // entries [begin, len) of the unpadded product array
    const int k0 = max(kSeg * tid, begin), k1 = min(kSeg * tid + kSeg, len);
    double tail = 0, head = 0;
    int head_row = -1, tail_starts = 1;  // tail_starts: the open segment (if any) began inside this thread
    P pv[kSeg];
    if (kSeg * tid < len) load8(&sm.prod[kSeg * tid], pv);  // this thread's 8 products, two 16-byte loads
    if (k0 < k1) {
        int lo = 0, hi = nrows - 1;  // the last row r with rptr[r] <= k0 (non-empty, since k0 < len)
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sm.rptr[mid] <= k0) lo = mid;
            else hi = mid - 1;
        }
        int r = lo;
        bool cont = sm.rptr[r] < k0, first = true, open = false;
        double acc = 0;
        for (int k = k0; k < k1; ++k) {
            acc += double(pv[k - kSeg * tid]);
            open = true;
            if (k + 1 == sm.rptr[r + 1]) {  // row r ends at k
                if (first && cont) head = acc, head_row = r;
                else sm.rowsum[r] = acc;
                acc = 0, first = false, cont = false, open = false;
                if (k + 1 < len)
                    for (++r; sm.rptr[r + 1] == sm.rptr[r]; ++r) {}  // skip rows without entries
            }
        }
        if (open) tail = acc, tail_starts = (first && cont) ? 0 : 1;  // a pure continuation carries on
    }
    // segmented inclusive scan of (tail, tail_starts) over the threads
    double v = tail;
    int f = tail_starts;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double pv = __shfl_up_sync(0xffffffffu, v, off);
        const int pf = __shfl_up_sync(0xffffffffu, f, off);
        if (lane >= off) {
            if (!f) v = pv + v;
            f |= pf;
        }
    }
    if (lane == 31) sm.segv[warp] = v, sm.segf[warp] = f;
    __syncthreads();
    double cv = 0;  // carry from the warps before this one
    for (int w = 0; w < warp; ++w) cv = sm.segf[w] ? sm.segv[w] : cv + sm.segv[w];
    const double incl = f ? v : cv + v;
    double before = __shfl_up_sync(0xffffffffu, incl, 1);  // the scan value of the previous thread
    if (lane == 0) before = cv;
    if (head_row >= 0) sm.rowsum[head_row] = before + head;
    __syncthreads();
}

// Sums of the block's rows into sm.rowsum[0, nrows) (a long row: sm.rowsum[0]). Ends with a barrier.
//   1. stage: each thread issues all of its 16-byte val / idx loads (up to kQuads quads), then all of its gathers
//      of the vector entries, then writes the products to shared memory;
//   2. reduce: a row of at most kShort nonzeros is summed sequentially by its own thread; longer rows are queued
//      and each is summed by one warp (lanes strided, shuffle tree). Every row's summation order is fixed.
template <class T, class X, bool VEC, class P>
__device__ __forceinline__ void block_sums(const int* __restrict__ ptr, const int* __restrict__ idx,
                                           const T* __restrict__ val, const X* __restrict__ xin, int4 meta,
                                           RowSmem<P>& sm) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = meta.x, nrows = meta.y & 0xffff, p0 = meta.z, p1 = meta.w, len = p1 - p0;
    if (len > kTile) {  // one long row: strided partial sums, fixed-order block reduction
        pdl_acquire();
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
        if (lane == 0) sm.rowsum[1 + warp] = s;
        __syncthreads();
        if (tid == 0) {
            double t = 0;
            for (int w = 0; w < kThreads / 32; ++w) t += sm.rowsum[1 + w];
            sm.rowsum[0] = t;
        }
        __syncthreads();
        return;
    }

    // 1. stage products (segmented blocks: unpadded, quad-aligned from a0 = p0 & ~3, for 16-byte accesses)
    const bool seg = (meta.y & kSegmented) != 0;
    const int base = seg ? (p0 & ~3) : p0;
    for (int t = tid; t <= nrows; t += kThreads) sm.rptr[t] = ptr[r0 + t] - base;
    if (tid == 0) sm.nlong = 0, sm.nmid = 0;
    if (seg)  // rows without entries stay zero; every other row is written once, after the barrier
        for (int t = tid; t < nrows; t += kThreads) sm.rowsum[t] = 0;
    if (VEC) {
        const int a0 = p0 & ~3;
        T v[kQuads][4];
        int c[kQuads][4];
#pragma unroll
        for (int i = 0; i < kQuads; ++i) {
            const int q = a0 + 4 * (tid + i * kThreads);
            if (q >= p0 && q + 4 <= p1) {
                Quad<T>::load(val + q, v[i]), load_idx4(idx + q, c[i]);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const bool in = q + e >= p0 && q + e < p1;
                    v[i][e] = in ? __ldg(val + q + e) : T(0);
                    c[i][e] = in ? __ldg(idx + q + e) : -1;
                }
            }
        }
        pdl_acquire();  // the matrix stream above is constant; the gathered vector is the predecessor's output
        X g[kQuads][4];
#pragma unroll
        for (int i = 0; i < kQuads; ++i)
#pragma unroll
            for (int e = 0; e < 4; ++e) g[i][e] = c[i][e] >= 0 ? gather(xin + c[i][e]) : X(0);
        if (seg) {
#pragma unroll
            for (int i = 0; i < kQuads; ++i) {
                const int q = a0 + 4 * (tid + i * kThreads);
                if (q < p1) {
                    P pq[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) pq[e] = c[i][e] >= 0 ? P(P(v[i][e]) * P(g[i][e])) : P(0);
                    store4(&sm.prod[q - a0], pq);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < kQuads; ++i) {
                const int q = a0 + 4 * (tid + i * kThreads);
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (c[i][e] >= 0) sm.prod[pidx(q + e - p0)] = P(v[i][e]) * P(g[i][e]);
            }
        }
    } else {
        pdl_acquire();
        for (int k = p0 + tid; k < p1; k += kThreads)
            sm.prod[seg ? k - base : pidx(k - p0)] = P(__ldg(val + k)) * P(__ldg(xin + __ldg(idx + k)));
    }
    __syncthreads();

    if (seg) {
        segmented_sums(sm, nrows);
        return;
    }
    // 2. reduce: short rows (every row of a uniform block) by their own thread, long rows by a warp each (with
    //    kMidGroups: rows up to kMid nonzeros by kGroup lanes each)
    const int thread_max = (meta.y & kUniformRows) ? kTile : kShort;
    const int mid_max = (meta.y & kMidGroups) ? kMid : thread_max;
    if (tid < nrows) {
        const int a = sm.rptr[tid], b = sm.rptr[tid + 1];
        if (b - a <= thread_max) {
            double s = 0;
            int k = a;
            for (; k + 4 <= b; k += 4) {  // four loads in flight, then the adds in entry order
                P t[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) t[e] = sm.prod[pidx(k + e)];
#pragma unroll
                for (int e = 0; e < 4; ++e) s += double(t[e]);
            }
            for (; k < b; ++k) s += double(sm.prod[pidx(k)]);
            sm.rowsum[tid] = s;
        } else if (b - a <= mid_max) {
            sm.midrow[atomicAdd(&sm.nmid, 1)] = short(tid);
        } else {
            sm.longrow[atomicAdd(&sm.nlong, 1)] = short(tid);
        }
    }
    __syncthreads();
    {  // rows of the mid list: group g of a warp takes list entry base + g; warp-uniform trip count
        const int grp = lane / kGroup, gl = lane % kGroup;
        for (int base = warp * (32 / kGroup); base < sm.nmid; base += kThreads / kGroup) {
            const int i = base + grp;
            double s = 0;
            if (i < sm.nmid) {
                const int t = sm.midrow[i];
                for (int k = sm.rptr[t] + gl; k < sm.rptr[t + 1]; k += kGroup) s += double(sm.prod[pidx(k)]);
            }
#pragma unroll
            for (int off = kGroup / 2; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (i < sm.nmid && gl == 0) sm.rowsum[sm.midrow[i]] = s;
        }
    }
    for (int i = warp; i < sm.nlong; i += kThreads / 32) {  // warp-uniform trip count: all lanes shuffle
        const int t = sm.longrow[i];
        double s = 0;
        for (int k = sm.rptr[t] + lane; k < sm.rptr[t + 1]; k += 32) s += double(sm.prod[pidx(k)]);
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) sm.rowsum[t] = s;
    }
    __syncthreads();
}

// One launch over all row blocks of one matrix; `skip` (may be NULL): return at once when *skip != 0.
template <class T, class X, class E, bool VEC>
__global__ void __launch_bounds__(kThreads, kMinBlocks<typename ProdT<T, X>::type>) k_rowblock(const int* __restrict__ ptr, const int* __restrict__ idx,
                                                         const T* __restrict__ val, const X* __restrict__ xin,
                                                         const int4* __restrict__ blk, const int* __restrict__ skip,
                                                         E epi) {
    using P = typename ProdT<T, X>::type;
    __shared__ RowSmem<P> sm;
    __shared__ typename E::Stage st;
    if (skip) {  // a flag the predecessor may set
        pdl_acquire();
        if (*skip) return;
    }
    const int tid = threadIdx.x;
    const int4 meta = __ldg(blk + blockIdx.x);
    const int r0 = meta.x, nrows = meta.y & 0xffff;
    const bool mine = tid < nrows;
    if (mine) epi.stage(r0 + tid, tid, st);  // this phase's own vectors: the other phase does not write them
    block_sums<T, X, VEC>(ptr, idx, val, xin, meta, sm);
    if (mine) epi.finish(r0 + tid, 0, tid, sm.rowsum[tid], st);
}

// One thread per row, its products summed in entry order: for a matrix whose rows all hold at most kShort nonzeros
// this is exactly block_sums' thread-per-row arithmetic (each product rounded to the product type, FP64 sums in
// entry order), so the results are bit-identical; it skips the staging, the metadata and the block barriers, which
// pays for very short rows (Engine::tune times both). `skip` as in k_rowblock.
template <class T, class X, class E>
__global__ void __launch_bounds__(kThreads) k_rowthread(int rows, const int* __restrict__ ptr,
                                                        const int* __restrict__ idx, const T* __restrict__ val,
                                                        const X* __restrict__ xin, const int* __restrict__ skip,
                                                        E epi) {
    using P = typename ProdT<T, X>::type;
    if (skip) {
        pdl_acquire();
        if (*skip) return;
    }
    const int r = blockIdx.x * kThreads + threadIdx.x;
    if (r >= rows) return;
    const typename E::Ops ops = epi.load(r, 0);
    const int a = __ldg(ptr + r), b = __ldg(ptr + r + 1);
    pdl_acquire();
    double s = 0;
    for (int k = a; k < b; ++k) s += double(mul_rn(P(__ldg(val + k)), P(gather(xin + __ldg(idx + k)))));
    epi.apply(r, s, ops);
}

// Batched form: a block list over many instances (block-diagonal batch). ext[b] = {instance, row shift, gather
// offset, 0}: the block's rows r of the (possibly shared) matrix are rows r + shift of the concatenated instance
// vectors, and its column indices address xin + offset. Blocks of instances with active[instance] == 0 return.
template <class T, class X, class E, bool VEC>
__global__ void __launch_bounds__(kThreads, kMinBlocks<typename ProdT<T, X>::type>) k_rowblock_batch(const int* __restrict__ ptr, const int* __restrict__ idx,
                                                               const T* __restrict__ val, const X* __restrict__ xin,
                                                               const int4* __restrict__ blk,
                                                               const int4* __restrict__ ext,
                                                               const int* __restrict__ active, E epi) {
    using P = typename ProdT<T, X>::type;
    __shared__ RowSmem<P> sm;
    __shared__ typename E::Stage st;
    const int4 e4 = __ldg(ext + blockIdx.x);
    if (!active[e4.x]) return;  // the running flags change only between blocks (decision kernel), never in a phase
    const int tid = threadIdx.x;
    const int4 meta = __ldg(blk + blockIdx.x);
    const int r0 = meta.x + e4.y, nrows = meta.y & 0xffff;
    const bool mine = tid < nrows;
    if (mine) epi.stage(r0 + tid, tid, st);
    block_sums<T, X, VEC>(ptr, idx, val, xin + e4.z, meta, sm);
    if (mine) epi.finish(r0 + tid, e4.x, tid, sm.rowsum[tid], st);
}

// Batched thread-per-row form: one warp per entry of a row-chunk list, chunk[e] = {first row in the concatenated
// row pointers, rows (at most 32), -, -} of one instance, ext[e] = {instance, row shift, gather offset, 0} as for
// k_rowblock_batch; lane t takes the chunk's row t. Bit-identical to k_rowblock_batch under policy 0 when every row
// of the matrix holds at most kShort nonzeros, for the reasons given at k_rowthread.
constexpr int kChunk = 32;  // rows per chunk: one warp
template <class T, class X, class E>
__global__ void __launch_bounds__(kThreads) k_rowthread_batch(int n, const int* __restrict__ ptr,
                                                              const int* __restrict__ idx, const T* __restrict__ val,
                                                              const X* __restrict__ xin,
                                                              const int4* __restrict__ chunk,
                                                              const int4* __restrict__ ext,
                                                              const int* __restrict__ active, E epi) {
    using P = typename ProdT<T, X>::type;
    const int e = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
    if (e >= n) return;
    const int4 e4 = __ldg(ext + e);
    if (!active[e4.x]) return;
    const int4 c4 = __ldg(chunk + e);
    const int t = threadIdx.x & 31;
    if (t >= c4.y) return;
    const int r = c4.x + t;  // row of the shared matrix; row r + e4.y of the batch's vectors
    const typename E::Ops ops = epi.load(r + e4.y, e4.x);
    const int a = __ldg(ptr + r), b = __ldg(ptr + r + 1);
    const X* xb = xin + e4.z;
    pdl_acquire();
    double s = 0;
    for (int k = a; k < b; ++k) s += double(mul_rn(P(__ldg(val + k)), P(gather(xb + __ldg(idx + k)))));
    epi.apply(r + e4.y, s, ops);
}

// First primal step of a block (gpu/pdhg.cu:208-214): x = clamp(x - tau (c + ATz), l, u), xs += x.
template <class T>
__global__ void k_xupd(int n, T* __restrict__ x, const T* __restrict__ ATz, const T* __restrict__ c,
                       const T* __restrict__ l, const T* __restrict__ u, const double* __restrict__ par,
                       double* __restrict__ xs) {
    const double tau = par[0];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const T xn = T(clampv(double(x[j]) - tau * (double(c[j]) + double(ATz[j])), double(l[j]), double(u[j])));
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

constexpr int kEvalBatch = 4;  // elements whose loads a KKT-evaluation thread issues before summing them

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
    auto add = [&](double ax, double zz, double lo, double up, double dr, double zl) {
        ax *= f, zz *= f;
        double r = ax < lo ? lo - ax : (ax > up ? ax - up : 0), ro = r / dr;
        double rr = ro * row_rel_weight(lo, up, dr);
        v[0] += r * r, v[1] += ro * ro, v[2] += rr * rr;
        if (zz > 0 && up < INFINITY) v[3] -= zz * up;
        if (zz < 0 && lo > -INFINITY) v[3] -= zz * lo;
        double dz = zz - zl;
        v[4] += dz * dz;
    };
    // each thread takes rows i, i + G, i + 2G, ... (G = the grid's threads) in that order; the loads of kEvalBatch
    // rows are issued before their sums, which keep the same order
    const int G = gridDim.x * blockDim.x;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + (kEvalBatch - 1) * G < m; i += kEvalBatch * G) {
        double a[kEvalBatch], zz[kEvalBatch], lo[kEvalBatch], up[kEvalBatch], dr[kEvalBatch], zl[kEvalBatch];
#pragma unroll
        for (int e = 0; e < kEvalBatch; ++e) {
            const int k = i + e * G;
            a[e] = double(Ax[k]), zz[e] = double(z[k]), lo[e] = rl[k], up[e] = ru[k], dr[e] = double(Dr[k]);
            zl[e] = double(zlast[k]);
        }
#pragma unroll
        for (int e = 0; e < kEvalBatch; ++e) add(a[e], zz[e], lo[e], up[e], dr[e], zl[e]);
    }
    for (; i < m; i += G) add(double(Ax[i]), double(z[i]), rl[i], ru[i], double(Dr[i]), double(zlast[i]));
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
    auto add = [&](double xx, double cj, double atz, double lo, double up, double dc, double xl) {
        xx *= f;
        double d = cj + atz * f, res = 0;
        v[2] += cj * xx;
        if (d > 0) {
            if (lo > -INFINITY) v[3] += d * lo;
            else res = d;
        } else if (d < 0) {
            if (up < INFINITY) v[3] += d * up;
            else res = -d;
        }
        double ro = res / dc, dx = xx - xl;
        v[0] += res * res, v[1] += ro * ro, v[4] += dx * dx;
    };
    const int G = gridDim.x * blockDim.x;  // columns j, j + G, ... in that order, loads batched as in k_eval_row
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    for (; j + (kEvalBatch - 1) * G < n; j += kEvalBatch * G) {
        double xx[kEvalBatch], cj[kEvalBatch], atz[kEvalBatch], lo[kEvalBatch], up[kEvalBatch], dc[kEvalBatch],
            xl[kEvalBatch];
#pragma unroll
        for (int e = 0; e < kEvalBatch; ++e) {
            const int k = j + e * G;
            xx[e] = double(x[k]), cj[e] = c[k], atz[e] = double(ATz[k]), lo[e] = l[k], up[e] = u[k];
            dc[e] = double(Dc[k]), xl[e] = double(xlast[k]);
        }
#pragma unroll
        for (int e = 0; e < kEvalBatch; ++e) add(xx[e], cj[e], atz[e], lo[e], up[e], dc[e], xl[e]);
    }
    for (; j < n; j += G) add(double(x[j]), c[j], double(ATz[j]), l[j], u[j], double(Dc[j]), double(xlast[j]));
    reduce_finish<5>(v, part, ticket, out);
}

// Power iteration on A_s^T A_s with the stop test on the device (gpu/pdhg.cu:425-434). st = {est, prev, scale,
// steps taken} (the step count lives on the device, so that a captured chunk of steps can be replayed);
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

static __global__ void k_power_update(const double* out, double* st, int* done) {  // one thread
    if (*done) return;
    const double s = out[0], prev = st[0], it = st[3];
    st[3] = it + 1;
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

static __global__ void k_set_par(double* par, double tau, double sigma) { par[0] = tau, par[1] = sigma; }

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
