// Batched PDHG: many LPs of one scenario family solved together on one GPU (include/taral_pdhg.h, part 5).
//
// The batch is one block-diagonal problem. Instances that have identical constraint matrices (the same period
// count of a scenario family) share one scaled copy of A and A^T; every instance has its own vectors. The
// row-block lists of the matrices are replicated per instance with an extension word {instance, row shift,
// gather offset}, and ordered matrix-major for the iteration (the CTAs that read one matrix tile for different
// instances run back to back, so the tile is served from L2) and instance-major for the evaluation (so the
// per-instance sums are taken in a fixed order). The driver logic of gpu/pdhg.cu:761-849 -- stopping rule,
// restart rule, primal-weight update -- runs per instance on the device (k_decide, FP64), so a block of
// eval_freq iterations plus its evaluation, decisions and restarts is one CUDA graph replayed until every
// instance has stopped; finished instances' blocks return at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/taral_pdhg.h"
#include "engine.hpp"
#include "host.hpp"
#include "kernels.cuh"
#include "scaling.cuh"
#include "solve.hpp"

namespace taral {
namespace {

struct BatchError {
    std::string msg;
};
#define BK(call)                                                                                            \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) throw BatchError{std::string(#call) + ": " + cudaGetErrorString(e_)};        \
    } while (0)

// Per-instance driver state (device resident, FP64): the restart schedule shared with the single-LP driver
// (schedule.hpp: weight, step scale, anchor, iteration counters) and what the batch keeps beside it -- the averages'
// scale f = 1 / (iterations since the restart), f at the last restart, the stopping test's norms, the better
// point's residuals, the operator norm and the status flags.
struct InstState {
    Schedule sch;
    double f, f_restart, bnorm, cnorm, best_p, best_d, best_g, norm;
    int status, avg_final, running, restart_flag;
};

// ---------------------------------------------------------------------------------------------- batch kernels
// ---------------------------------------------------------------------------------------------- pack layout
// Instances that share one constraint matrix are grouped in PACKS of W in {1, 2, 4, 8} slots. Every per-instance
// vector stores the entry of (slot t, row r) of a pack at base + r * W + t: the W instances' entries of one row (or
// column) are adjacent. One CTA takes one row block of the shared matrix for all W slots of a pack: the block's
// column indices and values are staged in shared memory once, and lane (row, slot) gathers x at gbase + col * W +
// slot, so the W slots of a column share one memory segment -- a gathered 32-byte sector serves up to 8 instances
// instead of one, and the matrix block is read once for the pack.
// Per slot, every row is summed in exactly the order of the single-instance skeleton (block_sums: products rounded
// to the product type, FP64 sums; a thread per row up to kShort nonzeros, a warp per longer row, the whole CTA for a
// row longer than kTile), so a batched instance follows the same iterates as the same instance solved alone.
// Per CTA: blk = {first row in the concatenated row pointers, rows, first nonzero, end}; ext = {pack, vector index
// of (first row, slot 0), gather base of the pack's other-side vector, W}. slot_inst[8 pack + t]: the instance in
// slot t, or -1 for an unused slot.
// Row blocks of a pack of width W hold at most pack_tile(W) nonzeros and kRowsMax / W rows, so that the block's
// (nonzero, slot) pairs fit the kTile-product staging of the single-instance skeleton: (tile + 3) W < kTile + 4.
__host__ __device__ constexpr int pack_tile(int W) { return (kTile + 4) / W - 4; }
constexpr int kPairs = (kTile + 4 + kThreads - 1) / kThreads;  // staged pairs per thread (8)
static_assert((pack_tile(8) + 3) * 8 <= kPairs * kThreads && (pack_tile(1) + 3) <= kPairs * kThreads, "pairs");

__device__ __forceinline__ int log2w(int W) { return W >= 8 ? 3 : W >= 4 ? 2 : W >= 2 ? 1 : 0; }

template <class P>
struct PackSmem {
    P prod[kPairs * kThreads + kPairs * kThreads / 32];  // pair q = (nonzero - a0) * W + slot at pidx(q)
    double rowsum[kRowsMax];                              // per (row, slot) item
    int rptr[kRowsMax + 1];
    short longq[kRowsMax];
    int nlong;
    double part[kThreads / 32];
};

template <class T, class X, class E>
__global__ void __launch_bounds__(kThreads, 6) k_pack_spmv(const int* __restrict__ ptr,
                                                                     const int* __restrict__ idx,
                                                                     const T* __restrict__ val,
                                                                     const X* __restrict__ xin,
                                                                     const int4* __restrict__ blk,
                                                                     const int4* __restrict__ ext,
                                                                     const int* __restrict__ slot_inst,
                                                                     const int* __restrict__ active, E epi) {
    using P = typename ProdT<T, X>::type;
    __shared__ PackSmem<P> sm;
    __shared__ typename E::Stage st;
    const int4 e4 = __ldg(ext + blockIdx.x);
    const int pack = e4.x, vbase = e4.y, gbase = e4.z, W = e4.w, lw = log2w(W);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, my_t = tid & (W - 1);
    const int my_inst = slot_inst[8 * pack + my_t];
    const bool my_live = my_inst >= 0 && active[my_inst] != 0;
    if (!__syncthreads_or(my_live)) return;
    const int4 meta = __ldg(blk + blockIdx.x);
    const int r0 = meta.x, nrows = meta.y & 0xffff, p0 = meta.z, p1 = meta.w, len = p1 - p0;
    if (len > pack_tile(W)) {  // one long row: per live slot, the whole CTA (block_sums' long-row order)
        const int a0 = p0 & ~3;
        for (int t = 0; t < W; ++t) {
            const int inst = slot_inst[8 * pack + t];
            if (inst < 0 || !active[inst]) continue;  // uniform over the CTA
            double s = 0;
            for (int q = a0 + 4 * tid; q < p1; q += 4 * kThreads)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int k = q + e;
                    if (k >= p0 && k < p1) s += double(__ldg(val + k)) * double(__ldg(xin + gbase + __ldg(idx + k) * W + t));
                }
            for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
            if (lane == 0) sm.part[warp] = s;
            __syncthreads();
            if (tid == 0) {
                double tot = 0;
                for (int w = 0; w < kThreads / 32; ++w) tot += sm.part[w];
                const int o = vbase + t;
                const auto ops = epi.load(o, inst);
                epi.apply(o, tot, ops);
            }
            __syncthreads();
        }
        return;
    }
    // item tid = (row tid >> lw, slot my_t): its epilogue operands are copied to shared memory before the matrix stream
    const bool mine = my_live && tid < (nrows << lw);
    if (mine) epi.stage(vbase + tid, tid, st);
    // 1. stage the products of the block's (nonzero, slot) pairs: all index / value loads, then all gathers
    const int a0 = p0 & ~3, npairs = (p1 - a0) << lw;
    int c[kPairs];
    T v[kPairs];
#pragma unroll
    for (int i = 0; i < kPairs; ++i) {
        const int q = tid + i * kThreads, k = a0 + (q >> lw);
        const bool in = my_live && q < npairs && k >= p0;
        c[i] = in ? __ldg(idx + k) : -1;
        v[i] = in ? __ldg(val + k) : T(0);
    }
    X g[kPairs];
#pragma unroll
    for (int i = 0; i < kPairs; ++i) g[i] = c[i] >= 0 ? gather(xin + gbase + c[i] * W + my_t) : X(0);
#pragma unroll
    for (int i = 0; i < kPairs; ++i)
        if (c[i] >= 0) sm.prod[pidx(tid + i * kThreads)] = mul_rn(P(v[i]), P(g[i]));
    for (int t = tid; t <= nrows; t += kThreads) sm.rptr[t] = ptr[r0 + t] - a0;
    if (tid == 0) sm.nlong = 0;
    __syncthreads();
    // 2. sums: an item of at most kShort nonzeros by its own thread, longer ones by a warp each
    if (mine) {
        const int rl = tid >> lw, a = sm.rptr[rl], b = sm.rptr[rl + 1];
        if (b - a <= ((meta.y & kUniformRows) ? kTile : kShort)) {
            double s = 0;
            int k = a;
            for (; k + 8 <= b; k += 8) {  // eight loads in flight, then the adds in entry order
                P t[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) t[e] = sm.prod[pidx(((k + e) << lw) + my_t)];
#pragma unroll
                for (int e = 0; e < 8; ++e) s += double(t[e]);
            }
            for (; k < b; ++k) s += double(sm.prod[pidx((k << lw) + my_t)]);
            sm.rowsum[tid] = s;
        } else {
            sm.longq[atomicAdd(&sm.nlong, 1)] = short(tid);
        }
    }
    __syncthreads();
    for (int i = warp; i < sm.nlong; i += kThreads / 32) {  // warp-uniform trip count: all lanes shuffle
        const int q = sm.longq[i], rl = q >> lw, t = q & (W - 1);
        double s = 0;
        for (int k = sm.rptr[rl] + lane; k < sm.rptr[rl + 1]; k += 32) s += double(sm.prod[pidx((k << lw) + t)]);
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) sm.rowsum[q] = s;
    }
    __syncthreads();
    if (mine) epi.finish(vbase + tid, my_inst, tid, sm.rowsum[tid], st);
}

// Per-(CTA, slot) partial sums of the row (ROW = true) or column KKT scalars over one pack block, CTAs in
// evaluation order (gpu/pdhg.cu:236-251 and :253-271); f per instance (1 for the current point).
// part[(cta * 8 + slot) * 5 + k].
template <class T, class V, bool ROW>
__global__ void __launch_bounds__(kThreads) k_pack_eval(const int4* __restrict__ blk, const int4* __restrict__ ext,
                                                         const int* __restrict__ slot_inst,
                                                         const int* __restrict__ active, const double* __restrict__ fi,
                                                         const V* __restrict__ a, const V* __restrict__ b,
                                                         const T* __restrict__ lo_v, const T* __restrict__ up_v,
                                                         const T* __restrict__ c_v, const T* __restrict__ D,
                                                         const T* __restrict__ last, double* part) {
    const int4 e4 = ext[blockIdx.x];
    const int pack = e4.x, vbase = e4.y, W = e4.w, lw = log2w(W);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, my_t = tid & (W - 1);
    const int inst = slot_inst[8 * pack + my_t];
    const bool live = inst >= 0 && active[inst] != 0;
    const int nrows = blk[blockIdx.x].y & 0xffff;
    const double f = live && fi ? fi[inst] : 1.0;
    double v[5] = {0, 0, 0, 0, 0};
    if (live)
        for (int q = tid; q < (nrows << lw); q += kThreads) {
            const int r = vbase + q;
            if (ROW) {  // a = Ax (or A xs), b = z (or zs)
                double ax = double(a[r]) * f, zz = double(b[r]) * f, lo = lo_v[r], up = up_v[r];
                double res = ax < lo ? lo - ax : (ax > up ? ax - up : 0), ro = res / double(D[r]);
                double rr = ro * row_rel_weight(lo, up, double(D[r]));
                v[0] += res * res, v[1] += ro * ro, v[2] += rr * rr;
                if (zz > 0 && up < INFINITY) v[3] -= zz * up;
                if (zz < 0 && lo > -INFINITY) v[3] -= zz * lo;
                double dz = zz - double(last[r]);
                v[4] += dz * dz;
            } else {  // a = x (or xs), b = ATz (or A^T zs); c_v = c, lo_v = l, up_v = u
                double xx = double(a[r]) * f, cj = c_v[r], d = cj + double(b[r]) * f, lo = lo_v[r], up = up_v[r],
                       res = 0;
                v[2] += cj * xx;
                if (d > 0) {
                    if (lo > -INFINITY) v[3] += d * lo;
                    else res = d;
                } else if (d < 0) {
                    if (up < INFINITY) v[3] += d * up;
                    else res = -d;
                }
                double ro = res / double(D[r]), dx = xx - double(last[r]);
                v[0] += res * res, v[1] += ro * ro, v[4] += dx * dx;
            }
        }
    __shared__ double sh[kThreads / 32][8][5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double s = v[k];
        for (int off = 16; off >= W; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);  // lanes of one slot
        if (lane < W) sh[w][lane][k] = s;
    }
    __syncthreads();
    if (tid < 8 * 5) {
        const int t = tid / 5, k = tid % 5;
        double s = 0;
        if (t < W)
            for (int i = 0; i < kThreads / 32; ++i) s += sh[i][t][k];
        part[(size_t(blockIdx.x) * 8 + t) * 5 + k] = s;
    }
}

// One warp per instance: kkt[inst*10 + k] = sum of its pack blocks' partials, in block order (deterministic).
__global__ void k_eval_finish(int ninst, const int2* __restrict__ where, const int* __restrict__ rr,
                              const int* __restrict__ cr, const double* __restrict__ prow,
                              const double* __restrict__ pcol, const int* __restrict__ active, double* kkt) {
    const int inst = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (inst >= ninst || !active[inst] || lane >= 10) return;
    const int2 pt = where[inst];  // {pack, slot}
    double s = 0;
    if (lane < 5)
        for (int b = rr[pt.x]; b < rr[pt.x + 1]; ++b) s += prow[(size_t(b) * 8 + pt.y) * 5 + lane];
    else
        for (int b = cr[pt.x]; b < cr[pt.x + 1]; ++b) s += pcol[(size_t(b) * 8 + pt.y) * 5 + lane - 5];
    kkt[inst * 10 + lane] = s;
}

// The schedule's decision after a block (schedule.hpp, judge_block) for every running instance, one thread each.
// External stops: the host's cancel flag (pinned host memory, read through its device mapping) and the deadline,
// compared with %globaltimer (0: none). rflag[i]: where instance i restarts (RestartTo).
template <class T>
__global__ void k_decide(int ninst, InstState* st, const double* __restrict__ kc_all, const double* __restrict__ ka_all,
                         double* par, int* running, int* rflag, double tol, double row_rel, long long max_iter,
                         const unsigned long long* deadline, const volatile int* cancel) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst) return;
    rflag[i] = kNoRestart;
    InstState& s = st[i];
    if (!s.running) return;
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    const StopRule rule{tol, row_rel, s.bnorm, s.cnorm, max_iter};
    const int stop = *cancel ? int(TARAL_CANCELLED) : (*deadline && now > *deadline) ? int(TARAL_TIME_LIMIT) : -1;
    const BlockDecision d = judge_block(s.sch, kc_all + 10 * i, ka_all + 10 * i, rule, stop);
    s.best_p = d.best.primal, s.best_d = d.best.dual, s.best_g = d.best.gap, s.avg_final = d.average_better;
    if (d.status >= 0) {
        s.status = d.status, s.running = 0, running[i] = 0;
        return;
    }
    if (d.restart != kNoRestart) {
        rflag[i] = d.restart;
        s.f_restart = s.f;
        if (d.new_weight) par[2 * i] = s.sch.eta / s.sch.weight, par[2 * i + 1] = s.sch.eta * s.sch.weight;
    }
}

__global__ void k_advance(int ninst, InstState* st, int steps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst || !st[i].running) return;
    Schedule& q = st[i].sch;
    q.iterations += steps, q.since_restart += steps;
    st[i].f = 1.0 / double(q.since_restart);
}

// Gather the per-instance f (running sums scale) into a flat array for the evaluation kernels.
__global__ void k_gather_f(int ninst, const InstState* st, double* f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ninst) f[i] = st[i].f;
}

// Elementwise work over the live (row, slot) entries of one pack block per CTA (evaluation-order block lists).
#define PACK_ENTRIES(ACTIVE_EXPR)                                                                   \
    const int4 e4 = ext[blockIdx.x];                                                                \
    const int pack = e4.x, vbase = e4.y, W = e4.w, lw = log2w(W);                                   \
    const int my_t = threadIdx.x & (W - 1), inst = slot_inst[8 * pack + my_t];                      \
    const int nrows = blk[blockIdx.x].y & 0xffff;                                                   \
    const bool live = inst >= 0 && (ACTIVE_EXPR);

// First primal step of the block for every running instance (gpu/pdhg.cu:208-214).
template <class T>
__global__ void k_pack_xupd(const int4* __restrict__ blk, const int4* __restrict__ ext,
                            const int* __restrict__ slot_inst, const int* __restrict__ active, T* __restrict__ x,
                            const T* __restrict__ ATz, const T* __restrict__ c, const T* __restrict__ l,
                            const T* __restrict__ u, const double* __restrict__ par, double* __restrict__ xs) {
    PACK_ENTRIES(active[inst] != 0)
    if (!live) return;
    const double tau = par[2 * inst];
    for (int q = threadIdx.x; q < (nrows << lw); q += blockDim.x) {
        const int j = vbase + q;
        const T xn = T(clampv(double(x[j]) - tau * (double(c[j]) + double(ATz[j])), double(l[j]), double(u[j])));
        x[j] = xn, xs[j] += double(xn);
    }
}

// Restart of the flagged instances (gpu/pdhg.cu:293-299): flag 2 -> average * f, 1 -> current point.
template <class T>
__global__ void k_pack_restart(const int4* __restrict__ blk, const int4* __restrict__ ext,
                               const int* __restrict__ slot_inst, const int* __restrict__ flag,
                               const InstState* __restrict__ st, T* __restrict__ x, double* __restrict__ xs,
                               T* __restrict__ xlast) {
    PACK_ENTRIES(flag[inst] != 0)
    if (!live) return;
    const int fl = flag[inst];
    const double fr = st[inst].f_restart;
    for (int q = threadIdx.x; q < (nrows << lw); q += blockDim.x) {
        const int j = vbase + q;
        const T v = fl == 2 ? T(xs[j] * fr) : x[j];
        x[j] = v, xlast[j] = v, xs[j] = 0;
    }
}

// Power iteration: per-(CTA, slot) partial ||v||^2 over one pack block (part[cta * 8 + slot]).
template <class T>
__global__ void __launch_bounds__(kThreads) k_pack_pow_part(const int4* __restrict__ blk, const int4* __restrict__ ext,
                                                             const int* __restrict__ slot_inst,
                                                             const int* __restrict__ active, const T* __restrict__ v,
                                                             double* part) {
    PACK_ENTRIES(active[inst] != 0)
    double a = 0;
    if (live)
        for (int q = threadIdx.x; q < (nrows << lw); q += kThreads) {
            const double t = double(v[vbase + q]);
            a += t * t;
        }
    for (int off = 16; off >= W; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    __shared__ double sh[kThreads / 32][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane < W) sh[w][lane] = a;
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0;
        if (int(threadIdx.x) < W)
            for (int i = 0; i < kThreads / 32; ++i) s += sh[i][threadIdx.x];
        part[size_t(blockIdx.x) * 8 + threadIdx.x] = s;
    }
}

__global__ void k_pow_update(int ninst, const int2* __restrict__ where, const int* __restrict__ cr,
                             const double* __restrict__ part, double* est, double* scale, int* active, int it) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst || !active[i]) return;
    const int2 pt = where[i];
    double s = 0;
    for (int b = cr[pt.x]; b < cr[pt.x + 1]; ++b) s += part[size_t(b) * 8 + pt.y];
    double prev = est[i];
    if (s <= 0) {
        est[i] = 0, active[i] = 0;
        return;
    }
    double e = sqrt(sqrt(s));
    est[i] = e, scale[i] = 1 / sqrt(s);
    if (it >= 10 && fabs(e - prev) <= 1e-7 * e) active[i] = 0;
}

template <class T>
__global__ void k_pack_pow_scale(const int4* __restrict__ blk, const int4* __restrict__ ext,
                                 const int* __restrict__ slot_inst, const int* __restrict__ active,
                                 const double* __restrict__ scale, T* __restrict__ v) {
    PACK_ENTRIES(active[inst] != 0)
    if (!live) return;
    const double sc = scale[inst];
    for (int q = threadIdx.x; q < (nrows << lw); q += blockDim.x) v[vbase + q] = T(double(v[vbase + q]) * sc);
}

// Download: out = (avg ? sum * f : point) for every used slot.
template <class T>
__global__ void k_pack_out(const int4* __restrict__ blk, const int4* __restrict__ ext,
                           const int* __restrict__ slot_inst, const InstState* __restrict__ st,
                           const T* __restrict__ x, const double* __restrict__ xs, double* __restrict__ out) {
    PACK_ENTRIES(true)
    if (!live) return;
    const InstState& s = st[inst];
    const double f = 1.0 / double(s.sch.since_restart > 1 ? s.sch.since_restart : 1);
    for (int q = threadIdx.x; q < (nrows << lw); q += blockDim.x) {
        const int j = vbase + q;
        out[j] = s.avg_final ? xs[j] * f : double(x[j]);
    }
}
#undef PACK_ENTRIES

__global__ void k_kkt_init(int ninst, InstState* st, const double* __restrict__ kc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst) return;
    st[i].sch.anchor = weighted_error(kc + 10 * i, st[i].sch.weight), st[i].sch.previous = INFINITY;
}

__global__ void k_set_deadline(unsigned long long* d, unsigned long long left_ns) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    *d = now + left_ns;
}

__global__ void k_count(int ninst, const int* __restrict__ running, int* count) {
    __shared__ int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    int c = 0;
    for (int i = threadIdx.x; i < ninst; i += blockDim.x) c += running[i] != 0;
    atomicAdd(&s, c);
    __syncthreads();
    if (threadIdx.x == 0) *count = s;
}

// ---------------------------------------------------------------------------------------------- host side
struct Shared {  // one distinct scaled matrix
    Scaled S;    // matrix part only: the unscaled A and AT on the host until they are uploaded, then Dr and Dc
    std::map<int, std::pair<std::vector<int4>, std::vector<int4>>> blk;  // pack width -> row blocks of A, A^T
    int pbaseA = 0, pbaseT = 0;
    int64_t nnzbase = 0, nnz = 0;
    int dr_off = 0, dc_off = 0;  // offsets of this matrix's Dr / Dc in the device scaling scratch
    int maxrowA = 0, maxrowT = 0;  // longest row of A and of A^T
};

uint64_t fnv(const void* p, size_t n, uint64_t h) {  // FNV-1a over 8-byte words, then the tail bytes
    const unsigned char* b = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 1099511628211ull;
    }
    for (; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

}  // namespace

struct BatchBase {
    virtual ~BatchBase() = default;
    // Returns TARAL_OK, or TARAL_ERR_CANCELLED when a cancel request stopped some instance.
    virtual int solve(const double* const* x0, const double* const* y0, const double* w0, taral_outcome* outs,
                      double* const* xo, double* const* yo) = 0;
    virtual void cancel() = 0;  // any host thread, also during solve()
    std::string err;
    int distinct = 0;
    size_t mem_used = 0;
    int64_t nnz_stored = 0, nnz_total = 0, launches = 0;
};

template <class T>
struct Batch final : BatchBase {
    int ninst = 0, M = 0, N = 0, nA = 0, nT = 0, freq = 64;
    int nA1 = 0, nT1 = 0, nAp = 0, nTp = 0;  // iteration CTAs: width-1 packs (k_rowblock_batch), wider packs
    Options opt;
    std::vector<const taral_model*> models;
    std::vector<int> mat_of;                 // instance -> distinct matrix
    std::vector<std::unique_ptr<Shared>> mats;
    std::vector<Scaled> vecs;                // per instance: vector part
    struct Pack {  // up to 8 instances sharing one matrix; vector entry (slot t, row r) at base + r * W + t
        int mat = 0, W = 1, rbase = 0, cbase = 0;
        int inst[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    };
    std::vector<Pack> packs;
    std::vector<int2> where;  // instance -> {pack, slot}
    int xidx(int i, int j) const { const Pack& q = packs[where[i].x]; return q.cbase + j * q.W + where[i].y; }
    int zidx(int i, int r) const { const Pack& q = packs[where[i].x]; return q.rbase + r * q.W + where[i].y; }
    // device
    int *Aptr = nullptr, *Aidx = nullptr, *Tptr = nullptr, *Tidx = nullptr;
    T *Aval = nullptr, *Tval = nullptr;
    int4 *A_it = nullptr, *Ae_it = nullptr, *T_it = nullptr, *Te_it = nullptr;
    int4 *A1_it = nullptr, *Ae1_it = nullptr, *T1_it = nullptr, *Te1_it = nullptr;
    // row-chunk lists of the width-1 packs for k_rowthread_batch: one warp per kChunk rows of one instance
    int nA1r = 0, nT1r = 0;
    int4 *A1_rc = nullptr, *Ae1_rc = nullptr, *T1_rc = nullptr, *Te1_rc = nullptr;
    std::vector<int4> h_a1r, h_ae1r, h_t1r, h_te1r, c_a1r, c_ae1r, c_t1r, c_te1r;
    std::vector<int4> h_a1, h_ap, h_t1, h_tp;  // host copies of the iteration block lists (autotuner)
    std::vector<int4> h_ae1, h_ae, h_te1, h_te;  // and of their extensions (instance or pack of each entry)
    std::vector<int4> c_a1, c_ae1, c_ap, c_ae, c_t1, c_te1, c_tp, c_te;  // the compacted lists last uploaded
    bool compacted = false;
    int tuned[2] = {0, 0};
    bool thread1[2] = {false, false};  // width-1 lists of A / A^T run on k_rowthread_batch
    int4 *A_ev = nullptr, *Ae_ev = nullptr, *T_ev = nullptr, *Te_ev = nullptr;
    int *rr = nullptr, *cr = nullptr, *slot_inst = nullptr;
    int2* d_where = nullptr;
    T *c = nullptr, *l = nullptr, *u = nullptr, *Dc = nullptr, *rl = nullptr, *ru = nullptr, *Dr = nullptr;
    double* par = nullptr;  // per instance {tau, sigma}
    T *x = nullptr, *ATz = nullptr, *xlast = nullptr, *z = nullptr, *Ax = nullptr, *zlast = nullptr;
    T *pv = nullptr, *pu = nullptr, *pw = nullptr;
    double *xs = nullptr, *zs = nullptr, *tmpM = nullptr, *tmpN = nullptr, *partA = nullptr, *partT = nullptr;
    double *kkt = nullptr, *fbuf = nullptr, *est = nullptr, *pscale = nullptr, *dout = nullptr;
    InstState* st = nullptr;
    unsigned long long* d_deadline = nullptr;
    int *running = nullptr, *rflag = nullptr, *pactive = nullptr, *count = nullptr, *h_count = nullptr;
    int* h_cancel = nullptr;        // pinned, mapped host memory: the cancel request (0 / 1)
    const int* d_cancel = nullptr;  // its device address
    cudaStream_t s = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<void*> allocs;

    template <class U>
    U* alloc(size_t n) {  // stream-ordered, from the device's memory pool (keep_pool_memory)
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(n, 1) * sizeof(U);
        if (!alloc_allowed(alloc_bytes, bytes))
            throw BatchError{"cudaMalloc: the device allocation limit (taral_set_device_alloc_limit) is reached"};
        cudaError_t e = cudaMallocAsync(&p, bytes, s);
        if (e != cudaSuccess) throw BatchError{std::string("cudaMalloc: ") + cudaGetErrorString(e)};
        allocs.push_back(p);
        alloc_bytes += bytes;
        return static_cast<U*>(p);
    }
    size_t alloc_bytes = 0;
    template <class U>
    U* put(const std::vector<U>& h) {
        U* p = alloc<U>(h.size());
        if (!h.empty()) BK(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(U), cudaMemcpyHostToDevice, s));
        BK(cudaStreamSynchronize(s));
        return p;
    }
    ~Batch() override {
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : allocs) cudaFreeAsync(p, s);
        if (s) cudaStreamSynchronize(s);
        if (h_count) cudaFreeHost(h_count);
        if (h_cancel) cudaFreeHost(h_cancel);
        if (s) cudaStreamDestroy(s);
    }

    void build(const taral_model* md, int count, const Options& o) {
        ninst = count, opt = o, freq = std::max(1, o.eval_freq);
        const auto tb = Clock::now();
        std::vector<std::pair<const char*, double>> marks;  // TARAL_TIMING: set-up steps, seconds since tb
        auto mark = [&](const char* what) { marks.emplace_back(what, since(tb)); };
        int dev = 0;
        BK(cudaGetDevice(&dev));
        keep_pool_memory(dev);
        BK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        if (const char* e = std::getenv("TARAL_PDL")) pdl = std::atoi(e) != 0;
        // 1. distinct matrices (same sizes and identical col_ptr / row_idx / val). Instances passing the very arrays
        //    of an earlier one share its matrix at once; otherwise a matrix is compared (FNV-1a hash, then bytes)
        //    only with the earlier distinct matrices of the same sizes, and hashed only when there are some.
        std::map<std::tuple<const void*, const void*, const void*, int, int>, int> same_arrays;
        std::map<std::tuple<int, int, int64_t>, std::vector<int>> by_size;  // (m, n, nnz) -> distinct matrices
        std::vector<uint64_t> mat_hash;
        std::vector<char> mat_hashed;
        auto hash_of = [](const taral_model& m) {
            const int64_t nz = m.col_ptr[m.n];
            uint64_t h = 1469598103934665603ull;
            h = fnv(m.col_ptr, size_t(m.n + 1) * sizeof(int64_t), h);
            h = fnv(m.row_idx, size_t(nz) * sizeof(int32_t), h);
            return fnv(m.val, size_t(nz) * sizeof(double), h);
        };
        mat_of.resize(count);
        for (int i = 0; i < count; ++i) {
            const taral_model& m = md[i];
            const int64_t nz = m.col_ptr[m.n];
            const auto akey = std::make_tuple((const void*)m.col_ptr, (const void*)m.row_idx, (const void*)m.val, m.m, m.n);
            auto sa = same_arrays.find(akey);
            if (sa != same_arrays.end()) {  // the very arrays of an earlier instance: the same matrix
                mat_of[i] = sa->second;
                continue;
            }
            std::vector<int>& ids = by_size[std::make_tuple(m.m, m.n, nz)];
            int found = -1;
            if (!ids.empty()) {
                const uint64_t h = hash_of(m);
                for (int id : ids) {
                    const taral_model& r = md[first_inst[id]];
                    if (!mat_hashed[id]) mat_hash[id] = hash_of(r), mat_hashed[id] = 1;
                    if (mat_hash[id] == h && !std::memcmp(r.col_ptr, m.col_ptr, size_t(m.n + 1) * sizeof(int64_t)) &&
                        !std::memcmp(r.row_idx, m.row_idx, size_t(nz) * sizeof(int32_t)) &&
                        !std::memcmp(r.val, m.val, size_t(nz) * sizeof(double))) {
                        found = id;
                        break;
                    }
                }
            }
            if (found < 0) {
                found = int(mats.size());
                mats.push_back(std::make_unique<Shared>());
                first_inst.push_back(i);
                mat_hash.push_back(0), mat_hashed.push_back(0);
                ids.push_back(found);
            }
            mat_of[i] = found;
            same_arrays[akey] = found;
        }
        distinct = int(mats.size());
        mark("match");
        // 2. unscaled matrices (host transposes, threads over matrices); scaled on the device in step 3
        unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        auto par_for = [&](int n, auto&& fn) {
            std::vector<std::thread> th;
            std::atomic<int> next{0};
            int nt = int(std::min<unsigned>(hw, unsigned(std::max(n, 1))));
            for (int t = 0; t < nt; ++t)
                th.emplace_back([&] {
                    for (int k = next++; k < n; k = next++) fn(k);
                });
            for (auto& t : th) t.join();
        };
        par_for(distinct, [&](int k) {
            Shared& sh = *mats[k];
            const taral_model& mk = md[first_inst[k]];
            model_matrices(mk, sh.S.A, sh.S.AT, 1);
            sh.S.m = mk.m, sh.S.n = mk.n, sh.nnz = int64_t(sh.S.A.idx.size());
        });
        mark("transposes");
        // 3. concatenated matrices (int32 offsets), uploaded unscaled and scaled on the device (scaling.cuh:
        //    bit-identical to the reference's host scaling), values narrowed to T in place
        std::vector<int> hAptr, hTptr;
        int64_t nzb = 0;
        int drn = 0, dcn = 0;
        for (auto& shp : mats) {
            Shared& sh = *shp;
            sh.pbaseA = int(hAptr.size()), sh.pbaseT = int(hTptr.size()), sh.nnzbase = nzb;
            sh.dr_off = drn, sh.dc_off = dcn;
            drn += sh.S.m, dcn += sh.S.n;
            for (int64_t v : sh.S.A.ptr) hAptr.push_back(int(v + nzb));
            for (int64_t v : sh.S.AT.ptr) hTptr.push_back(int(v + nzb));
            nzb += sh.nnz;
            if (nzb > INT32_MAX - 64) throw BatchError{"more than 2^31 distinct nonzeros in a batch"};
        }
        nnz_stored = nzb;
        Aptr = put(hAptr), Tptr = put(hTptr);
        Aidx = alloc<int>(size_t(nzb)), Tidx = alloc<int>(size_t(nzb));
        Aval = alloc<T>(size_t(nzb)), Tval = alloc<T>(size_t(nzb));
        {
            struct Scratch {
                std::vector<void*> p;
                cudaStream_t st;
                ~Scratch() { for (void* q : p) cudaFreeAsync(q, st); }
            } tmp{{}, s};
            auto scratch = [&](size_t k) {
                void* q = nullptr;
                BK(cudaMallocAsync(&q, std::max<size_t>(k, 1) * sizeof(double), s));
                tmp.p.push_back(q);
                return static_cast<double*>(q);
            };
            double *va, *vt;
            if (sizeof(T) == sizeof(double)) va = reinterpret_cast<double*>(Aval), vt = reinterpret_cast<double*>(Tval);
            else va = scratch(size_t(nzb)), vt = scratch(size_t(nzb));
            double *dr = scratch(size_t(drn)), *dc = scratch(size_t(dcn)), *rs = scratch(size_t(drn)),
                   *cs = scratch(size_t(dcn));
            for (auto& shp : mats) {
                Shared& sh = *shp;
                const size_t nz = size_t(sh.nnz), b = size_t(sh.nnzbase);
                if (nz) {
                    BK(cudaMemcpyAsync(Aidx + b, sh.S.A.idx.data(), nz * sizeof(int), cudaMemcpyHostToDevice, s));
                    BK(cudaMemcpyAsync(Tidx + b, sh.S.AT.idx.data(), nz * sizeof(int), cudaMemcpyHostToDevice, s));
                    BK(cudaMemcpyAsync(va + b, sh.S.A.val.data(), nz * sizeof(double), cudaMemcpyHostToDevice, s));
                    BK(cudaMemcpyAsync(vt + b, sh.S.AT.val.data(), nz * sizeof(double), cudaMemcpyHostToDevice, s));
                }
                scale_on_device(sh.S.m, sh.S.n, Aptr + sh.pbaseA, Aidx, va, Tptr + sh.pbaseT, Tidx, vt,
                                dr + sh.dr_off, dc + sh.dc_off, rs + sh.dr_off, cs + sh.dc_off, s);
            }
            if (sizeof(T) != sizeof(double) && nzb) {
                const int g = int(std::min<int64_t>((nzb + 255) / 256, 148 * 16));
                k_narrow<T><<<g, 256, 0, s>>>(nzb, va, Aval);
                k_narrow<T><<<g, 256, 0, s>>>(nzb, vt, Tval);
            }
            std::vector<double> hdr(static_cast<size_t>(drn)), hdc(static_cast<size_t>(dcn));
            if (drn) BK(cudaMemcpyAsync(hdr.data(), dr, size_t(drn) * sizeof(double), cudaMemcpyDeviceToHost, s));
            if (dcn) BK(cudaMemcpyAsync(hdc.data(), dc, size_t(dcn) * sizeof(double), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            BK(cudaGetLastError());
            for (auto& shp : mats) {
                Shared& sh = *shp;
                sh.S.Dr.assign(hdr.begin() + sh.dr_off, hdr.begin() + sh.dr_off + sh.S.m);
                sh.S.Dc.assign(hdc.begin() + sh.dc_off, hdc.begin() + sh.dc_off + sh.S.n);
                for (Csr* h : {&sh.S.A, &sh.S.AT}) {  // keep the row pointers (block lists), drop the entries
                    h->idx.clear(), h->idx.shrink_to_fit();
                    h->val.clear(), h->val.shrink_to_fit();
                }
            }
        }
        mark("upload+scaling");
        vecs.resize(count);
        par_for(count, [&](int i) {
            const Shared& sh = *mats[mat_of[i]];
            scale_vectors(md[i], md[i].maximize ? -1.0 : 1.0, sh.S.Dr, sh.S.Dc, vecs[i]);
        });
        // 4. packs (instances of one matrix, 8 slots, the remainder in the smallest power of two) and block lists
        std::vector<std::vector<int>> users(distinct);
        for (int i = 0; i < count; ++i) users[mat_of[i]].push_back(i);
        std::vector<std::vector<int>> packs_of(distinct);
        int pack_cap = 1;  // widest pack; TARAL_BATCH_PACK = 1, 2, 4 or 8 overrides
        if (const char* e = std::getenv("TARAL_BATCH_PACK")) {
            const int v = std::atoi(e);
            pack_cap = v >= 8 ? 8 : v >= 4 ? 4 : v >= 2 ? 2 : 1;
        }
        where.assign(count, make_int2(0, 0));
        int64_t Mt = 0, Nt = 0;
        for (int k = 0; k < distinct; ++k) {
            const Shared& sh = *mats[k];
            for (size_t u0 = 0; u0 < users[k].size();) {
                const int rem = int(users[k].size() - u0);
                Pack q;  // width: the smallest power of two holding the remaining instances, at most pack_cap
                q.mat = k, q.W = std::min(pack_cap, rem > 4 ? 8 : rem > 2 ? 4 : rem);
                const int used = std::min(rem, q.W);
                q.rbase = int(Mt), q.cbase = int(Nt);
                Mt += int64_t(sh.S.m) * q.W, Nt += int64_t(sh.S.n) * q.W;
                for (int t = 0; t < used; ++t) q.inst[t] = users[k][u0 + t], where[users[k][u0 + t]] = make_int2(int(packs.size()), t);
                packs_of[k].push_back(int(packs.size()));
                packs.push_back(q);
                u0 += size_t(used);
            }
            Shared& shw = *mats[k];
            for (int r = 0; r < shw.S.m; ++r)
                shw.maxrowA = std::max<int>(shw.maxrowA, int(shw.S.A.ptr[size_t(r) + 1] - shw.S.A.ptr[size_t(r)]));
            for (int r = 0; r < shw.S.n; ++r)
                shw.maxrowT = std::max<int>(shw.maxrowT, int(shw.S.AT.ptr[size_t(r) + 1] - shw.S.AT.ptr[size_t(r)]));
            for (int p : packs_of[k]) {
                const int W = packs[p].W;
                if (!shw.blk.count(W))
                    shw.blk[W] = {build_row_blocks(shw.S.A.ptr.data(), shw.S.m, pack_tile(W), kRowsMax / W),
                                  build_row_blocks(shw.S.AT.ptr.data(), shw.S.n, pack_tile(W), kRowsMax / W)};
            }
        }
        if (Mt + Nt > INT32_MAX - 1024) throw BatchError{"batch too large for int32 indexing"};
        M = int(Mt), N = int(Nt);
        std::vector<int4> a_it, ae_it, t_it, te_it, a_ev, ae_ev, t_ev, te_ev;
        std::vector<int> hrr{0}, hcr{0}, hslot;
        auto rebase = [](int4 b, int pbase, int64_t nzbase) {
            return make_int4(b.x + pbase, b.y, int(b.z + nzbase), int(b.w + nzbase));
        };
        auto extA = [&](int p, const int4& b) { const Pack& q = packs[p]; return make_int4(p, q.rbase + b.x * q.W, q.cbase, q.W); };
        auto extT = [&](int p, const int4& b) { const Pack& q = packs[p]; return make_int4(p, q.cbase + b.x * q.W, q.rbase, q.W); };
        for (int p = 0; p < int(packs.size()); ++p) {  // evaluation order: pack-major
            const Shared& sh = *mats[packs[p].mat];
            const auto& bl = sh.blk.at(packs[p].W);
            for (const int4& b : bl.first) a_ev.push_back(rebase(b, sh.pbaseA, sh.nnzbase)), ae_ev.push_back(extA(p, b));
            for (const int4& b : bl.second) t_ev.push_back(rebase(b, sh.pbaseT, sh.nnzbase)), te_ev.push_back(extT(p, b));
            hrr.push_back(int(a_ev.size())), hcr.push_back(int(t_ev.size()));
            for (int t = 0; t < 8; ++t) hslot.push_back(packs[p].inst[t]);
        }
        // iteration order: matrix-major, the packs of one width interleaved per block. Width-1 packs (one instance)
        // run on the single-instance skeleton k_rowblock_batch, whose block extension is {instance, row shift,
        // gather offset, 0}; wider packs on k_pack_spmv.
        std::vector<int4> a1_it, ae1_it, t1_it, te1_it;
        for (int k = 0; k < distinct; ++k) {
            const Shared& sh = *mats[k];
            for (const auto& wb : sh.blk) {
                const bool one = wb.first == 1;
                for (const int4& b : wb.second.first)
                    for (int p : packs_of[k]) {
                        if (packs[p].W != wb.first) continue;
                        const int4 rb = rebase(b, sh.pbaseA, sh.nnzbase);
                        if (one) a1_it.push_back(rb), ae1_it.push_back(make_int4(packs[p].inst[0], packs[p].rbase - sh.pbaseA, packs[p].cbase, 0));
                        else a_it.push_back(rb), ae_it.push_back(extA(p, b));
                    }
                for (const int4& b : wb.second.second)
                    for (int p : packs_of[k]) {
                        if (packs[p].W != wb.first) continue;
                        const int4 rb = rebase(b, sh.pbaseT, sh.nnzbase);
                        if (one) t1_it.push_back(rb), te1_it.push_back(make_int4(packs[p].inst[0], packs[p].cbase - sh.pbaseT, packs[p].rbase, 0));
                        else t_it.push_back(rb), te_it.push_back(extT(p, b));
                    }
            }
        }
        // row-chunk lists of the width-1 packs, in the same matrix-major order (a chunk, then its instances)
        for (int k = 0; k < distinct; ++k) {
            const Shared& sh = *mats[k];
            for (int r0 = 0; r0 < sh.S.m; r0 += kChunk)
                for (int p : packs_of[k])
                    if (packs[p].W == 1)
                        h_a1r.push_back(make_int4(sh.pbaseA + r0, std::min(kChunk, sh.S.m - r0), 0, 0)),
                            h_ae1r.push_back(make_int4(packs[p].inst[0], packs[p].rbase - sh.pbaseA, packs[p].cbase, 0));
            for (int r0 = 0; r0 < sh.S.n; r0 += kChunk)
                for (int p : packs_of[k])
                    if (packs[p].W == 1)
                        h_t1r.push_back(make_int4(sh.pbaseT + r0, std::min(kChunk, sh.S.n - r0), 0, 0)),
                            h_te1r.push_back(make_int4(packs[p].inst[0], packs[p].cbase - sh.pbaseT, packs[p].rbase, 0));
        }
        nA1r = int(h_a1r.size()), nT1r = int(h_t1r.size());
        A1_rc = put(h_a1r), Ae1_rc = put(h_ae1r), T1_rc = put(h_t1r), Te1_rc = put(h_te1r);
        nA = int(a_ev.size()), nT = int(t_ev.size());
        nA1 = int(a1_it.size()), nT1 = int(t1_it.size()), nAp = int(a_it.size()), nTp = int(t_it.size());
        A1_it = put(a1_it), Ae1_it = put(ae1_it), T1_it = put(t1_it), Te1_it = put(te1_it);
        h_a1 = a1_it, h_ap = a_it, h_t1 = t1_it, h_tp = t_it;
        h_ae1 = ae1_it, h_ae = ae_it, h_te1 = te1_it, h_te = te_it;
        slot_inst = put(hslot), d_where = put(where);
        // 5. upload
        A_it = put(a_it), Ae_it = put(ae_it), T_it = put(t_it), Te_it = put(te_it);
        A_ev = put(a_ev), Ae_ev = put(ae_ev), T_ev = put(t_ev), Te_ev = put(te_ev);
        rr = put(hrr), cr = put(hcr);
        std::vector<T> hc(N, T(0)), hl(N, T(0)), hu(N, T(0)), hDc(N, T(1)), hrl(M, T(0)), hru(M, T(0)), hDr(M, T(1));
        par_for(count, [&](int i) {  // every instance fills its own slots
            const Scaled& v = vecs[i];
            const Shared& sh = *mats[mat_of[i]];
            for (int j = 0; j < md[i].n; ++j) {
                const int g = xidx(i, j);
                hc[g] = T(v.c[j]), hl[g] = T(v.l[j]), hu[g] = T(v.u[j]), hDc[g] = T(sh.S.Dc[j]);
            }
            for (int r = 0; r < md[i].m; ++r) {
                const int g = zidx(i, r);
                hrl[g] = T(v.rl[r]), hru[g] = T(v.ru[r]), hDr[g] = T(sh.S.Dr[r]);
            }
        });
        c = put(hc), l = put(hl), u = put(hu), Dc = put(hDc), rl = put(hrl), ru = put(hru), Dr = put(hDr);
        x = alloc<T>(N), ATz = alloc<T>(N), xlast = alloc<T>(N), z = alloc<T>(M), Ax = alloc<T>(M), zlast = alloc<T>(M);
        pv = alloc<T>(N), pu = alloc<T>(N), pw = alloc<T>(M);
        xs = alloc<double>(N), zs = alloc<double>(M), tmpM = alloc<double>(M), tmpN = alloc<double>(N);
        dout = alloc<double>(size_t(std::max(M, N)));
        partA = alloc<double>(size_t(std::max(nA, 1)) * 40), partT = alloc<double>(size_t(std::max(nT, 1)) * 40);
        kkt = alloc<double>(size_t(count) * 20), fbuf = alloc<double>(count), est = alloc<double>(count);
        pscale = alloc<double>(count), st = alloc<InstState>(count), par = alloc<double>(2 * size_t(count));
        running = alloc<int>(count), rflag = alloc<int>(count), pactive = alloc<int>(count), this->count = alloc<int>(1);
        d_deadline = alloc<unsigned long long>(1);
        BK(cudaMallocHost(&h_count, sizeof(int)));
        BK(cudaHostAlloc(reinterpret_cast<void**>(&h_cancel), sizeof(int), cudaHostAllocMapped));
        __atomic_store_n(h_cancel, 0, __ATOMIC_SEQ_CST);
        void* dc = nullptr;
        BK(cudaHostGetDevicePointer(&dc, h_cancel, 0));
        d_cancel = static_cast<const int*>(dc);
        BK(cudaStreamSynchronize(s));
        mem_used = alloc_bytes;
        nnz_total = 0;
        for (int i = 0; i < count; ++i) nnz_total += mats[mat_of[i]]->nnz;
        models.clear();
        for (int i = 0; i < count; ++i) models.push_back(md + i);
        mark("vectors+lists");
        tune();
        mark("tune");
        if (std::getenv("TARAL_TIMING")) {
            std::fprintf(stderr, "taral: batch set-up");
            for (const auto& mk : marks) std::fprintf(stderr, " %s %.3f", mk.first, mk.second);
            std::fprintf(stderr, " s\n");
        }
    }

    // Autotuner, per phase over the whole batch (batches of at least 2^20 nonzeros), timed on the phase itself with
    // its fused step (5 launches after 2 warm-ups, on the not yet started state: solve() rewrites every vector the
    // steps write); a choice other than the default is kept only if it is at least 5 % faster:
    // 1. FP32 batches: the engine's five row-split policies (policies 1, 3, 4 only where some row exceeds kShort);
    // 2. k_rowthread_batch for the width-1 lists: any precision where no row exceeds kShort (bit-identical under
    //    policy 0), FP32 also for rows up to kMid (every row by its own thread, entry order).
    // TARAL_TUNE=0 keeps the defaults; TARAL_ROWSPLIT=0..4 and TARAL_ROWTHREAD=0|1 force a choice, untimed.
    void tune() {
        if (const char* e = std::getenv("TARAL_TUNE"))
            if (std::atoi(e) == 0) return;
        const int forced = forced_row_split();
        int forced_thread = -1;
        if (const char* e = std::getenv("TARAL_ROWTHREAD")) forced_thread = std::atoi(e) != 0 ? 1 : 0;
        const bool timing = forced < 0 && forced_thread < 0;
        if (timing && nnz_total < (int64_t(1) << 20)) return;  // small: timings are noise
        std::vector<int> ones(size_t(ninst), 1);
        BK(cudaMemcpyAsync(pactive, ones.data(), ones.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        BK(cudaMemsetAsync(par, 0, 2 * size_t(ninst) * sizeof(double), s));
        auto variant = [](const std::vector<int4>& h, int policy, bool& any) {
            std::vector<int4> a(h);
            if (policy > 0 && apply_row_split(a, policy)) any = true;
            return a;
        };
        for (int phase = 0; phase < 2; ++phase) {
            std::vector<int4>& h1 = phase ? h_t1 : h_a1;
            std::vector<int4>& hp = phase ? h_tp : h_ap;
            int4* d1 = phase ? T1_it : A1_it;
            int4* dp = phase ? T_it : A_it;
            int maxrow = 0;
            for (const auto& m : mats) maxrow = std::max(maxrow, phase ? m->maxrowT : m->maxrowA);
            const bool short_rows = maxrow <= kShort;
            const bool thread_ok = short_rows || (sizeof(T) == sizeof(float) && maxrow <= kMid);
            auto put_lists = [&](const std::vector<int4>& l1, const std::vector<int4>& lp) {
                if (!l1.empty()) BK(cudaMemcpyAsync(d1, l1.data(), l1.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
                if (!lp.empty()) BK(cudaMemcpyAsync(dp, lp.data(), lp.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
            };
            auto run = [&] {
                if (phase) spmv_T(z, EpiCol<T>{ATz, x, xs, c, l, u, par, 1}, pactive);
                else spmv_A(x, EpiRow<T>{Ax, z, zs, rl, ru, par}, pactive);
            };
            auto time_run = [&](int warm) {
                for (int r = 0; r < warm; ++r) run();
                cudaEvent_t e0, e1;
                BK(cudaEventCreate(&e0));
                BK(cudaEventCreate(&e1));
                BK(cudaEventRecord(e0, s));
                for (int r = 0; r < 5; ++r) run();
                BK(cudaEventRecord(e1, s));
                BK(cudaEventSynchronize(e1));
                float ms = 0;
                BK(cudaEventElapsedTime(&ms, e0, e1));
                cudaEventDestroy(e0), cudaEventDestroy(e1);
                return ms;
            };
            std::vector<int4> v1[kPolicies], vp[kPolicies];
            bool timed[kPolicies] = {true};
            for (int pol = 0; pol < kPolicies; ++pol) {
                bool any = pol == 0;
                v1[pol] = variant(h1, pol, any), vp[pol] = variant(hp, pol, any);
                if (pol > 0) timed[pol] = sizeof(T) == sizeof(float) && any && (!short_rows || pol == 2);
            }
            int best = 0;
            bool thread = false;
            if (!timing) {
                if (sizeof(T) == sizeof(float) && forced >= 0) best = forced;
                thread = thread_ok && best == 0 && forced_thread == 1;
            } else {
                put_lists(v1[0], vp[0]);
                const float t0 = time_run(6);
                float tb = t0;
                for (int k = 1; k < kPolicies; ++k) {
                    if (!timed[k]) continue;
                    put_lists(v1[k], vp[k]);
                    const float t = time_run(2);
                    if (t < 0.95f * t0 && t < tb) tb = t, best = k;
                }
                put_lists(v1[0], vp[0]);
                if (thread_ok && (phase ? nT1r : nA1r) > 0) {
                    thread1[phase] = true;
                    const float t = time_run(2);
                    thread1[phase] = false;
                    if (t < 0.95f * t0 && t < tb) tb = t, best = 0, thread = true;
                }
            }
            tuned[phase] = best;
            thread1[phase] = thread;
            if (std::getenv("TARAL_TIMING"))
                std::fprintf(stderr, "taral: batch tune %s: policy %d%s\n", phase ? "A^T" : "A", best,
                             thread ? ", thread per row" : "");
            h1 = v1[best], hp = vp[best];
            put_lists(h1, hp);
            BK(cudaStreamSynchronize(s));
        }
        launches = 0;
    }
    std::vector<int> first_inst;  // distinct matrix -> first instance that has it

    // ------------------------------------------------------------------ launches
    // `programmatic`: the width-1 kernels of an iteration's two phases start while their predecessor drains (they
    // wait for their predecessor before the first gather and release their successor after that wait); on with
    // TARAL_PDL=1. The wide-pack kernel always launches plainly.
    template <class K, class... Args>
    void launch(K kernel, int grid, bool programmatic, Args... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(grid)), cfg.blockDim = dim3(kThreads), cfg.dynamicSmemBytes = 0, cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr, cfg.numAttrs = programmatic ? 1 : 0;
        BK(cudaLaunchKernelEx(&cfg, kernel, args...));
        ++launches;
    }
    bool pdl = false;  // TARAL_PDL=1 (set at build)
    template <class X, class E>
    void spmv_A(const X* xin, const E& e, const int* act, bool programmatic = false) {
        if (thread1[0] && nA1r)
            launch(k_rowthread_batch<T, X, E>, (nA1r + 7) / 8, programmatic, nA1r, (const int*)Aptr, (const int*)Aidx,
                   (const T*)Aval, xin, (const int4*)A1_rc, (const int4*)Ae1_rc, act, e);
        else if (nA1)
            launch(k_rowblock_batch<T, X, E, true>, nA1, programmatic, (const int*)Aptr, (const int*)Aidx,
                   (const T*)Aval, xin, (const int4*)A1_it, (const int4*)Ae1_it, act, e);
        if (nAp) k_pack_spmv<T, X, E><<<nAp, kThreads, 0, s>>>(Aptr, Aidx, Aval, xin, A_it, Ae_it, slot_inst, act, e), ++launches;
    }
    template <class X, class E>
    void spmv_T(const X* xin, const E& e, const int* act, bool programmatic = false) {
        if (thread1[1] && nT1r)
            launch(k_rowthread_batch<T, X, E>, (nT1r + 7) / 8, programmatic, nT1r, (const int*)Tptr, (const int*)Tidx,
                   (const T*)Tval, xin, (const int4*)T1_rc, (const int4*)Te1_rc, act, e);
        else if (nT1)
            launch(k_rowblock_batch<T, X, E, true>, nT1, programmatic, (const int*)Tptr, (const int*)Tidx,
                   (const T*)Tval, xin, (const int4*)T1_it, (const int4*)Te1_it, act, e);
        if (nTp) k_pack_spmv<T, X, E><<<nTp, kThreads, 0, s>>>(Tptr, Tidx, Tval, xin, T_it, Te_it, slot_inst, act, e), ++launches;
    }
    void products(const int* act) {
        spmv_A(x, EpiStore<T>{Ax}, act);
        spmv_T(z, EpiStore<T>{ATz}, act);
    }
    void eval_into(double* dst, bool avg, const int* act) {
        const double* fi = avg ? fbuf : nullptr;
        if (!avg) {
            if (nA) k_pack_eval<T, T, true><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, slot_inst, act, fi, Ax, z, rl, ru, nullptr, Dr, zlast, partA);
            if (nT) k_pack_eval<T, T, false><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, act, fi, x, ATz, l, u, c, Dc, xlast, partT);
        } else {
            spmv_A(xs, EpiStore<double>{tmpM}, act);
            spmv_T(zs, EpiStore<double>{tmpN}, act);
            if (nA) k_pack_eval<T, double, true><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, slot_inst, act, fi, tmpM, zs, rl, ru, nullptr, Dr, zlast, partA);
            if (nT) k_pack_eval<T, double, false><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, act, fi, xs, tmpN, l, u, c, Dc, xlast, partT);
        }
        k_eval_finish<<<(ninst + 7) / 8, 256, 0, s>>>(ninst, d_where, rr, cr, partA, partT, act, dst);
        launches += 3;
    }
    // The iteration lists of the running instances only. A stopped instance's CTAs would return at once, but in the
    // tail of a batch they are most of the grid; dropping them changes no result: every running instance keeps all
    // its entries in the same order, and a stopped instance is never touched again. The next block re-captures the
    // graph with the smaller grids.
    void upload_lists(const std::vector<int4>& a1, const std::vector<int4>& ae1, const std::vector<int4>& ap,
                      const std::vector<int4>& ae, const std::vector<int4>& t1, const std::vector<int4>& te1,
                      const std::vector<int4>& tp, const std::vector<int4>& te) {
        auto up = [&](int4* d, const std::vector<int4>& h) {
            if (!h.empty()) BK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
        };
        up(A1_it, a1), up(Ae1_it, ae1), up(A_it, ap), up(Ae_it, ae), up(T1_it, t1), up(Te1_it, te1), up(T_it, tp),
            up(Te_it, te);
        nA1 = int(a1.size()), nAp = int(ap.size()), nT1 = int(t1.size()), nTp = int(tp.size());
        if (graph) {
            BK(cudaGraphExecDestroy(graph));
            graph = nullptr;
        }
    }
    void upload_chunks(const std::vector<int4>& a, const std::vector<int4>& ae, const std::vector<int4>& t,
                       const std::vector<int4>& te) {
        auto up = [&](int4* d, const std::vector<int4>& h) {
            if (!h.empty()) BK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
        };
        up(A1_rc, a), up(Ae1_rc, ae), up(T1_rc, t), up(Te1_rc, te);
        nA1r = int(a.size()), nT1r = int(t.size());
    }
    void compact_lists(const std::vector<int>& live) {
        auto pick = [&](const std::vector<int4>& blk, const std::vector<int4>& ext, bool one, std::vector<int4>& ob,
                        std::vector<int4>& oe) {
            ob.clear(), oe.clear();
            for (size_t k = 0; k < blk.size(); ++k) {
                bool keep = false;
                if (one) {
                    keep = live[size_t(ext[k].x)] != 0;
                } else {
                    const Pack& q = packs[size_t(ext[k].x)];
                    for (int t = 0; t < q.W; ++t) keep = keep || (q.inst[t] >= 0 && live[size_t(q.inst[t])] != 0);
                }
                if (keep) ob.push_back(blk[k]), oe.push_back(ext[k]);
            }
        };
        pick(h_a1, h_ae1, true, c_a1, c_ae1), pick(h_ap, h_ae, false, c_ap, c_ae);
        pick(h_t1, h_te1, true, c_t1, c_te1), pick(h_tp, h_te, false, c_tp, c_te);
        pick(h_a1r, h_ae1r, true, c_a1r, c_ae1r), pick(h_t1r, h_te1r, true, c_t1r, c_te1r);
        upload_lists(c_a1, c_ae1, c_ap, c_ae, c_t1, c_te1, c_tp, c_te);
        upload_chunks(c_a1r, c_ae1r, c_t1r, c_te1r);
        compacted = true;
    }
    void restore_lists() {
        if (!compacted) return;
        upload_lists(h_a1, h_ae1, h_ap, h_ae, h_t1, h_te1, h_tp, h_te);
        upload_chunks(h_a1r, h_ae1r, h_t1r, h_te1r);
        compacted = false;
    }

    void block(int steps) {
        if (nT) k_pack_xupd<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, running, x, ATz, c, l, u, par, xs), ++launches;
        for (int k = 0; k < steps; ++k) {
            spmv_A(x, EpiRow<T>{Ax, z, zs, rl, ru, par}, running, pdl);
            spmv_T(z, EpiCol<T>{ATz, x, xs, c, l, u, par, k + 1 < steps ? 1 : 0}, running, pdl);
        }
        int g = (ninst + 255) / 256;
        k_advance<<<g, 256, 0, s>>>(ninst, st, steps);
        k_gather_f<<<g, 256, 0, s>>>(ninst, st, fbuf);
        eval_into(kkt, false, running);
        eval_into(kkt + 10 * size_t(ninst), true, running);
        k_decide<T><<<g, 256, 0, s>>>(ninst, st, kkt, kkt + 10 * size_t(ninst), par, running, rflag, opt.tol,
                                      opt.row_rel, (long long)opt.max_iter, d_deadline, d_cancel);
        if (nT) k_pack_restart<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, rflag, st, x, xs, xlast);
        if (nA) k_pack_restart<T><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, slot_inst, rflag, st, z, zs, zlast);
        products(rflag);
        k_count<<<1, 256, 0, s>>>(ninst, running, count);
        launches += 7;
    }

    void cancel() override {
        if (h_cancel) __atomic_store_n(h_cancel, 1, __ATOMIC_SEQ_CST);
    }

    int solve(const double* const* x0, const double* const* y0, const double* w0, taral_outcome* outs,
              double* const* xo, double* const* yo) override {
        auto t0 = Clock::now();
        restore_lists();  // a previous solve may have left the lists compacted
        cudaEvent_t e0, e1;
        BK(cudaEventCreate(&e0));
        BK(cudaEventCreate(&e1));
        BK(cudaEventRecord(e0, s));
        // power iteration per instance (gpu/pdhg.cu:416-436)
        std::vector<double> h(N);
        for (int i = 0; i < ninst; ++i) {
            int n = models[i]->n;
            double nn = 0;
            std::vector<double> v0(static_cast<size_t>(n));
            for (int j = 0; j < n; ++j) v0[j] = 0.5 + double((uint32_t(j) * 2654435761u) % 1000u) / 1000.0;
            for (int j = 0; j < n; ++j) nn += v0[j] * v0[j];
            for (int j = 0; j < n; ++j) h[xidx(i, j)] = v0[j] / std::sqrt(nn);
        }
        BK(cudaMemcpyAsync(dout, h.data(), size_t(N) * sizeof(double), cudaMemcpyHostToDevice, s));
        k_cast<T><<<std::max(1, std::min((N + 255) / 256, 1184)), 256, 0, s>>>(N, dout, pv);
        // One estimate per distinct matrix: instances that share a matrix share its scaled copy, its row blocks and
        // the deterministic start vector, so their power iterations are the same numbers; only the first instance
        // of each matrix iterates, the others take its estimate.
        std::vector<int> rep(mats.size(), -1), first(static_cast<size_t>(ninst), 0);
        for (int i = 0; i < ninst; ++i)
            if (rep[size_t(mat_of[i])] < 0) rep[size_t(mat_of[i])] = i, first[size_t(i)] = 1;
        BK(cudaMemcpyAsync(pactive, first.data(), ninst * sizeof(int), cudaMemcpyHostToDevice, s));
        BK(cudaMemsetAsync(est, 0, ninst * sizeof(double), s));
        T *a = pv, *b = pu;
        int g = (ninst + 255) / 256;
        for (int it = 0; it < 200;) {
            int end = std::min(200, it + 8);
            for (; it < end; ++it) {
                spmv_A(a, EpiStore<T>{pw}, pactive);
                spmv_T(pw, EpiStore<T>{b}, pactive);
                if (nT) k_pack_pow_part<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, pactive, b, partT);
                k_pow_update<<<g, 256, 0, s>>>(ninst, d_where, cr, partT, est, pscale, pactive, it);
                if (nT) k_pack_pow_scale<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, pactive, pscale, b);
                launches += 3;
                std::swap(a, b);
            }
            k_count<<<1, 256, 0, s>>>(ninst, pactive, count);
            BK(cudaMemcpyAsync(h_count, count, sizeof(int), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            if (*h_count == 0) break;
        }
        std::vector<double> norms(ninst);
        BK(cudaMemcpyAsync(norms.data(), est, ninst * sizeof(double), cudaMemcpyDeviceToHost, s));
        BK(cudaStreamSynchronize(s));
        for (int i = 0; i < ninst; ++i) norms[size_t(i)] = norms[size_t(rep[size_t(mat_of[i])])];
        double power_s = since(t0);
        // step sizes and state (gpu/pdhg.cu:767-781)
        std::vector<InstState> hs(ninst);
        std::vector<double> hpar(2 * size_t(ninst));
        for (int i = 0; i < ninst; ++i) {
            const Scaled& v = vecs[i];
            StepScale sc = initial_steps(norms[i], v.c.data(), v.n, v.rl.data(), v.ru.data(), v.m);
            if (w0 && std::isfinite(w0[i]) && w0[i] > 0) sc.weight = w0[i];  // caller's initial primal weight
            InstState& q = hs[i];
            std::memset(&q, 0, sizeof q);
            q.sch.weight = sc.weight, q.sch.eta = sc.eta;  // anchor and previous: k_kkt_init, on the start point
            q.norm = norms[i];
            q.bnorm = v.bnorm, q.cnorm = v.cnorm, q.running = 1, q.status = TARAL_ITERATION_LIMIT;
            q.best_p = q.best_d = q.best_g = kInf;
            hpar[2 * i] = sc.eta / sc.weight, hpar[2 * i + 1] = sc.eta * sc.weight;
        }
        BK(cudaMemcpyAsync(st, hs.data(), ninst * sizeof(InstState), cudaMemcpyHostToDevice, s));
        BK(cudaMemcpyAsync(par, hpar.data(), hpar.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        const std::vector<int> ones(static_cast<size_t>(ninst), 1);
        BK(cudaMemcpyAsync(running, ones.data(), ninst * sizeof(int), cudaMemcpyHostToDevice, s));
        // start point (gpu/pdhg.cu:450-458), cold or warm per instance
        k_start_x<T><<<std::max(1, std::min((N + 255) / 256, 1184)), 256, 0, s>>>(N, l, u, x, xlast, xs);
        k_zero_point<T><<<std::max(1, std::min((M + 255) / 256, 1184)), 256, 0, s>>>(M, z, zlast, zs);
        bool warm = false;
        std::vector<double> wx, wy;
        for (int i = 0; i < ninst && !warm; ++i) warm = (x0 && x0[i]) || (y0 && y0[i]);
        if (warm) {
            std::vector<T> hx(N), hz(M);
            BK(cudaMemcpyAsync(hx.data(), x, N * sizeof(T), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            std::fill(hz.begin(), hz.end(), T(0));
            for (int i = 0; i < ninst; ++i) {
                const Shared& sh = *mats[mat_of[i]];
                if (x0 && x0[i])
                    for (int j = 0; j < models[i]->n; ++j) hx[xidx(i, j)] = T(x0[i][j] / sh.S.Dc[j]);
                if (y0 && y0[i])
                    for (int r = 0; r < models[i]->m; ++r) hz[zidx(i, r)] = T(y0[i][r] / sh.S.Dr[r]);
            }
            BK(cudaMemcpyAsync(x, hx.data(), N * sizeof(T), cudaMemcpyHostToDevice, s));
            BK(cudaMemcpyAsync(xlast, hx.data(), N * sizeof(T), cudaMemcpyHostToDevice, s));
            BK(cudaMemcpyAsync(z, hz.data(), M * sizeof(T), cudaMemcpyHostToDevice, s));
            BK(cudaMemcpyAsync(zlast, hz.data(), M * sizeof(T), cudaMemcpyHostToDevice, s));
            BK(cudaStreamSynchronize(s));
        }
        products(running);
        eval_into(kkt, false, running);
        k_kkt_init<<<g, 256, 0, s>>>(ninst, st, kkt);
        launches += 3;
        // the deadline on the device clock (%globaltimer, ns), read by k_decide from device memory so that the
        // captured graph serves every solve
        double left = std::min(std::max(opt.time_limit - since(t0), 0.0), 1e9);
        k_set_deadline<<<1, 1, 0, s>>>(d_deadline, (unsigned long long)(left * 1e9));
        ++launches;
        int64_t it = 0;
        // TARAL_COMPACT=0 keeps the full iteration lists; TARAL_TRACE=1 prints the running count per block
        const char* ce = std::getenv("TARAL_COMPACT");
        const bool compact = !(ce && std::atoi(ce) == 0);
        const bool trace = std::getenv("TARAL_TRACE") != nullptr;
        int live_lists = ninst;  // running instances when the lists were last built
        std::vector<int> live(static_cast<size_t>(ninst));
        // One graph launch runs `per_launch` blocks of eval_freq iterations (TARAL_BATCH_BLOCKS, default 4): the
        // decisions, restarts, the cancel flag and the deadline are all taken on the device after every block, and
        // the kernels of stopped instances return at once, so the host only reads the running count (and compacts
        // the iteration lists) between launches.
        const char* pb = std::getenv("TARAL_BATCH_BLOCKS");
        const int per_launch = std::max(1, std::min(64, pb ? std::atoi(pb) : 4));
        for (;;) {
            const int64_t left = opt.max_iter - it;
            if (left <= 0) break;
            if (opt.graph && left >= int64_t(freq) * per_launch) {
                if (!graph) {
                    cudaGraph_t gr;
                    int64_t before = launches;
                    BK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                    for (int q = 0; q < per_launch; ++q) block(freq);
                    BK(cudaStreamEndCapture(s, &gr));
                    BK(cudaGraphInstantiate(&graph, gr, 0));
                    BK(cudaGraphDestroy(gr));
                    per_graph = launches - before;
                }
                BK(cudaGraphLaunch(graph, s));
                launches += per_graph;
                it += int64_t(freq) * per_launch;
            } else {
                const int steps = int(std::min<int64_t>(freq, left));
                block(steps);
                it += steps;
            }
            BK(cudaMemcpyAsync(h_count, count, sizeof(int), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            if (trace) std::fprintf(stderr, "batch block it=%lld running=%d t=%.4f\n", (long long)it, *h_count, since(t0));
            if (*h_count == 0) break;
            if (compact && 4 * int64_t(*h_count) <= 3 * int64_t(live_lists)) {
                BK(cudaMemcpyAsync(live.data(), running, size_t(ninst) * sizeof(int), cudaMemcpyDeviceToHost, s));
                BK(cudaStreamSynchronize(s));
                compact_lists(live);
                live_lists = *h_count;
            }
        }
        BK(cudaGetLastError());
        // download
        std::vector<InstState> fin(ninst);
        BK(cudaMemcpyAsync(fin.data(), st, ninst * sizeof(InstState), cudaMemcpyDeviceToHost, s));
        std::vector<double> hx(N), hz(M);
        if (nT) k_pack_out<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, slot_inst, st, x, xs, dout);
        BK(cudaMemcpyAsync(hx.data(), dout, N * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (nA) k_pack_out<T><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, slot_inst, st, z, zs, dout);
        BK(cudaMemcpyAsync(hz.data(), dout, M * sizeof(double), cudaMemcpyDeviceToHost, s));
        BK(cudaEventRecord(e1, s));
        BK(cudaStreamSynchronize(s));
        launches += 2;
        float ms = 0;
        BK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0), cudaEventDestroy(e1);
        double solve_s = since(t0);
        const auto tf = Clock::now();
        // original-space check of every instance (independent: spread over the host threads)
        std::atomic<int> next{0};
        auto finish_one = [&](int i) {
            const InstState& q = fin[i];
            const Shared& sh = *mats[mat_of[i]];
            Outcome r;
            r.status = q.status, r.iterations = q.sch.iterations, r.restarts = q.sch.restarts;
            r.from_average = q.avg_final != 0;
            r.rel_primal = q.best_p, r.rel_dual = q.best_d, r.rel_gap = q.best_g, r.norm_a = q.norm;
            r.omega = q.sch.weight;
            r.x.resize(size_t(models[i]->n)), r.z.resize(size_t(models[i]->m));
            for (int j = 0; j < models[i]->n; ++j) r.x[j] = hx[xidx(i, j)];
            for (int q = 0; q < models[i]->m; ++q) r.z[q] = hz[zidx(i, q)];
            Scaled P;  // finish_point needs Dr, Dc and sizes
            P.m = models[i]->m, P.n = models[i]->n, P.Dr = sh.S.Dr, P.Dc = sh.S.Dc;
            Finished f = finish_point(*models[i], P, r);
            taral_outcome& o = outs[i];
            std::memset(&o, 0, sizeof o);
            o.status = r.status, o.iterations = r.iterations, o.restarts = r.restarts, o.from_average = r.from_average;
            o.rel_primal = r.rel_primal, o.rel_dual = r.rel_dual, o.rel_gap = r.rel_gap, o.norm_a = r.norm_a;
            o.primal_weight = r.omega, o.objective = f.objective, o.max_row_violation = f.max_row_violation;
            o.max_bound_violation = f.max_bound_violation, o.solve_s = solve_s, o.power_iter_s = power_s;
            o.device_mem_bytes = mem_used, o.kernel_launches = launches, o.nnz = sh.nnz;
            o.device_s = ms * 1e-3;
            if (xo && xo[i]) std::memcpy(xo[i], f.x.data(), f.x.size() * sizeof(double));
            if (yo && yo[i]) std::memcpy(yo[i], f.y.data(), f.y.size() * sizeof(double));
        };
        std::vector<std::thread> pool;
        const int nt = std::max(1, std::min(host_threads(), ninst));
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                for (int i = next++; i < ninst; i = next++) finish_one(i);
            });
        for (auto& th : pool) th.join();
        if (std::getenv("TARAL_TIMING"))
            std::fprintf(stderr, "taral: batch solve: power %.3f s, to the download %.3f s, check %.3f s, device %.3f s\n",
                         power_s, solve_s, since(tf), ms * 1e-3);
        __atomic_store_n(h_cancel, 0, __ATOMIC_SEQ_CST);  // a request applies to one solve
        for (int i = 0; i < ninst; ++i)
            if (fin[size_t(i)].status == TARAL_CANCELLED) return TARAL_ERR_CANCELLED;
        return TARAL_OK;
    }
    int64_t per_graph = 0;
};

}  // namespace taral

// ================================================================================================ C ABI
struct taral_batch {
    std::unique_ptr<taral::BatchBase> b;
};

extern "C" int taral_batch_create(const taral_model* models, int count, const taral_options* o, taral_batch** out) {
    if (!models || count <= 0 || !o || !out) return TARAL_ERR_INPUT;
    *out = nullptr;
    for (int i = 0; i < count; ++i) {
        if (taral::input_error(models[i])) return TARAL_ERR_UNSUPPORTED;
        if (!taral::check_model(models[i]).empty()) return TARAL_ERR_INPUT;
    }
    int dev = 0;
    if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) return TARAL_ERR_NO_DEVICE;
    taral::Options op;
    op.tol = o->tol, op.time_limit = o->time_limit, op.max_iter = o->max_iter;
    op.eval_freq = o->eval_freq > 0 ? o->eval_freq : 64, op.row_rel = o->row_rel, op.graph = o->graph != 0;
    op.precision = o->precision == TARAL_FP32 ? TARAL_FP32 : TARAL_FP64;
    auto* h = new taral_batch;
    try {
        if (op.precision == TARAL_FP32) {
            auto p = std::make_unique<taral::Batch<float>>();
            p->build(models, count, op);
            h->b = std::move(p);
        } else {
            auto p = std::make_unique<taral::Batch<double>>();
            p->build(models, count, op);
            h->b = std::move(p);
        }
    } catch (const taral::BatchError& e) {
        delete h;
        return e.msg.find("cudaMalloc") != std::string::npos ? TARAL_ERR_ALLOC : TARAL_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        delete h;
        return TARAL_ERR_ALLOC;
    }
    *out = h;
    return TARAL_OK;
}

extern "C" int taral_batch_solve(taral_batch* h, const double* const* x0, const double* const* y0,
                                 const double* w0, taral_outcome* outs, double* const* x_out, double* const* y_out) {
    if (!h || !outs) return TARAL_ERR_INPUT;
    try {
        return h->b->solve(x0, y0, w0, outs, x_out, y_out);
    } catch (const taral::BatchError& e) {
        h->b->err = e.msg;
        return TARAL_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        return TARAL_ERR_ALLOC;
    }
}

extern "C" int taral_batch_cancel(taral_batch* h) {
    if (!h || !h->b) return TARAL_ERR_INPUT;
    h->b->cancel();
    return TARAL_OK;
}

extern "C" int taral_batch_info(const taral_batch* h, int* distinct, size_t* mem, int64_t* nnz_stored,
                                int64_t* nnz_total) {
    if (!h) return TARAL_ERR_INPUT;
    if (distinct) *distinct = h->b->distinct;
    if (mem) *mem = h->b->mem_used;
    if (nnz_stored) *nnz_stored = h->b->nnz_stored;
    if (nnz_total) *nnz_total = h->b->nnz_total;
    return TARAL_OK;
}

extern "C" const char* taral_batch_last_error(const taral_batch* h) { return h ? h->b->err.c_str() : "NULL batch"; }
extern "C" void taral_batch_destroy(taral_batch* h) { delete h; }
