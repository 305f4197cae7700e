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
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/taral_pdhg.h"
#include "engine.hpp"
#include "host.hpp"
#include "kernels.cuh"
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

// Per-instance driver state (device resident, FP64 where the reference uses double).
struct InstState {
    double w, eta, k_last, k_prev, f, f_restart, bnorm, cnorm, best_p, best_d, best_g, norm;
    long long it, n_since;
    int status, restarts, avg_final, running, restart_flag, pad;
};

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }  // std::max semantics
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }  // std::min semantics

// ---------------------------------------------------------------------------------------------- batch kernels
// Per-block partial sums of the row (ROW = true) or column KKT scalars, blocks in evaluation order.
// Row part (gpu/pdhg.cu:236-251), column part (:253-271); f per instance (1 for the current point).
template <class T, class V, bool ROW>
__global__ void __launch_bounds__(kThreads) k_eval_blocks(const int4* __restrict__ blk, const int4* __restrict__ ext,
                                                          const int* __restrict__ active, const double* __restrict__ fi,
                                                          const V* __restrict__ a, const V* __restrict__ b,
                                                          const T* __restrict__ lo_v, const T* __restrict__ up_v,
                                                          const T* __restrict__ c_v, const T* __restrict__ D,
                                                          const T* __restrict__ last, double* part) {
    const int4 e4 = ext[blockIdx.x];
    if (!active[e4.x]) return;
    const int4 meta = blk[blockIdx.x];
    const int nrows = meta.y & 0xffff, r = meta.x + e4.y + threadIdx.x;
    const double f = fi ? fi[e4.x] : 1.0;
    double v[5] = {0, 0, 0, 0, 0};
    if (int(threadIdx.x) < nrows) {
        if (ROW) {  // a = Ax (or A xs), b = z (or zs)
            double ax = double(a[r]) * f, zz = double(b[r]) * f, lo = lo_v[r], up = up_v[r];
            double res = ax < lo ? lo - ax : (ax > up ? ax - up : 0), ro = res / double(D[r]);
            double rr = ro * row_rel_weight(lo, up, double(D[r]));
            v[0] = res * res, v[1] = ro * ro, v[2] = rr * rr;
            if (zz > 0 && up < INFINITY) v[3] -= zz * up;
            if (zz < 0 && lo > -INFINITY) v[3] -= zz * lo;
            double dz = zz - double(last[r]);
            v[4] = dz * dz;
        } else {  // a = x (or xs), b = ATz (or A^T zs); c_v = c, lo_v = l, up_v = u
            double xx = double(a[r]) * f, cj = c_v[r], d = cj + double(b[r]) * f, lo = lo_v[r], up = up_v[r], res = 0;
            v[2] = cj * xx;
            if (d > 0) {
                if (lo > -INFINITY) v[3] = d * lo;
                else res = d;
            } else if (d < 0) {
                if (up < INFINITY) v[3] = d * up;
                else res = -d;
            }
            double ro = res / double(D[r]), dx = xx - double(last[r]);
            v[0] = res * res, v[1] = ro * ro, v[4] = dx * dx;
        }
    }
    __shared__ double sh[5][kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double s = v[k];
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) sh[k][w] = s;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double s = 0;
        for (int i = 0; i < kThreads / 32; ++i) s += sh[threadIdx.x][i];
        part[size_t(blockIdx.x) * 5 + threadIdx.x] = s;
    }
}

// One warp per instance: kkt[inst*10 + k] = sum of its blocks' partials, in block order (deterministic).
__global__ void k_eval_finish(int ninst, const int* __restrict__ rr, const int* __restrict__ cr,
                              const double* __restrict__ prow, const double* __restrict__ pcol,
                              const int* __restrict__ active, double* kkt) {
    const int inst = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (inst >= ninst || !active[inst] || lane >= 10) return;
    double s = 0;
    if (lane < 5)
        for (int b = rr[inst]; b < rr[inst + 1]; ++b) s += prow[size_t(b) * 5 + lane];
    else
        for (int b = cr[inst]; b < cr[inst + 1]; ++b) s += pcol[size_t(b) * 5 + lane - 5];
    kkt[inst * 10 + lane] = s;
}

__device__ __forceinline__ double wkkt(const double* k, double w) {
    double g = k[POBJ] - (k[DROW] + k[DCOL]);
    return sqrt(w * k[PR2S] + k[DR2S] / w + g * g);
}

// The per-block decision of gpu/pdhg.cu:806-842 for every running instance (one thread each).
template <class T>
__global__ void k_decide(int ninst, InstState* st, const double* __restrict__ kc_all, const double* __restrict__ ka_all,
                         double* par, int* running, int* rflag, double tol, double row_rel, long long max_iter,
                         const unsigned long long* deadline) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst) return;
    rflag[i] = 0;
    InstState& s = st[i];
    if (!s.running) return;
    const double* kc = kc_all + 10 * i;
    const double* ka = ka_all + 10 * i;
    auto rel = [&](const double* k, double& p, double& d, double& g) {
        double po = k[POBJ], du = k[DROW] + k[DCOL];
        double prow = row_rel > 0 ? sqrt(k[PR2R]) / row_rel : 0;
        p = dmax(sqrt(k[PR2O]) / (1 + s.bnorm), prow), d = sqrt(k[DR2O]) / (1 + s.cnorm);
        g = fabs(po - du) / (1 + fabs(po) + fabs(du));
    };
    double cp, cd, cg, ap, ad, ag;
    rel(kc, cp, cd, cg), rel(ka, ap, ad, ag);
    double wc_ = dmax(cp, dmax(cd, cg)), wa_ = dmax(ap, dmax(ad, ag));
    bool use_avg = wa_ < wc_;
    s.best_p = use_avg ? ap : cp, s.best_d = use_avg ? ad : cd, s.best_g = use_avg ? ag : cg;
    s.avg_final = use_avg;
    double best = use_avg ? wa_ : wc_;
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    if (!isfinite(wc_) && !isfinite(wa_)) s.status = TARAL_NUMERICAL_FAILURE, s.running = 0;
    else if (best <= tol) s.status = TARAL_NEAR_OPTIMAL, s.running = 0;
    else if (*deadline && now > *deadline) s.status = TARAL_TIME_LIMIT, s.running = 0;
    else if (s.it >= max_iter) s.status = TARAL_ITERATION_LIMIT, s.running = 0;
    if (!s.running) {
        running[i] = 0;
        return;
    }
    double w = s.w, wc = wkkt(kc, w), wa = wkkt(ka, w);
    bool cand_avg = wa < wc;
    const double* kk = cand_avg ? ka : kc;
    double kcand = dmin(wa, wc);
    bool restart = double(s.n_since) >= 0.36 * double(s.it) || kcand <= 0.2 * s.k_last ||
                   (kcand <= 0.8 * s.k_last && kcand > s.k_prev);
    s.k_prev = kcand;
    if (restart) {
        double dx = sqrt(kk[DX2]), dz = sqrt(kk[DZ2]);
        rflag[i] = cand_avg ? 2 : 1;
        s.f_restart = s.f;
        if (dx > 1e-10 && dz > 1e-10) {
            w = exp(0.5 * log(dz / dx) + 0.5 * log(w));
            s.w = w;
            par[2 * i] = s.eta / w, par[2 * i + 1] = s.eta * w;
        }
        s.k_last = wkkt(kk, w), s.k_prev = INFINITY, s.n_since = 0, s.restarts++;
    }
}

__global__ void k_advance(int ninst, InstState* st, int steps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst || !st[i].running) return;
    st[i].it += steps, st[i].n_since += steps;
    st[i].f = 1.0 / double(st[i].n_since);
}

// Gather the per-instance f (running sums scale) into a flat array for the evaluation kernels.
__global__ void k_gather_f(int ninst, const InstState* st, double* f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ninst) f[i] = st[i].f;
}

// First primal step of the block for every running instance, over column blocks (rows of A^T).
template <class T>
__global__ void k_xupd_blocks(const int4* __restrict__ blk, const int4* __restrict__ ext, const int* __restrict__ active,
                              T* __restrict__ x, const T* __restrict__ ATz, const T* __restrict__ c,
                              const T* __restrict__ l, const T* __restrict__ u, const double* __restrict__ par,
                              double* __restrict__ xs) {
    const int4 e4 = ext[blockIdx.x];
    if (!active[e4.x]) return;
    const int4 meta = blk[blockIdx.x];
    const int nrows = meta.y & 0xffff;
    if (int(threadIdx.x) >= nrows) return;
    const int j = meta.x + e4.y + threadIdx.x;
    const T xn = T(clampv(double(x[j]) - par[2 * e4.x] * (double(c[j]) + double(ATz[j])), double(l[j]), double(u[j])));
    x[j] = xn, xs[j] += double(xn);
}

// Restart of the flagged instances (gpu/pdhg.cu:293-299): flag 2 -> average * f, 1 -> current point.
template <class T>
__global__ void k_restart_blocks(const int4* __restrict__ blk, const int4* __restrict__ ext, const int* __restrict__ flag,
                                 const InstState* __restrict__ st, T* __restrict__ x, double* __restrict__ xs,
                                 T* __restrict__ xlast) {
    const int4 e4 = ext[blockIdx.x];
    const int fl = flag[e4.x];
    if (!fl) return;
    const int4 meta = blk[blockIdx.x];
    const int nrows = meta.y & 0xffff;
    if (int(threadIdx.x) >= nrows) return;
    const int j = meta.x + e4.y + threadIdx.x;
    T v = fl == 2 ? T(xs[j] * st[e4.x].f_restart) : x[j];
    x[j] = v, xlast[j] = v, xs[j] = 0;
}

// Per-instance power-iteration step over column blocks: partial ||v||^2, then one thread per instance.
template <class T>
__global__ void k_pow_part(const int4* __restrict__ blk, const int4* __restrict__ ext, const int* __restrict__ active,
                           const T* __restrict__ v, double* part) {
    const int4 e4 = ext[blockIdx.x];
    if (!active[e4.x]) return;
    const int4 meta = blk[blockIdx.x];
    const int nrows = meta.y & 0xffff;
    double a = 0;
    if (int(threadIdx.x) < nrows) {
        double t = double(v[meta.x + e4.y + threadIdx.x]);
        a = t * t;
    }
    for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
    __shared__ double sh[kThreads / 32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < kThreads / 32; ++i) s += sh[i];
        part[blockIdx.x] = s;
    }
}

__global__ void k_pow_update(int ninst, const int* __restrict__ cr, const double* __restrict__ part, double* est,
                             double* scale, int* active, int it) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst || !active[i]) return;
    double s = 0;
    for (int b = cr[i]; b < cr[i + 1]; ++b) s += part[b];
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
__global__ void k_pow_scale(const int4* __restrict__ blk, const int4* __restrict__ ext, const int* __restrict__ active,
                            const double* __restrict__ scale, T* __restrict__ v) {
    const int4 e4 = ext[blockIdx.x];
    if (!active[e4.x]) return;
    const int4 meta = blk[blockIdx.x];
    if (int(threadIdx.x) >= (meta.y & 0xffff)) return;
    const int j = meta.x + e4.y + threadIdx.x;
    v[j] = T(double(v[j]) * scale[e4.x]);
}

// Download: out = (avg ? sum * f : point) for each instance's range.
template <class T>
__global__ void k_out_blocks(const int4* __restrict__ blk, const int4* __restrict__ ext, const InstState* __restrict__ st,
                             const T* __restrict__ x, const double* __restrict__ xs, double* __restrict__ out) {
    const int4 e4 = ext[blockIdx.x];
    const int4 meta = blk[blockIdx.x];
    if (int(threadIdx.x) >= (meta.y & 0xffff)) return;
    const int j = meta.x + e4.y + threadIdx.x;
    const InstState& s = st[e4.x];
    out[j] = s.avg_final ? xs[j] * (1.0 / double(s.n_since > 1 ? s.n_since : 1)) : double(x[j]);
}

__global__ void k_kkt_init(int ninst, InstState* st, const double* __restrict__ kc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst) return;
    st[i].k_last = wkkt(kc + 10 * i, st[i].w), st[i].k_prev = INFINITY;
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
    Scaled S;    // matrix part only (A, AT, Dr, Dc)
    std::vector<int4> blkA, blkT;
    int pbaseA = 0, pbaseT = 0;
    int64_t nnzbase = 0;
};

uint64_t fnv(const void* p, size_t n, uint64_t h) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

}  // namespace

struct BatchBase {
    virtual ~BatchBase() = default;
    virtual void solve(const double* const* x0, const double* const* y0, const double* w0, taral_outcome* outs,
                       double* const* xo,
                       double* const* yo) = 0;
    std::string err;
    int distinct = 0;
    size_t mem_used = 0;
    int64_t nnz_stored = 0, nnz_total = 0, launches = 0;
};

template <class T>
struct Batch final : BatchBase {
    int ninst = 0, M = 0, N = 0, nA = 0, nT = 0, freq = 64;
    Options opt;
    std::vector<const taral_model*> models;
    std::vector<int> mat_of;                 // instance -> distinct matrix
    std::vector<std::unique_ptr<Shared>> mats;
    std::vector<Scaled> vecs;                // per instance: vector part
    std::vector<int> row_off, col_off;
    // device
    int *Aptr = nullptr, *Aidx = nullptr, *Tptr = nullptr, *Tidx = nullptr;
    T *Aval = nullptr, *Tval = nullptr;
    int4 *A_it = nullptr, *Ae_it = nullptr, *T_it = nullptr, *Te_it = nullptr;
    int4 *A_ev = nullptr, *Ae_ev = nullptr, *T_ev = nullptr, *Te_ev = nullptr;
    int *rr = nullptr, *cr = nullptr;
    T *c = nullptr, *l = nullptr, *u = nullptr, *Dc = nullptr, *rl = nullptr, *ru = nullptr, *Dr = nullptr;
    double* par = nullptr;  // per instance {tau, sigma}
    T *x = nullptr, *ATz = nullptr, *xlast = nullptr, *z = nullptr, *Ax = nullptr, *zlast = nullptr;
    T *pv = nullptr, *pu = nullptr, *pw = nullptr;
    double *xs = nullptr, *zs = nullptr, *tmpM = nullptr, *tmpN = nullptr, *partA = nullptr, *partT = nullptr;
    double *kkt = nullptr, *fbuf = nullptr, *est = nullptr, *pscale = nullptr, *dout = nullptr;
    InstState* st = nullptr;
    unsigned long long* d_deadline = nullptr;
    int *running = nullptr, *rflag = nullptr, *pactive = nullptr, *count = nullptr, *h_count = nullptr;
    cudaStream_t s = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<void*> allocs;

    template <class U>
    U* alloc(size_t n) {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(U));
        if (e != cudaSuccess) throw BatchError{std::string("cudaMalloc: ") + cudaGetErrorString(e)};
        allocs.push_back(p);
        return static_cast<U*>(p);
    }
    template <class U>
    U* put(const std::vector<U>& h) {
        U* p = alloc<U>(h.size());
        if (!h.empty()) BK(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(U), cudaMemcpyHostToDevice, s));
        BK(cudaStreamSynchronize(s));
        return p;
    }
    ~Batch() override {
        if (graph) cudaGraphExecDestroy(graph);
        if (s) cudaStreamSynchronize(s);
        for (void* p : allocs) cudaFree(p);
        if (h_count) cudaFreeHost(h_count);
        if (s) cudaStreamDestroy(s);
    }

    void build(const taral_model* md, int count, const Options& o) {
        ninst = count, opt = o, freq = std::max(1, o.eval_freq);
        size_t free0, free1, total;
        BK(cudaMemGetInfo(&free0, &total));
        BK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        // 1. distinct matrices (same sizes and identical col_ptr / row_idx / val)
        std::map<std::pair<uint64_t, std::pair<int, int>>, int> seen;
        mat_of.resize(count);
        for (int i = 0; i < count; ++i) {
            const taral_model& m = md[i];
            int64_t nz = m.col_ptr[m.n];
            uint64_t h = 1469598103934665603ull;
            h = fnv(m.col_ptr, size_t(m.n + 1) * sizeof(int64_t), h);
            h = fnv(m.row_idx, size_t(nz) * sizeof(int32_t), h);
            h = fnv(m.val, size_t(nz) * sizeof(double), h);
            auto key = std::make_pair(h, std::make_pair(m.m, m.n));
            auto it = seen.find(key);
            bool same = false;
            if (it != seen.end()) {  // confirm byte equality against the first instance with this hash
                const taral_model& r = md[first_inst[it->second]];
                same = r.m == m.m && r.n == m.n && r.col_ptr[r.n] == nz &&
                       !std::memcmp(r.col_ptr, m.col_ptr, size_t(m.n + 1) * sizeof(int64_t)) &&
                       !std::memcmp(r.row_idx, m.row_idx, size_t(nz) * sizeof(int32_t)) &&
                       !std::memcmp(r.val, m.val, size_t(nz) * sizeof(double));
            }
            if (same) {
                mat_of[i] = it->second;
            } else {
                int id = int(mats.size());
                mats.push_back(std::make_unique<Shared>());
                first_inst.push_back(i);
                if (it == seen.end()) seen[key] = id;
                mat_of[i] = id;
            }
        }
        distinct = int(mats.size());
        // 2. scale: matrices (threads), then per-instance vectors
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
            scale_matrix(md[first_inst[k]], sh.S);
            sh.blkA = build_row_blocks(sh.S.A.ptr.data(), sh.S.A.rows);
            sh.blkT = build_row_blocks(sh.S.AT.ptr.data(), sh.S.AT.rows);
        });
        vecs.resize(count);
        par_for(count, [&](int i) {
            const Shared& sh = *mats[mat_of[i]];
            scale_vectors(md[i], md[i].maximize ? -1.0 : 1.0, sh.S.Dr, sh.S.Dc, vecs[i]);
        });
        // 3. concatenated matrices (int32 offsets)
        std::vector<int> hAptr, hTptr, hAidx, hTidx;
        std::vector<T> hAval, hTval;
        int64_t nzb = 0;
        for (auto& shp : mats) {
            Shared& sh = *shp;
            sh.pbaseA = int(hAptr.size()), sh.pbaseT = int(hTptr.size()), sh.nnzbase = nzb;
            for (int64_t v : sh.S.A.ptr) hAptr.push_back(int(v + nzb));
            for (int64_t v : sh.S.AT.ptr) hTptr.push_back(int(v + nzb));
            hAidx.insert(hAidx.end(), sh.S.A.idx.begin(), sh.S.A.idx.end());
            hTidx.insert(hTidx.end(), sh.S.AT.idx.begin(), sh.S.AT.idx.end());
            for (double v : sh.S.A.val) hAval.push_back(T(v));
            for (double v : sh.S.AT.val) hTval.push_back(T(v));
            nzb += int64_t(sh.S.A.val.size());
            if (nzb > INT32_MAX - 64) throw BatchError{"more than 2^31 distinct nonzeros in a batch"};
        }
        nnz_stored = nzb;
        // 4. instance offsets and block lists
        row_off.assign(count + 1, 0), col_off.assign(count + 1, 0);
        for (int i = 0; i < count; ++i) row_off[i + 1] = row_off[i] + md[i].m, col_off[i + 1] = col_off[i] + md[i].n;
        M = row_off[count], N = col_off[count];
        if (int64_t(M) + N > INT32_MAX - 1024) throw BatchError{"batch too large for int32 indexing"};
        std::vector<int4> a_it, ae_it, t_it, te_it, a_ev, ae_ev, t_ev, te_ev;
        std::vector<int> hrr{0}, hcr{0};
        auto shiftA = [&](int i) {
            const Shared& sh = *mats[mat_of[i]];
            return make_int4(i, row_off[i] - sh.pbaseA, col_off[i], 0);
        };
        auto shiftT = [&](int i) {
            const Shared& sh = *mats[mat_of[i]];
            return make_int4(i, col_off[i] - sh.pbaseT, row_off[i], 0);
        };
        auto rebase = [](int4 b, int pbase, int64_t nzbase) {
            return make_int4(b.x + pbase, b.y, int(b.z + nzbase), int(b.w + nzbase));
        };
        for (int i = 0; i < count; ++i) {  // evaluation order: instance-major
            const Shared& sh = *mats[mat_of[i]];
            for (const int4& b : sh.blkA) a_ev.push_back(rebase(b, sh.pbaseA, sh.nnzbase)), ae_ev.push_back(shiftA(i));
            for (const int4& b : sh.blkT) t_ev.push_back(rebase(b, sh.pbaseT, sh.nnzbase)), te_ev.push_back(shiftT(i));
            hrr.push_back(int(a_ev.size())), hcr.push_back(int(t_ev.size()));
        }
        std::vector<std::vector<int>> users(distinct);
        for (int i = 0; i < count; ++i) users[mat_of[i]].push_back(i);
        for (int k = 0; k < distinct; ++k) {  // iteration order: matrix-major, instances interleaved per tile
            const Shared& sh = *mats[k];
            for (const int4& b : sh.blkA)
                for (int i : users[k]) a_it.push_back(rebase(b, sh.pbaseA, sh.nnzbase)), ae_it.push_back(shiftA(i));
            for (const int4& b : sh.blkT)
                for (int i : users[k]) t_it.push_back(rebase(b, sh.pbaseT, sh.nnzbase)), te_it.push_back(shiftT(i));
        }
        nA = int(a_it.size()), nT = int(t_it.size());
        // 5. upload
        Aptr = put(hAptr), Tptr = put(hTptr), Aidx = put(hAidx), Tidx = put(hTidx), Aval = put(hAval), Tval = put(hTval);
        A_it = put(a_it), Ae_it = put(ae_it), T_it = put(t_it), Te_it = put(te_it);
        A_ev = put(a_ev), Ae_ev = put(ae_ev), T_ev = put(t_ev), Te_ev = put(te_ev);
        rr = put(hrr), cr = put(hcr);
        std::vector<T> hc(N), hl(N), hu(N), hDc(N), hrl(M), hru(M), hDr(M);
        for (int i = 0; i < count; ++i) {
            const Scaled& v = vecs[i];
            const Shared& sh = *mats[mat_of[i]];
            for (int j = 0; j < md[i].n; ++j) {
                int g = col_off[i] + j;
                hc[g] = T(v.c[j]), hl[g] = T(v.l[j]), hu[g] = T(v.u[j]), hDc[g] = T(sh.S.Dc[j]);
            }
            for (int r = 0; r < md[i].m; ++r) {
                int g = row_off[i] + r;
                hrl[g] = T(v.rl[r]), hru[g] = T(v.ru[r]), hDr[g] = T(sh.S.Dr[r]);
            }
        }
        c = put(hc), l = put(hl), u = put(hu), Dc = put(hDc), rl = put(hrl), ru = put(hru), Dr = put(hDr);
        x = alloc<T>(N), ATz = alloc<T>(N), xlast = alloc<T>(N), z = alloc<T>(M), Ax = alloc<T>(M), zlast = alloc<T>(M);
        pv = alloc<T>(N), pu = alloc<T>(N), pw = alloc<T>(M);
        xs = alloc<double>(N), zs = alloc<double>(M), tmpM = alloc<double>(M), tmpN = alloc<double>(N);
        dout = alloc<double>(size_t(std::max(M, N)));
        partA = alloc<double>(size_t(std::max(nA, 1)) * 5), partT = alloc<double>(size_t(std::max(nT, 1)) * 5);
        kkt = alloc<double>(size_t(count) * 20), fbuf = alloc<double>(count), est = alloc<double>(count);
        pscale = alloc<double>(count), st = alloc<InstState>(count), par = alloc<double>(2 * size_t(count));
        running = alloc<int>(count), rflag = alloc<int>(count), pactive = alloc<int>(count), this->count = alloc<int>(1);
        d_deadline = alloc<unsigned long long>(1);
        BK(cudaMallocHost(&h_count, sizeof(int)));
        BK(cudaStreamSynchronize(s));
        BK(cudaMemGetInfo(&free1, &total));
        mem_used = free0 - free1;
        nnz_total = 0;
        for (int i = 0; i < count; ++i) nnz_total += int64_t(mats[mat_of[i]]->S.A.val.size());
        models.clear();
        for (int i = 0; i < count; ++i) models.push_back(md + i);
    }
    std::vector<int> first_inst;  // distinct matrix -> first instance that has it

    // ------------------------------------------------------------------ launches
    template <class X, class E>
    void spmv_A(const X* xin, const E& e, const int* act) {
        if (nA) k_rowblock_batch<T, X, E, true><<<nA, kThreads, 0, s>>>(Aptr, Aidx, Aval, xin, A_it, Ae_it, act, e), ++launches;
    }
    template <class X, class E>
    void spmv_T(const X* xin, const E& e, const int* act) {
        if (nT) k_rowblock_batch<T, X, E, true><<<nT, kThreads, 0, s>>>(Tptr, Tidx, Tval, xin, T_it, Te_it, act, e), ++launches;
    }
    void products(const int* act) {
        spmv_A(x, EpiStore<T>{Ax}, act);
        spmv_T(z, EpiStore<T>{ATz}, act);
    }
    void eval_into(double* dst, bool avg, const int* act) {
        const double* fi = avg ? fbuf : nullptr;
        if (!avg) {
            if (nA) k_eval_blocks<T, T, true><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, act, fi, Ax, z, rl, ru, nullptr, Dr, zlast, partA);
            if (nT) k_eval_blocks<T, T, false><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, act, fi, x, ATz, l, u, c, Dc, xlast, partT);
        } else {
            spmv_A(xs, EpiStore<double>{tmpM}, act);
            spmv_T(zs, EpiStore<double>{tmpN}, act);
            if (nA) k_eval_blocks<T, double, true><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, act, fi, tmpM, zs, rl, ru, nullptr, Dr, zlast, partA);
            if (nT) k_eval_blocks<T, double, false><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, act, fi, xs, tmpN, l, u, c, Dc, xlast, partT);
        }
        k_eval_finish<<<(ninst + 7) / 8, 256, 0, s>>>(ninst, rr, cr, partA, partT, act, dst);
        launches += 3;
    }
    void block(int steps) {
        if (nT) k_xupd_blocks<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, running, x, ATz, c, l, u, par, xs), ++launches;
        for (int k = 0; k < steps; ++k) {
            spmv_A(x, EpiRow<T>{Ax, z, zs, rl, ru, par}, running);
            spmv_T(z, EpiCol<T>{ATz, x, xs, c, l, u, par, k + 1 < steps ? 1 : 0}, running);
        }
        int g = (ninst + 255) / 256;
        k_advance<<<g, 256, 0, s>>>(ninst, st, steps);
        k_gather_f<<<g, 256, 0, s>>>(ninst, st, fbuf);
        eval_into(kkt, false, running);
        eval_into(kkt + 10 * size_t(ninst), true, running);
        k_decide<T><<<g, 256, 0, s>>>(ninst, st, kkt, kkt + 10 * size_t(ninst), par, running, rflag, opt.tol,
                                      opt.row_rel, (long long)opt.max_iter, d_deadline);
        if (nT) k_restart_blocks<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, rflag, st, x, xs, xlast);
        if (nA) k_restart_blocks<T><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, rflag, st, z, zs, zlast);
        products(rflag);
        k_count<<<1, 256, 0, s>>>(ninst, running, count);
        launches += 7;
    }

    void solve(const double* const* x0, const double* const* y0, const double* w0, taral_outcome* outs,
               double* const* xo, double* const* yo) override {
        auto t0 = Clock::now();
        cudaEvent_t e0, e1;
        BK(cudaEventCreate(&e0));
        BK(cudaEventCreate(&e1));
        BK(cudaEventRecord(e0, s));
        // power iteration per instance (gpu/pdhg.cu:416-436)
        std::vector<double> h(N);
        for (int i = 0; i < ninst; ++i) {
            int n = models[i]->n;
            double nn = 0;
            for (int j = 0; j < n; ++j) h[col_off[i] + j] = 0.5 + double((uint32_t(j) * 2654435761u) % 1000u) / 1000.0;
            for (int j = 0; j < n; ++j) nn += h[col_off[i] + j] * h[col_off[i] + j];
            for (int j = 0; j < n; ++j) h[col_off[i] + j] = h[col_off[i] + j] / std::sqrt(nn);
        }
        BK(cudaMemcpyAsync(dout, h.data(), size_t(N) * sizeof(double), cudaMemcpyHostToDevice, s));
        k_cast<T><<<std::max(1, std::min((N + 255) / 256, 1184)), 256, 0, s>>>(N, dout, pv);
        std::vector<int> ones(ninst, 1);
        BK(cudaMemcpyAsync(pactive, ones.data(), ninst * sizeof(int), cudaMemcpyHostToDevice, s));
        BK(cudaMemsetAsync(est, 0, ninst * sizeof(double), s));
        T *a = pv, *b = pu;
        int g = (ninst + 255) / 256;
        for (int it = 0; it < 200;) {
            int end = std::min(200, it + 8);
            for (; it < end; ++it) {
                spmv_A(a, EpiStore<T>{pw}, pactive);
                spmv_T(pw, EpiStore<T>{b}, pactive);
                if (nT) k_pow_part<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, pactive, b, partT);
                k_pow_update<<<g, 256, 0, s>>>(ninst, cr, partT, est, pscale, pactive, it);
                if (nT) k_pow_scale<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, pactive, pscale, b);
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
        double power_s = since(t0);
        // step sizes and state (gpu/pdhg.cu:767-781)
        std::vector<InstState> hs(ninst);
        std::vector<double> hpar(2 * size_t(ninst));
        for (int i = 0; i < ninst; ++i) {
            const Scaled& v = vecs[i];
            double cs = 0, bs = 0;
            for (double cv : v.c) cs += cv * cv;
            for (int r = 0; r < v.m; ++r) {
                double lo = v.rl[r], up = v.ru[r];
                double q = std::isfinite(lo) && std::isfinite(up) ? std::max(std::fabs(lo), std::fabs(up))
                           : std::isfinite(lo)                    ? std::fabs(lo)
                           : std::isfinite(up)                    ? std::fabs(up)
                                                                  : 0;
                bs += q * q;
            }
            cs = std::sqrt(cs), bs = std::sqrt(bs);
            InstState& q = hs[i];
            std::memset(&q, 0, sizeof q);
            q.norm = norms[i];
            q.eta = norms[i] > 0 ? 0.95 / norms[i] : 1.0;
            q.w = cs > 1e-10 && bs > 1e-10 ? cs / bs : 1.0;
            if (w0 && std::isfinite(w0[i]) && w0[i] > 0) q.w = w0[i];  // caller's initial primal weight
            q.bnorm = v.bnorm, q.cnorm = v.cnorm, q.running = 1, q.status = TARAL_ITERATION_LIMIT;
            q.best_p = q.best_d = q.best_g = kInf;
            hpar[2 * i] = q.eta / q.w, hpar[2 * i + 1] = q.eta * q.w;
        }
        BK(cudaMemcpyAsync(st, hs.data(), ninst * sizeof(InstState), cudaMemcpyHostToDevice, s));
        BK(cudaMemcpyAsync(par, hpar.data(), hpar.size() * sizeof(double), cudaMemcpyHostToDevice, s));
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
                    for (int j = 0; j < models[i]->n; ++j) hx[col_off[i] + j] = T(x0[i][j] / sh.S.Dc[j]);
                if (y0 && y0[i])
                    for (int r = 0; r < models[i]->m; ++r) hz[row_off[i] + r] = T(y0[i][r] / sh.S.Dr[r]);
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
        for (;;) {
            int steps = int(std::min<int64_t>(freq, opt.max_iter - it));
            if (steps <= 0) break;
            if (steps == freq && opt.graph) {
                if (!graph) {
                    cudaGraph_t gr;
                    int64_t before = launches;
                    BK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                    block(steps);
                    BK(cudaStreamEndCapture(s, &gr));
                    BK(cudaGraphInstantiate(&graph, gr, 0));
                    BK(cudaGraphDestroy(gr));
                    per_graph = launches - before;
                }
                BK(cudaGraphLaunch(graph, s));
                launches += per_graph;
            } else {
                block(steps);
            }
            it += steps;
            BK(cudaMemcpyAsync(h_count, count, sizeof(int), cudaMemcpyDeviceToHost, s));
            BK(cudaStreamSynchronize(s));
            if (*h_count == 0) break;
        }
        BK(cudaGetLastError());
        // download
        std::vector<InstState> fin(ninst);
        BK(cudaMemcpyAsync(fin.data(), st, ninst * sizeof(InstState), cudaMemcpyDeviceToHost, s));
        std::vector<double> hx(N), hz(M);
        if (nT) k_out_blocks<T><<<nT, kThreads, 0, s>>>(T_ev, Te_ev, st, x, xs, dout);
        BK(cudaMemcpyAsync(hx.data(), dout, N * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (nA) k_out_blocks<T><<<nA, kThreads, 0, s>>>(A_ev, Ae_ev, st, z, zs, dout);
        BK(cudaMemcpyAsync(hz.data(), dout, M * sizeof(double), cudaMemcpyDeviceToHost, s));
        BK(cudaEventRecord(e1, s));
        BK(cudaStreamSynchronize(s));
        launches += 2;
        float ms = 0;
        BK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0), cudaEventDestroy(e1);
        double solve_s = since(t0);
        for (int i = 0; i < ninst; ++i) {
            const InstState& q = fin[i];
            const Shared& sh = *mats[mat_of[i]];
            Outcome r;
            r.status = q.status, r.iterations = q.it, r.restarts = q.restarts, r.from_average = q.avg_final != 0;
            r.rel_primal = q.best_p, r.rel_dual = q.best_d, r.rel_gap = q.best_g, r.norm_a = q.norm, r.omega = q.w;
            r.x.assign(hx.begin() + col_off[i], hx.begin() + col_off[i + 1]);
            r.z.assign(hz.begin() + row_off[i], hz.begin() + row_off[i + 1]);
            Scaled P;  // finish_point needs Dr, Dc and sizes
            P.m = models[i]->m, P.n = models[i]->n, P.Dr = sh.S.Dr, P.Dc = sh.S.Dc;
            Finished f = finish_point(*models[i], P, r);
            taral_outcome& o = outs[i];
            std::memset(&o, 0, sizeof o);
            o.status = r.status, o.iterations = r.iterations, o.restarts = r.restarts, o.from_average = r.from_average;
            o.rel_primal = r.rel_primal, o.rel_dual = r.rel_dual, o.rel_gap = r.rel_gap, o.norm_a = r.norm_a;
            o.primal_weight = r.omega, o.objective = f.objective, o.max_row_violation = f.max_row_violation;
            o.max_bound_violation = f.max_bound_violation, o.solve_s = solve_s, o.power_iter_s = power_s;
            o.device_mem_bytes = mem_used, o.kernel_launches = launches, o.nnz = int64_t(sh.S.A.val.size());
            o.device_s = ms * 1e-3;
            if (xo && xo[i]) std::memcpy(xo[i], f.x.data(), f.x.size() * sizeof(double));
            if (yo && yo[i]) std::memcpy(yo[i], f.y.data(), f.y.size() * sizeof(double));
        }
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
        h->b->solve(x0, y0, w0, outs, x_out, y_out);
    } catch (const taral::BatchError& e) {
        h->b->err = e.msg;
        return TARAL_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        return TARAL_ERR_ALLOC;
    }
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
