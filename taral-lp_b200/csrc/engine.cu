// Device context of the B200 PDHG engine and the C ABI of its backend concept (include/taral_pdhg.h, part 1 and 4).
//
// HBM layout of one context (T = double for TARAL_FP64, float for TARAL_FP32):
//   A   (m rows): ptr int32[m+1], idx int32[nnz], val T[nnz], row blocks int32[nblk+1]
//   A^T (n rows): the same for the transposed copy (products with A^T never use atomics)
//   data   c, l, u, Dc : T[n]        rl, ru, Dr : T[m]        par : T[2] = {tau, sigma}
//   state  x, ATz, xlast : T[n]      z, Ax, zlast : T[m]      xs : f64[n]  zs : f64[m]  (running sums)
//   eval   tmp_n f64[n], tmp_m f64[m] (products of the sums), partials, tickets, 20 result doubles
// The running sums of A x and A^T z that the reference keeps (gpu/pdhg.cu:188, :200) are not stored: the
// average's products are formed once per evaluation as A xs and A^T zs, which saves 16 bytes of state traffic
// per row and per column every iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/taral_pdhg.h"
#include "engine.hpp"
#include "host.hpp"
#include "kernels.cuh"
#include "scaling.cuh"

namespace taral {

// ---------------------------------------------------------------------------------------------- memory
// Device buffers come from the device's default memory pool (cudaMallocAsync / cudaFreeAsync on the context's
// stream). The pool keeps up to 32 GB of freed memory for the process, so a context's release is a stream-ordered
// return to the pool and the next context of the process reuses the memory without new device allocations.
// Fault-injection hook (taral_set_device_alloc_limit): the most bytes one context or batch may allocate, 0 = no limit.
static std::atomic<size_t> g_alloc_limit{0};
bool alloc_allowed(size_t used, size_t more) {
    const size_t lim = g_alloc_limit.load(std::memory_order_relaxed);
    return lim == 0 || used + more <= lim;
}

void keep_pool_memory(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = uint64_t(32) << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done.push_back(dev);
}

// The device's name, queried once per device (the full property query is slow next to a small LP's solve).
std::string device_name(int dev) {
    static std::mutex mu;
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> lock(mu);
    auto it = names.find(dev);
    if (it != names.end()) return it->second;
    char buf[256] = {0};
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) std::snprintf(buf, sizeof buf, "%s", prop.name);
    else cudaGetLastError();
    return names[dev] = buf;
}

// Pinned host blocks for the contexts' status reads, kept for the process once allocated: cudaMallocHost and
// cudaFreeHost cost up to milliseconds per call (and the free synchronises the device), a visible part of a small
// LP's solve. A block holds 32 doubles and an int.
constexpr size_t kPinnedBlock = 512;
static_assert(32 * sizeof(double) + sizeof(int) <= kPinnedBlock, "a status block holds 32 doubles and an int");
std::mutex g_pinned_mu;
std::vector<void*> g_pinned_free;
void* pinned_block() {
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        if (!g_pinned_free.empty()) {
            void* p = g_pinned_free.back();
            g_pinned_free.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    return cudaMallocHost(&p, kPinnedBlock) == cudaSuccess ? p : nullptr;
}
void pinned_return(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(p);
}

// ---------------------------------------------------------------------------------------------- row blocks
// Consecutive rows are packed into blocks of at most kTile nonzeros and kRowsMax rows; a longer row is a block of
// its own (block_sums sums it with the whole CTA).
std::vector<int4> build_row_blocks(const int64_t* ptr, int rows) { return build_row_blocks(ptr, rows, kTile, kRowsMax); }

// Policies: 0 the hybrid rule, 1 a thread per row in kUniformCandidate blocks, 2 segmented sums in every block, 3
// 8-lane groups for rows up to kMid nonzeros in every block, 4 policies 1 and 3 together.
bool apply_row_split(std::vector<int4>& blk, int policy) {
    bool changed = false;
    for (int4& b : blk) {
        const bool cand = (b.y & kUniformCandidate) != 0;
        if ((policy == 1 || policy == 4) && cand) b.y |= kUniformRows, changed = true;
        if (policy == 2) b.y |= kSegmented, changed = true;
        if (policy == 3 || policy == 4) b.y |= kMidGroups, changed = changed || policy == 3;
    }
    return changed;
}

int forced_row_split() {
    const char* e = std::getenv("TARAL_ROWSPLIT");
    return e ? std::max(0, std::min(kPolicies - 1, std::atoi(e))) : -1;
}

std::vector<int4> build_row_blocks(const int64_t* ptr, int rows, int tile, int rows_max) {
    std::vector<int4> out;
    auto close = [&](int r0, int r1) {  // y: rows | kUniformCandidate when no row is much longer than the mean
        int64_t mx = 0;
        for (int r = r0; r < r1; ++r) mx = std::max<int64_t>(mx, ptr[r + 1] - ptr[r]);
        const int64_t nz = ptr[r1] - ptr[r0], mean = (nz + (r1 - r0) - 1) / (r1 - r0);
        const bool uniform = r1 - r0 > 1 && mx > kShort && mx <= 2 * mean + 8;
        out.push_back(make_int4(r0, (r1 - r0) | (uniform ? kUniformCandidate : 0), int(ptr[r0]), int(ptr[r1])));
    };
    int start = 0, cur_rows = 0;
    int64_t cur_nnz = 0;
    for (int r = 0; r < rows; ++r) {
        int64_t L = ptr[r + 1] - ptr[r];
        if (L > tile) {  // a long row is a block of its own
            if (cur_rows) close(start, r);
            close(r, r + 1);
            start = r + 1, cur_rows = 0, cur_nnz = 0;
            continue;
        }
        if (cur_rows == rows_max || cur_nnz + L > tile) close(start, r), start = r, cur_rows = 0, cur_nnz = 0;
        ++cur_rows, cur_nnz += L;
    }
    if (cur_rows) close(start, rows);
    return out;
}

static int grid_for(int64_t k) {  // elementwise kernels: grid-stride, at most 8 CTAs of 256 per SM
    return int(std::max<int64_t>(1, std::min<int64_t>((k + 255) / 256, 148 * 8)));
}
static int red_grid(int64_t k) {  // reductions: fixed grid per size, so the partial-sum order is fixed
    return int(std::max<int64_t>(1, std::min<int64_t>((k + 255) / 256, 296)));
}

struct CudaError {
    std::string msg;
};
#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            throw CudaError{std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" +   \
                            std::to_string(__LINE__) + ")"};                                               \
    } while (0)

struct DevMat {
    int rows = 0, maxrow = 0;  // maxrow: the longest row's nonzeros
    bool per_thread = false;   // SpMV by k_rowthread (one thread per row) instead of the row blocks
    int64_t nnz = 0;
    int *ptr = nullptr, *idx = nullptr;
    int4* blk = nullptr;
    void* val = nullptr;
    int nblk = 0;
};

template <class T>
struct Engine final : EngineBase {
    int m = 0, n = 0, eval_freq = 64;
    bool use_graph = true;
    DevMat A, AT;
    T *c = nullptr, *l = nullptr, *u = nullptr, *rl = nullptr, *ru = nullptr, *Dr = nullptr, *Dc = nullptr;
    double* par = nullptr;  // {tau, sigma}
    T *x = nullptr, *z = nullptr, *Ax = nullptr, *ATz = nullptr, *xlast = nullptr, *zlast = nullptr;
    T *pv = nullptr, *pw = nullptr, *pu = nullptr;
    double *xs = nullptr, *zs = nullptr, *tmp_m = nullptr, *tmp_n = nullptr, *hbuf = nullptr, *part = nullptr,
           *out = nullptr, *pst = nullptr, *h_out = nullptr, *d_in = nullptr;
    unsigned* tickets = nullptr;
    int* pdone = nullptr;
    int* h_flag = nullptr;
    cudaStream_t st = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaGraphExec_t pgraph = nullptr;  // a chunk of power-iteration steps
    std::vector<void*> allocs;
    bool started = false;

    template <class U>
    U* alloc(size_t count) {  // stream-ordered, from the device's memory pool (see keep_pool_memory)
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(U);
        if (!alloc_allowed(alloc_bytes, bytes))
            throw CudaError{"cudaMalloc: the device allocation limit (taral_set_device_alloc_limit) is reached"};
        cudaError_t e = cudaMallocAsync(&p, bytes, st);
        if (e != cudaSuccess) throw CudaError{std::string("cudaMalloc: ") + cudaGetErrorString(e)};
        allocs.push_back(p);
        alloc_bytes += bytes;
        return static_cast<U*>(p);
    }
    size_t alloc_bytes = 0;
    T* upload(const double* v, size_t k) {
        std::vector<T> h(v, v + k);
        T* p = alloc<T>(k);
        if (k) CK(cudaMemcpyAsync(p, h.data(), k * sizeof(T), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return p;
    }
    template <class U>
    U* zeros(size_t k) {
        U* p = alloc<U>(k);
        CK(cudaMemsetAsync(p, 0, std::max<size_t>(k, 1) * sizeof(U), st));
        return p;
    }
    DevMat upload(const taral_csr& a) {
        DevMat d;
        d.rows = a.rows, d.nnz = a.nnz;
        std::vector<int> p32(size_t(a.rows) + 1);
        for (int r = 0; r <= a.rows; ++r) p32[r] = int(a.ptr[r]);
        for (int r = 0; r < a.rows; ++r) d.maxrow = std::max(d.maxrow, p32[r + 1] - p32[r]);
        std::vector<int4> blk = build_row_blocks(a.ptr, a.rows);
        d.nblk = int(blk.size());
        d.ptr = alloc<int>(p32.size()), d.idx = alloc<int>(size_t(a.nnz)), d.blk = alloc<int4>(blk.size());
        CK(cudaMemcpyAsync(d.ptr, p32.data(), p32.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        if (a.nnz) CK(cudaMemcpyAsync(d.idx, a.idx, size_t(a.nnz) * sizeof(int), cudaMemcpyHostToDevice, st));
        if (!blk.empty())
            CK(cudaMemcpyAsync(d.blk, blk.data(), blk.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
        d.val = upload(a.val, size_t(a.nnz));
        return d;
    }

    void begin(int m_, int n_, int freq, unsigned flags) {
        m = m_, n = n_, eval_freq = std::max(1, freq), use_graph = !(flags & TARAL_FLAG_NO_GRAPH);
        int dev;
        CK(cudaGetDevice(&dev));
        keep_pool_memory(dev);
        name = device_name(dev);
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        if (const char* e = std::getenv("TARAL_PDL")) pdl = std::atoi(e) != 0;
    }
    void init(const taral_csr& hA, const taral_csr& hAT, const double* hc_ptr, const double* hl, const double* hu,
              const double* hrl_ptr, const double* hru_ptr, const double* hDr, const double* hDc, int m_, int n_,
              int freq, unsigned flags) {
        begin(m_, n_, freq, flags);
        A = upload(hA), AT = upload(hAT);
        nnz = hA.nnz;
        finish_init(hc_ptr, hl, hu, hrl_ptr, hru_ptr, hDr, hDc);
    }
    // Internal row order (contexts built from a model whose rows are of both kinds, short (<= kShort nonzeros)
    // and long): rows sorted by ascending length (stable). The row phase's blocks then hold rows of similar length,
    // and the column phase's gathers of z concentrate on a contiguous tail (a long row of A is gathered by many
    // columns), which L1 and L2 serve far better. Every row's entries keep their order and A^T's entries keep
    // theirs (renumbered), so both phases add the same products in the same order as in the model's row order;
    // only the FP64 KKT sums over rows change order (in FP64 runs the reference's iteration counts hold: the
    // parity tests pin them). TARAL_ROWORDER=0 keeps the model's order. rperm[k] = model row at position k.
    std::vector<int> rperm;
    // ap: A with its rows in that order; at_idx: A^T's row indices renumbered (its pointers and values unchanged).
    // The copies run on the host threads.
    bool order_rows(const Csr& a, const CsrRef& at, Csr& ap, Entries<int32_t>& at_idx) {
        rperm.clear();
        const char* e = std::getenv("TARAL_ROWORDER");  // 0 off, otherwise (default) rows sorted by length
        const int mode = e ? std::atoi(e) : 1;
        if (mode <= 0 || a.rows == 0) return false;
        const int rows = a.rows;
        auto len = [&](int r) { return a.ptr[size_t(r) + 1] - a.ptr[size_t(r)]; };
        std::vector<int> perm(static_cast<size_t>(rows));
        int64_t longest = 0;
        for (int r = 0; r < rows; ++r) longest = std::max(longest, len(r));
        if (longest <= 16 * int64_t(rows) + 1024) {  // stable counting sort by length
            std::vector<int> at(size_t(longest) + 2, 0);
            for (int r = 0; r < rows; ++r) at[size_t(len(r)) + 1]++;
            for (size_t l = 1; l < at.size(); ++l) at[l] += at[l - 1];
            for (int r = 0; r < rows; ++r) perm[size_t(at[size_t(len(r))]++)] = r;
        } else {
            for (int r = 0; r < rows; ++r) perm[size_t(r)] = r;
            std::stable_sort(perm.begin(), perm.end(), [&](int x, int y) { return len(x) < len(y); });
        }
        int split = 0;
        while (split < rows && len(perm[size_t(split)]) <= kShort) ++split;
        if (split == rows || split == 0) return false;  // rows of one kind: nothing to separate
        std::vector<int> inv(static_cast<size_t>(rows));
        for (int k = 0; k < rows; ++k) inv[size_t(perm[size_t(k)])] = k;
        ap.rows = rows;
        ap.ptr.assign(size_t(rows) + 1, 0);
        for (int k = 0; k < rows; ++k) ap.ptr[size_t(k) + 1] = ap.ptr[size_t(k)] + len(perm[size_t(k)]);
        ap.idx.resize(a.idx.size()), ap.val.resize(a.val.size());
        const int threads = host_threads();
        const int64_t nnz = ap.ptr[size_t(rows)];
        split_ranges(threads, threads, [&](int, int64_t q0, int64_t q1) {  // rows cut into ranges of equal nonzeros
            for (int64_t q = q0; q < q1; ++q) {
                const auto row_at = [&](int64_t e) {
                    return int(std::lower_bound(ap.ptr.begin(), ap.ptr.end(), e) - ap.ptr.begin());
                };
                const int k0 = row_at(nnz * q / threads), k1 = q + 1 == threads ? rows : row_at(nnz * (q + 1) / threads);
                for (int k = k0; k < k1; ++k) {
                    const int64_t b = a.ptr[size_t(perm[size_t(k)])], l = len(perm[size_t(k)]), o = ap.ptr[size_t(k)];
                    std::copy(a.idx.begin() + b, a.idx.begin() + b + l, ap.idx.begin() + o);
                    std::copy(a.val.begin() + b, a.val.begin() + b + l, ap.val.begin() + o);
                }
            }
        });
        at_idx.resize(size_t(at.nnz()));
        split_ranges(at.nnz(), threads, [&](int, int64_t q0, int64_t q1) {
            for (int64_t q = q0; q < q1; ++q) at_idx[size_t(q)] = inv[size_t(at.idx[q])];
        });
        rperm = std::move(perm);
        return true;
    }
    std::vector<double> to_internal(const std::vector<double>& v) const {  // model row order -> internal
        std::vector<double> o(v.size());
        for (size_t k = 0; k < v.size(); ++k) o[k] = v[size_t(rperm[k])];
        return o;
    }
    std::vector<double> to_model(const std::vector<double>& v) const {  // internal -> model row order
        std::vector<double> o(v.size());
        for (size_t k = 0; k < v.size(); ++k) o[size_t(rperm[k])] = v[k];
        return o;
    }
    // Row pointers, column indices and row blocks of one matrix on the device; the values are left to the caller.
    DevMat upload_structure(const CsrRef& a) {
        DevMat d;
        d.rows = a.rows, d.nnz = a.nnz();
        std::vector<int> p32(size_t(a.rows) + 1);
        for (int r = 0; r <= a.rows; ++r) p32[r] = int(a.ptr[r]);
        for (int r = 0; r < a.rows; ++r) d.maxrow = std::max(d.maxrow, p32[r + 1] - p32[r]);
        std::vector<int4> blk = build_row_blocks(a.ptr, a.rows);
        d.nblk = int(blk.size());
        d.ptr = alloc<int>(p32.size()), d.idx = alloc<int>(size_t(d.nnz)), d.blk = alloc<int4>(blk.size());
        CK(cudaMemcpyAsync(d.ptr, p32.data(), p32.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        if (d.nnz) CK(cudaMemcpyAsync(d.idx, a.idx, size_t(d.nnz) * sizeof(int), cudaMemcpyHostToDevice, st));
        if (!blk.empty())
            CK(cudaMemcpyAsync(d.blk, blk.data(), blk.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
        d.val = alloc<T>(size_t(d.nnz));
        CK(cudaStreamSynchronize(st));  // the host vectors may be released after return
        return d;
    }
    // Set-up from the column-wise model with the scaling on the device (scaling.cuh): the host builds the unscaled
    // A and A^T (model_matrices, the reference's transposes), the device scales them in FP64 and narrows the values
    // to T in place. Fills P's Dr, Dc, vectors and norms (scale_vectors on the host, O(m + n)); P.A keeps the
    // UNSCALED row-wise copy (for finish_point), P.AT stays empty. host_s: seconds of host work.
    void init_model(const taral_model& md, double sign, Scaled& P, int freq, unsigned flags, double* host_s) {
        auto t0 = Clock::now();
        Csr hA, hAT;
        const CsrRef mAT = model_matrices_ref(md, hA, hAT);  // A^T: the model's own arrays when they are A^T
        // rows in ascending length internally (rperm: internal -> model row); A^T keeps its entry order (its
        // indices renumbered), so both phases sum exactly as before
        Csr hAp;
        Entries<int32_t> at_idx;
        const bool reorder = order_rows(hA, mAT, hAp, at_idx);
        const CsrRef uA = ref(reorder ? hAp : hA);
        CsrRef uAT = mAT;
        if (reorder) uAT.idx = at_idx.data();
        double hs = since(t0);
        begin(md.m, md.n, freq, flags);
        A = upload_structure(uA), AT = upload_structure(uAT);
        const int64_t nz = int64_t(hA.val.size());
        P.m = m, P.n = n;
        P.Dr.resize(size_t(m)), P.Dc.resize(size_t(n));
        {
        double *va = nullptr, *vt = nullptr, *dr = nullptr, *dc = nullptr, *rs = nullptr, *cs = nullptr;
        struct Scratch {  // FP64 working values and factors, released when the set-up ends
            std::vector<void*> p;
            cudaStream_t s;
            ~Scratch() { for (void* q : p) cudaFreeAsync(q, s); }
        } tmp{{}, st};
        auto scratch = [&](size_t count) {
            void* q = nullptr;
            CK(cudaMallocAsync(&q, std::max<size_t>(count, 1) * sizeof(double), st));
            tmp.p.push_back(q);
            return static_cast<double*>(q);
        };
        if (sizeof(T) == sizeof(double)) {
            va = reinterpret_cast<double*>(A.val), vt = reinterpret_cast<double*>(AT.val);
        } else {
            va = scratch(size_t(nz)), vt = scratch(size_t(nz));
        }
        dr = scratch(size_t(m)), dc = scratch(size_t(n)), rs = scratch(size_t(m)), cs = scratch(size_t(n));
        if (nz) {
            CK(cudaMemcpyAsync(va, uA.val, size_t(nz) * sizeof(double), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(vt, uAT.val, size_t(nz) * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        scale_on_device(m, n, A.ptr, A.idx, va, AT.ptr, AT.idx, vt, dr, dc, rs, cs, st);
        if (sizeof(T) != sizeof(double) && nz) {
            const int g = int(std::min<int64_t>((nz + 255) / 256, 148 * 16));
            k_narrow<T><<<g, 256, 0, st>>>(nz, va, static_cast<T*>(A.val));
            k_narrow<T><<<g, 256, 0, st>>>(nz, vt, static_cast<T*>(AT.val));
        }
        if (m) CK(cudaMemcpyAsync(P.Dr.data(), dr, size_t(m) * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (n) CK(cudaMemcpyAsync(P.Dc.data(), dc, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        }  // FP64 scratch released
        t0 = Clock::now();
        if (reorder) P.Dr = to_model(P.Dr);
        hAp = Csr(), at_idx = Entries<int32_t>();
        P.A = std::move(hA), P.AT = Csr();  // the unscaled row-wise copy serves the original-space check
        P.a_original = true;
        hAT = Csr();
        scale_vectors(md, sign, P.Dr, P.Dc, P);
        hs += since(t0);
        if (host_s) *host_s = hs;
        if (reorder) {
            const std::vector<double> rl_i = to_internal(P.rl), ru_i = to_internal(P.ru), dr_i = to_internal(P.Dr);
            finish_init(P.c.data(), P.l.data(), P.u.data(), rl_i.data(), ru_i.data(), dr_i.data(), P.Dc.data());
            hrl = P.rl, hru = P.ru;  // the driver's host copies stay in the model's order
        } else {
            finish_init(P.c.data(), P.l.data(), P.u.data(), P.rl.data(), P.ru.data(), P.Dr.data(), P.Dc.data());
        }
        nnz = nz;
    }
    void finish_init(const double* hc_ptr, const double* hl, const double* hu, const double* hrl_ptr,
                     const double* hru_ptr, const double* hDr, const double* hDc) {
        c = upload(hc_ptr, n), l = upload(hl, n), u = upload(hu, n), Dc = upload(hDc, n);
        rl = upload(hrl_ptr, m), ru = upload(hru_ptr, m), Dr = upload(hDr, m);
        par = zeros<double>(2);
        x = zeros<T>(n), ATz = zeros<T>(n), xlast = zeros<T>(n);
        z = zeros<T>(m), Ax = zeros<T>(m), zlast = zeros<T>(m);
        xs = zeros<double>(n), zs = zeros<double>(m), tmp_n = zeros<double>(n), tmp_m = zeros<double>(m);
        pv = zeros<T>(n), pw = zeros<T>(m), pu = zeros<T>(n);
        hbuf = alloc<double>(size_t(std::max(m, n)));
        d_in = alloc<double>(size_t(std::max(m, n)));
        part = zeros<double>(size_t(296) * 5 * 2);
        out = zeros<double>(32);
        pst = zeros<double>(4);
        tickets = zeros<unsigned>(4);
        pdone = zeros<int>(1);
        hc.assign(hc_ptr, hc_ptr + n), hrl.assign(hrl_ptr, hrl_ptr + m), hru.assign(hru_ptr, hru_ptr + m);
        h_out = static_cast<double*>(pinned_block());
        if (!h_out) throw CudaError{"cudaMallocHost: no pinned host memory for the status reads"};
        h_flag = reinterpret_cast<int*>(h_out + 32);
        CK(cudaStreamSynchronize(st));
        mem_used = alloc_bytes;
        tune();
    }
    ~Engine() override {
        if (ev0) cudaEventDestroy(ev0), cudaEventDestroy(ev1);
        if (graph) cudaGraphExecDestroy(graph);
        if (pgraph) cudaGraphExecDestroy(pgraph);
        for (void* p : allocs) cudaFreeAsync(p, st);  // back to the pool: no device-wide synchronisation
        if (st) cudaStreamSynchronize(st);
        pinned_return(h_out);  // after the synchronisation above: no copy into it is in flight
        if (st) cudaStreamDestroy(st);
    }

    // ------------------------------------------------------------------ autotuner
    // Per matrix of at least 2^20 nonzeros, timed on the matrix itself (CUDA-event time of 10 launches of its PDHG
    // phase, the SpMV with its fused step, after 3 warm-ups, 13 before the first candidate; a choice other than the
    // default is kept only if it is at least 5 % faster). Candidates that cannot change the arithmetic (policies 1,
    // 3, 4 when no row exceeds kShort) are not timed, so noise cannot pick them:
    // 1. FP32 contexts: the row-split policy of the block list (kernels.cuh): 0 the hybrid rule (thread per row up to
    //    48 nonzeros, warp per longer row), 1 thread per row in the kUniformCandidate blocks, 2 the balanced
    //    segmented sums (kSegmented) in every block, 3 the hybrid rule with 8-lane groups for rows up to 128
    //    nonzeros (kMidGroups), 4 policies 1 and 3 together. FP64 contexts keep policy 0 (the parity pins'
    //    summation order).
    // 2. k_rowthread instead of the block kernel: in any precision for matrices whose rows all hold at most kShort
    //    nonzeros (bit-identical results under policy 0, so FP64 may use it too); in FP32 also for rows up to kMid
    //    (every row summed by its own thread in entry order).
    // TARAL_TUNE=0 keeps the defaults; TARAL_ROWSPLIT=0..4 and TARAL_ROWTHREAD=0|1 force a choice, untimed.
    void tune() {
        if (const char* e = std::getenv("TARAL_TUNE"))
            if (std::atoi(e) == 0) return;
        const int forced = forced_row_split();
        int forced_thread = -1;
        if (const char* e = std::getenv("TARAL_ROWTHREAD")) forced_thread = std::atoi(e) != 0 ? 1 : 0;
        int which = 0;
        for (DevMat* d : {&A, &AT}) {
            const int slot = which++;
            if (d->nblk == 0) continue;
            const bool small = d->nnz < (int64_t(1) << 20);  // timings are noise
            const bool short_rows = d->maxrow <= kShort;      // every row on the thread path of policy 0
            // the thread-per-row kernel: bit-identical with short rows; otherwise (FP32, rows up to kMid) it sums
            // every row by its own thread, as policy 1 does in uniform blocks
            const bool thread_ok = short_rows || (sizeof(T) == sizeof(float) && d->maxrow <= kMid);
            // the phase itself with its fused step, on the not yet started state (start() rewrites every vector the
            // steps write: x, xs, z, zs, Ax, ATz)
            auto phase = [&] {
                if (d == &A) rowblock(A, x, EpiRow<T>{Ax, z, zs, rl, ru, par});
                else rowblock(AT, z, EpiCol<T>{ATz, x, xs, c, l, u, par, 1});
            };
            auto time_spmv = [&](int warm) {
                for (int r = 0; r < warm; ++r) phase();
                cudaEvent_t e0, e1;
                CK(cudaEventCreate(&e0));
                CK(cudaEventCreate(&e1));
                CK(cudaEventRecord(e0, st));
                for (int r = 0; r < 10; ++r) phase();
                CK(cudaEventRecord(e1, st));
                CK(cudaEventSynchronize(e1));
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                cudaEventDestroy(e0), cudaEventDestroy(e1);
                launches -= warm + 10;  // tuning launches are not part of the solve's count
                return ms;
            };
            std::vector<int4> base(size_t(d->nblk));
            CK(cudaMemcpyAsync(base.data(), d->blk, base.size() * sizeof(int4), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            std::vector<std::vector<int4>> cand(kPolicies, base);
            bool timed[kPolicies] = {true};
            for (int k = 1; k < kPolicies; ++k) {
                // FP32 only (FP64 keeps the parity pins' order); with short rows only policy 2 sums differently
                const bool differs = apply_row_split(cand[k], k);
                timed[k] = sizeof(T) == sizeof(float) && differs && (!short_rows || k == 2);
            }
            auto put = [&](const std::vector<int4>& list) {
                CK(cudaMemcpyAsync(d->blk, list.data(), list.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
            };
            int best = 0;
            bool thread = false;
            float t_pol[kPolicies] = {0}, t_thread = 0;
            if (forced >= 0 || forced_thread >= 0) {
                if (sizeof(T) == sizeof(float) && forced >= 0) best = forced;
                thread = thread_ok && best == 0 && forced_thread == 1;
            } else if (!small) {
                const float t0 = t_pol[0] = time_spmv(13);  // the first timings of a context also warm the GPU up
                float tb = t0;
                for (int k = 1; k < kPolicies; ++k) {
                    if (!timed[k]) continue;
                    put(cand[k]);
                    const float t = t_pol[k] = time_spmv(3);
                    if (t < 0.95f * t0 && t < tb) tb = t, best = k;
                }
                put(base);
                if (thread_ok) {
                    d->per_thread = true;
                    const float t = t_thread = time_spmv(3);
                    d->per_thread = false;
                    if (t < 0.95f * t0 && t < tb) tb = t, best = 0, thread = true;
                }
                if (std::getenv("TARAL_TIMING"))
                    std::fprintf(stderr, "taral: tune %s: policies %.1f %.1f %.1f %.1f %.1f, thread per row %.1f us/launch\n",
                                 slot ? "A^T" : "A", t_pol[0] * 100, t_pol[1] * 100, t_pol[2] * 100, t_pol[3] * 100,
                                 t_pol[4] * 100, t_thread * 100);
            }
            tuned[slot] = best;
            put(cand[best]);
            d->per_thread = per_thread[slot] = thread;
            CK(cudaStreamSynchronize(st));
        }
    }

    // ------------------------------------------------------------------ SpMV-shaped launches
    // `programmatic`: launch with programmatic stream serialisation, so the kernel may start while its predecessor
    // drains (both phase kernels wait for their predecessor before the first gather and release their successor
    // after that wait). Used for the two phase kernels of an iteration block when TARAL_PDL=1.
    template <class K, class... Args>
    void launch(K kernel, int grid, bool programmatic, Args... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(grid)), cfg.blockDim = dim3(kThreads), cfg.dynamicSmemBytes = 0, cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr, cfg.numAttrs = programmatic ? 1 : 0;
        CK(cudaLaunchKernelEx(&cfg, kernel, args...));
    }
    template <class X, class E>
    void rowblock(const DevMat& a, const X* xin, const E& epi, const int* skip = nullptr, bool programmatic = false) {
        if (a.nblk == 0) return;
        if (a.per_thread)
            launch(k_rowthread<T, X, E>, (a.rows + kThreads - 1) / kThreads, programmatic, a.rows,
                   (const int*)a.ptr, (const int*)a.idx, static_cast<const T*>(a.val), xin, skip, epi);
        else
            launch(k_rowblock<T, X, E, true>, a.nblk, programmatic, (const int*)a.ptr, (const int*)a.idx,
                   static_cast<const T*>(a.val), xin, (const int4*)a.blk, skip, epi);
        ++launches;
    }
    template <class X, class Y>
    void spmv(const DevMat& a, const X* xin, Y* y, const int* skip = nullptr) {
        rowblock(a, xin, EpiStore<Y>{y}, skip);
    }
    void products() {  // Ax = A x, ATz = A^T z exactly (gpu/pdhg.cu:446-449)
        spmv(A, x, Ax);
        spmv(AT, z, ATz);
    }

    // ------------------------------------------------------------------ backend concept
    double power_norm(int iters) override {
        std::vector<double> h(n);
        double nn = 0;
        for (int j = 0; j < n; ++j) h[j] = 0.5 + double((uint32_t(j) * 2654435761u) % 1000u) / 1000.0, nn += h[j] * h[j];
        for (int j = 0; j < n; ++j) h[j] = h[j] / std::sqrt(nn);
        if (n) CK(cudaMemcpyAsync(d_in, h.data(), size_t(n) * sizeof(double), cudaMemcpyHostToDevice, st));
        k_cast<T><<<grid_for(n), 256, 0, st>>>(n, d_in, pv);
        CK(cudaMemsetAsync(pst, 0, 4 * sizeof(double), st));
        CK(cudaMemsetAsync(pdone, 0, sizeof(int), st));
        launches += 1;
        T *a = pv, *b = pu;
        // steps queued between checks of the device-side stop flag; an even count, so that every chunk starts with
        // the vectors in the same roles and a chunk captured once replays as a CUDA graph
        const int chunk = 8;
        auto step = [&] {
            spmv(A, a, pw, pdone);
            spmv(AT, pw, b, pdone);
            k_power_sumsq<T><<<red_grid(n), kRedThreads, 0, st>>>(n, b, part, tickets + 2, out + 24, pdone);
            k_power_update<<<1, 1, 0, st>>>(out + 24, pst, pdone);
            k_power_scale<T><<<grid_for(n), 256, 0, st>>>(n, b, pst, pdone);
            launches += 3;
            std::swap(a, b);
        };
        for (int it = 0; it < iters;) {
            const int end = std::min(iters, it + chunk);
            if (use_graph && end - it == chunk) {
                if (!pgraph) {  // capturing swaps a and b `chunk` times: they end in their starting roles
                    const int64_t before = launches;
                    cudaGraph_t g;
                    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                    for (int k = 0; k < chunk; ++k) step();
                    CK(cudaStreamEndCapture(st, &g));
                    CK(cudaGraphInstantiate(&pgraph, g, 0));
                    CK(cudaGraphDestroy(g));
                    launches = before;
                }
                CK(cudaGraphLaunch(pgraph, st));
                launches += 5 * chunk;  // two SpMVs and three small kernels per step
                it = end;
            } else {
                for (; it < end; ++it) step();
            }
            CK(cudaMemcpyAsync(h_flag, pdone, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (*h_flag) break;
        }
        CK(cudaMemcpyAsync(h_out, pst, sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        return h_out[0];
    }
    void set_steps(double tau, double sigma) override {
        k_set_par<<<1, 1, 0, st>>>(par, tau, sigma);
        ++launches;
        CK(cudaGetLastError());
    }
    void start(const double* x0, const double* z0) override {
        if (x0) {
            CK(cudaMemcpyAsync(d_in, x0, size_t(n) * sizeof(double), cudaMemcpyHostToDevice, st));
            k_set_point<T><<<grid_for(n), 256, 0, st>>>(n, d_in, x, xlast, xs);
        } else {
            k_start_x<T><<<grid_for(n), 256, 0, st>>>(n, l, u, x, xlast, xs);
        }
        ++launches;
        std::vector<double> z0_i;
        if (z0 && !rperm.empty()) z0_i = to_internal(std::vector<double>(z0, z0 + m)), z0 = z0_i.data();
        if (z0) {  // the copy into d_in above has been consumed in stream order before this one lands
            CK(cudaMemcpyAsync(d_in, z0, size_t(m) * sizeof(double), cudaMemcpyHostToDevice, st));
            k_set_point<T><<<grid_for(m), 256, 0, st>>>(m, d_in, z, zlast, zs);
        } else {
            k_zero_point<T><<<grid_for(m), 256, 0, st>>>(m, z, zlast, zs);
        }
        ++launches;
        products();
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        started = true;
    }
    bool pdl = false;  // TARAL_PDL=1: programmatic launches of the phase kernels (set at init; measured slower)
    void launch_block(int steps) {
        k_xupd<T><<<grid_for(n), 256, 0, st>>>(n, x, ATz, c, l, u, par, xs);
        for (int s = 0; s < steps; ++s) {
            rowblock(A, x, EpiRow<T>{Ax, z, zs, rl, ru, par}, nullptr, pdl);
            rowblock(AT, z, EpiCol<T>{ATz, x, xs, c, l, u, par, s + 1 < steps ? 1 : 0}, nullptr, pdl);
        }
    }
    void iterate(int steps) override {
        if (steps <= 0) return;
        if (use_graph && steps == eval_freq) {
            if (!graph) {
                cudaGraph_t g;
                int64_t before = launches;
                CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                launch_block(steps);
                CK(cudaStreamEndCapture(st, &g));
                CK(cudaGraphInstantiate(&graph, g, 0));
                CK(cudaGraphDestroy(g));
                launches = before;
            }
            CK(cudaGraphLaunch(graph, st));
            launches += 1 + 2 * int64_t(steps);
        } else {
            launch_block(steps);
            launches += 1;
        }
        CK(cudaGetLastError());
    }
    void queue_eval(bool avg, double f, double* dst) {
        int gr = red_grid(m), gc = red_grid(n);
        if (!avg) {
            k_eval_row<T, T><<<gr, kRedThreads, 0, st>>>(m, 1.0 * f, Ax, z, rl, ru, Dr, zlast, part, tickets, dst);
            k_eval_col<T, T><<<gc, kRedThreads, 0, st>>>(n, 1.0 * f, x, ATz, c, l, u, Dc, xlast, part + 296 * 5,
                                                          tickets + 1, dst + 5);
        } else {
            spmv(A, xs, tmp_m);
            spmv(AT, zs, tmp_n);
            k_eval_row<T, double><<<gr, kRedThreads, 0, st>>>(m, f, tmp_m, zs, rl, ru, Dr, zlast, part, tickets, dst);
            k_eval_col<T, double><<<gc, kRedThreads, 0, st>>>(n, f, xs, tmp_n, c, l, u, Dc, xlast, part + 296 * 5,
                                                               tickets + 1, dst + 5);
        }
        launches += 2;
    }
    void eval(bool avg, double f, double* o10) override {
        queue_eval(avg, f, out);
        CK(cudaMemcpyAsync(h_out, out, 10 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        std::memcpy(o10, h_out, 10 * sizeof(double));
    }
    void eval_pair(double f, double* cur, double* avg) override {
        queue_eval(false, 1.0, out);
        queue_eval(true, f, out + 10);
        CK(cudaMemcpyAsync(h_out, out, 20 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        std::memcpy(cur, h_out, 10 * sizeof(double));
        std::memcpy(avg, h_out + 10, 10 * sizeof(double));
    }
    void restart(bool avg, double f) override {
        k_restart<T><<<grid_for(n), 256, 0, st>>>(n, avg ? 1 : 0, f, x, xs, xlast);
        k_restart<T><<<grid_for(m), 256, 0, st>>>(m, avg ? 1 : 0, f, z, zs, zlast);
        launches += 2;
        products();
        CK(cudaGetLastError());
    }
    void download(bool avg, double f, double* hx, double* hz) override {
        if (n) {
            if (avg) k_scale_out<double><<<grid_for(n), 256, 0, st>>>(n, f, xs, hbuf);
            else k_scale_out<T><<<grid_for(n), 256, 0, st>>>(n, 1.0, x, hbuf);
            CK(cudaMemcpyAsync(hx, hbuf, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        if (m) {
            if (avg) k_scale_out<double><<<grid_for(m), 256, 0, st>>>(m, f, zs, hbuf);
            else k_scale_out<T><<<grid_for(m), 256, 0, st>>>(m, 1.0, z, hbuf);
            CK(cudaMemcpyAsync(hz, hbuf, size_t(m) * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (!rperm.empty()) {
                const std::vector<double> zm = to_model(std::vector<double>(hz, hz + m));
                std::copy(zm.begin(), zm.end(), hz);
            }
        }
        launches += 2;
        CK(cudaGetLastError());
    }
    void sync() override { CK(cudaStreamSynchronize(st)); }
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void mark() override {
        if (!ev0) {
            CK(cudaEventCreate(&ev0));
            CK(cudaEventCreate(&ev1));
        }
        CK(cudaEventRecord(ev0, st));
    }
    double elapsed_ms() override {
        CK(cudaEventRecord(ev1, st));
        CK(cudaEventSynchronize(ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        return ms;
    }
    void scaled_values(double* hDr, double* hDc, double* a_val, double* at_val) override {
        auto fetch = [&](const void* d, size_t k) {
            std::vector<T> h(k);
            if (k) CK(cudaMemcpyAsync(h.data(), d, k * sizeof(T), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            return std::vector<double>(h.begin(), h.end());
        };
        if (hDr) {
            std::vector<double> v = fetch(Dr, size_t(m));
            if (!rperm.empty()) v = to_model(v);
            std::copy(v.begin(), v.end(), hDr);
        }
        if (hDc) {
            const std::vector<double> v = fetch(Dc, size_t(n));
            std::copy(v.begin(), v.end(), hDc);
        }
        if (at_val) {
            const std::vector<double> v = fetch(AT.val, size_t(AT.nnz));
            std::copy(v.begin(), v.end(), at_val);
        }
        if (a_val) {
            const std::vector<double> v = fetch(A.val, size_t(A.nnz));
            if (rperm.empty()) {
                std::copy(v.begin(), v.end(), a_val);
            } else {  // internal row k is model row rperm[k]: place each row at its model position
                std::vector<int> ip(size_t(m) + 1);
                if (m) CK(cudaMemcpyAsync(ip.data(), A.ptr, ip.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                std::vector<int64_t> mp(size_t(m) + 1, 0);  // model-order row pointers
                for (int k = 0; k < m; ++k) mp[size_t(rperm[size_t(k)]) + 1] = ip[size_t(k) + 1] - ip[size_t(k)];
                for (int r = 0; r < m; ++r) mp[size_t(r) + 1] += mp[size_t(r)];
                for (int k = 0; k < m; ++k)
                    std::copy(v.begin() + ip[size_t(k)], v.begin() + ip[size_t(k) + 1],
                              a_val + mp[size_t(rperm[size_t(k)])]);
            }
        }
    }
    void profile_phases(int reps, double* row_ms, double* col_ms) override {
        // reps row-phase launches back to back, then reps column-phase launches, each run bracketed by events:
        // the mean includes the graph-free launch gap but not the event overhead of a single launch.
        cudaEvent_t ev[3];
        for (auto& e : ev) CK(cudaEventCreate(&e));
        CK(cudaEventRecord(ev[0], st));
        for (int s = 0; s < reps; ++s) rowblock(A, x, EpiRow<T>{Ax, z, zs, rl, ru, par});
        CK(cudaEventRecord(ev[1], st));
        for (int s = 0; s < reps; ++s) rowblock(AT, z, EpiCol<T>{ATz, x, xs, c, l, u, par, 1});
        CK(cudaEventRecord(ev[2], st));
        CK(cudaStreamSynchronize(st));
        float a, b;
        CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
        CK(cudaEventElapsedTime(&b, ev[1], ev[2]));
        for (auto& e : ev) cudaEventDestroy(e);
        *row_ms = double(a) / reps, *col_ms = double(b) / reps;
    }
};

std::unique_ptr<EngineBase> make_engine(int precision) {
    if (precision == TARAL_FP32) return std::make_unique<Engine<float>>();
    return std::make_unique<Engine<double>>();
}

void engine_init(EngineBase& e, int precision, const taral_csr& A, const taral_csr& AT, const double* c,
                 const double* l, const double* u, const double* rl, const double* ru, const double* Dr,
                 const double* Dc, int m, int n, int freq, unsigned flags) {
    if (precision == TARAL_FP32)
        static_cast<Engine<float>&>(e).init(A, AT, c, l, u, rl, ru, Dr, Dc, m, n, freq, flags);
    else
        static_cast<Engine<double>&>(e).init(A, AT, c, l, u, rl, ru, Dr, Dc, m, n, freq, flags);
}

void engine_init_model(EngineBase& e, int precision, const taral_model& md, double sign, Scaled& P, int freq,
                       unsigned flags, double* host_s) {
    if (precision == TARAL_FP32)
        static_cast<Engine<float>&>(e).init_model(md, sign, P, freq, flags, host_s);
    else
        static_cast<Engine<double>&>(e).init_model(md, sign, P, freq, flags, host_s);
}

std::string cuda_error_message(const void* exc) { return static_cast<const CudaError*>(exc)->msg; }

}  // namespace taral

// ================================================================================================ C ABI
using taral::EngineBase;

struct pdhg_ctx {
    std::unique_ptr<EngineBase> e;
    int precision = TARAL_FP64;
    bool started = false;
    std::string err;
};

static int fail(pdhg_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define GUARD(ctx, ...)                                                              \
    try {                                                                            \
        __VA_ARGS__;                                                                 \
        return TARAL_OK;                                                             \
    } catch (const taral::CudaError& ex) {                                           \
        return fail(ctx, TARAL_ERR_CUDA, ex.msg);                                    \
    } catch (const std::bad_alloc&) {                                                \
        return fail(ctx, TARAL_ERR_ALLOC, "host allocation failed");                 \
    } catch (const std::exception& ex) {                                             \
        return fail(ctx, TARAL_ERR_INPUT, ex.what());                                \
    }

static std::string check_csr(const taral_csr* a, int rows, int cols, const char* name) {
    if (!a) return std::string(name) + " is NULL";
    if (a->rows != rows || a->cols != cols) return std::string(name) + " has the wrong shape";
    if (a->nnz < 0 || a->nnz > INT32_MAX - 64) return std::string(name) + ": nnz out of the int32 range";
    if (!a->ptr || (a->nnz && (!a->idx || !a->val))) return std::string(name) + ": NULL array";
    if (a->ptr[0] != 0 || a->ptr[rows] != a->nnz) return std::string(name) + ": ptr does not span [0, nnz]";
    for (int r = 0; r < rows; ++r)
        if (a->ptr[r + 1] < a->ptr[r]) return std::string(name) + ": ptr is not monotone";
    for (int64_t k = 0; k < a->nnz; ++k)
        if (a->idx[k] < 0 || a->idx[k] >= cols) return std::string(name) + ": column index out of range";
    return "";
}

extern "C" int pdhg_create(const taral_csr* A, const taral_csr* AT, const double* c, const double* l,
                           const double* u, const double* rl, const double* ru, const double* Dr, const double* Dc,
                           int m, int n, int precision, int eval_freq, unsigned flags, pdhg_ctx** out) {
    if (!out) return TARAL_ERR_INPUT;
    *out = nullptr;
    if (m < 0 || n < 0) return TARAL_ERR_INPUT;
    if (precision != TARAL_FP64 && precision != TARAL_FP32) return TARAL_ERR_INPUT;
    if (!check_csr(A, m, n, "A").empty() || !check_csr(AT, n, m, "AT").empty() || A->nnz != AT->nnz)
        return TARAL_ERR_INPUT;
    if ((n && (!c || !l || !u || !Dc)) || (m && (!rl || !ru || !Dr))) return TARAL_ERR_INPUT;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return TARAL_ERR_NO_DEVICE;
    auto* ctx = new pdhg_ctx;
    ctx->precision = precision;
    try {
        ctx->e = taral::make_engine(precision);
        taral::engine_init(*ctx->e, precision, *A, *AT, c, l, u, rl, ru, Dr, Dc, m, n, eval_freq, flags);
    } catch (const taral::CudaError& ex) {
        std::string msg = ex.msg;
        delete ctx;
        return msg.find("cudaMalloc") != std::string::npos ? TARAL_ERR_ALLOC : TARAL_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        delete ctx;
        return TARAL_ERR_ALLOC;
    }
    *out = ctx;
    return TARAL_OK;
}

int pdhg_create_model_ctx(const taral_model* md, int precision, int eval_freq, unsigned flags, taral::Scaled& P,
                          pdhg_ctx** out) {
    *out = nullptr;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return TARAL_ERR_NO_DEVICE;
    auto* ctx = new pdhg_ctx;
    ctx->precision = precision;
    try {
        ctx->e = taral::make_engine(precision);
        taral::engine_init_model(*ctx->e, precision, *md, md->maximize ? -1.0 : 1.0, P, eval_freq, flags, nullptr);
    } catch (const taral::CudaError& ex) {
        std::string msg = ex.msg;
        delete ctx;
        return msg.find("cudaMalloc") != std::string::npos ? TARAL_ERR_ALLOC : TARAL_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        delete ctx;
        return TARAL_ERR_ALLOC;
    }
    *out = ctx;
    return TARAL_OK;
}

extern "C" int pdhg_power_norm(pdhg_ctx* ctx, int iters, double* norm_out) {
    if (!ctx || !norm_out) return TARAL_ERR_INPUT;
    GUARD(ctx, *norm_out = ctx->e->power_norm(iters))
}
extern "C" int pdhg_set_steps(pdhg_ctx* ctx, double tau, double sigma) {
    if (!ctx) return TARAL_ERR_INPUT;
    GUARD(ctx, ctx->e->set_steps(tau, sigma))
}
extern "C" int pdhg_start(pdhg_ctx* ctx, const double* x0, const double* z0) {
    if (!ctx) return TARAL_ERR_INPUT;
    GUARD(ctx, ctx->e->start(x0, z0); ctx->started = true)
}
extern "C" int pdhg_iterate(pdhg_ctx* ctx, int steps) {
    if (!ctx || steps < 0) return TARAL_ERR_INPUT;
    if (!ctx->started) return fail(ctx, TARAL_ERR_STATE, "pdhg_iterate before pdhg_start");
    GUARD(ctx, ctx->e->iterate(steps))
}
extern "C" int pdhg_eval(pdhg_ctx* ctx, int avg, double f, double out[10]) {
    if (!ctx || !out) return TARAL_ERR_INPUT;
    if (!ctx->started) return fail(ctx, TARAL_ERR_STATE, "pdhg_eval before pdhg_start");
    GUARD(ctx, ctx->e->eval(avg != 0, f, out))
}
extern "C" int pdhg_eval_pair(pdhg_ctx* ctx, double f, double cur[10], double avg[10]) {
    if (!ctx || !cur || !avg) return TARAL_ERR_INPUT;
    if (!ctx->started) return fail(ctx, TARAL_ERR_STATE, "pdhg_eval_pair before pdhg_start");
    GUARD(ctx, ctx->e->eval_pair(f, cur, avg))
}
extern "C" int pdhg_restart(pdhg_ctx* ctx, int avg, double f) {
    if (!ctx) return TARAL_ERR_INPUT;
    if (!ctx->started) return fail(ctx, TARAL_ERR_STATE, "pdhg_restart before pdhg_start");
    GUARD(ctx, ctx->e->restart(avg != 0, f))
}
extern "C" int pdhg_download(pdhg_ctx* ctx, int avg, double f, double* x, double* z) {
    if (!ctx || !x || !z) return TARAL_ERR_INPUT;
    GUARD(ctx, ctx->e->download(avg != 0, f, x, z))
}
extern "C" int pdhg_solve_ctx(pdhg_ctx* ctx, double bnorm, double cnorm, const taral_options* o, const double* x0,
                              const double* z0, taral_outcome* out, double* x, double* z) {
    if (!ctx || !o || !out) return TARAL_ERR_INPUT;
    std::memset(out, 0, sizeof *out);
    taral::Options op;
    op.tol = o->tol, op.time_limit = o->time_limit, op.max_iter = o->max_iter;
    op.eval_freq = o->eval_freq > 0 ? o->eval_freq : 64, op.row_rel = o->row_rel, op.verbose = o->verbose != 0;
    EngineBase& e = *ctx->e;
    taral::DriverData P{int(e.hrl.size()), int(e.hc.size()), e.hc.data(), e.hrl.data(), e.hru.data(), bnorm, cnorm};
    GUARD(ctx, {
        int64_t l0 = e.launches;
        auto t0 = taral::Clock::now();
        e.mark();
        taral::Outcome r = taral::run(e, P, op, op.time_limit, x0, z0);
        out->device_s = e.elapsed_ms() * 1e-3;
        out->solve_s = taral::since(t0);
        ctx->started = true;
        out->status = r.status, out->iterations = r.iterations, out->restarts = r.restarts;
        out->from_average = r.from_average ? 1 : 0;
        out->rel_primal = r.rel_primal, out->rel_dual = r.rel_dual, out->rel_gap = r.rel_gap;
        out->norm_a = r.norm_a, out->primal_weight = r.omega, out->power_iter_s = r.power_s;
        out->device_mem_bytes = e.mem_used, out->kernel_launches = e.launches - l0;
        if (x) std::memcpy(x, r.x.data(), r.x.size() * sizeof(double));
        if (z) std::memcpy(z, r.z.data(), r.z.size() * sizeof(double));
    })
}

extern "C" int pdhg_profile_phases(pdhg_ctx* ctx, int reps, double* row_ms, double* col_ms) {
    if (!ctx || reps <= 0 || !row_ms || !col_ms) return TARAL_ERR_INPUT;
    if (!ctx->started) return fail(ctx, TARAL_ERR_STATE, "pdhg_profile_phases before pdhg_start");
    GUARD(ctx, ctx->e->profile_phases(reps, row_ms, col_ms))
}

extern "C" int pdhg_info(pdhg_ctx* ctx, char* name_out, size_t cap, size_t* mem_used) {
    if (!ctx) return TARAL_ERR_INPUT;
    if (name_out && cap) {
        std::snprintf(name_out, cap, "%s", ctx->e->name.c_str());
    }
    if (mem_used) *mem_used = ctx->e->mem_used;
    return TARAL_OK;
}
extern "C" int pdhg_scaled_problem(pdhg_ctx* ctx, double* Dr, double* Dc, double* A_val, double* AT_val) {
    if (!ctx) return TARAL_ERR_INPUT;
    GUARD(ctx, ctx->e->scaled_values(Dr, Dc, A_val, AT_val))
}
extern "C" int64_t pdhg_kernel_launches(const pdhg_ctx* ctx) { return ctx ? ctx->e->launches : 0; }
extern "C" const char* pdhg_last_error(const pdhg_ctx* ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }
extern "C" void pdhg_destroy(pdhg_ctx* ctx) { delete ctx; }
extern "C" void taral_set_device_alloc_limit(size_t bytes) { taral::g_alloc_limit.store(bytes); }

// ================================================================================================ SpMV plan
struct taral_spmv_plan {
    int rows = 0, cols = 0, dtype = TARAL_FP64, nblk = 0;
    bool per_thread = false;  // every row holds at most kShort nonzeros: k_rowthread (bit-identical, no staging)
    int4* blk = nullptr;
};

extern "C" int taral_spmv_plan_create(int rows, int cols, const int64_t* host_ptr, int dtype, taral_spmv_plan** out) {
    if (!out || rows < 0 || cols < 0 || !host_ptr) return TARAL_ERR_INPUT;
    if (dtype != TARAL_FP64 && dtype != TARAL_FP32) return TARAL_ERR_INPUT;
    *out = nullptr;
    for (int r = 0; r < rows; ++r)
        if (host_ptr[r + 1] < host_ptr[r]) return TARAL_ERR_INPUT;
    if (host_ptr[rows] > INT32_MAX - 64) return TARAL_ERR_INPUT;
    std::vector<int4> blk = taral::build_row_blocks(host_ptr, rows);
    const int forced = taral::forced_row_split();  // tests
    if (forced > 0) taral::apply_row_split(blk, forced);
    int64_t maxrow = 0;
    for (int r = 0; r < rows; ++r) maxrow = std::max<int64_t>(maxrow, host_ptr[r + 1] - host_ptr[r]);
    const char* rt = std::getenv("TARAL_ROWTHREAD");
    auto* p = new taral_spmv_plan;
    p->rows = rows, p->cols = cols, p->dtype = dtype, p->nblk = int(blk.size());
    p->per_thread = maxrow <= taral::kShort && forced <= 0 && !(rt && std::atoi(rt) == 0);
    if (cudaMalloc(&p->blk, std::max<size_t>(blk.size(), 1) * sizeof(int4)) != cudaSuccess) {
        delete p;
        return TARAL_ERR_ALLOC;
    }
    if (!blk.empty() &&
        cudaMemcpy(p->blk, blk.data(), blk.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(p->blk);
        delete p;
        return TARAL_ERR_CUDA;
    }
    *out = p;
    return TARAL_OK;
}

template <class T>
static void spmv_launch(const taral_spmv_plan* p, const int* ptr, const int* idx, const void* val, const void* x,
                        void* y, cudaStream_t s) {
    using namespace taral;
    bool vec = (reinterpret_cast<uintptr_t>(idx) % 16 == 0) && (reinterpret_cast<uintptr_t>(val) % 16 == 0);
    EpiStore<T> e{static_cast<T*>(y)};
    if (p->per_thread)
        k_rowthread<T, T, EpiStore<T>><<<(p->rows + kThreads - 1) / kThreads, kThreads, 0, s>>>(
            p->rows, ptr, idx, static_cast<const T*>(val), static_cast<const T*>(x), nullptr, e);
    else if (vec)
        k_rowblock<T, T, EpiStore<T>, true><<<p->nblk, kThreads, 0, s>>>(ptr, idx, static_cast<const T*>(val),
                                                                          static_cast<const T*>(x), p->blk, nullptr, e);
    else
        k_rowblock<T, T, EpiStore<T>, false><<<p->nblk, kThreads, 0, s>>>(ptr, idx, static_cast<const T*>(val),
                                                                           static_cast<const T*>(x), p->blk, nullptr, e);
}

extern "C" int taral_spmv_run(const taral_spmv_plan* p, const int32_t* d_ptr, const int32_t* d_idx, const void* d_val,
                              const void* d_x, void* d_y, void* stream) {
    if (!p || !d_ptr || !d_x || !d_y) return TARAL_ERR_INPUT;
    if (p->nblk == 0) return TARAL_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (p->dtype == TARAL_FP32) spmv_launch<float>(p, d_ptr, d_idx, d_val, d_x, d_y, s);
    else spmv_launch<double>(p, d_ptr, d_idx, d_val, d_x, d_y, s);
    return cudaGetLastError() == cudaSuccess ? TARAL_OK : TARAL_ERR_CUDA;
}
extern "C" int taral_spmv_plan_blocks(const taral_spmv_plan* p) { return p ? p->nblk : 0; }
extern "C" void taral_spmv_plan_destroy(taral_spmv_plan* p) {
    if (!p) return;
    cudaFree(p->blk);
    delete p;
}
