// Independent FP64 check of answers on the ORIGINAL models, on the device, over many models at once
// (include/taral_pdhg.h, part 8). Semantics of the reference's checker: the primal side of
// benchmarks/orig_check.py:63-88 (objective with the objective row's constant, the largest row violation relative to
// 1 + |b| with b the row's right-hand side, the largest bound violation) and the weak-duality bound of
// gpu/vector_check.py:46-74 (for y and -y: LB = const + sum_i min_{r in [lo_i, up_i]} y_i r + sum_j min_{x in [l_j,
// u_j]} d_j x, d = c - A'y; a term whose minimising bound is infinite -- |v| >= 1e20 -- is dropped and its size kept
// as dual infeasibility, |y_i| / (1 + |y_i|) for rows, |d_j| / (1 + |c_j|) for columns; the sign with the smaller
// largest dropped term is kept; minimisation models only). Shares no code with the solver: the models are uploaded
// unscaled in FP64, rows are summed from a row-wise copy and A'y from the model's own columns, each sequentially.
//
// One CTA takes 256 rows (or columns) of one model; its partial results (maxima, sums, dropped-term counts) are
// combined per model in CTA order by one thread: deterministic for a given input.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/taral_pdhg.h"
#include "engine.hpp"
#include "host.hpp"
#include "solve.hpp"

namespace taral {
namespace {

constexpr int kCT = 256;       // threads per CTA, rows / columns per CTA
constexpr double kBig = 1e20;  // the checker's infinity
constexpr int kParts = 8;

struct CheckError {
    std::string msg;
};
#define VK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) throw CheckError{std::string(#call) + ": " + cudaGetErrorString(e_)};       \
    } while (0)

// min over [lo, up] of coef * v: the value, or `dropped` with the coefficient's size when the bound is infinite
__device__ __forceinline__ double min_over(double coef, double lo, double up, bool& dropped) {
    dropped = false;
    if (coef == 0) return 0.0;
    const double v = coef > 0 ? lo : up;
    if (fabs(v) >= kBig) {
        dropped = true;
        return 0.0;
    }
    return coef * v;
}

// Block reduction of kParts values, slot k by op[k] (0 sum, 1 max), fixed order; thread 0 writes dst.
__device__ void reduce_parts(double (&v)[kParts], const int (&op)[kParts], double* dst) {
    __shared__ double sh[kParts][kCT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kParts; ++k) {
        double s = v[k];
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, s, off);
            s = op[k] ? (o > s ? o : s) : s + o;
        }
        if (lane == 0) sh[k][w] = s;
    }
    __syncthreads();
    if (threadIdx.x < kParts) {
        const int k = threadIdx.x;
        double s = sh[k][0];
        for (int i = 1; i < kCT / 32; ++i) s = op[k] ? (sh[k][i] > s ? sh[k][i] : s) : s + sh[k][i];
        dst[k] = s;
    }
}

// Per-CTA work item: {model, first row (or column) of the model, count, matrix}
struct Item {
    int model, first, count, mat;
};

struct Dev {  // device pointers of one model's data inside the concatenated arrays
    long long row0, col0;  // offsets of its rows / columns in the concatenated vectors
    int has_y, pad;
};

struct Mat {  // device pointers of one distinct matrix
    const int *rptr, *ridx, *cptr, *cidx;
    const double *rval, *cval;
};

// rows: act = a_i x, row violation, row dual terms for +y and -y
// parts: 0 max row violation, 1 sum t+, 2 sum t-, 3 max dropped+ , 4 max dropped-, 5 n dropped+, 6 n dropped-
__global__ void __launch_bounds__(kCT) k_check_rows(const Item* __restrict__ items, const Dev* __restrict__ dev,
                                                    const Mat* __restrict__ mats, const double* __restrict__ x,
                                                    const double* __restrict__ y, const double* __restrict__ lo,
                                                    const double* __restrict__ up, const double* __restrict__ b,
                                                    double* parts) {
    const Item it = items[blockIdx.x];
    const Dev d = dev[it.model];
    const Mat mt = mats[it.mat];
    double v[kParts] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int r = it.first + int(threadIdx.x);
    if (int(threadIdx.x) < it.count) {
        const long long g = d.row0 + r;
        double act = 0;
        for (int k = mt.rptr[r]; k < mt.rptr[r + 1]; ++k) act += mt.rval[k] * x[d.col0 + mt.ridx[k]];
        const double l = lo[g], u = up[g];
        double viol = l - act;
        viol = act - u > viol ? act - u : viol;
        v[0] = (viol > 0 ? viol : 0.0) / (1.0 + fabs(b[g]));
        if (d.has_y) {
            const double yi = y[g];
            bool dp, dm;
            const double tp = min_over(yi, l, u, dp), tm = min_over(-yi, l, u, dm);
            const double rel = fabs(yi) / (1.0 + fabs(yi));
            v[1] = tp, v[2] = tm;
            v[3] = dp ? rel : 0.0, v[4] = dm ? rel : 0.0, v[5] = dp, v[6] = dm;
        }
    }
    const int op[kParts] = {1, 0, 0, 1, 1, 0, 0, 0};
    reduce_parts(v, op, parts + size_t(blockIdx.x) * kParts);
}

// columns: objective, bound violation, column dual terms with d = c -+ A'y
// parts: 0 max bound violation, 1 sum c x, 2 sum t+, 3 sum t-, 4 max dropped+, 5 max dropped-, 6 n+, 7 n-
__global__ void __launch_bounds__(kCT) k_check_cols(const Item* __restrict__ items, const Dev* __restrict__ dev,
                                                    const Mat* __restrict__ mats, const double* __restrict__ x,
                                                    const double* __restrict__ y, const double* __restrict__ c,
                                                    const double* __restrict__ l, const double* __restrict__ u,
                                                    double* parts) {
    const Item it = items[blockIdx.x];
    const Dev d = dev[it.model];
    const Mat mt = mats[it.mat];
    double v[kParts] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int j = it.first + int(threadIdx.x);
    if (int(threadIdx.x) < it.count) {
        const long long g = d.col0 + j;
        const double xj = x[g], cj = c[g], lj = l[g], uj = u[g];
        double bv = lj - xj;
        bv = xj - uj > bv ? xj - uj : bv;
        v[0] = bv > 0 ? bv : 0.0;
        v[1] = cj * xj;
        if (d.has_y) {
            double aty = 0;
            for (int k = mt.cptr[j]; k < mt.cptr[j + 1]; ++k) aty += mt.cval[k] * y[d.row0 + mt.cidx[k]];
            bool dp, dm;
            const double ep = cj - aty, em = cj + aty;  // d for +y and for -y
            v[2] = min_over(ep, lj, uj, dp), v[3] = min_over(em, lj, uj, dm);
            v[4] = dp ? fabs(ep) / (1.0 + fabs(cj)) : 0.0, v[5] = dm ? fabs(em) / (1.0 + fabs(cj)) : 0.0;
            v[6] = dp, v[7] = dm;
        }
    }
    const int op[kParts] = {1, 0, 0, 0, 1, 1, 0, 0};
    reduce_parts(v, op, parts + size_t(blockIdx.x) * kParts);
}

// One thread per model: its CTAs' partials in order.
__global__ void k_check_finish(int count, const int* __restrict__ rr, const int* __restrict__ cr,
                               const double* __restrict__ prow, const double* __restrict__ pcol,
                               const double* __restrict__ cst, const int* __restrict__ dual, taral_check* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double rv = 0, bv = 0, obj = 0, sp = 0, sm = 0, ip = 0, im = 0, np_ = 0, nm = 0;
    for (int b = rr[i]; b < rr[i + 1]; ++b) {
        const double* p = prow + size_t(b) * kParts;
        rv = p[0] > rv ? p[0] : rv;
        sp += p[1], sm += p[2];
        ip = p[3] > ip ? p[3] : ip, im = p[4] > im ? p[4] : im;
        np_ += p[5], nm += p[6];
    }
    for (int b = cr[i]; b < cr[i + 1]; ++b) {
        const double* p = pcol + size_t(b) * kParts;
        bv = p[0] > bv ? p[0] : bv;
        obj += p[1], sp += p[2], sm += p[3];
        ip = p[4] > ip ? p[4] : ip, im = p[5] > im ? p[5] : im;
        np_ += p[6], nm += p[7];
    }
    taral_check r;
    r.objective = obj + cst[i], r.row_violation_rel = rv, r.bound_violation = bv;
    r.dual_bound = r.dual_obj_loose = r.dual_infeas_rel = r.dual_gap_rel = nan("");
    r.dual_sign = 0, r.pad = 0;
    if (dual[i]) {
        const bool plus = ip <= im;  // the reference keeps +y unless -y has strictly smaller infeasibility
        const double lb = cst[i] + (plus ? sp : sm);
        r.dual_sign = plus ? 1 : -1;
        r.dual_infeas_rel = plus ? ip : im;
        r.dual_obj_loose = lb;
        r.dual_bound = (plus ? np_ : nm) == 0 ? lb : nan("");
        const double ao = fabs(r.objective);
        r.dual_gap_rel = (r.objective - lb) / (ao > 1.0 ? ao : 1.0);
    }
    out[i] = r;
}

void check_models(const taral_model* md, int count, const double* const* rhs, const double* const* xs,
                  const double* const* ys, taral_check* out) {
    int dev = 0;
    VK(cudaGetDevice(&dev));
    keep_pool_memory(dev);
    cudaStream_t s;
    VK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::vector<void*> bufs;
    struct Release {
        std::vector<void*>& b;
        cudaStream_t s;
        ~Release() {
            for (void* p : b) cudaFreeAsync(p, s);
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } release{bufs, s};
    auto put = [&](const void* h, size_t bytes) {
        void* p = nullptr;
        VK(cudaMallocAsync(&p, std::max<size_t>(bytes, 8), s));
        bufs.push_back(p);
        if (bytes) VK(cudaMemcpyAsync(p, h, bytes, cudaMemcpyHostToDevice, s));
        return p;
    };
    // distinct matrices: the same arrays in more than one model are uploaded once
    std::map<std::tuple<const void*, const void*, const void*, int, int>, int> seen;
    std::vector<int> mat_of(static_cast<size_t>(count));
    std::vector<Mat> hmats;
    std::vector<std::vector<int>> keep;  // host staging kept alive until the copies are done
    std::vector<std::vector<double>> keepd;
    for (int i = 0; i < count; ++i) {
        const taral_model& m = md[i];
        const auto key = std::make_tuple((const void*)m.col_ptr, (const void*)m.row_idx, (const void*)m.val, m.m, m.n);
        auto it = seen.find(key);
        if (it != seen.end()) {
            mat_of[i] = it->second;
            continue;
        }
        Csr A, AT;
        model_matrices(m, A, AT);  // row-wise copy (zeros dropped: they add nothing to a row activity)
        Mat mt;
        keep.emplace_back(A.ptr.begin(), A.ptr.end());
        mt.rptr = static_cast<const int*>(put(keep.back().data(), keep.back().size() * sizeof(int)));
        mt.ridx = static_cast<const int*>(put(A.idx.data(), A.idx.size() * sizeof(int)));
        mt.rval = static_cast<const double*>(put(A.val.data(), A.val.size() * sizeof(double)));
        keep.emplace_back(m.col_ptr, m.col_ptr + m.n + 1);  // the model's own columns, as given
        mt.cptr = static_cast<const int*>(put(keep.back().data(), keep.back().size() * sizeof(int)));
        const int64_t nz = m.col_ptr[m.n];
        mt.cidx = static_cast<const int*>(put(m.row_idx, size_t(nz) * sizeof(int)));
        mt.cval = static_cast<const double*>(put(m.val, size_t(nz) * sizeof(double)));
        VK(cudaStreamSynchronize(s));  // A's host vectors go out of scope
        const int id = int(hmats.size());
        hmats.push_back(mt);
        seen[key] = id;
        mat_of[i] = id;
    }
    // concatenated vectors and work items
    int64_t M = 0, N = 0;
    for (int i = 0; i < count; ++i) M += md[i].m, N += md[i].n;
    const size_t nN = static_cast<size_t>(N), nM = static_cast<size_t>(M), nC = static_cast<size_t>(count);
    std::vector<double> hx(nN), hy(nM, 0.0), hc(nN), hl(nN), hu(nN), hlo(nM), hup(nM), hb(nM), hcst(nC);
    std::vector<int> hdual(nC), hrr{0}, hcr{0};
    std::vector<Dev> hdev(nC);
    std::vector<Item> rows, cols;
    int64_t r0 = 0, c0 = 0;
    for (int i = 0; i < count; ++i) {
        const taral_model& m = md[i];
        hdev[i] = {r0, c0, ys && ys[i] ? 1 : 0, 0};
        hdual[i] = ys && ys[i] && !m.maximize ? 1 : 0;
        hcst[i] = m.obj_const;
        for (int j = 0; j < m.n; ++j)
            hx[c0 + j] = xs[i][j], hc[c0 + j] = m.cost[j], hl[c0 + j] = m.col_lo[j], hu[c0 + j] = m.col_up[j];
        for (int r = 0; r < m.m; ++r) {
            const double lo = m.row_lo[r], up = m.row_up[r];
            hlo[r0 + r] = lo, hup[r0 + r] = up;
            hb[r0 + r] = rhs && rhs[i] ? rhs[i][r] : (std::isfinite(lo) ? lo : up);
            if (ys && ys[i]) hy[r0 + r] = ys[i][r];
        }
        for (int a = 0; a < m.m; a += kCT) rows.push_back({i, a, std::min(kCT, m.m - a), mat_of[i]});
        for (int a = 0; a < m.n; a += kCT) cols.push_back({i, a, std::min(kCT, m.n - a), mat_of[i]});
        hrr.push_back(int(rows.size())), hcr.push_back(int(cols.size()));
        r0 += m.m, c0 += m.n;
    }
    auto dput = [&](const auto& v) { return put(v.data(), v.size() * sizeof(v[0])); };
    const double *dx = (const double*)dput(hx), *dy = (const double*)dput(hy), *dc = (const double*)dput(hc),
                 *dl = (const double*)dput(hl), *du = (const double*)dput(hu), *dlo = (const double*)dput(hlo),
                 *dup = (const double*)dput(hup), *db = (const double*)dput(hb), *dcst = (const double*)dput(hcst);
    const int *ddual = (const int*)dput(hdual), *drr = (const int*)dput(hrr), *dcr = (const int*)dput(hcr);
    const Dev* ddev = (const Dev*)dput(hdev);
    const Mat* dmats = (const Mat*)dput(hmats);
    const Item *drows = (const Item*)dput(rows), *dcols = (const Item*)dput(cols);
    std::vector<double> zeros((rows.size() + cols.size()) * kParts + 2 * kParts, 0.0);
    double* parts = (double*)dput(zeros);
    double *prow = parts, *pcol = parts + rows.size() * kParts;
    taral_check* dout = nullptr;
    VK(cudaMallocAsync(reinterpret_cast<void**>(&dout), size_t(count) * sizeof(taral_check), s));
    bufs.push_back(dout);
    if (!rows.empty()) k_check_rows<<<int(rows.size()), kCT, 0, s>>>(drows, ddev, dmats, dx, dy, dlo, dup, db, prow);
    if (!cols.empty()) k_check_cols<<<int(cols.size()), kCT, 0, s>>>(dcols, ddev, dmats, dx, dy, dc, dl, du, pcol);
    k_check_finish<<<(count + 127) / 128, 128, 0, s>>>(count, drr, dcr, prow, pcol, dcst, ddual, dout);
    VK(cudaGetLastError());
    VK(cudaMemcpyAsync(out, dout, size_t(count) * sizeof(taral_check), cudaMemcpyDeviceToHost, s));
    VK(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace taral

extern "C" int taral_check_models(const taral_model* models, int count, const double* const* rhs,
                                  const double* const* x, const double* const* y, taral_check* out) {
    if (!models || count <= 0 || !x || !out) return TARAL_ERR_INPUT;
    for (int i = 0; i < count; ++i) {
        if (!x[i] || !taral::check_model(models[i]).empty()) return TARAL_ERR_INPUT;
        if (models[i].m > (1 << 30) || models[i].n > (1 << 30)) return TARAL_ERR_INPUT;
    }
    int devs = 0;
    if (cudaGetDeviceCount(&devs) != cudaSuccess || devs == 0) return TARAL_ERR_NO_DEVICE;
    try {
        taral::check_models(models, count, rhs, x, y, out);
    } catch (const taral::CheckError& e) {
        return e.msg.find("cudaMalloc") != std::string::npos ? TARAL_ERR_ALLOC : TARAL_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        return TARAL_ERR_ALLOC;
    }
    return TARAL_OK;
}
