// Host preprocessing: the CSR transposes of the model (gpu/pdhg.cu:55-70 semantics), the scaled vectors and norms
// (gpu/pdhg.cu:113-133) given the scaling factors computed on the device (scaling.cuh), and the original-space check
// of an answer (gpu/pdhg.cu:866-876).
#include <algorithm>
#include <cmath>
#include <thread>

#include "host.hpp"

namespace taral {

// CSR transpose by counting sort (gpu/pdhg.cu:55-70 semantics: rows of the output ascending), the scatter split
// over threads by ranges of output rows: every thread reads the whole input in order and writes only its own rows,
// so each output row is filled in the sequential order and the result does not depend on the thread count.
Csr transpose_par(const int64_t* ptr, const int32_t* idx, const double* val, int rows, int cols, int threads) {
    Csr t;
    t.rows = cols;
    const int64_t nnz = ptr[rows] - ptr[0];
    t.ptr.assign(size_t(cols) + 1, 0);
    for (int64_t k = ptr[0]; k < ptr[rows]; ++k) t.ptr[size_t(idx[k]) + 1]++;
    for (int j = 0; j < cols; ++j) t.ptr[j + 1] += t.ptr[j];
    t.idx.resize(size_t(nnz));
    t.val.resize(size_t(nnz));
    threads = int(std::max<int64_t>(1, std::min<int64_t>(threads, nnz / 65536)));
    std::vector<int> cut(size_t(threads) + 1, cols);  // output rows [cut[q], cut[q+1]) belong to thread q
    cut[0] = 0;
    for (int q = 1; q < threads; ++q)
        cut[q] = int(std::lower_bound(t.ptr.begin(), t.ptr.end(), nnz * q / threads) - t.ptr.begin());
    for (int q = 1; q <= threads; ++q) cut[q] = std::max(cut[q], cut[q - 1]);
    auto work = [&](int q) {
        const int lo = cut[q], hi = cut[q + 1];
        if (lo >= hi) return;
        std::vector<int64_t> pos(t.ptr.begin() + lo, t.ptr.begin() + hi);
        for (int i = 0; i < rows; ++i)
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
                const int j = idx[k];
                if (j < lo || j >= hi) continue;
                const int64_t p = pos[j - lo]++;
                t.idx[p] = i, t.val[p] = val[k];
            }
    };
    std::vector<std::thread> pool;
    for (int q = 1; q < threads; ++q) pool.emplace_back(work, q);
    work(0);
    for (auto& th : pool) th.join();
    return t;
}

int host_threads() {
    const unsigned h = std::thread::hardware_concurrency();
    return int(std::max(1u, std::min(h, 16u)));
}

void model_matrices(const taral_model& md, Csr& A, Csr& AT, int threads) {
    if (threads <= 0) threads = host_threads();
    const int64_t k0 = md.col_ptr[0], k1 = md.col_ptr[md.n];
    bool zeros = false;
    for (int64_t k = k0; k < k1 && !zeros; ++k) zeros = md.val[k] == 0;
    if (!zeros) {
        A = transpose_par(md.col_ptr, md.row_idx, md.val, md.n, md.m, threads);
    } else {  // drop explicit zeros first (the column-wise copy the reference builds)
        Csr T;
        T.rows = md.n;
        T.ptr.assign(size_t(md.n) + 1, 0);
        for (int j = 0; j < md.n; ++j) {
            for (int64_t k = md.col_ptr[j]; k < md.col_ptr[j + 1]; ++k)
                if (md.val[k] != 0) T.idx.push_back(md.row_idx[k]), T.val.push_back(md.val[k]);
            T.ptr[j + 1] = int64_t(T.idx.size());
        }
        A = transpose_par(T.ptr.data(), T.idx.data(), T.val.data(), md.n, md.m, threads);
    }
    // A^T = transpose(A) has ascending row indices in every column; a model whose columns already list their rows
    // in ascending order with no explicit zero is that matrix as it stands
    bool sorted = !zeros;
    for (int j = 0; j < md.n && sorted; ++j)
        for (int64_t k = md.col_ptr[j] + 1; k < md.col_ptr[j + 1] && sorted; ++k) sorted = md.row_idx[k - 1] < md.row_idx[k];
    if (sorted) {
        AT.rows = md.n;
        AT.ptr.assign(md.col_ptr, md.col_ptr + md.n + 1);
        for (int64_t& v : AT.ptr) v -= k0;
        AT.idx.assign(md.row_idx + k0, md.row_idx + k1);
        AT.val.assign(md.val + k0, md.val + k1);
    } else {
        AT = transpose_par(A.ptr.data(), A.idx.data(), A.val.data(), md.m, md.n, threads);
    }
}

void scale_vectors(const taral_model& md, double sign, const std::vector<double>& Dr, const std::vector<double>& Dc,
                   Scaled& P) {
    P.m = md.m, P.n = md.n;
    P.c.resize(size_t(P.n)), P.l.resize(size_t(P.n)), P.u.resize(size_t(P.n));
    P.rl.resize(size_t(P.m)), P.ru.resize(size_t(P.m));
    P.cnorm = P.bnorm = 0;
    for (int j = 0; j < P.n; ++j) {
        double c = sign * md.cost[j];
        P.cnorm += c * c;
        P.c[j] = c * Dc[j], P.l[j] = md.col_lo[j] / Dc[j], P.u[j] = md.col_up[j] / Dc[j];
    }
    for (int i = 0; i < P.m; ++i) {
        double lo = md.row_lo[i], up = md.row_up[i], b = 0;
        if (std::isfinite(lo) && std::isfinite(up)) b = std::max(std::fabs(lo), std::fabs(up));
        else if (std::isfinite(lo)) b = std::fabs(lo);
        else if (std::isfinite(up)) b = std::fabs(up);
        P.bnorm += b * b;
        P.rl[i] = lo * Dr[i], P.ru[i] = up * Dr[i];
    }
    P.bnorm = std::sqrt(P.bnorm), P.cnorm = std::sqrt(P.cnorm);
}

Finished finish_point(const taral_model& md, const Scaled& P, const Outcome& r) {
    Finished f;
    f.x.resize(size_t(P.n));
    f.y.resize(size_t(P.m));
    for (int j = 0; j < P.n; ++j) f.x[j] = r.x[j] * P.Dc[j];
    for (int i = 0; i < P.m; ++i) f.y[i] = P.Dr[i] * r.z[i];
    long double obj = md.obj_const;
    for (int j = 0; j < P.n; ++j) obj += (long double)md.cost[j] * f.x[j];
    double bviol = 0, rviol = 0;
    bool finite = true;
    for (int j = 0; j < P.n; ++j) {
        bviol = std::max(bviol, std::max(md.col_lo[j] - f.x[j], f.x[j] - md.col_up[j]));
        finite = finite && std::isfinite(f.x[j]);
    }
    if (finite && P.a_original && P.m > 0) {
        // Row activities from the unscaled row-wise copy: each row lists its entries in ascending column order, so
        // its sequential sum adds the same products in the same order as the column sweep below (explicit zeros
        // add nothing for finite x). Rows are split over threads; the maximum does not depend on the split.
        const int nt = std::max(1, std::min(host_threads(), P.m / 4096));
        std::vector<double> part(size_t(nt), 0.0);
        auto work = [&](int q) {
            const int i0 = int(int64_t(P.m) * q / nt), i1 = int(int64_t(P.m) * (q + 1) / nt);
            double v = 0;
            for (int i = i0; i < i1; ++i) {
                double a = 0.0;
                for (int64_t k = P.A.ptr[i]; k < P.A.ptr[i + 1]; ++k) a += P.A.val[k] * f.x[P.A.idx[k]];
                v = std::max(v, std::max(md.row_lo[i] - a, a - md.row_up[i]));
            }
            part[q] = v;
        };
        std::vector<std::thread> pool;
        for (int q = 1; q < nt; ++q) pool.emplace_back(work, q);
        work(0);
        for (auto& th : pool) th.join();
        for (double v : part) rviol = std::max(rviol, v);
    } else {
        std::vector<double> ax(size_t(P.m), 0.0);
        for (int j = 0; j < P.n; ++j)
            for (int64_t k = md.col_ptr[j]; k < md.col_ptr[j + 1]; ++k) ax[md.row_idx[k]] += md.val[k] * f.x[j];
        for (int i = 0; i < P.m; ++i) rviol = std::max(rviol, std::max(md.row_lo[i] - ax[i], ax[i] - md.row_up[i]));
    }
    f.objective = double(obj), f.max_row_violation = rviol, f.max_bound_violation = bviol;
    return f;
}

const char* status_name(int s) {
    switch (s) {
        case TARAL_NEAR_OPTIMAL: return "near_optimal";
        case TARAL_TIME_LIMIT: return "time_limit";
        case TARAL_NUMERICAL_FAILURE: return "numerical_failure";
        default: return "iteration_limit";
    }
}

}  // namespace taral
