// Host preprocessing: the CSR transposes of the model (gpu/pdhg.cu:55-70 semantics), the scaled vectors and norms
// (gpu/pdhg.cu:113-133 semantics) given the scaling factors computed on the device (scaling.cuh), and the
// original-space check of an answer (gpu/pdhg.cu:866-876 semantics).
#include <algorithm>
#include <cmath>
#include <thread>

#include "host.hpp"

namespace taral {

// CSR transpose by counting sort (gpu/pdhg.cu:55-70 semantics: rows of the output ascending). The input rows are
// cut into ranges of about equal nonzeros, one per thread; every range counts its entries per output row, each
// range's entries of an output row follow those of the ranges before it, and every range scatters its own entries:
// each output row is filled in the sequential order, so the result does not depend on the thread count.
Csr transpose_par(const int64_t* ptr, const int32_t* idx, const double* val, int rows, int cols, int threads) {
    Csr t;
    t.rows = cols;
    const int64_t nnz = ptr[rows] - ptr[0];
    t.ptr.assign(size_t(cols) + 1, 0);
    t.idx.resize(size_t(nnz));
    t.val.resize(size_t(nnz));
    const int parts = int(std::max<int64_t>(1, std::min<int64_t>(threads, nnz / 65536)));
    std::vector<int> cut(size_t(parts) + 1, rows);  // input rows [cut[q], cut[q+1]) form range q
    cut[0] = 0;
    for (int q = 1; q < parts; ++q)
        cut[q] = int(std::lower_bound(ptr, ptr + rows + 1, ptr[0] + nnz * q / parts) - ptr);
    for (int q = 1; q <= parts; ++q) cut[q] = std::max(cut[q], cut[q - 1]);
    // slot[q][j]: range q's count of output row j, then the offset of its first entry inside that row
    // (allocated here, so that an allocation failure reaches the caller rather than a worker thread)
    std::vector<std::vector<int32_t>> slot(static_cast<size_t>(parts), std::vector<int32_t>(size_t(cols), 0));
    split_ranges(parts, parts, [&](int, int64_t q0, int64_t q1) {
        for (int64_t q = q0; q < q1; ++q) {
            std::vector<int32_t>& c = slot[size_t(q)];
            for (int64_t k = ptr[cut[q]]; k < ptr[cut[q + 1]]; ++k) c[size_t(idx[k])]++;
        }
    });
    split_ranges(cols, threads, [&](int, int64_t j0, int64_t j1) {
        for (int64_t j = j0; j < j1; ++j) {
            int32_t run = 0;
            for (int q = 0; q < parts; ++q) {
                const int32_t c = slot[size_t(q)][size_t(j)];
                slot[size_t(q)][size_t(j)] = run;
                run += c;
            }
            t.ptr[size_t(j) + 1] = run;
        }
    });
    for (int j = 0; j < cols; ++j) t.ptr[size_t(j) + 1] += t.ptr[size_t(j)];
    split_ranges(parts, parts, [&](int, int64_t q0, int64_t q1) {
        for (int64_t q = q0; q < q1; ++q) {
            std::vector<int32_t>& c = slot[size_t(q)];
            for (int i = cut[q]; i < cut[q + 1]; ++i)
                for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
                    const int j = idx[k];
                    const int64_t p = t.ptr[size_t(j)] + c[size_t(j)]++;
                    t.idx[size_t(p)] = i, t.val[size_t(p)] = val[k];
                }
        }
    });
    return t;
}

int host_threads() {
    const unsigned h = std::thread::hardware_concurrency();
    return int(std::max(1u, std::min(h, 16u)));
}

CsrRef model_matrices_ref(const taral_model& md, Csr& A, Csr& AT, int threads) {
    if (threads <= 0) threads = host_threads();
    const int64_t k0 = md.col_ptr[0];
    // explicit zeros and the row order inside the columns, checked over column ranges in parallel
    std::vector<char> zero(size_t(threads), 0), unsorted(size_t(threads), 0);
    split_ranges(md.n, threads, [&](int q, int64_t j0, int64_t j1) {
        bool z = false, u = false;
        for (int64_t j = j0; j < j1 && !z; ++j)
            for (int64_t k = md.col_ptr[j]; k < md.col_ptr[j + 1]; ++k) {
                z = z || md.val[k] == 0;
                u = u || (k > md.col_ptr[j] && md.row_idx[k - 1] >= md.row_idx[k]);
            }
        zero[size_t(q)] = z, unsorted[size_t(q)] = u;
    });
    const bool zeros = std::find(zero.begin(), zero.end(), 1) != zero.end();
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
    // A^T = transpose(A) has ascending row indices in every column: a model whose columns already list their rows
    // in ascending order with no explicit zero is that matrix as it stands
    const bool sorted = !zeros && std::find(unsorted.begin(), unsorted.end(), 1) == unsorted.end();
    AT = Csr();
    if (sorted && k0 == 0) return {md.n, md.col_ptr, md.row_idx, md.val};
    if (sorted) {
        AT.rows = md.n;
        AT.ptr.assign(md.col_ptr, md.col_ptr + md.n + 1);
        for (int64_t& v : AT.ptr) v -= k0;
        AT.idx.assign(md.row_idx + k0, md.row_idx + md.col_ptr[md.n]);
        AT.val.assign(md.val + k0, md.val + md.col_ptr[md.n]);
    } else {
        AT = transpose_par(A.ptr.data(), A.idx.data(), A.val.data(), md.m, md.n, threads);
    }
    return ref(AT);
}

void model_matrices(const taral_model& md, Csr& A, Csr& AT, int threads) {
    const CsrRef at = model_matrices_ref(md, A, AT, threads);
    if (at.ptr == md.col_ptr) {  // the model's own arrays: copied
        AT.rows = md.n;
        AT.ptr.assign(at.ptr, at.ptr + md.n + 1);
        AT.idx.assign(at.idx, at.idx + at.nnz());
        AT.val.assign(at.val, at.val + at.nnz());
    }
}

namespace {

// sqrt of the sum of v(i)^2 over i = 0 .. count-1, accumulated in index order
template <class V>
double root_sum_squares(int count, V v) {
    double acc = 0;
    for (int i = 0; i < count; ++i) {
        const double e = v(i);
        acc += e * e;
    }
    return std::sqrt(acc);
}

// how far v lies outside [lo, hi] (negative inside), and the running maximum of such excesses from 0
inline double excess(double lo, double v, double hi) { return std::max(lo - v, v - hi); }
inline void keep_worst(double& worst, double e) { worst = std::max(worst, e); }

// largest row excess of the activities a = A x, rows [i0, i1) of the unscaled row-wise copy A (each row's entries
// in ascending column order, summed in that order)
double row_excess_range(const taral_model& md, const Csr& A, const std::vector<double>& x, int i0, int i1) {
    double worst = 0;
    for (int i = i0; i < i1; ++i) {
        double a = 0.0;
        for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) a += A.val[k] * x[A.idx[k]];
        keep_worst(worst, excess(md.row_lo[i], a, md.row_up[i]));
    }
    return worst;
}

}  // namespace

// The scaled problem's vectors: c_s = sign c Dc, l_s = l / Dc, u_s = u / Dc, rl_s = rl Dr, ru_s = ru Dr, and the
// stopping test's original-space norms ||sign c|| and ||b|| (b_i: the larger finite row bound in magnitude).
void scale_vectors(const taral_model& md, double sign, const std::vector<double>& Dr, const std::vector<double>& Dc,
                   Scaled& P) {
    const int n = md.n, m = md.m;
    P.m = m, P.n = n;
    P.cnorm = root_sum_squares(n, [&](int j) { return sign * md.cost[j]; });
    P.bnorm = root_sum_squares(m, [&](int i) { return bound_size(md.row_lo[i], md.row_up[i]); });
    P.c.resize(size_t(n)), P.l.resize(size_t(n)), P.u.resize(size_t(n));
    for (int j = 0; j < n; ++j) {
        const double d = Dc[size_t(j)];
        P.c[size_t(j)] = (sign * md.cost[j]) * d;
        P.l[size_t(j)] = md.col_lo[j] / d;
        P.u[size_t(j)] = md.col_up[j] / d;
    }
    P.rl.resize(size_t(m)), P.ru.resize(size_t(m));
    for (int i = 0; i < m; ++i) {
        const double d = Dr[size_t(i)];
        P.rl[size_t(i)] = md.row_lo[i] * d;
        P.ru[size_t(i)] = md.row_up[i] * d;
    }
}

// The answer in original units and how well it satisfies the original model: x = Dc x_s, y = Dr z_s, the
// objective c'x + obj_const accumulated in long double, the largest bound excess max(l - x, x - u) and the
// largest row excess max(lo - a, a - up) of the activities a = A x, all from 0. The activities come from the
// unscaled row-wise copy on several host threads when the set-up kept it (their sums add the same products in the
// same order as a sweep over the model's columns), otherwise from one sweep over the columns.
Finished finish_point(const taral_model& md, const Scaled& P, const Outcome& r) {
    const int n = P.n, m = P.m;
    Finished out;
    out.x.resize(size_t(n)), out.y.resize(size_t(m));
    for (int j = 0; j < n; ++j) out.x[size_t(j)] = r.x[size_t(j)] * P.Dc[size_t(j)];
    for (int i = 0; i < m; ++i) out.y[size_t(i)] = P.Dr[size_t(i)] * r.z[size_t(i)];

    long double objective = md.obj_const;
    for (int j = 0; j < n; ++j) objective += (long double)md.cost[j] * out.x[size_t(j)];
    out.objective = double(objective);

    bool all_finite = true;
    for (int j = 0; j < n; ++j) {
        const double v = out.x[size_t(j)];
        keep_worst(out.max_bound_violation, excess(md.col_lo[j], v, md.col_up[j]));
        all_finite = all_finite && std::isfinite(v);
    }

    if (all_finite && P.a_original && m > 0) {
        // explicit zeros of the model add nothing to a sum of finite products; the maximum is split-independent
        const int parts = std::max(1, std::min(host_threads(), m / 4096));
        std::vector<double> worst(size_t(parts), 0.0);
        auto part = [&](int q) {
            worst[size_t(q)] = row_excess_range(md, P.A, out.x, int(int64_t(m) * q / parts),
                                                int(int64_t(m) * (q + 1) / parts));
        };
        std::vector<std::thread> helpers;
        for (int q = 1; q < parts; ++q) helpers.emplace_back(part, q);
        part(0);
        for (std::thread& h : helpers) h.join();
        for (double w : worst) keep_worst(out.max_row_violation, w);
    } else {
        std::vector<double> activity(size_t(m), 0.0);
        for (int j = 0; j < n; ++j) {
            const double v = out.x[size_t(j)];
            for (int64_t k = md.col_ptr[j]; k < md.col_ptr[j + 1]; ++k) activity[size_t(md.row_idx[k])] += md.val[k] * v;
        }
        for (int i = 0; i < m; ++i) keep_worst(out.max_row_violation, excess(md.row_lo[i], activity[size_t(i)], md.row_up[i]));
    }
    return out;
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
