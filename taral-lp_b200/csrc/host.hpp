// Host side of the PDHG path: problem format, scaling, options/outcome and the driver loop.
#pragma once
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/taral_pdhg.h"

namespace taral {

constexpr double kInf = std::numeric_limits<double>::infinity();
using Clock = std::chrono::steady_clock;
inline double since(Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); }

// Column-wise LP with the field semantics of the reference Model (src/taral.hpp:22-35), stored as flat CSC.
struct Model {
    std::string name;
    std::vector<std::string> row_names, col_names;
    std::vector<int64_t> col_ptr{0};
    std::vector<int32_t> row_idx;
    std::vector<double> val, cost, col_lo, col_up, row_lo, row_up;
    double obj_const = 0;
    bool maximize = false;
    size_t sentinel_bounds = 0;        // finite |bound| >= 1e20 read as infinite
    std::vector<unsigned char> is_int; // MARKER INTORG..INTEND columns and BV/LI/UI bounds
    int64_t n_quadratic = 0;           // nonzero quadratic objective terms
    taral_model view() const;
};

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
Model read_mps(const std::string& path);  // src/mps.cpp:388-399 semantics

// Row-wise CSR (gpu/pdhg.cu:49-53), int64 row pointers.
struct Csr {
    int rows = 0;
    std::vector<int64_t> ptr;
    std::vector<int32_t> idx;
    std::vector<double> val;
    taral_csr view(int cols) const { return {rows, cols, int64_t(val.size()), ptr.data(), idx.data(), val.data()}; }
};
// Transpose of the CSR given by (ptr, idx, val) (gpu/pdhg.cu:55-70), the scatter on `threads` threads.
Csr transpose_par(const int64_t* ptr, const int32_t* idx, const double* val, int rows, int cols, int threads);
int host_threads();

// Scaled problem (gpu/pdhg.cu:72-78): A_s = diag(Dr) A diag(Dc).
struct Scaled {
    int m = 0, n = 0;
    Csr A, AT;
    std::vector<double> c, l, u, rl, ru, Dr, Dc;
    double bnorm = 0, cnorm = 0;  // original-space norms of the stopping test
    bool a_original = false;      // A holds the UNSCALED row-wise matrix (device-side set-up), used by finish_point
};
// The vector part of the scaled problem (c, l, u, rl, ru and the original-space norms) given Dr and Dc
// (gpu/pdhg.cu:113-133).
void scale_vectors(const taral_model& md, double sign, const std::vector<double>& Dr, const std::vector<double>& Dc,
                   Scaled& P);
// The unscaled A (the transpose of the column-wise model with explicit zeros dropped) and A^T (the transpose of A):
// the structure and entry order the reference's scaling works on (gpu/pdhg.cu:80-90, 131), before any scaling.
void model_matrices(const taral_model& md, Csr& A, Csr& AT, int threads = 0);  // threads <= 0: host_threads()

struct Options {  // gpu/pdhg.cu:744-750
    double tol = 1e-4, time_limit = 3600;
    int64_t max_iter = 2000000000LL;
    int eval_freq = 64;
    double row_rel = 0;
    bool verbose = false, graph = true;
    int precision = TARAL_FP64;
};

struct Outcome {  // gpu/pdhg.cu:752-759
    int status = TARAL_ITERATION_LIMIT;
    int64_t iterations = 0;
    int restarts = 0;
    bool from_average = false;
    double rel_primal = 0, rel_dual = 0, rel_gap = 0, norm_a = 0, omega = 1, power_s = 0, iterate_s = 0;
    std::vector<double> x, z;  // scaled space
};

const char* status_name(int s);

// What the driver reads of the scaled problem: sizes, c_s, [rl, ru]_s and the original-space norms.
struct DriverData {
    int m = 0, n = 0;
    const double *c = nullptr, *rl = nullptr, *ru = nullptr;
    double bnorm = 0, cnorm = 0;
    static DriverData of(const Scaled& P) { return {P.m, P.n, P.c.data(), P.rl.data(), P.ru.data(), P.bnorm, P.cnorm}; }
};

// KKT scalar slots (gpu/pdhg.cu:136, 145).
enum { PR2S, PR2O, PR2R, DROW, DZ2, DR2S, DR2O, POBJ, DCOL, DX2 };

// The restarted-average PDHG driver (gpu/pdhg.cu:761-849), generic over a backend with the concept's methods
// (power_norm, set_steps, start, iterate, eval_pair, restart, download). x0/z0: optional warm start (scaled
// space). The stopping rule, restart rule and primal-weight update follow the reference line by line; the
// KKT scalars of the current point and of the average come back together (one synchronisation per block).
template <class B>
Outcome run(B& b, const DriverData& P, const Options& o, double time_budget, const double* x0 = nullptr,
            const double* z0 = nullptr) {
    Outcome r;
    auto t0 = Clock::now();
    r.norm_a = b.power_norm(200);
    r.power_s = since(t0);
    double eta = r.norm_a > 0 ? 0.95 / r.norm_a : 1.0;
    double cs = 0, bs = 0;
    for (int j = 0; j < P.n; ++j) cs += P.c[j] * P.c[j];
    for (int i = 0; i < P.m; ++i) {
        double lo = P.rl[i], up = P.ru[i];
        double v = std::isfinite(lo) && std::isfinite(up) ? std::max(std::fabs(lo), std::fabs(up))
                   : std::isfinite(lo)                    ? std::fabs(lo)
                   : std::isfinite(up)                    ? std::fabs(up)
                                                          : 0;
        bs += v * v;
    }
    cs = std::sqrt(cs), bs = std::sqrt(bs);
    double w = cs > 1e-10 && bs > 1e-10 ? cs / bs : 1.0;
    b.set_steps(eta / w, eta * w);
    b.start(x0, z0);

    auto wkkt = [&](const double* k) {
        double g = k[POBJ] - (k[DROW] + k[DCOL]);
        return std::sqrt(w * k[PR2S] + k[DR2S] / w + g * g);
    };
    struct Rel {
        double p, d, g;
        double worst() const { return std::max(p, std::max(d, g)); }
    };
    auto rel = [&](const double* k) {
        double po = k[POBJ], du = k[DROW] + k[DCOL];
        double prow = o.row_rel > 0 ? std::sqrt(k[PR2R]) / o.row_rel : 0;
        return Rel{std::max(std::sqrt(k[PR2O]) / (1 + P.bnorm), prow), std::sqrt(k[DR2O]) / (1 + P.cnorm),
                   std::fabs(po - du) / (1 + std::fabs(po) + std::fabs(du))};
    };
    double kc[10], ka[10];
    b.eval(false, 1.0, kc);
    double k_last = wkkt(kc), k_prev = kInf;
    int64_t it = 0, n_since = 0;
    bool avg_final = false;
    Rel best{kInf, kInf, kInf};
    for (;;) {
        int steps = int(std::min<int64_t>(o.eval_freq, o.max_iter - it));
        if (steps <= 0) break;
        b.iterate(steps);
        it += steps, n_since += steps;
        double f = 1.0 / double(n_since);
        b.eval_pair(f, kc, ka);
        Rel rc = rel(kc), ra = rel(ka);
        bool use_avg = ra.worst() < rc.worst();
        best = use_avg ? ra : rc, avg_final = use_avg;
        if (o.verbose && (it / o.eval_freq) % 50 == 0)
            std::fprintf(stderr, "it %lld  w %.3e  cur %.2e %.2e %.2e  avg %.2e %.2e %.2e  pobj %.10g\n",
                         (long long)it, w, rc.p, rc.d, rc.g, ra.p, ra.d, ra.g, kc[POBJ]);
        if (!std::isfinite(rc.worst()) && !std::isfinite(ra.worst())) {
            r.status = TARAL_NUMERICAL_FAILURE;
            break;
        }
        if (best.worst() <= o.tol) {
            r.status = TARAL_NEAR_OPTIMAL;
            break;
        }
        if (since(t0) > time_budget) {
            r.status = TARAL_TIME_LIMIT;
            break;
        }
        if (it >= o.max_iter) break;
        double wc = wkkt(kc), wa = wkkt(ka);
        bool cand_avg = wa < wc;
        const double* kk = cand_avg ? ka : kc;
        double kcand = std::min(wa, wc);
        bool restart = double(n_since) >= 0.36 * double(it) || kcand <= 0.2 * k_last ||
                       (kcand <= 0.8 * k_last && kcand > k_prev);
        k_prev = kcand;
        if (restart) {
            double dx = std::sqrt(kk[DX2]), dz = std::sqrt(kk[DZ2]);
            b.restart(cand_avg, f);
            if (dx > 1e-10 && dz > 1e-10) {
                w = std::exp(0.5 * std::log(dz / dx) + 0.5 * std::log(w));
                b.set_steps(eta / w, eta * w);
            }
            k_last = wkkt(kk), k_prev = kInf, n_since = 0, r.restarts++;
        }
    }
    r.iterations = it;
    r.rel_primal = best.p, r.rel_dual = best.d, r.rel_gap = best.g, r.omega = w, r.from_average = avg_final;
    r.x.resize(P.n), r.z.resize(P.m);
    b.download(avg_final, 1.0 / double(std::max<int64_t>(n_since, 1)), r.x.data(), r.z.data());
    r.iterate_s = since(t0) - r.power_s;
    return r;
}

// Original-space figures of finish() (gpu/pdhg.cu:866-876): x = Dc x_s, objective (long double), max row and
// bound violation; y = Dr z_s.
struct Finished {
    std::vector<double> x, y;
    double objective = 0, max_row_violation = 0, max_bound_violation = 0;
};
Finished finish_point(const taral_model& md, const Scaled& P, const Outcome& r);

}  // namespace taral
