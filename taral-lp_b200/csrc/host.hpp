// Host side of the PDHG path: problem format, scaling, options/outcome and the driver loop.
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <stdexcept>
#include <memory>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/taral_pdhg.h"
#include "schedule.hpp"

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

// Allocator whose value-less construct leaves trivially constructible elements uninitialised: resize() of an entry
// array that is written in full right after, by several threads, does not first zero (and page in) all of it on one
// thread.
template <class T>
struct NoInit : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInit<U>;
    };
    NoInit() = default;
    template <class U>
    NoInit(const NoInit<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using Entries = std::vector<T, NoInit<T>>;

// Row-wise CSR (gpu/pdhg.cu:49-53), int64 row pointers.
struct Csr {
    int rows = 0;
    std::vector<int64_t> ptr;
    Entries<int32_t> idx;
    Entries<double> val;
    taral_csr view(int cols) const { return {rows, cols, int64_t(val.size()), ptr.data(), idx.data(), val.data()}; }
};
// A row-wise matrix held elsewhere (a Csr, or the column-wise arrays of a model read as its transpose): ptr[0] = 0,
// the entries of row r are [ptr[r], ptr[r + 1]).
struct CsrRef {
    int rows = 0;
    const int64_t* ptr = nullptr;
    const int32_t* idx = nullptr;
    const double* val = nullptr;
    int64_t nnz() const { return ptr ? ptr[rows] : 0; }
};
inline CsrRef ref(const Csr& a) { return {a.rows, a.ptr.data(), a.idx.data(), a.val.data()}; }
// Transpose of the CSR given by (ptr, idx, val) (gpu/pdhg.cu:55-70), counted and scattered on `threads` threads.
Csr transpose_par(const int64_t* ptr, const int32_t* idx, const double* val, int rows, int cols, int threads);
int host_threads();
// work(q, begin, end) over [0, count) cut into `parts` contiguous ranges of about equal length, range 0 on the
// calling thread and every other one on a thread of its own.
template <class F>
void split_ranges(int64_t count, int parts, F work) {
    parts = int(std::max<int64_t>(1, std::min<int64_t>(parts, count)));
    std::vector<std::thread> pool;
    for (int q = 1; q < parts; ++q)
        pool.emplace_back([&work, q, count, parts] { work(q, count * q / parts, count * (q + 1) / parts); });
    work(0, int64_t(0), count / parts);
    for (std::thread& t : pool) t.join();
}

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
// The same, except that when the model's columns already are A^T (rows ascending in every column, no explicit
// zero) AT is left empty and the result refers to the model's own arrays; otherwise it refers to AT.
CsrRef model_matrices_ref(const taral_model& md, Csr& A, Csr& AT, int threads = 0);

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

// The restarted-average PDHG on one LP (gpu/pdhg.cu:761-849 semantics), generic over a backend with the concept's
// methods (power_norm, set_steps, start, iterate, eval, eval_pair, restart, download). x0 / z0: optional warm start
// (scaled space). Blocks of eval_freq iterations alternate with one evaluation of the current point and of the
// average (a single synchronisation) and the schedule's decision (schedule.hpp), which the backend then carries
// out: a restart to the chosen point and, after a weight change, new step sizes.
template <class B>
Outcome run(B& b, const DriverData& P, const Options& o, double time_budget, const double* x0 = nullptr,
            const double* z0 = nullptr) {
    Outcome out;
    const auto t0 = Clock::now();
    out.norm_a = b.power_norm(200);
    out.power_s = since(t0);
    const StepScale scale = initial_steps(out.norm_a, P.c, P.n, P.rl, P.ru, P.m);
    b.set_steps(scale.eta / scale.weight, scale.eta * scale.weight);
    b.start(x0, z0);
    double cur[10], avg[10];
    b.eval(false, 1.0, cur);
    Schedule sch = make_schedule(scale, cur);
    const StopRule rule{o.tol, o.row_rel, P.bnorm, P.cnorm, int64_t(o.max_iter)};
    BlockDecision last{};
    last.best = {kInf, kInf, kInf}, last.average_better = false;
    while (sch.iterations < o.max_iter) {
        const int block = int(std::min<int64_t>(o.eval_freq, o.max_iter - sch.iterations));
        b.iterate(block);
        sch.iterations += block, sch.since_restart += block;
        const double f = 1.0 / double(sch.since_restart);
        b.eval_pair(f, cur, avg);
        last = judge_block(sch, cur, avg, rule, since(t0) > time_budget ? int(TARAL_TIME_LIMIT) : -1);
        if (o.verbose && (sch.iterations / o.eval_freq) % 50 == 0)
            std::fprintf(stderr, "[pdhg] iter=%lld weight=%.3e best(p,d,gap)=(%.2e, %.2e, %.2e) from=%s c'x=%.10g\n",
                         (long long)sch.iterations, sch.weight, last.best.primal, last.best.dual, last.best.gap,
                         last.average_better ? "average" : "current", cur[POBJ]);
        if (last.status >= 0) {
            out.status = last.status;
            break;
        }
        if (last.restart != kNoRestart) {
            b.restart(last.restart == kRestartAverage, f);
            if (last.new_weight) b.set_steps(sch.eta / sch.weight, sch.eta * sch.weight);
        }
    }
    out.iterations = sch.iterations, out.restarts = sch.restarts, out.omega = sch.weight;
    out.rel_primal = last.best.primal, out.rel_dual = last.best.dual, out.rel_gap = last.best.gap;
    out.from_average = last.average_better;
    out.x.resize(size_t(P.n)), out.z.resize(size_t(P.m));
    b.download(out.from_average, 1.0 / double(std::max<int64_t>(sch.since_restart, 1)), out.x.data(), out.z.data());
    out.iterate_s = since(t0) - out.power_s;
    return out;
}

// Original-space figures of finish() (gpu/pdhg.cu:866-876): x = Dc x_s, objective (long double), max row and
// bound violation; y = Dr z_s.
struct Finished {
    std::vector<double> x, y;
    double objective = 0, max_row_violation = 0, max_bound_violation = 0;
};
Finished finish_point(const taral_model& md, const Scaled& P, const Outcome& r);

}  // namespace taral
