// The restart schedule of the restarted-average PDHG (PDLP: Applegate et al., "Practical large-scale linear
// programming using primal-dual hybrid gradient", NeurIPS 2021, sections 3.1-3.3), as the reference applies it
// after every evaluation block (gpu/pdhg.cu:765-842): the stopping test on relative residuals, the adaptive
// restart to the better of the current point and the running average, and the smoothed primal-weight update.
//
// One implementation serves both engines: the single-LP driver calls it on the host after each block, and the
// batched engine calls it from its decision kernel, one thread per LP, with the state below in device memory.
// Every floating-point operation and comparison happens in the reference's order, with std::max / std::min
// semantics for NaN operands, so FP64 runs reproduce its iteration and restart counts exactly.
#pragma once
#include <cmath>

#include "../../include/taral_pdhg.h"

#if defined(__CUDACC__)
#define TARAL_HD __host__ __device__ inline
#else
#define TARAL_HD inline
#endif

namespace taral {

// Slots of the 10 KKT scalars of one evaluation (5 row terms, then 5 column terms).
enum KktSlot {
    PR2S,  // ||primal violation||^2, scaled space
    PR2O,  // ||primal violation||^2, original units
    PR2R,  // sum of (row violation / (1 + |b_i|))^2
    DROW,  // row part of the dual objective
    DZ2,   // ||z - z_last||^2
    DR2S,  // ||dual residual||^2, scaled space
    DR2O,  // ||dual residual||^2, original units
    POBJ,  // primal objective c'x
    DCOL,  // column part of the dual objective
    DX2    // ||x - x_last||^2
};

namespace sched {
#if defined(__CUDA_ARCH__)
TARAL_HD double root(double v) { return sqrt(v); }
TARAL_HD double ln(double v) { return log(v); }
TARAL_HD double ex(double v) { return exp(v); }
TARAL_HD double mag(double v) { return fabs(v); }
TARAL_HD bool finite(double v) { return isfinite(v); }
TARAL_HD double inf() { return INFINITY; }
#else
TARAL_HD double root(double v) { return std::sqrt(v); }
TARAL_HD double ln(double v) { return std::log(v); }
TARAL_HD double ex(double v) { return std::exp(v); }
TARAL_HD double mag(double v) { return std::fabs(v); }
TARAL_HD bool finite(double v) { return std::isfinite(v); }
TARAL_HD double inf() { return HUGE_VAL; }
#endif
// std::max(a, b) and std::min(a, b): a NaN in the second operand is never chosen
TARAL_HD double larger(double a, double b) { return a < b ? b : a; }
TARAL_HD double smaller(double a, double b) { return b < a ? b : a; }
}  // namespace sched

// A row's size in ||b||: the larger magnitude of its finite bounds, 0 for a free row.
TARAL_HD double bound_size(double lo, double up) {
    const bool has_lo = sched::finite(lo), has_up = sched::finite(up);
    if (has_lo && has_up) return sched::larger(sched::mag(lo), sched::mag(up));
    return has_lo ? sched::mag(lo) : has_up ? sched::mag(up) : 0.0;
}

// Step scale and initial primal weight of a scaled problem: eta = 0.95 / ||A_s||, w = ||c_s|| / ||b_s|| (1 when
// either norm is below 1e-10). The sums run in index order.
struct StepScale {
    double eta, weight;
};
TARAL_HD StepScale initial_steps(double norm_a, const double* c, int n, const double* rl, const double* ru, int m) {
    double c2 = 0, b2 = 0;
    for (int j = 0; j < n; ++j) c2 += c[j] * c[j];
    for (int i = 0; i < m; ++i) {
        const double b = bound_size(rl[i], ru[i]);
        b2 += b * b;
    }
    const double cn = sched::root(c2), bn = sched::root(b2);
    return {norm_a > 0 ? 0.95 / norm_a : 1.0, cn > 1e-10 && bn > 1e-10 ? cn / bn : 1.0};
}

// What the stopping test measures of one evaluation: relative primal, dual and gap errors in original units.
struct Residuals {
    double primal, dual, gap;
    TARAL_HD double worst() const { return sched::larger(primal, sched::larger(dual, gap)); }
};

// The stopping test's fixed inputs: tolerance, the optional per-row relative bound (0 = off), the iteration cap
// and the original-space norms ||b|| and ||c|| of the problem.
struct StopRule {
    double tol, row_rel, bnorm, cnorm;
    long long max_iter;
};

TARAL_HD Residuals residuals_of(const double* k, const StopRule& r) {
    const double pobj = k[POBJ], dobj = k[DROW] + k[DCOL];
    const double per_row = r.row_rel > 0 ? sched::root(k[PR2R]) / r.row_rel : 0;
    Residuals e;
    e.primal = sched::larger(sched::root(k[PR2O]) / (1 + r.bnorm), per_row);
    e.dual = sched::root(k[DR2O]) / (1 + r.cnorm);
    e.gap = sched::mag(pobj - dobj) / (1 + sched::mag(pobj) + sched::mag(dobj));
    return e;
}

// The restart criterion's measure: the KKT error in scaled space under primal weight w,
// sqrt(w ||primal viol||^2 + ||dual res||^2 / w + gap^2).
TARAL_HD double weighted_error(const double* k, double w) {
    const double gap = k[POBJ] - (k[DROW] + k[DCOL]);
    return sched::root(w * k[PR2S] + k[DR2S] / w + gap * gap);
}

// FP64 state of the schedule for one LP. `anchor` is the weighted error of the point the last restart went to (of
// the start point before the first restart); `previous` the candidate error one block ago, +inf after a restart.
struct Schedule {
    double weight, eta, anchor, previous;
    long long iterations, since_restart;
    int restarts, pad;
};

TARAL_HD Schedule make_schedule(const StepScale& s, const double* k_start) {
    Schedule q;
    q.weight = s.weight, q.eta = s.eta;
    q.anchor = weighted_error(k_start, s.weight), q.previous = sched::inf();
    q.iterations = 0, q.since_restart = 0, q.restarts = 0, q.pad = 0;
    return q;
}

enum RestartTo { kNoRestart = 0, kRestartCurrent = 1, kRestartAverage = 2 };

// The schedule's answer to one evaluation block.
struct BlockDecision {
    Residuals best;       // residuals of the better of the two points (by the worst relative error)
    bool average_better;  // that point is the running average
    int status;           // a taral_solve_status when the solve stops here, -1 to go on
    int restart;          // RestartTo: where the iterates restart before the next block
    bool new_weight;      // the primal weight changed: the step sizes become (eta / w, eta * w)
};

// Judge one block from the evaluations of the current point `cur` and of the average `avg` (the schedule's
// iteration counters already include the block). Stops on a non-finite error at both points
// (numerical_failure), on the better point's worst relative error <= tol (near_optimal), on an external stop
// request `stop` (a taral_solve_status such as time_limit or cancelled; -1: none) or on the iteration cap
// (iteration_limit), in that order. Otherwise the candidate (the point with
// the lower weighted error) restarts when a long time has passed since the last restart (36 % of all iterations),
// when its error fell to 20 % of the anchor, or when it fell to 80 % and rose since the last block; a restart
// re-anchors the schedule and, when both movements ||dx||, ||dz|| exceed 1e-10, moves log w halfway to
// log(||dz|| / ||dx||).
TARAL_HD BlockDecision judge_block(Schedule& s, const double* cur, const double* avg, const StopRule& rule,
                                   int stop) {
    BlockDecision d;
    const Residuals rc = residuals_of(cur, rule), ra = residuals_of(avg, rule);
    const double ec = rc.worst(), ea = ra.worst();
    d.average_better = ea < ec;
    d.best = d.average_better ? ra : rc;
    d.status = -1, d.restart = kNoRestart, d.new_weight = false;
    if (!sched::finite(ec) && !sched::finite(ea)) d.status = TARAL_NUMERICAL_FAILURE;
    else if (d.best.worst() <= rule.tol) d.status = TARAL_NEAR_OPTIMAL;
    else if (stop >= 0) d.status = stop;
    else if (s.iterations >= rule.max_iter) d.status = TARAL_ITERATION_LIMIT;
    if (d.status >= 0) return d;

    const double wc = weighted_error(cur, s.weight), wa = weighted_error(avg, s.weight);
    const bool to_average = wa < wc;
    const double candidate = sched::smaller(wa, wc);
    const bool stale = double(s.since_restart) >= 0.36 * double(s.iterations);
    const bool big_drop = candidate <= 0.2 * s.anchor;
    const bool drop_then_rise = candidate <= 0.8 * s.anchor && candidate > s.previous;
    s.previous = candidate;
    if (!(stale || big_drop || drop_then_rise)) return d;

    const double* chosen = to_average ? avg : cur;
    const double dx = sched::root(chosen[DX2]), dz = sched::root(chosen[DZ2]);
    if (dx > 1e-10 && dz > 1e-10) {
        s.weight = sched::ex(0.5 * sched::ln(dz / dx) + 0.5 * sched::ln(s.weight));
        d.new_weight = true;
    }
    s.anchor = weighted_error(chosen, s.weight), s.previous = sched::inf();
    s.since_restart = 0, s.restarts++;
    d.restart = to_average ? kRestartAverage : kRestartCurrent;
    return d;
}

}  // namespace taral
