// Test infrastructure: the engine's host driver (taral-lp_b200/csrc/host.hpp, run() with the restart schedule of
// schedule.hpp) over a backend made of the CPU oracle's FP64 step functions (oracle/pdhg_oracle.h). The oracle's
// own driver (orc_solve) restates the reference's; the two must take identical decisions block by block, which
// pins the engine's driver on the CPU without a GPU. Built and loaded by tests/test_driver_on_oracle.py.
#include <vector>

#include "host.hpp"
#include "pdhg_oracle.h"

namespace {

struct OracleBackend {
    const orc_scaled* P;
    orc_state S;
    explicit OracleBackend(const orc_scaled* p) : P(p) { orc_state_init(&S, p); }
    ~OracleBackend() { orc_state_free(&S); }
    double power_norm(int iters) { return orc_power_norm(P, iters); }
    void set_steps(double tau, double sigma) { orc_set_steps(&S, tau, sigma); }
    void start(const double* x0, const double*) { orc_start(&S, x0); }
    void iterate(int steps) { orc_iterate(&S, steps); }
    void eval(bool avg, double f, double* out) { orc_eval(&S, avg ? 1 : 0, f, out); }
    void eval_pair(double f, double* cur, double* avg) {
        orc_eval(&S, 0, 1.0, cur);
        orc_eval(&S, 1, f, avg);
    }
    void restart(bool avg, double f) { orc_restart(&S, avg ? 1 : 0, f); }
    void download(bool avg, double f, double* x, double* z) { orc_download(&S, avg ? 1 : 0, f, x, z); }
};

}  // namespace

extern "C" int drive_on_oracle(const orc_scaled* P, const orc_options* o, orc_outcome* r, double* x, double* z) {
    OracleBackend b(P);
    taral::DriverData d;
    d.m = P->m, d.n = P->n, d.c = P->c, d.rl = P->rl, d.ru = P->ru, d.bnorm = P->bnorm, d.cnorm = P->cnorm;
    taral::Options opt;
    opt.tol = o->tol, opt.time_limit = o->time_limit, opt.max_iter = o->max_iter, opt.eval_freq = o->eval_freq;
    opt.row_rel = o->row_rel;
    const taral::Outcome out = taral::run(b, d, opt, o->time_limit);
    r->status = out.status, r->iterations = out.iterations, r->restarts = out.restarts;
    r->from_average = out.from_average ? 1 : 0;
    r->rel_p = out.rel_primal, r->rel_d = out.rel_dual, r->rel_gap = out.rel_gap;
    r->norm_a = out.norm_a, r->omega = out.omega;
    for (int j = 0; j < P->n; ++j) x[j] = out.x[size_t(j)];
    for (int i = 0; i < P->m; ++i) z[i] = out.z[size_t(i)];
    return 0;
}
