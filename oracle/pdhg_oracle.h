/* CPU restatement of the TARAL-LP PDHG path, used ONLY as a test and benchmark checker.
 *
 * Nothing in the product links or calls this library; tests/, the smoke check and the CPU-baseline leg
 * of bench.py load it through ctypes to check the CUDA engine. Every function restates, in plain C and
 * FP64, the reference's algorithm in gpu/pdhg.cu (line numbers cited per function in pdhg_oracle.c).
 *
 * Pinned against the reference's own published ledgers (results/gpu_pdhg/synth_*_tol1e-{4,6}.csv) and
 * against outputs of the reference binary built from its sources by oracle/Makefile (tests/golden/). */
#ifndef PDHG_ORACLE_H
#define PDHG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Column-wise LP, the semantics of the reference Model (src/taral.hpp:22-35):
 * min cost'x + obj_const s.t. row_lo <= A x <= row_up, col_lo <= x <= col_up; +-INFINITY for absent bounds. */
typedef struct {
    int m, n;
    const int64_t* col_ptr; /* n+1 */
    const int* row_idx;     /* nnz, row-ascending within a column */
    const double* val;      /* nnz */
    const double *cost, *col_lo, *col_up, *row_lo, *row_up;
    double obj_const;
    int maximize;
} orc_model;

/* Row-wise CSR (the reference Csr, gpu/pdhg.cu:49-53). */
typedef struct {
    int rows;
    int64_t nnz;
    int64_t* ptr;
    int* idx;
    double* val;
} orc_csr;

/* Scaled problem (gpu/pdhg.cu:72-78). */
typedef struct {
    int m, n;
    orc_csr A, AT;
    double *c, *l, *u, *rl, *ru, *Dr, *Dc;
    double bnorm, cnorm;
} orc_scaled;

typedef struct {
    double tol, time_limit;
    int64_t max_iter;
    int eval_freq;
    double row_rel;
    int verbose;
} orc_options;

enum { ORC_NEAR_OPTIMAL = 0, ORC_ITERATION_LIMIT = 1, ORC_TIME_LIMIT = 2, ORC_NUMERICAL_FAILURE = 3 };

typedef struct {
    int status;
    int64_t iterations;
    int restarts;
    int from_average;
    double rel_p, rel_d, rel_gap, norm_a, omega;
    double objective;                  /* model sense, incl. obj_const */
    double max_row_viol, max_bound_viol;
    double power_s, iterate_s;
} orc_outcome;

/* The 10 KKT scalars of one evaluation, in the reference's order (gpu/pdhg.cu:136,145):
 * r = {PR2S, PR2O, PR2R, DROW, DZ2}, c = {DR2S, DR2O, POBJ, DCOL, DX2}. */
enum { ORC_PR2S, ORC_PR2O, ORC_PR2R, ORC_DROW, ORC_DZ2, ORC_DR2S, ORC_DR2O, ORC_POBJ, ORC_DCOL, ORC_DX2, ORC_NKKT };

/* Solver state of the FP64 twin backend (gpu/pdhg.cu:583-741). */
typedef struct {
    const orc_scaled* P;
    double tau, sigma;
    double *x, *z, *Ax, *ATz, *xs, *zs, *Axs, *ATzs, *xlast, *zlast;
} orc_state;

int orc_build_scaled(const orc_model* md, double sign, orc_scaled* out);
void orc_free_scaled(orc_scaled* P);
int orc_transpose(const orc_csr* a, int cols, orc_csr* out);
void orc_free_csr(orc_csr* a);
void orc_spmv(const orc_csr* a, const double* x, double* y);
double orc_power_norm(const orc_scaled* P, int iters);

int orc_state_init(orc_state* S, const orc_scaled* P);
void orc_state_free(orc_state* S);
void orc_set_steps(orc_state* S, double tau, double sigma);
void orc_start(orc_state* S, const double* x0); /* x0 == NULL: clamp(0, l, u) */
void orc_iterate(orc_state* S, int steps);
void orc_eval(const orc_state* S, int avg, double f, double out[ORC_NKKT]);
void orc_restart(orc_state* S, int avg, double f);
void orc_download(const orc_state* S, int avg, double f, double* x, double* z);

/* Whole solve + original-space check (gpu/pdhg.cu:761-911). x_orig (n) and y_orig (m, y = Dr z) may be NULL. */
int orc_solve(const orc_model* md, const orc_options* o, orc_outcome* r, double* x_orig, double* y_orig);

/* Fixed-seed start vector of the power iteration (gpu/pdhg.cu:153). */
double orc_start_vec(int j);

#ifdef __cplusplus
}
#endif
#endif
