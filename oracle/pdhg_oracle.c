/* CPU restatement of the TARAL-LP PDHG path (FP64), for checking the CUDA engine only.
 *
 * TEST INFRASTRUCTURE. The product never links or calls this file: only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load liboracle.so, and only as the checker. Each function names the lines of the
 * reference gpu/pdhg.cu whose behaviour it restates; the algorithm itself is the restarted-average PDHG of
 * Applegate et al., "Practical large-scale linear programming using primal-dual hybrid gradient" (2021), with
 * the reference's own constants (Ruiz 10 passes + Pock-Chambolle alpha 1, eta = 0.95/||A||, restart betas
 * 0.2 / 0.8 / artificial 0.36, primal-weight smoothing 0.5).
 *
 * Arithmetic follows the reference's CPU twin backend with one thread: sequential sums in index order, and
 * no contraction of a*b+c (the Makefile builds with -ffp-contract=off), so FP64 runs reproduce the reference's
 * iteration counts and objectives. */
#define _POSIX_C_SOURCE 199309L
#include "pdhg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <time.h>

static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* std::max / std::min as the reference uses them: max(a,b) = a < b ? b : a, min(a,b) = b < a ? b : a.
 * The NaN behaviour matters for the numerical-failure test, so it is kept. */
static double ref_max(double a, double b) { return a < b ? b : a; }
static double ref_min(double a, double b) { return b < a ? b : a; }
static double clampv(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

double orc_start_vec(int j) { /* gpu/pdhg.cu:153 */
    return 0.5 + (double)(((uint32_t)j * 2654435761u) % 1000u) / 1000.0;
}

void orc_free_csr(orc_csr* a) {
    free(a->ptr), free(a->idx), free(a->val);
    memset(a, 0, sizeof *a);
}

/* Counting-sort transpose, no atomics: gpu/pdhg.cu:55-70. Row order inside each output row is ascending. */
int orc_transpose(const orc_csr* a, int cols, orc_csr* t) {
    t->rows = cols;
    t->nnz = a->nnz;
    t->ptr = (int64_t*)calloc((size_t)cols + 1, sizeof(int64_t));
    t->idx = (int*)malloc((size_t)(a->nnz ? a->nnz : 1) * sizeof(int));
    t->val = (double*)malloc((size_t)(a->nnz ? a->nnz : 1) * sizeof(double));
    int64_t* pos = (int64_t*)malloc(((size_t)cols + 1) * sizeof(int64_t));
    if (!t->ptr || !t->idx || !t->val || !pos) return -1;
    for (int64_t k = 0; k < a->nnz; ++k) t->ptr[a->idx[k] + 1]++;
    for (int j = 0; j < cols; ++j) t->ptr[j + 1] += t->ptr[j];
    memcpy(pos, t->ptr, (size_t)cols * sizeof(int64_t));
    for (int i = 0; i < a->rows; ++i)
        for (int64_t k = a->ptr[i]; k < a->ptr[i + 1]; ++k) {
            int64_t p = pos[a->idx[k]]++;
            t->idx[p] = i, t->val[p] = a->val[k];
        }
    free(pos);
    return 0;
}

void orc_spmv(const orc_csr* a, const double* x, double* y) { /* Cpu::dot / spmv, gpu/pdhg.cu:625-634 */
    for (int r = 0; r < a->rows; ++r) {
        double s = 0;
        for (int64_t k = a->ptr[r]; k < a->ptr[r + 1]; ++k) s += a->val[k] * x[a->idx[k]];
        y[r] = s;
    }
}

/* Divide rows/cols by sqrt of their measures and fold the factors into Dr/Dc: gpu/pdhg.cu:95-102. */
static void apply_scaling(orc_scaled* P, double* rs, double* cs) {
    orc_csr* A = &P->A;
    for (int i = 0; i < P->m; ++i) rs[i] = rs[i] > 0 ? sqrt(rs[i]) : 1;
    for (int j = 0; j < P->n; ++j) cs[j] = cs[j] > 0 ? sqrt(cs[j]) : 1;
    for (int i = 0; i < P->m; ++i)
        for (int64_t k = A->ptr[i]; k < A->ptr[i + 1]; ++k) A->val[k] /= rs[i] * cs[A->idx[k]];
    for (int i = 0; i < P->m; ++i) P->Dr[i] /= rs[i];
    for (int j = 0; j < P->n; ++j) P->Dc[j] /= cs[j];
}

/* Ruiz (10 passes, inf-norm) then Pock-Chambolle (alpha 1), vectors and norms: gpu/pdhg.cu:80-133. */
int orc_build_scaled(const orc_model* md, double sign, orc_scaled* P) {
    memset(P, 0, sizeof *P);
    int m = md->m, n = md->n;
    P->m = m, P->n = n;
    orc_csr T; /* A^T straight from the column-wise model, zero entries dropped (gpu/pdhg.cu:83-90) */
    T.rows = n;
    int64_t cap = md->col_ptr[n] - md->col_ptr[0];
    T.ptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    T.idx = (int*)malloc((size_t)(cap ? cap : 1) * sizeof(int));
    T.val = (double*)malloc((size_t)(cap ? cap : 1) * sizeof(double));
    if (!T.ptr || !T.idx || !T.val) return -1;
    int64_t w = 0;
    for (int j = 0; j < n; ++j) {
        for (int64_t k = md->col_ptr[j]; k < md->col_ptr[j + 1]; ++k)
            if (md->val[k] != 0) T.idx[w] = md->row_idx[k], T.val[w] = md->val[k], ++w;
        T.ptr[j + 1] = w;
    }
    T.nnz = w;
    if (orc_transpose(&T, m, &P->A)) return -1;
    orc_free_csr(&T);
    orc_csr* A = &P->A;
    P->Dr = (double*)malloc((size_t)(m ? m : 1) * sizeof(double));
    P->Dc = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    double* rs = (double*)malloc((size_t)(m ? m : 1) * sizeof(double));
    double* cs = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    for (int i = 0; i < m; ++i) P->Dr[i] = 1;
    for (int j = 0; j < n; ++j) P->Dc[j] = 1;
    for (int pass = 0; pass < 10; ++pass) {
        memset(rs, 0, (size_t)m * sizeof(double)), memset(cs, 0, (size_t)n * sizeof(double));
        for (int i = 0; i < m; ++i)
            for (int64_t k = A->ptr[i]; k < A->ptr[i + 1]; ++k) {
                double a = fabs(A->val[k]);
                rs[i] = ref_max(rs[i], a), cs[A->idx[k]] = ref_max(cs[A->idx[k]], a);
            }
        apply_scaling(P, rs, cs);
    }
    memset(rs, 0, (size_t)m * sizeof(double)), memset(cs, 0, (size_t)n * sizeof(double));
    for (int i = 0; i < m; ++i)
        for (int64_t k = A->ptr[i]; k < A->ptr[i + 1]; ++k) rs[i] += fabs(A->val[k]), cs[A->idx[k]] += fabs(A->val[k]);
    apply_scaling(P, rs, cs);
    free(rs), free(cs);
    if (orc_transpose(A, n, &P->AT)) return -1;
    P->c = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    P->l = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    P->u = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    P->rl = (double*)malloc((size_t)(m ? m : 1) * sizeof(double));
    P->ru = (double*)malloc((size_t)(m ? m : 1) * sizeof(double));
    double cn = 0, bn = 0;
    for (int j = 0; j < n; ++j) {
        double c = sign * md->cost[j];
        cn += c * c;
        P->c[j] = c * P->Dc[j], P->l[j] = md->col_lo[j] / P->Dc[j], P->u[j] = md->col_up[j] / P->Dc[j];
    }
    for (int i = 0; i < m; ++i) {
        double lo = md->row_lo[i], up = md->row_up[i], b = 0;
        if (isfinite(lo) && isfinite(up)) b = ref_max(fabs(lo), fabs(up));
        else if (isfinite(lo)) b = fabs(lo);
        else if (isfinite(up)) b = fabs(up);
        bn += b * b;
        P->rl[i] = lo * P->Dr[i], P->ru[i] = up * P->Dr[i];
    }
    P->bnorm = sqrt(bn), P->cnorm = sqrt(cn);
    return 0;
}

void orc_free_scaled(orc_scaled* P) {
    orc_free_csr(&P->A), orc_free_csr(&P->AT);
    free(P->c), free(P->l), free(P->u), free(P->rl), free(P->ru), free(P->Dr), free(P->Dc);
    memset(P, 0, sizeof *P);
}

/* sigma_max(A_s) by power iteration on A_s^T A_s: gpu/pdhg.cu:635-654 (CPU) / :417-436 (GPU). */
double orc_power_norm(const orc_scaled* P, int iters) {
    int m = P->m, n = P->n;
    double* pv = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    double* pw = (double*)malloc((size_t)(m ? m : 1) * sizeof(double));
    double* pu = (double*)malloc((size_t)(n ? n : 1) * sizeof(double));
    double nn = 0;
    for (int j = 0; j < n; ++j) pv[j] = orc_start_vec(j), nn += pv[j] * pv[j];
    for (int j = 0; j < n; ++j) pv[j] = pv[j] / sqrt(nn);
    double est = 0;
    for (int it = 0; it < iters; ++it) {
        orc_spmv(&P->A, pv, pw);
        orc_spmv(&P->AT, pw, pu);
        double s = 0, prev = est;
        for (int j = 0; j < n; ++j) s += pu[j] * pu[j];
        if (s <= 0) { est = 0; break; }
        est = sqrt(sqrt(s));
        for (int j = 0; j < n; ++j) pu[j] = pu[j] * (1 / sqrt(s));
        double* t = pv; pv = pu; pu = t;
        if (it >= 10 && fabs(est - prev) <= 1e-7 * est) break;
    }
    free(pv), free(pw), free(pu);
    return est;
}

int orc_state_init(orc_state* S, const orc_scaled* P) { /* Cpu::init, gpu/pdhg.cu:617-624 */
    memset(S, 0, sizeof *S);
    S->P = P;
    size_t n = (size_t)(P->n ? P->n : 1), m = (size_t)(P->m ? P->m : 1);
    double** cols[] = {&S->x, &S->ATz, &S->xs, &S->ATzs, &S->xlast};
    double** rows[] = {&S->z, &S->Ax, &S->zs, &S->Axs, &S->zlast};
    for (int k = 0; k < 5; ++k) {
        *cols[k] = (double*)calloc(n, sizeof(double));
        *rows[k] = (double*)calloc(m, sizeof(double));
        if (!*cols[k] || !*rows[k]) return -1;
    }
    return 0;
}

void orc_state_free(orc_state* S) {
    free(S->x), free(S->ATz), free(S->xs), free(S->ATzs), free(S->xlast);
    free(S->z), free(S->Ax), free(S->zs), free(S->Axs), free(S->zlast);
    memset(S, 0, sizeof *S);
}

void orc_set_steps(orc_state* S, double tau, double sigma) { S->tau = tau, S->sigma = sigma; }

static void products(orc_state* S) { /* Ax = A x, ATz = A^T z exactly: gpu/pdhg.cu:656-659 */
    orc_spmv(&S->P->A, S->x, S->Ax);
    orc_spmv(&S->P->AT, S->z, S->ATz);
}

void orc_start(orc_state* S, const double* x0) { /* gpu/pdhg.cu:660-663 */
    const orc_scaled* P = S->P;
    for (int j = 0; j < P->n; ++j) {
        double v = x0 ? x0[j] : ref_min(ref_max(0.0, P->l[j]), P->u[j]);
        S->x[j] = S->xlast[j] = v;
    }
    products(S);
}

static void xupd(orc_state* S, int j) { /* gpu/pdhg.cu:665-668 */
    const orc_scaled* P = S->P;
    double xn = clampv(S->x[j] - S->tau * (P->c[j] + S->ATz[j]), P->l[j], P->u[j]);
    S->x[j] = xn, S->xs[j] += xn;
}

/* One block of PDHG steps: the first x update, then per step the row phase (A x, dual prox, sums) and the
 * column phase (A^T z, sums, and the next step's x update): gpu/pdhg.cu:669-691 (CPU) / :459-470 (GPU). */
void orc_iterate(orc_state* S, int steps) {
    const orc_scaled* P = S->P;
    const orc_csr *A = &P->A, *AT = &P->AT;
    double sig = S->sigma;
    for (int j = 0; j < P->n; ++j) xupd(S, j);
    for (int s = 0; s < steps; ++s) {
        for (int i = 0; i < P->m; ++i) {
            double ax = 0;
            for (int64_t k = A->ptr[i]; k < A->ptr[i + 1]; ++k) ax += A->val[k] * S->x[A->idx[k]];
            double v = S->z[i] + sig * (2 * ax - S->Ax[i]), q = v / sig;
            double zn = q < P->rl[i] ? v - sig * P->rl[i] : (q > P->ru[i] ? v - sig * P->ru[i] : 0.0);
            S->Ax[i] = ax, S->z[i] = zn, S->Axs[i] += ax, S->zs[i] += zn;
        }
        int upd = s + 1 < steps;
        for (int j = 0; j < P->n; ++j) {
            double v = 0;
            for (int64_t k = AT->ptr[j]; k < AT->ptr[j + 1]; ++k) v += AT->val[k] * S->z[AT->idx[k]];
            S->ATz[j] = v, S->ATzs[j] += v;
            if (upd) xupd(S, j);
        }
    }
}

/* Weight of row i in the per-row relative residual: gpu/pdhg.cu:138-144. */
static double row_rel_weight(double lo, double up, double dr) {
    double b = 0;
    if (lo > -INFINITY) b = lo < 0 ? -lo : lo;
    if (up < INFINITY) {
        double a = up < 0 ? -up : up;
        b = a > b ? a : b;
    }
    return 1.0 / (1.0 + b / dr);
}

/* The 10 FP64 KKT scalars of the current point or of the average scaled by f: gpu/pdhg.cu:692-730. */
void orc_eval(const orc_state* S, int avg, double f, double out[ORC_NKKT]) {
    const orc_scaled* P = S->P;
    for (int k = 0; k < ORC_NKKT; ++k) out[k] = 0;
    const double *Axv = avg ? S->Axs : S->Ax, *zv = avg ? S->zs : S->z;
    const double *xv = avg ? S->xs : S->x, *ATzv = avg ? S->ATzs : S->ATz;
    for (int i = 0; i < P->m; ++i) {
        double ax = Axv[i] * f, zz = zv[i] * f, lo = P->rl[i], up = P->ru[i];
        double r = ax < lo ? lo - ax : (ax > up ? ax - up : 0), ro = r / P->Dr[i];
        double rr = ro * row_rel_weight(lo, up, P->Dr[i]);
        out[ORC_PR2S] += r * r, out[ORC_PR2O] += ro * ro, out[ORC_PR2R] += rr * rr;
        if (zz > 0 && up < INFINITY) out[ORC_DROW] -= zz * up;
        if (zz < 0 && lo > -INFINITY) out[ORC_DROW] -= zz * lo;
        double dz = zz - S->zlast[i];
        out[ORC_DZ2] += dz * dz;
    }
    for (int j = 0; j < P->n; ++j) {
        double xx = xv[j] * f, cj = P->c[j], d = cj + ATzv[j] * f, lo = P->l[j], up = P->u[j], res = 0;
        out[ORC_POBJ] += cj * xx;
        if (d > 0) {
            if (lo > -INFINITY) out[ORC_DCOL] += d * lo;
            else res = d;
        } else if (d < 0) {
            if (up < INFINITY) out[ORC_DCOL] += d * up;
            else res = -d;
        }
        double ro = res / P->Dc[j], dx = xx - S->xlast[j];
        out[ORC_DR2S] += res * res, out[ORC_DR2O] += ro * ro, out[ORC_DX2] += dx * dx;
    }
}

void orc_restart(orc_state* S, int avg, double f) { /* gpu/pdhg.cu:731-735 */
    const orc_scaled* P = S->P;
    for (int j = 0; j < P->n; ++j) {
        double v = avg ? S->xs[j] * f : S->x[j];
        S->x[j] = S->xlast[j] = v, S->xs[j] = 0, S->ATzs[j] = 0;
    }
    for (int i = 0; i < P->m; ++i) {
        double v = avg ? S->zs[i] * f : S->z[i];
        S->z[i] = S->zlast[i] = v, S->zs[i] = 0, S->Axs[i] = 0;
    }
    products(S);
}

void orc_download(const orc_state* S, int avg, double f, double* x, double* z) { /* gpu/pdhg.cu:736-740 */
    for (int j = 0; j < S->P->n; ++j) x[j] = avg ? S->xs[j] * f : S->x[j];
    for (int i = 0; i < S->P->m; ++i) z[i] = avg ? S->zs[i] * f : S->z[i];
}

typedef struct { double p, d, g; } rel_t;
static double worst(rel_t r) { return ref_max(r.p, ref_max(r.d, r.g)); }

/* The driver: step sizes, primal weight, the eval/terminate/restart loop: gpu/pdhg.cu:761-849. Then the
 * original-space unscale, objective and violations of finish(): gpu/pdhg.cu:866-876, 905-909. */
int orc_solve(const orc_model* md, const orc_options* o, orc_outcome* r, double* x_orig, double* y_orig) {
    memset(r, 0, sizeof *r);
    r->status = ORC_ITERATION_LIMIT;
    r->omega = 1;
    orc_scaled P;
    if (orc_build_scaled(md, md->maximize ? -1.0 : 1.0, &P)) return -1;
    orc_state S;
    if (orc_state_init(&S, &P)) return -1;
    double t0 = now_s();
    r->norm_a = orc_power_norm(&P, 200);
    r->power_s = now_s() - t0;
    double eta = r->norm_a > 0 ? 0.95 / r->norm_a : 1.0;
    double cs = 0, bs = 0;
    for (int j = 0; j < P.n; ++j) cs += P.c[j] * P.c[j];
    for (int i = 0; i < P.m; ++i) {
        double lo = P.rl[i], up = P.ru[i];
        double v = isfinite(lo) && isfinite(up) ? ref_max(fabs(lo), fabs(up))
                   : isfinite(lo)               ? fabs(lo)
                   : isfinite(up)               ? fabs(up)
                                                : 0;
        bs += v * v;
    }
    cs = sqrt(cs), bs = sqrt(bs);
    double w = cs > 1e-10 && bs > 1e-10 ? cs / bs : 1.0;
    orc_set_steps(&S, eta / w, eta * w);
    orc_start(&S, NULL);

    double kc[ORC_NKKT], ka[ORC_NKKT];
#define WKKT(k) sqrt(w * (k)[ORC_PR2S] + (k)[ORC_DR2S] / w + \
                      ((k)[ORC_POBJ] - ((k)[ORC_DROW] + (k)[ORC_DCOL])) * ((k)[ORC_POBJ] - ((k)[ORC_DROW] + (k)[ORC_DCOL])))
    orc_eval(&S, 0, 1.0, kc);
    double k_last = WKKT(kc), k_prev = INFINITY;
    int64_t it = 0, n_since = 0;
    int avg_final = 0;
    rel_t best = {INFINITY, INFINITY, INFINITY};
    for (;;) {
        int64_t left = o->max_iter - it;
        int steps = (int)(left < o->eval_freq ? left : o->eval_freq);
        if (steps <= 0) break;
        orc_iterate(&S, steps);
        it += steps, n_since += steps;
        double f = 1.0 / (double)n_since;
        orc_eval(&S, 0, 1.0, kc);
        orc_eval(&S, 1, f, ka);
        rel_t rc, ra;
        for (int q = 0; q < 2; ++q) {
            const double* k = q ? ka : kc;
            double po = k[ORC_POBJ], du = k[ORC_DROW] + k[ORC_DCOL];
            double prow = o->row_rel > 0 ? sqrt(k[ORC_PR2R]) / o->row_rel : 0;
            rel_t v = {ref_max(sqrt(k[ORC_PR2O]) / (1 + P.bnorm), prow), sqrt(k[ORC_DR2O]) / (1 + P.cnorm),
                       fabs(po - du) / (1 + fabs(po) + fabs(du))};
            if (q) ra = v; else rc = v;
        }
        int use_avg = worst(ra) < worst(rc);
        best = use_avg ? ra : rc, avg_final = use_avg;
        if (o->verbose && (it / o->eval_freq) % 50 == 0)
            fprintf(stderr, "it %ld  w %.3e  cur %.2e %.2e %.2e  avg %.2e %.2e %.2e\n", (long)it, w, rc.p, rc.d, rc.g,
                    ra.p, ra.d, ra.g);
        if (!isfinite(worst(rc)) && !isfinite(worst(ra))) { r->status = ORC_NUMERICAL_FAILURE; break; }
        if (worst(best) <= o->tol) { r->status = ORC_NEAR_OPTIMAL; break; }
        if (now_s() - t0 > o->time_limit) { r->status = ORC_TIME_LIMIT; break; }
        if (it >= o->max_iter) break;
        double wc = WKKT(kc), wa = WKKT(ka);
        int cand_avg = wa < wc;
        const double* kk = cand_avg ? ka : kc;
        double kcand = ref_min(wa, wc);
        int restart = (double)n_since >= 0.36 * (double)it || kcand <= 0.2 * k_last ||
                      (kcand <= 0.8 * k_last && kcand > k_prev);
        k_prev = kcand;
        if (restart) {
            double dx = sqrt(kk[ORC_DX2]), dz = sqrt(kk[ORC_DZ2]);
            double kk_copy[ORC_NKKT];
            memcpy(kk_copy, kk, sizeof kk_copy);
            orc_restart(&S, cand_avg, f);
            if (dx > 1e-10 && dz > 1e-10) {
                w = exp(0.5 * log(dz / dx) + 0.5 * log(w));
                orc_set_steps(&S, eta / w, eta * w);
            }
            k_last = WKKT(kk_copy), k_prev = INFINITY, n_since = 0, r->restarts++;
        }
    }
#undef WKKT
    r->iterations = it;
    r->rel_p = best.p, r->rel_d = best.d, r->rel_gap = best.g, r->omega = w, r->from_average = avg_final;
    double* xs = (double*)malloc((size_t)(P.n ? P.n : 1) * sizeof(double));
    double* zs = (double*)malloc((size_t)(P.m ? P.m : 1) * sizeof(double));
    orc_download(&S, avg_final, 1.0 / (double)(n_since > 1 ? n_since : 1), xs, zs);
    r->iterate_s = now_s() - t0 - r->power_s;

    /* finish(): original space, FP64, objective in long double (gpu/pdhg.cu:866-876) */
    double* x = (double*)malloc((size_t)(P.n ? P.n : 1) * sizeof(double));
    double* ax = (double*)calloc((size_t)(P.m ? P.m : 1), sizeof(double));
    for (int j = 0; j < P.n; ++j) x[j] = xs[j] * P.Dc[j];
    long double obj = md->obj_const;
    for (int j = 0; j < P.n; ++j) obj += (long double)md->cost[j] * x[j];
    double bviol = 0, rviol = 0;
    for (int j = 0; j < P.n; ++j) {
        for (int64_t k = md->col_ptr[j]; k < md->col_ptr[j + 1]; ++k) ax[md->row_idx[k]] += md->val[k] * x[j];
        bviol = ref_max(bviol, ref_max(md->col_lo[j] - x[j], x[j] - md->col_up[j]));
    }
    for (int i = 0; i < P.m; ++i) rviol = ref_max(rviol, ref_max(md->row_lo[i] - ax[i], ax[i] - md->row_up[i]));
    r->objective = (double)obj, r->max_row_viol = rviol, r->max_bound_viol = bviol;
    if (x_orig) memcpy(x_orig, x, (size_t)P.n * sizeof(double));
    if (y_orig)
        for (int i = 0; i < P.m; ++i) y_orig[i] = P.Dr[i] * zs[i];
    free(xs), free(zs), free(x), free(ax);
    orc_state_free(&S);
    orc_free_scaled(&P);
    return 0;
}
