/* taral_pdhg.h -- C ABI of the B200 PDHG engine for continuous LPs (sm_100a).
 *
 * Drop-in boundary for the TARAL-LP PDHG path. Three layers, each replacing a reference interface:
 *
 *   1. Backend concept (pdhg_*): the eight methods the reference's driver template calls on a backend,
 *      gpu/pdhg.cu:313-514 (struct Gpu<T>) and :583-741 (struct Cpu<T>), over an opaque device context.
 *   2. Solver entry (taral_pdhg_solve): the reference's whole solve path for one model -- input gate
 *      (gpu/pdhg_input.hpp:7-26), scaling (gpu/pdhg.cu:80-133), driver run<B>() (gpu/pdhg.cu:761-849) and the
 *      original-space check of finish() (gpu/pdhg.cu:858-911).
 *   3. Problem format (taral_mps_*): the reference's MPS reader, src/mps.cpp:96-399 / src/taral.hpp:48,
 *      returning a model with the semantics of Model (src/taral.hpp:22-35).
 *
 * Conventions
 *   - Every call returns an int status: TARAL_OK (0) or a negative TARAL_ERR_*; the reference exits the
 *     process on any CUDA error (gpu/pdhg.cu:36-43) where this ABI returns TARAL_ERR_CUDA instead.
 *     pdhg_last_error() gives the message of the last failure on a context.
 *   - Host arrays passed in are read during the call only (copied); the context owns all device memory and
 *     its CUDA stream. One host thread per context; contexts are independent of each other.
 *   - Reductions are fixed-order: the same input gives bit-identical results on the same GPU.
 *   - Indices are 0-based; row/column pointer arrays are int64; infinite bounds are +-INFINITY.
 */
#ifndef TARAL_PDHG_H
#define TARAL_PDHG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TARAL_PDHG_ABI_VERSION 1

enum taral_status {
    TARAL_OK = 0,
    TARAL_ERR_CUDA = -1,        /* a CUDA runtime call failed (message in pdhg_last_error) */
    TARAL_ERR_ALLOC = -2,       /* device or host allocation failed */
    TARAL_ERR_INPUT = -3,       /* malformed arguments (sizes, pointers, index ranges) */
    TARAL_ERR_UNSUPPORTED = -4, /* integer or quadratic model (gpu/pdhg_input.hpp:7-17) */
    TARAL_ERR_PARSE = -5,       /* MPS file could not be read */
    TARAL_ERR_STATE = -6,       /* call out of order (e.g. iterate before start) */
    TARAL_ERR_NO_DEVICE = -7,   /* no CUDA device, or not an sm_100 part */
    TARAL_ERR_CANCELLED = -8    /* the solve stopped on a cancel request (taral_batch_cancel); outputs are filled */
};

/* Arithmetic of the iteration. FP64: everything in double (the reference's default).
 * FP32: matrix values, iterates x, z and the products Ax, A^T z in float; running averages, KKT
 * residuals, gap, restart tests and the primal weight in double. */
enum taral_precision { TARAL_FP64 = 0, TARAL_FP32 = 1 };

/* pdhg_create flags */
#define TARAL_FLAG_NO_GRAPH 1u /* launch each block's kernels directly instead of replaying a CUDA graph */

/* Row-wise CSR in host memory. ptr has rows+1 entries; column indices ascending within a row. */
typedef struct {
    int rows, cols;
    int64_t nnz;
    const int64_t* ptr;
    const int32_t* idx;
    const double* val;
} taral_csr;

/* ------------------------------------------------------------------------------------------------------------
 * 1. Backend concept. Replaces Gpu<T> (gpu/pdhg.cu:313-514). All vectors are in the SCALED space of
 *    gpu/pdhg.cu:72-78: A_s = diag(Dr) A diag(Dc), c_s = Dc c, [l,u]_s = [l,u]/Dc, [rl,ru]_s = Dr [rl,ru].
 * ------------------------------------------------------------------------------------------------------------ */
typedef struct pdhg_ctx pdhg_ctx;

/* Gpu::init (gpu/pdhg.cu:362-382): upload A and A^T (AT must be the transpose of A), the 7 vectors and
 * allocate the iteration state on the current CUDA device. eval_freq = steps per captured graph (64). */
int pdhg_create(const taral_csr* A, const taral_csr* AT, const double* c, const double* l, const double* u,
                const double* rl, const double* ru, const double* Dr, const double* Dc, int m, int n,
                int precision, int eval_freq, unsigned flags, pdhg_ctx** out);
/* Gpu::power_norm (gpu/pdhg.cu:416-436): sigma_max(A_s) by power iteration on A_s^T A_s, at most iters
 * steps, stopping after step 10 once the estimate changes by <= 1e-7 relative. */
int pdhg_power_norm(pdhg_ctx* ctx, int iters, double* norm_out);
/* Gpu::set_steps (gpu/pdhg.cu:442-445): primal step tau, dual step sigma. */
int pdhg_set_steps(pdhg_ctx* ctx, double tau, double sigma);
/* Gpu::start (gpu/pdhg.cu:450-458): x0 = clamp(0, l, u) when x0 is NULL, z0 = 0 when z0 is NULL (a warm start
 * passes both); x_last = x0, z_last = z0; averages cleared; Ax and A^T z recomputed exactly. */
int pdhg_start(pdhg_ctx* ctx, const double* x0, const double* z0);
/* Gpu::iterate (gpu/pdhg.cu:459-486): `steps` PDHG iterations; a block of exactly eval_freq steps replays a
 * CUDA graph captured on first use. Asynchronous: returns once the work is queued on the context stream. */
int pdhg_iterate(pdhg_ctx* ctx, int steps);
/* Gpu::eval (gpu/pdhg.cu:487-499): the 10 FP64 KKT scalars of the current point (avg = 0) or of the running
 * average scaled by f (avg = 1), in the order {PR2S, PR2O, PR2R, DROW, DZ2, DR2S, DR2O, POBJ, DCOL, DX2}
 * (gpu/pdhg.cu:136, 145). Synchronises the context stream. */
int pdhg_eval(pdhg_ctx* ctx, int avg, double f, double out[10]);
/* Both evaluations of one block (current, then average scaled by f) with one synchronisation. */
int pdhg_eval_pair(pdhg_ctx* ctx, double f, double cur[10], double avg[10]);
/* Gpu::restart (gpu/pdhg.cu:500-504): restart to the average scaled by f (avg = 1) or to the current point. */
int pdhg_restart(pdhg_ctx* ctx, int avg, double f);
/* Gpu::download (gpu/pdhg.cu:505-513): x (n) and z (m) of the current point or of the scaled average, FP64. */
int pdhg_download(pdhg_ctx* ctx, int avg, double f, double* x, double* z);
/* Gpu::name / Gpu::mem_used. name_out receives at most cap bytes (NUL-terminated). */
int pdhg_info(pdhg_ctx* ctx, char* name_out, size_t cap, size_t* mem_used);
/* Total kernels this context has launched (graph replays count their kernels). */
int64_t pdhg_kernel_launches(const pdhg_ctx* ctx);
const char* pdhg_last_error(const pdhg_ctx* ctx);
void pdhg_destroy(pdhg_ctx* ctx);

/* ------------------------------------------------------------------------------------------------------------
 * 2. Solver entry. Replaces main() -> build_scaled -> solve_with<T> -> run<Gpu<T>> -> finish
 *    (gpu/pdhg.cu:937-992, :913-935, :761-849, :858-911) for a model already in memory.
 * ------------------------------------------------------------------------------------------------------------ */

/* Column-wise model with the semantics of Model (src/taral.hpp:22-35). is_int may be NULL (all continuous);
 * n_quadratic is the number of nonzero quadratic objective terms (0 for an LP). */
typedef struct {
    int m, n;
    const int64_t* col_ptr; /* n+1 */
    const int32_t* row_idx; /* nnz, rows ascending within each column */
    const double* val;      /* nnz */
    const double *cost, *col_lo, *col_up, *row_lo, *row_up;
    double obj_const;
    int maximize;
    const unsigned char* is_int;
    int64_t n_quadratic;
} taral_model;

/* Options (gpu/pdhg.cu:744-750) plus the precision switch of the CLI's --fp32. */
typedef struct {
    double tol;         /* 1e-4 */
    double time_limit;  /* seconds, 3600 */
    int64_t max_iter;   /* 2e9 */
    int eval_freq;      /* 64 */
    double row_rel;     /* 0 = off */
    int verbose;        /* 0 */
    int graph;          /* 1 */
    int precision;      /* TARAL_FP64 */
} taral_options;

enum taral_solve_status { TARAL_NEAR_OPTIMAL = 0, TARAL_ITERATION_LIMIT = 1, TARAL_TIME_LIMIT = 2,
                          TARAL_NUMERICAL_FAILURE = 3, TARAL_CANCELLED = 4 /* batch: stopped by taral_batch_cancel */ };

/* Outcome (gpu/pdhg.cu:752-759) and the figures finish() prints (gpu/pdhg.cu:866-897). */
typedef struct {
    int status;             /* taral_solve_status */
    int64_t iterations;
    int restarts;
    int from_average;       /* 1: the answer is the running average, 0: the current iterate */
    double rel_primal, rel_dual, rel_gap;
    double norm_a, primal_weight;
    double objective;       /* model sense, including obj_const */
    double max_row_violation, max_bound_violation; /* original model, absolute */
    double scale_s, device_init_s, transfer_s, solve_s, power_iter_s;
    size_t device_mem_bytes;
    int64_t kernel_launches;
    int64_t nnz;
    double device_s;        /* pdhg_solve_ctx: CUDA-event time of the solve on the context stream */
} taral_outcome;

void taral_options_default(taral_options* o);
/* pdhg_input_error (gpu/pdhg_input.hpp:7-17): NULL for a continuous LP, else the rejection reason. */
const char* taral_pdhg_input_error(const taral_model* md);
/* Solve one LP. x_out (n, original space) and y_out (m, y = Dr z, minimisation form) may be NULL.
 * Returns TARAL_ERR_UNSUPPORTED (with nothing computed) for integer or quadratic models. */
int taral_pdhg_solve(const taral_model* md, const taral_options* o, taral_outcome* out, double* x_out,
                     double* y_out);
/* taral_pdhg_solve from a given start point instead of x = clamp(0, l, u), y = 0: x0 (n, original space) and y0
 * (m, minimisation-form row multipliers, as written by --dual) are scaled into the solver's space. Either may be
 * NULL. This is the warm-start hook of the learned initialiser; the reference has no counterpart (its only
 * restart across solves is the simplex crossover of src/crossover.cpp:15-60). */
int taral_pdhg_solve_warm(const taral_model* md, const taral_options* o, const double* x0, const double* y0,
                          taral_outcome* out, double* x_out, double* y_out);

/* Backend-level entries that take the solver's options and outcome types. */
/* Input gate + scaling (gpu/pdhg.cu:80-133) + pdhg_create for a column-wise model: the device context of the
 * model's scaled problem. bnorm / cnorm (may be NULL) receive the original-space norms pdhg_solve_ctx needs. An FP32
 * context may hold the rows in another order internally (sorted by length); every vector passed in or out
 * (pdhg_start, pdhg_download) is in the model's row order. */
int pdhg_create_model(const taral_model* md, int precision, int eval_freq, unsigned flags, pdhg_ctx** out,
                      double* bnorm, double* cnorm);
/* run<B> (gpu/pdhg.cu:761-849) on an existing context: power iteration, step sizes, the eval / terminate /
 * restart loop and the final download (x, z in the scaled space; either may be NULL). bnorm and cnorm are the
 * original-space norms of the stopping test (gpu/pdhg.cu:118-131); c, rl, ru are the ones given at creation.
 * x0 / z0: optional start point (scaled space). out->device_s is the device time of the whole solve. */
int pdhg_solve_ctx(pdhg_ctx* ctx, double bnorm, double cnorm, const taral_options* o, const double* x0,
                   const double* z0, taral_outcome* out, double* x, double* z);
/* Measurement hook: `reps` launches of the row-phase kernel (A x + dual step) back to back, then `reps` of the
 * column-phase kernel (A^T z + primal step), each run bracketed by CUDA events on the context stream. Returns the
 * mean milliseconds per launch of each. Leaves the iterate in an unspecified state: start again before solving. */
int pdhg_profile_phases(pdhg_ctx* ctx, int reps, double* row_ms, double* col_ms);
/* Inspection of the scaled problem a context holds (the reference's Scaled, gpu/pdhg.cu:72-78, which it keeps on the
 * host): Dr (m), Dc (n), the values of A_s = diag(Dr) A diag(Dc) (nnz; rows in the model's order, each row's entries
 * in column order, explicit zeros of the model dropped) and of A_s^T (nnz, its rows in column order, entries in row
 * order), copied from the device and widened to double (an FP32 context holds them narrowed to float). Any pointer
 * may be NULL. For checking the device-side set-up against a host computation of the same scaling. */
int pdhg_scaled_problem(pdhg_ctx* ctx, double* Dr, double* Dc, double* A_val, double* AT_val);

/* ------------------------------------------------------------------------------------------------------------
 * 3. Problem format. Replaces read_mps (src/taral.hpp:48, src/mps.cpp:388-399): free format first, fixed
 *    columns as fallback; RANGES, OBJSENSE, bound types, integer markers and quadratic sections are read;
 *    |bound| >= 1e20 is infinite. The handle owns the arrays its model view points into.
 * ------------------------------------------------------------------------------------------------------------ */
typedef struct taral_mps taral_mps;
/* On TARAL_ERR_PARSE, *out is NULL and taral_mps_error() returns the parser's message. */
int taral_mps_read(const char* path, taral_mps** out);
const char* taral_mps_error(void);
int taral_mps_model(const taral_mps* h, taral_model* view);
const char* taral_mps_col_name(const taral_mps* h, int j);
const char* taral_mps_row_name(const taral_mps* h, int i);
const char* taral_mps_name(const taral_mps* h);
void taral_mps_free(taral_mps* h);

/* ------------------------------------------------------------------------------------------------------------
 * 4. Standalone CSR SpMV on device buffers. Replaces the warp-per-row kernel of gpu/csr_matvec.cu:23-32:
 *    y = A x for a CSR matrix already resident on the device (int32 ptr/idx; float or double values and
 *    vectors). A plan holds the row-block partition of the matrix, built once from the host ptr array.
 * ------------------------------------------------------------------------------------------------------------ */
typedef struct taral_spmv_plan taral_spmv_plan;
/* dtype: TARAL_FP64 (double val/x/y) or TARAL_FP32 (float val/x/y, FP64 accumulation). */
int taral_spmv_plan_create(int rows, int cols, const int64_t* host_ptr, int dtype, taral_spmv_plan** out);
/* d_ptr (rows+1 int32), d_idx (nnz int32), d_val, d_x, d_y: device pointers (16-byte aligned idx/val take the
 * vector-load path); stream: a cudaStream_t, or NULL for the legacy default stream. Asynchronous. */
int taral_spmv_run(const taral_spmv_plan* plan, const int32_t* d_ptr, const int32_t* d_idx, const void* d_val,
                   const void* d_x, void* d_y, void* stream);
int taral_spmv_plan_blocks(const taral_spmv_plan* plan);
void taral_spmv_plan_destroy(taral_spmv_plan* plan);

/* ------------------------------------------------------------------------------------------------------------
 * 5. Batched solve: many LPs of one scenario family in one context (the batched scenario family). No
 *    counterpart in the reference, which solves one model per process (gpu/pdhg.cu:937-992); each instance
 *    follows the reference driver's rules (gpu/pdhg.cu:761-849) with its own step sizes, primal weight,
 *    restarts and stopping, evaluated on the device so a block of eval_freq iterations for the whole batch is
 *    one CUDA graph. Instances with identical constraint matrices share one scaled copy of A and A^T.
 * ------------------------------------------------------------------------------------------------------------ */
typedef struct taral_batch taral_batch;
/* Scale every model (matrices shared where identical) and upload the batch. The models and the arrays they
 * point into must stay valid until taral_batch_destroy (the final original-space check reads them). */
int taral_batch_create(const taral_model* models, int count, const taral_options* o, taral_batch** out);
/* Solve all instances. x0[i] / y0[i]: optional warm start of instance i (original space, y in the minimisation
 * form), x0 / y0 themselves may be NULL. w0: NULL, or per instance the initial primal weight (a value that is not
 * finite and positive keeps the default ||c|| / ||b|| of gpu/pdhg.cu:776). outs[i]: instance i's outcome (solve_s
 * and device_s are the whole batch's). x_out[i] (n_i) / y_out[i] (m_i) may be NULL, as may x_out / y_out. */
int taral_batch_solve(taral_batch* b, const double* const* x0, const double* const* y0, const double* w0,
                      taral_outcome* outs, double* const* x_out, double* const* y_out);
/* Ask a running taral_batch_solve on b to stop; callable from any host thread (the only call that may overlap a
 * solve on the same batch). The flag lives in pinned host memory that the device's decision kernel reads after every
 * block of eval_freq iterations: every instance still running then stops with status TARAL_CANCELLED, its best
 * point so far is downloaded and checked as usual, and taral_batch_solve returns TARAL_ERR_CANCELLED. A request made
 * while no solve runs applies to the next solve; a solve clears the flag when it returns. */
int taral_batch_cancel(taral_batch* b);
/* Distinct stored matrices, device bytes, nonzeros stored and nonzeros over all instances. */
int taral_batch_info(const taral_batch* b, int* distinct_matrices, size_t* device_mem, int64_t* nnz_stored,
                     int64_t* nnz_total);
const char* taral_batch_last_error(const taral_batch* b);
void taral_batch_destroy(taral_batch* b);

/* Fault-injection hook for tests (no counterpart in the reference, whose CHECK macro exits the process on any CUDA
 * error, gpu/pdhg.cu:36-43): from now on, a context or batch whose device allocations would exceed `bytes` in total
 * fails as if the device were out of memory, and its create call returns TARAL_ERR_ALLOC after releasing what it
 * had allocated. 0 (the default) removes the limit. Process-wide; set it while no create call runs. */
void taral_set_device_alloc_limit(size_t bytes);

/* ------------------------------------------------------------------------------------------------------------
 * 7. Learned warm start: an MLP (in -> hidden x depth with GELU -> out) trained and evaluated with this library's
 *    own BF16 tensor-core kernels (FP32 accumulate), mapping a scenario's perturbation vector to an initial
 *    (x, y) for taral_pdhg_solve_warm / taral_batch_solve. No counterpart in the reference.
 *    Parameters, in order per layer: W (in x out, row-major) then b (out), FP32 on the host.
 * ------------------------------------------------------------------------------------------------------------ */
typedef struct taral_mlp taral_mlp;
int taral_mlp_create(int in_dim, int hidden, int depth, int out_dim, int max_batch, taral_mlp** out);
int64_t taral_mlp_param_count(const taral_mlp* h);
int taral_mlp_set_params(taral_mlp* h, const float* params);
int taral_mlp_get_params(taral_mlp* h, float* params);
/* y (batch x out, host) = MLP(x (batch x in, host)). */
int taral_mlp_forward(taral_mlp* h, int batch, const float* x, float* y);
/* Loss mean((MLP(x) - target)^2) and its gradient with respect to every parameter (host, parameter order). */
int taral_mlp_gradients(taral_mlp* h, int batch, const float* x, const float* target, double* loss, float* grads);
/* Upload a training set once (count rows of x and target), then run Adam over shuffled mini-batches. */
int taral_mlp_set_dataset(taral_mlp* h, int count, const float* x, const float* target);
int taral_mlp_train(taral_mlp* h, int epochs, int batch, float lr, uint64_t seed, double* last_loss);
const char* taral_mlp_last_error(const taral_mlp* h);
void taral_mlp_destroy(taral_mlp* h);
/* The MLP's GEMM on device buffers: C (M x N, f32) = op(A) op(B) with bf16 A, B; ta: A is stored K x M; tb: B is
 * stored N x K; slices > 1: split-K with a workspace of slices * M * N floats. Asynchronous on `stream`. */
int taral_gemm_bf16(int M, int N, int K, int ta, int tb, const void* A, const void* B, float* C, int slices,
                    float* workspace, void* stream);
/* The MLP's forward GEMM on the tcgen05 tensor cores (accumulator in tensor memory): C (M x N, f32) = A Bt^T with
 * A (M x K) and Bt (N x K) bf16, row-major, 16-byte aligned, K a multiple of 8. err: a device int that is set to 1
 * if a completion wait gave up (C is then undefined); it is never cleared here. Asynchronous on `stream`. */
int taral_gemm_bf16_tc(int M, int N, int K, const void* A, const void* Bt, float* C, int* err, void* stream);
/* The general tcgen05 GEMM behind the MLP's three GEMMs: C (M x N, f32, row stride ldc) = sum_k A(m, k) B(n, k) with
 * bf16 operands brought in by TMA. a_mn = 0: A stored [M][lda] (K contiguous); a_mn = 1: A stored [K][lda] (M
 * contiguous); likewise b_mn for B with N. lda and ldb multiples of 8, A and B 16-byte aligned. slices > 1 splits K
 * into that many slices whose partials (in `workspace`, slices * M * ldc floats) are summed in slice order. err as
 * for taral_gemm_bf16_tc. Asynchronous on `stream`. */
int taral_gemm_bf16_umma(int M, int N, int K, const void* A, int lda, int a_mn, const void* B, int ldb, int b_mn,
                         float* C, int ldc, int slices, float* workspace, int* err, void* stream);

/* ------------------------------------------------------------------------------------------------------------
 * 6. KKT evaluation without device allocation. No counterpart in the reference: it is an addition for callers
 *    that cannot call cudaMalloc -- a host whose GPU memory is reserved up front by another allocator, or a loop
 *    that must not take cudaMalloc's implicit device synchronisation. It computes, on device vectors the caller
 *    holds, the same 10 FP64 KKT scalars as pdhg_eval(ctx, 0, f, out) (same kernels, same fixed-order sums).
 *
 *    Scratch: a file-scope device array of 23,696 bytes (2 x 296 x 5 partial sums + 2 tickets), held by every GPU
 *    that loads the library until the process exits. Every call shares it and it keeps the last call's contents;
 *    each call clears the tickets that must start at zero. Calls whose work overlaps on the GPU (different streams,
 *    threads or processes sharing the device) race on the array: serialise them. The first call on each device
 *    looks up the array's device address (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture. Nothing is allocated: no cudaMalloc, cudaFree or allocating library routine.
 *
 *    dtype: TARAL_FP64 (all 13 vectors double) or TARAL_FP32 (all float). Row vectors (length m): Ax, z, rl, ru,
 *    Dr, zlast; column vectors (length n): x, ATz, c, l, u, Dc, xlast -- all device pointers, in the scaled space
 *    of part 1. out10: device pointer to 10 doubles, written in the slot order of pdhg_eval. Asynchronous on
 *    `stream` (NULL: the legacy default stream). m and n above TARAL_NOALLOC_MAX_DIM are rejected with
 *    TARAL_ERR_INPUT (the kernels index with int and stride by 296 x 256).
 * ------------------------------------------------------------------------------------------------------------ */
#define TARAL_NOALLOC_MAX_DIM 2000000000
int taral_kkt_eval_noalloc(int m, int n, int dtype, double f, const void* Ax, const void* z, const void* rl,
                           const void* ru, const void* Dr, const void* zlast, const void* x, const void* ATz,
                           const void* c, const void* l, const void* u, const void* Dc, const void* xlast,
                           double* out10, void* stream);

/* ------------------------------------------------------------------------------------------------------------
 * 8. Independent check of answers on the original models, on the device (FP64), for one model or a whole batch:
 *    the reference checker's semantics -- benchmarks/orig_check.py:63-88 (objective incl. the objective row's
 *    constant, largest row violation relative to 1 + |b|, largest bound violation) and gpu/vector_check.py:46-74
 *    (weak-duality bound LB(y) for y and -y, d = c - A'y; a term whose minimising bound is infinite, |v| >= 1e20,
 *    is dropped and recorded as dual infeasibility; the sign with the smaller one is kept). Shares no code with the
 *    solver: the models are uploaded unscaled in FP64.
 * ------------------------------------------------------------------------------------------------------------ */
typedef struct taral_check {
    double objective;         /* c'x + obj_const */
    double row_violation_rel; /* max_i max(lo_i - a_i x, a_i x - up_i, 0) / (1 + |b_i|) */
    double bound_violation;   /* max_j max(l_j - x_j, x_j - u_j, 0) */
    double dual_bound;        /* strict weak-duality bound; NaN when a term was dropped or the dual is not checked */
    double dual_obj_loose;    /* LB with dropped terms left out (not a rigorous bound); NaN when not checked */
    double dual_infeas_rel;   /* the largest dropped term, relative; NaN when not checked */
    double dual_gap_rel;      /* (objective - dual_obj_loose) / max(1, |objective|); NaN when not checked */
    int dual_sign;            /* +1 or -1: the sign of y used; 0: not checked (no y, or a maximisation model) */
    int pad;
} taral_check;
/* x[i] (n_i, original space) and optional y[i] (m_i, row multipliers; y or y itself NULL: primal side only) of
 * model i. rhs: NULL, or per model NULL or the rows' right-hand sides b (the MPS RHS values; default: b = lo where
 * lo is finite, else up). out[i]: model i's check. */
int taral_check_models(const taral_model* models, int count, const double* const* rhs, const double* const* x,
                       const double* const* y, taral_check* out);

#ifdef __cplusplus
}
#endif
#endif /* TARAL_PDHG_H */
