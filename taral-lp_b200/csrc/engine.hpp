// Internal interface between the C ABI / host driver and the device engine (one object per context).
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <vector_types.h>

#include "../../include/taral_pdhg.h"

namespace taral {

// The backend concept of the reference driver (gpu/pdhg.cu:761-849 calls these on Gpu<T> / Cpu<T>).
struct EngineBase {
    std::string name;
    size_t mem_used = 0;
    int64_t launches = 0;
    int64_t nnz = 0;  // nonzeros of A
    int tuned[2] = {0, 0};  // row-split policy chosen by the autotuner for A and A^T
    bool per_thread[2] = {false, false};  // A, A^T use the one-thread-per-row SpMV kernel
    virtual ~EngineBase() = default;
    virtual double power_norm(int iters) = 0;
    virtual void set_steps(double tau, double sigma) = 0;
    virtual void start(const double* x0, const double* z0) = 0;
    virtual void iterate(int steps) = 0;
    virtual void eval(bool avg, double f, double* out10) = 0;
    virtual void eval_pair(double f, double* cur10, double* avg10) = 0;
    virtual void restart(bool avg, double f) = 0;
    virtual void download(bool avg, double f, double* x, double* z) = 0;
    virtual void sync() = 0;
    // Device time on the context stream between mark() and elapsed_ms() (CUDA events).
    virtual void mark() = 0;
    virtual double elapsed_ms() = 0;
    // `reps` PDHG iterations launched one kernel at a time, each row-phase and column-phase kernel bracketed by
    // CUDA events on the context stream; average milliseconds per launch of each.
    virtual void profile_phases(int reps, double* row_ms, double* col_ms) = 0;
    // The scaling factors and scaled matrix values held on the device, widened to double, in the model's row order
    // (any pointer may be NULL): Dr (m), Dc (n), A's values (nnz, rows in the model's order, each row's entries in
    // column order), A^T's values (nnz, A^T's entry order).
    virtual void scaled_values(double* Dr, double* Dc, double* a_val, double* at_val) = 0;
    // Host copies of the scaled c, rl, ru kept at creation (the driver's step-size and norm set-up reads them).
    std::vector<double> hc, hrl, hru;
};

std::unique_ptr<EngineBase> make_engine(int precision);
void engine_init(EngineBase& e, int precision, const taral_csr& A, const taral_csr& AT, const double* c,
                 const double* l, const double* u, const double* rl, const double* ru, const double* Dr,
                 const double* Dc, int m, int n, int eval_freq, unsigned flags);
std::vector<int4> build_row_blocks(const int64_t* ptr, int rows);
void keep_pool_memory(int dev);  // the device pool keeps freed memory for reuse by later contexts
// False when `more` bytes on top of `used` would pass the limit set by taral_set_device_alloc_limit.
bool alloc_allowed(size_t used, size_t more);
// Blocks of at most `tile` nonzeros and `rows_max` rows (a longer row is a block of its own).
std::vector<int4> build_row_blocks(const int64_t* ptr, int rows, int tile, int rows_max);
// The block list with the flags of row-split policy 0..4 (kernels.cuh, kPolicies); returns false when the policy
// changes nothing on this list (no block it applies to).
bool apply_row_split(std::vector<int4>& blk, int policy);
int forced_row_split();  // TARAL_ROWSPLIT (0..4) when set, else -1
// Set-up from the column-wise model with the scaling done on the device, bit-identical to the reference's: P gets
// Dr, Dc, the scaled vectors and the norms (its matrices stay empty); host_s: seconds of host work.
struct Scaled;
void engine_init_model(EngineBase& e, int precision, const taral_model& md, double sign, Scaled& P, int eval_freq,
                       unsigned flags, double* host_s);

}  // namespace taral

// A pdhg_ctx built by engine_init_model (the C ABI's pdhg_create_model); P as for engine_init_model.
int pdhg_create_model_ctx(const taral_model* md, int precision, int eval_freq, unsigned flags, taral::Scaled& P,
                          pdhg_ctx** out);

namespace taral {

}  // namespace taral
