// Solver entry of the C ABI (include/taral_pdhg.h, parts 2 and 3): input gate, scaling, device engine, the
// restarted-average driver and the original-space check, for one model in memory; plus the MPS handle.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "engine.hpp"
#include "host.hpp"
#include "solve.hpp"

namespace taral {

const char* input_error(const taral_model& md) {  // gpu/pdhg_input.hpp:7-17
    bool quadratic = md.n_quadratic > 0;
    bool integer = false;
    if (md.is_int)
        for (int j = 0; j < md.n && !integer; ++j) integer = md.is_int[j] != 0;
    if (quadratic && integer)
        return "PDHG supports continuous LPs only; quadratic objectives and integer variables are unsupported";
    if (quadratic) return "PDHG supports continuous LPs only; quadratic objectives are unsupported";
    if (integer)
        return "PDHG supports continuous LPs only; integer variables are unsupported (no LP relaxation is solved)";
    return nullptr;
}

std::string check_model(const taral_model& md) {
    if (md.m < 0 || md.n < 0) return "negative dimensions";
    if (!md.col_ptr) return "col_ptr is NULL";
    if (md.n && (!md.cost || !md.col_lo || !md.col_up)) return "column arrays are NULL";
    if (md.m && (!md.row_lo || !md.row_up)) return "row arrays are NULL";
    if (md.col_ptr[0] != 0) return "col_ptr[0] != 0";
    for (int j = 0; j < md.n; ++j)
        if (md.col_ptr[j + 1] < md.col_ptr[j]) return "col_ptr is not monotone";
    int64_t nnz = md.col_ptr[md.n];
    if (nnz && (!md.row_idx || !md.val)) return "entry arrays are NULL";
    if (nnz > INT32_MAX - 64) return "more than 2^31 nonzeros";
    for (int64_t k = 0; k < nnz; ++k)
        if (md.row_idx[k] < 0 || md.row_idx[k] >= md.m) return "row index out of range";
    return "";
}

int solve_model(const taral_model& md, const Options& o, SolveResult& res, const double* x0_orig,
                const double* y0_orig) {
    res = SolveResult();
    if (input_error(md)) return TARAL_ERR_UNSUPPORTED;
    std::string bad = check_model(md);
    if (!bad.empty()) {
        res.error = bad;
        return TARAL_ERR_INPUT;
    }
    auto t = Clock::now();
    Scaled P;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        res.error = "no CUDA device";
        return TARAL_ERR_NO_DEVICE;
    }
    if (cudaFree(nullptr) != cudaSuccess) {  // context creation, counted in setup
        res.error = "CUDA context creation failed";
        return TARAL_ERR_CUDA;
    }
    res.device_init_s = since(t);
    t = Clock::now();
    std::unique_ptr<EngineBase> e;
    try {
        e = make_engine(o.precision);
        engine_init_model(*e, o.precision, md, md.maximize ? -1.0 : 1.0, P, o.eval_freq,
                          o.graph ? 0u : TARAL_FLAG_NO_GRAPH, &res.scale_s);
    } catch (const std::bad_alloc&) {
        res.error = "host allocation failed";
        return TARAL_ERR_ALLOC;
    } catch (const std::exception& ex) {
        res.error = ex.what();
        return TARAL_ERR_CUDA;
    } catch (...) {
        res.error = "device initialisation failed (out of device memory?)";
        return TARAL_ERR_ALLOC;
    }
    res.transfer_s = since(t) - res.scale_s;  // upload, device scaling and narrowing
    res.device_mem_bytes = e->mem_used;
    res.device_name = e->name;
    // Warm start in the original space -> scaled space: x_s = x / Dc, z_s = y / Dr.
    std::vector<double> xs0, zs0;
    if (x0_orig) {
        xs0.resize(size_t(P.n));
        for (int j = 0; j < P.n; ++j) xs0[j] = x0_orig[j] / P.Dc[j];
    }
    if (y0_orig) {
        zs0.resize(size_t(P.m));
        for (int i = 0; i < P.m; ++i) zs0[i] = y0_orig[i] / P.Dr[i];
    }
    double setup = res.scale_s + res.device_init_s + res.transfer_s;
    t = Clock::now();
    try {
        res.outcome = run(*e, DriverData::of(P), o, o.time_limit - setup, x0_orig ? xs0.data() : nullptr,
                          y0_orig ? zs0.data() : nullptr);
    } catch (const std::exception& ex) {
        res.error = ex.what();
        return TARAL_ERR_CUDA;
    } catch (...) {
        res.error = "CUDA error during the solve";
        return TARAL_ERR_CUDA;
    }
    res.solve_s = since(t);
    res.kernel_launches = e->launches;
    res.nnz = e->nnz;
    const int tuned_a = e->tuned[0] + (e->per_thread[0] ? 10 : 0), tuned_t = e->tuned[1] + (e->per_thread[1] ? 10 : 0);
    t = Clock::now();
    res.fin = finish_point(md, P, res.outcome);
    const double finish_s = since(t);
    t = Clock::now();
    e.reset();  // device buffers, graph and stream released here rather than at scope exit, so they can be timed
    const double release_s = since(t);
    if (std::getenv("TARAL_TIMING"))
        std::fprintf(stderr, "taral: scale %.4f s, transfer %.4f s, solve %.4f s, finish %.4f s, release %.4f s, "
                     "row-split policy A %d A^T %d (10: thread per row)\n", res.scale_s, res.transfer_s, res.solve_s, finish_s, release_s,
                     tuned_a, tuned_t);
    res.m = P.m, res.n = P.n;
    return TARAL_OK;
}

}  // namespace taral

// ================================================================================================ C ABI
extern "C" void taral_options_default(taral_options* o) {
    if (!o) return;
    taral::Options d;
    o->tol = d.tol, o->time_limit = d.time_limit, o->max_iter = d.max_iter, o->eval_freq = d.eval_freq;
    o->row_rel = d.row_rel, o->verbose = 0, o->graph = 1, o->precision = TARAL_FP64;
}

extern "C" const char* taral_pdhg_input_error(const taral_model* md) { return md ? taral::input_error(*md) : nullptr; }

static int solve_c(const taral_model* md, const taral_options* o, taral_outcome* out, double* x_out, double* y_out,
                   const double* x0, const double* y0) {
    if (!md || !o || !out) return TARAL_ERR_INPUT;
    std::memset(out, 0, sizeof *out);
    taral::Options op;
    op.tol = o->tol, op.time_limit = o->time_limit, op.max_iter = o->max_iter;
    op.eval_freq = o->eval_freq > 0 ? o->eval_freq : 64;
    op.row_rel = o->row_rel, op.verbose = o->verbose != 0, op.graph = o->graph != 0;
    op.precision = o->precision == TARAL_FP32 ? TARAL_FP32 : TARAL_FP64;
    taral::SolveResult r;
    int rc = taral::solve_model(*md, op, r, x0, y0);
    if (rc != TARAL_OK) return rc;
    const taral::Outcome& oc = r.outcome;
    out->status = oc.status, out->iterations = oc.iterations, out->restarts = oc.restarts;
    out->from_average = oc.from_average ? 1 : 0;
    out->rel_primal = oc.rel_primal, out->rel_dual = oc.rel_dual, out->rel_gap = oc.rel_gap;
    out->norm_a = oc.norm_a, out->primal_weight = oc.omega;
    out->objective = r.fin.objective, out->max_row_violation = r.fin.max_row_violation;
    out->max_bound_violation = r.fin.max_bound_violation;
    out->scale_s = r.scale_s, out->device_init_s = r.device_init_s, out->transfer_s = r.transfer_s;
    out->solve_s = r.solve_s, out->power_iter_s = oc.power_s, out->device_mem_bytes = r.device_mem_bytes;
    out->kernel_launches = r.kernel_launches, out->nnz = r.nnz;
    if (x_out) std::memcpy(x_out, r.fin.x.data(), r.fin.x.size() * sizeof(double));
    if (y_out) std::memcpy(y_out, r.fin.y.data(), r.fin.y.size() * sizeof(double));
    return TARAL_OK;
}

extern "C" int taral_pdhg_solve(const taral_model* md, const taral_options* o, taral_outcome* out, double* x_out,
                                double* y_out) {
    return solve_c(md, o, out, x_out, y_out, nullptr, nullptr);
}

extern "C" int taral_pdhg_solve_warm(const taral_model* md, const taral_options* o, const double* x0,
                                     const double* y0, taral_outcome* out, double* x_out, double* y_out) {
    return solve_c(md, o, out, x_out, y_out, x0, y0);
}

extern "C" int pdhg_create_model(const taral_model* md, int precision, int eval_freq, unsigned flags, pdhg_ctx** out,
                                 double* bnorm, double* cnorm) {
    if (!md || !out) return TARAL_ERR_INPUT;
    *out = nullptr;
    if (taral::input_error(*md)) return TARAL_ERR_UNSUPPORTED;
    if (!taral::check_model(*md).empty()) return TARAL_ERR_INPUT;
    if (precision != TARAL_FP64 && precision != TARAL_FP32) return TARAL_ERR_INPUT;
    taral::Scaled P;
    int rc = pdhg_create_model_ctx(md, precision, eval_freq, flags, P, out);
    if (rc == TARAL_OK) {
        if (bnorm) *bnorm = P.bnorm;
        if (cnorm) *cnorm = P.cnorm;
    }
    return rc;
}

// ------------------------------------------------------------------------------------------------ MPS handle
struct taral_mps {
    taral::Model md;
};
static thread_local std::string g_mps_error;

extern "C" int taral_mps_read(const char* path, taral_mps** out) {
    if (!path || !out) return TARAL_ERR_INPUT;
    *out = nullptr;
    try {
        auto* h = new taral_mps;
        try {
            h->md = taral::read_mps(path);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        g_mps_error.clear();
        return TARAL_OK;
    } catch (const taral::ParseError& e) {
        g_mps_error = e.what();
        return TARAL_ERR_PARSE;
    } catch (const std::bad_alloc&) {
        g_mps_error = "out of memory";
        return TARAL_ERR_ALLOC;
    }
}
extern "C" const char* taral_mps_error(void) { return g_mps_error.c_str(); }
extern "C" int taral_mps_model(const taral_mps* h, taral_model* view) {
    if (!h || !view) return TARAL_ERR_INPUT;
    *view = h->md.view();
    return TARAL_OK;
}
extern "C" const char* taral_mps_col_name(const taral_mps* h, int j) {
    return h && j >= 0 && size_t(j) < h->md.col_names.size() ? h->md.col_names[j].c_str() : nullptr;
}
extern "C" const char* taral_mps_row_name(const taral_mps* h, int i) {
    return h && i >= 0 && size_t(i) < h->md.row_names.size() ? h->md.row_names[i].c_str() : nullptr;
}
extern "C" const char* taral_mps_name(const taral_mps* h) { return h ? h->md.name.c_str() : nullptr; }
extern "C" void taral_mps_free(taral_mps* h) { delete h; }
