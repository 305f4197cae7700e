// `pdhg` command line on the B200 engine. Interface kept from the reference CLI (gpu/pdhg.cu:851-992), because
// harnesses parse it: the flags, the status line, the JSON report's keys, the `.sol` / `.dual` line formats and
// the exit codes (0 any solve outcome, 1 parse or CUDA error, 2 usage or unsupported model). Any argument that is
// not a known flag names the model file. The engine has no CPU backend: `--device cpu` is refused after the input
// gate (exit 2), so unsupported models still report `status unsupported_model` on either device value.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host.hpp"
#include "solve.hpp"

using namespace taral;

namespace {

const char* const kUsage =
    "usage: pdhg MODEL.mps [--device gpu] [--tol 1e-4] [--time-limit S] [--max-iter N] [--json OUT.json] "
    "[--sol OUT.sol] [--dual OUT.dual] [--fp32] [--eval-freq 64] [--row-rel 0] [--no-graph] [--verbose]\n";

struct Invocation {
    const char* model = nullptr;
    const char* json = nullptr;
    const char* sol = nullptr;
    const char* dual = nullptr;
    std::string device = "gpu";
    Options opt;
};

enum class Opt { Device, Threads, Tol, TimeLimit, MaxIter, RowRel, EvalFreq, Json, Sol, Dual, Fp32, NoGraph, Verbose };

struct OptSpec {
    const char* flag;
    Opt id;
    bool has_value;
};

const OptSpec kOpts[] = {
    {"--device", Opt::Device, true},      {"--threads", Opt::Threads, true},   {"--tol", Opt::Tol, true},
    {"--time-limit", Opt::TimeLimit, true}, {"--max-iter", Opt::MaxIter, true}, {"--row-rel", Opt::RowRel, true},
    {"--eval-freq", Opt::EvalFreq, true}, {"--json", Opt::Json, true},         {"--sol", Opt::Sol, true},
    {"--dual", Opt::Dual, true},          {"--fp32", Opt::Fp32, false},        {"--no-graph", Opt::NoGraph, false},
    {"--verbose", Opt::Verbose, false},
};

const OptSpec* find_opt(const char* a) {
    for (const OptSpec& s : kOpts)
        if (std::strcmp(a, s.flag) == 0) return &s;
    return nullptr;
}

void apply(Invocation& inv, Opt id, const char* v) {
    Options& o = inv.opt;
    switch (id) {
        case Opt::Device: inv.device = v; break;
        case Opt::Threads: break;  // accepted for compatibility; the GPU engine has no host thread pool
        case Opt::Tol: o.tol = std::atof(v); break;
        case Opt::TimeLimit: o.time_limit = std::atof(v); break;
        case Opt::MaxIter: o.max_iter = std::atoll(v); break;
        case Opt::RowRel: o.row_rel = std::atof(v); break;
        case Opt::EvalFreq: o.eval_freq = std::atoi(v) < 1 ? 1 : std::atoi(v); break;
        case Opt::Json: inv.json = v; break;
        case Opt::Sol: inv.sol = v; break;
        case Opt::Dual: inv.dual = v; break;
        case Opt::Fp32: o.precision = TARAL_FP32; break;
        case Opt::NoGraph: o.graph = false; break;
        case Opt::Verbose: o.verbose = true; break;
    }
}

// Returns false (after a message on stderr) when a flag that needs a value ends the command line.
bool parse_args(int argc, char** argv, Invocation& inv) {
    int i = 1;
    while (i < argc) {
        const OptSpec* s = find_opt(argv[i]);
        if (!s) {
            inv.model = argv[i++];
            continue;
        }
        if (s->has_value && i + 1 >= argc) {
            std::fprintf(stderr, "option %s expects a value\n", argv[i]);
            return false;
        }
        apply(inv, s->id, s->has_value ? argv[i + 1] : nullptr);
        i += s->has_value ? 2 : 1;
    }
    return true;
}

// "name value" lines, value printed with 17 significant digits
void write_named(const char* path, const std::vector<std::string>& names, const std::vector<double>& v) {
    std::FILE* f = std::fopen(path, "w");
    if (!f) return;
    for (size_t k = 0; k < v.size(); ++k) std::fprintf(f, "%s %.17g\n", names[k].c_str(), v[k]);
    std::fclose(f);
}

struct Report {
    const SolveResult& r;
    const Options& o;
    double parse_s, setup_s, total_s;
};

void print_status(const Report& p) {
    const Outcome& oc = p.r.outcome;
    std::printf("status %s objective %.12g iterations %lld restarts %d rel_p %.2e rel_d %.2e rel_gap %.2e setup %.3fs "
                "solve %.3fs total %.3fs device %s\n",
                status_name(oc.status), p.r.fin.objective, (long long)oc.iterations, oc.restarts, oc.rel_primal,
                oc.rel_dual, oc.rel_gap, p.setup_s, p.r.solve_s, p.total_s, p.r.device_name.c_str());
}

void write_json(const char* path, const Report& p) {
    std::FILE* f = std::fopen(path, "w");
    if (!f) return;
    const SolveResult& r = p.r;
    const Outcome& oc = r.outcome;
    std::fprintf(f,
                 "{\"solver\": \"taral-pdhg-b200 (near-optimal)\", \"status\": \"%s\", \"objective\": %.17g, "
                 "\"rel_primal\": %.6e, \"rel_dual\": %.6e, \"rel_gap\": %.6e, \"tol\": %.3g, \"iterations\": %lld, "
                 "\"restarts\": %d, \"point\": \"%s\", \"max_row_violation\": %.6e, \"max_bound_violation\": %.6e, "
                 "\"setup_s\": %.6f, \"parse_s\": %.6f, \"scale_s\": %.6f, \"device_init_s\": %.6f, \"transfer_s\": %.6f, "
                 "\"solve_s\": %.6f, \"power_iter_s\": %.6f, \"total_s\": %.6f, \"device\": \"%s\", \"backend\": \"gpu\", "
                 "\"threads\": 0, \"precision\": \"%s\", \"rows\": %d, \"cols\": %d, \"nnz\": %lld, \"norm_a\": %.6e, "
                 "\"primal_weight\": %.6e, \"eval_freq\": %d, \"graph\": %s, \"device_mem_bytes\": %zu, "
                 "\"kernel_launches\": %lld}\n",
                 status_name(oc.status), r.fin.objective, oc.rel_primal, oc.rel_dual, oc.rel_gap, p.o.tol,
                 (long long)oc.iterations, oc.restarts, oc.from_average ? "average" : "current", r.fin.max_row_violation,
                 r.fin.max_bound_violation, p.setup_s, p.parse_s, r.scale_s, r.device_init_s, r.transfer_s, r.solve_s,
                 oc.power_s, p.total_s, r.device_name.c_str(), p.o.precision == TARAL_FP32 ? "fp32" : "fp64", r.m,
                 r.n, (long long)r.nnz, oc.norm_a, oc.omega, p.o.eval_freq, p.o.graph ? "true" : "false",
                 r.device_mem_bytes, (long long)r.kernel_launches);
    std::fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
    Invocation inv;
    if (!parse_args(argc, argv, inv)) return 2;
    if (!inv.model || (inv.device != "gpu" && inv.device != "cpu")) {
        std::fputs(kUsage, stderr);
        return 2;
    }
    const auto t_start = Clock::now();
    Model md;
    try {
        md = read_mps(inv.model);
    } catch (const ParseError& e) {
        std::printf("status parse_error: %s\n", e.what());
        return 1;
    }
    const taral_model v = md.view();
    if (const char* why = input_error(v)) {  // gpu/pdhg_input.hpp:20-26: before scaling, device init or any file
        std::printf("status unsupported_model\n");
        std::fprintf(stderr, "%s\n", why);
        return 2;
    }
    if (inv.device == "cpu") {
        std::fprintf(stderr, "this engine runs on the GPU only (no CPU backend); use --device gpu\n");
        return 2;
    }
    const double parse_s = since(t_start);
    SolveResult r;
    if (const int rc = solve_model(v, inv.opt, r); rc != TARAL_OK) {
        std::fprintf(stderr, "error %d: %s\n", rc, r.error.c_str());
        return 1;
    }
    const Report rep{r, inv.opt, parse_s, parse_s + r.scale_s + r.device_init_s + r.transfer_s, since(t_start)};
    print_status(rep);
    if (inv.json) write_json(inv.json, rep);
    if (inv.sol) write_named(inv.sol, md.col_names, r.fin.x);  // x in original units
    // y = Dr z in minimisation form: any y gives a weak-duality bound an independent checker can recompute
    if (inv.dual) write_named(inv.dual, md.row_names, r.fin.y);
    return 0;
}
