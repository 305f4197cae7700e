// `pdhg` command line: the reference CLI's flags, status line, JSON report, .sol and .dual files and exit codes
// (gpu/pdhg.cu:851-992), on the B200 engine. The engine has no CPU backend: `--device cpu` is refused after the
// input gate (exit 2), so unsupported models still report `status unsupported_model` on either device value.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "host.hpp"
#include "solve.hpp"

using namespace taral;

static const char* kUsage =
    "usage: pdhg MODEL.mps [--device gpu] [--tol 1e-4] [--time-limit S] [--max-iter N] [--json OUT.json] "
    "[--sol OUT.sol] [--dual OUT.dual] [--fp32] [--eval-freq 64] [--row-rel 0] [--no-graph] [--verbose]\n";

int main(int argc, char** argv) {
    const char *model = nullptr, *json = nullptr, *sol = nullptr, *dual = nullptr;
    std::string device = "gpu";
    Options o;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&] {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", a.c_str());
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--device") device = next();
        else if (a == "--threads") (void)next();  // accepted for compatibility; the GPU engine has no thread pool
        else if (a == "--tol") o.tol = std::atof(next());
        else if (a == "--time-limit") o.time_limit = std::atof(next());
        else if (a == "--max-iter") o.max_iter = std::atoll(next());
        else if (a == "--row-rel") o.row_rel = std::atof(next());
        else if (a == "--eval-freq") o.eval_freq = std::max(1, std::atoi(next()));
        else if (a == "--json") json = next();
        else if (a == "--sol") sol = next();
        else if (a == "--dual") dual = next();
        else if (a == "--fp32") o.precision = TARAL_FP32;
        else if (a == "--no-graph") o.graph = false;
        else if (a == "--verbose") o.verbose = true;
        else model = argv[i];
    }
    if (!model || (device != "gpu" && device != "cpu")) {
        std::fputs(kUsage, stderr);
        return 2;
    }
    auto t_start = Clock::now();
    Model md;
    try {
        md = read_mps(model);
    } catch (const ParseError& e) {
        std::printf("status parse_error: %s\n", e.what());
        return 1;
    }
    taral_model v = md.view();
    if (const char* why = input_error(v)) {  // gpu/pdhg_input.hpp:20-26: before scaling, device init or any file
        std::printf("status unsupported_model\n");
        std::fprintf(stderr, "%s\n", why);
        return 2;
    }
    if (device == "cpu") {
        std::fprintf(stderr, "this engine runs on the GPU only (no CPU backend); use --device gpu\n");
        return 2;
    }
    double parse_s = since(t_start);
    SolveResult r;
    int rc = solve_model(v, o, r);
    if (rc != TARAL_OK) {
        std::fprintf(stderr, "error %d: %s\n", rc, r.error.c_str());
        return 1;
    }
    const Outcome& oc = r.outcome;
    double setup = parse_s + r.scale_s + r.device_init_s + r.transfer_s;
    double total = since(t_start);
    const char* prec = o.precision == TARAL_FP32 ? "fp32" : "fp64";
    std::printf("status %s objective %.12g iterations %lld restarts %d rel_p %.2e rel_d %.2e rel_gap %.2e setup %.3fs "
                "solve %.3fs total %.3fs device %s\n",
                status_name(oc.status), r.fin.objective, (long long)oc.iterations, oc.restarts, oc.rel_primal,
                oc.rel_dual, oc.rel_gap, setup, r.solve_s, total, r.device_name.c_str());
    if (json)
        if (std::FILE* f = std::fopen(json, "w")) {
            std::fprintf(f,
                         "{\"solver\": \"taral-pdhg-b200 (near-optimal)\", \"status\": \"%s\", \"objective\": %.17g, "
                         "\"rel_primal\": %.6e, \"rel_dual\": %.6e, \"rel_gap\": %.6e, \"tol\": %.3g, \"iterations\": %lld, "
                         "\"restarts\": %d, \"point\": \"%s\", \"max_row_violation\": %.6e, \"max_bound_violation\": %.6e, "
                         "\"setup_s\": %.6f, \"parse_s\": %.6f, \"scale_s\": %.6f, \"device_init_s\": %.6f, \"transfer_s\": %.6f, "
                         "\"solve_s\": %.6f, \"power_iter_s\": %.6f, \"total_s\": %.6f, \"device\": \"%s\", \"backend\": \"gpu\", "
                         "\"threads\": 0, \"precision\": \"%s\", \"rows\": %d, \"cols\": %d, \"nnz\": %lld, \"norm_a\": %.6e, "
                         "\"primal_weight\": %.6e, \"eval_freq\": %d, \"graph\": %s, \"device_mem_bytes\": %zu, "
                         "\"kernel_launches\": %lld}\n",
                         status_name(oc.status), r.fin.objective, oc.rel_primal, oc.rel_dual, oc.rel_gap, o.tol,
                         (long long)oc.iterations, oc.restarts, oc.from_average ? "average" : "current",
                         r.fin.max_row_violation, r.fin.max_bound_violation, setup, parse_s, r.scale_s,
                         r.device_init_s, r.transfer_s, r.solve_s, oc.power_s, total, r.device_name.c_str(), prec, r.m,
                         r.n, (long long)r.nnz, oc.norm_a, oc.omega, o.eval_freq, o.graph ? "true" : "false",
                         r.device_mem_bytes, (long long)r.kernel_launches);
            std::fclose(f);
        }
    if (sol)
        if (std::FILE* f = std::fopen(sol, "w")) {
            for (int j = 0; j < r.n; ++j) std::fprintf(f, "%s %.17g\n", md.col_names[j].c_str(), r.fin.x[j]);
            std::fclose(f);
        }
    if (dual)  // y = Dr z in minimisation form: any y gives a weak-duality bound an independent checker can recompute
        if (std::FILE* f = std::fopen(dual, "w")) {
            for (int i = 0; i < r.m; ++i) std::fprintf(f, "%s %.17g\n", md.row_names[i].c_str(), r.fin.y[i]);
            std::fclose(f);
        }
    return 0;
}
