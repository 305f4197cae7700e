// Whole-solve entry shared by the C ABI and the CLI.
#pragma once
#include <string>

#include "host.hpp"

namespace taral {

struct SolveResult {
    Outcome outcome;
    Finished fin;
    double scale_s = 0, device_init_s = 0, transfer_s = 0, solve_s = 0;
    size_t device_mem_bytes = 0;
    int64_t kernel_launches = 0, nnz = 0;
    int m = 0, n = 0;
    std::string device_name, error;
};

const char* input_error(const taral_model& md);
std::string check_model(const taral_model& md);
// Scale, upload, run the driver and check the point on the original model. x0_orig / y0_orig: optional warm
// start (original space; y in the minimisation form of the dual output). Returns a taral_status.
int solve_model(const taral_model& md, const Options& o, SolveResult& res, const double* x0_orig = nullptr,
                const double* y0_orig = nullptr);

}  // namespace taral
