// Test shim over the engine's host set-up code (taral-lp_b200/csrc/scaling.cpp): the threaded CSR transpose and the
// model matrices, copied out into caller buffers so that a test can compare them with a plain restatement.
#include <algorithm>

#include "host.hpp"

using namespace taral;

extern "C" int64_t transpose_into(const int64_t* ptr, const int32_t* idx, const double* val, int rows, int cols,
                                  int threads, int64_t* optr, int32_t* oidx, double* oval) {
    const Csr t = transpose_par(ptr, idx, val, rows, cols, threads);
    std::copy(t.ptr.begin(), t.ptr.end(), optr);
    std::copy(t.idx.begin(), t.idx.end(), oidx);
    std::copy(t.val.begin(), t.val.end(), oval);
    return int64_t(t.idx.size());
}

// by_ref = 1: model_matrices_ref, A^T read through the returned reference; 0: model_matrices (copies).
// Returns A's nonzero count; *refers_to_model = 1 when A^T is the model's own arrays.
extern "C" int64_t model_matrices_into(int m, int n, const int64_t* col_ptr, const int32_t* row_idx, const double* val,
                                       int threads, int by_ref, int64_t* aptr, int32_t* aidx, double* aval,
                                       int64_t* tptr, int32_t* tidx, double* tval, int* refers_to_model) {
    taral_model md{};
    md.m = m, md.n = n, md.col_ptr = col_ptr, md.row_idx = row_idx, md.val = val;
    Csr A, AT;
    CsrRef at;
    if (by_ref) {
        at = model_matrices_ref(md, A, AT, threads);
    } else {
        model_matrices(md, A, AT, threads);
        at = ref(AT);
    }
    *refers_to_model = at.ptr == col_ptr;
    std::copy(A.ptr.begin(), A.ptr.end(), aptr);
    std::copy(A.idx.begin(), A.idx.end(), aidx);
    std::copy(A.val.begin(), A.val.end(), aval);
    std::copy(at.ptr, at.ptr + n + 1, tptr);
    std::copy(at.idx, at.idx + at.nnz(), tidx);
    std::copy(at.val, at.val + at.nnz(), tval);
    return int64_t(A.idx.size());
}
