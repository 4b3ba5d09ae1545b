/*
 * chol_ref_bridge.cpp — C entry points over the reference's own
 * IncrementalCholesky (src/deformation/IncrementalCholesky.cpp, compiled as
 * it lies in the reference tree with oracle/shim_chol/core/Types.h).  TEST
 * INFRASTRUCTURE ONLY: built into oracle/_ref/libpbfref_chol.so.
 *
 * cholref_run replays a script on one matrix: analyze, then for each of
 * `steps` constraint masks either a full factorization (full[s] != 0) or an
 * update of the listed changed columns, then a solve of rhs; the solutions
 * are written to out (steps x n).
 */
#include <vector>

#include "deformation/IncrementalCholesky.h"

extern "C" int cholref_run(int n, const int* colptr, const int* rows, const double* vals, int steps,
                           const char* masks, const int* full, const int* changed_ptr, const int* changed,
                           const double* rhs, double* out)
{
    const int nnz = colptr[n];
    ESparseMatrix A(n, std::vector<int>(colptr, colptr + n + 1), std::vector<int>(rows, rows + nnz),
                    std::vector<double>(vals, vals + nnz));
    IncrementalCholesky L;
    L.analyze(A);
    for (int s = 0; s < steps; ++s) {
        L.setConstrained(std::vector<char>(masks + (size_t)s * n, masks + (size_t)(s + 1) * n));
        if (full[s]) {
            L.factorizeFull(A);
        } else {
            L.updateColumns(A, std::vector<int>(changed + changed_ptr[s], changed + changed_ptr[s + 1]));
        }
        EVecX b((size_t)n);
        for (int i = 0; i < n; ++i) b[(size_t)i] = rhs[(size_t)s * n + i];
        L.solveInPlace(b);
        for (int i = 0; i < n; ++i) out[(size_t)s * n + i] = b[(size_t)i];
    }
    return L.ok() ? 0 : 1;
}
