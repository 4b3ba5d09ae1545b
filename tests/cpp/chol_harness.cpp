// chol_harness.cpp — the library's IncrementalCholesky
// (realtime-fsi-engine_b200/host/IncrementalCholesky.cpp) behind the same C
// script interface as the reference bridge oracle/chol_ref_bridge.cpp, so a
// test can replay one script on both and compare the solutions.  Built by
// tests/test_deform_cpu.py.
#include <vector>

#include "deformation/IncrementalCholesky.h"

extern "C" int chol_run(int n, const int* colptr, const int* rows, const double* vals, int steps, const char* masks,
                        const int* full, const int* changed_ptr, const int* changed, const double* rhs, double* out)
{
    pbfdrop::SymCsc A;
    A.n = n;
    A.colptr.assign(colptr, colptr + n + 1);
    A.rows.assign(rows, rows + colptr[n]);
    A.vals.assign(vals, vals + colptr[n]);
    pbfdrop::IncrementalCholesky L;
    L.analyze(A);
    for (int s = 0; s < steps; ++s) {
        L.setConstrained(std::vector<char>(masks + (size_t)s * n, masks + (size_t)(s + 1) * n));
        if (full[s])
            L.factorizeFull(A);
        else
            L.updateColumns(A, std::vector<int>(changed + changed_ptr[s], changed + changed_ptr[s + 1]));
        std::vector<double> b(rhs + (size_t)s * n, rhs + (size_t)(s + 1) * n);
        L.solveInPlace(b);
        for (int i = 0; i < n; ++i) out[(size_t)s * n + i] = b[(size_t)i];
    }
    return L.ok() ? 0 : 1;
}
