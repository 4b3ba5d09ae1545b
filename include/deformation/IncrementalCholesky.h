// IncrementalCholesky.h — LDL^T of a fixed-pattern symmetric matrix whose
// constraint set changes, with column updates along elimination-tree paths.
//
// Replaces the reference's IncrementalCholesky (include/deformation/
// IncrementalCholesky.h:1-96, src/deformation/IncrementalCholesky.cpp) without
// Eigen.  Method (Herholz & Alexa / Davis):
//   * the working matrix A^B equals A with row and column k replaced by the
//     k-th unit vector for every constrained k (it only removes entries, so
//     one symbolic analysis of the unconstrained A — elimination tree and
//     nonzero pattern of L — serves every constraint state);
//   * the numeric factor is computed column by column with the up-looking
//     LDL^T recurrence;
//   * after a constraint change only the columns on elimination-tree paths
//     from the changed columns to the root are recomputed, in ascending order.
// L is unit lower triangular (strict lower part stored by columns, rows
// ascending), D its diagonal.  Host code, FP64.
#pragma once

#include <cstdint>
#include <vector>

namespace pbfdrop {

// Symmetric sparse matrix, both triangles, compressed by columns with
// ascending row indices.
struct SymCsc {
    int n = 0;
    std::vector<int> colptr, rows;
    std::vector<double> vals;
    double at(int i, int j) const;  // A(i, j), 0 when not stored
};

// Build a SymCsc from (row, col, value) triplets (duplicates summed; the
// caller supplies both triangles).
SymCsc sym_from_triplets(int n, const std::vector<int>& r, const std::vector<int>& c,
                         const std::vector<double>& v);

class IncrementalCholesky {
public:
    // Symbolic analysis of the unconstrained A (upper triangle is read).
    void analyze(const SymCsc& A);
    // constrained[k] != 0 detaches k (row/column k of A^B = e_k).
    void setConstrained(std::vector<char> constrained);
    // Numeric factorization of A^B, every column.
    void factorizeFull(const SymCsc& A);
    // Recompute the columns on the tree paths from `changed` to the root.
    void updateColumns(const SymCsc& A, const std::vector<int>& changed);
    // Solve A^B x = b in place.
    void solveInPlace(std::vector<double>& b) const;

    int size() const { return n_; }
    bool ok() const { return ok_; }
    const std::vector<int>& parent() const { return parent_; }
    size_t factorNonzeros() const { return li_.size(); }

private:
    int n_ = 0;
    bool ok_ = false;
    std::vector<int> parent_;          // elimination tree, -1 at roots
    std::vector<int> lp_, li_;         // pattern of strict lower L by columns
    std::vector<double> lx_, d_;
    std::vector<char> cons_;
    std::vector<double> work_;         // dense accumulator of the current row
    std::vector<int> stack_, visit_;   // row-pattern scratch and visit stamps
    int stamp_ = 0;

    int slot(int col, int row) const;  // position of L(row, col) in li_/lx_
    void column(const SymCsc& A, int k);
};

}  // namespace pbfdrop
