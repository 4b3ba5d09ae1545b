/*
 * Stand-in for the reference's include/core/Types.h, used only to compile
 * the reference's own src/deformation/IncrementalCholesky.cpp under
 * oracle/_ref (Eigen/Core, Eigen/Sparse and CHOLMOD are absent from the
 * reference tree and from this machine).  It provides the two types that
 * file uses, written here: ESparseMatrix, a column-compressed sparse matrix
 * of doubles with rows() and the InnerIterator (row(), value(), advance,
 * test for end) the file walks columns with, and EVecX, a dense vector with
 * operator[].  Nothing else of Types.h is declared.
 */
#ifndef TYPES_H
#define TYPES_H
#include <cstddef>
#include <vector>

class ESparseMatrix {
public:
    ESparseMatrix() = default;
    // CSC with ascending row indices per column (the order the reference's
    // matrices have after setFromTriplets).
    ESparseMatrix(int n, std::vector<int> colptr, std::vector<int> rowidx, std::vector<double> vals)
        : n_(n), p_(std::move(colptr)), i_(std::move(rowidx)), x_(std::move(vals)) {}
    long rows() const { return n_; }
    long cols() const { return n_; }
    class InnerIterator {
    public:
        InnerIterator(const ESparseMatrix& A, int col) : A_(A), k_(A.p_[(size_t)col]), end_(A.p_[(size_t)col + 1]) {}
        explicit operator bool() const { return k_ < end_; }
        InnerIterator& operator++() { ++k_; return *this; }
        long row() const { return A_.i_[(size_t)k_]; }
        double value() const { return A_.x_[(size_t)k_]; }
    private:
        const ESparseMatrix& A_;
        int k_, end_;
    };
private:
    int n_ = 0;
    std::vector<int> p_, i_;
    std::vector<double> x_;
};

class EVecX {
public:
    explicit EVecX(std::size_t n = 0) : v_(n, 0.0) {}
    double& operator[](std::size_t i) { return v_[i]; }
    double operator[](std::size_t i) const { return v_[i]; }
    std::size_t size() const { return v_.size(); }
    double* data() { return v_.data(); }
private:
    std::vector<double> v_;
};

#endif
