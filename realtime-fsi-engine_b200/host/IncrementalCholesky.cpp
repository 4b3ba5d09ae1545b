// IncrementalCholesky.cpp — see include/deformation/IncrementalCholesky.h.
//
// Symbolic step: elimination tree and column counts of L from the upper
// triangle (Liu's tree via path compression-free ancestor walks, as in
// Davis' LDL).  Numeric step (per column k, "up-looking"): the nonzero
// pattern of row k of L is the union of the tree paths from every i with
// A(i, k) != 0, i < k, up to k; solving the triangular system along that
// pattern in topological order yields L(k, :) and D(k).  Constrained
// columns (Herholz et al. 2017, Eq. 14) get L(k, :) = 0 and D(k) = 1.
#include "../../include/deformation/IncrementalCholesky.h"

#include <algorithm>
#include <map>

namespace pbfdrop {

double SymCsc::at(int i, int j) const
{
    const auto b = rows.begin() + colptr[j], e = rows.begin() + colptr[j + 1];
    const auto it = std::lower_bound(b, e, i);
    return (it != e && *it == i) ? vals[it - rows.begin()] : 0.0;
}

SymCsc sym_from_triplets(int n, const std::vector<int>& r, const std::vector<int>& c, const std::vector<double>& v)
{
    std::vector<std::map<int, double>> cols(n);
    for (size_t t = 0; t < r.size(); ++t) cols[c[t]][r[t]] += v[t];
    SymCsc A;
    A.n = n;
    A.colptr.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) {
        A.colptr[j + 1] = A.colptr[j] + (int)cols[j].size();
        for (const auto& kv : cols[j]) {
            A.rows.push_back(kv.first);
            A.vals.push_back(kv.second);
        }
    }
    return A;
}

void IncrementalCholesky::analyze(const SymCsc& A)
{
    n_ = A.n;
    ok_ = false;
    parent_.assign(n_, -1);
    std::vector<int> count(n_, 0), mark(n_, -1);
    for (int k = 0; k < n_; ++k) {
        mark[k] = k;
        for (int q = A.colptr[k]; q < A.colptr[k + 1] && A.rows[q] < k; ++q) {
            for (int j = A.rows[q]; mark[j] != k; j = parent_[j]) {
                if (parent_[j] == -1) parent_[j] = k;
                ++count[j];
                mark[j] = k;
            }
        }
    }
    lp_.assign(n_ + 1, 0);
    for (int j = 0; j < n_; ++j) lp_[j + 1] = lp_[j] + count[j];
    li_.assign(lp_[n_], 0);
    lx_.assign(lp_[n_], 0.0);
    d_.assign(n_, 0.0);
    std::vector<int> fill(n_, 0);
    std::fill(mark.begin(), mark.end(), -1);
    for (int k = 0; k < n_; ++k) {  // rows appended in increasing k: ascending per column
        mark[k] = k;
        for (int q = A.colptr[k]; q < A.colptr[k + 1] && A.rows[q] < k; ++q) {
            for (int j = A.rows[q]; mark[j] != k; j = parent_[j]) {
                li_[lp_[j] + fill[j]++] = k;
                mark[j] = k;
            }
        }
    }
    cons_.assign(n_, 0);
    work_.assign(n_, 0.0);
    stack_.assign(n_, 0);
    visit_.assign(n_, 0);
    stamp_ = 0;
    ok_ = n_ > 0;
}

void IncrementalCholesky::setConstrained(std::vector<char> constrained)
{
    cons_ = std::move(constrained);
    if ((int)cons_.size() != n_) cons_.assign(n_, 0);
}

int IncrementalCholesky::slot(int col, int row) const
{
    const auto b = li_.begin() + lp_[col], e = li_.begin() + lp_[col + 1];
    return (int)(std::lower_bound(b, e, row) - li_.begin());
}

void IncrementalCholesky::column(const SymCsc& A, int k)
{
    const int stamp = ++stamp_;
    visit_[k] = stamp;
    int top = n_;
    // scatter A^B(:, k) above the diagonal and collect the row-k pattern
    for (int q = A.colptr[k]; q < A.colptr[k + 1] && A.rows[q] < k; ++q) {
        const int i = A.rows[q];
        work_[i] += cons_[i] ? 0.0 : A.vals[q];
        int len = 0;
        for (int j = i; visit_[j] != stamp; j = parent_[j]) {
            stack_[len++] = j;
            visit_[j] = stamp;
        }
        while (len > 0) stack_[--top] = stack_[--len];
    }
    if (cons_[k]) {  // detached: L(k, :) = 0, D(k) = 1
        d_[k] = 1.0;
        for (int p = top; p < n_; ++p) {
            const int j = stack_[p];
            lx_[slot(j, k)] = 0.0;
            work_[j] = 0.0;
        }
        return;
    }
    double dk = A.at(k, k);
    for (int p = top; p < n_; ++p) {
        const int j = stack_[p];
        const double y = work_[j];
        work_[j] = 0.0;
        const int s = slot(j, k);
        for (int q = lp_[j]; q < s; ++q) work_[li_[q]] -= lx_[q] * y;
        const double l = d_[j] != 0.0 ? y / d_[j] : 0.0;
        dk -= l * y;
        lx_[s] = l;
    }
    d_[k] = dk;
}

void IncrementalCholesky::factorizeFull(const SymCsc& A)
{
    if (!ok_) return;
    std::fill(lx_.begin(), lx_.end(), 0.0);
    std::fill(work_.begin(), work_.end(), 0.0);
    for (int k = 0; k < n_; ++k) column(A, k);
}

void IncrementalCholesky::updateColumns(const SymCsc& A, const std::vector<int>& changed)
{
    if (!ok_ || changed.empty()) return;
    // union of the tree paths from the changed columns to their roots
    const int stamp = ++stamp_;
    std::vector<int> cols;
    for (int c : changed)
        for (int j = c; j != -1 && visit_[j] != stamp; j = parent_[j]) {
            visit_[j] = stamp;
            cols.push_back(j);
        }
    std::sort(cols.begin(), cols.end());
    for (int k : cols) column(A, k);
}

void IncrementalCholesky::solveInPlace(std::vector<double>& b) const
{
    for (int k = 0; k < n_; ++k) {  // L z = b
        const double bk = b[k];
        for (int p = lp_[k]; p < lp_[k + 1]; ++p) b[li_[p]] -= lx_[p] * bk;
    }
    for (int k = 0; k < n_; ++k) b[k] /= d_[k];  // D y = z
    for (int k = n_ - 1; k >= 0; --k) {          // L^T x = y
        double x = b[k];
        for (int p = lp_[k]; p < lp_[k + 1]; ++p) x -= lx_[p] * b[li_[p]];
        b[k] = x;
    }
}

}  // namespace pbfdrop
