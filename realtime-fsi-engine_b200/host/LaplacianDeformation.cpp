// LaplacianDeformation.cpp — see include/deformation/LaplacianDeformation.h.
//
// Restates src/deformation/LaplacianDeformation.cpp of the reference:
//   cotangent weights  w_e = max(0.5 * sum over the edge's faces of cot(opposite angle), 1e-4)
//                      (cot = cos / sin, a face skipped when sin <= 1e-6)  (:69-114)
//   Laplacian          L_ii = 1, L_ij = -w_ij / sum_j w_ij                 (:116-160)
//   delta              L * V at rest                                        (:162-183)
//   local patch        k-ring of the handles minus anchors; Lii, Li_notI, rest delta;
//                      (Lii^T Lii + I_handles) x = Lii^T (delta - Li_notI x_notI) + targets (:215-417)
//   soft global        [L; rows e_anchor, e_control, e_handles] least squares (:497-616)
//   incremental        A = L^T L + 1e-8 I, b = L^T delta, hard constraints on the
//                      detached factor, RHS corrected by A_IC c_C              (:25-66, :430-497, :620-675)
// Vertex neighbourhoods are kept in ascending index order (the reference walks
// OpenMesh one-rings, which only reorders floating-point sums).
#include "../../include/deformation/LaplacianDeformation.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <set>

namespace pbfdrop {

namespace {
inline Vec3 sub(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline double dot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Vec3 cross(const Vec3& a, const Vec3& b)
{
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double len(const Vec3& a) { return std::sqrt(dot(a, a)); }

// y = M x for rows given as (col, value) lists
std::vector<double> rows_times(const std::vector<std::vector<std::pair<int, double>>>& M, const std::vector<double>& x)
{
    std::vector<double> y(M.size(), 0.0);
    for (size_t i = 0; i < M.size(); ++i)
        for (const auto& e : M[i]) y[i] += e.second * x[e.first];
    return y;
}

// M^T M for rows of an (m x n) matrix, plus `diag` added on given indices.
SymCsc normal_matrix(const std::vector<std::vector<std::pair<int, double>>>& M, int n,
                     const std::vector<int>& diagIdx, double diagVal, double reg)
{
    std::vector<std::map<int, double>> cols(n);
    for (const auto& row : M)
        for (const auto& a : row)
            for (const auto& b : row) cols[b.first][a.first] += a.second * b.second;
    for (int k : diagIdx) cols[k][k] += diagVal;
    if (reg != 0.0)
        for (int k = 0; k < n; ++k) cols[k][k] += reg;
    SymCsc A;
    A.n = n;
    A.colptr.assign(n + 1, 0);
    for (int j = 0; j < n; ++j) {
        for (const auto& kv : cols[j]) {
            if (kv.second == 0.0 && kv.first != j) continue;
            A.rows.push_back(kv.first);
            A.vals.push_back(kv.second);
        }
        A.colptr[j + 1] = (int)A.rows.size();
    }
    return A;
}

// Reverse Cuthill-McKee order of the graph of A (perm[new] = old).
std::vector<int> rcm(const SymCsc& A)
{
    const int n = A.n;
    std::vector<int> deg(n), perm;
    perm.reserve(n);
    for (int j = 0; j < n; ++j) deg[j] = A.colptr[j + 1] - A.colptr[j];
    std::vector<char> seen(n, 0);
    std::vector<int> byDeg(n);
    for (int i = 0; i < n; ++i) byDeg[i] = i;
    std::stable_sort(byDeg.begin(), byDeg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    for (int s : byDeg) {
        if (seen[s]) continue;
        std::deque<int> q{s};
        seen[s] = 1;
        while (!q.empty()) {
            const int v = q.front();
            q.pop_front();
            perm.push_back(v);
            std::vector<int> nb;
            for (int p = A.colptr[v]; p < A.colptr[v + 1]; ++p)
                if (!seen[A.rows[p]]) {
                    seen[A.rows[p]] = 1;
                    nb.push_back(A.rows[p]);
                }
            std::stable_sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            for (int u : nb) q.push_back(u);
        }
    }
    std::reverse(perm.begin(), perm.end());
    return perm;
}

SymCsc permuted(const SymCsc& A, const std::vector<int>& inv)
{
    std::vector<int> r, c;
    std::vector<double> v;
    for (int j = 0; j < A.n; ++j)
        for (int p = A.colptr[j]; p < A.colptr[j + 1]; ++p) {
            r.push_back(inv[A.rows[p]]);
            c.push_back(inv[j]);
            v.push_back(A.vals[p]);
        }
    return sym_from_triplets(A.n, r, c, v);
}
}  // namespace

LaplacianDeformation::LaplacianDeformation(DeformMesh& mesh) : mesh_(mesh) {}

void LaplacianDeformation::initialize()
{
    buildLaplacian();
    local_ = Patch{};
    softReady_ = false;
    incReady_ = false;
    A_ = SymCsc{};
    prevConstrained_.clear();
}

void LaplacianDeformation::buildLaplacian()
{
    n_ = (int)mesh_.points.size();
    // edges with the opposite vertex of each adjacent face
    std::map<std::pair<int, int>, std::vector<int>> opp;
    for (const auto& f : mesh_.faces)
        for (int e = 0; e < 3; ++e) {
            const int a = f[e], b = f[(e + 1) % 3], c = f[(e + 2) % 3];
            opp[{std::min(a, b), std::max(a, b)}].push_back(c);
        }
    std::vector<std::map<int, double>> w(n_);
    for (const auto& kv : opp) {
        const int a = kv.first.first, b = kv.first.second;
        double cot = 0.0;
        for (int c : kv.second) {
            const Vec3 s = sub(mesh_.points[a], mesh_.points[c]), e = sub(mesh_.points[b], mesh_.points[c]);
            const double cs = dot(s, e), sn = len(cross(s, e));
            if (sn > 1e-6) cot += cs / sn;
        }
        const double wt = std::max(0.5 * cot, 1e-4);
        w[a][b] = wt;
        w[b][a] = wt;
    }
    L_.assign(n_, {});
    ring_.assign(n_, {});
    for (int i = 0; i < n_; ++i) {
        double sum = 0.0;
        for (const auto& kv : w[i]) sum += kv.second;
        std::map<int, double> row;
        row[i] += 1.0;
        for (const auto& kv : w[i]) {
            row[kv.first] += -kv.second / sum;
            ring_[i].push_back(kv.first);
        }
        for (const auto& kv : row) L_[i].push_back(kv);
    }
    std::vector<double> X(n_), Y(n_), Z(n_);
    for (int i = 0; i < n_; ++i) {
        X[i] = mesh_.points[i][0];
        Y[i] = mesh_.points[i][1];
        Z[i] = mesh_.points[i][2];
    }
    dx_ = rows_times(L_, X);
    dy_ = rows_times(L_, Y);
    dz_ = rows_times(L_, Z);
}

void LaplacianDeformation::addAnchor(int v)
{
    if (v < 0 || v >= n_ || std::find(anchors_.begin(), anchors_.end(), v) != anchors_.end()) return;
    anchors_.push_back(v);
    anchorPos_.push_back(mesh_.points[v]);
}

void LaplacianDeformation::setControlPoint(int v, const Vec3& t)
{
    controlIndex_ = v;
    controlTarget_ = t;
}

void LaplacianDeformation::setControlPoints(const std::vector<int>& idx, const std::vector<Vec3>& t)
{
    controlIndices_ = idx;
    controlTargets_ = t;
}

void LaplacianDeformation::clearControlPoints()
{
    controlIndices_.clear();
    controlTargets_.clear();
}

void LaplacianDeformation::clearConstraints()
{
    anchors_.clear();
    anchorPos_.clear();
    controlIndex_ = -1;
    controlTarget_ = {0, 0, 0};
    clearControlPoints();
}

void LaplacianDeformation::clearControlPoint()
{
    controlIndex_ = -1;
    controlTarget_ = {0, 0, 0};
}

Vec3 LaplacianDeformation::targetOf(int v) const
{
    Vec3 t{0, 0, 0};
    for (size_t i = 0; i < controlIndices_.size(); ++i)
        if (controlIndices_[i] == v) {
            t = controlTargets_[i];
            break;
        }
    if (controlIndex_ == v) t = controlTarget_;
    return t;
}

// ---- local patch --------------------------------------------------------------------------
void LaplacianDeformation::precomputeLocal()
{
    local_.ready = false;
    std::vector<int> seeds = controlIndices_;
    if (controlIndex_ >= 0) seeds.push_back(controlIndex_);
    if (seeds.empty()) return;
    std::set<int> anchorSet(anchors_.begin(), anchors_.end());
    // k-ring by breadth-first hops over the one-rings
    std::vector<char> inRing(n_, 0);
    std::vector<int> frontier;
    for (int s : seeds)
        if (s >= 0 && s < n_ && !inRing[s]) {
            inRing[s] = 1;
            frontier.push_back(s);
        }
    for (int hop = 0; hop < kring_; ++hop) {
        std::vector<int> next;
        for (int v : frontier)
            for (int j : ring_[v])
                if (!inRing[j]) {
                    inRing[j] = 1;
                    next.push_back(j);
                }
        frontier.swap(next);
    }
    Patch& P = local_;
    P.interior.clear();
    P.outer.clear();
    P.g2l.assign(n_, -1);
    std::vector<int> o2l(n_, -1);
    for (int v = 0; v < n_; ++v) {
        if (!inRing[v]) continue;
        if (anchorSet.count(v)) {
            o2l[v] = (int)P.outer.size();
            P.outer.push_back(v);
        } else {
            P.g2l[v] = (int)P.interior.size();
            P.interior.push_back(v);
        }
    }
    const int ni = (int)P.interior.size();
    if (ni == 0) return;
    P.Lii.assign(ni, {});
    P.Lio.assign(ni, {});
    for (int li = 0; li < ni; ++li) {
        for (const auto& e : L_[P.interior[li]]) {
            const int g = e.first;
            if (P.g2l[g] >= 0) {
                P.Lii[li].push_back({P.g2l[g], e.second});
            } else {
                if (o2l[g] < 0) {
                    o2l[g] = (int)P.outer.size();
                    P.outer.push_back(g);
                }
                P.Lio[li].push_back({o2l[g], e.second});
            }
        }
    }
    P.rdx.resize(ni);
    P.rdy.resize(ni);
    P.rdz.resize(ni);
    for (int li = 0; li < ni; ++li) {
        P.rdx[li] = dx_[P.interior[li]];
        P.rdy[li] = dy_[P.interior[li]];
        P.rdz[li] = dz_[P.interior[li]];
    }
    P.handleLocal.clear();
    P.handleGlobal.clear();
    for (int h : controlIndices_)
        if (h >= 0 && h < n_ && P.g2l[h] >= 0) {
            P.handleLocal.push_back(P.g2l[h]);
            P.handleGlobal.push_back(h);
        }
    if (controlIndex_ >= 0 && controlIndex_ < n_ && P.g2l[controlIndex_] >= 0) {
        P.handleLocal.push_back(P.g2l[controlIndex_]);
        P.handleGlobal.push_back(controlIndex_);
    }
    if (P.handleLocal.empty()) return;
    P.AtA = normal_matrix(P.Lii, ni, P.handleLocal, 1.0, 0.0);
    P.factor.analyze(P.AtA);
    P.factor.setConstrained(std::vector<char>(ni, 0));
    P.factor.factorizeFull(P.AtA);
    P.ready = P.factor.ok();
}

void LaplacianDeformation::solveLocal()
{
    Patch& P = local_;
    if (!P.ready) return;
    const int ni = (int)P.interior.size();
    const int no = (int)P.outer.size();
    std::vector<double> ox(no), oy(no), oz(no);
    for (int i = 0; i < no; ++i) {
        ox[i] = mesh_.points[P.outer[i]][0];
        oy[i] = mesh_.points[P.outer[i]][1];
        oz[i] = mesh_.points[P.outer[i]][2];
    }
    const std::vector<double> cx = rows_times(P.Lio, ox), cy = rows_times(P.Lio, oy), cz = rows_times(P.Lio, oz);
    std::vector<double> bx(ni), by(ni), bz(ni);
    for (int i = 0; i < ni; ++i) {
        bx[i] = P.rdx[i] - cx[i];
        by[i] = P.rdy[i] - cy[i];
        bz[i] = P.rdz[i] - cz[i];
    }
    // rhs = Lii^T b
    std::vector<double> rx(ni, 0.0), ry(ni, 0.0), rz(ni, 0.0);
    for (int i = 0; i < ni; ++i)
        for (const auto& e : P.Lii[i]) {
            rx[e.first] += e.second * bx[i];
            ry[e.first] += e.second * by[i];
            rz[e.first] += e.second * bz[i];
        }
    for (size_t c = 0; c < P.handleLocal.size(); ++c) {
        const Vec3 t = targetOf(P.handleGlobal[c]);
        rx[P.handleLocal[c]] += t[0];
        ry[P.handleLocal[c]] += t[1];
        rz[P.handleLocal[c]] += t[2];
    }
    P.factor.solveInPlace(rx);
    P.factor.solveInPlace(ry);
    P.factor.solveInPlace(rz);
    for (int i = 0; i < ni; ++i) mesh_.points[P.interior[i]] = {rx[i], ry[i], rz[i]};
}

// ---- incremental -------------------------------------------------------------------------
void LaplacianDeformation::buildNormalSystem()
{
    A_ = normal_matrix(L_, n_, {}, 0.0, 1e-8);
    // b = L^T delta
    bx_.assign(n_, 0.0);
    by_.assign(n_, 0.0);
    bz_.assign(n_, 0.0);
    for (int i = 0; i < n_; ++i)
        for (const auto& e : L_[i]) {
            bx_[e.first] += e.second * dx_[i];
            by_[e.first] += e.second * dy_[i];
            bz_[e.first] += e.second * dz_[i];
        }
    perm_ = rcm(A_);
    invPerm_.assign(n_, 0);
    for (int i = 0; i < n_; ++i) invPerm_[perm_[i]] = i;
    Aperm_ = permuted(A_, invPerm_);
    incReady_ = false;
    prevConstrained_.clear();
}

std::vector<int> LaplacianDeformation::constrainedSorted() const
{
    std::vector<int> c = anchors_;
    if (controlIndex_ >= 0) c.push_back(controlIndex_);
    c.insert(c.end(), controlIndices_.begin(), controlIndices_.end());
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    return c;
}

void LaplacianDeformation::targets(std::vector<double>& tx, std::vector<double>& ty, std::vector<double>& tz) const
{
    tx.assign(n_, 0.0);
    ty.assign(n_, 0.0);
    tz.assign(n_, 0.0);
    auto set = [&](int v, const Vec3& p) {
        tx[v] = p[0];
        ty[v] = p[1];
        tz[v] = p[2];
    };
    for (size_t i = 0; i < anchors_.size(); ++i) set(anchors_[i], anchorPos_[i]);
    if (controlIndex_ >= 0) set(controlIndex_, controlTarget_);
    for (size_t i = 0; i < controlIndices_.size(); ++i) set(controlIndices_[i], controlTargets_[i]);
}

void LaplacianDeformation::solveAxisIncremental(const std::vector<double>& b, const std::vector<double>& t,
                                                std::vector<double>& x) const
{
    // free rows: b - A_IC t_C; constrained rows: their targets
    std::vector<double> rhs = b;
    for (int k = 0; k < n_; ++k) {
        if (!mask_[k]) continue;
        for (int p = A_.colptr[k]; p < A_.colptr[k + 1]; ++p) rhs[A_.rows[p]] -= A_.vals[p] * t[k];
    }
    for (int k = 0; k < n_; ++k)
        if (mask_[k]) rhs[k] = t[k];
    std::vector<double> rp(n_);
    for (int i = 0; i < n_; ++i) rp[i] = rhs[perm_[i]];
    inc_.solveInPlace(rp);
    x.assign(n_, 0.0);
    for (int i = 0; i < n_; ++i) x[perm_[i]] = rp[i];
}

double LaplacianDeformation::verifyIncremental()
{
    if (!useIncremental_ || !incReady_) return -1.0;
    // dense LDL^T of the detached system
    std::vector<double> M((size_t)n_ * n_, 0.0);
    for (int j = 0; j < n_; ++j)
        for (int p = A_.colptr[j]; p < A_.colptr[j + 1]; ++p) {
            const int i = A_.rows[p];
            if (mask_[i] || mask_[j]) {
                if (i == j) M[(size_t)i * n_ + j] = 1.0;
            } else {
                M[(size_t)i * n_ + j] = A_.vals[p];
            }
        }
    std::vector<double> tx, ty, tz;
    targets(tx, ty, tz);
    std::vector<double> rhs = bx_;
    for (int k = 0; k < n_; ++k) {
        if (!mask_[k]) continue;
        for (int p = A_.colptr[k]; p < A_.colptr[k + 1]; ++p) rhs[A_.rows[p]] -= A_.vals[p] * tx[k];
    }
    for (int k = 0; k < n_; ++k)
        if (mask_[k]) rhs[k] = tx[k];
    // Gaussian elimination on the symmetric positive-definite dense matrix
    std::vector<double> y = rhs;
    for (int k = 0; k < n_; ++k) {
        const double piv = M[(size_t)k * n_ + k];
        for (int i = k + 1; i < n_; ++i) {
            const double f = M[(size_t)i * n_ + k] / piv;
            if (f == 0.0) continue;
            for (int j = k; j < n_; ++j) M[(size_t)i * n_ + j] -= f * M[(size_t)k * n_ + j];
            y[i] -= f * y[k];
        }
    }
    for (int k = n_ - 1; k >= 0; --k) {
        double s = y[k];
        for (int j = k + 1; j < n_; ++j) s -= M[(size_t)k * n_ + j] * y[j];
        y[k] = s / M[(size_t)k * n_ + k];
    }
    std::vector<double> xi;
    solveAxisIncremental(bx_, tx, xi);
    double m = 0.0;
    for (int i = 0; i < n_; ++i) m = std::max(m, std::fabs(xi[i] - y[i]));
    return m;
}

// ---- dispatch ------------------------------------------------------------------------------
void LaplacianDeformation::precomputeSystem()
{
    if (useLocal_) {
        precomputeLocal();
        return;
    }
    if (useIncremental_) {
        std::vector<int> cur = constrainedSorted();
        if (cur.empty()) return;
        if (!incReady_ && A_.n != n_) buildNormalSystem();
        if (!incReady_) {
            inc_.analyze(Aperm_);
            incReady_ = true;
        }
        mask_.assign(n_, 0);
        std::vector<char> mp(n_, 0);
        for (int v : cur) {
            mask_[v] = 1;
            mp[invPerm_[v]] = 1;
        }
        inc_.setConstrained(mp);
        if (prevConstrained_.empty()) {
            inc_.factorizeFull(Aperm_);
        } else {
            // changed columns: the symmetric difference of the sets and every
            // column that shares a nonzero with them
            std::vector<int> diff;
            std::set_symmetric_difference(cur.begin(), cur.end(), prevConstrained_.begin(), prevConstrained_.end(),
                                          std::back_inserter(diff));
            std::vector<char> seen(n_, 0);
            std::vector<int> changed;
            for (int v : diff)
                for (int p = A_.colptr[v]; p < A_.colptr[v + 1]; ++p) {
                    const int q = invPerm_[A_.rows[p]];
                    if (!seen[q]) {
                        seen[q] = 1;
                        changed.push_back(q);
                    }
                }
            inc_.updateColumns(Aperm_, changed);
        }
        prevConstrained_ = std::move(cur);
        return;
    }
    // soft global: rows L, then one unit row per constraint
    std::vector<std::vector<std::pair<int, double>>> rows = L_;
    for (int a : anchors_) rows.push_back({{a, 1.0}});
    if (controlIndex_ >= 0) rows.push_back({{controlIndex_, 1.0}});
    for (int h : controlIndices_) rows.push_back({{h, 1.0}});
    if (rows.size() == L_.size()) return;  // needs at least one constraint
    soft_ = normal_matrix(rows, n_, {}, 0.0, 0.0);
    softFactor_.analyze(soft_);
    softFactor_.setConstrained(std::vector<char>(n_, 0));
    softFactor_.factorizeFull(soft_);
    softReady_ = softFactor_.ok();
}

void LaplacianDeformation::solve()
{
    if (useLocal_) {
        solveLocal();
        return;
    }
    if (useIncremental_) {
        if (!incReady_) return;
        std::vector<double> tx, ty, tz, x, y, z;
        targets(tx, ty, tz);
        solveAxisIncremental(bx_, tx, x);
        solveAxisIncremental(by_, ty, y);
        solveAxisIncremental(bz_, tz, z);
        for (int i = 0; i < n_; ++i) mesh_.points[i] = {x[i], y[i], z[i]};
        return;
    }
    if (!softReady_) return;
    // A^T b: L^T delta plus the constraint targets on their columns
    std::vector<double> rx(n_, 0.0), ry(n_, 0.0), rz(n_, 0.0);
    for (int i = 0; i < n_; ++i)
        for (const auto& e : L_[i]) {
            rx[e.first] += e.second * dx_[i];
            ry[e.first] += e.second * dy_[i];
            rz[e.first] += e.second * dz_[i];
        }
    auto add = [&](int v, const Vec3& p) {
        rx[v] += p[0];
        ry[v] += p[1];
        rz[v] += p[2];
    };
    for (size_t i = 0; i < anchors_.size(); ++i) add(anchors_[i], anchorPos_[i]);
    if (controlIndex_ >= 0) add(controlIndex_, controlTarget_);
    for (size_t i = 0; i < controlIndices_.size(); ++i) add(controlIndices_[i], controlTargets_[i]);
    softFactor_.solveInPlace(rx);
    softFactor_.solveInPlace(ry);
    softFactor_.solveInPlace(rz);
    for (int i = 0; i < n_; ++i) mesh_.points[i] = {rx[i], ry[i], rz[i]};
}

// ---- per-frame handle logic (src/main.cpp:870-944) ------------------------------------------
bool LaplacianDeformation::deformStep(const std::vector<Vec3>& forces, float dt, const DeformParams& prm,
                                      const std::vector<Vec3>& rest, std::vector<int>& lastHandles,
                                      int* handleCount, bool* refactored)
{
    if (handleCount) *handleCount = 0;
    if (refactored) *refactored = false;
    if ((int)rest.size() != n_ || (int)forces.size() != n_) return false;
    std::set<int> anchorSet(anchors_.begin(), anchors_.end());
    std::vector<int> handles;
    std::vector<Vec3> tg;
    for (int i = 0; i < n_; ++i) {
        if (anchorSet.count(i)) continue;
        const Vec3 cur = mesh_.points[i];
        const Vec3& r = rest[i];
        // forces and the per-frame displacement are single precision, as the
        // reference's PVec3 vertex forces (main.cpp:886,903-905)
        const float fx = (float)forces[i][0], fy = (float)forces[i][1], fz = (float)forces[i][2];
        const float fmag = std::sqrt(fx * fx + fy * fy + fz * fz);
        const bool wasH = std::binary_search(lastHandles.begin(), lastHandles.end(), i);
        const bool pushed = (fmag >= prm.controlThreshold) || (wasH && fmag >= prm.controlThresholdLow);
        const double offset = len(sub(cur, r));
        const bool relaxing = prm.restoreEnabled && wasH && offset > 1e-3;
        if (!pushed && !relaxing) continue;
        Vec3 t = cur;
        if (pushed) {
            const float g = prm.stiffness * dt;
            float ex = fx * g, ey = fy * g, ez = fz * g;
            const float dm = std::sqrt(ex * ex + ey * ey + ez * ez);
            if (dm > prm.maxDisplacement && dm > 1e-12f) {
                const float s = prm.maxDisplacement / dm;
                ex *= s;
                ey *= s;
                ez *= s;
            }
            t = {t[0] + ex, t[1] + ey, t[2] + ez};
        }
        if (prm.restoreEnabled) {
            const double k = (double)prm.restoreStrength;
            t = {t[0] + k * (r[0] - t[0]), t[1] + k * (r[1] - t[1]), t[2] + k * (r[2] - t[2])};
        }
        const Vec3 fr = sub(t, r);
        const double off = len(fr);
        if (off > prm.maxTotalDisp) {
            const double s = prm.maxTotalDisp / off;
            t = {r[0] + fr[0] * s, r[1] + fr[1] * s, r[2] + fr[2] * s};
        }
        handles.push_back(i);
        tg.push_back(t);
    }
    if (handleCount) *handleCount = (int)handles.size();
    const bool changed = handles != lastHandles;
    setControlPoints(handles, tg);
    if (changed) {
        precomputeSystem();
        if (refactored) *refactored = true;
    }
    lastHandles = handles;
    if (!handles.empty() || changed) {
        solve();
        return true;
    }
    return false;
}

}  // namespace pbfdrop
