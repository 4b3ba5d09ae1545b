// LaplacianDeformation.h — cotangent-Laplacian surface deformation driven by
// per-vertex handle targets, the host consumer of the fluid's vertex forces.
//
// Replaces the reference's LaplacianDeformation (include/deformation/
// LaplacianDeformation.h:11-157, src/deformation/LaplacianDeformation.cpp)
// with the same public members and the same three solve paths, without
// Eigen, CHOLMOD or OpenMesh (none of which is available to this build):
//   * local patch (default): only the k-ring of the handles is solved, with
//     the vertices around it held where they are;
//   * soft global: least squares of [L; constraint rows] over all vertices;
//   * incremental: hard constraints on the persistent factor of L^T L
//     (IncrementalCholesky), updated along tree paths when the handle set
//     changes.
// The mesh is a triangle list; positions are FP64.  deformStep() restates the
// application's per-frame handle logic (src/main.cpp:870-944).
#pragma once

#include <array>
#include <vector>

#include "deformation/IncrementalCholesky.h"

namespace pbfdrop {

using Vec3 = std::array<double, 3>;

struct DeformMesh {
    std::vector<Vec3> points;
    std::vector<std::array<int, 3>> faces;
};

// Per-frame handle policy (the reference's SceneDeform, include/core/Scene.h:17-27,
// and main.cpp's g_* tuning globals).
struct DeformParams {
    float stiffness = 1.0f;            // force -> displacement gain
    float maxDisplacement = 0.02f;     // per-frame displacement clamp
    float maxTotalDisp = 0.40f;        // clamp on |deformed - rest|
    bool restoreEnabled = true;        // spring back toward the rest shape
    float restoreStrength = 0.05f;     // fraction of the offset removed per frame
    float controlThreshold = 0.50f;    // |force| to enter the handle set
    float controlThresholdLow = 0.30f; // |force| to leave it (hysteresis)
};

class LaplacianDeformation {
public:
    explicit LaplacianDeformation(DeformMesh& mesh);

    void initialize();

    void addAnchor(int vertexIndex);
    void setControlPoint(int vertexIndex, const Vec3& targetPosition);
    void setControlPoints(const std::vector<int>& indices, const std::vector<Vec3>& targets);
    void clearControlPoints();
    const std::vector<int>& getControlIndices() const { return controlIndices_; }
    void clearConstraints();
    void clearControlPoint();

    void precomputeSystem();
    void solve();

    void setUseLocal(bool on) { useLocal_ = on; }
    bool isUsingLocal() const { return useLocal_; }
    void setLocalKRing(int k) { kring_ = k; }
    int getLocalPatchSize() const { return local_.ready ? (int)local_.interior.size() : 0; }
    void setUseIncremental(bool on) { useIncremental_ = on; }
    bool isUsingIncremental() const { return useIncremental_; }
    // max |x_incremental - x_dense| of the x axis against a dense LDL^T of the
    // same detached system; -1 when the incremental path is not ready.
    double verifyIncremental();

    const std::vector<int>& getAnchorIndices() const { return anchors_; }
    const std::vector<Vec3>& getAnchorPositions() const { return anchorPos_; }
    int getControlIndex() const { return controlIndex_; }
    Vec3 getControlTarget() const { return controlTarget_; }
    const DeformMesh& getMesh() const { return mesh_; }
    const SymCsc& laplacianNormal() const { return A_; }

    // One frame of fluid-driven deformation (src/main.cpp:870-944): forms the
    // handle set from the per-vertex forces (hysteresis, per-frame and total
    // clamps, elastic restore), refactors only when the set changes, solves.
    // Returns true when the mesh moved.  `rest` = rest positions; `lastHandles`
    // carries the previous frame's sorted handle set.
    bool deformStep(const std::vector<Vec3>& forces, float dt, const DeformParams& prm,
                    const std::vector<Vec3>& rest, std::vector<int>& lastHandles, int* handleCount,
                    bool* refactored);

private:
    DeformMesh& mesh_;
    int n_ = 0;
    std::vector<std::vector<std::pair<int, double>>> L_;  // rows of the Laplacian (sorted cols)
    std::vector<std::vector<int>> ring_;                   // one-ring neighbours (sorted)
    std::vector<double> dx_, dy_, dz_;                     // differential coordinates at rest

    std::vector<int> anchors_;
    std::vector<Vec3> anchorPos_;
    int controlIndex_ = -1;
    Vec3 controlTarget_{0, 0, 0};
    std::vector<int> controlIndices_;
    std::vector<Vec3> controlTargets_;

    bool useLocal_ = true;
    int kring_ = 3;
    bool useIncremental_ = false;

    struct Patch {
        bool ready = false;
        std::vector<int> interior, outer;
        std::vector<int> g2l;                                  // global -> interior index or -1
        std::vector<std::vector<std::pair<int, double>>> Lio;  // interior row -> outer entries
        std::vector<std::vector<std::pair<int, double>>> Lii;  // interior row -> interior entries
        std::vector<double> rdx, rdy, rdz;
        std::vector<int> handleLocal, handleGlobal;
        SymCsc AtA;
        IncrementalCholesky factor;
    } local_;

    // soft global path
    SymCsc soft_;
    IncrementalCholesky softFactor_;
    bool softReady_ = false;

    // incremental path (factor in reverse Cuthill-McKee order)
    SymCsc A_, Aperm_;
    std::vector<double> bx_, by_, bz_;
    std::vector<int> perm_, invPerm_;
    IncrementalCholesky inc_;
    bool incReady_ = false;
    std::vector<char> mask_;
    std::vector<int> prevConstrained_;

    void buildLaplacian();
    void buildNormalSystem();
    std::vector<int> constrainedSorted() const;
    void targets(std::vector<double>& tx, std::vector<double>& ty, std::vector<double>& tz) const;
    void solveAxisIncremental(const std::vector<double>& b, const std::vector<double>& t,
                              std::vector<double>& x) const;
    void precomputeLocal();
    void solveLocal();
    Vec3 targetOf(int v) const;
};

}  // namespace pbfdrop
