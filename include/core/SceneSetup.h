// core/SceneSetup.h — headless scene set-up: mesh assets, placement and
// particle spawning.
//
// The reference performs these steps inside its application (src/main.cpp):
// loadOFF (:364-415), fitMeshToDomain (:419-432), the mesh centre chosen by
// loadMeshBoundary (:500-512), the placement of applyMeshTransform
// (:747-770), spawnParticles (:160-188) and the order loadScene /
// confirmAnchorsAndSpawn apply them in (:1192-1243, :959-993).  Here they are
// library functions, so a caller without a window can build the reference's
// scenes and step them.
#ifndef PBF_B200_CORE_SCENESETUP_H
#define PBF_B200_CORE_SCENESETUP_H

#include <array>
#include <string>
#include <vector>

#include "core/Scene.h"
#include "core/Types.h"
#include "core/config.h"
#include "fluid/Particle.h"

class PBFluids;
class SDFBoundary;

// A triangle mesh in double precision (src/main.cpp:216-219).
struct MeshData {
    std::vector<std::array<double, 3>> verts;
    std::vector<std::array<int, 3>> faces;  // triangulated
};

// Reads an OFF file: comment ('#') and blank lines are skipped, the header
// line must contain "OFF" (OFF, NOFF, COFF, ...), the first three numbers of
// each vertex line are its position (normals, colours after them are
// ignored), polygons are fan-triangulated from their first vertex.  Returns
// false (and leaves `out` untouched) when the file cannot be opened, is not
// an OFF file, ends before the counts it declares, or names a vertex index
// outside [0, vertex count) or a polygon of more than 4096 vertices.
bool loadOFF(const std::string& path, MeshData& out);

// Centres the mesh's bounding box on `center` and scales its largest extent
// to `targetSize` (an extent below 1e-9 counts as 1e-9).
void fitMeshToDomain(MeshData& m, const PVec3& center, double targetSize);

// The point loadMeshBoundary fits a scene's mesh around: the middle of the
// walls in x and z, 40 % of the way up in y.
PVec3 meshFitCenter(const FluidConfig& c);

// Rotates the mesh about its bounding-box centre by rotDeg (degrees about
// X, then Y, then Z, composed as Rx * Ry * Rz) and translates it, in single
// precision as the reference does.
void placeMesh(MeshData& m, const PVec3& translate, const PVec3& rotDeg);

// The reference's particle spawner: a lattice from spawnMin stepping by
// `spacing` (z outermost, x innermost, float accumulation, at most
// particleCount particles), or, with spawnRandom, particleCount uniform
// points inside [spawnMin + spacing, spawnMax - spacing] from
// std::mt19937(1337).  predPos = pos, vel = initialVelocity.
std::vector<Particle> spawnParticles(const FluidConfig& c);

// A preset turned into its initial state: the fitted and placed mesh and
// the spawned particles.
struct SceneState {
    MeshData mesh;
    std::vector<Particle> particles;
};

// loadOFF(assetDir/meshFile), fitMeshToDomain(meshFitCenter, meshFitSize),
// placeMesh(meshTranslate, meshRotDeg), spawnParticles.  `meshPath`, when
// not empty, replaces assetDir/meshFile.  Returns false if the mesh cannot be
// loaded.
bool buildSceneState(const Scene& sc, const std::string& assetDir, SceneState& out,
                     const std::string& meshPath = std::string());

// Applies a preset to a solver and an SDF the caller owns, as the
// reference's loadScene + confirmAnchorsAndSpawn do: fluid parameters and
// walls, the SDF built from the placed mesh at sdfCell, padding and
// obstacle/container mode, the spawned particles.  Anchors and the
// deformation solver are left to the caller.  Returns false if the mesh
// cannot be loaded or the SDF cannot be built.
bool loadScene(const Scene& sc, const std::string& assetDir, PBFluids& fluid, SDFBoundary& sdf,
               SceneState* state = nullptr, const std::string& meshPath = std::string());

#endif
