// core/Scene.h — the scene presets the reference's demo boots with.
//
// Drop-in for the reference's include/core/Scene.h:17-306: SceneDeform,
// Scene and getScenes() with the same fields in the same order.  A preset is
// data a caller selects by index: a FluidConfig, the mesh asset and its fit
// size, SDF resolution and padding, obstacle or container, the mesh placement
// and the deformation tuning.  The four presets carry the reference's values.
// The camera fields are kept for source compatibility; nothing here renders.
// The headless set-up that turns a preset into a running scene is
// core/SceneSetup.h.
#ifndef PBF_B200_CORE_SCENE_H
#define PBF_B200_CORE_SCENE_H

#include <vector>

#include "core/Types.h"
#include "core/config.h"

struct SceneDeform {
    float stiffness;            // force -> displacement gain
    float maxDisplacement;      // per-frame displacement clamp
    float maxTotalDisp;         // clamp on |deformed - rest|
    bool restoreEnabled;        // elastic spring-back toward the rest shape
    float restoreStrength;      // fraction of the remaining offset removed per frame
    float controlThreshold;     // |force| to enter the handle set
    float controlThresholdLow;  // |force| to leave it (hysteresis, below the entry threshold)
    int localKRing;             // ring radius of the local solve patch
    float contactRadius;        // surface band counted as fluid contact
};

struct Scene {
    const char* name;
    FluidConfig fluid;
    float camYaw;
    float camPitch;
    float camDist;
    float pointSize;

    const char* meshFile;  // asset file name, e.g. "cube1538.off"
    float meshFitSize;     // the mesh's largest extent is scaled to this
    float sdfCell;         // SDF voxel size
    float sdfPadding;      // particle centres are kept this far off the surface
    bool sdfContainer;     // false: obstacle (fluid pours onto it); true: fluid held inside

    PVec3 meshTranslate;  // offset from the fitted, centred pose
    PVec3 meshRotDeg;     // rotation about the mesh centre, degrees about X, then Y, then Z

    SceneDeform deform;
};

// The four presets: 0 Container Cube, 1 Surface Cube, 2 Surface Bull,
// 3 Surface Hand.
const std::vector<Scene>& getScenes();

#endif
