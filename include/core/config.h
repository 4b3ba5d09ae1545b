// core/config.h — FluidConfig, the solver parameter block.
//
// Drop-in for the reference's include/core/config.h:9-63: the same fields,
// types, order and in-class defaults (the field list is the interface; the
// defaults are the reference's tuning).  Also reachable as "core/Config.h",
// the spelling the reference's sources include.
#ifndef PBF_B200_CORE_CONFIG_H
#define PBF_B200_CORE_CONFIG_H

#include "core/Types.h"

struct FluidConfig {
    F32 dt = 1.0f / 60.0f;
    PVec3 gravity = {0.0f, -3.81f, 0.0f};

    F32 h = 0.15f;
    F32 rho0 = 1200.0f;
    U32 solverIterations = 3;
    U32 substepIterations = 2;
    F32 eps = 0.0001f;

    U32 particleCount = 1 << 12;
    PVec3 spawnMin = {2.f, 0.2f, 2.f};
    PVec3 spawnMax = {5.f, 5.f, 5.f};
    bool spawnRandom = false;
    F32 spacing = 0.1f;
    PVec3 initialVelocity = {0.0f, 0.0f, 0.0f};

    PVec3 boundsMin = {0.0f, 0.0f, 0.0f};
    PVec3 boundsMax = {6.0f, 6.0f, 6.0f};
    F32 boundDamping = 0.5f;

    U32 hashSize = 1 << 17;

    bool enableSCorr = true;
    F32 kCorr = 0.001f;
    F32 nCorr = 4.0f;
    F32 deltaQ = 0.3f;

    F32 cohesionStrength = 0.001f;

    bool enableViscosity = true;
    F32 viscosity = 0.1f;

    F32 interactionRadius = 1.5f;
    F32 interactionStrength = 25.0f;

    bool enableVorticity = true;
    F32 vorticityEpsilon = 0.05f;

    bool enableAPBF = false;
    U32 minLOD = 2;
    U32 maxLOD = 7;
    F32 lodMaxDist = 15.0f;
};

struct DeformConfig {
    bool enabled = false;
    F32 stiffness = 1.0f;
};

struct ViewerConfig {
    bool showParticles = true;
    F32 pointRadius = 0.02f;
};

struct Config {
    FluidConfig fluid;
    DeformConfig deform;
    ViewerConfig viewer;
};

#endif
