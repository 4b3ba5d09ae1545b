// fluid/Particle.h — per-particle state as the caller sees it.
//
// Drop-in for the reference's include/fluid/Particle.h:8-12: three vec3
// each followed by a pad word (48 bytes).  predPos is carried through
// unchanged; the solver's prediction lives on the GPU.
#ifndef PBF_B200_FLUID_PARTICLE_H
#define PBF_B200_FLUID_PARTICLE_H

#include "core/Types.h"

struct Particle {
    PVec3 pos;
    F32 _pad0 = 0.f;
    PVec3 predPos;
    F32 _pad1 = 0.f;
    PVec3 vel;
    F32 _pad2 = 0.f;
};

static_assert(sizeof(Particle) == 48, "Particle must stay 48 bytes");

#endif
