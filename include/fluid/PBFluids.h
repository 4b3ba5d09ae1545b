// fluid/PBFluids.h — position-based fluids solver, B200 engine.
//
// Drop-in for the reference's include/fluid/PBFluids.h:88-163: the same public
// members with the same meaning, backed by the C ABI of pbf_b200.h (one CUDA
// stream and one set of device buffers per instance).  Empty or unready states
// stay silent no-ops as in the reference; device errors are reported on stderr
// with pbf_last_error() (the reference prints shader errors the same way).
#ifndef PBF_B200_FLUID_PBFLUIDS_H
#define PBF_B200_FLUID_PBFLUIDS_H

#include <vector>

#include "core/Types.h"
#include "core/config.h"
#include "fluid/Particle.h"
#include "fluid/SDFBoundary.h"

struct pbf_handle;

// FluidConfigUBO (include/fluid/PBFluids.h:21-61 of the reference)
struct FluidConfigUBO {
    PVec4 boundsMin;
    PVec4 boundsMax;
    PVec4 gravity_dt;
    F32 h, rho0, eps, wq;
    F32 kCorr, nCorr, viscosity, boundDamping;
    U32 hashSize, particleCount, enableSCorr, enableViscosity;
    F32 cohesionStrength, interactionRadius, interactionStrength, w0_self;
    U32 hashMask;
    F32 poly6Coeff, spikyCoeff, invRho0;
    U32 minLOD, maxLOD;
    F32 lodMaxDist;
    U32 enableAPBF;
};

// ContactCandidate (include/fluid/PBFluids.h:67-70 of the reference)
struct ContactCandidate {
    PVec4 pos;
    PVec4 vel;
};

class PBFluids {
public:
    PBFluids();
    explicit PBFluids(const FluidConfig& p, int device = 0);
    ~PBFluids();
    PBFluids(const PBFluids&) = delete;
    PBFluids& operator=(const PBFluids&) = delete;

    void setParams(const FluidConfig& p);
    const FluidConfig& params() const { return _params; }
    void setCameraPos(const PVec3& pos);

    void setParticles(const std::vector<Particle>& particles);
    std::vector<Particle>& particles() { return _particles; }
    const std::vector<Particle>& particles() const { return _particles; }

    void setCollisionPadding(F32 p);
    F32 _collisionPadding = 0.0f;
    void setBounds(const PVec3& minBound, const PVec3& maxBound, F32 damping = 0.0f);

    void setSDFBoundary(const SDFBoundary* sdf);
    void setSDFPadding(F32 padding);
    void setSDFContainment(bool inside);

    void setInteraction(bool active, const PVec3& pos);

    void step();

    // Device pointers of the committed state (float4 pos, float4 vel), in
    // place of binding the particle SSBO for the renderer.
    struct DeviceParticles {
        void* pos4 = nullptr;
        void* vel4 = nullptr;
        U32 count = 0;
    };
    DeviceParticles bindParticlesForRendering() const;

    void readbackParticles(std::vector<Particle>& out);
    void filterContactCandidates(float contactBand);
    void readbackContactCandidates(std::vector<ContactCandidate>& out);

    // computeContactForces (src/main.cpp:604-710 of the reference) on the GPU:
    // per-vertex push of the current candidates on the attached mesh SDF.
    int computeContactForces(float band, bool useVelMagnitude, std::vector<PVec3>& vertForces);

    pbf_handle* handle() const { return _h; }

private:
    static void toC(const FluidConfig& p, void* out);
    void report(int rc, const char* what) const;
    pbf_handle* _h = nullptr;
    FluidConfig _params;
    std::vector<Particle> _particles;
    const SDFBoundary* _sdf = nullptr;
    F32 _sdfPadding = 0.0f;
    bool _sdfContainment = false;
};

#endif
