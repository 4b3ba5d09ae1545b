// PBFluids.cpp / SDFBoundary — the reference's C++ fluid interface
// (include/fluid/PBFluids.h:88-163, include/fluid/SDFBoundary.h:38-167)
// implemented over the C ABI of pbf_b200.h.
#include "fluid/PBFluids.h"

#include <cstdio>
#include <cstring>

#include "pbf_b200.h"
#include "config_c.h"

// ---- SDFBoundary -------------------------------------------------------------------------
SDFBoundary::SDFBoundary() : SDFBoundary(0) {}

SDFBoundary::SDFBoundary(int device)
{
    pbf_fluid_config c;
    pbf_default_config(&c);
    if (pbf_create(&c, device, &_h) != PBF_OK) {
        std::fprintf(stderr, "SDFBoundary: %s\n", pbf_last_error());
        _h = nullptr;
    }
}

SDFBoundary::~SDFBoundary() { pbf_destroy(_h); }

void SDFBoundary::refreshInfo()
{
    int32_t d[3];
    double o[3], cs = 0.0;
    if (pbf_sdf_grid_info(_h, d, o, &cs) != PBF_OK) return;
    for (int a = 0; a < 3; ++a) {
        _dimensions.v[a] = d[a];
        _origin.v[a] = o[a];
    }
    _cellSize = cs;
    _distancesStale = true;
}

void SDFBoundary::buildFromMesh(const std::vector<std::array<double, 3>>& verts,
                                const std::vector<std::array<int, 3>>& faces, double resolution, bool verbose)
{
    if (!_h) return;
    const bool same_faces = _valid && resolution == _buildResolution && faces == _buildFaces &&
                            verts.size() == _buildVerts.size();
    const int rc = same_faces ? pbf_rebuild_mesh(_h, verts[0].data(), (int32_t)verts.size())
                              : pbf_set_sdf_mesh(_h, verts.empty() ? nullptr : verts[0].data(), (int32_t)verts.size(),
                                                 faces.empty() ? nullptr : faces[0].data(), (int32_t)faces.size(),
                                                 resolution);
    if (rc != PBF_OK) {
        std::fprintf(stderr, "SDFBoundary::buildFromMesh: %s\n", pbf_last_error());
        _valid = false;
        return;
    }
    _valid = true;
    _buildVerts = verts;
    if (!same_faces) {
        _buildFaces = faces;
        _buildResolution = resolution;
    }
    refreshInfo();
    if (verbose)
        std::printf("SDF computed: %dx%dx%d (%d voxels, %zu triangles, LBVH)\n", _dimensions.x(), _dimensions.y(),
                    _dimensions.z(), _dimensions.x() * _dimensions.y() * _dimensions.z(), faces.size());
}

void SDFBoundary::refitFromMesh(const std::vector<std::array<double, 3>>& verts)
{
    if (!_h || !_valid) return;
    if (pbf_update_mesh_vertices(_h, verts.empty() ? nullptr : verts[0].data(), (int32_t)verts.size()) != PBF_OK) {
        std::fprintf(stderr, "SDFBoundary::refitFromMesh: %s\n", pbf_last_error());
        return;
    }
    _buildVerts = verts;
    _distancesStale = true;
}

bool SDFBoundary::refitDirty(const std::vector<std::array<double, 3>>& newVerts, double /*bandRadius*/, double moveEps)
{
    bool moved = _buildVerts.size() != newVerts.size();
    const double e2 = moveEps * moveEps;
    for (size_t i = 0; !moved && i < newVerts.size(); ++i) {
        const double dx = newVerts[i][0] - _buildVerts[i][0], dy = newVerts[i][1] - _buildVerts[i][1],
                     dz = newVerts[i][2] - _buildVerts[i][2];
        moved = dx * dx + dy * dy + dz * dz > e2;
    }
    refitFromMesh(newVerts);  // the whole grid is recomputed on the GPU
    return moved;
}

const std::vector<float>& SDFBoundary::distances() const
{
    if (_distancesStale && _valid) {
        _distances.resize((size_t)_dimensions.x() * _dimensions.y() * _dimensions.z());
        if (pbf_read_sdf_grid(_h, _distances.data(), _distances.size()) != PBF_OK)
            std::fprintf(stderr, "SDFBoundary::distances: %s\n", pbf_last_error());
        _distancesStale = false;
    }
    return _distances;
}

SDFBoundary::ClosestSurface SDFBoundary::closestTriangle(const PVec3& p) const
{
    ClosestSurface out;
    if (!_valid) return out;
    const float q[3] = {p.x, p.y, p.z};
    int32_t face = -1;
    float pt[3] = {0, 0, 0};
    if (pbf_closest_triangle(_h, q, 1, &face, pt) == PBF_OK) {
        out.face = face;
        out.point = PVec3{pt[0], pt[1], pt[2]};
    }
    return out;
}

// ---- PBFluids ---------------------------------------------------------------------------------
void pbfhost::fluid_config_to_c(const FluidConfig& p, pbf_fluid_config* out)
{
    pbf_fluid_config& c = *out;
    std::memset(&c, 0, sizeof(c));
    c.dt = p.dt;
    c.gravity[0] = p.gravity.x; c.gravity[1] = p.gravity.y; c.gravity[2] = p.gravity.z;
    c.h = p.h;
    c.rho0 = p.rho0;
    c.solver_iterations = p.solverIterations;
    c.substep_iterations = p.substepIterations;
    c.eps = p.eps;
    c.particle_count = p.particleCount;
    c.spawn_min[0] = p.spawnMin.x; c.spawn_min[1] = p.spawnMin.y; c.spawn_min[2] = p.spawnMin.z;
    c.spawn_max[0] = p.spawnMax.x; c.spawn_max[1] = p.spawnMax.y; c.spawn_max[2] = p.spawnMax.z;
    c.spawn_random = p.spawnRandom ? 1u : 0u;
    c.spacing = p.spacing;
    c.initial_velocity[0] = p.initialVelocity.x; c.initial_velocity[1] = p.initialVelocity.y;
    c.initial_velocity[2] = p.initialVelocity.z;
    c.bounds_min[0] = p.boundsMin.x; c.bounds_min[1] = p.boundsMin.y; c.bounds_min[2] = p.boundsMin.z;
    c.bounds_max[0] = p.boundsMax.x; c.bounds_max[1] = p.boundsMax.y; c.bounds_max[2] = p.boundsMax.z;
    c.bound_damping = p.boundDamping;
    c.hash_size = p.hashSize;
    c.enable_scorr = p.enableSCorr ? 1u : 0u;
    c.k_corr = p.kCorr;
    c.n_corr = p.nCorr;
    c.delta_q = p.deltaQ;
    c.cohesion_strength = p.cohesionStrength;
    c.enable_viscosity = p.enableViscosity ? 1u : 0u;
    c.viscosity = p.viscosity;
    c.interaction_radius = p.interactionRadius;
    c.interaction_strength = p.interactionStrength;
    c.enable_vorticity = p.enableVorticity ? 1u : 0u;
    c.vorticity_epsilon = p.vorticityEpsilon;
    c.enable_apbf = p.enableAPBF ? 1u : 0u;
    c.min_lod = p.minLOD;
    c.max_lod = p.maxLOD;
    c.lod_max_dist = p.lodMaxDist;
}

FluidConfig pbfhost::fluid_config_from_c(const pbf_fluid_config& c)
{
    FluidConfig p;
    p.dt = c.dt;
    p.gravity = {c.gravity[0], c.gravity[1], c.gravity[2]};
    p.h = c.h;
    p.rho0 = c.rho0;
    p.solverIterations = c.solver_iterations;
    p.substepIterations = c.substep_iterations;
    p.eps = c.eps;
    p.particleCount = c.particle_count;
    p.spawnMin = {c.spawn_min[0], c.spawn_min[1], c.spawn_min[2]};
    p.spawnMax = {c.spawn_max[0], c.spawn_max[1], c.spawn_max[2]};
    p.spawnRandom = c.spawn_random != 0;
    p.spacing = c.spacing;
    p.initialVelocity = {c.initial_velocity[0], c.initial_velocity[1], c.initial_velocity[2]};
    p.boundsMin = {c.bounds_min[0], c.bounds_min[1], c.bounds_min[2]};
    p.boundsMax = {c.bounds_max[0], c.bounds_max[1], c.bounds_max[2]};
    p.boundDamping = c.bound_damping;
    p.hashSize = c.hash_size;
    p.enableSCorr = c.enable_scorr != 0;
    p.kCorr = c.k_corr;
    p.nCorr = c.n_corr;
    p.deltaQ = c.delta_q;
    p.cohesionStrength = c.cohesion_strength;
    p.enableViscosity = c.enable_viscosity != 0;
    p.viscosity = c.viscosity;
    p.interactionRadius = c.interaction_radius;
    p.interactionStrength = c.interaction_strength;
    p.enableVorticity = c.enable_vorticity != 0;
    p.vorticityEpsilon = c.vorticity_epsilon;
    p.enableAPBF = c.enable_apbf != 0;
    p.minLOD = c.min_lod;
    p.maxLOD = c.max_lod;
    p.lodMaxDist = c.lod_max_dist;
    return p;
}

void PBFluids::toC(const FluidConfig& p, void* out) { pbfhost::fluid_config_to_c(p, static_cast<pbf_fluid_config*>(out)); }

void PBFluids::report(int rc, const char* what) const
{
    if (rc != PBF_OK) std::fprintf(stderr, "PBFluids::%s: %s\n", what, pbf_last_error());
}

PBFluids::PBFluids() : PBFluids(FluidConfig{}) {}

PBFluids::PBFluids(const FluidConfig& p, int device) : _params(p)
{
    pbf_fluid_config c;
    toC(p, &c);
    const int rc = pbf_create(&c, device, &_h);
    if (rc != PBF_OK) {
        report(rc, "PBFluids");
        _h = nullptr;
    }
}

PBFluids::~PBFluids() { pbf_destroy(_h); }

void PBFluids::setParams(const FluidConfig& p)
{
    _params = p;
    if (!_h) return;
    pbf_fluid_config c;
    toC(p, &c);
    report(pbf_set_collision_padding(_h, _collisionPadding), "setParams");
    report(pbf_set_params(_h, &c), "setParams");
}

void PBFluids::setCameraPos(const PVec3& pos)
{
    const float q[3] = {pos.x, pos.y, pos.z};
    if (_h) report(pbf_set_camera_pos(_h, q), "setCameraPos");
}

void PBFluids::setParticles(const std::vector<Particle>& particles)
{
    _particles = particles;
    _params.particleCount = (U32)particles.size();
    if (!_h) return;
    static_assert(sizeof(Particle) == sizeof(pbf_particle), "Particle layout");
    report(pbf_set_particles(_h, reinterpret_cast<const pbf_particle*>(particles.data()), (uint32_t)particles.size()),
           "setParticles");
}

void PBFluids::setCollisionPadding(F32 p)
{
    _collisionPadding = p;
    if (_h) report(pbf_set_collision_padding(_h, p), "setCollisionPadding");
}

void PBFluids::setBounds(const PVec3& minBound, const PVec3& maxBound, F32 damping)
{
    const float mn[3] = {minBound.x, minBound.y, minBound.z}, mx[3] = {maxBound.x, maxBound.y, maxBound.z};
    if (_h) report(pbf_set_bounds(_h, mn, mx, damping), "setBounds");
}

void PBFluids::setSDFBoundary(const SDFBoundary* sdf)
{
    _sdf = sdf;
    if (!_h) return;
    if (sdf && sdf->valid() && sdf->handle())
        report(pbf_attach_sdf(_h, sdf->handle()), "setSDFBoundary");
    else
        report(pbf_attach_sdf(_h, nullptr), "setSDFBoundary");
}

void PBFluids::setSDFPadding(F32 padding)
{
    _sdfPadding = padding;
    if (_h) report(pbf_set_sdf_mode(_h, _sdfPadding, _sdfContainment ? 1 : 0), "setSDFPadding");
}

void PBFluids::setSDFContainment(bool inside)
{
    _sdfContainment = inside;
    if (_h) report(pbf_set_sdf_mode(_h, _sdfPadding, _sdfContainment ? 1 : 0), "setSDFContainment");
}

void PBFluids::setInteraction(bool active, const PVec3& pos)
{
    const float q[3] = {pos.x, pos.y, pos.z};
    if (_h) report(pbf_set_interaction(_h, active ? 1 : 0, q), "setInteraction");
}

void PBFluids::step()
{
    if (_particles.empty() || !_h) return;  // PBFluids.cpp:325
    report(pbf_step(_h), "step");
}

PBFluids::DeviceParticles PBFluids::bindParticlesForRendering() const
{
    DeviceParticles d;
    if (!_h) return d;
    size_t b = 0;
    pbf_buffer_device_ptr(_h, PBF_BUF_POS, &d.pos4, &b);
    pbf_buffer_device_ptr(_h, PBF_BUF_VEL, &d.vel4, &b);
    uint32_t n = 0;
    pbf_particle_count(_h, &n);
    d.count = n;
    return d;
}

void PBFluids::readbackParticles(std::vector<Particle>& out)
{
    uint32_t n = 0;
    if (_h) pbf_particle_count(_h, &n);
    out.resize(n);
    if (n == 0) return;
    report(pbf_read_particles(_h, reinterpret_cast<pbf_particle*>(out.data()), n), "readbackParticles");
}

void PBFluids::filterContactCandidates(float contactBand)
{
    if (!_sdf || !_sdf->valid() || contactBand <= 0.0f || !_h) return;  // PBFluids.cpp:195
    report(pbf_filter_contacts(_h, contactBand), "filterContactCandidates");
}

void PBFluids::readbackContactCandidates(std::vector<ContactCandidate>& out)
{
    out.clear();
    if (!_h) return;
    uint32_t count = 0;
    if (pbf_read_contacts(_h, nullptr, 0, &count) != PBF_OK || count == 0) return;
    out.resize(count);
    static_assert(sizeof(ContactCandidate) == sizeof(pbf_contact_candidate), "ContactCandidate layout");
    report(pbf_read_contacts(_h, reinterpret_cast<pbf_contact_candidate*>(out.data()), count, &count),
           "readbackContactCandidates");
    out.resize(count);
}

int PBFluids::computeContactForces(float band, bool useVelMagnitude, std::vector<PVec3>& vertForces)
{
    if (!_h || !_sdf || !_sdf->valid()) return 0;
    int32_t contacts = 0;
    static_assert(sizeof(PVec3) == 3 * sizeof(float), "PVec3 layout");
    const int rc = pbf_vertex_forces(_h, band, useVelMagnitude ? 1 : 0, reinterpret_cast<float*>(vertForces.data()),
                                     (int32_t)vertForces.size(), &contacts);
    report(rc, "computeContactForces");
    return contacts;
}
