// Scenes.cpp — the scene presets (include/core/Scene.h) and the headless
// set-up of include/core/SceneSetup.h, plus their C ABI (pbf_scene_*,
// pbf_off_*, pbf_mesh_*, pbf_spawn_particles).  Host code only.
#include "core/SceneSetup.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <random>
#include <sstream>

#include "config_c.h"
#include "fluid/PBFluids.h"
#include "fluid/SDFBoundary.h"
#include "pbf_b200.h"

namespace pbf {
int set_error(int code, const char* fmt, ...);
}

// ---- presets (include/core/Scene.h:70-306) ---------------------------------------------------
namespace {

// What the four presets share: a 6^3 domain, h = 0.15, rho0 = 1000, two
// substeps of a 1/60 s frame, 16,384 lattice particles, 2^15 hash buckets,
// s_corr k = 0.001, n = 4, dq = 0.3, viscosity 0.1, vorticity off.  Fields
// a preset does not list keep FluidConfig's defaults (APBF off).
FluidConfig preset_fluid(U32 iterations, PVec3 spawnLo, PVec3 spawnHi, F32 spacing, F32 damping, F32 interactionRadius)
{
    FluidConfig f;
    f.dt = 1.0f / 60.0f;
    f.gravity = {0.0f, -9.81f, 0.0f};
    f.h = 0.15f;
    f.rho0 = 1000.0f;
    f.solverIterations = iterations;
    f.substepIterations = 2;
    f.eps = 0.0001f;
    f.particleCount = 1u << 14;
    f.spawnMin = spawnLo;
    f.spawnMax = spawnHi;
    f.spawnRandom = false;
    f.spacing = spacing;
    f.initialVelocity = {0.0f, 0.0f, 0.0f};
    f.boundsMin = {0.0f, 0.0f, 0.0f};
    f.boundsMax = {6.0f, 6.0f, 6.0f};
    f.boundDamping = damping;
    f.hashSize = 1u << 15;
    f.enableSCorr = true;
    f.kCorr = 0.001f;
    f.nCorr = 4.0f;
    f.deltaQ = 0.3f;
    f.cohesionStrength = 0.001f;
    f.enableViscosity = true;
    f.viscosity = 0.1f;
    f.interactionRadius = interactionRadius;
    f.interactionStrength = 25.0f;
    f.enableVorticity = false;
    f.vorticityEpsilon = 0.05f;
    return f;
}

Scene preset(const char* name, const FluidConfig& fluid, float pitch, float dist, const char* mesh, float fit, float cell,
             bool container, PVec3 translate, PVec3 rot, SceneDeform deform)
{
    Scene s;
    s.name = name;
    s.fluid = fluid;
    s.camYaw = 0.6f;
    s.camPitch = pitch;
    s.camDist = dist;
    s.pointSize = 8.0f;
    s.meshFile = mesh;
    s.meshFitSize = fit;
    s.sdfCell = cell;
    s.sdfPadding = 0.05f;
    s.sdfContainer = container;
    s.meshTranslate = translate;
    s.meshRotDeg = rot;
    s.deform = deform;
    return s;
}

std::vector<Scene> make_presets()
{
    const PVec3 above_lo{0.2f, 0.2f, 0.2f}, above_hi{5.8f, 1.0f, 5.8f};
    const PVec3 zero{0.0f, 0.0f, 0.0f};
    std::vector<Scene> v;
    // fluid spawned inside a closed cube and held there by the SDF
    v.push_back(preset("Container Cube",
                       preset_fluid(3, {1.0f, 1.0f, 1.0f}, {5.0f, 2.5f, 5.0f}, 0.11f, 0.3f, 2.0f), 0.35f, 13.0f,
                       "cube1538.off", 4.5f, 0.10f, true, {0.0f, 0.5f, 0.0f}, zero,
                       SceneDeform{1.0f, 0.02f, 0.25f, true, 0.02f, 1.8f, 1.5f, 2, 0.12f}));
    // a block pouring onto the outside of a cube
    v.push_back(preset("Surface Cube", preset_fluid(4, above_lo, above_hi, 0.1f, 0.4f, 2.5f), 0.35f, 12.0f,
                       "cube1538.off", 3.0f, 0.10f, false, {0.0f, 0.5f, 0.0f}, zero,
                       SceneDeform{1.0f, 0.02f, 0.30f, true, 0.02f, 1.20f, 1.0f, 3, 0.12f}));
    // onto a bull figure
    v.push_back(preset("Surface Bull", preset_fluid(5, above_lo, above_hi, 0.1f, 0.4f, 2.5f), 0.30f, 12.0f, "386.off",
                       4.0f, 0.08f, false, zero, {270.0f, 0.0f, 0.0f},
                       SceneDeform{2.0f, 0.020f, 0.40f, true, 0.04f, 0.5f, 0.3f, 2, 0.12f}));
    // onto a hand
    v.push_back(preset("Surface Hand", preset_fluid(4, above_lo, above_hi, 0.1f, 0.4f, 1.5f), 0.30f, 12.0f, "200.off",
                       4.5f, 0.08f, false, zero, {90.0f, 0.0f, 0.0f},
                       SceneDeform{1.5f, 0.025f, 0.45f, true, 0.05f, 0.45f, 0.28f, 3, 0.12f}));
    return v;
}

}  // namespace

const std::vector<Scene>& getScenes()
{
    static const std::vector<Scene> scenes = make_presets();
    return scenes;
}

// ---- OFF assets (src/main.cpp:364-415) ------------------------------------------------------
namespace {

// Next line that is neither empty nor a comment; false at end of file.
bool next_content_line(std::istream& in, std::string& line)
{
    while (std::getline(in, line)) {
        while (!line.empty() && (line.back() == '\r' || line.back() == ' ' || line.back() == '\t')) line.pop_back();
        if (!line.empty() && line[0] != '#') return true;
    }
    return false;
}

}  // namespace

bool loadOFF(const std::string& path, MeshData& out)
{
    std::ifstream f(path);
    if (!f) {
        std::fprintf(stderr, "loadOFF: cannot open %s\n", path.c_str());
        return false;
    }
    std::string line;
    if (!next_content_line(f, line) || line.find("OFF") == std::string::npos) {
        std::fprintf(stderr, "loadOFF: not an OFF file: %s\n", path.c_str());
        return false;
    }
    // Some writers put the counts on the header line itself ("OFF 8 12 0").
    long nv = -1, nf = -1, ne = 0;
    {
        std::istringstream hs(line.substr(line.find("OFF") + 3));
        if (!(hs >> nv >> nf)) nv = nf = -1;
    }
    while (nv < 0) {
        if (!next_content_line(f, line)) return false;
        std::istringstream ss(line);
        if (ss >> nv >> nf) {
            ss >> ne;
            break;
        }
        nv = nf = -1;
    }
    // counts past 2^30 are malformed; storage grows with the lines actually
    // read, so a count larger than the file allocates nothing up front
    if (nv < 0 || nf < 0 || nv > (1L << 30) || nf > (1L << 30)) return false;
    MeshData m;
    for (long i = 0; i < nv; ++i) {
        if (!next_content_line(f, line)) return false;
        std::istringstream ss(line);
        double x = 0.0, y = 0.0, z = 0.0;
        ss >> x >> y >> z;
        m.verts.push_back({x, y, z});
    }
    for (long i = 0; i < nf; ++i) {
        if (!next_content_line(f, line)) return false;
        std::istringstream ss(line);
        int k = 0;
        ss >> k;
        if (k < 0 || k > 4096) return false;  // a polygon's vertex count
        std::vector<int> poly((size_t)k);
        for (auto& q : poly) {
            if (!(ss >> q) || q < 0 || q >= nv) return false;  // a missing or out-of-range vertex index
        }
        for (int j = 1; j + 1 < k; ++j) m.faces.push_back({poly[0], poly[(size_t)j], poly[(size_t)j + 1]});
    }
    out = std::move(m);
    return true;
}

// ---- placement (src/main.cpp:419-432, 500-512, 747-770) -----------------------------------------
namespace {

void bbox(const MeshData& m, double lo[3], double hi[3])
{
    for (int k = 0; k < 3; ++k) {
        lo[k] = 1e30;
        hi[k] = -1e30;
    }
    for (const auto& v : m.verts)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], v[(size_t)k]);
            hi[k] = std::max(hi[k], v[(size_t)k]);
        }
}

// Column-major 3x3 rotation by `rad` about unit axis a, in float (the
// Rodrigues form: c I + (1 - c) a a^T + s [a]x).
struct M3 {
    float m[3][3];  // m[col][row]
};

M3 axis_rotation(float rad, int axis)
{
    const float c = std::cos(rad), s = std::sin(rad);
    float a[3] = {0.0f, 0.0f, 0.0f};
    a[axis] = 1.0f;
    M3 r;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) r.m[col][row] = (1.0f - c) * a[col] * a[row] + (col == row ? c : 0.0f);
    // skew part: column col, row row gets s * (a x e_col)_row
    r.m[0][1] += s * a[2];
    r.m[0][2] -= s * a[1];
    r.m[1][0] -= s * a[2];
    r.m[1][2] += s * a[0];
    r.m[2][0] += s * a[1];
    r.m[2][1] -= s * a[0];
    return r;
}

M3 mul(const M3& A, const M3& B)
{
    M3 r;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row)
            r.m[col][row] = A.m[0][row] * B.m[col][0] + A.m[1][row] * B.m[col][1] + A.m[2][row] * B.m[col][2];
    return r;
}

}  // namespace

void fitMeshToDomain(MeshData& m, const PVec3& center, double targetSize)
{
    if (m.verts.empty()) return;
    double lo[3], hi[3];
    bbox(m, lo, hi);
    double mid[3], ext = 1e-9;
    for (int k = 0; k < 3; ++k) {
        mid[k] = 0.5 * (lo[k] + hi[k]);
        ext = std::max(ext, hi[k] - lo[k]);
    }
    const double s = targetSize / ext;
    const double c[3] = {center.x, center.y, center.z};
    for (auto& v : m.verts)
        for (int k = 0; k < 3; ++k) v[(size_t)k] = (v[(size_t)k] - mid[k]) * s + c[k];
}

PVec3 meshFitCenter(const FluidConfig& c)
{
    return PVec3{0.5f * (c.boundsMin.x + c.boundsMax.x), c.boundsMin.y + 0.40f * (c.boundsMax.y - c.boundsMin.y),
                 0.5f * (c.boundsMin.z + c.boundsMax.z)};
}

void placeMesh(MeshData& m, const PVec3& translate, const PVec3& rotDeg)
{
    if (m.verts.empty()) return;
    double lo[3], hi[3];
    bbox(m, lo, hi);
    const float pivot[3] = {0.5f * (float)(lo[0] + hi[0]), 0.5f * (float)(lo[1] + hi[1]), 0.5f * (float)(lo[2] + hi[2])};
    const float deg = 0.01745329251994329577f;
    const M3 R = mul(mul(axis_rotation(rotDeg.x * deg, 0), axis_rotation(rotDeg.y * deg, 1)),
                     axis_rotation(rotDeg.z * deg, 2));
    const float t[3] = {translate.x, translate.y, translate.z};
    for (auto& v : m.verts) {
        const float p[3] = {(float)v[0] - pivot[0], (float)v[1] - pivot[1], (float)v[2] - pivot[2]};
        for (int row = 0; row < 3; ++row) {
            const float q = R.m[0][row] * p[0] + R.m[1][row] * p[1] + R.m[2][row] * p[2];
            v[(size_t)row] = (double)(q + pivot[row] + t[row]);
        }
    }
}

// ---- particles (src/main.cpp:155-188) -----------------------------------------------------------
std::vector<Particle> spawnParticles(const FluidConfig& c)
{
    std::vector<Particle> out;
    out.reserve(c.particleCount);
    if (c.spawnRandom) {
        std::mt19937 rng(1337);
        std::uniform_real_distribution<float> u01(0.0f, 1.0f);
        const PVec3 lo{c.spawnMin.x + c.spacing, c.spawnMin.y + c.spacing, c.spawnMin.z + c.spacing};
        const PVec3 hi{c.spawnMax.x - c.spacing, c.spawnMax.y - c.spacing, c.spawnMax.z - c.spacing};
        for (U32 i = 0; i < c.particleCount; ++i) {
            Particle p{};
            // one draw per axis, x first
            const float ux = u01(rng);
            const float uy = u01(rng);
            const float uz = u01(rng);
            p.pos = {lo.x + (hi.x - lo.x) * ux, lo.y + (hi.y - lo.y) * uy, lo.z + (hi.z - lo.z) * uz};
            p.predPos = p.pos;
            p.vel = c.initialVelocity;
            out.push_back(p);
        }
        return out;
    }
    const float step = std::max(1e-6f, c.spacing);
    const auto full = [&] { return (U32)out.size() >= c.particleCount; };
    for (float z = c.spawnMin.z; z <= c.spawnMax.z && !full(); z += step)
        for (float y = c.spawnMin.y; y <= c.spawnMax.y && !full(); y += step)
            for (float x = c.spawnMin.x; x <= c.spawnMax.x && !full(); x += step) {
                Particle p{};
                p.pos = {x, y, z};
                p.predPos = p.pos;
                p.vel = c.initialVelocity;
                out.push_back(p);
            }
    return out;
}

// ---- whole scenes (src/main.cpp:959-993, 1192-1243) ---------------------------------------------
bool buildSceneState(const Scene& sc, const std::string& assetDir, SceneState& out, const std::string& meshPath)
{
    const std::string path = !meshPath.empty() ? meshPath
                             : assetDir.empty() ? std::string(sc.meshFile)
                                                : assetDir + "/" + sc.meshFile;
    MeshData m;
    if (!loadOFF(path, m)) return false;
    fitMeshToDomain(m, meshFitCenter(sc.fluid), sc.meshFitSize);
    placeMesh(m, sc.meshTranslate, sc.meshRotDeg);
    out.mesh = std::move(m);
    out.particles = spawnParticles(sc.fluid);
    return true;
}

bool loadScene(const Scene& sc, const std::string& assetDir, PBFluids& fluid, SDFBoundary& sdf, SceneState* state,
               const std::string& meshPath)
{
    SceneState st;
    if (!buildSceneState(sc, assetDir, st, meshPath)) return false;
    fluid.setParams(sc.fluid);
    fluid.setBounds(sc.fluid.boundsMin, sc.fluid.boundsMax, sc.fluid.boundDamping);
    sdf.buildFromMesh(st.mesh.verts, st.mesh.faces, sc.sdfCell, false);
    if (!sdf.valid()) return false;
    fluid.setSDFBoundary(&sdf);
    fluid.setSDFPadding(sc.sdfPadding);
    fluid.setSDFContainment(sc.sdfContainer);
    fluid.setParticles(st.particles);
    if (state) *state = std::move(st);
    return true;
}

// ---- C ABI ----------------------------------------------------------------------------------------
using pbf::set_error;

extern "C" int pbf_scene_count(void) { return (int)getScenes().size(); }

extern "C" int pbf_scene_get(int32_t index, pbf_scene_preset* out)
{
    const auto& all = getScenes();
    if (!out) return set_error(PBF_ERR_INVALID, "null output");
    if (index < 0 || index >= (int32_t)all.size())
        return set_error(PBF_ERR_INVALID, "scene index %d out of range [0, %zu)", index, all.size());
    const Scene& s = all[(size_t)index];
    std::memset(out, 0, sizeof(*out));
    std::snprintf(out->name, sizeof(out->name), "%s", s.name);
    pbfhost::fluid_config_to_c(s.fluid, &out->fluid);
    out->cam_yaw = s.camYaw;
    out->cam_pitch = s.camPitch;
    out->cam_dist = s.camDist;
    out->point_size = s.pointSize;
    std::snprintf(out->mesh_file, sizeof(out->mesh_file), "%s", s.meshFile);
    out->mesh_fit_size = s.meshFitSize;
    out->sdf_cell = s.sdfCell;
    out->sdf_padding = s.sdfPadding;
    out->sdf_container = s.sdfContainer ? 1u : 0u;
    const PVec3 t = s.meshTranslate, r = s.meshRotDeg;
    out->mesh_translate[0] = t.x, out->mesh_translate[1] = t.y, out->mesh_translate[2] = t.z;
    out->mesh_rot_deg[0] = r.x, out->mesh_rot_deg[1] = r.y, out->mesh_rot_deg[2] = r.z;
    const SceneDeform& d = s.deform;
    out->deform.stiffness = d.stiffness;
    out->deform.max_displacement = d.maxDisplacement;
    out->deform.max_total_disp = d.maxTotalDisp;
    out->deform.restore_enabled = d.restoreEnabled ? 1u : 0u;
    out->deform.restore_strength = d.restoreStrength;
    out->deform.control_threshold = d.controlThreshold;
    out->deform.control_threshold_low = d.controlThresholdLow;
    out->local_kring = d.localKRing;
    out->contact_radius = d.contactRadius;
    return PBF_OK;
}

extern "C" int pbf_off_load(const char* path, double* verts3, int32_t vcap, int32_t* faces3, int32_t fcap,
                            int32_t* nv, int32_t* nf)
{
    if (!path || !nv || !nf) return set_error(PBF_ERR_INVALID, "null argument");
    MeshData m;
    try {
        if (!loadOFF(path, m)) return set_error(PBF_ERR_INVALID, "pbf_off_load: cannot read an OFF mesh from %s", path);
    } catch (const std::exception& e) {
        return set_error(PBF_ERR_ALLOC, "pbf_off_load: %s", e.what());
    }
    if (m.verts.size() > (size_t)INT32_MAX || m.faces.size() > (size_t)INT32_MAX)
        return set_error(PBF_ERR_INVALID, "pbf_off_load: mesh too large");
    *nv = (int32_t)m.verts.size();
    *nf = (int32_t)m.faces.size();
    if (verts3 && vcap >= *nv)
        for (size_t i = 0; i < m.verts.size(); ++i)
            for (int k = 0; k < 3; ++k) verts3[3 * i + (size_t)k] = m.verts[i][(size_t)k];
    if (faces3 && fcap >= *nf)
        for (size_t i = 0; i < m.faces.size(); ++i)
            for (int k = 0; k < 3; ++k) faces3[3 * i + (size_t)k] = m.faces[i][(size_t)k];
    return PBF_OK;
}

namespace {
MeshData wrap(const double* verts3, int32_t nv)
{
    MeshData m;
    m.verts.resize((size_t)nv);
    for (int32_t i = 0; i < nv; ++i) m.verts[(size_t)i] = {verts3[3 * i], verts3[3 * i + 1], verts3[3 * i + 2]};
    return m;
}
void unwrap(const MeshData& m, double* verts3)
{
    for (size_t i = 0; i < m.verts.size(); ++i)
        for (int k = 0; k < 3; ++k) verts3[3 * i + (size_t)k] = m.verts[i][(size_t)k];
}
}  // namespace

extern "C" int pbf_mesh_fit(double* verts3, int32_t nv, const float center[3], double target_size)
{
    if (!verts3 || !center || nv < 0) return set_error(PBF_ERR_INVALID, "bad mesh arguments");
    try {
        MeshData m = wrap(verts3, nv);
        fitMeshToDomain(m, PVec3{center[0], center[1], center[2]}, target_size);
        unwrap(m, verts3);
    } catch (const std::exception& e) {
        return set_error(PBF_ERR_ALLOC, "pbf_mesh_fit: %s", e.what());
    }
    return PBF_OK;
}

extern "C" int pbf_mesh_fit_center(const pbf_fluid_config* cfg, float center_out[3])
{
    if (!cfg || !center_out) return set_error(PBF_ERR_INVALID, "null argument");
    const PVec3 c = meshFitCenter(pbfhost::fluid_config_from_c(*cfg));
    center_out[0] = c.x, center_out[1] = c.y, center_out[2] = c.z;
    return PBF_OK;
}

extern "C" int pbf_mesh_place(double* verts3, int32_t nv, const float translate[3], const float rot_deg[3])
{
    if (!verts3 || !translate || !rot_deg || nv < 0) return set_error(PBF_ERR_INVALID, "bad mesh arguments");
    try {
        MeshData m = wrap(verts3, nv);
        placeMesh(m, PVec3{translate[0], translate[1], translate[2]}, PVec3{rot_deg[0], rot_deg[1], rot_deg[2]});
        unwrap(m, verts3);
    } catch (const std::exception& e) {
        return set_error(PBF_ERR_ALLOC, "pbf_mesh_place: %s", e.what());
    }
    return PBF_OK;
}

extern "C" int pbf_spawn_particles(const pbf_fluid_config* cfg, pbf_particle* out, uint32_t capacity, uint32_t* count)
{
    if (!cfg || !count) return set_error(PBF_ERR_INVALID, "null argument");
    std::vector<Particle> ps;
    try {
        ps = spawnParticles(pbfhost::fluid_config_from_c(*cfg));
    } catch (const std::exception& e) {
        return set_error(PBF_ERR_ALLOC, "pbf_spawn_particles: %s", e.what());
    }
    *count = (uint32_t)ps.size();
    if (out && capacity >= *count) std::memcpy(out, ps.data(), ps.size() * sizeof(Particle));
    return PBF_OK;
}
