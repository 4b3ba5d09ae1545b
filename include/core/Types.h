// core/Types.h — plain value types of the fluid path.
//
// Drop-in for the reference's include/core/Types.h:37-77 ("Fluid (GPU) -
// Plain Vectors"): same names and layouts, so code written against the
// reference's PBFluids compiles unchanged.  The Eigen/CHOLMOD aliases of the
// reference header belong to the host deformation solver, which is not part
// of this library, and are not declared here.
#ifndef PBF_B200_CORE_TYPES_H
#define PBF_B200_CORE_TYPES_H

#include <cmath>
#include <cstdint>

using F32 = float;
using I32 = std::int32_t;
using U32 = std::uint32_t;

struct PVec3 {
    F32 x, y, z;
};
struct PVec4 {
    F32 x, y, z, w;
};
struct UVec2 {
    U32 x, y;
};
struct IVec2 {
    I32 x, y;
};

inline PVec3 make_pvec3(F32 x, F32 y, F32 z) { return PVec3{x, y, z}; }
inline PVec3 operator+(PVec3 a, PVec3 b) { return PVec3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline PVec3 operator-(PVec3 a, PVec3 b) { return PVec3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline PVec3 operator*(PVec3 a, F32 s) { return PVec3{a.x * s, a.y * s, a.z * s}; }
inline PVec3 operator*(F32 s, PVec3 a) { return a * s; }
inline PVec3& operator+=(PVec3& a, PVec3 b) { return a = a + b; }
inline PVec3& operator-=(PVec3& a, PVec3 b) { return a = a - b; }
inline PVec3& operator*=(PVec3& a, F32 s) { return a = a * s; }
inline F32 dot(PVec3 a, PVec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F32 norm2(PVec3 a) { return dot(a, a); }
inline F32 norm(PVec3 a) { return std::sqrt(norm2(a)); }

#endif
