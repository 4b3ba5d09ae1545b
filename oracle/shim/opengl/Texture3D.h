/* Stand-in for the reference's opengl/Texture3D.h: the methods
 * SDFBoundary.cpp calls, as no-ops (nothing is uploaded; the CPU grid is what
 * the oracle reads). */
#ifndef PBF_ORACLE_SHIM_TEXTURE3D_H
#define PBF_ORACLE_SHIM_TEXTURE3D_H
#include <vector>
#include "glad/glad.h"
class Texture3D {
public:
    void upload(int, int, int, const std::vector<float>&) {}
    void uploadSubRegion(int, int, int, int, int, int, const std::vector<float>&) {}
    void bindToUnit(GLuint) const {}
};
#endif
