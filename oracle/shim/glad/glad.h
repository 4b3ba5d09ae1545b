/* Stand-in for glad/glad.h: the GL scalar types the reference's
 * include/fluid/SDFBoundary.h names.  No GL function exists here. */
#ifndef PBF_ORACLE_SHIM_GLAD_H
#define PBF_ORACLE_SHIM_GLAD_H
typedef unsigned int GLuint;
typedef int GLint;
typedef unsigned int GLenum;
#endif
