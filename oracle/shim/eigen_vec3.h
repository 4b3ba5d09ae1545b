/*
 * eigen_vec3.h — the small part of Eigen's fixed-size vector interface that
 * the reference's src/fluid/SDFBoundary.cpp uses (Vector3d / Vector3i:
 * construction, Zero/Ones, x/y/z, arithmetic, dot, cross, norm,
 * squaredNorm, normalized, cwiseMin/cwiseMax and array() for coefficient-wise
 * arithmetic with scalars), written here so that file compiles as test
 * infrastructure under oracle/_ref.  The reference vendors no usable Eigen
 * (thirdparty/eigen lacks Eigen/Core) and none is installed.  Arithmetic is
 * plain IEEE double / int per coefficient, the order Eigen evaluates these
 * 3-vector expressions in.
 */
#ifndef PBF_ORACLE_SHIM_EIGEN_VEC3_H
#define PBF_ORACLE_SHIM_EIGEN_VEC3_H
#include <algorithm>
#include <cmath>

namespace Eigen {

template <typename T>
struct Vec3 {
    T c[3];
    Vec3() : c{T(0), T(0), T(0)} {}
    Vec3(T x, T y, T z) : c{x, y, z} {}
    static Vec3 Zero() { return Vec3(T(0), T(0), T(0)); }
    static Vec3 Ones() { return Vec3(T(1), T(1), T(1)); }
    T& x() { return c[0]; }
    T& y() { return c[1]; }
    T& z() { return c[2]; }
    const T& x() const { return c[0]; }
    const T& y() const { return c[1]; }
    const T& z() const { return c[2]; }
    T& operator[](int i) { return c[i]; }
    const T& operator[](int i) const { return c[i]; }
    T& operator()(int i) { return c[i]; }
    const T& operator()(int i) const { return c[i]; }
    // coefficient-wise view: the same object (scalar +/- below apply to it)
    const Vec3& array() const { return *this; }
    Vec3& array() { return *this; }
    T dot(const Vec3& o) const { return c[0] * o.c[0] + c[1] * o.c[1] + c[2] * o.c[2]; }
    Vec3 cross(const Vec3& o) const
    {
        return Vec3(c[1] * o.c[2] - c[2] * o.c[1], c[2] * o.c[0] - c[0] * o.c[2], c[0] * o.c[1] - c[1] * o.c[0]);
    }
    T squaredNorm() const { return dot(*this); }
    T norm() const { return std::sqrt(squaredNorm()); }
    Vec3 normalized() const
    {
        const T n = norm();
        return n > T(0) ? Vec3(c[0] / n, c[1] / n, c[2] / n) : *this;
    }
    void normalize() { *this = normalized(); }
    Vec3 cwiseMin(const Vec3& o) const
    {
        return Vec3(std::min(c[0], o.c[0]), std::min(c[1], o.c[1]), std::min(c[2], o.c[2]));
    }
    Vec3 cwiseMax(const Vec3& o) const
    {
        return Vec3(std::max(c[0], o.c[0]), std::max(c[1], o.c[1]), std::max(c[2], o.c[2]));
    }
    Vec3& operator+=(const Vec3& o) { c[0] += o.c[0]; c[1] += o.c[1]; c[2] += o.c[2]; return *this; }
    Vec3& operator-=(const Vec3& o) { c[0] -= o.c[0]; c[1] -= o.c[1]; c[2] -= o.c[2]; return *this; }
    Vec3& operator*=(T s) { c[0] *= s; c[1] *= s; c[2] *= s; return *this; }
    Vec3& operator/=(T s) { c[0] /= s; c[1] /= s; c[2] /= s; return *this; }
};

template <typename T> Vec3<T> operator+(const Vec3<T>& a, const Vec3<T>& b) { return Vec3<T>(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <typename T> Vec3<T> operator-(const Vec3<T>& a, const Vec3<T>& b) { return Vec3<T>(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <typename T> Vec3<T> operator-(const Vec3<T>& a) { return Vec3<T>(-a[0], -a[1], -a[2]); }
template <typename T> Vec3<T> operator*(const Vec3<T>& a, T s) { return Vec3<T>(a[0] * s, a[1] * s, a[2] * s); }
template <typename T> Vec3<T> operator*(T s, const Vec3<T>& a) { return Vec3<T>(s * a[0], s * a[1], s * a[2]); }
template <typename T> Vec3<T> operator/(const Vec3<T>& a, T s) { return Vec3<T>(a[0] / s, a[1] / s, a[2] / s); }
// array() arithmetic with a scalar
template <typename T> Vec3<T> operator+(const Vec3<T>& a, T s) { return Vec3<T>(a[0] + s, a[1] + s, a[2] + s); }
template <typename T> Vec3<T> operator-(const Vec3<T>& a, T s) { return Vec3<T>(a[0] - s, a[1] - s, a[2] - s); }

using Vector3d = Vec3<double>;
using Vector3i = Vec3<int>;

}  // namespace Eigen
#endif
