// Small 3-vector used by the host API in place of Eigen::Vector3d.
//
// The reference API (include/FEM/NavierStokes.hpp:66-72, include/Mesh/Mesh.hpp:37-45)
// exposes Eigen::Vector3d; this type offers the accessors that callers of that API use
// (x(), y(), z(), operator(), dot, cross, norm, normalized, cwiseMin/Max) so that caller
// code reads the same. Arithmetic is written out in the natural left-to-right order
// ((a0*b0 + a1*b1) + a2*b2) with no fused multiply-add, so host geometry is reproducible.
#pragma once

#include <cmath>
#include <cstddef>

struct Vec3 {
  double v[3] = {0.0, 0.0, 0.0};

  Vec3() = default;
  Vec3(double x, double y, double z) : v{x, y, z} {}

  static Vec3 Zero() { return Vec3(0.0, 0.0, 0.0); }

  double &x() { return v[0]; }
  double &y() { return v[1]; }
  double &z() { return v[2]; }
  double x() const { return v[0]; }
  double y() const { return v[1]; }
  double z() const { return v[2]; }
  double &operator()(std::size_t i) { return v[i]; }
  double operator()(std::size_t i) const { return v[i]; }
  double &operator[](std::size_t i) { return v[i]; }
  double operator[](std::size_t i) const { return v[i]; }
  const double *data() const { return v; }
  double *data() { return v; }

  Vec3 operator+(const Vec3 &o) const { return Vec3(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]); }
  Vec3 operator-(const Vec3 &o) const { return Vec3(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
  Vec3 operator-() const { return Vec3(-v[0], -v[1], -v[2]); }
  Vec3 operator*(double s) const { return Vec3(v[0] * s, v[1] * s, v[2] * s); }
  Vec3 operator/(double s) const { return Vec3(v[0] / s, v[1] / s, v[2] / s); }
  Vec3 &operator+=(const Vec3 &o) { v[0] += o.v[0]; v[1] += o.v[1]; v[2] += o.v[2]; return *this; }
  Vec3 &operator-=(const Vec3 &o) { v[0] -= o.v[0]; v[1] -= o.v[1]; v[2] -= o.v[2]; return *this; }
  bool operator==(const Vec3 &o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }

  double dot(const Vec3 &o) const { return (v[0] * o.v[0] + v[1] * o.v[1]) + v[2] * o.v[2]; }
  Vec3 cross(const Vec3 &o) const {
    return Vec3(v[1] * o.v[2] - v[2] * o.v[1], v[2] * o.v[0] - v[0] * o.v[2],
                v[0] * o.v[1] - v[1] * o.v[0]);
  }
  double squaredNorm() const { return dot(*this); }
  double norm() const { return std::sqrt(squaredNorm()); }
  Vec3 normalized() const {
    const double n = norm();
    return n > 0.0 ? (*this) / n : *this;
  }
  Vec3 cwiseMin(const Vec3 &o) const {
    return Vec3(o.v[0] < v[0] ? o.v[0] : v[0], o.v[1] < v[1] ? o.v[1] : v[1],
                o.v[2] < v[2] ? o.v[2] : v[2]);
  }
  Vec3 cwiseMax(const Vec3 &o) const {
    return Vec3(v[0] < o.v[0] ? o.v[0] : v[0], v[1] < o.v[1] ? o.v[1] : v[1],
                v[2] < o.v[2] ? o.v[2] : v[2]);
  }
  bool hasNaN() const { return std::isnan(v[0]) || std::isnan(v[1]) || std::isnan(v[2]); }
};

inline Vec3 operator*(double s, const Vec3 &a) { return a * s; }
