// Minimal stand-in for the FDPS umbrella header, written for this repository.
//
// TEST INFRASTRUCTURE ONLY. It lets the reference's own physics headers
// (src/param.h, src/kernel.h, src/EoS.h, src/class.h, src/force.h,
// src/integral.h) compile unmodified so that their CPU functors can serve as
// the parity oracle.  FDPS itself (https://github.com/FDPS/FDPS.git, unpinned
// in CloneFDPS.sh:1) is not vendored by the reference and is absent here; only
// the handful of names those headers touch are provided:
//   * scalar typedefs  PS::F64, PS::F32, PS::S32, PS::S64, PS::U32, PS::U64
//   * PS::F64vec       a 3-D vector with FDPS's operator set (operator* between
//                      two vectors is the dot product, as in FDPS Vector3)
//   * PS::DIMENSION    3 (the oracle is always 3-D)
//   * PS::Comm         single-process getMinValue / getRank / broadcast
//   * PS::ParticleSystem<T>  a std::vector with the two accessors the headers use
//   * PS::DomainInfo   an empty tag type (named in a class.h:271 signature)
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>
#include <algorithm>
#include <iostream>
#include <iomanip>
#include <chrono>

namespace PS {
typedef double F64;
typedef float F32;
typedef int32_t S32;
typedef int64_t S64;
typedef uint32_t U32;
typedef uint64_t U64;

static const S32 DIMENSION = 3;

template <typename T> struct Vec3 {
  T x, y, z;
  Vec3() : x(0), y(0), z(0) {}
  Vec3(T a) : x(a), y(a), z(a) {}
  Vec3(T a, T b, T c) : x(a), y(b), z(c) {}
  Vec3& operator=(T a) { x = y = z = a; return *this; }
  Vec3 operator+(const Vec3& o) const { return Vec3(x + o.x, y + o.y, z + o.z); }
  Vec3 operator-(const Vec3& o) const { return Vec3(x - o.x, y - o.y, z - o.z); }
  Vec3 operator-() const { return Vec3(-x, -y, -z); }
  // FDPS Vector3: vector * vector is the inner product.
  T operator*(const Vec3& o) const { return x * o.x + y * o.y + z * o.z; }
  Vec3 operator*(T s) const { return Vec3(x * s, y * s, z * s); }
  Vec3 operator/(T s) const { return Vec3(x / s, y / s, z / s); }
  Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  Vec3& operator-=(const Vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  Vec3& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
  Vec3& operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
};
template <typename T> inline Vec3<T> operator*(T s, const Vec3<T>& v) { return v * s; }

typedef Vec3<F64> F64vec;

struct Comm {
  static S32 getRank() { return 0; }
  static S32 getNumberOfProc() { return 1; }
  static S32 getNumberOfThread() { return 1; }
  template <typename T> static T getMinValue(const T v) { return v; }
  template <typename T> static void broadcast(T*, S32, S32) {}
  static void barrier() {}
};

class DomainInfo {};

template <typename T> class ParticleSystem {
 public:
  std::vector<T> p;
  S32 getNumberOfParticleLocal() const { return (S32)p.size(); }
  void setNumberOfParticleLocal(S32 n) { p.resize(n); }
  T& operator[](S32 i) { return p[i]; }
  const T& operator[](S32 i) const { return p[i]; }
};
}  // namespace PS
