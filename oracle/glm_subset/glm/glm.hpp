// Project-written stand-in for the subset of GLM 0.9.9.8 (environment.yml:19)
// that the reference rasterizer uses; GLM itself is not available here.
//
// Written from GLM's documented semantics, not from its sources:
//   * vec3 / vec4: packed float components x, y, z(, w); component-wise
//     arithmetic; scalar operands broadcast;
//   * mat3: column-major, m[c] is column c, m[c][r] row r of that column;
//     mat3(s) is s on the diagonal; mat3(9 scalars) fills column 0 first;
//   * A * B is the matrix product, (A*B)[c][r] = sum_k A[k][r] * B[c][k] with k
//     ascending; s * A scales every element; transpose swaps [c][r];
//   * dot(a, b) = a.x*b.x + a.y*b.y + a.z*b.z; length(v) = sqrt(dot(v, v)).
// Used only by oracle/build_ref.py to compile the reference as a checker.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define GLMS_FN __host__ __device__ inline
#else
#define GLMS_FN inline
#endif

namespace glm {

struct vec3 {
  float x, y, z;
  GLMS_FN vec3() : x(0.f), y(0.f), z(0.f) {}
  GLMS_FN explicit vec3(float s) : x(s), y(s), z(s) {}
  GLMS_FN vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  GLMS_FN float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  GLMS_FN const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  GLMS_FN vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  GLMS_FN vec3& operator-=(const vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  GLMS_FN vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
};

struct vec4 {
  float x, y, z, w;
  GLMS_FN vec4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
  GLMS_FN explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
  GLMS_FN vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};

GLMS_FN vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
GLMS_FN vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
GLMS_FN vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
GLMS_FN vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
GLMS_FN vec3 operator*(float s, const vec3& v) { return vec3(s * v.x, s * v.y, s * v.z); }
GLMS_FN vec3 operator*(const vec3& v, float s) { return vec3(v.x * s, v.y * s, v.z * s); }
GLMS_FN vec3 operator/(const vec3& v, float s) { return vec3(v.x / s, v.y / s, v.z / s); }

GLMS_FN float dot(const vec3& a, const vec3& b) {
  const vec3 t = a * b;
  return t.x + t.y + t.z;
}
GLMS_FN float length(const vec3& v) { return sqrtf(dot(v, v)); }

struct mat3 {
  vec3 col[3];
  GLMS_FN mat3() { col[0] = vec3(1.f, 0.f, 0.f); col[1] = vec3(0.f, 1.f, 0.f); col[2] = vec3(0.f, 0.f, 1.f); }
  GLMS_FN explicit mat3(float s) { col[0] = vec3(s, 0.f, 0.f); col[1] = vec3(0.f, s, 0.f); col[2] = vec3(0.f, 0.f, s); }
  GLMS_FN mat3(float a0, float a1, float a2, float b0, float b1, float b2, float c0, float c1, float c2) {
    col[0] = vec3(a0, a1, a2); col[1] = vec3(b0, b1, b2); col[2] = vec3(c0, c1, c2);
  }
  GLMS_FN vec3& operator[](int c) { return col[c]; }
  GLMS_FN const vec3& operator[](int c) const { return col[c]; }
};

GLMS_FN mat3 operator*(const mat3& A, const mat3& B) {
  mat3 o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o[c][r] = A[0][r] * B[c][0] + A[1][r] * B[c][1] + A[2][r] * B[c][2];
  return o;
}
GLMS_FN mat3 operator*(float s, const mat3& A) {
  mat3 o;
  for (int c = 0; c < 3; ++c) o[c] = A[c] * s;
  return o;
}
GLMS_FN mat3 operator*(const mat3& A, float s) { return s * A; }
GLMS_FN mat3 transpose(const mat3& A) {
  mat3 o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o[c][r] = A[r][c];
  return o;
}

}  // namespace glm
