// Device math for the per-world kernels: 3-vectors, quaternions (w, x, y, z), 3x3 row-major
// matrices, 6-D spatial vectors (angular, linear) and 10-element inertias
// (xx, yy, zz, xy, xz, yz, m*cx, m*cy, m*cz, m).  The formulas are the ones the reference's
// mujoco_warp/_src/math.py states (cited per function); Warp's normalize() returns the zero vector
// for zero input and so do ours.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mjb {

constexpr float kMinVal = 1e-15f;   // mjMINVAL
constexpr float kMinImp = 0.0001f;  // mjMINIMP
constexpr float kMaxImp = 0.9999f;  // mjMAXIMP
constexpr float kPi = 3.14159265358979323846f;

enum { JNT_FREE = 0, JNT_BALL = 1, JNT_SLIDE = 2, JNT_HINGE = 3 };
enum { GEOM_PLANE = 0, GEOM_SPHERE = 2, GEOM_CAPSULE = 3, GEOM_BOX = 6 };
enum : int32_t {
  DSBL_CONSTRAINT = 1 << 0, DSBL_LIMIT = 1 << 3, DSBL_CONTACT = 1 << 4, DSBL_PASSIVE = 1 << 5,
  DSBL_GRAVITY = 1 << 6, DSBL_CLAMPCTRL = 1 << 7, DSBL_FILTERPARENT = 1 << 9,
  DSBL_ACTUATION = 1 << 10, DSBL_REFSAFE = 1 << 11, DSBL_EULERDAMP = 1 << 14
};

struct f3 {
  float x, y, z;
};
struct q4 {
  float w, x, y, z;
};
struct m33 {
  float m[9];
};

__device__ __forceinline__ f3 mk3(float a, float b, float c) { return f3{a, b, c}; }
__device__ __forceinline__ f3 ld3(const float* p) { return f3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(float* p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
__device__ __forceinline__ q4 ld4(const float* p) { return q4{p[0], p[1], p[2], p[3]}; }
__device__ __forceinline__ void st4(float* p, q4 q) { p[0] = q.w; p[1] = q.x; p[2] = q.y; p[3] = q.z; }
__device__ __forceinline__ m33 ld9(const float* p) {
  m33 r;
#pragma unroll
  for (int i = 0; i < 9; i++) r.m[i] = p[i];
  return r;
}
__device__ __forceinline__ void st9(float* p, const m33& r) {
#pragma unroll
  for (int i = 0; i < 9; i++) p[i] = r.m[i];
}

__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return f3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 normalize(f3 a) {
  float l = length(a);
  return l > 0.f ? a * (1.f / l) : f3{0.f, 0.f, 0.f};
}
__device__ __forceinline__ q4 qnormalize(q4 q) {
  float l = sqrtf(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  if (l > 0.f) {
    float s = 1.f / l;
    return q4{q.w * s, q.x * s, q.y * s, q.z * s};
  }
  return q4{0.f, 0.f, 0.f, 0.f};
}

// math.py:23-30
__device__ __forceinline__ q4 mul_quat(q4 u, q4 v) {
  return q4{u.w * v.w - u.x * v.x - u.y * v.y - u.z * v.z,
            u.w * v.x + u.x * v.w + u.y * v.z - u.z * v.y,
            u.w * v.y - u.x * v.z + u.y * v.w + u.z * v.x,
            u.w * v.z + u.x * v.y - u.y * v.x + u.z * v.w};
}
// math.py:33-38
__device__ __forceinline__ f3 rot_vec_quat(f3 v, q4 q) {
  f3 u{q.x, q.y, q.z};
  float s = q.w;
  f3 r = (2.f * dot(u, v)) * u + (s * s - dot(u, u)) * v;
  return r + (2.f * s) * cross(u, v);
}
// math.py:41-45
__device__ __forceinline__ q4 axis_angle_to_quat(f3 a, float ang) {
  float s, c;
  sincosf(ang * 0.5f, &s, &c);
  return q4{c, a.x * s, a.y * s, a.z * s};
}
// math.py:48-64
__device__ __forceinline__ m33 quat_to_mat(q4 q) {
  float a = q.w, b = q.x, c = q.y, d = q.z;
  m33 r;
  r.m[0] = a * a + b * b - c * c - d * d;
  r.m[1] = 2.f * (b * c - a * d);
  r.m[2] = 2.f * (b * d + a * c);
  r.m[3] = 2.f * (b * c + a * d);
  r.m[4] = a * a - b * b + c * c - d * d;
  r.m[5] = 2.f * (c * d - a * b);
  r.m[6] = 2.f * (b * d - a * c);
  r.m[7] = 2.f * (c * d + a * b);
  r.m[8] = a * a - b * b - c * c + d * d;
  return r;
}
__device__ __forceinline__ f3 mulmv(const m33& a, f3 v) {
  return f3{a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
            a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z};
}
__device__ __forceinline__ f3 col(const m33& a, int j) { return f3{a.m[j], a.m[3 + j], a.m[6 + j]}; }
// math.py:115-128
__device__ __forceinline__ f3 quat_to_vel(q4 q) {
  f3 axis{q.x, q.y, q.z};
  float s = length(axis);
  if (s == 0.f) return f3{0.f, 0.f, 0.f};
  float speed = 2.f * atan2f(s, q.w);
  if (speed > kPi) speed -= 2.f * kPi;
  return axis * (speed / s);
}
// math.py:131-139
__device__ __forceinline__ f3 quat_sub(q4 qa, q4 qb) {
  return quat_to_vel(mul_quat(q4{qb.w, -qb.x, -qb.y, -qb.z}, qa));
}
// math.py:142-152
__device__ __forceinline__ q4 quat_integrate(q4 q, f3 v, float dt) {
  float n = length(v);
  v = normalize(v);
  q4 r = axis_angle_to_quat(v, dt * n);
  return qnormalize(mul_quat(q, r));
}
// math.py:155-180
__device__ __forceinline__ m33 make_frame(f3 a) {
  a = normalize(a);
  f3 b = (-0.5f < a.y && a.y < 0.5f) ? f3{0.f, 1.f, 0.f} : f3{0.f, 0.f, 1.f};
  b = b - a * dot(a, b);
  b = normalize(b);
  if (length(a) == 0.f) b = f3{0.f, 0.f, 0.f};
  f3 c = cross(a, b);
  return m33{{a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z}};
}
// math.py:191-206
__device__ __forceinline__ f3 closest_segment_point(f3 a, f3 b, f3 pt) {
  f3 ab = b - a;
  float t = dot(pt - a, ab) / (dot(ab, ab) + 1e-6f);
  t = fminf(fmaxf(t, 0.f), 1.f);
  return a + t * ab;
}
// math.py:209-242
__device__ __forceinline__ void closest_segment_to_segment_points(f3 a0, f3 a1, f3 b0, f3 b1,
                                                                  f3& pa, f3& pb) {
  f3 da = a1 - a0, db = b1 - b0;
  float la = length(da), lb = length(db);
  f3 dir_a = la == 0.f ? da : da * (1.f / la);
  f3 dir_b = lb == 0.f ? db : db * (1.f / lb);
  float ha = la * 0.5f, hb = lb * 0.5f;
  f3 amid = a0 + dir_a * ha, bmid = b0 + dir_b * hb;
  f3 trans = amid - bmid;
  float dd = dot(dir_a, dir_b), dat = dot(dir_a, trans), dbt = dot(dir_b, trans);
  float denom = 1.f - dd * dd;
  float ta0 = (-dat + dd * dbt) / (denom + 1e-6f);
  float tb0 = dbt + ta0 * dd;
  float ta = fminf(fmaxf(ta0, -ha), ha);
  float tb = fminf(fmaxf(tb0, -hb), hb);
  f3 best_a = amid + dir_a * ta, best_b = bmid + dir_b * tb;
  f3 na = closest_segment_point(a0, a1, best_b);
  f3 nb = closest_segment_point(b0, b1, best_a);
  float d1 = dot(best_b - na, best_b - na), d2 = dot(best_a - nb, best_a - nb);
  if (d1 < d2) {
    pa = na;
    pb = best_b;
  } else {
    pa = best_a;
    pb = nb;
  }
}

// spatial algebra ---------------------------------------------------------------------------

struct s6 {
  float v[6];
};
__device__ __forceinline__ s6 ld6(const float* p) {
  s6 r;
#pragma unroll
  for (int i = 0; i < 6; i++) r.v[i] = p[i];
  return r;
}
__device__ __forceinline__ void st6(float* p, const s6& r) {
#pragma unroll
  for (int i = 0; i < 6; i++) p[i] = r.v[i];
}
__device__ __forceinline__ float dot6(const s6& a, const s6& b) {
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 6; i++) s += a.v[i] * b.v[i];
  return s;
}
// math.py:72-82 (mju_mulInertVec)
__device__ __forceinline__ s6 inert_vec(const float* i, const s6& v) {
  s6 r;
  r.v[0] = i[0] * v.v[0] + i[3] * v.v[1] + i[4] * v.v[2] - i[8] * v.v[4] + i[7] * v.v[5];
  r.v[1] = i[3] * v.v[0] + i[1] * v.v[1] + i[5] * v.v[2] + i[8] * v.v[3] - i[6] * v.v[5];
  r.v[2] = i[4] * v.v[0] + i[5] * v.v[1] + i[2] * v.v[2] - i[7] * v.v[3] + i[6] * v.v[4];
  r.v[3] = i[8] * v.v[1] - i[7] * v.v[2] + i[9] * v.v[3];
  r.v[4] = i[6] * v.v[2] - i[8] * v.v[0] + i[9] * v.v[4];
  r.v[5] = i[7] * v.v[0] - i[6] * v.v[1] + i[9] * v.v[5];
  return r;
}
// math.py:85-97
__device__ __forceinline__ s6 motion_cross(const s6& u, const s6& v) {
  f3 u0{u.v[0], u.v[1], u.v[2]}, u1{u.v[3], u.v[4], u.v[5]};
  f3 v0{v.v[0], v.v[1], v.v[2]}, v1{v.v[3], v.v[4], v.v[5]};
  f3 a = cross(u0, v0), b = cross(u1, v0) + cross(u0, v1);
  return s6{{a.x, a.y, a.z, b.x, b.y, b.z}};
}
// math.py:100-112
__device__ __forceinline__ s6 motion_cross_force(const s6& v, const s6& f) {
  f3 v0{v.v[0], v.v[1], v.v[2]}, v1{v.v[3], v.v[4], v.v[5]};
  f3 f0{f.v[0], f.v[1], f.v[2]}, f1{f.v[3], f.v[4], f.v[5]};
  f3 a = cross(v0, f0) + cross(v1, f1), b = cross(v0, f1);
  return s6{{a.x, a.y, a.z, b.x, b.y, b.z}};
}

// warp collectives ------------------------------------------------------------------------------

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum_t(float v) { return warp_sum(v); }
__device__ __forceinline__ double warp_sum_t(double v) { return warp_sum_d(v); }
__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// exclusive prefix sum of v over the warp's lanes; total returned in *total
__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

}  // namespace mjb
