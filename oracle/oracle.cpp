// ORACLE — test infrastructure only.
//
// CPU restatement of the reference's batched physics step (mujoco_warp/_src/*.py), one world at a
// time, templated on the scalar type: float mode follows the reference's FP32 arithmetic, double
// mode stands in for an FP64 evaluation of the same algorithm.  It is the checker for the CUDA
// path (tests/, __graft_entry__.smoke()) and the timed CPU baseline of bench.py; the product
// never links, imports or calls it.
//
// Parity: only the reference tests' known-answer vectors (math_test.py, broad_phase_test.py,
// forward_test.py:130-145) pin this restatement; everything the reference compares against
// MuJoCo C is unpinned here because neither MuJoCo nor Warp can run in this environment.
//
// Canonical ordering (the reference orders contacts / efc rows by global atomics,
// collision_primitive.py:64, constraint.py:119,162): per world, limit rows in
// jnt_limited_slide_hinge_adr order, then contact rows in contact order, 4 pyramid edges each;
// contacts in broadphase pair order (g1 < g2 lexicographic, collision_driver.py:465-478), then
// contact index within the pair.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Host description of a compiled model (all float arrays are float64, int arrays int32).
// Field names follow mujoco_warp/_src/types.py:366-612.
typedef struct OracleModelDesc {
  int nq, nv, na, nu, nbody, njnt, ngeom, nsite, nmocap, nlimit, nlevel, nblock;
  int integrator, cone, solver, iterations, ls_iterations, disableflags, ls_parallel, nlsp;
  int actuator_affine_bias_gain;
  double timestep, impratio, tolerance, ls_tolerance, meaninertia;
  double gravity[3];
  const int *body_tree, *body_treeadr, *body_parentid, *body_rootid, *body_weldid, *body_jntnum,
      *body_jntadr, *body_dofnum, *body_dofadr;
  const double *body_pos, *body_quat, *body_ipos, *body_iquat, *body_mass, *subtree_mass,
      *body_inertia, *body_invweight0;
  const int *jnt_type, *jnt_qposadr, *jnt_dofadr, *jnt_bodyid, *jnt_limited, *jnt_actfrclimited,
      *jnt_limited_slide_hinge_adr;
  const double *jnt_solref, *jnt_solimp, *jnt_pos, *jnt_axis, *jnt_stiffness, *jnt_range,
      *jnt_actfrcrange, *jnt_margin;
  const int *dof_bodyid, *dof_jntid, *dof_parentid;
  const double *dof_armature, *dof_damping, *dof_invweight0;
  const int *block_adr, *block_size;
  const int *geom_type, *geom_contype, *geom_conaffinity, *geom_condim, *geom_bodyid,
      *geom_priority;
  const double *geom_pos, *geom_quat, *geom_size, *geom_rbound, *geom_solmix, *geom_solref,
      *geom_solimp, *geom_friction, *geom_margin, *geom_gap;
  const int* site_bodyid;
  const double *site_pos, *site_quat;
  const int *actuator_trntype, *actuator_dyntype, *actuator_gaintype, *actuator_biastype,
      *actuator_trnid, *actuator_actadr, *actuator_ctrllimited, *actuator_forcelimited,
      *actuator_actlimited;
  const double *actuator_dynprm, *actuator_gainprm, *actuator_biasprm, *actuator_ctrlrange,
      *actuator_forcerange, *actuator_actrange, *actuator_gear;
  const double *qpos0, *qpos_spring;
} OracleModelDesc;
}

namespace {

constexpr double kMinVal = 1e-15;   // mjMINVAL
constexpr double kMinImp = 0.0001;  // mjMINIMP
constexpr double kMaxImp = 0.9999;  // mjMAXIMP

enum { JNT_FREE = 0, JNT_BALL = 1, JNT_SLIDE = 2, JNT_HINGE = 3 };
enum { GEOM_PLANE = 0, GEOM_SPHERE = 2, GEOM_CAPSULE = 3, GEOM_BOX = 6 };
enum {
  DSBL_CONSTRAINT = 1 << 0, DSBL_LIMIT = 1 << 3, DSBL_CONTACT = 1 << 4, DSBL_PASSIVE = 1 << 5,
  DSBL_GRAVITY = 1 << 6, DSBL_CLAMPCTRL = 1 << 7, DSBL_FILTERPARENT = 1 << 9,
  DSBL_ACTUATION = 1 << 10, DSBL_REFSAFE = 1 << 11, DSBL_EULERDAMP = 1 << 14
};

template <typename T>
struct V3 {
  T x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(T a, T b, T c) : x(a), y(b), z(c) {}
  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <typename T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> V3<T> operator*(T s, V3<T> a) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename T> T length(V3<T> a) { return std::sqrt(dot(a, a)); }
// warp's normalize: zero vector stays zero
template <typename T> V3<T> normalize(V3<T> a) {
  T l = length(a);
  return l > T(0) ? a * (T(1) / l) : V3<T>();
}

template <typename T>
struct Q4 {
  T w, x, y, z;
};
template <typename T> Q4<T> qnormalize(Q4<T> q) {
  T l = std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  if (l > T(0)) { T s = T(1) / l; return {q.w * s, q.x * s, q.y * s, q.z * s}; }
  return {T(0), T(0), T(0), T(0)};
}
// math.py:23-30
template <typename T> Q4<T> mul_quat(Q4<T> u, Q4<T> v) {
  return {u.w * v.w - u.x * v.x - u.y * v.y - u.z * v.z,
          u.w * v.x + u.x * v.w + u.y * v.z - u.z * v.y,
          u.w * v.y - u.x * v.z + u.y * v.w + u.z * v.x,
          u.w * v.z + u.x * v.y - u.y * v.x + u.z * v.w};
}
// math.py:33-38
template <typename T> V3<T> rot_vec_quat(V3<T> v, Q4<T> q) {
  V3<T> u(q.x, q.y, q.z);
  T s = q.w;
  V3<T> r = (T(2) * dot(u, v)) * u + (s * s - dot(u, u)) * v;
  return r + (T(2) * s) * cross(u, v);
}
// math.py:41-45
template <typename T> Q4<T> axis_angle_to_quat(V3<T> a, T ang) {
  T s = std::sin(ang * T(0.5)), c = std::cos(ang * T(0.5));
  return {c, a.x * s, a.y * s, a.z * s};
}
template <typename T>
struct M3 {
  T m[9];
  T& operator()(int i, int j) { return m[3 * i + j]; }
  T operator()(int i, int j) const { return m[3 * i + j]; }
  V3<T> col(int j) const { return {m[j], m[3 + j], m[6 + j]}; }
  V3<T> row(int i) const { return {m[3 * i], m[3 * i + 1], m[3 * i + 2]}; }
};
template <typename T> V3<T> mulmv(const M3<T>& a, V3<T> v) {
  return {a(0, 0) * v.x + a(0, 1) * v.y + a(0, 2) * v.z, a(1, 0) * v.x + a(1, 1) * v.y + a(1, 2) * v.z,
          a(2, 0) * v.x + a(2, 1) * v.y + a(2, 2) * v.z};
}
// math.py:48-64
template <typename T> M3<T> quat_to_mat(Q4<T> q) {
  T a = q.w, b = q.x, c = q.y, d = q.z;
  M3<T> r;
  r.m[0] = a * a + b * b - c * c - d * d;
  r.m[1] = T(2) * (b * c - a * d);
  r.m[2] = T(2) * (b * d + a * c);
  r.m[3] = T(2) * (b * c + a * d);
  r.m[4] = a * a - b * b + c * c - d * d;
  r.m[5] = T(2) * (c * d - a * b);
  r.m[6] = T(2) * (b * d - a * c);
  r.m[7] = T(2) * (c * d + a * b);
  r.m[8] = a * a - b * b - c * c + d * d;
  return r;
}
// math.py:115-128
template <typename T> V3<T> quat_to_vel(Q4<T> q) {
  V3<T> axis(q.x, q.y, q.z);
  T s = length(axis);
  if (s == T(0)) return V3<T>();
  T speed = T(2) * std::atan2(s, q.w);
  if (speed > T(M_PI)) speed -= T(2 * M_PI);
  return axis * (speed / s);
}
// math.py:131-139
template <typename T> V3<T> quat_sub(Q4<T> qa, Q4<T> qb) {
  Q4<T> qneg{qb.w, -qb.x, -qb.y, -qb.z};
  return quat_to_vel(mul_quat(qneg, qa));
}
// math.py:142-152
template <typename T> Q4<T> quat_integrate(Q4<T> q, V3<T> v, T dt) {
  T n = length(v);
  v = normalize(v);
  T ang = dt * n;
  Q4<T> r = axis_angle_to_quat(v, ang);
  return qnormalize(mul_quat(q, r));
}
// math.py:155-180
template <typename T> M3<T> make_frame(V3<T> a) {
  a = normalize(a);
  V3<T> b = (T(-0.5) < a.y && a.y < T(0.5)) ? V3<T>(0, 1, 0) : V3<T>(0, 0, 1);
  b = b - a * dot(a, b);
  b = normalize(b);
  if (length(a) == T(0)) b = V3<T>();
  V3<T> c = cross(a, b);
  M3<T> f;
  f.m[0] = a.x; f.m[1] = a.y; f.m[2] = a.z;
  f.m[3] = b.x; f.m[4] = b.y; f.m[5] = b.z;
  f.m[6] = c.x; f.m[7] = c.y; f.m[8] = c.z;
  return f;
}
// math.py:191-206
template <typename T> V3<T> closest_segment_point(V3<T> a, V3<T> b, V3<T> pt) {
  V3<T> ab = b - a;
  T t = dot(pt - a, ab) / (dot(ab, ab) + T(1e-6));
  t = std::min(std::max(t, T(0)), T(1));
  return a + t * ab;
}
// math.py:209-242
template <typename T>
void closest_segment_to_segment_points(V3<T> a0, V3<T> a1, V3<T> b0, V3<T> b1, V3<T>& pa,
                                       V3<T>& pb) {
  V3<T> da = a1 - a0, db = b1 - b0;
  T la = length(da), lb = length(db);
  V3<T> dir_a = la == T(0) ? da : da * (T(1) / la);
  V3<T> dir_b = lb == T(0) ? db : db * (T(1) / lb);
  T ha = la * T(0.5), hb = lb * T(0.5);
  V3<T> amid = a0 + dir_a * ha, bmid = b0 + dir_b * hb;
  V3<T> trans = amid - bmid;
  T dd = dot(dir_a, dir_b), dat = dot(dir_a, trans), dbt = dot(dir_b, trans);
  T denom = T(1) - dd * dd;
  T ta0 = (-dat + dd * dbt) / (denom + T(1e-6));
  T tb0 = dbt + ta0 * dd;
  T ta = std::min(std::max(ta0, -ha), ha);
  T tb = std::min(std::max(tb0, -hb), hb);
  V3<T> best_a = amid + dir_a * ta, best_b = bmid + dir_b * tb;
  V3<T> na = closest_segment_point(a0, a1, best_b);
  V3<T> nb = closest_segment_point(b0, b1, best_a);
  T d1 = dot(best_b - na, best_b - na), d2 = dot(best_a - nb, best_a - nb);
  if (d1 < d2) { pa = na; pb = best_b; } else { pa = best_a; pb = nb; }
}

template <typename T> using S6 = std::array<T, 6>;

// math.py:72-82  (mju_mulInertVec)
template <typename T> S6<T> inert_vec(const T* i, const S6<T>& v) {
  return {i[0] * v[0] + i[3] * v[1] + i[4] * v[2] - i[8] * v[4] + i[7] * v[5],
          i[3] * v[0] + i[1] * v[1] + i[5] * v[2] + i[8] * v[3] - i[6] * v[5],
          i[4] * v[0] + i[5] * v[1] + i[2] * v[2] - i[7] * v[3] + i[6] * v[4],
          i[8] * v[1] - i[7] * v[2] + i[9] * v[3],
          i[6] * v[2] - i[8] * v[0] + i[9] * v[4],
          i[7] * v[0] - i[6] * v[1] + i[9] * v[5]};
}
// math.py:85-97
template <typename T> S6<T> motion_cross(const S6<T>& u, const S6<T>& v) {
  V3<T> u0(u[0], u[1], u[2]), u1(u[3], u[4], u[5]), v0(v[0], v[1], v[2]), v1(v[3], v[4], v[5]);
  V3<T> a = cross(u0, v0), b = cross(u1, v0) + cross(u0, v1);
  return {a.x, a.y, a.z, b.x, b.y, b.z};
}
// math.py:100-112
template <typename T> S6<T> motion_cross_force(const S6<T>& v, const S6<T>& f) {
  V3<T> v0(v[0], v[1], v[2]), v1(v[3], v[4], v[5]), f0(f[0], f[1], f[2]), f1(f[3], f[4], f[5]);
  V3<T> a = cross(v0, f0) + cross(v1, f1), b = cross(v0, f1);
  return {a.x, a.y, a.z, b.x, b.y, b.z};
}
template <typename T> T dot6(const T* a, const S6<T>& b) {
  T s = 0;
  for (int i = 0; i < 6; i++) s += a[i] * b[i];
  return s;
}

template <typename T>
std::vector<T> cvt(const double* p, size_t n) {
  std::vector<T> v(n);
  for (size_t i = 0; i < n; i++) v[i] = T(p[i]);
  return v;
}
std::vector<int> cvti(const int* p, size_t n) { return std::vector<int>(p, p + n); }

template <typename T>
struct Model {
  int nq, nv, na, nu, nbody, njnt, ngeom, nsite, nmocap, nlimit, nlevel, nblock;
  int integrator, cone, solver, iterations, ls_iterations, disableflags, ls_parallel, nlsp;
  bool affine;
  T timestep, impratio, tolerance, ls_tolerance, meaninertia;
  V3<T> gravity;
  std::vector<int> body_tree, body_treeadr, body_parentid, body_rootid, body_weldid, body_jntnum,
      body_jntadr, body_dofnum, body_dofadr;
  std::vector<T> body_pos, body_quat, body_ipos, body_iquat, body_mass, subtree_mass,
      body_inertia, body_invweight0;
  std::vector<int> jnt_type, jnt_qposadr, jnt_dofadr, jnt_bodyid, jnt_limited,
      jnt_actfrclimited, jnt_limited_slide_hinge_adr;
  std::vector<T> jnt_solref, jnt_solimp, jnt_pos, jnt_axis, jnt_stiffness, jnt_range,
      jnt_actfrcrange, jnt_margin;
  std::vector<int> dof_bodyid, dof_jntid, dof_parentid;
  std::vector<T> dof_armature, dof_damping, dof_invweight0;
  std::vector<int> block_adr, block_size;
  std::vector<int> geom_type, geom_contype, geom_conaffinity, geom_condim, geom_bodyid,
      geom_priority;
  std::vector<T> geom_pos, geom_quat, geom_size, geom_rbound, geom_solmix, geom_solref,
      geom_solimp, geom_friction, geom_margin, geom_gap;
  std::vector<int> site_bodyid;
  std::vector<T> site_pos, site_quat;
  std::vector<int> actuator_trntype, actuator_dyntype, actuator_gaintype, actuator_biastype,
      actuator_trnid, actuator_actadr, actuator_ctrllimited, actuator_forcelimited,
      actuator_actlimited;
  std::vector<T> actuator_dynprm, actuator_gainprm, actuator_biasprm, actuator_ctrlrange,
      actuator_forcerange, actuator_actrange, actuator_gear;
  std::vector<T> qpos0, qpos_spring;
  std::vector<T> alpha_candidate;

  explicit Model(const OracleModelDesc& d) {
    nq = d.nq; nv = d.nv; na = d.na; nu = d.nu; nbody = d.nbody; njnt = d.njnt; ngeom = d.ngeom;
    nsite = d.nsite; nmocap = d.nmocap; nlimit = d.nlimit; nlevel = d.nlevel; nblock = d.nblock;
    integrator = d.integrator; cone = d.cone; solver = d.solver; iterations = d.iterations;
    ls_iterations = d.ls_iterations; disableflags = d.disableflags; ls_parallel = d.ls_parallel;
    nlsp = d.nlsp; affine = d.actuator_affine_bias_gain != 0;
    timestep = T(d.timestep); impratio = T(d.impratio); tolerance = T(d.tolerance);
    ls_tolerance = T(d.ls_tolerance); meaninertia = T(d.meaninertia);
    gravity = V3<T>(T(d.gravity[0]), T(d.gravity[1]), T(d.gravity[2]));
    int nb = nbody, nj = njnt, ng = ngeom;
    body_tree = cvti(d.body_tree, nb); body_treeadr = cvti(d.body_treeadr, nlevel + 1);
    body_parentid = cvti(d.body_parentid, nb); body_rootid = cvti(d.body_rootid, nb);
    body_weldid = cvti(d.body_weldid, nb); body_jntnum = cvti(d.body_jntnum, nb);
    body_jntadr = cvti(d.body_jntadr, nb); body_dofnum = cvti(d.body_dofnum, nb);
    body_dofadr = cvti(d.body_dofadr, nb);
    body_pos = cvt<T>(d.body_pos, 3 * nb); body_quat = cvt<T>(d.body_quat, 4 * nb);
    body_ipos = cvt<T>(d.body_ipos, 3 * nb); body_iquat = cvt<T>(d.body_iquat, 4 * nb);
    body_mass = cvt<T>(d.body_mass, nb); subtree_mass = cvt<T>(d.subtree_mass, nb);
    body_inertia = cvt<T>(d.body_inertia, 3 * nb);
    body_invweight0 = cvt<T>(d.body_invweight0, 2 * nb);
    jnt_type = cvti(d.jnt_type, nj); jnt_qposadr = cvti(d.jnt_qposadr, nj);
    jnt_dofadr = cvti(d.jnt_dofadr, nj); jnt_bodyid = cvti(d.jnt_bodyid, nj);
    jnt_limited = cvti(d.jnt_limited, nj); jnt_actfrclimited = cvti(d.jnt_actfrclimited, nj);
    jnt_limited_slide_hinge_adr = cvti(d.jnt_limited_slide_hinge_adr, nlimit);
    jnt_solref = cvt<T>(d.jnt_solref, 2 * nj); jnt_solimp = cvt<T>(d.jnt_solimp, 5 * nj);
    jnt_pos = cvt<T>(d.jnt_pos, 3 * nj); jnt_axis = cvt<T>(d.jnt_axis, 3 * nj);
    jnt_stiffness = cvt<T>(d.jnt_stiffness, nj); jnt_range = cvt<T>(d.jnt_range, 2 * nj);
    jnt_actfrcrange = cvt<T>(d.jnt_actfrcrange, 2 * nj); jnt_margin = cvt<T>(d.jnt_margin, nj);
    dof_bodyid = cvti(d.dof_bodyid, nv); dof_jntid = cvti(d.dof_jntid, nv);
    dof_parentid = cvti(d.dof_parentid, nv);
    dof_armature = cvt<T>(d.dof_armature, nv); dof_damping = cvt<T>(d.dof_damping, nv);
    dof_invweight0 = cvt<T>(d.dof_invweight0, nv);
    block_adr = cvti(d.block_adr, nblock); block_size = cvti(d.block_size, nblock);
    geom_type = cvti(d.geom_type, ng); geom_contype = cvti(d.geom_contype, ng);
    geom_conaffinity = cvti(d.geom_conaffinity, ng); geom_condim = cvti(d.geom_condim, ng);
    geom_bodyid = cvti(d.geom_bodyid, ng); geom_priority = cvti(d.geom_priority, ng);
    geom_pos = cvt<T>(d.geom_pos, 3 * ng); geom_quat = cvt<T>(d.geom_quat, 4 * ng);
    geom_size = cvt<T>(d.geom_size, 3 * ng); geom_rbound = cvt<T>(d.geom_rbound, ng);
    geom_solmix = cvt<T>(d.geom_solmix, ng); geom_solref = cvt<T>(d.geom_solref, 2 * ng);
    geom_solimp = cvt<T>(d.geom_solimp, 5 * ng); geom_friction = cvt<T>(d.geom_friction, 3 * ng);
    geom_margin = cvt<T>(d.geom_margin, ng); geom_gap = cvt<T>(d.geom_gap, ng);
    site_bodyid = cvti(d.site_bodyid, nsite);
    site_pos = cvt<T>(d.site_pos, 3 * nsite); site_quat = cvt<T>(d.site_quat, 4 * nsite);
    actuator_trntype = cvti(d.actuator_trntype, nu); actuator_dyntype = cvti(d.actuator_dyntype, nu);
    actuator_gaintype = cvti(d.actuator_gaintype, nu);
    actuator_biastype = cvti(d.actuator_biastype, nu);
    actuator_trnid = cvti(d.actuator_trnid, 2 * nu); actuator_actadr = cvti(d.actuator_actadr, nu);
    actuator_ctrllimited = cvti(d.actuator_ctrllimited, nu);
    actuator_forcelimited = cvti(d.actuator_forcelimited, nu);
    actuator_actlimited = cvti(d.actuator_actlimited, nu);
    actuator_dynprm = cvt<T>(d.actuator_dynprm, 10 * nu);
    actuator_gainprm = cvt<T>(d.actuator_gainprm, 10 * nu);
    actuator_biasprm = cvt<T>(d.actuator_biasprm, 10 * nu);
    actuator_ctrlrange = cvt<T>(d.actuator_ctrlrange, 2 * nu);
    actuator_forcerange = cvt<T>(d.actuator_forcerange, 2 * nu);
    actuator_actrange = cvt<T>(d.actuator_actrange, 2 * nu);
    actuator_gear = cvt<T>(d.actuator_gear, 6 * nu);
    qpos0 = cvt<T>(d.qpos0, nq); qpos_spring = cvt<T>(d.qpos_spring, nq);
    alpha_candidate.resize(std::max(nlsp, 0));
    for (int i = 0; i < nlsp; i++)
      alpha_candidate[i] = nlsp > 1 ? T(double(i) / double(nlsp - 1)) : T(0);  // io.py:233
  }
  V3<T> v3(const std::vector<T>& a, int i) const { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
  Q4<T> q4(const std::vector<T>& a, int i) const {
    return {a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]};
  }
};

// Per-world state and intermediates (the reference's Data fields for one world).
template <typename T>
struct World {
  // state
  std::vector<T> qpos, qvel, act, ctrl, qacc, qacc_warmstart, qfrc_applied, xfrc_applied;
  // position / velocity stages
  std::vector<T> xpos, xquat, xmat, xipos, ximat, xanchor, xaxis, geom_xpos, geom_xmat, site_xpos,
      site_xmat, subtree_com, cinert, crb, cdof, cvel, cdof_dot, qM, qLD, qLDiagInv,
      actuator_length, actuator_velocity, actuator_force, actuator_moment, qfrc_bias, qfrc_spring,
      qfrc_damper, qfrc_passive, qfrc_actuator, qfrc_smooth, qfrc_constraint, qacc_smooth,
      act_dot, rne_cacc, rne_cfrc, qacc_integration;
  // collision: pairs and contacts
  std::vector<int> pair;  // 2 per pair
  std::vector<T> con_dist, con_pos, con_frame, con_includemargin, con_friction, con_solref,
      con_solimp;
  std::vector<int> con_dim, con_geom;
  // constraints
  std::vector<T> efc_J, efc_pos, efc_margin, efc_D, efc_aref, efc_force, efc_Jaref;
  std::vector<int> efc_active;
  // solver
  std::vector<T> Ma, grad, Mgrad, search, mv, jv, quad, h;
  T grad_dot = 0, search_dot = 0, gauss = 0, cost = 0, prev_cost = 0, gtol = 0, alpha = 0;
  T quad_gauss[3] = {0, 0, 0};
  int solver_niter = 0;
  int iters_run = 0;
  bool done = false;
  std::vector<T> prev_grad, prev_Mgrad;
  T beta = 0;

  int ncon() const { return int(con_dist.size()); }
  int nefc() const { return int(efc_D.size()); }
  int npair() const { return int(pair.size() / 2); }

  void init(const Model<T>& m) {
    int nv = m.nv, nb = m.nbody, nj = m.njnt, ng = m.ngeom, ns = m.nsite, nu = m.nu;
    qpos.assign(m.qpos0.begin(), m.qpos0.end());
    qvel.assign(nv, 0); act.assign(m.na, 0); ctrl.assign(nu, 0); qacc.assign(nv, 0);
    qacc_warmstart.assign(nv, 0); qfrc_applied.assign(nv, 0); xfrc_applied.assign(6 * nb, 0);
    xpos.assign(3 * nb, 0); xquat.assign(4 * nb, 0); xmat.assign(9 * nb, 0);
    xipos.assign(3 * nb, 0); ximat.assign(9 * nb, 0); xanchor.assign(3 * nj, 0);
    xaxis.assign(3 * nj, 0); geom_xpos.assign(3 * ng, 0); geom_xmat.assign(9 * ng, 0);
    site_xpos.assign(3 * ns, 0); site_xmat.assign(9 * ns, 0); subtree_com.assign(3 * nb, 0);
    cinert.assign(10 * nb, 0); crb.assign(10 * nb, 0); cdof.assign(6 * nv, 0);
    cvel.assign(6 * nb, 0); cdof_dot.assign(6 * nv, 0); qM.assign(nv * nv, 0);
    qLD.assign(nv * nv, 0); qLDiagInv.assign(nv, 0); actuator_length.assign(nu, 0);
    actuator_velocity.assign(nu, 0); actuator_force.assign(nu, 0);
    actuator_moment.assign(nu * nv, 0); qfrc_bias.assign(nv, 0); qfrc_spring.assign(nv, 0);
    qfrc_damper.assign(nv, 0); qfrc_passive.assign(nv, 0); qfrc_actuator.assign(nv, 0);
    qfrc_smooth.assign(nv, 0); qfrc_constraint.assign(nv, 0); qacc_smooth.assign(nv, 0);
    act_dot.assign(m.na, 0); rne_cacc.assign(6 * nb, 0); rne_cfrc.assign(6 * nb, 0);
    qacc_integration.assign(nv, 0);
    Ma.assign(nv, 0); grad.assign(nv, 0); Mgrad.assign(nv, 0); search.assign(nv, 0);
    mv.assign(nv, 0); h.assign(nv * nv, 0); prev_grad.assign(nv, 0); prev_Mgrad.assign(nv, 0);
  }
};

// ------------------------------------------------------------------------------------------
// smooth.py

// smooth.py:32-145
template <typename T>
void kinematics(const Model<T>& m, World<T>& w) {
  // _root (smooth.py:37-43)
  w.xpos[0] = w.xpos[1] = w.xpos[2] = 0;
  w.xquat[0] = 1; w.xquat[1] = w.xquat[2] = w.xquat[3] = 0;
  w.xipos[0] = w.xipos[1] = w.xipos[2] = 0;
  for (int i = 0; i < 9; i++) w.xmat[i] = w.ximat[i] = (i % 4 == 0) ? T(1) : T(0);
  // _level for each BFS level (smooth.py:46-109)
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    for (int n = m.body_treeadr[lvl]; n < m.body_treeadr[lvl + 1]; n++) {
      int b = m.body_tree[n];
      int jntadr = m.body_jntadr[b], jntnum = m.body_jntnum[b];
      V3<T> xpos;
      Q4<T> xquat;
      if (jntnum == 1 && m.jnt_type[jntadr] == JNT_FREE) {
        int a = m.jnt_qposadr[jntadr];
        xpos = V3<T>(w.qpos[a], w.qpos[a + 1], w.qpos[a + 2]);
        xquat = Q4<T>{w.qpos[a + 3], w.qpos[a + 4], w.qpos[a + 5], w.qpos[a + 6]};
        for (int k = 0; k < 3; k++) {
          w.xanchor[3 * jntadr + k] = xpos[k];
          w.xaxis[3 * jntadr + k] = m.jnt_axis[3 * jntadr + k];
        }
      } else {
        int p = m.body_parentid[b];
        M3<T> pm;
        std::memcpy(pm.m, &w.xmat[9 * p], sizeof(pm.m));
        V3<T> ppos(w.xpos[3 * p], w.xpos[3 * p + 1], w.xpos[3 * p + 2]);
        xpos = mulmv(pm, m.v3(m.body_pos, b)) + ppos;
        xquat = mul_quat(Q4<T>{w.xquat[4 * p], w.xquat[4 * p + 1], w.xquat[4 * p + 2], w.xquat[4 * p + 3]},
                         m.q4(m.body_quat, b));
        for (int j = jntadr; j < jntadr + jntnum; j++) {
          int a = m.jnt_qposadr[j];
          int t = m.jnt_type[j];
          V3<T> jaxis = m.v3(m.jnt_axis, j), jpos = m.v3(m.jnt_pos, j);
          V3<T> xanchor = rot_vec_quat(jpos, xquat) + xpos;
          V3<T> xaxis = rot_vec_quat(jaxis, xquat);
          if (t == JNT_BALL) {
            Q4<T> qloc{w.qpos[a], w.qpos[a + 1], w.qpos[a + 2], w.qpos[a + 3]};
            xquat = mul_quat(xquat, qloc);
            xpos = xanchor - rot_vec_quat(jpos, xquat);
          } else if (t == JNT_SLIDE) {
            xpos = xpos + xaxis * (w.qpos[a] - m.qpos0[a]);
          } else if (t == JNT_HINGE) {
            Q4<T> qloc = axis_angle_to_quat(jaxis, w.qpos[a] - m.qpos0[a]);
            xquat = mul_quat(xquat, qloc);
            xpos = xanchor - rot_vec_quat(jpos, xquat);
          }
          for (int k = 0; k < 3; k++) {
            w.xanchor[3 * j + k] = xanchor[k];
            w.xaxis[3 * j + k] = xaxis[k];
          }
        }
      }
      for (int k = 0; k < 3; k++) w.xpos[3 * b + k] = xpos[k];
      xquat = qnormalize(xquat);
      w.xquat[4 * b] = xquat.w; w.xquat[4 * b + 1] = xquat.x;
      w.xquat[4 * b + 2] = xquat.y; w.xquat[4 * b + 3] = xquat.z;
      M3<T> xm = quat_to_mat(xquat);
      std::memcpy(&w.xmat[9 * b], xm.m, sizeof(xm.m));
      V3<T> xipos = xpos + rot_vec_quat(m.v3(m.body_ipos, b), xquat);
      for (int k = 0; k < 3; k++) w.xipos[3 * b + k] = xipos[k];
      M3<T> xim = quat_to_mat(mul_quat(xquat, m.q4(m.body_iquat, b)));
      std::memcpy(&w.ximat[9 * b], xim.m, sizeof(xim.m));
    }
  }
  // geom_local_to_global / site_local_to_global (smooth.py:111-131)
  for (int g = 0; g < m.ngeom; g++) {
    int b = m.geom_bodyid[g];
    Q4<T> q{w.xquat[4 * b], w.xquat[4 * b + 1], w.xquat[4 * b + 2], w.xquat[4 * b + 3]};
    V3<T> p = V3<T>(w.xpos[3 * b], w.xpos[3 * b + 1], w.xpos[3 * b + 2]) +
              rot_vec_quat(m.v3(m.geom_pos, g), q);
    for (int k = 0; k < 3; k++) w.geom_xpos[3 * g + k] = p[k];
    M3<T> r = quat_to_mat(mul_quat(q, m.q4(m.geom_quat, g)));
    std::memcpy(&w.geom_xmat[9 * g], r.m, sizeof(r.m));
  }
  for (int s = 0; s < m.nsite; s++) {
    int b = m.site_bodyid[s];
    Q4<T> q{w.xquat[4 * b], w.xquat[4 * b + 1], w.xquat[4 * b + 2], w.xquat[4 * b + 3]};
    V3<T> p = V3<T>(w.xpos[3 * b], w.xpos[3 * b + 1], w.xpos[3 * b + 2]) +
              rot_vec_quat(m.v3(m.site_pos, s), q);
    for (int k = 0; k < 3; k++) w.site_xpos[3 * s + k] = p[k];
    M3<T> r = quat_to_mat(mul_quat(q, m.q4(m.site_quat, s)));
    std::memcpy(&w.site_xmat[9 * s], r.m, sizeof(r.m));
  }
}

// smooth.py:148-245
template <typename T>
void com_pos(const Model<T>& m, World<T>& w) {
  int nb = m.nbody;
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < 3; k++) w.subtree_com[3 * b + k] = w.xipos[3 * b + k] * m.body_mass[b];
  // reverse levels, including level 0 which adds the world into itself (smooth.py:238-241)
  for (int lvl = m.nlevel - 1; lvl >= 0; lvl--) {
    for (int n = m.body_treeadr[lvl]; n < m.body_treeadr[lvl + 1]; n++) {
      int b = m.body_tree[n], p = m.body_parentid[b];
      T v[3] = {w.subtree_com[3 * b], w.subtree_com[3 * b + 1], w.subtree_com[3 * b + 2]};
      for (int k = 0; k < 3; k++) w.subtree_com[3 * p + k] += v[k];
    }
  }
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < 3; k++) w.subtree_com[3 * b + k] /= m.subtree_mass[b];
  // cinert (smooth.py:169-201)
  for (int b = 0; b < nb; b++) {
    M3<T> mat;
    std::memcpy(mat.m, &w.ximat[9 * b], sizeof(mat.m));
    V3<T> inert = m.v3(m.body_inertia, b);
    T mass = m.body_mass[b];
    int r = m.body_rootid[b];
    V3<T> dif(w.xipos[3 * b] - w.subtree_com[3 * r], w.xipos[3 * b + 1] - w.subtree_com[3 * r + 1],
              w.xipos[3 * b + 2] - w.subtree_com[3 * r + 2]);
    T tmp[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        T s = 0;
        for (int k = 0; k < 3; k++) s += mat(i, k) * inert[k] * mat(j, k);
        tmp[i][j] = s;
      }
    T* res = &w.cinert[10 * b];
    res[0] = tmp[0][0] + mass * (dif.y * dif.y + dif.z * dif.z);
    res[1] = tmp[1][1] + mass * (dif.x * dif.x + dif.z * dif.z);
    res[2] = tmp[2][2] + mass * (dif.x * dif.x + dif.y * dif.y);
    res[3] = tmp[0][1] - mass * dif.x * dif.y;
    res[4] = tmp[0][2] - mass * dif.x * dif.z;
    res[5] = tmp[1][2] - mass * dif.y * dif.z;
    res[6] = mass * dif.x;
    res[7] = mass * dif.y;
    res[8] = mass * dif.z;
    res[9] = mass;
  }
  // cdof (smooth.py:203-232)
  for (int j = 0; j < m.njnt; j++) {
    int b = m.jnt_bodyid[j], d = m.jnt_dofadr[j], t = m.jnt_type[j], r = m.body_rootid[b];
    V3<T> xaxis(w.xaxis[3 * j], w.xaxis[3 * j + 1], w.xaxis[3 * j + 2]);
    M3<T> xm;
    std::memcpy(xm.m, &w.xmat[9 * b], sizeof(xm.m));
    V3<T> off(w.subtree_com[3 * r] - w.xanchor[3 * j], w.subtree_com[3 * r + 1] - w.xanchor[3 * j + 1],
              w.subtree_com[3 * r + 2] - w.xanchor[3 * j + 2]);
    auto put = [&](int dof, V3<T> a, V3<T> l) {
      T* c = &w.cdof[6 * dof];
      c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = l.x; c[4] = l.y; c[5] = l.z;
    };
    if (t == JNT_FREE) {
      put(d + 0, V3<T>(), V3<T>(1, 0, 0));
      put(d + 1, V3<T>(), V3<T>(0, 1, 0));
      put(d + 2, V3<T>(), V3<T>(0, 0, 1));
      for (int k = 0; k < 3; k++) put(d + 3 + k, xm.col(k), cross(xm.col(k), off));
    } else if (t == JNT_BALL) {
      for (int k = 0; k < 3; k++) put(d + k, xm.col(k), cross(xm.col(k), off));
    } else if (t == JNT_SLIDE) {
      put(d, V3<T>(), xaxis);
    } else {
      put(d, xaxis, cross(xaxis, off));
    }
  }
}

// smooth.py:248-314 (dense qM)
template <typename T>
void crb(const Model<T>& m, World<T>& w) {
  w.crb = w.cinert;
  for (int lvl = m.nlevel - 1; lvl >= 0; lvl--) {
    for (int n = m.body_treeadr[lvl]; n < m.body_treeadr[lvl + 1]; n++) {
      int b = m.body_tree[n], p = m.body_parentid[b];
      if (p == 0) continue;
      for (int k = 0; k < 10; k++) w.crb[10 * p + k] += w.crb[10 * b + k];
    }
  }
  int nv = m.nv;
  std::fill(w.qM.begin(), w.qM.end(), T(0));
  for (int i = 0; i < nv; i++) {
    int b = m.dof_bodyid[i];
    S6<T> cd;
    for (int k = 0; k < 6; k++) cd[k] = w.cdof[6 * i + k];
    S6<T> buf = inert_vec(&w.crb[10 * b], cd);
    w.qM[i * nv + i] = m.dof_armature[i] + dot6(&w.cdof[6 * i], buf);
    for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j]) {
      T v = dot6(&w.cdof[6 * j], buf);
      w.qM[i * nv + j] += v;
      w.qM[j * nv + i] += v;
    }
  }
}

// Dense Cholesky of each tree block of an inertia-like matrix (smooth.py:353-379: tile_cholesky
// per qLD_tile group). L is written lower-triangular into L (nv x nv), zero elsewhere.
template <typename T>
void factor_blocks(const Model<T>& m, const std::vector<T>& M, std::vector<T>& L) {
  int nv = m.nv;
  std::fill(L.begin(), L.end(), T(0));
  for (int blk = 0; blk < m.nblock; blk++) {
    int a = m.block_adr[blk], n = m.block_size[blk];
    for (int j = 0; j < n; j++) {
      T s = M[(a + j) * nv + a + j];
      for (int k = 0; k < j; k++) s -= L[(a + j) * nv + a + k] * L[(a + j) * nv + a + k];
      T d = std::sqrt(s);
      L[(a + j) * nv + a + j] = d;
      for (int i = j + 1; i < n; i++) {
        T t = M[(a + i) * nv + a + j];
        for (int k = 0; k < j; k++) t -= L[(a + i) * nv + a + k] * L[(a + j) * nv + a + k];
        L[(a + i) * nv + a + j] = t / d;
      }
    }
  }
}

// x = (L L^T)^-1 y per tree block (smooth.py:654-681 tile_cholesky_solve)
template <typename T>
void solve_blocks(const Model<T>& m, const std::vector<T>& L, T* x, const T* y) {
  int nv = m.nv;
  std::vector<T> z(nv);
  for (int blk = 0; blk < m.nblock; blk++) {
    int a = m.block_adr[blk], n = m.block_size[blk];
    for (int i = 0; i < n; i++) {
      T s = y[a + i];
      for (int k = 0; k < i; k++) s -= L[(a + i) * nv + a + k] * z[a + k];
      z[a + i] = s / L[(a + i) * nv + a + i];
    }
    for (int i = n - 1; i >= 0; i--) {
      T s = z[a + i];
      for (int k = i + 1; k < n; k++) s -= L[(a + k) * nv + a + i] * x[a + k];
      x[a + i] = s / L[(a + i) * nv + a + i];
    }
  }
}

// Dense Cholesky factor + solve of a full nv x nv lower-triangular-stored matrix (solver.py:279-290)
template <typename T>
void cholesky_full_solve(int nv, const std::vector<T>& H, T* x, const T* y) {
  std::vector<T> L(nv * nv, T(0)), z(nv);
  for (int j = 0; j < nv; j++) {
    T s = H[j * nv + j];
    for (int k = 0; k < j; k++) s -= L[j * nv + k] * L[j * nv + k];
    T d = std::sqrt(s);
    L[j * nv + j] = d;
    for (int i = j + 1; i < nv; i++) {
      T t = H[i * nv + j];
      for (int k = 0; k < j; k++) t -= L[i * nv + k] * L[j * nv + k];
      L[i * nv + j] = t / d;
    }
  }
  for (int i = 0; i < nv; i++) {
    T s = y[i];
    for (int k = 0; k < i; k++) s -= L[i * nv + k] * z[k];
    z[i] = s / L[i * nv + i];
  }
  for (int i = nv - 1; i >= 0; i--) {
    T s = z[i];
    for (int k = i + 1; k < nv; k++) s -= L[k * nv + i] * x[k];
    x[i] = s / L[i * nv + i];
  }
}

template <typename T>
void factor_m(const Model<T>& m, World<T>& w) { factor_blocks(m, w.qM, w.qLD); }

// smooth.py:398-466
template <typename T>
void rne(const Model<T>& m, World<T>& w) {
  int nb = m.nbody;
  for (int k = 0; k < 6; k++) w.rne_cacc[k] = 0;
  if (!(m.disableflags & DSBL_GRAVITY)) {
    w.rne_cacc[3] = -m.gravity.x; w.rne_cacc[4] = -m.gravity.y; w.rne_cacc[5] = -m.gravity.z;
  }
  for (int lvl = 0; lvl < m.nlevel; lvl++) {
    for (int n = m.body_treeadr[lvl]; n < m.body_treeadr[lvl + 1]; n++) {
      int b = m.body_tree[n], p = m.body_parentid[b];
      T acc[6];
      for (int k = 0; k < 6; k++) acc[k] = w.rne_cacc[6 * p + k];
      for (int i = 0; i < m.body_dofnum[b]; i++) {
        int d = m.body_dofadr[b] + i;
        for (int k = 0; k < 6; k++) acc[k] += w.cdof_dot[6 * d + k] * w.qvel[d];
      }
      for (int k = 0; k < 6; k++) w.rne_cacc[6 * b + k] = acc[k];
    }
  }
  for (int b = 0; b < nb; b++) {
    S6<T> cacc, cvel;
    for (int k = 0; k < 6; k++) { cacc[k] = w.rne_cacc[6 * b + k]; cvel[k] = w.cvel[6 * b + k]; }
    S6<T> f = inert_vec(&w.cinert[10 * b], cacc);
    S6<T> g = motion_cross_force(cvel, inert_vec(&w.cinert[10 * b], cvel));
    for (int k = 0; k < 6; k++) w.rne_cfrc[6 * b + k] = f[k] + g[k];
  }
  for (int lvl = m.nlevel - 1; lvl >= 0; lvl--) {
    for (int n = m.body_treeadr[lvl]; n < m.body_treeadr[lvl + 1]; n++) {
      int b = m.body_tree[n], p = m.body_parentid[b];
      T v[6];
      for (int k = 0; k < 6; k++) v[k] = w.rne_cfrc[6 * b + k];
      for (int k = 0; k < 6; k++) w.rne_cfrc[6 * p + k] += v[k];
    }
  }
  for (int i = 0; i < m.nv; i++) {
    int b = m.dof_bodyid[i];
    T s = 0;
    for (int k = 0; k < 6; k++) s += w.cdof[6 * i + k] * w.rne_cfrc[6 * b + k];
    w.qfrc_bias[i] = s;
  }
}

// smooth.py:469-536
template <typename T>
void transmission(const Model<T>& m, World<T>& w) {
  int nv = m.nv;
  for (int a = 0; a < m.nu; a++) {
    int j = m.actuator_trnid[2 * a], t = m.jnt_type[j], qa = m.jnt_qposadr[j], va = m.jnt_dofadr[j];
    int trn = m.actuator_trntype[a];
    const T* gear = &m.actuator_gear[6 * a];
    T* mom = &w.actuator_moment[a * nv];
    for (int i = 0; i < nv; i++) mom[i] = 0;
    if (trn != 0 && trn != 1) continue;
    if (t == JNT_FREE) {
      w.actuator_length[a] = 0;
      if (trn == 1) {
        Q4<T> qn{w.qpos[qa + 3], -w.qpos[qa + 4], -w.qpos[qa + 5], -w.qpos[qa + 6]};
        V3<T> ga = rot_vec_quat(V3<T>(gear[3], gear[4], gear[5]), qn);
        mom[va] = gear[0]; mom[va + 1] = gear[1]; mom[va + 2] = gear[2];
        mom[va + 3] = ga.x; mom[va + 4] = ga.y; mom[va + 5] = ga.z;
      } else {
        for (int i = 0; i < 6; i++) mom[va + i] = gear[i];
      }
    } else if (t == JNT_BALL) {
      Q4<T> q{w.qpos[qa], w.qpos[qa + 1], w.qpos[qa + 2], w.qpos[qa + 3]};
      V3<T> aa = quat_to_vel(q);
      V3<T> ga(gear[0], gear[1], gear[2]);
      if (trn == 1) ga = rot_vec_quat(ga, Q4<T>{q.w, -q.x, -q.y, -q.z});
      w.actuator_length[a] = dot(aa, ga);
      mom[va] = ga.x; mom[va + 1] = ga.y; mom[va + 2] = ga.z;
    } else {
      w.actuator_length[a] = w.qpos[qa] * gear[0];
      mom[va] = gear[0];
    }
  }
}

// smooth.py:539-606
template <typename T>
void com_vel(const Model<T>& m, World<T>& w) {
  for (int k = 0; k < 6; k++) w.cvel[k] = 0;
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    for (int n = m.body_treeadr[lvl]; n < m.body_treeadr[lvl + 1]; n++) {
      int b = m.body_tree[n], p = m.body_parentid[b];
      S6<T> cvel;
      for (int k = 0; k < 6; k++) cvel[k] = w.cvel[6 * p + k];
      int d = m.body_dofadr[b];
      auto cd = [&](int i) { S6<T> c; for (int k = 0; k < 6; k++) c[k] = w.cdof[6 * i + k]; return c; };
      auto add = [&](int i) { for (int k = 0; k < 6; k++) cvel[k] += w.cdof[6 * i + k] * w.qvel[i]; };
      auto setdot = [&](int i) { S6<T> r = motion_cross(cvel, cd(i)); for (int k = 0; k < 6; k++) w.cdof_dot[6 * i + k] = r[k]; };
      for (int j = m.body_jntadr[b]; j < m.body_jntadr[b] + m.body_jntnum[b]; j++) {
        int t = m.jnt_type[j];
        if (t == JNT_FREE) {
          add(d); add(d + 1); add(d + 2);
          for (int k = 0; k < 6; k++) w.cdof_dot[6 * d + k] = w.cdof_dot[6 * (d + 1) + k] = w.cdof_dot[6 * (d + 2) + k] = 0;
          setdot(d + 3); setdot(d + 4); setdot(d + 5);
          add(d + 3); add(d + 4); add(d + 5);
          d += 6;
        } else if (t == JNT_BALL) {
          setdot(d); setdot(d + 1); setdot(d + 2);
          add(d); add(d + 1); add(d + 2);
          d += 3;
        } else {
          setdot(d);
          add(d);
          d += 1;
        }
      }
      for (int k = 0; k < 6; k++) w.cvel[6 * b + k] = cvel[k];
    }
  }
}

// passive.py:27-108
template <typename T>
void passive(const Model<T>& m, World<T>& w) {
  if (m.disableflags & DSBL_PASSIVE) {
    std::fill(w.qfrc_passive.begin(), w.qfrc_passive.end(), T(0));
    return;
  }
  std::fill(w.qfrc_spring.begin(), w.qfrc_spring.end(), T(0));
  for (int j = 0; j < m.njnt; j++) {
    T k = m.jnt_stiffness[j];
    int d = m.jnt_dofadr[j];
    if (k == T(0)) continue;
    int t = m.jnt_type[j], a = m.jnt_qposadr[j];
    if (t == JNT_FREE) {
      for (int i = 0; i < 3; i++) w.qfrc_spring[d + i] = -k * (w.qpos[a + i] - m.qpos_spring[a + i]);
      Q4<T> rot{w.qpos[a + 3], w.qpos[a + 4], w.qpos[a + 5], w.qpos[a + 6]};
      Q4<T> ref{m.qpos_spring[a + 3], m.qpos_spring[a + 4], m.qpos_spring[a + 5], m.qpos_spring[a + 6]};
      V3<T> dif = quat_sub(rot, ref);
      for (int i = 0; i < 3; i++) w.qfrc_spring[d + 3 + i] = -k * dif[i];
    } else if (t == JNT_BALL) {
      Q4<T> rot{w.qpos[a], w.qpos[a + 1], w.qpos[a + 2], w.qpos[a + 3]};
      Q4<T> ref{m.qpos_spring[a], m.qpos_spring[a + 1], m.qpos_spring[a + 2], m.qpos_spring[a + 3]};
      V3<T> dif = quat_sub(rot, ref);
      for (int i = 0; i < 3; i++) w.qfrc_spring[d + i] = -k * dif[i];
    } else {
      w.qfrc_spring[d] = -k * (w.qpos[a] - m.qpos_spring[a]);
    }
  }
  for (int i = 0; i < m.nv; i++) {
    T damper = -m.dof_damping[i] * w.qvel[i];
    w.qfrc_damper[i] = damper;
    w.qfrc_passive[i] = damper + w.qfrc_spring[i];
  }
}

// ------------------------------------------------------------------------------------------
// collision_driver.py / collision_primitive.py

// collision_driver.py:27-49
template <typename T>
bool geom_filter(const Model<T>& m, int g1, int g2, bool filterparent) {
  int b1 = m.geom_bodyid[g1], b2 = m.geom_bodyid[g2];
  int w1 = m.body_weldid[b1], w2 = m.body_weldid[b2];
  int wp1 = m.body_weldid[m.body_parentid[w1]], wp2 = m.body_weldid[m.body_parentid[w2]];
  bool self = w1 == w2;
  bool pc = filterparent && w1 != 0 && w2 != 0 && (w1 == wp2 || w2 == wp1);
  bool mask = (m.geom_contype[g1] & m.geom_conaffinity[g2]) || (m.geom_contype[g2] & m.geom_conaffinity[g1]);
  return mask && !self && !pc;
}

// collision_driver.py:458-512: every pair (g1 < g2) in element order, bounding test, filter,
// append with the type-ordering swap of _add_geom_pair (:52-68)
template <typename T>
void nxn_broadphase(const Model<T>& m, World<T>& w) {
  w.pair.clear();
  bool filterparent = !(m.disableflags & DSBL_FILTERPARENT);
  for (int g1 = 0; g1 < m.ngeom; g1++) {
    for (int g2 = g1 + 1; g2 < m.ngeom; g2++) {
      T m1 = m.geom_margin[g1], m2 = m.geom_margin[g2];
      T s1 = m.geom_rbound[g1], s2 = m.geom_rbound[g2];
      T bound = s1 + s2 + std::max(m1, m2);
      V3<T> p1(w.geom_xpos[3 * g1], w.geom_xpos[3 * g1 + 1], w.geom_xpos[3 * g1 + 2]);
      V3<T> p2(w.geom_xpos[3 * g2], w.geom_xpos[3 * g2 + 1], w.geom_xpos[3 * g2 + 2]);
      V3<T> dif = p2 - p1;
      bool bf;
      if (s1 != T(0) && s2 != T(0)) {
        T dsq = dot(dif, dif);
        bf = dsq <= bound * bound;
      } else if (s1 == T(0)) {
        const T* x = &w.geom_xmat[9 * g1];
        T dist = dot(dif, V3<T>(x[2], x[5], x[8]));
        bf = dist <= bound;
      } else {
        const T* x = &w.geom_xmat[9 * g2];
        V3<T> nd = V3<T>() - dif;
        T dist = dot(nd, V3<T>(x[2], x[5], x[8]));
        bf = dist <= bound;
      }
      if (bf && geom_filter(m, g1, g2, filterparent)) {
        if (m.geom_type[g1] > m.geom_type[g2]) {
          w.pair.push_back(g2); w.pair.push_back(g1);
        } else {
          w.pair.push_back(g1); w.pair.push_back(g2);
        }
      }
    }
  }
}

// collision_driver.py:350-455 — sweep-and-prune: project bounding spheres on the fixed direction
// (:72-92), stable sort of the lower bounds (the segmented radix sort, :373-378), reorder into
// spheres / encoded planes (:134-156), then every sorted position i against positions
// i+1 .. min(ngeom-1, first position whose lower bound exceeds i's upper bound) (:219-236), with
// the filter and the overlap test (:163-184, 272-300).  encode_plane / decode_plane (:98-130) as
// the reference evaluates them: the decoded offset magnitude is the length of the whole 4-vector,
// w code included.  Pairs in sweep order.
template <typename T>
V3<T> sap_normalize(V3<T> v) {
  T l = std::sqrt(dot(v, v));
  return l > T(0) ? V3<T>(v[0] / l, v[1] / l, v[2] / l) : v;
}

template <typename T>
void sap_encode_plane(V3<T> normal, V3<T> point, T margin, T out[4]) {
  V3<T> n = sap_normalize(normal);
  V3<T> q(point[0] + n[0] * margin, point[1] + n[1] * margin, point[2] + n[2] * margin);
  T off = -dot(n, q);
  T scale = std::fabs(off);
  if (std::fabs(off) < T(1e-6)) {
    out[0] = n[0]; out[1] = n[1]; out[2] = n[2]; out[3] = T(-1);
  } else {
    out[0] = scale * n[0]; out[1] = scale * n[1]; out[2] = scale * n[2];
    out[3] = off < T(0) ? T(-2) : T(-3);
  }
}

template <typename T>
bool sap_overlap(const T* a, const T* b) {
  if (a[3] < T(0) && b[3] < T(0)) return false;
  if (a[3] < T(0) || b[3] < T(0)) {
    if (b[3] < T(0)) std::swap(a, b);
    V3<T> e(a[0], a[1], a[2]);
    T mag = std::sqrt(dot(e, e) + a[3] * a[3]);
    V3<T> n = sap_normalize(e);
    T off = a[3] == T(-1) ? T(0) : (a[3] == T(-2) ? -mag : mag);
    T dist = dot(V3<T>(b[0], b[1], b[2]), n) + off;
    return dist <= b[3];
  }
  V3<T> dlt(a[0] - b[0], a[1] - b[1], a[2] - b[2]);
  T r = a[3] + b[3];
  return dot(dlt, dlt) <= r * r;
}

template <typename T>
void sap_broadphase(const Model<T>& m, World<T>& w) {
  w.pair.clear();
  const int ng = m.ngeom;
  bool filterparent = !(m.disableflags & DSBL_FILTERPARENT);
  V3<T> dir = sap_normalize(V3<T>(T(0.5935f), T(0.7790f), T(0.1235f)));
  std::vector<T> lo(ng), up(ng), S(4 * ng);
  std::vector<int> idx(ng);
  for (int g = 0; g < ng; g++) {
    T r = m.geom_rbound[g];
    if (r == T(0)) r = T(1e9f);
    T sr = r + m.geom_margin[g];
    T c = dot(dir, V3<T>(w.geom_xpos[3 * g], w.geom_xpos[3 * g + 1], w.geom_xpos[3 * g + 2]));
    lo[g] = c - sr;
    up[g] = c + sr;
    idx[g] = g;
  }
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return lo[a] < lo[b]; });
  std::vector<T> los(ng);
  for (int i = 0; i < ng; i++) los[i] = lo[idx[i]];
  for (int i = 0; i < ng; i++) {
    int g = idx[i];
    V3<T> c(w.geom_xpos[3 * g], w.geom_xpos[3 * g + 1], w.geom_xpos[3 * g + 2]);
    T r = m.geom_rbound[g], margin = m.geom_margin[g];
    if (r == T(0)) {
      const T* x = &w.geom_xmat[9 * g];
      sap_encode_plane(V3<T>(x[2], x[5], x[8]), c, margin, &S[4 * i]);
    } else {
      S[4 * i] = c[0]; S[4 * i + 1] = c[1]; S[4 * i + 2] = c[2]; S[4 * i + 3] = r + margin;
    }
  }
  for (int i = 0; i < ng; i++) {
    int g1 = idx[i];
    T end = up[g1];
    int a = i + 1, b = ng;
    while (a < b) {
      int mid = (a + b) >> 1;
      if (los[mid] > end) b = mid;
      else a = mid + 1;
    }
    int limit = std::min(ng - 1, a);
    for (int j = i + 1; j <= limit; j++) {
      int g2 = idx[j];
      if (!geom_filter(m, g1, g2, filterparent) || !sap_overlap(&S[4 * i], &S[4 * j])) continue;
      if (m.geom_type[g1] > m.geom_type[g2]) {
        w.pair.push_back(g2); w.pair.push_back(g1);
      } else {
        w.pair.push_back(g1); w.pair.push_back(g2);
      }
    }
  }
}

template <typename T>
void write_contact(World<T>& w, T dist, V3<T> pos, const M3<T>& frame, T margin, int g1, int g2) {
  // collision_primitive.py:52-70
  if ((dist - margin) < T(0)) {
    w.con_dist.push_back(dist);
    for (int k = 0; k < 3; k++) w.con_pos.push_back(pos[k]);
    for (int k = 0; k < 9; k++) w.con_frame.push_back(frame.m[k]);
    w.con_geom.push_back(g1);
    w.con_geom.push_back(g2);
  }
}

template <typename T>
void plane_sphere_raw(V3<T> n, V3<T> ppos, V3<T> spos, T r, T& dist, V3<T>& pos) {
  dist = dot(spos - ppos, n) - r;
  pos = spos - n * (r + T(0.5) * dist);
}

template <typename T>
void sphere_sphere_raw(World<T>& w, V3<T> p1, T r1, V3<T> p2, T r2, T margin, int g1, int g2) {
  V3<T> dir = p2 - p1;
  T dist = length(dir);
  V3<T> n = dist == T(0) ? V3<T>(1, 0, 0) : dir * (T(1) / dist);
  dist = dist - (r1 + r2);
  V3<T> pos = p1 + n * (r1 + T(0.5) * dist);
  write_contact(w, dist, pos, make_frame(n), margin, g1, g2);
}

// collision_primitive.py:235-268 per pair, then get_contact_solver_params (collision_driver.py:304-347)
template <typename T>
void narrowphase(const Model<T>& m, World<T>& w) {
  w.con_dist.clear(); w.con_pos.clear(); w.con_frame.clear(); w.con_geom.clear();
  for (int p = 0; p < w.npair(); p++) {
    int g1 = w.pair[2 * p], g2 = w.pair[2 * p + 1];
    int t1 = m.geom_type[g1], t2 = m.geom_type[g2];
    V3<T> pos1(w.geom_xpos[3 * g1], w.geom_xpos[3 * g1 + 1], w.geom_xpos[3 * g1 + 2]);
    V3<T> pos2(w.geom_xpos[3 * g2], w.geom_xpos[3 * g2 + 1], w.geom_xpos[3 * g2 + 2]);
    M3<T> r1, r2;
    std::memcpy(r1.m, &w.geom_xmat[9 * g1], sizeof(r1.m));
    std::memcpy(r2.m, &w.geom_xmat[9 * g2], sizeof(r2.m));
    V3<T> n1 = r1.col(2);
    V3<T> sz1 = m.v3(m.geom_size, g1), sz2 = m.v3(m.geom_size, g2);
    T margin = std::max(m.geom_margin[g1], m.geom_margin[g2]);
    if (t1 == GEOM_PLANE && t2 == GEOM_SPHERE) {
      T dist; V3<T> pos;
      plane_sphere_raw(n1, pos1, pos2, sz2.x, dist, pos);
      write_contact(w, dist, pos, make_frame(n1), margin, g1, g2);
    } else if (t1 == GEOM_SPHERE && t2 == GEOM_SPHERE) {
      sphere_sphere_raw(w, pos1, sz1.x, pos2, sz2.x, margin, g1, g2);
    } else if (t1 == GEOM_PLANE && t2 == GEOM_CAPSULE) {
      // collision_primitive.py:166-195
      V3<T> n = n1, axis = r2.col(2);
      V3<T> bv = axis - n * dot(n, axis);
      T bn = length(bv);
      V3<T> b = bn == T(0) ? bv : bv * (T(1) / bn);
      if (bn < T(0.5)) b = (T(-0.5) < n.y && n.y < T(0.5)) ? V3<T>(0, 1, 0) : V3<T>(0, 0, 1);
      V3<T> c = cross(n, b);
      M3<T> frame;
      frame.m[0] = n.x; frame.m[1] = n.y; frame.m[2] = n.z;
      frame.m[3] = b.x; frame.m[4] = b.y; frame.m[5] = b.z;
      frame.m[6] = c.x; frame.m[7] = c.y; frame.m[8] = c.z;
      V3<T> seg = axis * sz2.y;
      T dist; V3<T> pos;
      plane_sphere_raw(n, pos1, pos2 + seg, sz2.x, dist, pos);
      write_contact(w, dist, pos, frame, margin, g1, g2);
      plane_sphere_raw(n, pos1, pos2 - seg, sz2.x, dist, pos);
      write_contact(w, dist, pos, frame, margin, g1, g2);
    } else if (t1 == GEOM_PLANE && t2 == GEOM_BOX) {
      // collision_primitive.py:198-232
      int count = 0;
      T dist = dot(pos2 - pos1, n1);
      for (int i = 0; i < 8; i++) {
        V3<T> corner((i & 1) ? sz2.x : -sz2.x, (i & 2) ? sz2.y : -sz2.y, (i & 4) ? sz2.z : -sz2.z);
        corner = mulmv(r2, corner);
        T ldist = dot(n1, corner);
        if (dist + ldist > margin || ldist > T(0)) continue;
        T cdist = dist + ldist;
        V3<T> pos = corner + pos2 + n1 * (cdist / T(-2));
        write_contact(w, cdist, pos, make_frame(n1), margin, g1, g2);
        if (++count >= 4) break;
      }
    } else if (t1 == GEOM_CAPSULE && t2 == GEOM_CAPSULE) {
      // collision_primitive.py:140-163
      V3<T> s1 = r1.col(2) * sz1.y, s2 = r2.col(2) * sz2.y;
      V3<T> pa, pb;
      closest_segment_to_segment_points(pos1 - s1, pos1 + s1, pos2 - s2, pos2 + s2, pa, pb);
      sphere_sphere_raw(w, pa, sz1.x, pb, sz2.x, margin, g1, g2);
    }
  }
  // get_contact_solver_params_kernel (collision_driver.py:304-347)
  int nc = w.ncon();
  w.con_dim.assign(nc, 0);
  w.con_includemargin.assign(nc, 0);
  w.con_friction.assign(5 * nc, 0);
  w.con_solref.assign(2 * nc, 0);
  w.con_solimp.assign(5 * nc, 0);
  for (int i = 0; i < nc; i++) {
    int g1 = w.con_geom[2 * i], g2 = w.con_geom[2 * i + 1];
    T margin = std::max(m.geom_margin[g1], m.geom_margin[g2]);
    T gap = std::max(m.geom_gap[g1], m.geom_gap[g2]);
    T sm1 = m.geom_solmix[g1], sm2 = m.geom_solmix[g2];
    T mix = sm1 / (sm1 + sm2);
    if (sm1 < T(kMinVal) && sm2 < T(kMinVal)) mix = T(0.5);
    else if (sm1 < T(kMinVal)) mix = T(0);
    else if (sm2 < T(kMinVal)) mix = T(1);
    int p1 = m.geom_priority[g1], p2 = m.geom_priority[g2];
    if (p1 != p2) mix = p1 > p2 ? T(1) : T(0);
    int c1 = m.geom_condim[g1], c2 = m.geom_condim[g2];
    w.con_dim[i] = p1 == p2 ? std::max(c1, c2) : (p1 > p2 ? c1 : c2);
    if (m.geom_solref[2 * g1] > T(0) && m.geom_solref[2 * g2] > T(0)) {
      for (int k = 0; k < 2; k++)
        w.con_solref[2 * i + k] = mix * m.geom_solref[2 * g1 + k] + (T(1) - mix) * m.geom_solref[2 * g2 + k];
    } else {
      for (int k = 0; k < 2; k++)
        w.con_solref[2 * i + k] = std::min(m.geom_solref[2 * g1 + k], m.geom_solref[2 * g2 + k]);
    }
    w.con_includemargin[i] = margin - gap;
    T f[3];
    for (int k = 0; k < 3; k++) f[k] = std::max(m.geom_friction[3 * g1 + k], m.geom_friction[3 * g2 + k]);
    T f5[5] = {f[0], f[0], f[1], f[2], f[2]};
    for (int k = 0; k < 5; k++) w.con_friction[5 * i + k] = f5[k];
    for (int k = 0; k < 5; k++)
      w.con_solimp[5 * i + k] = mix * m.geom_solimp[5 * g1 + k] + (T(1) - mix) * m.geom_solimp[5 * g2 + k];
  }
}

template <typename T>
void collision(const Model<T>& m, World<T>& w) {
  if (m.ngeom > 100) sap_broadphase(m, w);  // collision_driver.py:537-540
  else nxn_broadphase(m, w);
  narrowphase(m, w);
}

// ------------------------------------------------------------------------------------------
// constraint.py

// constraint.py:22-73
template <typename T>
void update_efc_row(const Model<T>& m, World<T>& w, int r, T pos_aref, T pos_imp, T invweight,
                    const T* solref, const T* solimp, T margin, bool refsafe, T Jqvel) {
  T timeconst = solref[0], dampratio = solref[1];
  T dmin = solimp[0], dmax = solimp[1], width = solimp[2], mid = solimp[3], power = solimp[4];
  if (refsafe) timeconst = std::max(timeconst, T(2) * m.timestep);
  dmin = std::min(std::max(dmin, T(kMinImp)), T(kMaxImp));
  dmax = std::min(std::max(dmax, T(kMinImp)), T(kMaxImp));
  width = std::max(T(kMinVal), width);
  mid = std::min(std::max(mid, T(kMinImp)), T(kMaxImp));
  power = std::max(T(1), power);
  T k = T(1) / (dmax * dmax * timeconst * timeconst * dampratio * dampratio);
  T b = T(2) / (dmax * timeconst);
  if (solref[0] <= T(0)) k = -solref[0] / (dmax * dmax);
  if (solref[1] <= T(0)) b = -solref[1] / dmax;
  T imp_x = std::abs(pos_imp) / width;
  T imp;
  if (imp_x > T(1)) {
    imp = dmax;
  } else {
    T imp_y;
    if (imp_x < mid) imp_y = (T(1) / std::pow(mid, power - T(1))) * std::pow(imp_x, power);
    else imp_y = T(1) - (T(1) / std::pow(T(1) - mid, power - T(1))) * std::pow(T(1) - imp_x, power);
    imp = dmin + imp_y * (dmax - dmin);
    imp = std::min(std::max(imp, dmin), dmax);
  }
  w.efc_D[r] = T(1) / std::max(invweight * (T(1) - imp) / imp, T(kMinVal));
  w.efc_aref[r] = -k * imp * pos_aref - b * Jqvel;
  w.efc_pos[r] = pos_aref + margin;
  w.efc_margin[r] = margin;
}

template <typename T>
void make_constraint(const Model<T>& m, World<T>& w) {
  int nv = m.nv;
  w.efc_J.clear(); w.efc_pos.clear(); w.efc_margin.clear(); w.efc_D.clear(); w.efc_aref.clear();
  if (m.disableflags & DSBL_CONSTRAINT) return;
  bool refsafe = !(m.disableflags & DSBL_REFSAFE);
  auto newrow = [&]() {
    int r = w.nefc();
    w.efc_J.resize((r + 1) * nv, T(0));
    w.efc_pos.push_back(0); w.efc_margin.push_back(0); w.efc_D.push_back(0); w.efc_aref.push_back(0);
    return r;
  };
  // constraint.py:104-141
  if (!(m.disableflags & DSBL_LIMIT)) {
    for (int l = 0; l < m.nlimit; l++) {
      int j = m.jnt_limited_slide_hinge_adr[l];
      T q = w.qpos[m.jnt_qposadr[j]];
      T dmin = q - m.jnt_range[2 * j], dmax = m.jnt_range[2 * j + 1] - q;
      T pos = std::min(dmin, dmax) - m.jnt_margin[j];
      if (pos < T(0)) {
        int r = newrow();
        int d = m.jnt_dofadr[j];
        T J = T(dmin < dmax ? 1 : 0) * T(2) - T(1);
        w.efc_J[r * nv + d] = J;
        T Jqvel = J * w.qvel[d];
        update_efc_row(m, w, r, pos, pos, m.dof_invweight0[d], &m.jnt_solref[2 * j],
                       &m.jnt_solimp[5 * j], m.jnt_margin[j], refsafe, Jqvel);
      }
    }
  }
  // constraint.py:144-210
  if (!(m.disableflags & DSBL_CONTACT) && m.cone == 0) {
    for (int c = 0; c < w.ncon(); c++) {
      if (w.con_dim[c] != 3) continue;
      T pos = w.con_dist[c] - w.con_includemargin[c];
      if (!(pos < T(0))) continue;
      int b1 = m.geom_bodyid[w.con_geom[2 * c]], b2 = m.geom_bodyid[w.con_geom[2 * c + 1]];
      T fri0 = w.con_friction[5 * c];
      T invweight = m.body_invweight0[2 * b1] + m.body_invweight0[2 * b2];
      invweight = invweight + fri0 * fri0 * invweight;
      invweight = invweight * T(2) * fri0 * fri0 / m.impratio;
      V3<T> cp(w.con_pos[3 * c], w.con_pos[3 * c + 1], w.con_pos[3 * c + 2]);
      const T* fr = &w.con_frame[9 * c];
      // per-dof translational jacobian difference at the contact point (constraint.py:76-101)
      std::vector<V3<T>> jdif(nv);
      for (int i = 0; i < nv; i++) {
        V3<T> j12[2];
        int bodies[2] = {b1, b2};
        for (int s = 0; s < 2; s++) {
          int body = bodies[s];
          int db = m.dof_bodyid[i];
          int in_tree = db == 0;
          for (int p = body; p != 0; p = m.body_parentid[p])
            if (p == db) { in_tree = 1; break; }
          int r = m.body_rootid[body];
          V3<T> off = cp - V3<T>(w.subtree_com[3 * r], w.subtree_com[3 * r + 1], w.subtree_com[3 * r + 2]);
          const T* cd = &w.cdof[6 * i];
          V3<T> jac = V3<T>(cd[3], cd[4], cd[5]) + cross(V3<T>(cd[0], cd[1], cd[2]), off);
          j12[s] = jac * T(in_tree);
        }
        jdif[i] = j12[1] - j12[0];
      }
      for (int dimid = 0; dimid < 4; dimid++) {
        int r = newrow();
        int d2 = dimid / 2 + 1;
        T Jqvel = 0;
        for (int i = 0; i < nv; i++) {
          T diff0 = 0, diffi = 0;
          for (int xyz = 0; xyz < 3; xyz++) {
            diff0 += fr[xyz] * jdif[i][xyz];
            diffi += fr[3 * d2 + xyz] * jdif[i][xyz];
          }
          T f = w.con_friction[5 * c + d2 - 1];
          T J = (dimid % 2 == 0) ? diff0 + diffi * f : diff0 - diffi * f;
          w.efc_J[r * nv + i] = J;
          Jqvel += J * w.qvel[i];
        }
        update_efc_row(m, w, r, pos, pos, invweight, &w.con_solref[2 * c], &w.con_solimp[5 * c],
                       w.con_includemargin[c], refsafe, Jqvel);
      }
    }
  }
  int n = w.nefc();
  w.efc_force.assign(n, 0);
  w.efc_Jaref.assign(n, 0);
  w.efc_active.assign(n, 0);
  w.jv.assign(n, 0);
  w.quad.assign(3 * n, 0);
}

// ------------------------------------------------------------------------------------------
// forward.py / support.py

// support.py:140-172
template <typename T>
void xfrc_accumulate(const Model<T>& m, World<T>& w, T* qfrc) {
  for (int i = 0; i < m.nv; i++) {
    const T* cd = &w.cdof[6 * i];
    V3<T> rot(cd[0], cd[1], cd[2]), lin(cd[3], cd[4], cd[5]);
    int db = m.dof_bodyid[i];
    T acc = 0;
    for (int b = db; b < m.nbody; b++) {
      int p = b;
      while (p != 0 && p != db) p = m.body_parentid[p];
      if (p == 0) continue;
      int r = m.body_rootid[b];
      V3<T> off(w.xipos[3 * b] - w.subtree_com[3 * r], w.xipos[3 * b + 1] - w.subtree_com[3 * r + 1],
                w.xipos[3 * b + 2] - w.subtree_com[3 * r + 2]);
      const T* f = &w.xfrc_applied[6 * b];
      V3<T> force(f[0], f[1], f[2]), torque(f[3], f[4], f[5]);
      acc += dot(lin, force) + dot(rot, torque) + dot(cross(rot, off), force);
    }
    qfrc[i] += acc;
  }
}

template <typename T>
void mul_m(const Model<T>& m, const World<T>& w, T* res, const T* vec) {
  int nv = m.nv;
  for (int i = 0; i < nv; i++) {
    T s = 0;
    for (int j = 0; j < nv; j++) s += w.qM[i * nv + j] * vec[j];
    res[i] = s;
  }
}

// forward.py:423-500
template <typename T>
void fwd_velocity(const Model<T>& m, World<T>& w) {
  for (int a = 0; a < m.nu; a++) {
    T s = 0;
    for (int i = 0; i < m.nv; i++) s += w.actuator_moment[a * m.nv + i] * w.qvel[i];
    w.actuator_velocity[a] = s;
  }
  com_vel(m, w);
  passive(m, w);
  rne(m, w);
}

// forward.py:503-641
template <typename T>
void fwd_actuation(const Model<T>& m, World<T>& w) {
  if (!m.nu || (m.disableflags & DSBL_ACTUATION)) {
    std::fill(w.act_dot.begin(), w.act_dot.end(), T(0));
    std::fill(w.qfrc_actuator.begin(), w.qfrc_actuator.end(), T(0));
    return;
  }
  for (int a = 0; a < m.nu; a++) {
    const T* gp = &m.actuator_gainprm[10 * a];
    const T* bp = &m.actuator_biasprm[10 * a];
    T len = w.actuator_length[a], vel = w.actuator_velocity[a];
    T gain = gp[0] + gp[1] * len + gp[2] * vel;
    T bias = bp[0] + bp[1] * len + bp[2] * vel;
    T ctrl = w.ctrl[a];
    if (m.actuator_ctrllimited[a] && !(m.disableflags & DSBL_CLAMPCTRL))
      ctrl = std::min(std::max(ctrl, m.actuator_ctrlrange[2 * a]), m.actuator_ctrlrange[2 * a + 1]);
    w.actuator_force[a] = gain * ctrl + bias;
  }
  for (int i = 0; i < m.nv; i++) {
    T s = 0;
    for (int a = 0; a < m.nu; a++) s += w.actuator_moment[a * m.nv + i] * w.actuator_force[a];
    int j = m.dof_jntid[i];
    if (m.jnt_actfrclimited[j])
      s = std::min(std::max(s, m.jnt_actfrcrange[2 * j]), m.jnt_actfrcrange[2 * j + 1]);
    w.qfrc_actuator[i] = s;
  }
}

// forward.py:644-661
template <typename T>
void fwd_acceleration(const Model<T>& m, World<T>& w) {
  for (int i = 0; i < m.nv; i++)
    w.qfrc_smooth[i] = w.qfrc_passive[i] - w.qfrc_bias[i] + w.qfrc_actuator[i] + w.qfrc_applied[i];
  xfrc_accumulate(m, w, w.qfrc_smooth.data());
  solve_blocks(m, w.qLD, w.qacc_smooth.data(), w.qfrc_smooth.data());
}

// ------------------------------------------------------------------------------------------
// solver.py (per world; a world that is done skips all further work, solver.py:80-82 etc.)

template <typename T> T safe_div(T x, T y) { return x / (y != T(0) ? y : T(kMinVal)); }
template <typename T> void eval_pt(const T* q, T a, T* out) {
  out[0] = a * a * q[2] + a * q[1] + q[0];
  out[1] = T(2) * a * q[2] + q[1];
  out[2] = T(2) * q[2];
}
template <typename T> bool in_bracket(const T* x, const T* y) {
  return (x[1] < y[1] && y[1] < T(0)) || (x[1] > y[1] && y[1] > T(0));
}

template <typename T>
void update_constraint(const Model<T>& m, World<T>& w) {
  // solver.py:75-173
  int nv = m.nv, n = w.nefc();
  w.prev_cost = w.cost;
  w.cost = 0;
  w.gauss = 0;
  for (int r = 0; r < n; r++) {
    T Jaref = w.efc_Jaref[r], D = w.efc_D[r];
    int active = Jaref < T(0);
    w.efc_active[r] = active;
    if (active) {
      w.efc_force[r] = T(-1) * D * Jaref;
      w.cost += T(0.5) * D * Jaref * Jaref;
    } else {
      w.efc_force[r] = 0;
    }
  }
  for (int i = 0; i < nv; i++) {
    T s = 0;
    for (int r = 0; r < n; r++) s += w.efc_J[r * nv + i] * w.efc_force[r];
    w.qfrc_constraint[i] = s;
  }
  T g = 0;
  for (int i = 0; i < nv; i++)
    g += T(0.5) * (w.Ma[i] - w.qfrc_smooth[i]) * (w.qacc[i] - w.qacc_smooth[i]);
  w.gauss += g;
  w.cost += g;
}

template <typename T>
void update_gradient(const Model<T>& m, World<T>& w) {
  // solver.py:176-312
  int nv = m.nv, n = w.nefc();
  w.grad_dot = 0;
  for (int i = 0; i < nv; i++) {
    T g = w.Ma[i] - w.qfrc_smooth[i] - w.qfrc_constraint[i];
    w.grad[i] = g;
    w.grad_dot += g * g;
  }
  if (m.solver == 1) {  // CG
    solve_blocks(m, w.qLD, w.Mgrad.data(), w.grad.data());
  } else {  // Newton
    for (int i = 0; i < nv; i++)
      for (int j = 0; j < nv; j++) w.h[i * nv + j] = j <= i ? w.qM[i * nv + j] : T(0);
    for (int r = 0; r < n; r++) {
      T D = w.efc_D[r];
      if (D == T(0) || !w.efc_active[r]) continue;
      const T* J = &w.efc_J[r * nv];
      for (int i = 0; i < nv; i++)
        for (int j = 0; j <= i; j++) w.h[i * nv + j] += J[i] * J[j] * D;
    }
    cholesky_full_solve(nv, w.h, w.Mgrad.data(), w.grad.data());
  }
}

template <typename T>
void linesearch(const Model<T>& m, World<T>& w) {
  // solver.py:737-869
  int nv = m.nv, n = w.nefc();
  mul_m(m, w, w.mv.data(), w.search.data());
  for (int r = 0; r < n; r++) {
    T s = 0;
    for (int i = 0; i < nv; i++) s += w.efc_J[r * nv + i] * w.search[i];
    w.jv[r] = s;
  }
  T qg[3] = {0, 0, 0};
  for (int i = 0; i < nv; i++) {
    qg[0] += w.gauss / T(nv);
    qg[1] += w.search[i] * (w.Ma[i] - w.qfrc_smooth[i]);
    qg[2] += T(0.5) * w.search[i] * w.mv[i];
  }
  for (int k = 0; k < 3; k++) w.quad_gauss[k] = qg[k];
  for (int r = 0; r < n; r++) {
    T Jaref = w.efc_Jaref[r], jv = w.jv[r], D = w.efc_D[r];
    w.quad[3 * r] = T(0.5) * Jaref * Jaref * D;
    w.quad[3 * r + 1] = jv * Jaref * D;
    w.quad[3 * r + 2] = T(0.5) * jv * jv * D;
  }
  auto total = [&](T a, T* out) {
    eval_pt(qg, a, out);
    for (int r = 0; r < n; r++) {
      if (w.efc_Jaref[r] + a * w.jv[r] < T(0)) {
        T p[3];
        eval_pt(&w.quad[3 * r], a, p);
        out[0] += p[0]; out[1] += p[1]; out[2] += p[2];
      }
    }
  };
  if (m.ls_parallel) {
    // solver.py:667-734
    int best = 0;
    T bestc = std::numeric_limits<T>::infinity();
    for (int k = 0; k < m.nlsp; k++) {
      T a = m.alpha_candidate[k];
      T tq[3] = {qg[0], qg[1], qg[2]};
      for (int r = 0; r < n; r++)
        if (w.efc_Jaref[r] + a * w.jv[r] < T(0))
          for (int c = 0; c < 3; c++) tq[c] += w.quad[3 * r + c];
      T cost = a * a * tq[2] + a * tq[1] + tq[0];
      if (cost < bestc) { bestc = cost; best = k; }
    }
    w.alpha = m.alpha_candidate[best];
  } else {
    // solver.py:339-664
    T snorm = std::sqrt(w.search_dot);
    T scale = m.meaninertia * T(std::max(1, nv));
    w.gtol = m.tolerance * m.ls_tolerance * snorm * scale;
    T p0[3] = {qg[0], qg[1], T(2) * qg[2]};
    for (int r = 0; r < n; r++) {
      if (w.efc_Jaref[r] >= T(0)) continue;
      p0[0] += w.quad[3 * r]; p0[1] += w.quad[3 * r + 1]; p0[2] += T(2) * w.quad[3 * r + 2];
    }
    T lo_alpha = -safe_div(p0[1], p0[2]);
    T lo[3];
    total(lo_alpha, lo);
    T hi[3], hi_alpha;
    bool lo_less = lo[1] < p0[1];
    if (lo_less) {
      hi[0] = p0[0]; hi[1] = p0[1]; hi[2] = p0[2]; hi_alpha = 0;
    } else {
      hi[0] = lo[0]; hi[1] = lo[1]; hi[2] = lo[2]; hi_alpha = lo_alpha;
      lo[0] = p0[0]; lo[1] = p0[1]; lo[2] = p0[2]; lo_alpha = 0;
    }
    bool done = false;
    for (int it = 0; it < m.ls_iterations && !done; it++) {
      T lon_a = lo_alpha - safe_div(lo[1], lo[2]);
      T hin_a = hi_alpha - safe_div(hi[1], hi[2]);
      T mid_a = T(0.5) * (lo_alpha + hi_alpha);
      T lon[3], hin[3], mid[3];
      total(lon_a, lon);
      total(hin_a, hin);
      total(mid_a, mid);
      // _swap (solver.py:537-617)
      auto copy3 = [](T* d, const T* s) { d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; };
      bool s1 = in_bracket(lo, lon);
      if (s1) { copy3(lo, lon); lo_alpha = lon_a; }
      bool s2 = in_bracket(lo, mid);
      if (s2) { copy3(lo, mid); lo_alpha = mid_a; }
      bool s3 = in_bracket(lo, hin);
      if (s3) { copy3(lo, hin); lo_alpha = hin_a; }
      bool swap_lo = s1 || s2 || s3;
      bool t1 = in_bracket(hi, hin);
      if (t1) { copy3(hi, hin); hi_alpha = hin_a; }
      bool t2 = in_bracket(hi, mid);
      if (t2) { copy3(hi, mid); hi_alpha = mid_a; }
      bool t3 = in_bracket(hi, lon);
      if (t3) { copy3(hi, lon); hi_alpha = lon_a; }
      bool swap_hi = t1 || t2 || t3;
      done = (!swap_lo && !swap_hi) || (lo[1] < T(0) && lo[1] > -w.gtol) ||
             (hi[1] > T(0) && hi[1] < w.gtol);
      T alpha = 0;
      bool improved = lo[0] < p0[0] || hi[0] < p0[0];
      bool lo_better = lo[0] < hi[0];
      if (improved && lo_better) alpha = lo_alpha;
      if (improved && !lo_better) alpha = hi_alpha;
      w.alpha = alpha;
    }
  }
  // solver.py:816-841
  for (int i = 0; i < nv; i++) {
    w.qacc[i] += w.alpha * w.search[i];
    w.Ma[i] += w.alpha * w.mv[i];
  }
  for (int r = 0; r < n; r++) w.efc_Jaref[r] += w.alpha * w.jv[r];
}

template <typename T>
void solve(const Model<T>& m, World<T>& w) {
  // solver.py:872-1000
  int nv = m.nv, n = w.nefc();
  w.qacc = w.qacc_warmstart;
  // _create_context (solver.py:26-72)
  w.cost = std::numeric_limits<T>::infinity();
  w.solver_niter = 0;
  w.iters_run = 0;
  w.done = false;
  w.search_dot = 0;
  for (int r = 0; r < n; r++) {
    T s = 0;
    for (int i = 0; i < nv; i++) s += w.efc_J[r * nv + i] * w.qacc[i];
    w.efc_Jaref[r] = s - w.efc_aref[r];
  }
  mul_m(m, w, w.Ma.data(), w.qacc.data());
  update_constraint(m, w);
  update_gradient(m, w);
  for (int i = 0; i < nv; i++) {
    w.search[i] = -w.Mgrad[i];
    w.search_dot += w.search[i] * w.search[i];
  }
  for (int it = 0; it < m.iterations; it++) {
    if (w.done) break;
    linesearch(m, w);
    if (m.solver == 1) { w.prev_grad = w.grad; w.prev_Mgrad = w.Mgrad; }
    update_constraint(m, w);
    update_gradient(m, w);
    if (m.solver == 1) {
      T num = 0, den = 0;
      for (int i = 0; i < nv; i++) {
        num += w.grad[i] * (w.Mgrad[i] - w.prev_Mgrad[i]);
        den += w.prev_grad[i] * w.prev_Mgrad[i];
      }
      w.beta = std::max(T(0), num / std::max(T(kMinVal), den));
    }
    w.search_dot = 0;
    for (int i = 0; i < nv; i++) {
      T s = -w.Mgrad[i];
      if (m.solver == 1) s += w.beta * w.search[i];
      w.search[i] = s;
      w.search_dot += s * s;
    }
    T scale = m.meaninertia * T(std::max(1, nv));
    T improvement = (w.prev_cost - w.cost) / scale;
    T gradient = std::sqrt(w.grad_dot) / scale;
    w.done = improvement < m.tolerance || gradient < m.tolerance;
    // the reference never advances efc.solver_niter (solver.py:30 sets it to 0 and nothing
    // increments it); the count is kept separately for diagnostics
    w.iters_run++;
  }
  w.qacc_warmstart = w.qacc;
}

// forward.py:43-162
template <typename T>
void advance(const Model<T>& m, World<T>& w, const T* qacc) {
  T dt = m.timestep;
  for (int i = 0; i < m.nv; i++) w.qvel[i] = w.qvel[i] + qacc[i] * dt;
  for (int j = 0; j < m.njnt; j++) {
    int t = m.jnt_type[j], a = m.jnt_qposadr[j], d = m.jnt_dofadr[j];
    if (t == JNT_FREE) {
      for (int k = 0; k < 3; k++) w.qpos[a + k] = w.qpos[a + k] + dt * w.qvel[d + k];
      Q4<T> q{w.qpos[a + 3], w.qpos[a + 4], w.qpos[a + 5], w.qpos[a + 6]};
      Q4<T> r = quat_integrate(q, V3<T>(w.qvel[d + 3], w.qvel[d + 4], w.qvel[d + 5]), dt);
      w.qpos[a + 3] = r.w; w.qpos[a + 4] = r.x; w.qpos[a + 5] = r.y; w.qpos[a + 6] = r.z;
    } else if (t == JNT_BALL) {
      Q4<T> q{w.qpos[a], w.qpos[a + 1], w.qpos[a + 2], w.qpos[a + 3]};
      Q4<T> r = quat_integrate(q, V3<T>(w.qvel[d], w.qvel[d + 1], w.qvel[d + 2]), dt);
      w.qpos[a] = r.w; w.qpos[a + 1] = r.x; w.qpos[a + 2] = r.y; w.qpos[a + 3] = r.z;
    } else {
      w.qpos[a] = w.qpos[a] + dt * w.qvel[d];
    }
  }
}

// forward.py:165-242
template <typename T>
void euler(const Model<T>& m, World<T>& w) {
  int nv = m.nv;
  if (!(m.disableflags & DSBL_EULERDAMP)) {
    std::vector<T> M(w.qM), L(nv * nv), f(nv);
    for (int i = 0; i < nv; i++) {
      M[i * nv + i] += m.timestep * m.dof_damping[i];
      f[i] = w.qfrc_smooth[i] + w.qfrc_constraint[i];
    }
    factor_blocks(m, M, L);
    solve_blocks(m, L, w.qacc_integration.data(), f.data());
    advance(m, w, w.qacc_integration.data());
  } else {
    advance(m, w, w.qacc.data());
  }
}

// forward.py:245-405 (implicitfast, dense)
template <typename T>
void implicit(const Model<T>& m, World<T>& w) {
  int nv = m.nv;
  bool passive_on = !(m.disableflags & DSBL_PASSIVE);
  bool act_on = !(m.disableflags & DSBL_ACTUATION) && m.affine;
  if (!(passive_on || act_on)) {
    advance(m, w, w.qacc.data());
    return;
  }
  std::vector<T> qderiv(nv * nv, T(0));
  if (act_on) {
    std::vector<T> vel(m.nu);
    for (int a = 0; a < m.nu; a++) {
      T bv = m.actuator_biastype[a] == 1 ? m.actuator_biasprm[10 * a + 2] : T(0);
      T gv = m.actuator_gaintype[a] == 1 ? m.actuator_gainprm[10 * a + 2] : T(0);
      T c = m.actuator_dyntype[a] != 0 ? w.act[a] : w.ctrl[a];
      vel[a] = bv + gv * c;
    }
    for (int i = 0; i < nv; i++)
      for (int j = 0; j < nv; j++) {
        T s = 0;
        for (int a = 0; a < m.nu; a++)
          s += w.actuator_moment[a * nv + i] * vel[a] * w.actuator_moment[a * nv + j];
        qderiv[i * nv + j] = s;
      }
  }
  if (passive_on)
    for (int i = 0; i < nv; i++) qderiv[i * nv + i] -= m.dof_damping[i];
  std::vector<T> M(nv * nv), L(nv * nv), f(nv);
  for (int i = 0; i < nv * nv; i++) M[i] = w.qM[i] - qderiv[i] * m.timestep;
  for (int i = 0; i < nv; i++) f[i] = w.qfrc_smooth[i] + w.qfrc_constraint[i];
  factor_blocks(m, M, L);
  solve_blocks(m, L, w.qacc_integration.data(), f.data());
  advance(m, w, w.qacc_integration.data());
}

template <typename T>
void fwd_position(const Model<T>& m, World<T>& w) {
  kinematics(m, w);
  com_pos(m, w);
  crb(m, w);
  factor_m(m, w);
  collision(m, w);
  make_constraint(m, w);
  transmission(m, w);
}

template <typename T>
void forward(const Model<T>& m, World<T>& w, bool njmax_zero) {
  fwd_position(m, w);
  fwd_velocity(m, w);
  fwd_actuation(m, w);
  fwd_acceleration(m, w);
  if (njmax_zero) w.qacc = w.qacc_smooth;
  else solve(m, w);
}

template <typename T>
void step(const Model<T>& m, World<T>& w, bool njmax_zero) {
  forward(m, w, njmax_zero);
  if (m.integrator == 0) euler(m, w);
  else implicit(m, w);
}

enum Stage {
  ST_STEP = 0, ST_FORWARD, ST_FWD_POSITION, ST_FWD_VELOCITY, ST_FWD_ACTUATION,
  ST_FWD_ACCELERATION, ST_KINEMATICS, ST_COM_POS, ST_CRB, ST_FACTOR_M, ST_COLLISION,
  ST_NXN_BROADPHASE, ST_NARROWPHASE, ST_MAKE_CONSTRAINT, ST_TRANSMISSION, ST_COM_VEL, ST_PASSIVE,
  ST_RNE, ST_SOLVE, ST_EULER, ST_IMPLICIT, ST_FORWARD_NOSOLVE, ST_SAP_BROADPHASE
};

template <typename T>
void run_stage(const Model<T>& m, World<T>& w, int stage, bool njmax_zero) {
  switch (stage) {
    case ST_STEP: step(m, w, njmax_zero); break;
    case ST_FORWARD: forward(m, w, njmax_zero); break;
    case ST_FWD_POSITION: fwd_position(m, w); break;
    case ST_FWD_VELOCITY: fwd_velocity(m, w); break;
    case ST_FWD_ACTUATION: fwd_actuation(m, w); break;
    case ST_FWD_ACCELERATION: fwd_acceleration(m, w); break;
    case ST_KINEMATICS: kinematics(m, w); break;
    case ST_COM_POS: com_pos(m, w); break;
    case ST_CRB: crb(m, w); break;
    case ST_FACTOR_M: factor_m(m, w); break;
    case ST_COLLISION: collision(m, w); break;
    case ST_NXN_BROADPHASE: nxn_broadphase(m, w); break;
    case ST_SAP_BROADPHASE: sap_broadphase(m, w); break;
    case ST_NARROWPHASE: narrowphase(m, w); break;
    case ST_MAKE_CONSTRAINT: make_constraint(m, w); break;
    case ST_TRANSMISSION: transmission(m, w); break;
    case ST_COM_VEL: com_vel(m, w); break;
    case ST_PASSIVE: passive(m, w); break;
    case ST_RNE: rne(m, w); break;
    case ST_SOLVE: solve(m, w); break;
    case ST_EULER: euler(m, w); break;
    case ST_IMPLICIT: implicit(m, w); break;
    case ST_FORWARD_NOSOLVE:
      fwd_position(m, w); fwd_velocity(m, w); fwd_actuation(m, w); fwd_acceleration(m, w);
      break;
  }
}

struct BatchBase {
  virtual ~BatchBase() {}
  virtual int run(int stage, int nstep, int nthreads, int njmax_zero) = 0;
  virtual int field(const char* name, double* out, const double* in, int world) = 0;
  virtual int rows(const char* name, int* counts, double* out, const double* in) = 0;
  virtual int solver_scalar(const char* name, double* out) = 0;
};

template <typename T>
struct Batch : BatchBase {
  Model<T> m;
  std::vector<World<T>> w;
  Batch(const OracleModelDesc& d, int nworld) : m(d), w(nworld) {
    for (auto& x : w) x.init(m);
  }
  int run(int stage, int nstep, int nthreads, int njmax_zero) override {
    int nw = int(w.size());
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int i = 0; i < nw; i++)
      for (int s = 0; s < nstep; s++) run_stage(m, w[i], stage, njmax_zero != 0);
    return 0;
  }
  std::vector<T>* vec(World<T>& x, const std::string& n) {
    static const std::map<std::string, std::vector<T> World<T>::*> table = {
      {"qpos", &World<T>::qpos}, {"qvel", &World<T>::qvel}, {"act", &World<T>::act},
      {"ctrl", &World<T>::ctrl}, {"qacc", &World<T>::qacc},
      {"qacc_warmstart", &World<T>::qacc_warmstart}, {"qfrc_applied", &World<T>::qfrc_applied},
      {"xfrc_applied", &World<T>::xfrc_applied}, {"xpos", &World<T>::xpos},
      {"xquat", &World<T>::xquat}, {"xmat", &World<T>::xmat}, {"xipos", &World<T>::xipos},
      {"ximat", &World<T>::ximat}, {"xanchor", &World<T>::xanchor}, {"xaxis", &World<T>::xaxis},
      {"geom_xpos", &World<T>::geom_xpos}, {"geom_xmat", &World<T>::geom_xmat},
      {"site_xpos", &World<T>::site_xpos}, {"site_xmat", &World<T>::site_xmat},
      {"subtree_com", &World<T>::subtree_com}, {"cinert", &World<T>::cinert},
      {"crb", &World<T>::crb}, {"cdof", &World<T>::cdof}, {"cvel", &World<T>::cvel},
      {"cdof_dot", &World<T>::cdof_dot}, {"qM", &World<T>::qM}, {"qLD", &World<T>::qLD},
      {"actuator_length", &World<T>::actuator_length},
      {"actuator_velocity", &World<T>::actuator_velocity},
      {"actuator_force", &World<T>::actuator_force},
      {"actuator_moment", &World<T>::actuator_moment}, {"qfrc_bias", &World<T>::qfrc_bias},
      {"qfrc_spring", &World<T>::qfrc_spring}, {"qfrc_damper", &World<T>::qfrc_damper},
      {"qfrc_passive", &World<T>::qfrc_passive}, {"qfrc_actuator", &World<T>::qfrc_actuator},
      {"qfrc_smooth", &World<T>::qfrc_smooth}, {"qfrc_constraint", &World<T>::qfrc_constraint},
      {"qacc_smooth", &World<T>::qacc_smooth}, {"act_dot", &World<T>::act_dot},
      {"rne_cacc", &World<T>::rne_cacc}, {"rne_cfrc", &World<T>::rne_cfrc},
      {"qacc_integration", &World<T>::qacc_integration}, {"efc_Ma", &World<T>::Ma},
      {"efc_grad", &World<T>::grad}, {"efc_Mgrad", &World<T>::Mgrad},
      {"efc_search", &World<T>::search}, {"efc_mv", &World<T>::mv}, {"efc_h", &World<T>::h},
    };
    auto it = table.find(n);
    if (it == table.end()) return nullptr;
    return &(x.*(it->second));
  }
  // per-world fixed-size field: copy all worlds in (in != null) or out
  int field(const char* name, double* out, const double* in, int world) override {
    int lo = world < 0 ? 0 : world, hi = world < 0 ? int(w.size()) : world + 1;
    size_t off = 0;
    for (int i = lo; i < hi; i++) {
      std::vector<T>* v = vec(w[i], name);
      if (!v) return -1;
      for (size_t k = 0; k < v->size(); k++) {
        if (in) (*v)[k] = T(in[off + k]);
        if (out) out[off + k] = double((*v)[k]);
      }
      off += v->size();
    }
    return int(off);
  }
  // variable-count rows (pairs, contacts, efc): counts[world] in/out, data concatenated in world order
  int rows(const char* name_c, int* counts, double* out, const double* in) override {
    std::string name(name_c);
    size_t off = 0;
    for (size_t i = 0; i < w.size(); i++) {
      World<T>& x = w[i];
      int width = 1;
      std::vector<T>* tv = nullptr;
      std::vector<int>* iv = nullptr;
      if (name == "pair") { iv = &x.pair; width = 2; }
      else if (name == "contact_dist") { tv = &x.con_dist; }
      else if (name == "contact_pos") { tv = &x.con_pos; width = 3; }
      else if (name == "contact_frame") { tv = &x.con_frame; width = 9; }
      else if (name == "contact_includemargin") { tv = &x.con_includemargin; }
      else if (name == "contact_friction") { tv = &x.con_friction; width = 5; }
      else if (name == "contact_solref") { tv = &x.con_solref; width = 2; }
      else if (name == "contact_solimp") { tv = &x.con_solimp; width = 5; }
      else if (name == "contact_dim") { iv = &x.con_dim; }
      else if (name == "contact_geom") { iv = &x.con_geom; width = 2; }
      else if (name == "efc_J") { tv = &x.efc_J; width = m.nv; }
      else if (name == "efc_pos") { tv = &x.efc_pos; }
      else if (name == "efc_margin") { tv = &x.efc_margin; }
      else if (name == "efc_D") { tv = &x.efc_D; }
      else if (name == "efc_aref") { tv = &x.efc_aref; }
      else if (name == "efc_force") { tv = &x.efc_force; }
      else if (name == "efc_Jaref") { tv = &x.efc_Jaref; }
      else if (name == "efc_active") { iv = &x.efc_active; }
      else if (name == "efc_jv") { tv = &x.jv; }
      else if (name == "efc_quad") { tv = &x.quad; width = 3; }
      else return -1;
      if (in) {
        size_t n = size_t(counts[i]) * width;
        if (tv) { tv->resize(n); for (size_t k = 0; k < n; k++) (*tv)[k] = T(in[off + k]); }
        else { iv->resize(n); for (size_t k = 0; k < n; k++) (*iv)[k] = int(in[off + k]); }
        off += n;
      } else {
        size_t n = tv ? tv->size() : iv->size();
        counts[i] = int(n / width);
        if (out) for (size_t k = 0; k < n; k++) out[off + k] = tv ? double((*tv)[k]) : double((*iv)[k]);
        off += n;
      }
    }
    return int(off);
  }
  int solver_scalar(const char* name_c, double* out) override {
    std::string n(name_c);
    for (size_t i = 0; i < w.size(); i++) {
      World<T>& x = w[i];
      double v;
      if (n == "cost") v = x.cost;
      else if (n == "gauss") v = x.gauss;
      else if (n == "prev_cost") v = x.prev_cost;
      else if (n == "grad_dot") v = x.grad_dot;
      else if (n == "search_dot") v = x.search_dot;
      else if (n == "alpha") v = x.alpha;
      else if (n == "gtol") v = x.gtol;
      else if (n == "solver_niter") v = x.solver_niter;
      else if (n == "iters_run") v = x.iters_run;
      else if (n == "done") v = x.done;
      else return -1;
      out[i] = v;
    }
    return int(w.size());
  }
};

}  // namespace

extern "C" {

// Creates a batch of nworld worlds at qpos0 computing in float (precision 32) or double (64).
void* oracle_create(const OracleModelDesc* desc, int nworld, int precision) {
  if (precision == 64) return new Batch<double>(*desc, nworld);
  return new Batch<float>(*desc, nworld);
}
void oracle_destroy(void* b) { delete static_cast<BatchBase*>(b); }
// Runs `stage` (enum Stage) nstep times on every world; nthreads <= 0 keeps the OpenMP default.
int oracle_run(void* b, int stage, int nstep, int nthreads, int njmax_zero) {
  return static_cast<BatchBase*>(b)->run(stage, nstep, nthreads, njmax_zero);
}
// Gets (out) and/or sets (in) a fixed-size per-world field; world < 0 means all worlds.
int oracle_field(void* b, const char* name, double* out, const double* in, int world) {
  return static_cast<BatchBase*>(b)->field(name, out, in, world);
}
// Gets or sets variable-length per-world rows (pairs, contacts, efc rows).
int oracle_rows(void* b, const char* name, int* counts, double* out, const double* in) {
  return static_cast<BatchBase*>(b)->rows(name, counts, out, in);
}
int oracle_solver_scalar(void* b, const char* name, double* out) {
  return static_cast<BatchBase*>(b)->solver_scalar(name, out);
}
// Closest points between two segments (math.py:209-242), double precision, for the known-answer
// tests of math_test.py.
void oracle_closest_segments(const double* a0, const double* a1, const double* b0, const double* b1,
                             double* pa, double* pb, int precision) {
  if (precision == 32) {
    V3<float> A0(a0[0], a0[1], a0[2]), A1(a1[0], a1[1], a1[2]), B0(b0[0], b0[1], b0[2]),
        B1(b1[0], b1[1], b1[2]), PA, PB;
    closest_segment_to_segment_points(A0, A1, B0, B1, PA, PB);
    for (int k = 0; k < 3; k++) { pa[k] = PA[k]; pb[k] = PB[k]; }
  } else {
    V3<double> A0(a0[0], a0[1], a0[2]), A1(a1[0], a1[1], a1[2]), B0(b0[0], b0[1], b0[2]),
        B1(b1[0], b1[1], b1[2]), PA, PB;
    closest_segment_to_segment_points(A0, A1, B0, B1, PA, PB);
    for (int k = 0; k < 3; k++) { pa[k] = PA[k]; pb[k] = PB[k]; }
  }
}

}  // extern "C"
