// Pieces of the analytic qpos adjoint of one step (no counterpart in the reference, whose API has
// no derivatives).  Every qpos dependence of the step reaches the dynamics through a few position
// quantities: the motion subspaces cdof, the body inertias cinert, the roots' subtree_com, the
// contact geometry (position, frame, distance) and the rows' impedance.  The routines below turn
// adjoint vectors into bars on those quantities, the bars into per-body force / torque pairs
// (F, T about the world origin: a point x with bar xb adds F += xb, T += x x xb; a direction u
// with bar ub adds T += u x ub), and those into the tangent-space qpos gradient by one reverse
// walk over the joints.
#pragma once

#include "mjb_solver.cuh"

namespace mjb {

// ---------------------------------------------------------------------------------------------
// Forward-mode dual numbers for the contact geometry: one lane carries the tangent of one of the
// 12 pose directions of a contact's two geoms (translation / world rotation about the geom's
// origin, per axis) through the narrowphase formulas, taking the same branches as the forward
// by value.

struct Dl {
  float v, d;
};
__device__ __forceinline__ Dl dc(float v) { return Dl{v, 0.f}; }
__device__ __forceinline__ Dl operator+(Dl a, Dl b) { return Dl{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dl operator-(Dl a, Dl b) { return Dl{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dl operator-(Dl a) { return Dl{-a.v, -a.d}; }
__device__ __forceinline__ Dl operator*(Dl a, Dl b) { return Dl{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dl operator*(Dl a, float s) { return Dl{a.v * s, a.d * s}; }
__device__ __forceinline__ Dl operator/(Dl a, Dl b) {
  const float q = a.v / b.v;
  return Dl{q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dl dsqrt(Dl a) {
  const float s = sqrtf(a.v);
  return Dl{s, s > 0.f ? a.d * 0.5f / s : 0.f};
}
__device__ __forceinline__ Dl dclamp(Dl a, float lo, float hi) {  // fminf(fmaxf(a, lo), hi)
  if (!(a.v > lo)) return dc(lo);
  if (!(a.v < hi)) return dc(hi);
  return a;
}
__device__ __forceinline__ Dl dclamp(Dl a, Dl lo, Dl hi) {
  if (!(a.v > lo.v)) a = lo;
  if (!(a.v < hi.v)) a = hi;
  return a;
}

struct D3 {
  Dl x, y, z;
};
__device__ __forceinline__ D3 dc3(f3 a) { return D3{dc(a.x), dc(a.y), dc(a.z)}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, Dl s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator*(D3 a, float s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Dl ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
  return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ Dl dlength(D3 a) { return dsqrt(ddot(a, a)); }
__device__ __forceinline__ D3 dnormalize(D3 a) {
  const Dl l = dlength(a);
  return l.v > 0.f ? a * (dc(1.f) / l) : dc3(mk3(0.f, 0.f, 0.f));
}
__device__ __forceinline__ f3 val(D3 a) { return mk3(a.x.v, a.y.v, a.z.v); }
__device__ __forceinline__ f3 tan3(D3 a) { return mk3(a.x.d, a.y.d, a.z.d); }

// frame rows (normal, first tangent, second tangent), as make_frame
struct DFrame {
  D3 r[3];
};
__device__ DFrame dmake_frame(D3 a) {
  a = dnormalize(a);
  D3 b = (-0.5f < a.y.v && a.y.v < 0.5f) ? dc3(mk3(0.f, 1.f, 0.f)) : dc3(mk3(0.f, 0.f, 1.f));
  b = b - a * ddot(a, b);
  b = dnormalize(b);
  if (dlength(a).v == 0.f) b = dc3(mk3(0.f, 0.f, 0.f));
  return DFrame{{a, b, dcross(a, b)}};
}
__device__ D3 dclosest_segment_point(D3 a, D3 b, D3 pt) {
  const D3 ab = b - a;
  Dl t = ddot(pt - a, ab) / (ddot(ab, ab) + dc(1e-6f));
  t = dclamp(t, 0.f, 1.f);
  return a + ab * t;
}
__device__ void dclosest_segment_to_segment_points(D3 a0, D3 a1, D3 b0, D3 b1, D3& pa, D3& pb) {
  const D3 da = a1 - a0, db = b1 - b0;
  const Dl la = dlength(da), lb = dlength(db);
  const D3 dir_a = la.v == 0.f ? da : da * (dc(1.f) / la);
  const D3 dir_b = lb.v == 0.f ? db : db * (dc(1.f) / lb);
  const Dl ha = la * 0.5f, hb = lb * 0.5f;
  const D3 amid = a0 + dir_a * ha, bmid = b0 + dir_b * hb;
  const D3 trans = amid - bmid;
  const Dl dd = ddot(dir_a, dir_b), dat = ddot(dir_a, trans), dbt = ddot(dir_b, trans);
  const Dl denom = dc(1.f) - dd * dd;
  const Dl ta0 = (-dat + dd * dbt) / (denom + dc(1e-6f));
  const Dl tb0 = dbt + ta0 * dd;
  const Dl ta = dclamp(ta0, -ha, ha), tb = dclamp(tb0, -hb, hb);
  const D3 best_a = amid + dir_a * ta, best_b = bmid + dir_b * tb;
  const D3 na = dclosest_segment_point(a0, a1, best_b);
  const D3 nb = dclosest_segment_point(b0, b1, best_a);
  const Dl d1 = ddot(best_b - na, best_b - na), d2 = ddot(best_a - nb, best_a - nb);
  if (d1.v < d2.v) {
    pa = na;
    pb = best_b;
  } else {
    pa = best_a;
    pb = nb;
  }
}

struct DContact {
  Dl dist;
  D3 pos;
  DFrame frame;
};
__device__ __forceinline__ void dplane_sphere(D3 n, D3 ppos, D3 spos, Dl r, DContact& c) {
  c.dist = ddot(spos - ppos, n) - r;
  c.pos = spos - n * (r + c.dist * 0.5f);
}
__device__ __forceinline__ void dsphere_sphere(D3 p1, Dl r1, D3 p2, Dl r2, DContact& c) {
  const D3 dir = p2 - p1;
  Dl dist = dlength(dir);
  const D3 n = dist.v == 0.f ? dc3(mk3(1.f, 0.f, 0.f)) : dir * (dc(1.f) / dist);
  dist = dist - (r1 + r2);
  c.dist = dist;
  c.pos = p1 + n * (r1 + dist * 0.5f);
  c.frame = dmake_frame(n);
}

// Candidate j of the narrowphase of one geom pair (narrow_pair's formulas and branches), the two
// geom poses given as dual numbers.  Returns false when the pair has no candidate j.
__device__ bool dcontact_candidate(const MjbModel& m, int g1, int g2, D3 p1, const D3* R1, D3 p2,
                                   const D3* R2, float margin, int j, DContact& c) {
  // R1 / R2: the columns of the geoms' rotation matrices
  const int t1 = m.geom_type[g1], t2 = m.geom_type[g2];
  const f3 sz1 = ld3(m.geom_size + 3 * g1), sz2 = ld3(m.geom_size + 3 * g2);
  const D3 n1 = R1[2];
  if (t1 == GEOM_PLANE && t2 == GEOM_SPHERE) {
    if (j != 0) return false;
    dplane_sphere(n1, p1, p2, dc(sz2.x), c);
    c.frame = dmake_frame(n1);
    return true;
  }
  if (t1 == GEOM_SPHERE && t2 == GEOM_SPHERE) {
    if (j != 0) return false;
    dsphere_sphere(p1, dc(sz1.x), p2, dc(sz2.x), c);
    return true;
  }
  if (t1 == GEOM_PLANE && t2 == GEOM_CAPSULE) {
    if (j > 1) return false;
    const D3 n = n1, axis = R2[2];
    const D3 bv = axis - n * ddot(n, axis);
    const Dl bn = dlength(bv);
    D3 b = bn.v == 0.f ? bv : bv * (dc(1.f) / bn);
    if (bn.v < 0.5f)
      b = (-0.5f < n.y.v && n.y.v < 0.5f) ? dc3(mk3(0.f, 1.f, 0.f)) : dc3(mk3(0.f, 0.f, 1.f));
    c.frame = DFrame{{n, b, dcross(n, b)}};
    const D3 seg = axis * sz2.y;
    dplane_sphere(n, p1, j == 0 ? p2 + seg : p2 - seg, dc(sz2.x), c);
    return true;
  }
  if (t1 == GEOM_PLANE && t2 == GEOM_BOX) {
    const Dl dist = ddot(p2 - p1, n1);
    int cnt = 0;
    for (int i = 0; i < 8; i++) {
      const float cx = (i & 1) ? sz2.x : -sz2.x, cy = (i & 2) ? sz2.y : -sz2.y;
      const float cz = (i & 4) ? sz2.z : -sz2.z;
      const D3 corner = R2[0] * cx + R2[1] * cy + R2[2] * cz;
      const Dl ldist = ddot(n1, corner);
      if (dist.v + ldist.v > margin || ldist.v > 0.f) continue;
      if (cnt == j) {
        c.dist = dist + ldist;
        c.pos = corner + p2 + n1 * (c.dist * -0.5f);
        c.frame = dmake_frame(n1);
        return true;
      }
      if (++cnt >= 4) break;
    }
    return false;
  }
  if (t1 == GEOM_CAPSULE && t2 == GEOM_CAPSULE) {
    if (j != 0) return false;
    const D3 s1 = R1[2] * sz1.y, s2 = R2[2] * sz2.y;
    D3 pa, pb;
    dclosest_segment_to_segment_points(p1 - s1, p1 + s1, p2 - s2, p2 + s2, pa, pb);
    dsphere_sphere(pa, dc(sz1.x), pb, dc(sz2.x), c);
    return true;
  }
  return false;
}

// Pose bars of contact c's two geoms from the bars of its distance, position and frame rows:
// lane k < 12 differentiates along pose direction k (geom k / 6; translation for k % 6 < 3, else
// rotation about world axis k % 3), the candidate whose position matches the stored contact is
// taken, and the lane returns d(dist, pos, frame) / d(direction k) . bars.
__device__ float contact_pose_bar(const MjbModel& m, const MjbData& d, int w, int c, float distb,
                                  f3 posb, const float* frameb, int lane) {
  const int g1 = d.contact_geom[2 * c], g2 = d.contact_geom[2 * c + 1];
  const float* gxpos = d.geom_xpos + W(w, 3 * m.ngeom);
  const float* gxmat = d.geom_xmat + W(w, 9 * m.ngeom);
  const float margin = fmaxf(m.geom_margin[g1], m.geom_margin[g2]);
  const int k = lane % 12, gsel = k / 6, axis = k % 3;
  const bool rot = (k % 6) >= 3, seed = lane < 12;
  D3 P[2], R[2][3];
  for (int s = 0; s < 2; s++) {
    const int g = s == 0 ? g1 : g2;
    const f3 p = ld3(gxpos + 3 * g);
    const m33 mat = ld9(gxmat + 9 * g);
    const bool mine = seed && gsel == s;
    const f3 e = mk3(axis == 0 ? 1.f : 0.f, axis == 1 ? 1.f : 0.f, axis == 2 ? 1.f : 0.f);
    const f3 dp = (mine && !rot) ? e : mk3(0.f, 0.f, 0.f);
    P[s] = D3{Dl{p.x, dp.x}, Dl{p.y, dp.y}, Dl{p.z, dp.z}};
    for (int cc = 0; cc < 3; cc++) {
      const f3 u = col(mat, cc);
      const f3 du = (mine && rot) ? cross(e, u) : mk3(0.f, 0.f, 0.f);
      R[s][cc] = D3{Dl{u.x, du.x}, Dl{u.y, du.y}, Dl{u.z, du.z}};
    }
  }
  const f3 cpos = ld3(d.contact_pos + 3 * c);
  DContact best, cand;
  float bestd = 3.4e38f;
  for (int j = 0; j < 8; j++) {
    if (!dcontact_candidate(m, g1, g2, P[0], R[0], P[1], R[1], margin, j, cand)) break;
    const f3 dp = val(cand.pos) - cpos;
    const float dd = dot(dp, dp);
    if (dd < bestd) {
      bestd = dd;
      best = cand;
    }
  }
  if (!seed || bestd == 3.4e38f) return 0.f;
  float g = best.dist.d * distb + dot(tan3(best.pos), posb);
  for (int r = 0; r < 3; r++) g += dot(tan3(best.frame.r[r]), ld3(frameb + 3 * r));
  return g;
}

// ---------------------------------------------------------------------------------------------
// Constraint row parameters (constraint.py:22-73 restated) with the impedance's derivative.

struct EfcPar {
  float k, b, imp, dimp;  // stiffness, damping, impedance, d imp / d pos
};
__device__ EfcPar efc_params(const MjbModel& m, const float* solref, const float* solimp, float pos,
                             bool refsafe) {
  float timeconst = solref[0], dampratio = solref[1];
  float dmin = solimp[0], dmax = solimp[1], width = solimp[2], mid = solimp[3], power = solimp[4];
  if (refsafe) timeconst = fmaxf(timeconst, 2.f * m.timestep);
  dmin = fminf(fmaxf(dmin, kMinImp), kMaxImp);
  dmax = fminf(fmaxf(dmax, kMinImp), kMaxImp);
  width = fmaxf(kMinVal, width);
  mid = fminf(fmaxf(mid, kMinImp), kMaxImp);
  power = fmaxf(1.f, power);
  EfcPar p;
  p.k = 1.f / (dmax * dmax * timeconst * timeconst * dampratio * dampratio);
  p.b = 2.f / (dmax * timeconst);
  if (solref[0] <= 0.f) p.k = -solref[0] / (dmax * dmax);
  if (solref[1] <= 0.f) p.b = -solref[1] / dmax;
  const float imp_x = fabsf(pos) / width;
  if (imp_x > 1.f) {
    p.imp = dmax;
    p.dimp = 0.f;
    return p;
  }
  float imp_y, dy;
  if (imp_x < mid) {
    const float a = 1.f / powf(mid, power - 1.f);
    imp_y = a * powf(imp_x, power);
    dy = a * power * powf(imp_x, power - 1.f);
  } else {
    const float a = 1.f / powf(1.f - mid, power - 1.f);
    imp_y = 1.f - a * powf(1.f - imp_x, power);
    dy = a * power * powf(1.f - imp_x, power - 1.f);
  }
  const float imp = dmin + imp_y * (dmax - dmin);
  p.imp = fminf(fmaxf(imp, dmin), dmax);
  const bool inside = imp > dmin && imp < dmax;
  p.dimp = inside ? dy * (dmax - dmin) * (pos < 0.f ? -1.f : 1.f) / width : 0.f;
  return p;
}

// d (a' I(c) b) / d c accumulated into cb (10), I(c) the 6x6 map of inert_vec
__device__ __forceinline__ void inert_bilin_add(float* cb, const s6& a, const s6& b) {
  const float* x = a.v;
  const float* y = b.v;
  cb[0] += x[0] * y[0];
  cb[1] += x[1] * y[1];
  cb[2] += x[2] * y[2];
  cb[3] += x[0] * y[1] + x[1] * y[0];
  cb[4] += x[0] * y[2] + x[2] * y[0];
  cb[5] += x[1] * y[2] + x[2] * y[1];
  cb[6] += -x[1] * y[5] + x[2] * y[4] + x[4] * y[2] - x[5] * y[1];
  cb[7] += x[0] * y[5] - x[2] * y[3] - x[3] * y[2] + x[5] * y[0];
  cb[8] += -x[0] * y[4] + x[1] * y[3] + x[3] * y[1] - x[4] * y[0];
  cb[9] += x[3] * y[3] + x[4] * y[4] + x[5] * y[5];
}

__device__ __forceinline__ s6 s6add(const s6& a, const s6& b) {
  s6 r;
#pragma unroll
  for (int k = 0; k < 6; k++) r.v[k] = a.v[k] + b.v[k];
  return r;
}
__device__ __forceinline__ s6 s6axpy(float s, const s6& a, const s6& b) {  // s a + b
  s6 r;
#pragma unroll
  for (int k = 0; k < 6; k++) r.v[k] = s * a.v[k] + b.v[k];
  return r;
}
__device__ __forceinline__ void add6(float* p, const s6& a) {
#pragma unroll
  for (int k = 0; k < 6; k++) p[k] += a.v[k];
}

// U_b = sum of u_i cdof_i over the dofs from the root to body b (a top-down sweep)
__device__ void tree_sum_down(const MjbModel& m, const float* cdof, const float* u, float* U,
                              int lane) {
  if (lane < 6) U[lane] = 0.f;
  __syncwarp();
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += 32) {
      const int b = m.body_tree[n];
      s6 acc = ld6(U + 6 * m.body_parentid[b]);
      const int da = m.body_dofadr[b];
      for (int i = 0; i < m.body_dofnum[b]; i++) acc = s6axpy(u[da + i], ld6(cdof + 6 * (da + i)), acc);
      st6(U + 6 * b, acc);
    }
    __syncwarp();
  }
}
// A_b += sum of A over b's children, deepest level first: subtree sums (body 0 untouched)
__device__ void tree_sum_up(const MjbModel& m, float* A, int lane) {
  for (int lvl = m.nlevel - 1; lvl >= 1; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += 32) {
      const int b = m.body_tree[n];
      s6 acc = ld6(A + 6 * b);
      const int ca = m.body_childadr[b], cn = m.body_childnum[b];
      for (int c = 0; c < cn; c++) acc = s6add(acc, ld6(A + 6 * m.body_child[ca + c]));
      st6(A + 6 * b, acc);
    }
    __syncwarp();
  }
}

// Bars of u' M(q) x: with U_b, X_b the tree sums of u and x, u' M x = sum_b U_b . I_b X_b, so
// cinert_b gets d(U_b' I X_b)/dc and cdof_i gets u_i (subtree sum of I X) + x_i (of I U).
// Scratch: SA..SD, 6 nbody floats each.
__device__ void mass_product_bars(const MjbModel& m, const MjbData& d, int w, int lane,
                                  const float* u, const float* x, float* cdof_bar, float* cinert_bar,
                                  float* SA, float* SB, float* SC, float* SD) {
  const int nb = m.nbody, nv = m.nv;
  const float* cdof = d.cdof + W(w, 6 * nv);
  const float* cinert = d.cinert + W(w, 10 * nb);
  tree_sum_down(m, cdof, u, SA, lane);
  tree_sum_down(m, cdof, x, SB, lane);
  for (int b = lane; b < nb; b += 32) {
    if (b == 0) {
      for (int k = 0; k < 6; k++) SC[k] = SD[k] = 0.f;
      continue;
    }
    const s6 U = ld6(SA + 6 * b), X = ld6(SB + 6 * b);
    st6(SC + 6 * b, inert_vec(cinert + 10 * b, U));
    st6(SD + 6 * b, inert_vec(cinert + 10 * b, X));
    inert_bilin_add(cinert_bar + 10 * b, U, X);
  }
  __syncwarp();
  tree_sum_up(m, SC, lane);
  tree_sum_up(m, SD, lane);
  for (int i = lane; i < nv; i += 32) {
    const int b = m.dof_bodyid[i];
    add6(cdof_bar + 6 * i, s6axpy(u[i], ld6(SD + 6 * b), s6axpy(x[i], ld6(SC + 6 * b), s6{})));
  }
  __syncwarp();
}

// Bars of u' qfrc_bias(q, v) on cdof and cinert (v = qv, the step's starting velocity): the
// com_vel / rne recursions of the forward run backwards (see rne_vel_vjp for the velocity part).
__device__ void bias_q_bars(const MjbModel& m, const MjbData& d, int w, int lane, const float* u,
                            const float* qv, float* cdof_bar, float* cinert_bar, float* SA, float* SB,
                            float* SC) {
  const int nb = m.nbody, nv = m.nv;
  const float* cdof = d.cdof + W(w, 6 * nv);
  const float* cvel = d.cvel + W(w, 6 * nb);
  const float* cacc = d.rne_cacc + W(w, 6 * nb);
  const float* cfrc = d.rne_cfrc + W(w, 6 * nb);
  const float* cinert = d.cinert + W(w, 10 * nb);
  tree_sum_down(m, cdof, u, SA, lane);
  for (int b = lane; b < nb; b += 32) {
    if (b == 0) {
      for (int k = 0; k < 6; k++) SB[k] = SC[k] = 0.f;
      continue;
    }
    const s6 U = ld6(SA + 6 * b), V = ld6(cvel + 6 * b);
    const float* I = cinert + 10 * b;
    st6(SB + 6 * b, inert_vec(I, U));
    const s6 uxv = motion_cross(U, V);
    const s6 a = inert_vec(I, uxv);
    const s6 c = motion_cross_force(U, inert_vec(I, V));
    s6 r;
    for (int k = 0; k < 6; k++) r.v[k] = a.v[k] - c.v[k];
    st6(SC + 6 * b, r);
    inert_bilin_add(cinert_bar + 10 * b, U, ld6(cacc + 6 * b));
    inert_bilin_add(cinert_bar + 10 * b, uxv, V);
  }
  __syncwarp();
  for (int lvl = m.nlevel - 1; lvl >= 1; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += 32) {
      const int b = m.body_tree[n];
      s6 g = ld6(SB + 6 * b), r = ld6(SC + 6 * b);
      const int ca = m.body_childadr[b], cn = m.body_childnum[b];
      for (int c = 0; c < cn; c++) {
        const int ch = m.body_child[ca + c];
        g = s6add(g, ld6(SB + 6 * ch));
        r = s6add(r, ld6(SC + 6 * ch));
      }
      st6(SB + 6 * b, g);
      const s6 ftot = ld6(cfrc + 6 * b);
      s6 V = ld6(cvel + 6 * b);  // the body velocity after the joint being undone
      const int j0 = m.body_jntadr[b];
      int dof_end = m.body_dofadr[b] + m.body_dofnum[b];
      for (int j = j0 + m.body_jntnum[b] - 1; j >= j0; j--) {
        const int t = m.jnt_type[j];
        const int nd = t == JNT_FREE ? 6 : (t == JNT_BALL ? 3 : 1);
        const int dof = dof_end - nd;
        const int rot = t == JNT_FREE ? 3 : 0;
        s6 Vpre = V;
        for (int i = dof + rot; i < dof_end; i++) Vpre = s6axpy(-qv[i], ld6(cdof + 6 * i), Vpre);
        const s6 vg = motion_cross_force(Vpre, g);
        s6 acc{};
        for (int i = dof + rot; i < dof_end; i++) {
          const s6 c = ld6(cdof + 6 * i);
          s6 bar = s6axpy(u[i], ftot, s6axpy(qv[i], r, s6{}));
          bar = s6axpy(-qv[i], vg, bar);
          add6(cdof_bar + 6 * i, bar);
          acc = s6axpy(qv[i], motion_cross_force(c, g), acc);
        }
        r = s6add(r, acc);
        V = Vpre;
        for (int i = dof; i < dof + rot; i++) {
          add6(cdof_bar + 6 * i, s6axpy(u[i], ftot, s6axpy(qv[i], r, s6{})));
          V = s6axpy(-qv[i], ld6(cdof + 6 * i), V);
        }
        dof_end = dof;
      }
      st6(SC + 6 * b, r);
    }
    __syncwarp();
  }
}

// Row terms: for the active rows i (joint limits first, then 4 pyramid rows per active condim-3
// contact, make_constraint's order), with t_i = J_i s and e_i = aref_i - J_i qacc (= -Jaref_i),
//   dD_i t_i e_i + D_i t_i daref_i + D_i dJ_i . (e_i s - t_i qacc - b_i t_i v).
// A limit row's pos moves with its dof (d pos / d q = J); a contact row's J moves with cdof, the
// contact position and frame and the roots' subtree_com, and its pos with the contact distance.
// Writes: Q (limits), cdof_bar, and for contacts BF / BT of the geoms' bodies and SCB (bars of
// subtree_com[root(b)] kept in body b's slot).
// With GV non-null the rows' velocity term -D_i b_i J_i (J_i s) of d loss / d qvel is subtracted
// from GV (per dof) as well; with cdof_bar null only that is done.
__device__ void row_q_bars(const MjbModel& m, const MjbData& d, int w, int lane, const float* S,
                           const float* qv, float* Q, float* cdof_bar, float* BF, float* BT,
                           float* SCB, float* GV) {
  const bool posq = cdof_bar != nullptr;
  const int nv = m.nv;
  const int adr = d.world_efcadr[w], n = d.world_nefc[w];
  if (n == 0) return;
  const bool on = !(m.disableflags & DSBL_CONSTRAINT);
  const bool do_con = on && !(m.disableflags & DSBL_CONTACT) && m.cone == 0;
  const bool refsafe = !(m.disableflags & DSBL_REFSAFE);
  const int ca = d.world_conadr[w], nc = d.world_ncon[w];
  auto con_active = [&](int c) {
    return d.contact_dim[c] == 3 && (d.contact_dist[c] - d.contact_includemargin[c]) < 0.f;
  };
  int ncact = 0;
  if (do_con)
    for (int base = 0; base < nc; base += 32)
      ncact += __popc(__ballot_sync(0xffffffffu, base + lane < nc && con_active(ca + base + lane)));
  const int nlim = n - 4 * ncact;
  if (nlim < 0) return;
  const float* qacc = d.qacc + W(w, nv);
  for (int k = 0; k < nlim; k++) {
    const int r = adr + k;
    if (!d.efc_active[r] || d.efc_D[r] == 0.f) continue;
    const float* J = d.efc_J + size_t(r) * nv;
    int dof = -1;
    for (int base = 0; base < nv; base += 32) {
      const unsigned msk = __ballot_sync(0xffffffffu, base + lane < nv && J[base + lane] != 0.f);
      if (msk && dof < 0) dof = base + __ffs(msk) - 1;
    }
    if (dof >= 0 && lane == 0) {
      const float Js = J[dof];
      const int j = m.dof_jntid[dof];
      const float pos = d.efc_pos[r] - d.efc_margin[r];
      const EfcPar p = efc_params(m, m.jnt_solref + 2 * j, m.jnt_solimp + 5 * j, pos, refsafe);
      const float D = d.efc_D[r], t = Js * S[dof], e = -d.efc_Jaref[r];
      if (GV) GV[dof] -= D * p.b * t * Js;
      if (posq) {
        const float dD = D / (p.imp * (1.f - p.imp)) * p.dimp;
        const float posb = dD * t * e - D * t * p.k * (p.imp + pos * p.dimp);
        Q[dof] += posb * Js;
      }
    }
    __syncwarp();
  }
  __syncwarp();
  if (!do_con || ncact == 0) return;
  const float* cdof = d.cdof + W(w, 6 * nv);
  const float* sc = d.subtree_com + W(w, 3 * m.nbody);
  int r = adr + nlim;
  for (int k = 0; k < nc; k++) {
    const int c = ca + k;
    if (!con_active(c)) continue;
    const int r0 = r;
    r += 4;
    float D[4], t[4], ee[4];
    bool any = false;
    for (int e = 0; e < 4; e++) {
      const bool act = d.efc_active[r0 + e] && d.efc_D[r0 + e] != 0.f;
      const float* J = d.efc_J + size_t(r0 + e) * nv;
      float part = 0.f;
      for (int i = lane; i < nv; i += 32) part += J[i] * S[i];
      t[e] = warp_sum(part);
      D[e] = act ? d.efc_D[r0 + e] : 0.f;
      ee[e] = -d.efc_Jaref[r0 + e];
      any |= act;
    }
    if (!any) continue;
    const float pos = d.contact_dist[c] - d.contact_includemargin[c];
    const EfcPar p = efc_params(m, d.contact_solref + 2 * c, d.contact_solimp + 5 * c, pos, refsafe);
    if (GV) {
      for (int i = lane; i < nv; i += 32) {
        float g = 0.f;
        for (int e = 0; e < 4; e++) g += D[e] * t[e] * d.efc_J[size_t(r0 + e) * nv + i];
        GV[i] -= p.b * g;
      }
    }
    if (!posq) continue;
    float posb = 0.f;
    for (int e = 0; e < 4; e++) {
      if (D[e] == 0.f) continue;
      const float dD = D[e] / (p.imp * (1.f - p.imp)) * p.dimp;
      posb += dD * t[e] * ee[e] - D[e] * t[e] * p.k * (p.imp + pos * p.dimp);
    }
    const int b1 = m.geom_bodyid[d.contact_geom[2 * c]], b2 = m.geom_bodyid[d.contact_geom[2 * c + 1]];
    const float* fr = d.contact_frame + 9 * c;
    const f3 nrm = ld3(fr), t1 = ld3(fr + 3), t2 = ld3(fr + 6);
    const float mu0 = d.contact_friction[5 * c], mu1 = d.contact_friction[5 * c + 1];
    const f3 dir[4] = {nrm + t1 * mu0, nrm - t1 * mu0, nrm + t2 * mu1, nrm - t2 * mu1};
    const f3 cp = ld3(d.contact_pos + 3 * c);
    const f3 off1 = cp - ld3(sc + 3 * m.body_rootid[b1]);
    const f3 off2 = cp - ld3(sc + 3 * m.body_rootid[b2]);
    f3 db[4] = {mk3(0, 0, 0), mk3(0, 0, 0), mk3(0, 0, 0), mk3(0, 0, 0)};
    f3 o1b = mk3(0, 0, 0), o2b = mk3(0, 0, 0);
    for (int i = lane; i < nv; i += 32) {
      const s6 cd = ld6(cdof + 6 * i);
      const f3 ang{cd.v[0], cd.v[1], cd.v[2]}, lin{cd.v[3], cd.v[4], cd.v[5]};
      const int dbd = m.dof_bodyid[i];
      const float in1 = (dbd != 0 && dbd <= b1 && b1 < m.body_subtreeend[dbd]) ? 1.f : 0.f;
      const float in2 = (dbd != 0 && dbd <= b2 && b2 < m.body_subtreeend[dbd]) ? 1.f : 0.f;
      if (in1 == in2) continue;  // the dof moves both bodies or neither: its J entries are 0
      const f3 jd = (lin + cross(ang, off2)) * in2 - (lin + cross(ang, off1)) * in1;
      f3 ab = mk3(0, 0, 0), lb = mk3(0, 0, 0);
      for (int e = 0; e < 4; e++) {
        if (D[e] == 0.f) continue;
        const float cw = D[e] * (ee[e] * S[i] - t[e] * qacc[i] - p.b * t[e] * qv[i]);
        lb = lb + dir[e] * (cw * (in2 - in1));
        ab = ab + (cross(off2, dir[e]) * in2 - cross(off1, dir[e]) * in1) * cw;
        db[e] = db[e] + jd * cw;
        const f3 da = cross(dir[e], ang) * cw;
        o2b = o2b + da * in2;
        o1b = o1b - da * in1;
      }
      float* cb = cdof_bar + 6 * i;
      cb[0] += ab.x; cb[1] += ab.y; cb[2] += ab.z;
      cb[3] += lb.x; cb[4] += lb.y; cb[5] += lb.z;
    }
    for (int e = 0; e < 4; e++) db[e] = mk3(warp_sum(db[e].x), warp_sum(db[e].y), warp_sum(db[e].z));
    o1b = mk3(warp_sum(o1b.x), warp_sum(o1b.y), warp_sum(o1b.z));
    o2b = mk3(warp_sum(o2b.x), warp_sum(o2b.y), warp_sum(o2b.z));
    const f3 nb = db[0] + db[1] + db[2] + db[3];
    const f3 t1b = (db[0] - db[1]) * mu0, t2b = (db[2] - db[3]) * mu1;
    const float frameb[9] = {nb.x, nb.y, nb.z, t1b.x, t1b.y, t1b.z, t2b.x, t2b.y, t2b.z};
    const float g = contact_pose_bar(m, d, w, c, posb, o1b + o2b, frameb, lane);
    float gs[12];
    for (int q = 0; q < 12; q++) gs[q] = __shfl_sync(0xffffffffu, g, q);
    if (lane == 0) {
      float* s1 = SCB + 3 * b1;
      float* s2 = SCB + 3 * b2;
      s1[0] -= o1b.x; s1[1] -= o1b.y; s1[2] -= o1b.z;
      s2[0] -= o2b.x; s2[1] -= o2b.y; s2[2] -= o2b.z;
      const float* gxpos = d.geom_xpos + W(w, 3 * m.ngeom);
      for (int sgeom = 0; sgeom < 2; sgeom++) {
        const int gg = d.contact_geom[2 * c + sgeom], bb = m.geom_bodyid[gg];
        const f3 pb = mk3(gs[6 * sgeom], gs[6 * sgeom + 1], gs[6 * sgeom + 2]);
        const f3 tb = mk3(gs[6 * sgeom + 3], gs[6 * sgeom + 4], gs[6 * sgeom + 5]);
        const f3 tq = cross(ld3(gxpos + 3 * gg), pb) + tb;
        BF[3 * bb] += pb.x; BF[3 * bb + 1] += pb.y; BF[3 * bb + 2] += pb.z;
        BT[3 * bb] += tq.x; BT[3 * bb + 1] += tq.y; BT[3 * bb + 2] += tq.z;
      }
    }
    __syncwarp();
  }
}

// cdof bars -> bars of the joints' anchors (JA) and axes (JX), of the roots' subtree_com (JS, per
// joint) and torques of the body frames whose columns free / ball cdof use (BT).  com_pos: a hinge
// has cdof = (axis; axis x off), a slide (0; axis), a free / ball rotational dof (x_k; x_k x off)
// with x_k the body frame's column k, off = subtree_com[root] - anchor.
__device__ void cdof_joint_bars(const MjbModel& m, const MjbData& d, int w, int lane,
                                const float* cdof_bar, float* JA, float* JX, float* JS, float* BT) {
  const float* xmat = d.xmat + W(w, 9 * m.nbody);
  const float* xanchor = d.xanchor + W(w, 3 * m.njnt);
  const float* xaxis = d.xaxis + W(w, 3 * m.njnt);
  const float* sc = d.subtree_com + W(w, 3 * m.nbody);
  for (int j = lane; j < m.njnt; j += 32) {
    const int b = m.jnt_bodyid[j], dof = m.jnt_dofadr[j], t = m.jnt_type[j];
    const f3 off = ld3(sc + 3 * m.body_rootid[b]) - ld3(xanchor + 3 * j);
    f3 ja = mk3(0, 0, 0), jx = mk3(0, 0, 0), js = mk3(0, 0, 0), bt = mk3(0, 0, 0);
    if (t == JNT_FREE || t == JNT_BALL) {
      const m33 xm = ld9(xmat + 9 * b);
      const int d0 = t == JNT_FREE ? dof + 3 : dof;
      for (int k = 0; k < 3; k++) {
        const float* cb = cdof_bar + 6 * (d0 + k);
        const f3 ab = ld3(cb), lb = ld3(cb + 3), c = col(xm, k);
        bt = bt + cross(c, ab + cross(off, lb));
        js = js + cross(lb, c);
        ja = ja - cross(lb, c);
      }
    } else if (t == JNT_SLIDE) {
      jx = ld3(cdof_bar + 6 * dof + 3);
    } else {
      const float* cb = cdof_bar + 6 * dof;
      const f3 ab = ld3(cb), lb = ld3(cb + 3), ax = ld3(xaxis + 3 * j);
      jx = ab + cross(off, lb);
      js = cross(lb, ax);
      ja = mk3(0, 0, 0) - cross(lb, ax);
    }
    st3(JA + 3 * j, ja);
    st3(JX + 3 * j, jx);
    st3(JS + 3 * j, js);
    if (t == JNT_FREE || t == JNT_BALL) {
      BT[3 * b] += bt.x; BT[3 * b + 1] += bt.y; BT[3 * b + 2] += bt.z;
    }
  }
  __syncwarp();
}

// cinert bars -> body force / torque (xipos point, ximat columns) and SCB.  com_pos: cinert holds
// R diag(inertia) R' (R = ximat) plus the parallel-axis terms of dif = xipos - subtree_com[root].
__device__ void cinert_body_bars(const MjbModel& m, const MjbData& d, int w, int lane,
                                 const float* cinert_bar, float* BF, float* BT, float* SCB) {
  const int nb = m.nbody;
  const float* xipos = d.xipos + W(w, 3 * nb);
  const float* ximat = d.ximat + W(w, 9 * nb);
  const float* sc = d.subtree_com + W(w, 3 * nb);
  for (int b = lane; b < nb; b += 32) {
    if (b == 0) continue;
    const float* cb = cinert_bar + 10 * b;
    const m33 R = ld9(ximat + 9 * b);
    const f3 in = ld3(m.body_inertia + 3 * b);
    const float mass = m.body_mass[b];
    const float A[3][3] = {{cb[0], 0.5f * cb[3], 0.5f * cb[4]},
                           {0.5f * cb[3], cb[1], 0.5f * cb[5]},
                           {0.5f * cb[4], 0.5f * cb[5], cb[2]}};
    const float ink[3] = {in.x, in.y, in.z};
    f3 tq = mk3(0, 0, 0);
    for (int k = 0; k < 3; k++) {  // column k of Rbar = 2 A R diag(inertia)
      f3 rb;
      rb.x = 2.f * ink[k] * (A[0][0] * R.m[k] + A[0][1] * R.m[3 + k] + A[0][2] * R.m[6 + k]);
      rb.y = 2.f * ink[k] * (A[1][0] * R.m[k] + A[1][1] * R.m[3 + k] + A[1][2] * R.m[6 + k]);
      rb.z = 2.f * ink[k] * (A[2][0] * R.m[k] + A[2][1] * R.m[3 + k] + A[2][2] * R.m[6 + k]);
      tq = tq + cross(col(R, k), rb);
    }
    const f3 xi = ld3(xipos + 3 * b);
    const f3 df = xi - ld3(sc + 3 * m.body_rootid[b]);
    f3 dfb;
    dfb.x = mass * (2.f * df.x * (cb[1] + cb[2]) - cb[3] * df.y - cb[4] * df.z + cb[6]);
    dfb.y = mass * (2.f * df.y * (cb[0] + cb[2]) - cb[3] * df.x - cb[5] * df.z + cb[7]);
    dfb.z = mass * (2.f * df.z * (cb[0] + cb[1]) - cb[4] * df.x - cb[5] * df.y + cb[8]);
    tq = tq + cross(xi, dfb);
    BF[3 * b] += dfb.x; BF[3 * b + 1] += dfb.y; BF[3 * b + 2] += dfb.z;
    BT[3 * b] += tq.x; BT[3 * b + 1] += tq.y; BT[3 * b + 2] += tq.z;
    SCB[3 * b] -= dfb.x; SCB[3 * b + 1] -= dfb.y; SCB[3 * b + 2] -= dfb.z;
  }
  __syncwarp();
}

// subtree_com[r] = sum over r's subtree of mass_c xipos_c / subtree_mass_r: the bars collected
// for each root r (SCB of its bodies, JS of its joints) become xipos forces on its bodies.
// Scratch SR: 3 nbody floats.
__device__ void subtree_com_bars(const MjbModel& m, const MjbData& d, int w, int lane,
                                 const float* SCB, const float* JS, float* BF, float* BT, float* SR) {
  const int nb = m.nbody;
  const float* xipos = d.xipos + W(w, 3 * nb);
  for (int r = lane; r < nb; r += 32) {
    if (r == 0 || m.body_parentid[r] != 0) continue;
    const int end = m.body_subtreeend[r];
    f3 s = mk3(0, 0, 0);
    for (int b = r; b < end; b++) s = s + ld3(SCB + 3 * b);
    for (int j = 0; j < m.njnt; j++) {
      const int jb = m.jnt_bodyid[j];
      if (jb >= r && jb < end) s = s + ld3(JS + 3 * j);
    }
    st3(SR + 3 * r, s);
  }
  __syncwarp();
  for (int b = lane; b < nb; b += 32) {
    if (b == 0) continue;
    const int r = m.body_rootid[b];
    const f3 xb = ld3(SR + 3 * r) * (m.body_mass[b] / m.subtree_mass[r]);
    const f3 tq = cross(ld3(xipos + 3 * b), xb);
    BF[3 * b] += xb.x; BF[3 * b + 1] += xb.y; BF[3 * b + 2] += xb.z;
    BT[3 * b] += tq.x; BT[3 * b + 1] += tq.y; BT[3 * b + 2] += tq.z;
  }
  __syncwarp();
}

// Reverse walk of kinematics (smooth.py:46-109): a joint's motion moves everything downstream
// rigidly (the body's final frame and what hangs on it, later joints' anchors and axes on the same
// body, the descendant bodies), so with (F, T) summed over the downstream bars, a hinge gets
// axis . (T - anchor x F), a slide axis . F, a free joint F (translation) and x_k . (T - pos x F)
// (rotation about local axis k), a ball x_k . (T - anchor x F).  Adds to Q (per dof).
__device__ void kinematic_sweep(const MjbModel& m, const MjbData& d, int w, int lane,
                                const float* JA, const float* JX, float* BF, float* BT, float* Q) {
  const int nb = m.nbody;
  const float* xpos = d.xpos + W(w, 3 * nb);
  const float* xmat = d.xmat + W(w, 9 * nb);
  const float* xanchor = d.xanchor + W(w, 3 * m.njnt);
  const float* xaxis = d.xaxis + W(w, 3 * m.njnt);
  for (int lvl = m.nlevel - 1; lvl >= 1; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += 32) {
      const int b = m.body_tree[n];
      f3 F = ld3(BF + 3 * b), T = ld3(BT + 3 * b);
      const int ca = m.body_childadr[b], cn = m.body_childnum[b];
      for (int c = 0; c < cn; c++) {
        const int ch = m.body_child[ca + c];
        F = F + ld3(BF + 3 * ch);
        T = T + ld3(BT + 3 * ch);
      }
      const int j0 = m.body_jntadr[b];
      for (int j = j0 + m.body_jntnum[b] - 1; j >= j0; j--) {
        const int t = m.jnt_type[j], dof = m.jnt_dofadr[j];
        const f3 anchor = ld3(xanchor + 3 * j), ax = ld3(xaxis + 3 * j);
        const f3 ja = ld3(JA + 3 * j), jx = ld3(JX + 3 * j);
        if (t == JNT_FREE) {  // the anchor is the body position, which the joint itself sets
          F = F + ja;
          T = T + cross(anchor, ja);
          Q[dof] += F.x;
          Q[dof + 1] += F.y;
          Q[dof + 2] += F.z;
          const m33 R = ld9(xmat + 9 * b);
          const f3 tau = T - cross(ld3(xpos + 3 * b), F);
          for (int k = 0; k < 3; k++) Q[dof + 3 + k] += dot(col(R, k), tau);
          continue;
        }
        if (t == JNT_BALL) {
          const m33 R = ld9(xmat + 9 * b);
          const f3 tau = T - cross(anchor, F);
          for (int k = 0; k < 3; k++) Q[dof + k] += dot(col(R, k), tau);
        } else if (t == JNT_SLIDE) {
          Q[dof] += dot(ax, F);
        } else {
          Q[dof] += dot(ax, T - cross(anchor, F));
        }
        F = F + ja;
        T = T + cross(anchor, ja) + cross(ax, jx);
      }
      st3(BF + 3 * b, F);
      st3(BT + 3 * b, T);
    }
    __syncwarp();
  }
}

}  // namespace mjb
