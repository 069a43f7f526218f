// Finite-difference transition Jacobians of the batched step and their vector-Jacobian products.
//
// The reference has no derivative API; the scheme is MuJoCo's mjd_transitionFD, applied to a
// whole batch at once.  The state is x = (qpos in the tangent space (nv), qvel (nv), act (na)) and
// the input u = ctrl (nu); ncol = 2 nv + na + nu columns are differenced.  For each base world w
// the perturbed batch holds K = 1 + ncol (forward differences) or 1 + 2 ncol (centered) worlds:
// slot w K is an unperturbed copy and slot w K + 1 + c (forward), or w K + 1 + 2c and
// w K + 2 + 2c (centered, +eps and -eps), carries a perturbation of column c.  One step of the
// perturbed batch (any launch form) advances every slot; the differences of the slots' next
// states, divided by eps (2 eps), are the columns of A = dx'/dx (nx x nx, nx = 2 nv + na) and
// B = dx'/du (nx x nu), stored row-major per world.  Position perturbations and differences live
// in the tangent space: a free or ball joint's quaternion is rotated by quat_integrate about a
// local axis and differenced by quat_sub (the rotation vector in the first state's frame), as
// mj_integratePos / mj_differentiatePos do.  qacc_warmstart, qfrc_applied and xfrc_applied are
// copied unperturbed.
#pragma once

#include "mjb_adjoint.cuh"

namespace mjb {

// flags of the finite-difference entry points: bit 0 centered differences, bit 1 state columns
// only (the nu control columns are left out, e.g. when their derivative is taken analytically),
// bit 2 the nv qpos columns only (velocities and controls by step_vjp_world)
constexpr int kFdCentered = 1, kFdStateOnly = 2, kFdQposOnly = 4;
__host__ __device__ __forceinline__ int fd_ncol(const MjbModel& m, int flags = 0) {
  if (flags & kFdQposOnly) return m.nv;
  return 2 * m.nv + m.na + ((flags & kFdStateOnly) ? 0 : m.nu);
}
__host__ __device__ __forceinline__ int fd_slots(const MjbModel& m, int flags) {
  return 1 + fd_ncol(m, flags) * ((flags & kFdCentered) ? 2 : 1);
}

// Writes base world w's state into perturbed slot pw and perturbs column col by delta (col < 0:
// an unperturbed copy).
__device__ void fd_perturb_world(const MjbModel& m, const MjbData& b, const MjbData& p, int w,
                                 int pw, int col, float delta, int lane) {
  auto copy = [&](float* dst, const float* src, int n) {
    if (!dst || !src) return;
    for (int i = lane; i < n; i += 32) dst[W(pw, n) + i] = src[W(w, n) + i];
  };
  copy(p.qpos, b.qpos, m.nq);
  copy(p.qvel, b.qvel, m.nv);
  copy(p.act, b.act, m.na);
  copy(p.ctrl, b.ctrl, m.nu);
  copy(p.qacc_warmstart, b.qacc_warmstart, m.nv);
  copy(p.qfrc_applied, b.qfrc_applied, m.nv);
  copy(p.xfrc_applied, b.xfrc_applied, 6 * m.nbody);
  __syncwarp();
  if (lane != 0 || col < 0) return;
  const int nv = m.nv;
  if (col < nv) {  // mj_integratePos along tangent dof col
    float* qpos = p.qpos + W(pw, m.nq);
    const int j = m.dof_jntid[col], t = m.jnt_type[j], adr = m.jnt_qposadr[j];
    const int r = col - m.jnt_dofadr[j];
    if (t == JNT_FREE && r < 3) {
      qpos[adr + r] += delta;
    } else if (t == JNT_FREE || t == JNT_BALL) {
      const int qa = t == JNT_FREE ? adr + 3 : adr;
      const int k = t == JNT_FREE ? r - 3 : r;
      const f3 axis = f3{k == 0 ? 1.f : 0.f, k == 1 ? 1.f : 0.f, k == 2 ? 1.f : 0.f};
      st4(qpos + qa, quat_integrate(ld4(qpos + qa), axis, delta));
    } else {
      qpos[adr] += delta;
    }
  } else if (col < 2 * nv) {
    p.qvel[W(pw, nv) + col - nv] += delta;
  } else if (col < 2 * nv + m.na) {
    p.act[W(pw, m.na) + col - 2 * nv] += delta;
  } else {
    p.ctrl[W(pw, m.nu) + col - 2 * nv - m.na] += delta;
  }
}

// One column of A or B for base world w from the stepped perturbed batch.
__device__ void fd_column(const MjbModel& m, const MjbData& p, int w, int col, int flags,
                          float eps, float* A, float* B, int lane) {
  const int centered = flags & kFdCentered;
  const int nv = m.nv, na = m.na, nx = 2 * nv + na, K = fd_slots(m, flags);
  const int P = w * K + 1 + (centered ? 2 * col : col);
  const int R = centered ? P + 1 : w * K;
  const float scale = 1.f / (centered ? 2.f * eps : eps);
  float* out = col < nx ? A + W(w, nx * nx) + col : B + W(w, nx * m.nu) + (col - nx);
  const int ld = col < nx ? nx : m.nu;
  const float* qP = p.qpos + W(P, m.nq);
  const float* qR = p.qpos + W(R, m.nq);
  for (int j = lane; j < m.njnt; j += 32) {  // mj_differentiatePos
    const int t = m.jnt_type[j], adr = m.jnt_qposadr[j], dof = m.jnt_dofadr[j];
    if (t == JNT_FREE) {
      for (int k = 0; k < 3; k++) out[(dof + k) * ld] = (qP[adr + k] - qR[adr + k]) * scale;
      const f3 v = quat_sub(ld4(qP + adr + 3), ld4(qR + adr + 3));
      out[(dof + 3) * ld] = v.x * scale;
      out[(dof + 4) * ld] = v.y * scale;
      out[(dof + 5) * ld] = v.z * scale;
    } else if (t == JNT_BALL) {
      const f3 v = quat_sub(ld4(qP + adr), ld4(qR + adr));
      out[dof * ld] = v.x * scale;
      out[(dof + 1) * ld] = v.y * scale;
      out[(dof + 2) * ld] = v.z * scale;
    } else {
      out[dof * ld] = (qP[adr] - qR[adr]) * scale;
    }
  }
  for (int i = lane; i < nv; i += 32)
    out[(nv + i) * ld] = (p.qvel[W(P, nv) + i] - p.qvel[W(R, nv) + i]) * scale;
  for (int i = lane; i < na; i += 32)
    out[(2 * nv + i) * ld] = (p.act[W(P, na) + i] - p.act[W(R, na) + i]) * scale;
}

// lam_out = A^T lam and grad_ctrl = B^T lam for world w (row-major A: nx x nx, B: nx x nu).
__device__ void transition_vjp_world(const MjbModel& m, const float* A, const float* B,
                                     const float* lam, float* lam_out, float* grad_ctrl, int w,
                                     int lane) {
  const int nx = 2 * m.nv + m.na, nu = m.nu;
  const float* Aw = A + W(w, nx * nx);
  const float* l = lam + W(w, nx);
  for (int j = lane; j < nx; j += 32) {
    float s = 0.f;
    for (int i = 0; i < nx; i++) s += Aw[i * nx + j] * l[i];
    lam_out[W(w, nx) + j] = s;
  }
  if (B && grad_ctrl) {
    const float* Bw = B + W(w, nx * nu);
    for (int j = lane; j < nu; j += 32) {
      float s = 0.f;
      for (int i = 0; i < nx; i++) s += Bw[i * nu + j] * l[i];
      grad_ctrl[W(w, nu) + j] = s;
    }
  }
}

// Shared-memory floats per warp of step_vjp_world: the Hessian tile (nv <= 32) or the sparse-row
// assembly / blocked-Cholesky scratch (nv > 32), eight vectors of 32 ceil(nv / 32) floats and,
// for the velocity or position adjoint, four spatial vectors per body; for the position adjoint
// also the cdof bars (6 per dof), body force / torque / cinert / subtree_com bars (19 per body)
// and the joints' anchor / axis / subtree_com bars (9 per joint).
__host__ __device__ __forceinline__ int step_vjp_vec(int nv) { return 32 * ((nv + 31) / 32); }
__host__ __device__ __forceinline__ int step_vjp_floats(const MjbModel& m, bool vel, bool pos) {
  int n = (m.nv <= 32 ? tile_floats(m.nv) : generic_nz_floats(m.nv)) + 8 * step_vjp_vec(m.nv);
  if (vel || pos) n += 24 * m.nbody;
  if (pos) n += 6 * m.nv + 19 * m.nbody + 9 * m.njnt;
  return n;
}

// Reverse sweep of the bias forces' velocity dependence (smooth.py:539-606 com_vel and
// smooth.py:398-466 rne run backwards): rq_i = d (s . qfrc_bias) / d qvel_i, for s (nv, shared).
// With u_b = sum of s_i cdof_i over the dofs from the root to body b, s . qfrc_bias =
// sum_b u_b . cfrc_b, cfrc_b = I_b cacc_b + cvel_b x* (I_b cvel_b).  The adjoint of cacc_b is
// G_b = sum over b's subtree of I_c u_c; cvel_b gets I_b (u_b x cvel_b) - u_b x* (I_b cvel_b)
// directly, and the adjoint of the velocity entering each dof's cdof_dot = v x cdof gets
// qvel_i cdof_i x* G_b.  Walking every body's joints backwards (the order com_vel adds them in),
// rq_i = G_b . cdof_dot_i + cdof_i . (adjoint of the body velocity after dof i's joint).
__device__ void rne_vel_vjp(const MjbModel& m, const MjbData& d, int w, int lane, const float* s,
                            const float* qvel, float* rq, float* U, float* G, float* R) {
  const int nb = m.nbody, nv = m.nv;
  const float* cdof = d.cdof + W(w, 6 * nv);
  const float* cdd = d.cdof_dot + W(w, 6 * nv);
  const float* cvel = d.cvel + W(w, 6 * nb);
  const float* cinert = d.cinert + W(w, 10 * nb);
  if (lane < 6) U[lane] = G[lane] = R[lane] = 0.f;
  __syncwarp();
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += 32) {
      const int b = m.body_tree[n];
      s6 u = ld6(U + 6 * m.body_parentid[b]);
      const int da = m.body_dofadr[b];
      for (int i = 0; i < m.body_dofnum[b]; i++) {
        const s6 c = ld6(cdof + 6 * (da + i));
        for (int k = 0; k < 6; k++) u.v[k] += c.v[k] * s[da + i];
      }
      st6(U + 6 * b, u);
      const s6 v = ld6(cvel + 6 * b);
      st6(G + 6 * b, inert_vec(cinert + 10 * b, u));
      const s6 a = inert_vec(cinert + 10 * b, motion_cross(u, v));
      const s6 c = motion_cross_force(u, inert_vec(cinert + 10 * b, v));
      s6 r;
      for (int k = 0; k < 6; k++) r.v[k] = a.v[k] - c.v[k];
      st6(R + 6 * b, r);
    }
    __syncwarp();
  }
  for (int lvl = m.nlevel - 1; lvl >= 1; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += 32) {
      const int b = m.body_tree[n];
      s6 g = ld6(G + 6 * b), r = ld6(R + 6 * b);
      const int ca = m.body_childadr[b], cn = m.body_childnum[b];
      for (int c = 0; c < cn; c++) {
        const int ch = m.body_child[ca + c];
        const s6 x = ld6(G + 6 * ch), y = ld6(R + 6 * ch);
        for (int k = 0; k < 6; k++) {
          g.v[k] += x.v[k];
          r.v[k] += y.v[k];
        }
      }
      st6(G + 6 * b, g);
      // joints of b in reverse; r is the adjoint of the body velocity after the joint
      const int j0 = m.body_jntadr[b];
      int dof_end = m.body_dofadr[b] + m.body_dofnum[b];
      for (int j = j0 + m.body_jntnum[b] - 1; j >= j0; j--) {
        const int t = m.jnt_type[j];
        const int nd = t == JNT_FREE ? 6 : (t == JNT_BALL ? 3 : 1);
        const int dof = dof_end - nd;
        const int rot = t == JNT_FREE ? 3 : 0;  // a free joint's cdof_dot uses v after its translation
        s6 acc{{0, 0, 0, 0, 0, 0}};
        for (int i = dof + rot; i < dof_end; i++) {
          const s6 c = ld6(cdof + 6 * i);
          rq[i] = dot6(g, ld6(cdd + 6 * i)) + dot6(c, r);
          const s6 x = motion_cross_force(c, g);
          for (int k = 0; k < 6; k++) acc.v[k] += qvel[i] * x.v[k];
        }
        for (int k = 0; k < 6; k++) r.v[k] += acc.v[k];
        for (int i = dof; i < dof + rot; i++) rq[i] = dot6(g, ld6(cdd + 6 * i)) + dot6(ld6(cdof + 6 * i), r);
        dof_end = dof;
      }
      st6(R + 6 * b, r);  // now the adjoint of the parent's velocity, summed by the parent
    }
    __syncwarp();
  }
}

// VJP of one step by implicit differentiation at the solver's final active set A (no counterpart
// in the reference).  With qacc = H^-1 (qfrc_smooth + J_A' D_A aref_A) at the Newton solution
// (H = M + J_A' D_A J_A), qfrc_constraint = -J_A' D_A (J_A qacc - aref_A), and the integrator's
// qacc_int = Mt^-1 (qfrc_smooth + qfrc_constraint) (Mt = M - dt qDeriv, qLD_integration its
// factor; Euler without eulerdamp advances with qacc itself), v' = v + dt qacc_int and
// q' = q (+) dt v', whose tangent responds to dv' by dt J_r(dt v') on a quaternion's three dofs
// (J_r the right Jacobian of the rotation exponential) and by dt elsewhere.  With
//   y = lam_v + dt J_r' lam_q,   z = Mt^-1 y,   s = H^-1 M z   (z = 0, s = H^-1 y without Mt):
// controls enter qfrc_smooth through moment' (gain * [ctrl inside its range]), masked (mask) where
// the joint's actuator force is clamped:  d loss / d ctrl = dt G' moment mask s;
// velocities enter through the identity in v', the damper -damping v, the bias forces (rne), the
// actuator velocity terms (force += (gainprm[2] ctrl + biasprm[2]) moment v) and
// aref = -k imp pos - b J v:
//   d loss / d qvel = y + dt (-damping s - d(s . qfrc_bias)/dv + moment' K moment mask s
//                             - J_A' D_A b_A J_A s);
// positions enter through q' directly (a quaternion's tangent is carried by R(dt v'), the rotation
// of the step) and through every position-dependent quantity of the step:
//   d loss / d qpos = R' lam_q + dt d/dq [z' M (qacc - qacc_int) - s' M qacc + s' qfrc_smooth
//                                         + sum_A (D t e + D t aref)]
// with the row terms of row_q_bars (t = J s, e = aref - J qacc, every factor but the
// differentiated one held fixed).  d holds the step's intermediates (qM, the final efc rows and
// active flags, contacts, qLD_integration, qacc_integration, kinematics, com / rne arrays,
// actuator arrays) and the post-step qvel; qvel_prev is the pre-step qvel; lam = (lam_q (nv),
// lam_v (nv)) of the next state.  Any of grad_qpos / grad_qvel / grad_ctrl may be null.  One warp
// per world (scratch: step_vjp_floats; for nv > 32 the Newton solver's factor of H in efc_h is
// reused, and with CG H and its factor are written there), dense qM, na = 0.
__device__ void step_vjp_world(const MjbModel& m, const MjbData& d, int w, int lane,
                               const float* lam, const float* qvel_prev, float* grad_ctrl,
                               float* grad_qvel, float* grad_qpos, float* tile) {
  const int nv = m.nv, nu = m.nu, nb = m.nbody, VL = step_vjp_vec(nv);
  const float dt = m.timestep;
  const bool velg = grad_qvel != nullptr, posg = grad_qpos != nullptr;
  const float* lq = lam + W(w, 2 * nv + m.na);
  const float* lv = lq + nv;
  const float* qvel = d.qvel + W(w, nv);
  const float* qv = qvel_prev ? qvel_prev + W(w, nv) : nullptr;
  float* Y = tile + (nv <= 32 ? tile_floats(nv) : generic_nz_floats(nv));
  float* Z = Y + VL;
  float* S = Z + VL;
  float* St = S + VL;
  float* WV = St + VL;
  float* Q = WV + VL;
  float* GV = Q + VL;
  float* DIR = GV + VL;
  float* SA = DIR + VL;
  float* SB = SA + 6 * nb;
  float* SC = SB + 6 * nb;
  float* SD = SC + 6 * nb;
  float* CB = SD + 6 * nb;
  float* BF = CB + 6 * nv;
  float* BT = BF + 3 * nb;
  float* CIB = BT + 3 * nb;
  float* SCB = CIB + 10 * nb;
  float* JA = SCB + 3 * nb;
  float* JX = JA + 3 * m.njnt;
  float* JS = JX + 3 * m.njnt;
  // y = lam_v + dt J_r' lam_q, and for the position part R(dt v') lam_q
  for (int i = lane; i < VL; i += 32) {
    float y = 0.f, direct = 0.f;
    if (i < nv) {
      float rl = lq[i];
      direct = lq[i];
      const int j = m.dof_jntid[i], t = m.jnt_type[j], r = i - m.jnt_dofadr[j];
      if ((t == JNT_FREE && r >= 3) || t == JNT_BALL) {
        const int b = i - (t == JNT_FREE ? r - 3 : r);  // first rotational dof of the joint
        const int k = i - b;
        const f3 phi = ld3(qvel + b) * dt;
        const float th2 = dot(phi, phi), th = sqrtf(th2);
        float c1, c2, sa;  // (1 - cos th) / th^2, (th - sin th) / th^3, sin th / th
        if (th < 1e-3f) {
          c1 = 0.5f - th2 / 24.f;
          c2 = 1.f / 6.f - th2 / 120.f;
          sa = 1.f - th2 / 6.f;
        } else {
          c1 = (1.f - cosf(th)) / th2;
          c2 = (th - sinf(th)) / (th2 * th);
          sa = sinf(th) / th;
        }
        // J_r = I - c1 [phi]x + c2 [phi]x^2; row k of J_r^T = column k of J_r
        const float p[3] = {phi.x, phi.y, phi.z};
        float colk[3];
        for (int e = 0; e < 3; e++) {
          // [phi]x (e, k) = -eps_ekl phi_l ; [phi]x^2 = phi phi^T - |phi|^2 I
          const float cx = (e == k) ? 0.f : ((e + 1) % 3 == k ? -p[(k + 1) % 3] : p[(e + 1) % 3]);
          const float cx2 = p[e] * p[k] - (e == k ? th2 : 0.f);
          colk[e] = (e == k ? 1.f : 0.f) - c1 * cx + c2 * cx2;
        }
        rl = colk[0] * lq[b] + colk[1] * lq[b + 1] + colk[2] * lq[b + 2];
        // R(phi) lam = lam + sa phi x lam + c1 phi x (phi x lam), component k
        const f3 l3 = ld3(lq + b);
        const f3 a = cross(phi, l3), a2 = cross(phi, a);
        const f3 rv = l3 + a * sa + a2 * c1;
        direct = k == 0 ? rv.x : (k == 1 ? rv.y : rv.z);
      }
      y = lv[i] + dt * rl;
    }
    Y[i] = y;
    Z[i] = y;
    DIR[i] = direct;
    Q[i] = 0.f;
    GV[i] = 0.f;
  }
  __syncwarp();
  // z = Mt^-1 y and w = M z (implicitfast, eulerdamp), else w = y
  const bool passive_on = !(m.disableflags & DSBL_PASSIVE);
  const bool mt = m.integrator == 0 ? !(m.disableflags & DSBL_EULERDAMP) : passive_on;
  if (mt) {
    solve_blocks(m, d.qLD_integration + W(w, nv * nv), Z, Z, lane, tile, false);
    mul_m_world(d.qM + W(w, nv * nv), nv, WV, Z, lane);
  } else {
    for (int i = lane; i < VL; i += 32) {
      WV[i] = Y[i];
      Z[i] = 0.f;
    }
  }
  __syncwarp();
  // s = H^-1 w with H assembled at the final active set: in the tile (nv <= 32) or in efc_h
  const float* qM = d.qM + W(w, nv * nv);
  const int adr = d.world_efcadr[w], n = d.world_nefc[w];
  if (nv <= 32) {
    const int ld = tile_ld(nv);
    const bool own = lane < nv;
    copy_rows(qM, nv, tile, ld, nv, nv, 4 * ((nv + 3) >> 2), lane);
    __syncwarp();
    if (own) {
      float h[32];
      for (int c = 0; c < nv; c++) h[c] = tile[lane * ld + c];
      for (int k = 0; k < n; k++) {
        const int r = adr + k;
        if (!d.efc_active[r]) continue;
        const float D = d.efc_D[r];
        if (D == 0.f) continue;
        const float* J = d.efc_J + size_t(r) * nv;
        const float a = D * J[lane];
        for (int c = 0; c < nv; c++) h[c] += a * J[c];
      }
      for (int c = 0; c < nv; c++) tile[lane * ld + c] = h[c];
    }
    __syncwarp();
    chol_tile(tile, ld, nv, lane);
    const float sv = cho_solve_tile(tile, ld, nv, own ? WV[lane] : 0.f, lane);
    __syncwarp();
    S[lane] = own ? sv : 0.f;
  } else {
    // the Newton solver (generic path) leaves the factor of H at the final active set in efc_h:
    // its iterations end with update_gradient, which factors H in place (or keeps the factor
    // while the active set is unchanged); CG has no H, and without constraint capacity
    // (njmax = 0) the solver does not run, so there H is assembled and factored here
    float* H = d.efc_h + W(w, nv * nv);
    if (m.solver != 2 || d.njmax == 0) {
      assemble_hessian(m, d, qM, H, adr, n, tile, lane);
      chol_any(H, nv, nv, lane, tile);
    }
    warp_cho_solve(H, nv, nv, S, WV, lane);
    for (int i = nv + lane; i < VL; i += 32) S[i] = 0.f;
  }
  __syncwarp();
  for (int i = lane; i < VL; i += 32) St[i] = S[i];
  __syncwarp();
  // velocity: bias forces, damper, rows
  if (velg) {
    rne_vel_vjp(m, d, w, lane, S, qv, WV, SA, SB, SC);
    for (int i = lane; i < nv; i += 32)
      GV[i] = -WV[i] - (passive_on ? m.dof_damping[i] * S[i] : 0.f);
    __syncwarp();
    row_q_bars(m, d, w, lane, S, qv, Q, nullptr, nullptr, nullptr, nullptr, GV);
  }
  // mask of the dofs whose actuator force is not clamped
  const bool act = nu > 0 && !(m.disableflags & DSBL_ACTUATION);
  const float* moment = d.actuator_moment + W(w, nu * nv);
  const float* force = d.actuator_force + W(w, nu);
  if (act) {
    for (int i = lane; i < nv; i += 32) {
      float f = 0.f;
      for (int a = 0; a < nu; a++) f += moment[a * nv + i] * force[a];
      const int j = m.dof_jntid[i];
      const bool clamped = m.jnt_actfrclimited[j] &&
                           !(f > m.jnt_actfrcrange[2 * j] && f < m.jnt_actfrcrange[2 * j + 1]);
      if (clamped) St[i] = 0.f;
    }
  }
  __syncwarp();
  // controls, and the actuators' velocity (GV) and length (Q) terms
  const float* len = d.actuator_length + W(w, nu);
  const float* vel = d.actuator_velocity + W(w, nu);
  const float* ctrl = d.ctrl + W(w, nu);
  for (int a0 = 0; a0 < nu; a0 += 32) {
    const int a = a0 + lane;
    float kv = 0.f, kq = 0.f;  // (gainprm[2] ctrl + biasprm[2]), (gainprm[1] ctrl + biasprm[1]) x moment_a . St
    if (a < nu) {
      float g = 0.f;
      if (act) {
        const float* gp = m.actuator_gainprm + 10 * a;
        const float* bp = m.actuator_biasprm + 10 * a;
        const float gain = gp[0] + gp[1] * len[a] + gp[2] * vel[a];
        float c = ctrl[a];
        const bool limited = m.actuator_ctrllimited[a] && !(m.disableflags & DSBL_CLAMPCTRL);
        const bool clamp = limited && !(c > m.actuator_ctrlrange[2 * a] &&
                                        c < m.actuator_ctrlrange[2 * a + 1]);
        if (limited) c = fminf(fmaxf(c, m.actuator_ctrlrange[2 * a]), m.actuator_ctrlrange[2 * a + 1]);
        float ms = 0.f;
        for (int i = 0; i < nv; i++) ms += moment[a * nv + i] * St[i];
        if (!clamp) g = dt * gain * ms;
        kv = (gp[2] * c + bp[2]) * ms;
        kq = (gp[1] * c + bp[1]) * ms;
      }
      if (grad_ctrl) grad_ctrl[W(w, nu) + a] = g;
    }
    const int cnt = min(32, nu - a0);
    for (int k = 0; k < cnt; k++) {
      const float cv = __shfl_sync(0xffffffffu, kv, k), cq = __shfl_sync(0xffffffffu, kq, k);
      if (cv == 0.f && cq == 0.f) continue;
      const float* mo = moment + (a0 + k) * nv;
      for (int i = lane; i < nv; i += 32) {
        GV[i] += cv * mo[i];
        Q[i] += cq * mo[i];
      }
    }
  }
  __syncwarp();
  if (velg)
    for (int i = lane; i < nv; i += 32) grad_qvel[W(w, nv) + i] = Y[i] + dt * GV[i];
  if (!posg) {
    __syncwarp();
    return;
  }
  // position: bars on cdof / cinert / subtree_com / contacts, then the joints
  for (int e = lane; e < 6 * nv; e += 32) CB[e] = 0.f;
  for (int e = lane; e < 19 * nb; e += 32) BF[e] = 0.f;  // BF, BT, CIB, SCB are contiguous
  for (int e = lane; e < 9 * m.njnt; e += 32) JA[e] = 0.f;  // JA, JX, JS
  __syncwarp();
  const float* qacc = d.qacc + W(w, nv);
  if (mt) {
    const float* aint = d.qacc_integration + W(w, nv);
    for (int i = lane; i < VL; i += 32) WV[i] = i < nv ? qacc[i] - aint[i] : 0.f;
    __syncwarp();
    mass_product_bars(m, d, w, lane, Z, WV, CB, CIB, SA, SB, SC, SD);
  }
  for (int i = lane; i < VL; i += 32) WV[i] = -S[i];
  __syncwarp();
  mass_product_bars(m, d, w, lane, WV, qacc, CB, CIB, SA, SB, SC, SD);
  bias_q_bars(m, d, w, lane, WV, qv, CB, CIB, SA, SB, SC);
  if (passive_on) {  // hinge / slide springs -k (q - q_spring)
    for (int j = lane; j < m.njnt; j += 32) {
      const int t = m.jnt_type[j];
      if ((t == JNT_HINGE || t == JNT_SLIDE) && m.jnt_stiffness[j] != 0.f) {
        const int dof = m.jnt_dofadr[j];
        Q[dof] -= m.jnt_stiffness[j] * S[dof];
      }
    }
    __syncwarp();
  }
  row_q_bars(m, d, w, lane, S, qv, Q, CB, BF, BT, SCB, nullptr);
  cdof_joint_bars(m, d, w, lane, CB, JA, JX, JS, BT);
  cinert_body_bars(m, d, w, lane, CIB, BF, BT, SCB);
  subtree_com_bars(m, d, w, lane, SCB, JS, BF, BT, SA);
  kinematic_sweep(m, d, w, lane, JA, JX, BF, BT, Q);
  for (int i = lane; i < nv; i += 32) grad_qpos[W(w, nv) + i] = DIR[i] + dt * Q[i];
  __syncwarp();
}

}  // namespace mjb
