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

#include "mjb_solver.cuh"

namespace mjb {

// flags of the finite-difference entry points: bit 0 centered differences, bit 1 state columns
// only (the nu control columns are left out, e.g. when their derivative is taken analytically)
constexpr int kFdCentered = 1, kFdStateOnly = 2;
__host__ __device__ __forceinline__ int fd_ncol(const MjbModel& m, int flags = 0) {
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

// d loss / d ctrl of one step by implicit differentiation at the solver's final active set A
// (no counterpart in the reference).  With qacc = H^-1 (qfrc_smooth + J_A' D_A aref_A) at the
// Newton solution (H = M + J_A' D_A J_A), qfrc_constraint = -J_A' D_A (J_A qacc - aref_A), and the
// integrator's qacc_int = Mt^-1 (qfrc_smooth + qfrc_constraint) (Mt = M - dt qDeriv, qLD_integration
// its factor; Euler without eulerdamp advances with qacc itself), d qacc_int / d qfrc_smooth is
// Mt^-1 M H^-1.  Then v' = v + dt qacc_int and q' = q (+) dt v', whose tangent responds to dv' by
// dt J_r(dt v') on a quaternion's three dofs (J_r the right Jacobian of the rotation exponential)
// and by dt elsewhere; qfrc_smooth depends on ctrl through moment' (gain * [ctrl inside its range])
// masked where the joint's actuator force is clamped.  Hence
//   d loss / d ctrl = dt G' moment mask H^-1 M Mt^-1 (lam_v + dt R' lam_q).
// d holds the step's intermediates (qM, the final efc rows and active flags, qLD_integration,
// actuator arrays) and the post-step qvel; lam = (lam_q (nv), lam_v (nv)) of the next state.
// One warp per world, nv <= 32 (tile: tile_floats(nv) + 64 floats of warp scratch), dense qM,
// na = 0.
__device__ void ctrl_vjp_world(const MjbModel& m, const MjbData& d, int w, int lane,
                               const float* lam, float* grad_ctrl, float* tile) {
  const int nv = m.nv, nu = m.nu;
  const float dt = m.timestep;
  const bool own = lane < nv;
  const float* lq = lam + W(w, 2 * nv + m.na);
  const float* lv = lq + nv;
  const float* qvel = d.qvel + W(w, nv);
  // y = lam_v + dt R' lam_q
  float y = 0.f;
  if (own) {
    float rl = lq[lane];
    const int j = m.dof_jntid[lane], t = m.jnt_type[j], r = lane - m.jnt_dofadr[j];
    if ((t == JNT_FREE && r >= 3) || t == JNT_BALL) {
      const int b = lane - (t == JNT_FREE ? r - 3 : r);  // first rotational dof of the joint
      const int k = lane - b;
      const f3 phi = ld3(qvel + b) * dt;
      const float th2 = dot(phi, phi), th = sqrtf(th2);
      float c1, c2;  // (1 - cos th) / th^2, (th - sin th) / th^3
      if (th < 1e-3f) {
        c1 = 0.5f - th2 / 24.f;
        c2 = 1.f / 6.f - th2 / 120.f;
      } else {
        c1 = (1.f - cosf(th)) / th2;
        c2 = (th - sinf(th)) / (th2 * th);
      }
      // J_r = I - c1 [phi]x + c2 [phi]x^2; row k of J_r^T = column k of J_r
      const float p[3] = {phi.x, phi.y, phi.z};
      float col[3];
      for (int i = 0; i < 3; i++) {
        // [phi]x (i, k) = -eps_ikl phi_l ; [phi]x^2 = phi phi^T - |phi|^2 I
        const float cx = (i == k) ? 0.f : ((i + 1) % 3 == k ? -p[(k + 1) % 3] : p[(i + 1) % 3]);
        const float cx2 = p[i] * p[k] - (i == k ? th2 : 0.f);
        col[i] = (i == k ? 1.f : 0.f) - c1 * cx + c2 * cx2;
      }
      rl = col[0] * lq[b] + col[1] * lq[b + 1] + col[2] * lq[b + 2];
    }
    y = lv[lane] + dt * rl;
  }
  // w = M Mt^-1 y (implicitfast, eulerdamp), else y
  const bool passive_on = !(m.disableflags & DSBL_PASSIVE);
  const bool mt = m.integrator == 0 ? !(m.disableflags & DSBL_EULERDAMP) : passive_on;
  float* zv = tile + tile_floats(nv);  // two 32-float vectors after the tile
  float* wv = zv + 32;
  if (own) zv[lane] = y;
  __syncwarp();
  if (mt) {
    solve_blocks(m, d.qLD_integration + W(w, nv * nv), zv, zv, lane, tile, false);
    mul_m_world(d.qM + W(w, nv * nv), nv, wv, zv, lane);
  } else if (own) {
    wv[lane] = zv[lane];
  }
  __syncwarp();
  // s = H^-1 w, H assembled at the final active set in the tile
  const int ld = tile_ld(nv);
  const float* qM = d.qM + W(w, nv * nv);
  const int adr = d.world_efcadr[w], n = d.world_nefc[w];
  for (int r = 0; r < nv; r++)
    if (lane < 4 * ((nv + 3) >> 2)) tile[r * ld + lane] = lane < nv ? qM[r * nv + lane] : 0.f;
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
  const float sv = cho_solve_tile(tile, ld, nv, own ? wv[lane] : 0.f, lane);
  __syncwarp();
  if (own) zv[lane] = sv;
  // mask of the dofs whose actuator force is not clamped
  const float* moment = d.actuator_moment + W(w, nu * nv);
  const float* force = d.actuator_force + W(w, nu);
  if (own) {
    float f = 0.f;
    for (int a = 0; a < nu; a++) f += moment[a * nv + lane] * force[a];
    const int j = m.dof_jntid[lane];
    const bool clamped = m.jnt_actfrclimited[j] &&
                         !(f > m.jnt_actfrcrange[2 * j] && f < m.jnt_actfrcrange[2 * j + 1]);
    if (clamped) zv[lane] = 0.f;
  }
  __syncwarp();
  const float* len = d.actuator_length + W(w, nu);
  const float* vel = d.actuator_velocity + W(w, nu);
  const float* ctrl = d.ctrl + W(w, nu);
  for (int a = lane; a < nu; a += 32) {
    const float* gp = m.actuator_gainprm + 10 * a;
    const float gain = gp[0] + gp[1] * len[a] + gp[2] * vel[a];
    const float c = ctrl[a];
    const bool clamp = m.actuator_ctrllimited[a] && !(m.disableflags & DSBL_CLAMPCTRL) &&
                       !(c > m.actuator_ctrlrange[2 * a] && c < m.actuator_ctrlrange[2 * a + 1]);
    float g = 0.f;
    if (!clamp) {
      for (int i = 0; i < nv; i++) g += moment[a * nv + i] * zv[i];
      g *= dt * gain;
    }
    grad_ctrl[W(w, nu) + a] = g;
  }
  __syncwarp();
}

}  // namespace mjb
