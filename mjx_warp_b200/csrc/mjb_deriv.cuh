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

#include "mjb_collide.cuh"

namespace mjb {

__host__ __device__ __forceinline__ int fd_ncol(const MjbModel& m) { return 2 * m.nv + m.na + m.nu; }
__host__ __device__ __forceinline__ int fd_slots(const MjbModel& m, int centered) {
  return 1 + fd_ncol(m) * (centered ? 2 : 1);
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
__device__ void fd_column(const MjbModel& m, const MjbData& p, int w, int col, int centered,
                          float eps, float* A, float* B, int lane) {
  const int nv = m.nv, na = m.na, nx = 2 * nv + na, K = fd_slots(m, centered);
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

}  // namespace mjb
