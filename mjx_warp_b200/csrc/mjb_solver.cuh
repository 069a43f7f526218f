// Primal Newton / CG constraint solver (mujoco_warp/_src/solver.py:26-1000), one warp per world.
//
// The reference runs each solver phase as a kernel over all njmax rows or nworld*nv dofs with
// float atomics into per-world accumulators; here one warp owns a world for the whole solve:
// lanes stride over the world's constraint rows (contiguous in the flat efc arrays) or over its
// dofs, per-world sums are warp reductions (identical in every lane, so control flow stays
// uniform), and a world that is done simply leaves the iteration loop, which is what the
// reference's per-kernel `done` early exits amount to.  The Newton Hessian
// H = tril(qM) + sum_active D J^T J and its Cholesky factor live in the per-warp scratch `hs`
// (nv x nv floats).
#pragma once

#include "mjb_collide.cuh"
#include "mjb_tc.cuh"

namespace mjb {

struct SolverCtx {
  const MjbModel& m;
  const MjbData& d;
  int w, lane, nv, adr, n;
  float *qacc, *Ma, *grad, *Mgrad, *search, *mv, *qfrc_constraint;
  const float *qM, *qLD, *qfrc_smooth, *qacc_smooth;
  float* hs;
  float* nz;                 // warp scratch of generic_nz_floats(nv) floats, or null
  bool reuse = false;        // keep the Hessian factor while the active set is unchanged
  bool factored = false;     // hs holds the factor of the current active set's Hessian
  bool changed = true;       // the last update_constraint changed an active flag
  float cost, prev_cost, gauss, grad_dot, search_dot, gtol, alpha;
  float qg[3];
};

__host__ __device__ __forceinline__ int round4i(int x) { return (x + 3) & ~3; }
// warp scratch of the generic (nv > 32) solver: a constraint row's nonzero columns and values
// during the Hessian assembly, then the blocked Cholesky's 32 x 36 tile
__host__ __device__ __forceinline__ int generic_nz_floats(int nv) {
  return 2 * round4i(nv) > 32 * 36 ? 2 * round4i(nv) : 32 * 36;
}

__device__ __forceinline__ float safe_div(float x, float y) { return x / (y != 0.f ? y : kMinVal); }

// M vec for one world (support.py:45-92; dense qM is symmetric, so rows = columns)
__device__ __forceinline__ void mul_m_world(const float* qM, int nv, float* res, const float* vec, int lane) {
  for (int i = lane; i < nv; i += 32) {
    float s = 0.f;
    for (int j = 0; j < nv; j++) s += qM[i * nv + j] * vec[j];
    res[i] = s;
  }
  __syncwarp();
}

// res = M vec for the world's mass matrix, dense or sparse (res must not alias vec)
__device__ __forceinline__ void mul_m_ctx(SolverCtx& s, float* res, const float* vec) {
  if (s.m.is_sparse) mul_m_sparse(s.m, s.qM, res, vec, s.lane);
  else mul_m_world(s.qM, s.nv, res, vec, s.lane);
}

// solver.py:75-173
__device__ void update_constraint(SolverCtx& s) {
  const MjbData& d = s.d;
  const int nv = s.nv;
  s.prev_cost = s.cost;
  float c = 0.f;
  bool changed = false;
  for (int k = s.lane; k < s.n; k += 32) {
    const int r = s.adr + k;
    const float Jaref = d.efc_Jaref[r], D = d.efc_D[r];
    const int active = Jaref < 0.f;
    changed |= d.efc_active[r] != active;
    d.efc_active[r] = active;
    if (active) {
      d.efc_force[r] = -1.f * D * Jaref;
      c += 0.5f * D * Jaref * Jaref;
    } else {
      d.efc_force[r] = 0.f;
    }
  }
  s.changed = __any_sync(WARP_FULL, changed);
  c = warp_sum(c);
  __syncwarp();
  for (int i = s.lane; i < nv; i += 32) {
    float f = 0.f;
    for (int k = 0; k < s.n; k++) f += d.efc_J[size_t(s.adr + k) * nv + i] * d.efc_force[s.adr + k];
    s.qfrc_constraint[i] = f;
  }
  float g = 0.f;
  for (int i = s.lane; i < nv; i += 32)
    g += 0.5f * (s.Ma[i] - s.qfrc_smooth[i]) * (s.qacc[i] - s.qacc_smooth[i]);
  g = warp_sum(g);
  s.gauss = g;
  s.cost = c + g;
  __syncwarp();
}

// solver.py:176-312
// H = tril(qM) + sum over the world's active rows of D J'J: the lower triangle of the dense
// nv x nv matrix at H (update_gradient's Newton Hessian, solver.py:249-276).  nz: null or
// generic_nz_floats(nv) floats of warp scratch for the sparse-row assembly.
__device__ void assemble_hessian(const MjbModel& m, const MjbData& d, const float* qM, float* H,
                                 int adr, int n, float* nz, int lane) {
  const int nv = m.nv;
  if (nz) {
    // Each row's outer product touches only the row's nonzero columns (a contact row has the
    // dofs of two kinematic chains): the columns are compacted in order into the warp's
    // scratch and the lower-triangle pairs updated, row by row, with the per-entry arithmetic
    // of the dense form (h += J_i * J_j * D in row order; zero terms are skipped).
    if (m.is_sparse) {
      sparse_to_lower(m, qM, H, lane);
    } else {
      for (int e = lane; e < nv * nv; e += 32) {
        const int i = e / nv, j = e - i * nv;
        if (j <= i) H[e] = qM[e];
      }
      __syncwarp();
    }
    int* nzi = reinterpret_cast<int*>(nz);
    float* nzv = nz + round4i(nv);
    for (int k = 0; k < n; k++) {
      const int r = adr + k;
      if (!d.efc_active[r]) continue;
      const float D = d.efc_D[r];
      if (D == 0.f) continue;
      const float* J = d.efc_J + size_t(r) * nv;
      int cnt = 0;
      for (int base = 0; base < nv; base += 32) {
        const int c = base + lane;
        const float v = c < nv ? J[c] : 0.f;
        const unsigned mk = __ballot_sync(WARP_FULL, v != 0.f);
        if (v != 0.f) {
          const int p = cnt + __popc(mk & ((1u << lane) - 1u));
          nzi[p] = c;
          nzv[p] = v;
        }
        cnt += __popc(mk);
      }
      __syncwarp();
      const int npair = cnt * (cnt + 1) / 2;
      for (int t = lane; t < npair; t += 32) {  // pair t = (a, b), b <= a, in triangle order
        int a = int((sqrtf(8.f * float(t) + 1.f) - 1.f) * 0.5f);
        while (a * (a + 1) / 2 > t) a--;
        while ((a + 1) * (a + 2) / 2 <= t) a++;
        const int b = t - a * (a + 1) / 2;
        H[nzi[a] * nv + nzi[b]] += nzv[a] * nzv[b] * D;
      }
      __syncwarp();
    }
  } else {
    if (m.is_sparse) sparse_to_lower(m, qM, H, lane);
    for (int e = lane; e < nv * nv; e += 32) {
      const int i = e / nv, j = e - i * nv;
      if (j > i) continue;
      float h = m.is_sparse ? H[e] : qM[e];
      for (int k = 0; k < n; k++) {
        const int r = adr + k;
        if (!d.efc_active[r]) continue;
        const float D = d.efc_D[r];
        if (D == 0.f) continue;
        const float* J = d.efc_J + size_t(r) * nv;
        h += J[i] * J[j] * D;
      }
      H[e] = h;
    }
    __syncwarp();
  }
}

__device__ void update_gradient(SolverCtx& s) {
  const MjbModel& m = s.m;
  const MjbData& d = s.d;
  const int nv = s.nv, lane = s.lane;
  float gd = 0.f;
  for (int i = lane; i < nv; i += 32) {
    const float g = s.Ma[i] - s.qfrc_smooth[i] - s.qfrc_constraint[i];
    s.grad[i] = g;
    gd += g * g;
  }
  s.grad_dot = warp_sum(gd);
  __syncwarp();
  if (m.solver == 1) {  // CG: Mgrad = M^-1 grad
    solve_m_world(m, d, s.w, s.Mgrad, s.grad, lane);
    return;
  }
  // Newton: H = tril(qM) + sum_active D J^T J, then dense Cholesky solve.  With s.reuse the
  // factor of the previous call is kept while no active flag changed (the same H, the same bits).
  float* H = s.hs;
  if (!(s.reuse && s.factored && !s.changed)) {
    assemble_hessian(m, d, s.qM, H, s.adr, s.n, s.nz, lane);
    if (d.efc_h) {  // keep the assembled Hessian observable (lower triangle), as the reference does
      float* out = d.efc_h + W(s.w, nv * nv);
      if (out != H)
        for (int e = lane; e < nv * nv; e += 32) out[e] = H[e];
    }
    chol_any(H, nv, nv, lane, s.nz);
    s.factored = true;
  }
  warp_cho_solve(H, nv, nv, s.Mgrad, s.grad, lane);
}

__device__ __forceinline__ void eval_pt3(const float* q, float a, float* out) {
  out[0] = a * a * q[2] + a * q[1] + q[0];
  out[1] = 2.f * a * q[2] + q[1];
  out[2] = 2.f * q[2];
}
__device__ __forceinline__ bool in_bracket(const float* x, const float* y) {
  return (x[1] < y[1] && y[1] < 0.f) || (x[1] > y[1] && y[1] > 0.f);
}

// solver.py:737-869 with the iterative (:339-664) or parallel (:667-734) line search
__device__ void linesearch(SolverCtx& s) {
  const MjbModel& m = s.m;
  const MjbData& d = s.d;
  const int nv = s.nv, lane = s.lane;
  mul_m_ctx(s, s.mv, s.search);
  float q1 = 0.f, q2 = 0.f, q0 = 0.f;
  for (int i = lane; i < nv; i += 32) {
    q0 += s.gauss / float(nv);
    q1 += s.search[i] * (s.Ma[i] - s.qfrc_smooth[i]);
    q2 += 0.5f * s.search[i] * s.mv[i];
  }
  s.qg[0] = warp_sum(q0);
  s.qg[1] = warp_sum(q1);
  s.qg[2] = warp_sum(q2);
  for (int k = lane; k < s.n; k += 32) {
    const int r = s.adr + k;
    const float* J = d.efc_J + size_t(r) * nv;
    float jv = 0.f;
    for (int i = 0; i < nv; i++) jv += J[i] * s.search[i];
    const float Jaref = d.efc_Jaref[r], D = d.efc_D[r];
    d.efc_jv[r] = jv;
    d.efc_quad[3 * r] = 0.5f * Jaref * Jaref * D;
    d.efc_quad[3 * r + 1] = jv * Jaref * D;
    d.efc_quad[3 * r + 2] = 0.5f * jv * jv * D;
  }
  __syncwarp();
  if (m.ls_parallel) {
    int best = 0;
    float bestc = 0.f;
    for (int c = 0; c < m.nlsp; c++) {
      const float a = m.alpha_candidate[c];
      float t0 = 0.f, t1 = 0.f, t2 = 0.f;
      for (int k = lane; k < s.n; k += 32) {
        const int r = s.adr + k;
        if (d.efc_Jaref[r] + a * d.efc_jv[r] < 0.f) {
          t0 += d.efc_quad[3 * r];
          t1 += d.efc_quad[3 * r + 1];
          t2 += d.efc_quad[3 * r + 2];
        }
      }
      t0 = warp_sum(t0) + s.qg[0];
      t1 = warp_sum(t1) + s.qg[1];
      t2 = warp_sum(t2) + s.qg[2];
      const float cost = a * a * t2 + a * t1 + t0;
      if (c == 0 || cost < bestc) {
        bestc = cost;
        best = c;
      }
    }
    s.alpha = m.alpha_candidate[best];
  } else {
    const float snorm = sqrtf(s.search_dot);
    const float scale = m.meaninertia * float(max(1, nv));
    s.gtol = m.tolerance * m.ls_tolerance * snorm * scale;
    float p0[3];
    {
      float a0 = 0.f, a1 = 0.f, a2 = 0.f;
      for (int k = lane; k < s.n; k += 32) {
        const int r = s.adr + k;
        if (d.efc_Jaref[r] >= 0.f) continue;
        a0 += d.efc_quad[3 * r];
        a1 += d.efc_quad[3 * r + 1];
        a2 += 2.f * d.efc_quad[3 * r + 2];
      }
      p0[0] = s.qg[0] + warp_sum(a0);
      p0[1] = s.qg[1] + warp_sum(a1);
      p0[2] = 2.f * s.qg[2] + warp_sum(a2);
    }
    // evaluates the total cost polynomial at up to three step sizes at once
    auto totals = [&](int na, const float* al, float (*out)[3]) {
      float acc[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
      for (int k = lane; k < s.n; k += 32) {
        const int r = s.adr + k;
        const float jaref = d.efc_Jaref[r], jv = d.efc_jv[r];
        const float* q = d.efc_quad + 3 * r;
        for (int t = 0; t < na; t++) {
          if (jaref + al[t] * jv < 0.f) {
            float p[3];
            eval_pt3(q, al[t], p);
            acc[t][0] += p[0];
            acc[t][1] += p[1];
            acc[t][2] += p[2];
          }
        }
      }
      for (int t = 0; t < na; t++) {
        float g[3];
        eval_pt3(s.qg, al[t], g);
        out[t][0] = g[0] + warp_sum(acc[t][0]);
        out[t][1] = g[1] + warp_sum(acc[t][1]);
        out[t][2] = g[2] + warp_sum(acc[t][2]);
      }
    };
    float lo_alpha = -safe_div(p0[1], p0[2]);
    float lo[3], hi[3], hi_alpha;
    {
      float o[1][3];
      totals(1, &lo_alpha, o);
      lo[0] = o[0][0]; lo[1] = o[0][1]; lo[2] = o[0][2];
    }
    if (lo[1] < p0[1]) {
      hi[0] = p0[0]; hi[1] = p0[1]; hi[2] = p0[2];
      hi_alpha = 0.f;
    } else {
      hi[0] = lo[0]; hi[1] = lo[1]; hi[2] = lo[2];
      hi_alpha = lo_alpha;
      lo[0] = p0[0]; lo[1] = p0[1]; lo[2] = p0[2];
      lo_alpha = 0.f;
    }
    bool done = false;
    for (int it = 0; it < m.ls_iterations && !done; it++) {
      float al[3] = {lo_alpha - safe_div(lo[1], lo[2]), hi_alpha - safe_div(hi[1], hi[2]),
                     0.5f * (lo_alpha + hi_alpha)};
      float o[3][3];
      totals(3, al, o);
      float *lon = o[0], *hin = o[1], *mid = o[2];
      // _swap (solver.py:537-617)
      const bool s1 = in_bracket(lo, lon);
      if (s1) { lo[0] = lon[0]; lo[1] = lon[1]; lo[2] = lon[2]; lo_alpha = al[0]; }
      const bool s2 = in_bracket(lo, mid);
      if (s2) { lo[0] = mid[0]; lo[1] = mid[1]; lo[2] = mid[2]; lo_alpha = al[2]; }
      const bool s3 = in_bracket(lo, hin);
      if (s3) { lo[0] = hin[0]; lo[1] = hin[1]; lo[2] = hin[2]; lo_alpha = al[1]; }
      const bool t1 = in_bracket(hi, hin);
      if (t1) { hi[0] = hin[0]; hi[1] = hin[1]; hi[2] = hin[2]; hi_alpha = al[1]; }
      const bool t2 = in_bracket(hi, mid);
      if (t2) { hi[0] = mid[0]; hi[1] = mid[1]; hi[2] = mid[2]; hi_alpha = al[2]; }
      const bool t3 = in_bracket(hi, lon);
      if (t3) { hi[0] = lon[0]; hi[1] = lon[1]; hi[2] = lon[2]; hi_alpha = al[0]; }
      done = (!(s1 || s2 || s3) && !(t1 || t2 || t3)) || (lo[1] < 0.f && lo[1] > -s.gtol) ||
             (hi[1] > 0.f && hi[1] < s.gtol);
      float alpha = 0.f;
      const bool improved = lo[0] < p0[0] || hi[0] < p0[0];
      const bool lo_better = lo[0] < hi[0];
      if (improved && lo_better) alpha = lo_alpha;
      if (improved && !lo_better) alpha = hi_alpha;
      s.alpha = alpha;
    }
  }
  // solver.py:816-841
  for (int i = lane; i < nv; i += 32) {
    s.qacc[i] += s.alpha * s.search[i];
    s.Ma[i] += s.alpha * s.mv[i];
  }
  for (int k = lane; k < s.n; k += 32) d.efc_Jaref[s.adr + k] += s.alpha * d.efc_jv[s.adr + k];
  __syncwarp();
}

// solver.py:872-1000, any nv; hs: per-world nv*nv floats (the Newton Hessian and its factor);
// nz: null or generic_nz_floats(nv) floats of warp scratch for the sparse-row Hessian assembly;
// reuse: keep the factor while the active set is unchanged
__device__ __noinline__ void solve_generic(const MjbModel& m, const MjbData& d, int w, int lane,
                                           float* hs, float* nz, bool reuse) {
  const int nv = m.nv;
  SolverCtx s{m, d, w, lane, nv, d.world_efcadr[w], d.world_nefc[w]};
  s.nz = nz;
  s.reuse = reuse;
  s.qacc = d.qacc + W(w, nv);
  s.Ma = d.efc_Ma + W(w, nv);
  s.grad = d.efc_grad + W(w, nv);
  s.Mgrad = d.efc_Mgrad + W(w, nv);
  s.search = d.efc_search + W(w, nv);
  s.mv = d.efc_mv + W(w, nv);
  s.qfrc_constraint = d.qfrc_constraint + W(w, nv);
  s.qM = d.qM + (m.is_sparse ? W(w, m.nM) : W(w, nv * nv));
  s.qLD = d.qLD + (m.is_sparse ? W(w, m.nM) : W(w, nv * nv));
  s.qfrc_smooth = d.qfrc_smooth + W(w, nv);
  s.qacc_smooth = d.qacc_smooth + W(w, nv);
  s.hs = hs;
  s.alpha = 0.f;
  s.gtol = 0.f;
  const float* ws = d.qacc_warmstart + W(w, nv);
  for (int i = lane; i < nv; i += 32) s.qacc[i] = ws[i];
  __syncwarp();
  // _create_context (solver.py:26-72)
  s.cost = __int_as_float(0x7f800000);
  s.search_dot = 0.f;
  bool done = false;
  for (int k = lane; k < s.n; k += 32) {
    const int r = s.adr + k;
    const float* J = d.efc_J + size_t(r) * nv;
    float v = 0.f;
    for (int i = 0; i < nv; i++) v += J[i] * s.qacc[i];
    d.efc_Jaref[r] = v - d.efc_aref[r];
  }
  mul_m_ctx(s, s.Ma, s.qacc);
  update_constraint(s);
  update_gradient(s);
  float sd = 0.f;
  for (int i = lane; i < nv; i += 32) {
    const float v = -s.Mgrad[i];
    s.search[i] = v;
    sd += v * v;
  }
  s.search_dot = warp_sum(sd);
  __syncwarp();
  float* prev_grad = d.efc_prev_grad ? d.efc_prev_grad + W(w, nv) : nullptr;
  float* prev_Mgrad = d.efc_prev_Mgrad ? d.efc_prev_Mgrad + W(w, nv) : nullptr;
  float beta = 0.f;
  for (int it = 0; it < m.iterations && !done; it++) {
    linesearch(s);
    if (m.solver == 1) {
      for (int i = lane; i < nv; i += 32) {
        prev_grad[i] = s.grad[i];
        prev_Mgrad[i] = s.Mgrad[i];
      }
      __syncwarp();
    }
    update_constraint(s);
    update_gradient(s);
    if (m.solver == 1) {  // Polak-Ribiere (solver.py:918-970)
      float num = 0.f, den = 0.f;
      for (int i = lane; i < nv; i += 32) {
        num += s.grad[i] * (s.Mgrad[i] - prev_Mgrad[i]);
        den += prev_grad[i] * prev_Mgrad[i];
      }
      num = warp_sum(num);
      den = warp_sum(den);
      beta = fmaxf(0.f, num / fmaxf(kMinVal, den));
    }
    sd = 0.f;
    for (int i = lane; i < nv; i += 32) {
      float v = -s.Mgrad[i];
      if (m.solver == 1) v += beta * s.search[i];
      s.search[i] = v;
      sd += v * v;
    }
    s.search_dot = warp_sum(sd);
    __syncwarp();
    const float scale = m.meaninertia * float(max(1, nv));
    const float improvement = (s.prev_cost - s.cost) / scale;
    const float gradient = sqrtf(s.grad_dot) / scale;
    done = improvement < m.tolerance || gradient < m.tolerance;
  }
  float* wsw = d.qacc_warmstart + W(w, nv);
  for (int i = lane; i < nv; i += 32) wsw[i] = s.qacc[i];
  if (lane == 0) {
    if (d.efc_cost) d.efc_cost[w] = s.cost;
    if (d.efc_prev_cost) d.efc_prev_cost[w] = s.prev_cost;
    if (d.efc_gauss) d.efc_gauss[w] = s.gauss;
    if (d.efc_grad_dot) d.efc_grad_dot[w] = s.grad_dot;
    if (d.efc_search_dot) d.efc_search_dot[w] = s.search_dot;
    if (d.efc_gtol) d.efc_gtol[w] = s.gtol;
    if (d.efc_alpha) d.efc_alpha[w] = s.alpha;
    if (d.efc_beta) d.efc_beta[w] = beta;
    if (d.efc_done) d.efc_done[w] = done ? 1 : 0;
    if (d.efc_solver_niter) d.efc_solver_niter[w] = 0;  // never advanced by the reference
    if (d.efc_quad_gauss) {
      d.efc_quad_gauss[3 * w] = s.qg[0];
      d.efc_quad_gauss[3 * w + 1] = s.qg[1];
      d.efc_quad_gauss[3 * w + 2] = s.qg[2];
    }
  }
  __syncwarp();
}


// ------------------------------------------------------------------------------------------
// Solver for nv <= 32: lane i owns dof i, so every per-dof vector (qacc, Ma, grad, Mgrad, search,
// mv, ...) lives in one register per lane; qM, the constraint Jacobian rows (when a world has at
// most kSolverRows rows) and the Hessian factor live in the warp's shared-memory slice; per-row
// scalars stay in the flat efc arrays, each touched only by the lane that owns the row.

#ifndef MJB_JROWS
#define MJB_JROWS 32
#endif
constexpr int kSolverRows = MJB_JROWS;

__host__ __device__ __forceinline__ int round4(int x) { return (x + 3) & ~3; }
// Per-warp layout, every part 16-byte aligned, every matrix row tile_ld(nv) floats with the
// columns from nv to the next multiple of 4 zero: Ls (the factor tile, nv rows) | Js (kSolverRows
// rows) | Ms (qM, nv rows) | vs (32) | F (kSolverRows).  The tile comes first so the fused step can
// use it for the mass-matrix factorisations too.  Lanes read their own rows as float4 without bank
// conflicts (see tile_ld).
__host__ __device__ __forceinline__ size_t solver_smem_floats(int nv) {
  return size_t(round4(2 * tile_floats(nv) + kSolverRows * tile_ld(nv) + 32 + kSolverRows));
}

// sum_j a_j b_j over the first 4 * nq columns of two 16-byte aligned rows (four partial sums)
__device__ __forceinline__ float dotq(const float* a, const float* b, int nq) {
  const float4* a4 = reinterpret_cast<const float4*>(a);
  const float4* b4 = reinterpret_cast<const float4*>(b);
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    if (q < nq) {
      const float4 x = a4[q], y = b4[q];
      s0 += x.x * y.x;
      s1 += x.y * y.y;
      s2 += x.z * y.z;
      s3 += x.w * y.w;
    }
  }
  return (s0 + s1) + (s2 + s3);
}

struct Small {
  const MjbModel& m;
  const MjbData& d;
  int w, lane, nv, adr, n, ldj;
  int ld, nq;                   // staged row stride and float4 count per row (4 * nq >= nv)
  bool staged;                  // J rows copied to shared memory (else read from efc_J)
  bool own;
  // With staged rows (n <= 32) lane k owns row k and keeps its scalars in registers; the flat
  // efc arrays are then only written (they stay the observable outputs).
  float rJaref = 0.f, rjv = 0.f, rD = 0.f, rq0 = 0.f, rq1 = 0.f, rq2 = 0.f;
  int ract = 0;
  bool reuse = false;           // keep the factor of H while the active set is unchanged
  bool factored = false;        // Ls holds the factor of H for the active set factored_mask
  unsigned factored_mask = 0u;
  float *Ms, *Ls, *vs, *F;
  double* Ld = nullptr;         // precision form: the FP64 factor tile
  const float* J;
  // per-dof registers
  float qacc, Ma, grad, Mgrad, search, mv, qfs, qas, qfc;
  // per-world scalars (uniform across lanes)
  float cost, prev_cost, gauss, grad_dot, search_dot, gtol, alpha;
  float qg[3];

  // (M v)_lane
  __device__ __forceinline__ float mulM(float v) {
    vs[lane] = own ? v : 0.f;
    __syncwarp();
    const float s = own ? dotq(Ms + lane * ld, vs, nq) : 0.f;
    __syncwarp();
    return s;
  }
  // publishes v for row-wise dot products; call before rowdot, __syncwarp() after the last use
  __device__ __forceinline__ void publish(float v) {
    vs[lane] = own ? v : 0.f;
    __syncwarp();
  }
  template <bool ST>
  __device__ __forceinline__ float rowdot(int k) const {
    const float* Jr = J + size_t(k) * ldj;
    if (ST) return dotq(Jr, vs, nq);
    float s = 0.f;
    for (int j = 0; j < nv; j++) s += Jr[j] * vs[j];
    return s;
  }
};

// H = tril(qM) + sum_k c_k J_k^T J_k for nv <= 32 on the tensor pipe, in split TF32 (mjb_tc.cuh):
// H = qM + A B with A = J^T (nv x na) and B = diag(c) J (na x nv) over the na rows listed in idx
// (the rows with c != 0), one warp.  The output is computed in the m16n8 tiles that touch the lower
// triangle, (rows 16 mt .., columns 8 nt ..) = (0, 0), (0, 1) and, for nv > 16, (1, 0) .. (1, 3);
// the k dimension runs over the listed rows eight at a time.  Ms / Js: qM and the staged rows
// (stride ld floats, zero padded to 4 ceil(nv / 4) columns); writes rows and columns < nv (and the
// padding column of an odd nv) of H (stride ldh elements of T), entries above the diagonal too.
template <typename T>
__device__ __forceinline__ void hessian_tc(const float* Ms, const float* Js, int ld, const float* c,
                                           const int* idx, int na, int nv, T* H, int ldh,
                                           int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int ncol = (nv + 3) & ~3;
  const bool two = nv > 16;
  constexpr int kMt[6] = {0, 0, 1, 1, 1, 1}, kNt[6] = {0, 1, 0, 1, 2, 3};
  float acc[6][4];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    const int r0 = 16 * kMt[i] + g, r1 = r0 + 8, cc = 8 * kNt[i] + 2 * t;
    const float2 z = make_float2(0.f, 0.f);
    const float2 v0 = (r0 < nv && cc < ncol) ? *reinterpret_cast<const float2*>(Ms + r0 * ld + cc) : z;
    const float2 v1 = (r1 < nv && cc < ncol) ? *reinterpret_cast<const float2*>(Ms + r1 * ld + cc) : z;
    acc[i][0] = v0.x;
    acc[i][1] = v0.y;
    acc[i][2] = v1.x;
    acc[i][3] = v1.y;
  }
  for (int k0 = 0; k0 < na; k0 += 8) {
    const int ka = k0 + t, kb = ka + 4;
    const int ra = ka < na ? idx[ka] : -1, rb = kb < na ? idx[kb] : -1;
    const float ca = ra >= 0 ? c[ra] : 0.f, cb = rb >= 0 ? c[rb] : 0.f;
    float ja[4], jb[4];  // J[ra][g + 8 q], J[rb][g + 8 q]
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int col = g + 8 * q;
      ja[q] = (ra >= 0 && col < ncol) ? Js[ra * ld + col] : 0.f;
      jb[q] = (rb >= 0 && col < ncol) ? Js[rb * ld + col] : 0.f;
    }
    const FragA a0 = frag_a(ja[0], ja[1], jb[0], jb[1]);  // rows 0..15 of A: dofs g, g + 8
    FragB b[4];
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = frag_b(ca * ja[q], cb * jb[q]);
    mma_3xtf32(acc[0], a0, b[0]);
    mma_3xtf32(acc[1], a0, b[1]);
    if (two) {
      const FragA a1 = frag_a(ja[2], ja[3], jb[2], jb[3]);  // rows 16..31: dofs g + 16, g + 24
#pragma unroll
      for (int q = 0; q < 4; q++) mma_3xtf32(acc[2 + q], a1, b[q]);
    }
  }
#pragma unroll
  for (int i = 0; i < 6; i++) {
    if (i >= 2 && !two) break;
    const int r0 = 16 * kMt[i] + g, r1 = r0 + 8, cc = 8 * kNt[i] + 2 * t;
    if (cc < nv) {  // cc + 1 < nv, or the padding column of an odd nv (< ldh)
      if (r0 < nv) {
        H[r0 * ldh + cc] = T(acc[i][0]);
        H[r0 * ldh + cc + 1] = T(acc[i][1]);
      }
      if (r1 < nv) {
        H[r1 * ldh + cc] = T(acc[i][2]);
        H[r1 * ldh + cc + 1] = T(acc[i][3]);
      }
    }
  }
}

// Newton step direction H^-1 grad for nv <= 32 (solver.py:234-290).  When `refactor` is set,
// lane i assembles row i of H = tril(qM) + sum_k c_k J_k^T J_k in registers (c_k = D_k for active
// rows, 0 otherwise; inactive rows are skipped), stores it to the tile Ls and factors it in place;
// otherwise Ls already holds the factor of the same H.  The coefficients come from C
// (staged rows) or, when C is null, from the rows' active flags and D.  Returns element `lane` of the
// solution.  Staged Jacobian rows are read as float4 broadcasts.
// TC (staged rows only): H is assembled by hessian_tc on the tensor pipe instead; ix is 32 ints
// of warp scratch for its row list.
template <bool PREC, bool ST, bool TC = false>
__device__ __forceinline__ float newton_direction(const float* Ms, int ld, const float* J, int ldj,
                                               const float* C, const int* act,
                                               const float* D, int n, float* Ls, int nv,
                                               float grad, int lane, bool refactor,
                                               double* Ld = nullptr, int* ix = nullptr) {
  const int nq = (nv + 3) >> 2;
  const bool own = lane < nv;
  if (TC && ST && refactor) {  // n <= 32: lane k owns row k; list the rows with a nonzero coefficient
    const bool on = lane < n && C[lane] != 0.f;
    const unsigned mk = __ballot_sync(WARP_FULL, on);
    if (on) ix[__popc(mk & ((1u << lane) - 1u))] = lane;
    __syncwarp();
    if (PREC) {
      hessian_tc(Ms, J, ldj, C, ix, __popc(mk), nv, Ld, ld, lane);
      __syncwarp();
      chol_tile_d(Ld, ld, nv, lane);
    } else {
      hessian_tc(Ms, J, ldj, C, ix, __popc(mk), nv, Ls, ld, lane);
      __syncwarp();
      chol_tile(Ls, ld, nv, lane);
    }
  } else if (refactor) {
    float h[32];  // row `lane` of qM (columns past nv are zero; entries above the diagonal unused)
    const float4* M4 = reinterpret_cast<const float4*>(Ms + min(lane, nv - 1) * ld);
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float4 v = q < nq ? M4[q] : make_float4(0.f, 0.f, 0.f, 0.f);
      h[4 * q] = v.x;
      h[4 * q + 1] = v.y;
      h[4 * q + 2] = v.z;
      h[4 * q + 3] = v.w;
    }
    if (ST) {
      // staged rows (n <= 32, zero-padded, 16-byte aligned): the rows with c != 0 taken from a
      // ballot mask in increasing order, two per pass (each h[j] still adds the rows' terms in
      // row order)
      unsigned mk = __ballot_sync(WARP_FULL, lane < n && C[lane] != 0.f);
      while (mk) {
        const int k0 = __ffs(mk) - 1;
        mk &= mk - 1u;
        const float* J0 = J + k0 * ldj;
        const float a0 = own ? C[k0] * J0[lane] : 0.f;
        const float4* A4 = reinterpret_cast<const float4*>(J0);
        if (mk) {
          const int k1 = __ffs(mk) - 1;
          mk &= mk - 1u;
          const float* J1 = J + k1 * ldj;
          const float a1 = own ? C[k1] * J1[lane] : 0.f;
          const float4* B4 = reinterpret_cast<const float4*>(J1);
#pragma unroll
          for (int q = 0; q < 8; q++) {
            if (q < nq) {
              const float4 u = A4[q], v = B4[q];
              h[4 * q] += a0 * u.x;
              h[4 * q + 1] += a0 * u.y;
              h[4 * q + 2] += a0 * u.z;
              h[4 * q + 3] += a0 * u.w;
              h[4 * q] += a1 * v.x;
              h[4 * q + 1] += a1 * v.y;
              h[4 * q + 2] += a1 * v.z;
              h[4 * q + 3] += a1 * v.w;
            }
          }
        } else {
#pragma unroll
          for (int q = 0; q < 8; q++) {
            if (q < nq) {
              const float4 u = A4[q];
              h[4 * q] += a0 * u.x;
              h[4 * q + 1] += a0 * u.y;
              h[4 * q + 2] += a0 * u.z;
              h[4 * q + 3] += a0 * u.w;
            }
          }
        }
      }
    } else {
      for (int k = 0; k < n; k++) {
        const float c = C ? C[k] : (act[k] ? D[k] : 0.f);
        if (c == 0.f) continue;
        const float* Jr = J + size_t(k) * ldj;
        const float a = own ? c * Jr[lane] : 0.f;
#pragma unroll
        for (int j = 0; j < 32; j++)
          if (j < nv) h[j] += a * Jr[j];
      }
    }
    if (PREC) {  // precision form: the FP32-assembled row, factored and solved in FP64
      if (own)
#pragma unroll
        for (int j = 0; j < 32; j++)
          if (j < nv) Ld[lane * ld + j] = h[j];
      __syncwarp();
      chol_tile_d(Ld, ld, nv, lane);
    } else {
      if (own) {  // the whole row (entries above the diagonal are never read)
        float4* row = reinterpret_cast<float4*>(Ls + lane * ld);
#pragma unroll
        for (int q = 0; q < 8; q++)
          if (q < nq) row[q] = make_float4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
      }
      __syncwarp();
      chol_tile(Ls, ld, nv, lane);
    }
  }
  if (PREC) return float(cho_solve_tile_d(Ld, ld, nv, double(grad), lane));
  return cho_solve_tile(Ls, ld, nv, grad, lane);
}

// Line-search coefficient sums across the warp: base + sum of x, accumulated in FP64 in the
// precision form.
__device__ __forceinline__ float ls_sum(float base, float x, bool prec) {
  if (prec) return float(double(base) + warp_sum_d(double(x)));
  return base + warp_sum(x);
}

// solver.py:75-173
template <bool ST>
__device__ void small_update_constraint(Small& s) {
  const MjbData& d = s.d;
  s.prev_cost = s.cost;
  float c = 0.f;
  if (ST) {
    if (s.lane < s.n) {
      const int r = s.adr + s.lane;
      const float Jaref = s.rJaref, D = s.rD;
      const int active = Jaref < 0.f;
      s.ract = active;
      d.efc_active[r] = active;
      const float f = active ? -1.f * D * Jaref : 0.f;
      d.efc_force[r] = f;
      s.F[s.lane] = f;
      if (active) c += 0.5f * D * Jaref * Jaref;
    }
  } else {
    for (int k = s.lane; k < s.n; k += 32) {
      const int r = s.adr + k;
      const float Jaref = d.efc_Jaref[r], D = d.efc_D[r];
      const int active = Jaref < 0.f;
      d.efc_active[r] = active;
      const float f = active ? -1.f * D * Jaref : 0.f;
      d.efc_force[r] = f;
      s.F[k] = f;
      if (active) c += 0.5f * D * Jaref * Jaref;
    }
  }
  c = warp_sum(c);
  __syncwarp();
  float q = 0.f;
  if (s.own)
    for (int k = 0; k < s.n; k++) q += s.J[size_t(k) * s.ldj + s.lane] * s.F[k];
  s.qfc = q;
  float g = s.own ? 0.5f * (s.Ma - s.qfs) * (s.qacc - s.qas) : 0.f;
  g = warp_sum(g);
  s.gauss = g;
  s.cost = c + g;
  __syncwarp();
}

// solver.py:176-312
template <bool PREC, bool ST, bool CG, bool TC>
__device__ void small_update_gradient(Small& s) {
  const MjbModel& m = s.m;
  const MjbData& d = s.d;
  const int nv = s.nv, lane = s.lane;
  s.grad = s.own ? s.Ma - s.qfs - s.qfc : 0.f;
  s.grad_dot = warp_sum(s.grad * s.grad);
  if (CG) {  // CG: Mgrad = M^-1 grad with the qLD factor
    float* gg = d.efc_grad + W(s.w, nv);
    float* mg = d.efc_Mgrad + W(s.w, nv);
    if (s.own) gg[lane] = s.grad;
    __syncwarp();
    solve_blocks(m, d.qLD + W(s.w, nv * nv), mg, gg, lane);
    s.Mgrad = s.own ? mg[lane] : 0.f;
    __syncwarp();
    return;
  }
  // H depends on the solve's inputs only through the active set, so with s.reuse the factor of
  // the previous call is kept (bit-identical) while the set of active rows is unchanged; rows
  // past the first 32 are not tracked, so such worlds refactor every time.  Without s.reuse every
  // call refactors, as the reference does.
  constexpr bool staged = ST;  // unstaged rows keep F in efc_force, which must survive
  const unsigned mask = __ballot_sync(
      WARP_FULL, lane < s.n && (staged ? s.ract != 0 : d.efc_active[s.adr + lane] != 0));
  const bool refactor = !s.reuse || !s.factored || s.n > 32 || mask != s.factored_mask;
  if (refactor && staged) {  // coefficient of each row in J^T D J: D when active, else 0
    if (lane < s.n) s.F[lane] = s.ract ? s.rD : 0.f;
    __syncwarp();
  }
  s.Mgrad = newton_direction<PREC, ST, TC>(s.Ms, s.ld, s.J, s.ldj, staged ? s.F : nullptr,
                             d.efc_active + s.adr, d.efc_D + s.adr, s.n, s.Ls, nv, s.grad, lane,
                             refactor, s.Ld, reinterpret_cast<int*>(s.vs));
  s.factored = true;
  s.factored_mask = mask;
}

// solver.py:737-869
template <bool PREC, bool ST, bool LSP>
__device__ void small_linesearch(Small& s) {
  const MjbModel& m = s.m;
  const MjbData& d = s.d;
  const int nv = s.nv, lane = s.lane;
  constexpr bool prec = PREC;
  // f(Jaref, jv, quad0, quad1, quad2) for each of this lane's rows (registers when staged)
  auto rows = [&](auto&& f) {
    if (ST) {
      if (lane < s.n) f(s.rJaref, s.rjv, s.rq0, s.rq1, s.rq2);
    } else {
      for (int k = lane; k < s.n; k += 32) {
        const int r = s.adr + k;
        const float* q = d.efc_quad + 3 * r;
        f(d.efc_Jaref[r], d.efc_jv[r], q[0], q[1], q[2]);
      }
    }
  };
  s.mv = s.mulM(s.search);
  {
    float q0 = s.own ? s.gauss / float(nv) : 0.f;
    float q1 = s.own ? s.search * (s.Ma - s.qfs) : 0.f;
    float q2 = s.own ? 0.5f * s.search * s.mv : 0.f;
    s.qg[0] = ls_sum(0.f, q0, prec);
    s.qg[1] = ls_sum(0.f, q1, prec);
    s.qg[2] = ls_sum(0.f, q2, prec);
  }
  s.publish(s.search);
  if (ST) {
    if (lane < s.n) {
      const int r = s.adr + lane;
      const float jv = s.template rowdot<ST>(lane);
      const float Jaref = s.rJaref, D = s.rD;
      s.rjv = jv;
      s.rq0 = 0.5f * Jaref * Jaref * D;
      s.rq1 = jv * Jaref * D;
      s.rq2 = 0.5f * jv * jv * D;
      d.efc_jv[r] = jv;
      d.efc_quad[3 * r] = s.rq0;
      d.efc_quad[3 * r + 1] = s.rq1;
      d.efc_quad[3 * r + 2] = s.rq2;
    }
  } else {
    for (int k = lane; k < s.n; k += 32) {
      const int r = s.adr + k;
      const float jv = s.template rowdot<ST>(k);
      const float Jaref = d.efc_Jaref[r], D = d.efc_D[r];
      d.efc_jv[r] = jv;
      d.efc_quad[3 * r] = 0.5f * Jaref * Jaref * D;
      d.efc_quad[3 * r + 1] = jv * Jaref * D;
      d.efc_quad[3 * r + 2] = 0.5f * jv * jv * D;
    }
  }
  __syncwarp();
  if (LSP) {
    int best = 0;
    float bestc = 0.f;
    for (int c = 0; c < m.nlsp; c++) {
      const float a = m.alpha_candidate[c];
      float t0 = 0.f, t1 = 0.f, t2 = 0.f;
      rows([&](float jaref, float jv, float q0, float q1, float q2) {
        if (jaref + a * jv < 0.f) {
          t0 += q0;
          t1 += q1;
          t2 += q2;
        }
      });
      t0 = ls_sum(s.qg[0], t0, prec);
      t1 = ls_sum(s.qg[1], t1, prec);
      t2 = ls_sum(s.qg[2], t2, prec);
      const float cost = a * a * t2 + a * t1 + t0;
      if (c == 0 || cost < bestc) {
        bestc = cost;
        best = c;
      }
    }
    s.alpha = m.alpha_candidate[best];
  } else {
    const float scale = m.meaninertia * float(max(1, nv));
    s.gtol = m.tolerance * m.ls_tolerance * sqrtf(s.search_dot) * scale;
    float p0[3];
    {
      float a0 = 0.f, a1 = 0.f, a2 = 0.f;
      rows([&](float jaref, float, float q0, float q1, float q2) {
        if (jaref >= 0.f) return;
        a0 += q0;
        a1 += q1;
        a2 += 2.f * q2;
      });
      p0[0] = ls_sum(s.qg[0], a0, prec);
      p0[1] = ls_sum(s.qg[1], a1, prec);
      p0[2] = ls_sum(2.f * s.qg[2], a2, prec);
    }
    auto totals = [&](int na, const float* al, float (*out)[3]) {
      float acc[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
      rows([&](float jaref, float jv, float q0, float q1, float q2) {
        const float q[3] = {q0, q1, q2};
        for (int t = 0; t < na; t++) {
          if (jaref + al[t] * jv < 0.f) {
            float p[3];
            eval_pt3(q, al[t], p);
            acc[t][0] += p[0];
            acc[t][1] += p[1];
            acc[t][2] += p[2];
          }
        }
      });
      for (int t = 0; t < na; t++) {
        float g[3];
        eval_pt3(s.qg, al[t], g);
        out[t][0] = ls_sum(g[0], acc[t][0], prec);
        out[t][1] = ls_sum(g[1], acc[t][1], prec);
        out[t][2] = ls_sum(g[2], acc[t][2], prec);
      }
    };
    float lo_alpha = -safe_div(p0[1], p0[2]);
    float lo[3], hi[3], hi_alpha;
    {
      float o[1][3];
      totals(1, &lo_alpha, o);
      lo[0] = o[0][0]; lo[1] = o[0][1]; lo[2] = o[0][2];
    }
    if (lo[1] < p0[1]) {
      hi[0] = p0[0]; hi[1] = p0[1]; hi[2] = p0[2];
      hi_alpha = 0.f;
    } else {
      hi[0] = lo[0]; hi[1] = lo[1]; hi[2] = lo[2];
      hi_alpha = lo_alpha;
      lo[0] = p0[0]; lo[1] = p0[1]; lo[2] = p0[2];
      lo_alpha = 0.f;
    }
    bool done = false;
    for (int it = 0; it < m.ls_iterations && !done; it++) {
      float al[3] = {lo_alpha - safe_div(lo[1], lo[2]), hi_alpha - safe_div(hi[1], hi[2]),
                     0.5f * (lo_alpha + hi_alpha)};
      float o[3][3];
      totals(3, al, o);
      float *lon = o[0], *hin = o[1], *mid = o[2];
      const bool s1 = in_bracket(lo, lon);
      if (s1) { lo[0] = lon[0]; lo[1] = lon[1]; lo[2] = lon[2]; lo_alpha = al[0]; }
      const bool s2 = in_bracket(lo, mid);
      if (s2) { lo[0] = mid[0]; lo[1] = mid[1]; lo[2] = mid[2]; lo_alpha = al[2]; }
      const bool s3 = in_bracket(lo, hin);
      if (s3) { lo[0] = hin[0]; lo[1] = hin[1]; lo[2] = hin[2]; lo_alpha = al[1]; }
      const bool t1 = in_bracket(hi, hin);
      if (t1) { hi[0] = hin[0]; hi[1] = hin[1]; hi[2] = hin[2]; hi_alpha = al[1]; }
      const bool t2 = in_bracket(hi, mid);
      if (t2) { hi[0] = mid[0]; hi[1] = mid[1]; hi[2] = mid[2]; hi_alpha = al[2]; }
      const bool t3 = in_bracket(hi, lon);
      if (t3) { hi[0] = lon[0]; hi[1] = lon[1]; hi[2] = lon[2]; hi_alpha = al[0]; }
      done = (!(s1 || s2 || s3) && !(t1 || t2 || t3)) || (lo[1] < 0.f && lo[1] > -s.gtol) ||
             (hi[1] > 0.f && hi[1] < s.gtol);
      float alpha = 0.f;
      const bool improved = lo[0] < p0[0] || hi[0] < p0[0];
      const bool lo_better = lo[0] < hi[0];
      if (improved && lo_better) alpha = lo_alpha;
      if (improved && !lo_better) alpha = hi_alpha;
      s.alpha = alpha;
    }
  }
  if (s.own) {
    s.qacc += s.alpha * s.search;
    s.Ma += s.alpha * s.mv;
  }
  if (ST) {
    if (lane < s.n) {
      s.rJaref += s.alpha * s.rjv;
      d.efc_Jaref[s.adr + lane] = s.rJaref;
    }
  } else {
    for (int k = lane; k < s.n; k += 32) d.efc_Jaref[s.adr + k] += s.alpha * d.efc_jv[s.adr + k];
  }
  __syncwarp();
}

// The iterations of solve_small once the world's rows are placed.  ST: rows staged in shared
// memory (n <= kSolverRows); CG: the CG solver (else Newton); LSP: the parallel line search (else
// the iterative one) -- compile-time choices, so that each path's code is straight.
template <bool PREC, bool ST, bool CG, bool LSP, bool TC>
__device__ void solve_small_run(Small& s) {
  const MjbModel& m = s.m;
  const MjbData& d = s.d;
  const int nv = s.nv, lane = s.lane, w = s.w, adr = s.adr, n = s.n;
  // _create_context (solver.py:26-72)
  s.cost = __int_as_float(0x7f800000);
  s.publish(s.qacc);
  if (ST) {
    if (lane < n) {
      s.rD = d.efc_D[adr + lane];
      s.rJaref = s.template rowdot<ST>(lane) - d.efc_aref[adr + lane];
      d.efc_Jaref[adr + lane] = s.rJaref;
    }
  } else {
    for (int k = lane; k < n; k += 32) d.efc_Jaref[adr + k] = s.template rowdot<ST>(k) - d.efc_aref[adr + k];
  }
  __syncwarp();
  s.Ma = s.mulM(s.qacc);
  small_update_constraint<ST>(s);
  small_update_gradient<PREC, ST, CG, TC>(s);
  s.search = -s.Mgrad;
  s.search_dot = warp_sum(s.search * s.search);
  bool done = false;
  float beta = 0.f, prev_grad = 0.f, prev_Mgrad = 0.f;
  for (int it = 0; it < m.iterations && !done; it++) {
    small_linesearch<PREC, ST, LSP>(s);
    prev_grad = s.grad;
    prev_Mgrad = s.Mgrad;
    small_update_constraint<ST>(s);
    small_update_gradient<PREC, ST, CG, TC>(s);
    if (CG) {  // Polak-Ribiere (solver.py:918-970)
      const float num = warp_sum(s.own ? s.grad * (s.Mgrad - prev_Mgrad) : 0.f);
      const float den = warp_sum(s.own ? prev_grad * prev_Mgrad : 0.f);
      beta = fmaxf(0.f, num / fmaxf(kMinVal, den));
    }
    float v = -s.Mgrad;
    if (CG) v += beta * s.search;
    s.search = s.own ? v : 0.f;
    s.search_dot = warp_sum(s.search * s.search);
    const float scale = m.meaninertia * float(max(1, nv));
    done = (s.prev_cost - s.cost) / scale < m.tolerance || sqrtf(s.grad_dot) / scale < m.tolerance;
  }
  if (s.own) {
    const size_t o = W(w, nv) + lane;
    d.qacc[o] = s.qacc;
    d.qacc_warmstart[o] = s.qacc;
    d.qfrc_constraint[o] = s.qfc;
    d.efc_Ma[o] = s.Ma;
    d.efc_grad[o] = s.grad;
    d.efc_Mgrad[o] = s.Mgrad;
    d.efc_search[o] = s.search;
    d.efc_mv[o] = s.mv;
    if (d.efc_prev_grad) d.efc_prev_grad[o] = prev_grad;
    if (d.efc_prev_Mgrad) d.efc_prev_Mgrad[o] = prev_Mgrad;
  }
  if (lane == 0) {
    if (d.efc_cost) d.efc_cost[w] = s.cost;
    if (d.efc_prev_cost) d.efc_prev_cost[w] = s.prev_cost;
    if (d.efc_gauss) d.efc_gauss[w] = s.gauss;
    if (d.efc_grad_dot) d.efc_grad_dot[w] = s.grad_dot;
    if (d.efc_search_dot) d.efc_search_dot[w] = s.search_dot;
    if (d.efc_gtol) d.efc_gtol[w] = s.gtol;
    if (d.efc_alpha) d.efc_alpha[w] = s.alpha;
    if (d.efc_beta) d.efc_beta[w] = beta;
    if (d.efc_done) d.efc_done[w] = done ? 1 : 0;
    if (d.efc_solver_niter) d.efc_solver_niter[w] = 0;
    if (d.efc_quad_gauss) {
      d.efc_quad_gauss[3 * w] = s.qg[0];
      d.efc_quad_gauss[3 * w + 1] = s.qg[1];
      d.efc_quad_gauss[3 * w + 2] = s.qg[2];
    }
  }
  __syncwarp();
}

// solver.py:872-1000 for nv <= 32; sm: solver_smem_floats(nv) floats of warp-private scratch
// PREC: the precision form (FP64 Hessian factor-solve and line-search sums; the double tile at
// sm + solver_smem_floats(nv))
template <bool PREC = false, bool TC = false>
__device__ void solve_small(const MjbModel& m, const MjbData& d, int w, int lane, float* sm,
                            bool reuse) {
  const int nv = m.nv;
  const int adr = d.world_efcadr[w], n = d.world_nefc[w];
  Small s{m, d, w, lane, nv, adr, n};
  s.own = lane < nv;
  s.reuse = reuse;
  s.ld = tile_ld(nv);
  s.nq = (nv + 3) >> 2;
  s.Ls = sm;
  if (PREC) s.Ld = reinterpret_cast<double*>(sm + solver_smem_floats(nv));
  float* Js = sm + tile_floats(nv);
  s.Ms = Js + kSolverRows * s.ld;
  s.vs = s.Ms + tile_floats(nv);
  s.F = s.vs + 32;
  const int ncol = 4 * s.nq;  // staged columns: nv, zero padded to a multiple of 4
  const float* Jg = d.efc_J + size_t(adr) * nv;
  if (n <= kSolverRows) {
    copy_rows(Jg, nv, Js, s.ld, n, nv, ncol, lane);  // rows zero padded for float4 reads
    s.J = Js;
    s.ldj = s.ld;
    s.staged = true;
  } else {
    s.J = Jg;
    s.ldj = nv;
    s.staged = false;
    s.F = d.efc_force + adr;  // rows beyond the staged capacity broadcast through global memory
  }
  const float* qMg = d.qM + W(w, nv * nv);
  copy_rows(qMg, nv, s.Ms, s.ld, nv, nv, ncol, lane);
  s.qacc = s.own ? d.qacc_warmstart[W(w, nv) + lane] : 0.f;
  s.qfs = s.own ? d.qfrc_smooth[W(w, nv) + lane] : 0.f;
  s.qas = s.own ? d.qacc_smooth[W(w, nv) + lane] : 0.f;
  s.alpha = 0.f;
  s.gtol = 0.f;
  s.qg[0] = s.qg[1] = s.qg[2] = 0.f;
  __syncwarp();
  const bool cg = m.solver == 1, lsp = m.ls_parallel != 0;
  if (s.staged) {
    if (!cg && !lsp) solve_small_run<PREC, true, false, false, TC>(s);
    else if (!cg) solve_small_run<PREC, true, false, true, TC>(s);
    else if (!lsp) solve_small_run<PREC, true, true, false, TC>(s);
    else solve_small_run<PREC, true, true, true, TC>(s);
  } else {
    if (!cg && !lsp) solve_small_run<PREC, false, false, false, TC>(s);
    else if (!cg) solve_small_run<PREC, false, false, true, TC>(s);
    else if (!lsp) solve_small_run<PREC, false, true, false, TC>(s);
    else solve_small_run<PREC, false, true, true, TC>(s);
  }
}

// Dispatch: the register / shared-memory solver when nv <= 32 and the caller provides its scratch
// (solver_smem_floats(nv) floats), else the generic solver with an nv x nv Hessian tile `hs`.
// reuse: keep the Newton Hessian's factor across iterations with an unchanged active set.
// For nv > 32 or a sparse mass matrix, sm (when given) is the generic solver's scratch of at least
// generic_nz_floats(nv) floats.
// TC: the Newton Hessian of staged rows assembled on the tensor pipe (split TF32, hessian_tc)
template <bool PREC = false, bool TC = false>
__device__ __forceinline__ void solve(const MjbModel& m, const MjbData& d, int w, int lane,
                                      float* sm, float* hs, bool reuse = false) {
  if (m.nv <= 32 && sm && !m.is_sparse) solve_small<PREC, TC>(m, d, w, lane, sm, reuse);
  else solve_generic(m, d, w, lane, hs, (m.nv > 32 || m.is_sparse) ? sm : nullptr, reuse);
}

}  // namespace mjb
