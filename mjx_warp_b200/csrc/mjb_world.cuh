// Per-world stages of the batched step, executed by one warp per world.
//
// Each function evaluates one stage of the reference pipeline (mujoco_warp/_src/*.py, cited per
// function) for world `w` with the 32 lanes of the calling warp cooperating: lanes stride over
// the bodies of a tree level, over joints, dofs, geoms, candidate pairs, contacts or constraint
// rows.  Tree recursions run level by level from the BFS tables (body_tree / body_treeadr) with
// a __syncwarp() between levels; accumulations into a parent gather over that parent's children
// (body_child tables) instead of the reference's float atomics, so every result is
// deterministic.  All pointers are generic: the plain per-stage kernels pass global memory, the
// fused step passes the same layout.
#pragma once

#include "../../include/mjb200.h"
#include "mjb_math.cuh"

// Cholesky for n <= 32 blocks: 0 = memory rows (chol_lower, the faster one measured), 1 = register rows (chol32)
#ifndef MJB_CHOL
#define MJB_CHOL 0
#endif
// the shared-memory factor / solve routines: called (1) or inlined into each caller (0)
#ifndef MJB_TILE_CALL
#define MJB_TILE_CALL 1
#endif
#if MJB_TILE_CALL
#define MJB_TILE_FN __noinline__
#else
#define MJB_TILE_FN __forceinline__
#endif

namespace mjb {

#define WARP_FULL 0xffffffffu

__device__ __forceinline__ size_t W(int w, int n) { return size_t(w) * size_t(n); }

// Stages written for L lanes per world (L = 32: one world per warp; L = 8 or 16: 32 / L worlds per
// warp, the world's lanes an aligned group): `lane` is the lane within the world's group, loops
// stride by L and lsync<L> synchronises the group.
template <int L>
__device__ __forceinline__ void lsync() {
  static_assert(L == 8 || L == 16 || L == 32, "lanes per world");
  if constexpr (L == 32) __syncwarp();
  else __syncwarp(((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1)));
}

// ------------------------------------------------------------------------------------------
// smooth.py:32-145 — forward kinematics
template <int L = 32>
__device__ void kinematics(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nb = m.nbody;
  const float* qpos = d.qpos + W(w, m.nq);
  float* xpos = d.xpos + W(w, 3 * nb);
  float* xquat = d.xquat + W(w, 4 * nb);
  float* xmat = d.xmat + W(w, 9 * nb);
  float* xipos = d.xipos + W(w, 3 * nb);
  float* ximat = d.ximat + W(w, 9 * nb);
  float* xanchor = d.xanchor + W(w, 3 * m.njnt);
  float* xaxis = d.xaxis + W(w, 3 * m.njnt);
  if (lane == 0) {  // _root (smooth.py:37-43)
    st3(xpos, mk3(0, 0, 0));
    st4(xquat, q4{1, 0, 0, 0});
    st3(xipos, mk3(0, 0, 0));
    m33 eye{{1, 0, 0, 0, 1, 0, 0, 0, 1}};
    st9(xmat, eye);
    st9(ximat, eye);
  }
  lsync<L>();
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += L) {  // _level (smooth.py:46-109)
      const int b = m.body_tree[n];
      const int jntadr = m.body_jntadr[b], jntnum = m.body_jntnum[b];
      f3 pos;
      q4 quat;
      if (jntnum == 1 && m.jnt_type[jntadr] == JNT_FREE) {
        const int a = m.jnt_qposadr[jntadr];
        pos = ld3(qpos + a);
        quat = ld4(qpos + a + 3);
        st3(xanchor + 3 * jntadr, pos);
        st3(xaxis + 3 * jntadr, ld3(m.jnt_axis + 3 * jntadr));
      } else {
        const int p = m.body_parentid[b];
        pos = mulmv(ld9(xmat + 9 * p), ld3(m.body_pos + 3 * b)) + ld3(xpos + 3 * p);
        quat = mul_quat(ld4(xquat + 4 * p), ld4(m.body_quat + 4 * b));
        for (int j = jntadr; j < jntadr + jntnum; j++) {
          const int a = m.jnt_qposadr[j];
          const int t = m.jnt_type[j];
          const f3 jaxis = ld3(m.jnt_axis + 3 * j), jpos = ld3(m.jnt_pos + 3 * j);
          const f3 anchor = rot_vec_quat(jpos, quat) + pos;
          const f3 axis = rot_vec_quat(jaxis, quat);
          if (t == JNT_BALL) {
            quat = mul_quat(quat, ld4(qpos + a));
            pos = anchor - rot_vec_quat(jpos, quat);
          } else if (t == JNT_SLIDE) {
            pos = pos + axis * (qpos[a] - m.qpos0[a]);
          } else if (t == JNT_HINGE) {
            quat = mul_quat(quat, axis_angle_to_quat(jaxis, qpos[a] - m.qpos0[a]));
            pos = anchor - rot_vec_quat(jpos, quat);
          }
          st3(xanchor + 3 * j, anchor);
          st3(xaxis + 3 * j, axis);
        }
      }
      st3(xpos + 3 * b, pos);
      quat = qnormalize(quat);
      st4(xquat + 4 * b, quat);
      st9(xmat + 9 * b, quat_to_mat(quat));
      st3(xipos + 3 * b, pos + rot_vec_quat(ld3(m.body_ipos + 3 * b), quat));
      st9(ximat + 9 * b, quat_to_mat(mul_quat(quat, ld4(m.body_iquat + 4 * b))));
    }
    lsync<L>();
  }
  // geom_local_to_global / site_local_to_global (smooth.py:111-131)
  float* gxpos = d.geom_xpos + W(w, 3 * m.ngeom);
  float* gxmat = d.geom_xmat + W(w, 9 * m.ngeom);
  for (int g = lane; g < m.ngeom; g += L) {
    const int b = m.geom_bodyid[g];
    const q4 q = ld4(xquat + 4 * b);
    st3(gxpos + 3 * g, ld3(xpos + 3 * b) + rot_vec_quat(ld3(m.geom_pos + 3 * g), q));
    st9(gxmat + 9 * g, quat_to_mat(mul_quat(q, ld4(m.geom_quat + 4 * g))));
  }
  if (d.site_xpos) {
    float* sxpos = d.site_xpos + W(w, 3 * m.nsite);
    float* sxmat = d.site_xmat + W(w, 9 * m.nsite);
    for (int s = lane; s < m.nsite; s += L) {
      const int b = m.site_bodyid[s];
      const q4 q = ld4(xquat + 4 * b);
      st3(sxpos + 3 * s, ld3(xpos + 3 * b) + rot_vec_quat(ld3(m.site_pos + 3 * s), q));
      st9(sxmat + 9 * s, quat_to_mat(mul_quat(q, ld4(m.site_quat + 4 * s))));
    }
  }
  lsync<L>();
}

// ------------------------------------------------------------------------------------------
// smooth.py:148-245 — subtree CoM, cinert, cdof
template <int L = 32>
__device__ void com_pos(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nb = m.nbody;
  const float* xipos = d.xipos + W(w, 3 * nb);
  const float* ximat = d.ximat + W(w, 9 * nb);
  const float* xmat = d.xmat + W(w, 9 * nb);
  const float* xanchor = d.xanchor + W(w, 3 * m.njnt);
  const float* xaxis = d.xaxis + W(w, 3 * m.njnt);
  float* sc = d.subtree_com + W(w, 3 * nb);
  for (int b = lane; b < nb; b += L) st3(sc + 3 * b, ld3(xipos + 3 * b) * m.body_mass[b]);
  lsync<L>();
  // bottom-up gather over children; the world also adds itself (smooth.py:238-241 runs the
  // accumulation on level 0, where body 0 is its own parent)
  for (int lvl = m.nlevel - 1; lvl >= 0; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += L) {
      const int b = m.body_tree[n];
      f3 acc = ld3(sc + 3 * b);
      const int ca = m.body_childadr[b], cn = m.body_childnum[b];
      for (int k = 0; k < cn; k++) acc = acc + ld3(sc + 3 * m.body_child[ca + k]);
      if (b == 0) acc = acc + acc;
      st3(sc + 3 * b, acc);
    }
    lsync<L>();
  }
  for (int b = lane; b < nb; b += L) {
    const float sm = m.subtree_mass[b];
    f3 v = ld3(sc + 3 * b);
    st3(sc + 3 * b, mk3(v.x / sm, v.y / sm, v.z / sm));
  }
  lsync<L>();
  // cinert (smooth.py:169-201)
  float* cinert = d.cinert + W(w, 10 * nb);
  for (int b = lane; b < nb; b += L) {
    const m33 mat = ld9(ximat + 9 * b);
    const f3 inert = ld3(m.body_inertia + 3 * b);
    const float mass = m.body_mass[b];
    const f3 dif = ld3(xipos + 3 * b) - ld3(sc + 3 * m.body_rootid[b]);
    float t[6];
    const int ij[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
#pragma unroll
    for (int e = 0; e < 6; e++) {
      const int i = ij[e][0], j = ij[e][1];
      t[e] = mat.m[3 * i] * inert.x * mat.m[3 * j] + mat.m[3 * i + 1] * inert.y * mat.m[3 * j + 1] +
             mat.m[3 * i + 2] * inert.z * mat.m[3 * j + 2];
    }
    float* r = cinert + 10 * b;
    r[0] = t[0] + mass * (dif.y * dif.y + dif.z * dif.z);
    r[1] = t[1] + mass * (dif.x * dif.x + dif.z * dif.z);
    r[2] = t[2] + mass * (dif.x * dif.x + dif.y * dif.y);
    r[3] = t[3] - mass * dif.x * dif.y;
    r[4] = t[4] - mass * dif.x * dif.z;
    r[5] = t[5] - mass * dif.y * dif.z;
    r[6] = mass * dif.x;
    r[7] = mass * dif.y;
    r[8] = mass * dif.z;
    r[9] = mass;
  }
  // cdof (smooth.py:203-232)
  float* cdof = d.cdof + W(w, 6 * m.nv);
  for (int j = lane; j < m.njnt; j += L) {
    const int b = m.jnt_bodyid[j], dof = m.jnt_dofadr[j], t = m.jnt_type[j];
    const f3 off = ld3(sc + 3 * m.body_rootid[b]) - ld3(xanchor + 3 * j);
    const m33 xm = ld9(xmat + 9 * b);
    auto put = [&](int i, f3 a, f3 l) {
      float* c = cdof + 6 * i;
      c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = l.x; c[4] = l.y; c[5] = l.z;
    };
    if (t == JNT_FREE) {
      put(dof + 0, mk3(0, 0, 0), mk3(1, 0, 0));
      put(dof + 1, mk3(0, 0, 0), mk3(0, 1, 0));
      put(dof + 2, mk3(0, 0, 0), mk3(0, 0, 1));
      for (int k = 0; k < 3; k++) put(dof + 3 + k, col(xm, k), cross(col(xm, k), off));
    } else if (t == JNT_BALL) {
      for (int k = 0; k < 3; k++) put(dof + k, col(xm, k), cross(col(xm, k), off));
    } else if (t == JNT_SLIDE) {
      put(dof, mk3(0, 0, 0), ld3(xaxis + 3 * j));
    } else {
      const f3 ax = ld3(xaxis + 3 * j);
      put(dof, ax, cross(ax, off));
    }
  }
  lsync<L>();
}

// ------------------------------------------------------------------------------------------
// Sparse mass matrix (the reference's layout when opt.is_sparse; MuJoCo's qM / qLD): row i holds
// M(i,i), M(i,parent(i)), M(i,parent(parent(i))), ... at dof_Madr[i], dof_Madr[i] + 1, ... (the
// dof's ancestor chain, smooth.py:264-279); qLD holds the L'DL factor in the same slots (D on the
// diagonal slot, the unit factor's entries below it) and qLDiagInv = 1 / D.  Every kinematic
// tree's dofs are contiguous (block_adr / block_size) and couple only within the tree, so one
// lane owns one tree and runs the serial algorithms on it; results do not depend on the lane
// count.

__device__ __forceinline__ int madr_row_len(const MjbModel& m, int i) {
  return (i + 1 < m.nv ? m.dof_Madr[i + 1] : m.nM) - m.dof_Madr[i];
}

// smooth.py:317-351 (mj_factorI): in-place L'DL, each tree's dofs eliminated from its last to its
// first, each elimination updating its ancestors' rows; Dinv (may be null) = 1 / D
__device__ void factor_sparse(const MjbModel& m, float* L, float* Dinv, int lane) {
  for (int blk = lane; blk < m.nblock; blk += 32) {
    const int a = m.block_adr[blk], n = m.block_size[blk];
    for (int k = a + n - 1; k >= a; k--) {
      const int Mkk = m.dof_Madr[k];
      int Mki = Mkk + 1;
      for (int i = m.dof_parentid[k]; i >= 0; i = m.dof_parentid[i], Mki++) {
        const float tmp = L[Mki] / L[Mkk];
        const int Mi = m.dof_Madr[i], cnt = madr_row_len(m, i);
        for (int j = 0; j < cnt; j++) L[Mi + j] -= L[Mki + j] * tmp;
        L[Mki] = tmp;
      }
    }
    if (Dinv)
      for (int k = a; k < a + n; k++) Dinv[k] = 1.f / L[m.dof_Madr[k]];
  }
  __syncwarp();
}

// x = M^-1 y from the L'DL factor (smooth.py:609-652, mj_solveLD): x <- L'^-1 x from the leaves
// up, x <- D^-1 x, x <- L^-1 x from the roots down.  Dinv may be null (1 / D is then formed from
// L).  x may alias y.
__device__ void solve_sparse(const MjbModel& m, const float* L, const float* Dinv, float* x,
                             const float* y, int lane) {
  for (int blk = lane; blk < m.nblock; blk += 32) {
    const int a = m.block_adr[blk], n = m.block_size[blk];
    for (int k = a; k < a + n; k++) x[k] = y[k];
    for (int k = a + n - 1; k >= a; k--) {
      int Mki = m.dof_Madr[k] + 1;
      for (int i = m.dof_parentid[k]; i >= 0; i = m.dof_parentid[i], Mki++) x[i] -= L[Mki] * x[k];
    }
    for (int k = a; k < a + n; k++) x[k] *= Dinv ? Dinv[k] : 1.f / L[m.dof_Madr[k]];
    for (int k = a; k < a + n; k++) {
      int Mki = m.dof_Madr[k] + 1;
      for (int i = m.dof_parentid[k]; i >= 0; i = m.dof_parentid[i], Mki++) x[k] -= L[Mki] * x[i];
    }
  }
  __syncwarp();
}

// res = M vec for the sparse M (support.py:96-137: the diagonal, then each stored off-diagonal
// entry applied to both of its rows); res must not alias vec
__device__ void mul_m_sparse(const MjbModel& m, const float* M, float* res, const float* vec,
                             int lane) {
  for (int blk = lane; blk < m.nblock; blk += 32) {
    const int a = m.block_adr[blk], n = m.block_size[blk];
    for (int i = a; i < a + n; i++) res[i] = M[m.dof_Madr[i]] * vec[i];
    for (int i = a; i < a + n; i++) {
      int Mij = m.dof_Madr[i] + 1;
      for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j], Mij++) {
        res[i] += M[Mij] * vec[j];
        res[j] += M[Mij] * vec[i];
      }
    }
  }
  __syncwarp();
}

// Scatters the sparse M into the lower triangle of a dense nv x nv matrix H (upper left alone)
__device__ void sparse_to_lower(const MjbModel& m, const float* M, float* H, int lane) {
  const int nv = m.nv;
  for (int e = lane; e < nv * nv; e += 32) {
    const int i = e / nv, j = e - i * nv;
    if (j <= i) H[e] = 0.f;
  }
  __syncwarp();
  for (int i = lane; i < nv; i += 32) {
    int a = m.dof_Madr[i];
    H[i * nv + i] = M[a];
    for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j]) H[i * nv + j] = M[++a];
  }
  __syncwarp();
}

// ------------------------------------------------------------------------------------------
// smooth.py:248-314 — composite rigid body inertia and dense qM
template <int L = 32>
__device__ void crb(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nb = m.nbody, nv = m.nv;
  const float* cinert = d.cinert + W(w, 10 * nb);
  float* crb = d.crb + W(w, 10 * nb);
  // bottom-up gather; children of the world do not add into it (smooth.py:259-260)
  for (int lvl = m.nlevel - 1; lvl >= 0; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += L) {
      const int b = m.body_tree[n];
      float acc[10];
#pragma unroll
      for (int k = 0; k < 10; k++) acc[k] = cinert[10 * b + k];
      if (b != 0) {
        const int ca = m.body_childadr[b], cn = m.body_childnum[b];
        for (int c = 0; c < cn; c++) {
          const float* src = crb + 10 * m.body_child[ca + c];
#pragma unroll
          for (int k = 0; k < 10; k++) acc[k] += src[k];
        }
      }
#pragma unroll
      for (int k = 0; k < 10; k++) crb[10 * b + k] = acc[k];
    }
    lsync<L>();
  }
  const float* cdof = d.cdof + W(w, 6 * nv);
  if (m.is_sparse) {  // qM_sparse (smooth.py:263-279)
    float* qMs = d.qM + W(w, m.nM);
    for (int i = lane; i < nv; i += L) {
      const s6 ci = ld6(cdof + 6 * i);
      const s6 buf = inert_vec(crb + 10 * m.dof_bodyid[i], ci);
      int a = m.dof_Madr[i];
      qMs[a] = m.dof_armature[i] + dot6(ci, buf);
      for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j]) qMs[++a] = dot6(ld6(cdof + 6 * j), buf);
    }
    lsync<L>();
    return;
  }
  // qM_dense (smooth.py:281-302)
  float* qM = d.qM + W(w, nv * nv);
  for (int e = lane; e < nv * nv; e += L) qM[e] = 0.f;
  lsync<L>();
  for (int i = lane; i < nv; i += L) {
    const s6 ci = ld6(cdof + 6 * i);
    const s6 buf = inert_vec(crb + 10 * m.dof_bodyid[i], ci);
    qM[i * nv + i] = m.dof_armature[i] + dot6(ci, buf);
    for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j]) {
      const float v = dot6(ld6(cdof + 6 * j), buf);
      qM[i * nv + j] = v;
      qM[j * nv + i] = v;
    }
  }
  lsync<L>();
}

// In-place Cholesky A = L L^T (left-looking, column by column) of the n x n SPD matrix at A with
// leading dimension ld (shared or global memory); only the lower triangle is read and written.
// Column k: lane j takes row k + j (+ 32 t) and forms the dot product of that row with row k over
// the finished columns (four independent partial sums); lane 0's row is row k itself, so its
// result is the pivot, which is broadcast by shuffle before every lane scales its entry.
// Compiled once (no inlining) so every caller shares one copy of the code.
// correctly rounded reciprocal (the value of 1 / x)
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }

template <typename T>
__device__ __forceinline__ T chol_dot(const T* a, const T* b, int k) {
  T s0 = T(0), s1 = T(0), s2 = T(0), s3 = T(0);
  int m = 0;
  for (; m + 3 < k; m += 4) {
    s0 += a[m] * b[m];
    s1 += a[m + 1] * b[m + 1];
    s2 += a[m + 2] * b[m + 2];
    s3 += a[m + 3] * b[m + 3];
  }
  for (; m < k; m++) s0 += a[m] * b[m];
  return (s0 + s1) + (s2 + s3);
}

template <typename T>
__device__ __noinline__ void chol_lower(T* A, int ld, int n, int lane) {
  for (int k = 0; k < n; k++) {
    const T* Ak = A + k * ld;
    if (n - k <= 32) {  // one row per lane: the pivot and the column in a single pass
      const int i = k + lane;
      T s = T(0);
      if (i < n) s = A[i * ld + k] - chol_dot(A + i * ld, Ak, k);
      const T lkk = sqrt(__shfl_sync(0xffffffffu, s, 0));
      const T inv = rcp_rn(lkk);
      __syncwarp();
      if (lane == 0) A[k * ld + k] = lkk;
      else if (i < n) A[i * ld + k] = s * inv;
    } else {
      T s = T(0);
      if (lane == 0) s = Ak[k] - chol_dot(Ak, Ak, k);
      const T lkk = sqrt(__shfl_sync(0xffffffffu, s, 0));
      const T inv = rcp_rn(lkk);
      for (int i = k + 1 + lane; i < n; i += 32) {
        T* Ai = A + i * ld;
        Ai[k] = (Ai[k] - chol_dot(Ai, Ak, k)) * inv;
      }
      __syncwarp();
      if (lane == 0) A[k * ld + k] = lkk;
    }
    __syncwarp();
  }
}

// Cholesky of an n x n (n <= 32) SPD matrix, in place, with the forward substitution of one
// right-hand side folded in.  The lower triangle is read from L (leading dimension ldl, shared or
// global memory); lane i keeps row i in registers.  Right-looking: at column k every lane takes
// the updated diagonal from lane k by shuffle, scales its entry L[i][k], publishes it to a 32-float
// per-warp buffer and subtracts L[i][k] * L[j][k] from the rest of its row — independent FMAs fed
// by broadcast reads.  On exit L holds the factor; the return value is (1 / L[i][i], z_i) with
// z = L^-1 y for the lane's y_i (0 for lanes >= n).  Blocks of up to 4 warps (one buffer each).
__device__ __noinline__ float2 chol32(float* L, int ldl, int n, int lane, float y) {
  __shared__ float colbuf[4][32];
  float* col = colbuf[(threadIdx.x >> 5) & 3];
  float r[32];
#pragma unroll
  for (int j = 0; j < 32; j++) r[j] = (lane < n && j <= lane) ? L[lane * ldl + j] : 0.f;
  float z = lane < n ? y : 0.f, invd = 0.f;
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 32; k++) {
    if (k >= n) break;
    const float lkk = sqrtf(__shfl_sync(0xffffffffu, r[k], k));
    const float inv = 1.f / lkk;
    const float zk = __shfl_sync(0xffffffffu, z, k) * inv;
    if (lane == k) {
      r[k] = lkk;
      invd = inv;
      z = zk;
    } else if (lane > k) {
      r[k] *= inv;
      z -= r[k] * zk;
    }
    col[lane] = r[k];
    __syncwarp();
    if (lane > k && lane < n) {
      const float lik = r[k];
#pragma unroll
      for (int j = k + 1; j < 32; j++)
        if (j <= lane) r[j] -= lik * col[j];
    }
    __syncwarp();
  }
  if (lane < n) {
#pragma unroll
    for (int j = 0; j < 32; j++)
      if (j <= lane) L[lane * ldl + j] = r[j];
  }
  __syncwarp();
  return make_float2(invd, z);
}

// Back substitution x = L^-T z for a chol32 factor; lane i holds z_i and 1 / L_ii, returns x_i.
__device__ __forceinline__ float cho_back32(const float* L, int ldl, int n, float invd, float z,
                                            int lane) {
  float x = lane < n ? z : 0.f;
  for (int k = n - 1; k >= 0; k--) {
    const float lk = lane < k ? L[k * ldl + lane] : 0.f;
    const float xk = __shfl_sync(0xffffffffu, x, k) * __shfl_sync(0xffffffffu, invd, k);
    if (lane == k) x = xk;
    else if (lane < k) x -= lk * xk;
  }
  return x;
}

// x = (L L^T)^-1 y for a chol32 factor (n <= 32) with lane i holding y_i and invd_i = 1/L_ii;
// returns x_i.  No divisions: the reciprocal diagonal is broadcast by shuffle.
__device__ __forceinline__ float cho_solve32(const float* L, int ldl, int n, float invd, float y,
                                             int lane) {
  float z = lane < n ? y : 0.f;
  for (int k = 0; k < n; k++) {
    const float lk = (lane > k && lane < n) ? L[lane * ldl + k] : 0.f;
    const float zk = __shfl_sync(0xffffffffu, z, k) * __shfl_sync(0xffffffffu, invd, k);
    if (lane == k) z = zk;
    else if (lane > k && lane < n) z -= lk * zk;
  }
  return cho_back32(L, ldl, n, invd, z, lane);
}


// Per-warp factor tiles for blocks of n <= 32 in shared memory.  Rows are tile_ld(nv) floats:
// the padded width 4 * ceil(n / 4) rounded so that ld / 4 is odd, which keeps rows 16-byte
// aligned and lets the 8 lanes of a quarter warp read their own rows as float4 from 8 distinct
// groups of 4 banks (no conflict); entries above the diagonal are never read.
__host__ __device__ __forceinline__ int tile_ld(int nv) {
  const int r = ((nv < 32 ? nv : 32) + 3) & ~3;
  return (r & 4) ? r : r + 4;
}
__host__ __device__ __forceinline__ int tile_floats(int nv) {
  return (nv < 32 ? nv : 32) * tile_ld(nv);
}

// Copies an nrows x ncols block (ncols <= 32; lane = column) from src (row stride sld) to dst (row
// stride dld), writing lanes [ncols, pad) as zero.  Eight rows are loaded before they are stored,
// so the loads overlap: row-by-row copies wait out each load, because dst (shared memory reached
// through a generic pointer) may alias src as far as the compiler can tell.
__device__ __forceinline__ void copy_rows(const float* src, int sld, float* dst, int dld, int nrows,
                                          int ncols, int pad, int lane) {
  for (int r0 = 0; r0 < nrows; r0 += 8) {
    float v[8];
#pragma unroll
    for (int t = 0; t < 8; t++)
      v[t] = (r0 + t < nrows && lane < ncols) ? src[size_t(r0 + t) * sld + lane] : 0.f;
#pragma unroll
    for (int t = 0; t < 8; t++)
      if (r0 + t < nrows && lane < pad) dst[size_t(r0 + t) * dld + lane] = v[t];
  }
}

// In-place Cholesky of an n x n (n <= 32) SPD tile with row stride ld (lower triangle): the
// partial sums of chol_lower with float4 row reads; the pivot and its reciprocal come from one
// rsqrtf (within 2 ulp of the correctly rounded sqrt and reciprocal).  Lane i works on row i,
// four columns per step: one pass over the row's finished columns (whole float4 chunks, k being a
// multiple of 4) feeds the four columns' partial sums, its row loads shared; then column k + j
// adds the terms L[i][k + t] L[k + j][k + t], t < j, with L[k + j][k + t] shuffled from lane k + j,
// and one __syncwarp() publishes the four columns.  Every sum is formed in the order of the
// one-column form (the same float4 chunks, then the remaining terms in column order into the first
// partial sum), so the factor is the same bit for bit.
__device__ MJB_TILE_FN void chol_tile(float* A, int ld, int n, int lane) {
  float* Ar = A + min(lane, n - 1) * ld;  // lanes past the last row repeat it
  for (int k = 0; k < n; k += 4) {
    const int nb = min(4, n - k);  // columns of this step
    const float* Ak[4];
#pragma unroll
    for (int j = 0; j < 4; j++) Ak[j] = A + (k + (j < nb ? j : 0)) * ld;
    float s[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++) s[j][0] = s[j][1] = s[j][2] = s[j][3] = 0.f;
    for (int m = 0; m < k; m += 4) {
      const float4 a = *reinterpret_cast<const float4*>(Ar + m);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float4 b = *reinterpret_cast<const float4*>(Ak[j] + m);
        s[j][0] += a.x * b.x;
        s[j][1] += a.y * b.y;
        s[j][2] += a.z * b.z;
        s[j][3] += a.w * b.w;
      }
    }
    float l[4] = {0.f, 0.f, 0.f, 0.f};  // L[i][k + j]; on lane k + j the pivot
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (j < nb) {
#pragma unroll
        for (int t = 0; t < j; t++) s[j][0] += l[t] * __shfl_sync(WARP_FULL, l[t], k + j);
        const float x = Ar[k + j] - ((s[j][0] + s[j][1]) + (s[j][2] + s[j][3]));
        l[j] = x * rsqrtf(__shfl_sync(WARP_FULL, x, k + j));
        if (lane >= k + j && lane < n) Ar[k + j] = l[j];
      }
    }
    __syncwarp();
  }
}

// x = (L L^T)^-1 y for an n <= 32 tile factor; lane i holds y_i and returns x_i (the arithmetic of
// cho_solve32).  The forward pass reads the lane's own row four columns at a time, the backward
// pass row k across the lanes; neither load depends on the substitution chain.
__device__ MJB_TILE_FN float cho_solve_tile(const float* L, int ld, int n, float y, int lane) {
  const bool own = lane < n;
  const float* Li = L + min(lane, n - 1) * ld;
  const float invd = own ? __frcp_rn(Li[lane]) : 0.f;
  float z = own ? y : 0.f;
  for (int q = 0; 4 * q < n; q++) {  // the lane's row, four columns per float4 read
    const float4 l4 = *reinterpret_cast<const float4*>(Li + 4 * q);
    const float lq[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int k = 4 * q + t;
      if (k < n) {  // lane k scales its entry, one shuffle broadcasts it
        if (lane == k) z *= invd;
        const float zk = __shfl_sync(WARP_FULL, z, k);
        if (lane > k && own) z -= lq[t] * zk;
      }
    }
  }
  float x = z;
#pragma unroll 4
  for (int k = n - 1; k >= 0; k--) {
    const float lk = L[k * ld + (lane < k ? lane : 0)];
    if (lane == k) x *= invd;
    const float xk = __shfl_sync(WARP_FULL, x, k);
    if (lane < k) x -= lk * xk;
  }
  return own ? x : 0.f;
}

// FP64 counterparts of chol_tile / cho_solve_tile for the precision form (MJB_FORM_PRECISION):
// the same lane-per-row scheme on a tile of doubles (row stride ld doubles), the pivot and its
// reciprocal from one double rsqrt (L_kk = s_k rsqrt(s_k), L_ik = s_i rsqrt(s_k)) as in chol_tile.
// chol_tile_d takes four columns per step as chol_tile does: one pass over the row's finished
// columns (pairs of partial sums, k a multiple of 4) feeds the four columns, then column k + j
// adds the terms of columns k .. k + j - 1 as the one-column form orders them (the pair
// (k, k + 1) into the two partial sums, column k + 2 as the tail term).
__device__ __noinline__ void chol_tile_d(double* A, int ld, int n, int lane) {
  double* Ar = A + min(lane, n - 1) * ld;  // lane i on row i; lanes past the last row repeat it
  for (int k = 0; k < n; k += 4) {
    const int nb = min(4, n - k);
    const double* Ak[4];
#pragma unroll
    for (int j = 0; j < 4; j++) Ak[j] = A + (k + (j < nb ? j : 0)) * ld;
    double s[4][2];
#pragma unroll
    for (int j = 0; j < 4; j++) s[j][0] = s[j][1] = 0.0;
    for (int m = 0; m < k; m += 2) {
      const double a0 = Ar[m], a1 = Ar[m + 1];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        s[j][0] += a0 * Ak[j][m];
        s[j][1] += a1 * Ak[j][m + 1];
      }
    }
    double l[4] = {0.0, 0.0, 0.0, 0.0};  // L[i][k + j]; on lane k + j the pivot
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (j < nb) {
        if (j >= 1) s[j][0] += l[0] * __shfl_sync(WARP_FULL, l[0], k + j);
        if (j >= 2) s[j][1] += l[1] * __shfl_sync(WARP_FULL, l[1], k + j);
        if (j >= 3) s[j][0] += l[2] * __shfl_sync(WARP_FULL, l[2], k + j);
        const double x = Ar[k + j] - (s[j][0] + s[j][1]);
        l[j] = x * rsqrt(__shfl_sync(WARP_FULL, x, k + j));
        if (lane >= k + j && lane < n) Ar[k + j] = l[j];
      }
    }
    __syncwarp();
  }
}
// The substitutions multiply by each lane's reciprocal pivot, formed once (one FP64 division per
// lane instead of one per step of each pass); lane k scales its entry, one shuffle broadcasts it.
__device__ __noinline__ double cho_solve_tile_d(const double* L, int ld, int n, double y, int lane) {
  const bool own = lane < n;
  const double* Li = L + min(lane, n - 1) * ld;
  const double invd = own ? 1.0 / Li[lane] : 0.0;
  double z = own ? y : 0.0;
  for (int k = 0; k < n; k++) {
    if (lane == k) z *= invd;
    const double zk = __shfl_sync(WARP_FULL, z, k);
    if (lane > k && own) z -= Li[k] * zk;
  }
  double x = z;
  for (int k = n - 1; k >= 0; k--) {
    const double lk = L[k * ld + (lane < k ? lane : 0)];
    if (lane == k) x *= invd;
    const double xk = __shfl_sync(WARP_FULL, x, k);
    if (lane < k) x -= lk * xk;
  }
  return own ? x : 0.0;
}
// Floats of per-warp scratch the precision form adds for its double tile.
__host__ __device__ __forceinline__ int prec_tile_floats(int nv) { return 2 * tile_floats(nv); }

// Copies the lower triangle of an n <= 32 tile to L (leading dimension ld) with zeros above the
// diagonal, one coalesced row at a time.
__device__ __forceinline__ void tile_store_lower(const float* T, int tld, int n, float* L, int ld, int lane) {
  for (int r0 = 0; r0 < n; r0 += 8) {  // eight rows read before they are written (see copy_rows)
    float v[8];
#pragma unroll
    for (int t = 0; t < 8; t++) v[t] = (r0 + t < n && lane <= r0 + t) ? T[(r0 + t) * tld + lane] : 0.f;
#pragma unroll
    for (int t = 0; t < 8; t++)
      if (r0 + t < n && lane < n) L[(r0 + t) * ld + lane] = v[t];
  }
}

// Right-looking blocked Cholesky of the n x n SPD lower triangle of A (row stride ld, shared or
// global memory) in panels of 32 columns, with a warp scratch tile T of 32 x 36 floats (16-byte
// aligned).  Per panel: (a) the diagonal block is staged in T, factored by chol_tile and written
// back; (b) every row below it solves L_i = A_i L_pp^-T against the factored block (lane per row,
// the row's 32 panel entries in registers, the block and its reciprocal diagonal read from T by
// broadcast); (c) the trailing lower triangle is updated, A_ij -= L_i . L_j over the panel, one
// chunk of 32 rows j at a time staged in T, lane per row i, float4 broadcast reads.  The column
// dot products are accumulated panel by panel, so the bits differ from chol_lower's.
__device__ __noinline__ void chol_blocked(float* A, int ld, int n, int lane, float* T) {
  constexpr int TL = 36;
  for (int p0 = 0; p0 < n; p0 += 32) {
    const int pn = min(32, n - p0);
    // (a)
    for (int r = 0; r < pn; r++)
      if (lane < pn) T[r * TL + lane] = lane <= r ? A[size_t(p0 + r) * ld + p0 + lane] : 0.f;
    __syncwarp();
    chol_tile(T, TL, pn, lane);
    for (int r = 0; r < pn; r++)
      if (lane <= r) A[size_t(p0 + r) * ld + p0 + lane] = T[r * TL + lane];
    if (lane < pn) T[lane * TL + 32] = __frcp_rn(T[lane * TL + lane]);
    __syncwarp();
    // (b)
    for (int i = p0 + pn + lane; i < n; i += 32) {
      float* Ai = A + size_t(i) * ld + p0;
      float x[32];
#pragma unroll
      for (int c = 0; c < 32; c++) x[c] = c < pn ? Ai[c] : 0.f;
#pragma unroll
      for (int c = 0; c < 32; c++) {
        if (c < pn) {
          float v = x[c];
#pragma unroll
          for (int q = 0; q < c; q++) v -= x[q] * T[c * TL + q];
          x[c] = v * T[c * TL + 32];
        }
      }
#pragma unroll
      for (int c = 0; c < 32; c++)
        if (c < pn) Ai[c] = x[c];
    }
    __syncwarp();
    // (c)
    for (int j0 = p0 + pn; j0 < n; j0 += 32) {
      const int jn = min(32, n - j0);
      for (int jj = 0; jj < jn; jj++)
        T[jj * TL + lane] = lane < pn ? A[size_t(j0 + jj) * ld + p0 + lane] : 0.f;
      __syncwarp();
      for (int i = j0 + lane; i < n; i += 32) {
        const float* Li = A + size_t(i) * ld + p0;
        float x[32];
#pragma unroll
        for (int c = 0; c < 32; c++) x[c] = c < pn ? Li[c] : 0.f;
        float* Ai = A + size_t(i) * ld + j0;
        const int jm = min(jn, i - j0 + 1);
        for (int jj = 0; jj < jm; jj++) {
          const float4* P4 = reinterpret_cast<const float4*>(T + jj * TL);
          float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const float4 pv = P4[q];
            s0 += x[4 * q] * pv.x;
            s1 += x[4 * q + 1] * pv.y;
            s2 += x[4 * q + 2] * pv.z;
            s3 += x[4 * q + 3] * pv.w;
          }
          Ai[jj] -= (s0 + s1) + (s2 + s3);
        }
      }
      __syncwarp();
    }
  }
}

// Cholesky of an n x n SPD block: blocked (chol_blocked) when n > 32 and a 32 x 36 warp scratch
// tile is given, else chol_lower.
__device__ __forceinline__ void chol_any(float* A, int ld, int n, int lane, float* tile) {
  if (n > 32 && tile) chol_blocked(A, ld, n, lane, tile);
  else chol_lower(A, ld, n, lane);
}

// x = (L L^T)^-1 y for the n x n lower factor at L (leading dimension ld); x may alias y.
__device__ void warp_cho_solve(const float* L, int ld, int n, float* x, const float* y, int lane) {
  if (n <= 32) {
    float xi = lane < n ? y[lane] : 0.f;
    for (int k = 0; k < n; k++) {  // L z = y
      float xk = __shfl_sync(WARP_FULL, xi, k) / L[k * ld + k];
      if (lane == k) xi = xk;
      else if (lane > k && lane < n) xi -= L[lane * ld + k] * xk;
    }
    for (int k = n - 1; k >= 0; k--) {  // L^T x = z
      float xk = __shfl_sync(WARP_FULL, xi, k) / L[k * ld + k];
      if (lane == k) xi = xk;
      else if (lane < k) xi -= L[k * ld + lane] * xk;
    }
    __syncwarp();
    if (lane < n) x[lane] = xi;
    __syncwarp();
    return;
  }
  for (int i = lane; i < n; i += 32) x[i] = y[i];
  __syncwarp();
  for (int k = 0; k < n; k++) {
    const float xk = x[k] / L[k * ld + k];
    __syncwarp();
    if (lane == (k & 31)) x[k] = xk;
    for (int i = k + 1 + lane; i < n; i += 32) x[i] -= L[i * ld + k] * xk;
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; k--) {
    const float xk = x[k] / L[k * ld + k];
    __syncwarp();
    if (lane == (k & 31)) x[k] = xk;
    for (int i = lane; i < k; i += 32) x[i] -= L[k * ld + i] * xk;
    __syncwarp();
  }
}

// Factor every tree block of the nv x nv matrix M (+ scale * diag(dadd) when dadd is given) into
// L: dense storage, zero outside the lower block triangles.  smooth.py:353-379 (tile_cholesky per
// qLD_tile group) and the fused damping tiles of forward.py:195-232.
// Dense Cholesky of each tree block of the inertia-like matrix M (+ scale * dadd on the diagonal)
// into L (smooth.py:353-379, qLD_tile semantics; zeros outside the blocks' lower triangles).  With
// a per-warp tile, blocks of n <= 32 are factored in shared memory and written back row by row;
// the tile then holds the factor of the last block.
__device__ void factor_blocks(const MjbModel& m, const float* M, float* L, int lane,
                              const float* dadd = nullptr, float scale = 0.f, float* tile = nullptr) {
  const int nv = m.nv;
  // one tiled block covering every dof is written whole by tile_store_lower
  if (!(tile && m.nblock == 1 && nv <= 32)) {
    for (int e = lane; e < nv * nv; e += 32) L[e] = 0.f;
    __syncwarp();
  }
  for (int blk = 0; blk < m.nblock; blk++) {
    const int a = m.block_adr[blk], n = m.block_size[blk];
    if (tile && n <= 32) {
      const int tld = tile_ld(nv);
      copy_rows(M + a * nv + a, nv, tile, tld, n, n, n, lane);  // coalesced row reads of the block
      __syncwarp();
      if (dadd && lane < n) {
        float v = tile[lane * tld + lane];
        v += scale * dadd[a + lane];
        tile[lane * tld + lane] = v;
      }
      __syncwarp();
      chol_tile(tile, tld, n, lane);
      tile_store_lower(tile, tld, n, L + a * nv + a, nv, lane);
      __syncwarp();
      continue;
    }
    for (int i = lane; i < n; i += 32) {  // row i of the block's lower triangle (+ damping on the diagonal)
      const float* src = M + (a + i) * nv + a;
      float* dst = L + (a + i) * nv + a;
      for (int j = 0; j < i; j++) dst[j] = src[j];
      dst[i] = src[i] + (dadd ? scale * dadd[a + i] : 0.f);
    }
    __syncwarp();
#if MJB_CHOL == 1
    if (n <= 32) chol32(L + a * nv + a, nv, n, lane, 0.f);
    else chol_any(L + a * nv + a, nv, n, lane, tile);
#else
    chol_any(L + a * nv + a, nv, n, lane, tile);
#endif
  }
}

// x = M^-1 y per tree block from the block factor L (smooth.py:654-681); x may alias y.  With a
// tile, blocks of n <= 32 are staged into it row by row first, unless tile_has_factor says that
// the tile already holds the factor of the model's only block.
__device__ void solve_blocks(const MjbModel& m, const float* L, float* x, const float* y,
                             int lane, float* tile = nullptr, bool tile_has_factor = false) {
  const int nv = m.nv;
  for (int blk = 0; blk < m.nblock; blk++) {
    const int a = m.block_adr[blk], n = m.block_size[blk];
    if (n <= 32) {
      const float yi = lane < n ? y[a + lane] : 0.f;
      float xi;
      if (tile) {
        const int tld = tile_ld(nv);
        if (!(tile_has_factor && m.nblock == 1)) {
          copy_rows(L + a * nv + a, nv, tile, tld, n, n, n, lane);
          __syncwarp();
        }
        xi = cho_solve_tile(tile, tld, n, yi, lane);
      } else {
        const float* Lb = L + a * nv + a;
        const float invd = lane < n ? 1.f / Lb[lane * nv + lane] : 0.f;
        xi = cho_solve32(Lb, nv, n, invd, yi, lane);
      }
      __syncwarp();
      if (lane < n) x[a + lane] = xi;
      __syncwarp();
    } else {
      warp_cho_solve(L + a * nv + a, nv, n, x + a, y + a, lane);
    }
  }
}

// x = (M + scale diag(dadd))^-1 y per tree block, factored and solved in FP64 in the double tile
// dt (precision form; blocks of n <= 32, dense M with leading dimension nv).
__device__ void factor_solve_blocks_d(const MjbModel& m, const float* M, const float* dadd,
                                      float scale, float* x, const float* y, int lane, double* dt) {
  const int nv = m.nv, ld = tile_ld(nv);
  for (int blk = 0; blk < m.nblock; blk++) {
    const int a = m.block_adr[blk], n = m.block_size[blk];
    for (int r = 0; r < n; r++)
      if (lane < n) {
        double v = M[(a + r) * nv + a + lane];
        if (dadd && lane == r) v += double(scale) * double(dadd[a + r]);
        dt[r * ld + lane] = v;
      }
    __syncwarp();
    chol_tile_d(dt, ld, n, lane);
    const double xi = cho_solve_tile_d(dt, ld, n, lane < n ? double(y[a + lane]) : 0.0, lane);
    __syncwarp();
    if (lane < n) x[a + lane] = float(xi);
    __syncwarp();
  }
}

// smooth.py:392-395
__device__ void factor_m(const MjbModel& m, const MjbData& d, int w, int lane, float* tile = nullptr) {
  const int nv = m.nv;
  if (m.is_sparse) {  // smooth.py:317-351
    const float* M = d.qM + W(w, m.nM);
    float* L = d.qLD + W(w, m.nM);
    for (int e = lane; e < m.nM; e += 32) L[e] = M[e];
    __syncwarp();
    factor_sparse(m, L, d.qLDiagInv + W(w, nv), lane);
    return;
  }
  factor_blocks(m, d.qM + W(w, nv * nv), d.qLD + W(w, nv * nv), lane, nullptr, 0.f, tile);
}

// x = M^-1 y with the world's mass-matrix factor (qLD), dense or sparse
__device__ __forceinline__ void solve_m_world(const MjbModel& m, const MjbData& d, int w, float* x,
                                              const float* y, int lane, float* tile = nullptr,
                                              bool tile_has_factor = false) {
  if (m.is_sparse) solve_sparse(m, d.qLD + W(w, m.nM), d.qLDiagInv + W(w, m.nv), x, y, lane);
  else solve_blocks(m, d.qLD + W(w, m.nv * m.nv), x, y, lane, tile, tile_has_factor);
}

// ------------------------------------------------------------------------------------------
// smooth.py:469-536 — transmission (JOINT, JOINTINPARENT)
template <int L = 32>
__device__ void transmission(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nv = m.nv;
  const float* qpos = d.qpos + W(w, m.nq);
  float* length = d.actuator_length + W(w, m.nu);
  float* moment = d.actuator_moment + W(w, m.nu * nv);
  for (int e = lane; e < m.nu * nv; e += L) moment[e] = 0.f;  // coalesced; then the nonzeros
  lsync<L>();
  for (int a = lane; a < m.nu; a += L) {
    const int j = m.actuator_trnid[2 * a], t = m.jnt_type[j];
    const int qa = m.jnt_qposadr[j], va = m.jnt_dofadr[j], trn = m.actuator_trntype[a];
    const float* gear = m.actuator_gear + 6 * a;
    float* mom = moment + a * nv;
    if (trn != 0 && trn != 1) continue;
    if (t == JNT_FREE) {
      length[a] = 0.f;
      if (trn == 1) {
        const q4 qn{qpos[qa + 3], -qpos[qa + 4], -qpos[qa + 5], -qpos[qa + 6]};
        const f3 ga = rot_vec_quat(mk3(gear[3], gear[4], gear[5]), qn);
        mom[va] = gear[0]; mom[va + 1] = gear[1]; mom[va + 2] = gear[2];
        mom[va + 3] = ga.x; mom[va + 4] = ga.y; mom[va + 5] = ga.z;
      } else {
        for (int i = 0; i < 6; i++) mom[va + i] = gear[i];
      }
    } else if (t == JNT_BALL) {
      const q4 q = ld4(qpos + qa);
      const f3 aa = quat_to_vel(q);
      f3 ga = mk3(gear[0], gear[1], gear[2]);
      if (trn == 1) ga = rot_vec_quat(ga, q4{q.w, -q.x, -q.y, -q.z});
      length[a] = dot(aa, ga);
      mom[va] = ga.x; mom[va + 1] = ga.y; mom[va + 2] = ga.z;
    } else {
      length[a] = qpos[qa] * gear[0];
      mom[va] = gear[0];
    }
  }
  lsync<L>();
}

// ------------------------------------------------------------------------------------------
// smooth.py:539-606 — cvel, cdof_dot
template <int L = 32>
__device__ void com_vel(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nb = m.nbody, nv = m.nv;
  float* cvel = d.cvel + W(w, 6 * nb);
  float* cdd = d.cdof_dot + W(w, 6 * nv);
  const float* cdof = d.cdof + W(w, 6 * nv);
  const float* qvel = d.qvel + W(w, nv);
  if (lane < 6) cvel[lane] = 0.f;
  lsync<L>();
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += L) {
      const int b = m.body_tree[n];
      s6 v = ld6(cvel + 6 * m.body_parentid[b]);
      int dof = m.body_dofadr[b];
      for (int j = m.body_jntadr[b]; j < m.body_jntadr[b] + m.body_jntnum[b]; j++) {
        const int t = m.jnt_type[j];
        const int nd = t == JNT_FREE ? 6 : (t == JNT_BALL ? 3 : 1);
        if (t == JNT_FREE) {
          for (int i = 0; i < 3; i++) {
            const s6 c = ld6(cdof + 6 * (dof + i));
            for (int k = 0; k < 6; k++) v.v[k] += c.v[k] * qvel[dof + i];
            st6(cdd + 6 * (dof + i), s6{{0, 0, 0, 0, 0, 0}});
          }
          for (int i = 3; i < 6; i++) st6(cdd + 6 * (dof + i), motion_cross(v, ld6(cdof + 6 * (dof + i))));
          for (int i = 3; i < 6; i++) {
            const s6 c = ld6(cdof + 6 * (dof + i));
            for (int k = 0; k < 6; k++) v.v[k] += c.v[k] * qvel[dof + i];
          }
        } else {
          for (int i = 0; i < nd; i++) st6(cdd + 6 * (dof + i), motion_cross(v, ld6(cdof + 6 * (dof + i))));
          for (int i = 0; i < nd; i++) {
            const s6 c = ld6(cdof + 6 * (dof + i));
            for (int k = 0; k < 6; k++) v.v[k] += c.v[k] * qvel[dof + i];
          }
        }
        dof += nd;
      }
      st6(cvel + 6 * b, v);
    }
    lsync<L>();
  }
}

// passive.py:27-108
template <int L = 32>
__device__ void passive(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nv = m.nv;
  float* qfrc_passive = d.qfrc_passive + W(w, nv);
  if (m.disableflags & DSBL_PASSIVE) {
    for (int i = lane; i < nv; i += L) qfrc_passive[i] = 0.f;
    lsync<L>();
    return;
  }
  const float* qpos = d.qpos + W(w, m.nq);
  const float* qvel = d.qvel + W(w, nv);
  float* spring = d.qfrc_spring + W(w, nv);
  float* damper = d.qfrc_damper + W(w, nv);
  for (int i = lane; i < nv; i += L) spring[i] = 0.f;
  lsync<L>();
  for (int j = lane; j < m.njnt; j += L) {
    const float k = m.jnt_stiffness[j];
    if (k == 0.f) continue;
    const int dof = m.jnt_dofadr[j], t = m.jnt_type[j], a = m.jnt_qposadr[j];
    if (t == JNT_FREE) {
      for (int i = 0; i < 3; i++) spring[dof + i] = -k * (qpos[a + i] - m.qpos_spring[a + i]);
      const f3 dif = quat_sub(ld4(qpos + a + 3), ld4(m.qpos_spring + a + 3));
      spring[dof + 3] = -k * dif.x; spring[dof + 4] = -k * dif.y; spring[dof + 5] = -k * dif.z;
    } else if (t == JNT_BALL) {
      const f3 dif = quat_sub(ld4(qpos + a), ld4(m.qpos_spring + a));
      spring[dof] = -k * dif.x; spring[dof + 1] = -k * dif.y; spring[dof + 2] = -k * dif.z;
    } else {
      spring[dof] = -k * (qpos[a] - m.qpos_spring[a]);
    }
  }
  lsync<L>();
  for (int i = lane; i < nv; i += L) {
    const float dm = -m.dof_damping[i] * qvel[i];
    damper[i] = dm;
    qfrc_passive[i] = dm + spring[i];
  }
  lsync<L>();
}

// smooth.py:398-466 — recursive Newton-Euler bias forces
template <int L = 32>
__device__ void rne(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nb = m.nbody, nv = m.nv;
  float* cacc = d.rne_cacc + W(w, 6 * nb);
  float* cfrc = d.rne_cfrc + W(w, 6 * nb);
  const float* cdd = d.cdof_dot + W(w, 6 * nv);
  const float* qvel = d.qvel + W(w, nv);
  const float* cinert = d.cinert + W(w, 10 * nb);
  const float* cvel = d.cvel + W(w, 6 * nb);
  if (lane < 6) {
    const bool grav = !(m.disableflags & DSBL_GRAVITY);
    cacc[lane] = (lane >= 3 && grav) ? -m.gravity[lane - 3] : 0.f;
  }
  lsync<L>();
  for (int lvl = 1; lvl < m.nlevel; lvl++) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += L) {
      const int b = m.body_tree[n];
      s6 a = ld6(cacc + 6 * m.body_parentid[b]);
      const int da = m.body_dofadr[b];
      for (int i = 0; i < m.body_dofnum[b]; i++) {
        const s6 c = ld6(cdd + 6 * (da + i));
        for (int k = 0; k < 6; k++) a.v[k] += c.v[k] * qvel[da + i];
      }
      st6(cacc + 6 * b, a);
    }
    lsync<L>();
  }
  for (int b = lane; b < nb; b += L) {
    const s6 v = ld6(cvel + 6 * b);
    const s6 f = inert_vec(cinert + 10 * b, ld6(cacc + 6 * b));
    const s6 g = motion_cross_force(v, inert_vec(cinert + 10 * b, v));
    s6 r;
    for (int k = 0; k < 6; k++) r.v[k] = f.v[k] + g.v[k];
    st6(cfrc + 6 * b, r);
  }
  lsync<L>();
  // bottom-up gather; level 0 adds the world into itself as smooth.py:461-464 does
  for (int lvl = m.nlevel - 1; lvl >= 0; lvl--) {
    const int beg = m.body_treeadr[lvl], end = m.body_treeadr[lvl + 1];
    for (int n = beg + lane; n < end; n += L) {
      const int b = m.body_tree[n];
      s6 acc = ld6(cfrc + 6 * b);
      const int ca = m.body_childadr[b], cn = m.body_childnum[b];
      for (int c = 0; c < cn; c++) {
        const s6 x = ld6(cfrc + 6 * m.body_child[ca + c]);
        for (int k = 0; k < 6; k++) acc.v[k] += x.v[k];
      }
      if (b == 0)
        for (int k = 0; k < 6; k++) acc.v[k] += acc.v[k];
      st6(cfrc + 6 * b, acc);
    }
    lsync<L>();
  }
  const float* cdof = d.cdof + W(w, 6 * nv);
  float* bias = d.qfrc_bias + W(w, nv);
  for (int i = lane; i < nv; i += L) bias[i] = dot6(ld6(cdof + 6 * i), ld6(cfrc + 6 * m.dof_bodyid[i]));
  lsync<L>();
}

// forward.py:423-500 (dense path)
template <int L = 32>
__device__ void fwd_velocity(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nv = m.nv;
  const float* moment = d.actuator_moment + W(w, m.nu * nv);
  const float* qvel = d.qvel + W(w, nv);
  float* vel = d.actuator_velocity + W(w, m.nu);
  for (int a = lane; a < m.nu; a += L) {
    float s = 0.f;
    for (int i = 0; i < nv; i++) s += moment[a * nv + i] * qvel[i];
    vel[a] = s;
  }
  lsync<L>();
  com_vel<L>(m, d, w, lane);
  passive<L>(m, d, w, lane);
  rne<L>(m, d, w, lane);
}

// forward.py:503-641
template <int L = 32>
__device__ void fwd_actuation(const MjbModel& m, const MjbData& d, int w, int lane) {
  const int nv = m.nv, nu = m.nu;
  float* qfrc = d.qfrc_actuator + W(w, nv);
  if (!nu || (m.disableflags & DSBL_ACTUATION)) {
    if (d.act_dot)
      for (int i = lane; i < m.na; i += L) d.act_dot[W(w, m.na) + i] = 0.f;
    for (int i = lane; i < nv; i += L) qfrc[i] = 0.f;
    lsync<L>();
    return;
  }
  const float* len = d.actuator_length + W(w, nu);
  const float* vel = d.actuator_velocity + W(w, nu);
  const float* ctrl = d.ctrl + W(w, nu);
  float* force = d.actuator_force + W(w, nu);
  for (int a = lane; a < nu; a += L) {
    const float* gp = m.actuator_gainprm + 10 * a;
    const float* bp = m.actuator_biasprm + 10 * a;
    float gain = gp[0];
    gain += gp[1] * len[a];
    gain += gp[2] * vel[a];
    float bias = bp[0];
    bias += bp[1] * len[a];
    bias += bp[2] * vel[a];
    float c = ctrl[a];
    if (m.actuator_ctrllimited[a] && !(m.disableflags & DSBL_CLAMPCTRL))
      c = fminf(fmaxf(c, m.actuator_ctrlrange[2 * a]), m.actuator_ctrlrange[2 * a + 1]);
    force[a] = gain * c + bias;  // forcerange is not applied (forward.py:539-541)
  }
  lsync<L>();
  const float* moment = d.actuator_moment + W(w, nu * nv);
  for (int i = lane; i < nv; i += L) {
    float s = 0.f;
    for (int a = 0; a < nu; a++) s += moment[a * nv + i] * force[a];
    const int j = m.dof_jntid[i];
    if (m.jnt_actfrclimited[j]) s = fminf(fmaxf(s, m.jnt_actfrcrange[2 * j]), m.jnt_actfrcrange[2 * j + 1]);
    qfrc[i] = s;
  }
  lsync<L>();
}

// support.py:140-172 — qfrc += J^T xfrc_applied (Jacobian at each body's xipos)
__device__ void xfrc_accumulate(const MjbModel& m, const MjbData& d, int w, float* qfrc, int lane) {
  const int nv = m.nv, nb = m.nbody;
  const float* cdof = d.cdof + W(w, 6 * nv);
  const float* xipos = d.xipos + W(w, 3 * nb);
  const float* sc = d.subtree_com + W(w, 3 * nb);
  const float* xfrc = d.xfrc_applied + W(w, 6 * nb);
  // a world with no applied body force adds only zeros (for finite states): skip its walk
  bool any = false;
  for (int e = lane; e < 6 * nb; e += 32) any |= xfrc[e] != 0.f;
  if (!__any_sync(WARP_FULL, any)) return;
  for (int i = lane; i < nv; i += 32) {
    const s6 c = ld6(cdof + 6 * i);
    const f3 rot{c.v[0], c.v[1], c.v[2]}, lin{c.v[3], c.v[4], c.v[5]};
    const int db = m.dof_bodyid[i];
    float acc = 0.f;
    for (int b = db; b < m.body_subtreeend[db]; b++) {  // bodies in the subtree of db
      const f3 off = ld3(xipos + 3 * b) - ld3(sc + 3 * m.body_rootid[b]);
      const f3 force = ld3(xfrc + 6 * b), torque = ld3(xfrc + 6 * b + 3);
      acc += (dot(lin, force) + dot(rot, torque)) + dot(cross(rot, off), force);
    }
    qfrc[i] += acc;
  }
  __syncwarp();
}

// forward.py:644-661
// tile_has_qLD: the per-warp tile still holds the factor left by factor_m
__device__ void fwd_acceleration(const MjbModel& m, const MjbData& d, int w, int lane,
                                 float* tile = nullptr, bool tile_has_qLD = false) {
  const int nv = m.nv;
  float* sm = d.qfrc_smooth + W(w, nv);
  const float* pas = d.qfrc_passive + W(w, nv);
  const float* bias = d.qfrc_bias + W(w, nv);
  const float* act = d.qfrc_actuator + W(w, nv);
  const float* app = d.qfrc_applied + W(w, nv);
  for (int i = lane; i < nv; i += 32) sm[i] = pas[i] - bias[i] + act[i] + app[i];
  __syncwarp();
  xfrc_accumulate(m, d, w, sm, lane);
  if (m.precision && tile) {  // FP64 factor-solve in the double tile after the float tile
    factor_solve_blocks_d(m, d.qM + W(w, nv * nv), nullptr, 0.f, d.qacc_smooth + W(w, nv), sm, lane,
                          reinterpret_cast<double*>(tile + tile_floats(nv)));
    return;
  }
  solve_m_world(m, d, w, d.qacc_smooth + W(w, nv), sm, lane, tile, tile_has_qLD);
}

// ------------------------------------------------------------------------------------------
// forward.py:43-162 — advance velocities and positions (semi-implicit)
__device__ void advance(const MjbModel& m, const MjbData& d, int w, const float* qacc, int lane) {
  const int nv = m.nv;
  const float dt = m.timestep;
  float* qvel = d.qvel + W(w, nv);
  float* qpos = d.qpos + W(w, m.nq);
  for (int i = lane; i < nv; i += 32) qvel[i] = qvel[i] + qacc[i] * dt;
  __syncwarp();
  for (int j = lane; j < m.njnt; j += 32) {
    const int t = m.jnt_type[j], a = m.jnt_qposadr[j], dof = m.jnt_dofadr[j];
    if (t == JNT_FREE) {
      for (int k = 0; k < 3; k++) qpos[a + k] = qpos[a + k] + dt * qvel[dof + k];
      st4(qpos + a + 3, quat_integrate(ld4(qpos + a + 3), ld3(qvel + dof + 3), dt));
    } else if (t == JNT_BALL) {
      st4(qpos + a, quat_integrate(ld4(qpos + a), ld3(qvel + dof), dt));
    } else {
      qpos[a] = qpos[a] + dt * qvel[dof];
    }
  }
  __syncwarp();
}

// forward.py:165-242 — Euler with implicit joint damping unless EULERDAMP is disabled
__device__ void euler(const MjbModel& m, const MjbData& d, int w, int lane, float* tile = nullptr) {
  const int nv = m.nv;
  if (m.disableflags & DSBL_EULERDAMP) {
    advance(m, d, w, d.qacc + W(w, nv), lane);
    return;
  }
  float* x = d.qacc_integration + W(w, nv);
  const float* sm = d.qfrc_smooth + W(w, nv);
  const float* qc = d.qfrc_constraint + W(w, nv);
  if (m.is_sparse) {  // eulerdamp_sparse (forward.py:171-193)
    const float* M = d.qM + W(w, m.nM);
    float* Mi = d.qM_integration ? d.qM_integration + W(w, m.nM) : nullptr;
    float* Ls = d.qLD_integration + W(w, m.nM);
    float* f = d.qfrc_integration ? d.qfrc_integration + W(w, nv) : x;
    for (int e = lane; e < m.nM; e += 32) {
      if (Mi) Mi[e] = M[e];
      Ls[e] = M[e];
    }
    __syncwarp();
    for (int i = lane; i < nv; i += 32) {
      const int a = m.dof_Madr[i];
      const float v = M[a] + m.timestep * m.dof_damping[i];
      if (Mi) Mi[a] = v;
      Ls[a] = v;
      f[i] = sm[i] + qc[i];
    }
    __syncwarp();
    factor_sparse(m, Ls, nullptr, lane);
    solve_sparse(m, Ls, nullptr, x, f, lane);
    advance(m, d, w, x, lane);
    return;
  }
  float* L = d.qLD_integration + W(w, nv * nv);
  factor_blocks(m, d.qM + W(w, nv * nv), L, lane, m.dof_damping, m.timestep, tile);
  for (int i = lane; i < nv; i += 32) x[i] = sm[i] + qc[i];
  __syncwarp();
  if (m.precision && tile)  // the float factor stays in qLD_integration; x in FP64
    factor_solve_blocks_d(m, d.qM + W(w, nv * nv), m.dof_damping, m.timestep, x, x, lane,
                          reinterpret_cast<double*>(tile + tile_floats(nv)));
  else
    solve_blocks(m, L, x, x, lane, tile, true);
  advance(m, d, w, x, lane);
}

// forward.py:245-405 — implicitfast (dense): (M - dt qDeriv) qacc = qfrc_smooth + qfrc_constraint
// with qDeriv = moment^T diag(bias_vel + gain_vel * ctrl) moment - diag(damping)
__device__ void implicit(const MjbModel& m, const MjbData& d, int w, int lane, float* tile = nullptr) {
  const int nv = m.nv, nu = m.nu;
  const bool passive_on = !(m.disableflags & DSBL_PASSIVE);
  const bool act_on = !(m.disableflags & DSBL_ACTUATION) && m.actuator_affine_bias_gain;
  if (!passive_on && !act_on) {
    advance(m, d, w, d.qacc + W(w, nv), lane);
    return;
  }
  float* vel = d.act_vel_integration + W(w, nu);
  const float* moment = d.actuator_moment + W(w, nu * nv);
  if (act_on) {  // actuator_bias_gain_vel (forward.py:277-299)
    for (int a = lane; a < nu; a += 32) {
      const float bv = m.actuator_biastype[a] == 1 ? m.actuator_biasprm[10 * a + 2] : 0.f;
      const float gv = m.actuator_gaintype[a] == 1 ? m.actuator_gainprm[10 * a + 2] : 0.f;
      const float c = m.actuator_dyntype[a] != 0 ? d.act[W(w, m.na) + a] : d.ctrl[W(w, nu) + a];
      vel[a] = bv + gv * c;
    }
    __syncwarp();
  }
  bool tiled = tile != nullptr;  // every block small enough for the tile
  for (int blk = 0; blk < m.nblock; blk++) tiled &= m.block_size[blk] <= 32;
  const float* qM = d.qM + W(w, nv * nv);
  float* Mi = d.qM_integration + W(w, nv * nv);
  float* f = d.qfrc_integration + W(w, nv);
  const float* sm = d.qfrc_smooth + W(w, nv);
  const float* qc = d.qfrc_constraint + W(w, nv);
  float* L = d.qLD_integration + W(w, nv * nv);
  float* x = d.qacc_integration + W(w, nv);
  for (int i = lane; i < nv; i += 32) f[i] = sm[i] + qc[i];
  if (tiled && !(m.nblock == 1 && m.block_size[0] == nv))  // else tile_store_lower writes it all
    for (int e = lane; e < nv * nv; e += 32) L[e] = 0.f;
  __syncwarp();
  // qderiv_actuator_fused_kernel, per tree tile: Mi = qM - dt qDeriv, one coalesced row at a time
  for (int blk = 0; blk < m.nblock; blk++) {
    const int a0 = m.block_adr[blk], n = m.block_size[blk];
    if (tiled && !act_on) {  // damping only: the block's rows loaded into the tile eight at a time
      const int tld = tile_ld(nv);
      copy_rows(qM + a0 * nv + a0, nv, tile, tld, n, n, n, lane);
      __syncwarp();
      if (passive_on && lane < n) {
        const int i = a0 + lane;
        tile[lane * tld + lane] = tile[lane * tld + lane] - (-m.dof_damping[i]) * m.timestep;
      }
      __syncwarp();
      copy_rows(tile, tld, Mi + a0 * nv + a0, nv, n, n, n, lane);
      __syncwarp();
    } else
    for (int r = 0; r < n; r++) {
      const int i = a0 + r;
      for (int jj = lane; jj < n; jj += 32) {
        const int j = a0 + jj;
        float qd = 0.f;
        if (act_on)
          for (int a = 0; a < nu; a++) qd += moment[a * nv + i] * vel[a] * moment[a * nv + j];
        if (passive_on && i == j) qd -= m.dof_damping[i];
        const float v = qM[i * nv + j] - qd * m.timestep;
        Mi[i * nv + j] = v;
        if (tiled) tile[r * tile_ld(nv) + jj] = v;
      }
    }
    __syncwarp();
    if (tiled) {  // factor and solve this block in the tile
      const int tld = tile_ld(nv);
      chol_tile(tile, tld, n, lane);
      tile_store_lower(tile, tld, n, L + a0 * nv + a0, nv, lane);
      const float xi = cho_solve_tile(tile, tld, n, lane < n ? f[a0 + lane] : 0.f, lane);
      __syncwarp();
      if (lane < n) x[a0 + lane] = xi;
      __syncwarp();
    }
  }
  if (!tiled) {
    factor_blocks(m, Mi, L, lane, nullptr, 0.f, tile);
    solve_blocks(m, L, x, f, lane);
  }
  if (m.precision && tile)  // the float factor stays in qLD_integration; x again in FP64
    factor_solve_blocks_d(m, Mi, nullptr, 0.f, x, f, lane,
                          reinterpret_cast<double*>(tile + tile_floats(nv)));
  advance(m, d, w, x, lane);
}

}  // namespace mjb
