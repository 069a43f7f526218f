// The chosen form's constraint solver for large models (nv > 32, dense or sparse mass matrix): one
// CTA of NW warps per world (solver.py:26-1000, the same algorithm as solve_generic).
//
// A world with hundreds of dofs and constraint rows is too much for one warp: the Newton
// Hessian's factorisation (nv^3 / 3 multiply-adds) and the row loops (dense nv-wide Jacobian
// rows) serialise on 32 lanes, and with 16 such warps per SM the per-world matrices (nv^2 floats
// each) no longer fit in L2.  Here all NW warps of a CTA work on one world: per-row dot products
// are warp-per-row (coalesced reads of the dense Jacobian rows), per-row scalars thread-per-row,
// per-dof vectors thread-per-dof, and every per-world sum is a CTA reduction in a fixed order
// (warp sums, then the warps' partials in warp order), identical in every thread, so control flow
// stays uniform across the CTA.  The Hessian H = tril(qM) + sum_active D J'J is assembled in efc_h
// (each warp updates the H rows it owns, row by row in constraint order, so no two warps touch the
// same entry; or, selected by the autotuner and always in the precision form, as split-TF32
// tensor-core tiles, assemble_hessian_tc) and factored by chol_cta: a left-looking blocked
// Cholesky with 32-column panels whose panel updates A[r, p] -= L[r, :p] L[p, :p]^T run on the
// tensor pipe in split TF32 (mjb_tc.cuh), the 32 x 32 diagonal blocks by chol_tile and the panel
// rows below by substitution.  The precision form factors and solves in FP64 in shared memory.
#pragma once

#include "mjb_solver.cuh"

namespace mjb {

// CTA sums of K values: warp sums, then the NW warps' partials added in warp order; every thread
// returns the totals.  red: K * NW elements of shared memory.
template <int NW, int K, typename T>
__device__ __forceinline__ void cta_sum(T (&v)[K], T* red, int warp, int lane) {
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = warp_sum_t(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) red[k * NW + warp] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) {
    T s = red[k * NW];
#pragma unroll
    for (int q = 1; q < NW; q++) s += red[k * NW + q];
    v[k] = s;
  }
  __syncthreads();
}

// the dof tree block [a, a + size) that contains dof i (binary search over block_adr)
__device__ __forceinline__ void dof_block(const MjbModel& m, int i, int& a, int& size) {
  int lo = 0, hi = m.nblock - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (m.block_adr[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  a = m.block_adr[lo];
  size = m.block_size[lo];
}

// Left-looking blocked Cholesky of the n x n SPD lower triangle of A (row stride ld, global
// memory) by a CTA of NW warps: per 32-column panel p, (i) the panel's rows are updated with the
// finished columns, A[r, p] -= L[r, :p] L[p, :p]^T for every row r >= p, as m16n8k8 tensor-core
// tiles in split TF32 (16-row m-tiles dealt to the warps, the panel's 32 columns as 4 n-tiles),
// (ii) warp 0 factors the 32 x 32 diagonal block in the shared tile T (chol_tile) and writes it
// back with its reciprocal diagonal in T's column 32, (iii) every row below solves
// L[r, p] = A[r, p] L_pp^-T, one thread per row.  T: 32 x 36 + 32 floats of shared memory.
template <int NW>
__device__ __noinline__ void chol_cta(float* A, int ld, int n, float* T, int warp, int lane) {
  constexpr int TL = 36, kMt = 3;
  const int g = lane >> 2, t = lane & 3;
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int pn = min(32, n - c0);
    if (c0 > 0) {
      const int nmt = (n - c0 + 15) >> 4;
      for (int mt0 = warp; mt0 < nmt; mt0 += NW * kMt) {
        float acc[kMt][4][4];
#pragma unroll
        for (int q = 0; q < kMt; q++)
#pragma unroll
          for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[q][nt][e] = 0.f;
        // raw loads of chunk k0 + 8 are issued before chunk k0's splits and products
        float rb[4][2], ra[kMt][4];
        auto load = [&](int k0, float (&xb)[4][2], float (&xa)[kMt][4]) {
#pragma unroll
          for (int nt = 0; nt < 4; nt++) {  // B[k][j] = L[c0 + j][k0 + k], j = 8 nt + g
            const int r = c0 + 8 * nt + g;
            const float* Ar = A + size_t(r) * ld + k0;
            xb[nt][0] = r < n ? Ar[t] : 0.f;
            xb[nt][1] = r < n ? Ar[t + 4] : 0.f;
          }
#pragma unroll
          for (int q = 0; q < kMt; q++) {
            const int mt = mt0 + q * NW;
            const int r0 = c0 + 16 * mt + g, r1 = r0 + 8;
            const bool ok0 = mt < nmt && r0 < n, ok1 = mt < nmt && r1 < n;
            const float* A0 = A + size_t(r0) * ld + k0;
            const float* A1 = A + size_t(r1) * ld + k0;
            xa[q][0] = ok0 ? A0[t] : 0.f;
            xa[q][1] = ok1 ? A1[t] : 0.f;
            xa[q][2] = ok0 ? A0[t + 4] : 0.f;
            xa[q][3] = ok1 ? A1[t + 4] : 0.f;
          }
        };
        load(0, rb, ra);
        for (int k0 = 0; k0 < c0; k0 += 8) {
          float nb[4][2], na[kMt][4];
          if (k0 + 8 < c0) load(k0 + 8, nb, na);
          FragB b[4];
#pragma unroll
          for (int nt = 0; nt < 4; nt++) b[nt] = frag_b(rb[nt][0], rb[nt][1]);
#pragma unroll
          for (int q = 0; q < kMt; q++) {
            const int mt = mt0 + q * NW;
            if (mt < nmt) {
              const FragA a = frag_a(ra[q][0], ra[q][1], ra[q][2], ra[q][3]);
#pragma unroll
              for (int nt = 0; nt < 4; nt++) mma_3xtf32(acc[q][nt], a, b[nt]);
            }
          }
          if (k0 + 8 < c0) {
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
              rb[nt][0] = nb[nt][0];
              rb[nt][1] = nb[nt][1];
            }
#pragma unroll
            for (int q = 0; q < kMt; q++)
#pragma unroll
              for (int e = 0; e < 4; e++) ra[q][e] = na[q][e];
          }
        }
#pragma unroll
        for (int q = 0; q < kMt; q++) {
          const int mt = mt0 + q * NW;
          if (mt >= nmt) break;
          const int r0 = c0 + 16 * mt + g, r1 = r0 + 8;
#pragma unroll
          for (int nt = 0; nt < 4; nt++) {
            const int cc = c0 + 8 * nt + 2 * t;
#pragma unroll
            for (int e = 0; e < 2; e++) {
              if (cc + e < c0 + pn) {  // lower triangle only (the diagonal block's upper part
                                       // is not part of the factor)
                if (r0 < n && cc + e <= r0) A[size_t(r0) * ld + cc + e] -= acc[q][nt][e];
                if (r1 < n && cc + e <= r1) A[size_t(r1) * ld + cc + e] -= acc[q][nt][2 + e];
              }
            }
          }
        }
      }
    }
    __syncthreads();
    if (warp == 0) {  // (ii)
      for (int r = 0; r < pn; r++)
        if (lane < pn) T[r * TL + lane] = lane <= r ? A[size_t(c0 + r) * ld + c0 + lane] : 0.f;
      __syncwarp();
      chol_tile(T, TL, pn, lane);
      for (int r = 0; r < pn; r++)
        if (lane <= r) A[size_t(c0 + r) * ld + c0 + lane] = T[r * TL + lane];
      if (lane < pn) T[lane * TL + 32] = __frcp_rn(T[lane * TL + lane]);
    }
    __syncthreads();
    const bool vec = (ld & 3) == 0 && pn == 32;  // rows 16-byte aligned: float4 reads and writes
    for (int i = c0 + pn + int(threadIdx.x); i < n; i += NW * 32) {  // (iii)
      float* Ai = A + size_t(i) * ld + c0;
      float x[32];
      if (vec) {
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const float4 v = reinterpret_cast<const float4*>(Ai)[q];
          x[4 * q] = v.x;
          x[4 * q + 1] = v.y;
          x[4 * q + 2] = v.z;
          x[4 * q + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int c = 0; c < 32; c++) x[c] = c < pn ? Ai[c] : 0.f;
      }
#pragma unroll
      for (int c = 0; c < 32; c++) {
        if (c < pn) {
          float v = x[c];
#pragma unroll
          for (int q = 0; q < c; q++) v -= x[q] * T[c * TL + q];
          x[c] = v * T[c * TL + 32];
        }
      }
      if (vec) {
#pragma unroll
        for (int q = 0; q < 8; q++)
          reinterpret_cast<float4*>(Ai)[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
      } else {
#pragma unroll
        for (int c = 0; c < 32; c++)
          if (c < pn) Ai[c] = x[c];
      }
    }
    __syncthreads();
  }
}

// x = (L L^T)^-1 y by a CTA of NW warps for the n x n lower factor L in global memory (row stride
// ld), blocked by 32: forward, each block's partial y_b - L[b, :b] z[:b] is a row-per-warp dot
// product over the finished part (coalesced row reads, warp sums), then warp 0 solves the 32 x 32
// diagonal block with its rows in registers; backward, each block's partial
// z_b - L[b+:, b]^T x[b+:] is accumulated warp-per-row over the rows below (lane j reads the
// row's entry in column j of the block, coalesced), reduced across the warps in red, then warp 0
// solves L_bb^T.  z: n floats of shared memory (the intermediate vector); red: 32 NW floats.
// x and y are in global memory (x may alias y).
template <int NW>
__device__ __noinline__ void cho_solve_cta(const float* L, int ld, int n, float* x, const float* y,
                                           float* z, float* red, int warp, int lane) {
  for (int c0 = 0; c0 < n; c0 += 32) {  // L z = y
    const int pn = min(32, n - c0);
    for (int j = warp; j < pn; j += NW) {
      const float* Lr = L + size_t(c0 + j) * ld;
      float a = 0.f;
      for (int k = lane; k < c0; k += 32) a += Lr[k] * z[k];
      a = warp_sum(a);
      if (lane == 0) z[c0 + j] = y[c0 + j] - a;
    }
    __syncthreads();
    if (warp == 0) {
      float r[32];  // row `lane` of the diagonal block
      const float* Lr = L + size_t(c0 + min(lane, pn - 1)) * ld + c0;
#pragma unroll
      for (int q = 0; q < 32; q++) r[q] = (q < pn && q <= lane && lane < pn) ? Lr[q] : 1.f;
      float zi = lane < pn ? z[c0 + lane] : 0.f;
#pragma unroll
      for (int q = 0; q < 32; q++) {
        if (q < pn) {
          const float zq = __shfl_sync(WARP_FULL, zi, q) / __shfl_sync(WARP_FULL, r[q], q);
          if (lane == q) zi = zq;
          else if (lane > q && lane < pn) zi -= r[q] * zq;
        }
      }
      if (lane < pn) z[c0 + lane] = zi;
    }
    __syncthreads();
  }
  const int nb = (n + 31) / 32;
  for (int b = nb - 1; b >= 0; b--) {  // L^T x = z
    const int c0 = 32 * b, pn = min(32, n - c0);
    float acc = 0.f;  // lane j: sum over this warp's rows i below the block of L[i][c0 + j] x[i]
    for (int i = c0 + pn + warp; i < n; i += NW)
      if (lane < pn) acc += L[size_t(i) * ld + c0 + lane] * z[i];
    red[warp * 32 + lane] = acc;
    __syncthreads();
    if (warp == 0) {
      float t = 0.f;
#pragma unroll
      for (int q = 0; q < NW; q++) t += red[q * 32 + lane];
      float xi = lane < pn ? z[c0 + lane] - t : 0.f;
      // back substitution with L_bb^T: column lane of L_bb is row lane of L_bb^T
      for (int q = pn - 1; q >= 0; q--) {
        const float lq = lane < q ? L[size_t(c0 + q) * ld + c0 + lane] : 0.f;
        const float xq = __shfl_sync(WARP_FULL, xi, q) / L[size_t(c0 + q) * ld + c0 + q];
        if (lane == q) xi = xq;
        else if (lane < q) xi -= lq * xq;
      }
      if (lane < pn) z[c0 + lane] = xi;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += NW * 32) x[i] = z[i];
  __syncthreads();
}

// Per-CTA shared memory of the solver (floats): reductions (16 NW, as doubles 32 NW), the
// diagonal tile (32 x 36 + 32), each warp's row-compaction scratch and the triangular solves'
// vector (nv); the precision form adds the FP64 Hessian factor, its lower triangle packed row by
// row (row i at i (i + 1) / 2), then the FP64 solve's vector and the factor's reciprocal
// diagonal (nv doubles each), 16-byte aligned after the floats.
__host__ __device__ __forceinline__ int tri(int i) { return i * (i + 1) / 2; }
__host__ __device__ __forceinline__ int cta_solver_smem_base(int nv, int nw) {
  return round4i(32 * nw + 32 * 36 + 32 + nw * 2 * round4i(nv) + round4i(nv));
}
__host__ __device__ __forceinline__ int cta_solver_smem_floats(int nv, int nw, bool prec = false) {
  const int base = cta_solver_smem_base(nv, nw);
  return prec ? base + 2 * (tri(nv) + 2 * nv + 1) : base;
}

// FP64 counterpart of chol_cta for the precision form, on the packed lower triangle P of an
// n x n SPD matrix in shared memory: per 32-column panel, (i) every entry (r, j) of the panel's
// rows r >= p subtracts its dot product over the finished columns (4 x 1 strips of entries per
// thread, so each loaded L[j][k] serves four rows); (ii) warp 0 factors the diagonal block in
// place, lane per row, with the pivot's reciprocal kept in rd; (iii) the rows below solve
// against it, one thread per row, multiplying by rd.
template <int NW>
__device__ __noinline__ void chol_cta_d(double* P, double* rd, int n, int warp, int lane) {
  constexpr int NT = NW * 32;
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int pn = min(32, n - c0);
    if (c0 > 0) {
      const int nr4 = (n - c0 + 3) / 4;  // strips of four rows
      for (int e = int(threadIdx.x); e < nr4 * pn; e += NT) {
        const int r = c0 + 4 * (e / pn), j = c0 + e % pn;
        const double* Lj = P + tri(j);
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        const double* R0 = P + tri(r);
        const double* R1 = P + tri(min(r + 1, n - 1));
        const double* R2 = P + tri(min(r + 2, n - 1));
        const double* R3 = P + tri(min(r + 3, n - 1));
        for (int k = 0; k < c0; k++) {
          const double l = Lj[k];
          s0 += R0[k] * l;
          s1 += R1[k] * l;
          s2 += R2[k] * l;
          s3 += R3[k] * l;
        }
        if (j <= r) P[tri(r) + j] -= s0;
        if (r + 1 < n && j <= r + 1) P[tri(r + 1) + j] -= s1;
        if (r + 2 < n && j <= r + 2) P[tri(r + 2) + j] -= s2;
        if (r + 3 < n && j <= r + 3) P[tri(r + 3) + j] -= s3;
      }
      __syncthreads();
    }
    if (warp == 0) {  // (ii): column k of the block, lanes over its rows (left-looking)
      for (int k = 0; k < pn; k++) {
        const int i = c0 + k + lane;
        const double* Lk = P + tri(c0 + k) + c0;
        double s = 0.0;
        if (k + lane < pn) {
          const double* Li = P + tri(i) + c0;
          s = Li[k];
          for (int q = 0; q < k; q++) s -= Li[q] * Lk[q];
        }
        const double sk = __shfl_sync(WARP_FULL, s, 0);
        const double inv = rsqrt(sk);  // the pivot's reciprocal; L_kk = s_k rsqrt(s_k)
        const double lkk = sk * inv;
        __syncwarp();
        if (lane == 0) {
          P[tri(c0 + k) + c0 + k] = lkk;
          rd[c0 + k] = inv;
        } else if (k + lane < pn) {
          P[tri(i) + c0 + k] = s * inv;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int i = c0 + pn + int(threadIdx.x); i < n; i += NT) {  // (iii)
      double* Ai = P + tri(i) + c0;
      for (int c = 0; c < pn; c++) {
        double v = Ai[c];
        const double* Lc = P + tri(c0 + c) + c0;
        for (int q = 0; q < c; q++) v -= Ai[q] * Lc[q];
        Ai[c] = v * rd[c0 + c];
      }
    }
    __syncthreads();
  }
}

// x = (L L^T)^-1 y for the packed FP64 factor in shared memory, one warp, in FP64 with the
// intermediate vector in v (n doubles of shared memory) and the reciprocal diagonal rd; x and y
// are n floats in global memory (x may alias y).
__device__ void cho_solve_d_warp(const double* P, const double* rd, int n, double* v, float* x,
                                 const float* y, int lane) {
  for (int i = lane; i < n; i += 32) v[i] = double(y[i]);
  __syncwarp();
  for (int k = 0; k < n; k++) {  // L z = y, a column at a time; lanes update the rows below
    const double zk = v[k] * rd[k];
    __syncwarp();
    if (lane == (k & 31)) v[k] = zk;
    for (int i = k + 1 + lane; i < n; i += 32) v[i] -= P[tri(i) + k] * zk;
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; k--) {  // L^T x = z: row k of L is column k of L^T
    const double xk = v[k] * rd[k];
    __syncwarp();
    if (lane == (k & 31)) v[k] = xk;
    const double* Lk = P + tri(k);
    for (int i = lane; i < k; i += 32) v[i] -= Lk[i] * xk;
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) x[i] = float(v[i]);
  __syncwarp();
}

template <int NW, bool PREC>
struct CtaSolver {
  const MjbModel& m;
  const MjbData& d;
  int w, tid, lane, warp, nv, adr, n;
  float *qacc, *Ma, *grad, *Mgrad, *search, *mv, *qfrc_constraint, *H;
  const float *qM, *qfrc_smooth, *qacc_smooth;
  float* red;    // 32 NW floats (cta sums of up to 9 values, as floats or doubles; the solves)
  float* T;      // chol_cta's diagonal tile
  float* nz;     // this warp's row compaction: round4(nv) ints, then round4(nv) floats
  float* zv;     // the triangular solves' intermediate vector (nv floats)
  double* Ld;    // precision form: the Hessian's FP64 factor, lower triangle packed by rows
  double* vd;    // precision form: the FP64 solve's vector (nv doubles)
  double* rdg;   // precision form: the factor's reciprocal diagonal (nv doubles)
  bool reuse = true, factored = false, changed = true;
  bool tc = false;  // FP32 form: the Hessian assembled on the tensor pipe (assemble_hessian_tc)
  float cost, prev_cost, gauss, grad_dot, search_dot, gtol, alpha, beta;
  float qg[3];
  static constexpr int NT = NW * 32;

  template <int K>
  __device__ __forceinline__ void sum(float (&v)[K]) { cta_sum<NW, K, float>(v, red, warp, lane); }
  // line-search coefficient sums: base + the CTA's sum of x, in FP64 in the precision form
  template <int K>
  __device__ __forceinline__ void ls_sums(const float (&base)[K], float (&x)[K]) {
    if (PREC) {
      double v[K];
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = double(x[k]);
      cta_sum<NW, K, double>(v, reinterpret_cast<double*>(red), warp, lane);
#pragma unroll
      for (int k = 0; k < K; k++) x[k] = float(double(base[k]) + v[k]);
    } else {
      sum<K>(x);
#pragma unroll
      for (int k = 0; k < K; k++) x[k] = base[k] + x[k];
    }
  }

  // res = M vec (support.py:35-137): the dense mass matrix within each dof tree block, or the
  // sparse one's diagonal-plus-ancestor products, one tree per thread
  __device__ void mul_m(float* res, const float* vec) {
    if (m.is_sparse) {
      for (int blk = tid; blk < m.nblock; blk += NT) {
        const int a = m.block_adr[blk], size = m.block_size[blk];
        for (int i = a; i < a + size; i++) res[i] = qM[m.dof_Madr[i]] * vec[i];
        for (int i = a; i < a + size; i++) {
          int Mij = m.dof_Madr[i] + 1;
          for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j], Mij++) {
            res[i] += qM[Mij] * vec[j];
            res[j] += qM[Mij] * vec[i];
          }
        }
      }
      __syncthreads();
      return;
    }
    for (int i = tid; i < nv; i += NT) {
      int a, size;
      dof_block(m, i, a, size);
      const float* row = qM + size_t(i) * nv;
      float s = 0.f;
      for (int j = a; j < a + size; j++) s += row[j] * vec[j];
      res[i] = s;
    }
    __syncthreads();
  }

  // out[r] = J_r . x - sub[r] for every row (warp per row); sub may be null
  __device__ void rows_dot(const float* x, float* out, const float* sub) {
    for (int k = warp; k < n; k += NW) {
      const float* J = d.efc_J + size_t(adr + k) * nv;
      float v = 0.f;
      for (int i = lane; i < nv; i += 32) v += J[i] * x[i];
      v = warp_sum(v);
      if (lane == 0) out[adr + k] = sub ? v - sub[adr + k] : v;
    }
    __syncthreads();
  }

  // solver.py:75-173
  __device__ void update_constraint() {
    prev_cost = cost;
    float c[2] = {0.f, 0.f};
    bool ch = false;
    for (int k = tid; k < n; k += NT) {
      const int r = adr + k;
      const float Jaref = d.efc_Jaref[r], D = d.efc_D[r];
      const int active = Jaref < 0.f;
      ch |= d.efc_active[r] != active;
      d.efc_active[r] = active;
      if (active) {
        d.efc_force[r] = -1.f * D * Jaref;
        c[0] += 0.5f * D * Jaref * Jaref;
      } else {
        d.efc_force[r] = 0.f;
      }
    }
    changed = __syncthreads_or(ch) != 0;
    for (int i = tid; i < nv; i += NT) {
      float f = 0.f;
      for (int k = 0; k < n; k++) {
        const float fk = d.efc_force[adr + k];
        if (fk != 0.f) f += d.efc_J[size_t(adr + k) * nv + i] * fk;
      }
      qfrc_constraint[i] = f;
      c[1] += 0.5f * (Ma[i] - qfrc_smooth[i]) * (qacc[i] - qacc_smooth[i]);
    }
    sum<2>(c);
    gauss = c[1];
    cost = c[0] + c[1];
  }

  // H = tril(qM) + sum over active rows of D J'J in efc_h (update_gradient's Newton Hessian,
  // solver.py:249-276): warp q owns the H rows i with i % NW == q, and applies each row's outer
  // product over the row's nonzero columns to those rows in constraint order, so every entry sees
  // the reference's sequence of additions and no two warps write the same entry.
  // the lower triangle of the mass matrix into Out (row stride ldh, or packed by rows): the
  // dense qM a coalesced row per warp; the sparse one zeros, then each dof's row of its
  // ancestors (smooth.py:264-279's layout), one dof per thread
  template <typename TH, bool PACKED = false>
  __device__ void lower_mass(TH* Out, int ldh) {
    auto at = [&](int i) { return PACKED ? size_t(tri(i)) : size_t(i) * ldh; };
    if (!m.is_sparse) {
      for (int i = warp; i < nv; i += NW) {
        const float* Mi = qM + size_t(i) * nv;
        TH* Hi = Out + at(i);
        for (int j = lane; j <= i; j += 32) Hi[j] = TH(Mi[j]);
      }
      __syncthreads();
      return;
    }
    for (int i = warp; i < nv; i += NW) {
      TH* Hi = Out + at(i);
      for (int j = lane; j <= i; j += 32) Hi[j] = TH(0);
    }
    __syncthreads();
    for (int i = tid; i < nv; i += NT) {
      int a = m.dof_Madr[i];
      TH* Hi = Out + at(i);
      Hi[i] = TH(qM[a]);
      for (int j = m.dof_parentid[i]; j >= 0; j = m.dof_parentid[j]) Hi[j] = TH(qM[++a]);
    }
    __syncthreads();
  }

  __device__ void assemble_hessian() {
    lower_mass<float>(H, nv);
    int* nzi = reinterpret_cast<int*>(nz);
    float* nzv = nz + round4i(nv);
    for (int k = 0; k < n; k++) {
      const int r = adr + k;
      if (!d.efc_active[r]) continue;
      const float D = d.efc_D[r];
      if (D == 0.f) continue;
      const float* J = d.efc_J + size_t(r) * nv;
      int cnt = 0;
      for (int base = 0; base < nv; base += 256) {  // eight 32-column chunks loaded, then compacted
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int c = base + 32 * q + lane;
          v[q] = c < nv ? J[c] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const unsigned mk = __ballot_sync(WARP_FULL, v[q] != 0.f);
          if (v[q] != 0.f) {
            const int p = cnt + __popc(mk & ((1u << lane) - 1u));
            nzi[p] = base + 32 * q + lane;
            nzv[p] = v[q];
          }
          cnt += __popc(mk);
        }
      }
      __syncwarp();
      for (int a = 0; a < cnt; a++) {
        const int i = nzi[a];
        if (i % NW != warp) continue;
        float* Hi = H + size_t(i) * nv;
        const float va = nzv[a];
        for (int b = lane; b <= a; b += 32) Hi[nzi[b]] += va * nzv[b] * D;
      }
      __syncwarp();
    }
    __syncthreads();
  }

  // H = tril(qM) + sum over active rows of D J'J on the tensor pipe in split TF32 (mjb_tc.cuh):
  // H = qM + A B with A = J^T (nv x n) and B = diag(c) J (n x nv), c = D on active rows and 0
  // elsewhere; warp q takes the 16-row m-tiles mt = q, q + NW, ... and, four at a time, the m16n8
  // tiles of that row band that touch the lower triangle; the k dimension runs over the world's
  // rows eight at a time, the accumulators start from qM; writes the lower triangle of Hout (row
  // stride ldh elements: efc_h; or, PACKED, the precision form's packed FP64 triangle).
  template <typename TH, bool PACKED = false>
  __device__ void assemble_hessian_tc(TH* Hout, int ldh) {
    const int g = lane >> 2, t = lane & 3;
    const int nmt = (nv + 15) >> 4, ncol8 = (nv + 7) >> 3;
    const float* J = d.efc_J + size_t(adr) * nv;
    // the accumulators start from the mass matrix: read from qM when dense; the sparse layout is
    // first expanded into Hout's lower triangle and read back from there
    const bool sparse = m.is_sparse;
    if (sparse) lower_mass<TH, PACKED>(Hout, ldh);
    auto mass = [&](int r, int c) -> float {
      if (r >= nv || c >= nv) return 0.f;
      if (!sparse) return qM[size_t(r) * nv + c];
      return c <= r ? float(Hout[(PACKED ? size_t(tri(r)) : size_t(r) * ldh) + c]) : 0.f;
    };
    for (int mt = warp; mt < nmt; mt += NW) {
      const int r0 = 16 * mt + g, r1 = r0 + 8;
      const int nnt = min((16 * mt + 15) / 8 + 1, ncol8);
      for (int nt0 = 0; nt0 < nnt; nt0 += 4) {
        float acc[4][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int c = 8 * (nt0 + q) + 2 * t;
          acc[q][0] = mass(r0, c);
          acc[q][1] = mass(r0, c + 1);
          acc[q][2] = mass(r1, c);
          acc[q][3] = mass(r1, c + 1);
        }
        for (int k0 = 0; k0 < n; k0 += 8) {
          const int ka = k0 + t, kb = ka + 4;
          const bool va = ka < n, vb = kb < n;
          const float ca = (va && d.efc_active[adr + ka]) ? d.efc_D[adr + ka] : 0.f;
          const float cb = (vb && d.efc_active[adr + kb]) ? d.efc_D[adr + kb] : 0.f;
          const float* Ja = J + size_t(va ? ka : 0) * nv;
          const float* Jb = J + size_t(vb ? kb : 0) * nv;
          const FragA a = frag_a((va && r0 < nv) ? Ja[r0] : 0.f, (va && r1 < nv) ? Ja[r1] : 0.f,
                                 (vb && r0 < nv) ? Jb[r0] : 0.f, (vb && r1 < nv) ? Jb[r1] : 0.f);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int c = 8 * (nt0 + q) + g;
            if (nt0 + q < nnt) {
              const FragB b = frag_b((va && c < nv) ? ca * Ja[c] : 0.f, (vb && c < nv) ? cb * Jb[c] : 0.f);
              mma_3xtf32(acc[q], a, b);
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int c = 8 * (nt0 + q) + 2 * t;
#pragma unroll
          for (int e = 0; e < 2; e++) {
            if (r0 < nv && c + e <= r0)
              Hout[(PACKED ? size_t(tri(r0)) : size_t(r0) * ldh) + c + e] = TH(acc[q][e]);
            if (r1 < nv && c + e <= r1)
              Hout[(PACKED ? size_t(tri(r1)) : size_t(r1) * ldh) + c + e] = TH(acc[q][2 + e]);
          }
        }
      }
    }
    __syncthreads();
  }

  // solver.py:176-312
  __device__ void update_gradient() {
    float gd[1] = {0.f};
    for (int i = tid; i < nv; i += NT) {
      const float g = Ma[i] - qfrc_smooth[i] - qfrc_constraint[i];
      grad[i] = g;
      gd[0] += g * g;
    }
    sum<1>(gd);
    grad_dot = gd[0];
    if (m.solver == 1) {  // CG: Mgrad = M^-1 grad
      if (warp == 0) solve_m_world(m, d, w, Mgrad, grad, lane);
      __syncthreads();
      return;
    }
    if (!(reuse && factored && !changed)) {
      if (PREC) {  // H in split TF32 straight into the FP64 tile, factored there in FP64
        assemble_hessian_tc<double, true>(Ld, 0);
        chol_cta_d<NW>(Ld, rdg, nv, warp, lane);
        for (int e = tid; e < nv * nv; e += NT) {  // efc_h keeps the factor (FP32-rounded)
          const int i = e / nv, j = e - i * nv;
          if (j <= i) H[e] = float(Ld[tri(i) + j]);
        }
      } else {
        if (tc) assemble_hessian_tc(H, nv);
        else assemble_hessian();
        chol_cta<NW>(H, nv, nv, T, warp, lane);
      }
      factored = true;
    }
    if (warp == 0) {
      if (PREC) cho_solve_d_warp(Ld, rdg, nv, vd, Mgrad, grad, lane);
    }
    if (!PREC) cho_solve_cta<NW>(H, nv, nv, Mgrad, grad, zv, red, warp, lane);
    __syncthreads();
  }

  // solver.py:737-869 with the iterative (:339-664) or parallel (:667-734) line search
  __device__ void linesearch() {
    mul_m(mv, search);
    {
      float q[3] = {0.f, 0.f, 0.f};
      for (int i = tid; i < nv; i += NT) {
        q[0] += gauss / float(nv);
        q[1] += search[i] * (Ma[i] - qfrc_smooth[i]);
        q[2] += 0.5f * search[i] * mv[i];
      }
      const float z[3] = {0.f, 0.f, 0.f};
      ls_sums<3>(z, q);
      qg[0] = q[0];
      qg[1] = q[1];
      qg[2] = q[2];
    }
    rows_dot(search, d.efc_jv, nullptr);
    for (int k = tid; k < n; k += NT) {
      const int r = adr + k;
      const float jv = d.efc_jv[r], Jaref = d.efc_Jaref[r], D = d.efc_D[r];
      d.efc_quad[3 * r] = 0.5f * Jaref * Jaref * D;
      d.efc_quad[3 * r + 1] = jv * Jaref * D;
      d.efc_quad[3 * r + 2] = 0.5f * jv * jv * D;
    }
    __syncthreads();
    if (m.ls_parallel) {
      int best = 0;
      float bestc = 0.f;
      for (int c = 0; c < m.nlsp; c++) {
        const float a = m.alpha_candidate[c];
        float tt[3] = {0.f, 0.f, 0.f};
        for (int k = tid; k < n; k += NT) {
          const int r = adr + k;
          if (d.efc_Jaref[r] + a * d.efc_jv[r] < 0.f) {
            tt[0] += d.efc_quad[3 * r];
            tt[1] += d.efc_quad[3 * r + 1];
            tt[2] += d.efc_quad[3 * r + 2];
          }
        }
        ls_sums<3>(qg, tt);
        const float cst = a * a * tt[2] + a * tt[1] + tt[0];
        if (c == 0 || cst < bestc) {
          bestc = cst;
          best = c;
        }
      }
      alpha = m.alpha_candidate[best];
    } else {
      const float scale = m.meaninertia * float(max(1, nv));
      gtol = m.tolerance * m.ls_tolerance * sqrtf(search_dot) * scale;
      float p0[3] = {0.f, 0.f, 0.f};
      for (int k = tid; k < n; k += NT) {
        const int r = adr + k;
        if (d.efc_Jaref[r] >= 0.f) continue;
        p0[0] += d.efc_quad[3 * r];
        p0[1] += d.efc_quad[3 * r + 1];
        p0[2] += 2.f * d.efc_quad[3 * r + 2];
      }
      {
        const float base[3] = {qg[0], qg[1], 2.f * qg[2]};
        ls_sums<3>(base, p0);
      }
      // the total cost polynomial's value and derivatives at up to three step sizes at once
      auto totals = [&](int na, const float* al, float (*out)[3]) {
        float acc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int k = tid; k < n; k += NT) {
          const int r = adr + k;
          const float jaref = d.efc_Jaref[r], jv = d.efc_jv[r];
          const float* q = d.efc_quad + 3 * r;
          for (int t = 0; t < na; t++) {
            if (jaref + al[t] * jv < 0.f) {
              float p[3];
              eval_pt3(q, al[t], p);
              acc[3 * t] += p[0];
              acc[3 * t + 1] += p[1];
              acc[3 * t + 2] += p[2];
            }
          }
        }
        float base[9];
        for (int t = 0; t < 3; t++) {
          float gq[3] = {0.f, 0.f, 0.f};
          if (t < na) eval_pt3(qg, al[t], gq);
          base[3 * t] = gq[0];
          base[3 * t + 1] = gq[1];
          base[3 * t + 2] = gq[2];
        }
        ls_sums<9>(base, acc);
        for (int t = 0; t < na; t++) {
          out[t][0] = acc[3 * t];
          out[t][1] = acc[3 * t + 1];
          out[t][2] = acc[3 * t + 2];
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
        done = (!(s1 || s2 || s3) && !(t1 || t2 || t3)) || (lo[1] < 0.f && lo[1] > -gtol) ||
               (hi[1] > 0.f && hi[1] < gtol);
        float a = 0.f;
        const bool improved = lo[0] < p0[0] || hi[0] < p0[0];
        const bool lo_better = lo[0] < hi[0];
        if (improved && lo_better) a = lo_alpha;
        if (improved && !lo_better) a = hi_alpha;
        alpha = a;
      }
    }
    // solver.py:816-841
    for (int i = tid; i < nv; i += NT) {
      qacc[i] += alpha * search[i];
      Ma[i] += alpha * mv[i];
    }
    for (int k = tid; k < n; k += NT) d.efc_Jaref[adr + k] += alpha * d.efc_jv[adr + k];
    __syncthreads();
  }

  // search = -Mgrad (+ beta search for CG); returns search . search
  __device__ void new_search() {
    float sd[1] = {0.f};
    for (int i = tid; i < nv; i += NT) {
      float v = -Mgrad[i];
      if (m.solver == 1) v += beta * search[i];
      search[i] = v;
      sd[0] += v * v;
    }
    sum<1>(sd);
    search_dot = sd[0];
  }

  __device__ void run() {
    const float* ws = d.qacc_warmstart + W(w, nv);
    for (int i = tid; i < nv; i += NT) qacc[i] = ws[i];
    __syncthreads();
    // _create_context (solver.py:26-72)
    cost = __int_as_float(0x7f800000);
    search_dot = 0.f;
    alpha = 0.f;
    gtol = 0.f;
    beta = 0.f;
    qg[0] = qg[1] = qg[2] = 0.f;
    rows_dot(qacc, d.efc_Jaref, d.efc_aref);
    mul_m(Ma, qacc);
    update_constraint();
    update_gradient();
    new_search();
    float* prev_grad = d.efc_prev_grad ? d.efc_prev_grad + W(w, nv) : nullptr;
    float* prev_Mgrad = d.efc_prev_Mgrad ? d.efc_prev_Mgrad + W(w, nv) : nullptr;
    bool done = false;
    for (int it = 0; it < m.iterations && !done; it++) {
      linesearch();
      if (m.solver == 1) {
        for (int i = tid; i < nv; i += NT) {
          prev_grad[i] = grad[i];
          prev_Mgrad[i] = Mgrad[i];
        }
        __syncthreads();
      }
      update_constraint();
      update_gradient();
      if (m.solver == 1) {  // Polak-Ribiere (solver.py:918-970)
        float nd[2] = {0.f, 0.f};
        for (int i = tid; i < nv; i += NT) {
          nd[0] += grad[i] * (Mgrad[i] - prev_Mgrad[i]);
          nd[1] += prev_grad[i] * prev_Mgrad[i];
        }
        sum<2>(nd);
        beta = fmaxf(0.f, nd[0] / fmaxf(kMinVal, nd[1]));
      }
      new_search();
      const float scale = m.meaninertia * float(max(1, nv));
      done = (prev_cost - cost) / scale < m.tolerance || sqrtf(grad_dot) / scale < m.tolerance;
    }
    float* wsw = d.qacc_warmstart + W(w, nv);
    for (int i = tid; i < nv; i += NT) wsw[i] = qacc[i];
    if (tid == 0) {
      if (d.efc_cost) d.efc_cost[w] = cost;
      if (d.efc_prev_cost) d.efc_prev_cost[w] = prev_cost;
      if (d.efc_gauss) d.efc_gauss[w] = gauss;
      if (d.efc_grad_dot) d.efc_grad_dot[w] = grad_dot;
      if (d.efc_search_dot) d.efc_search_dot[w] = search_dot;
      if (d.efc_gtol) d.efc_gtol[w] = gtol;
      if (d.efc_alpha) d.efc_alpha[w] = alpha;
      if (d.efc_beta) d.efc_beta[w] = beta;
      if (d.efc_done) d.efc_done[w] = done ? 1 : 0;
      if (d.efc_solver_niter) d.efc_solver_niter[w] = 0;  // never advanced by the reference
      if (d.efc_quad_gauss) {
        d.efc_quad_gauss[3 * w] = qg[0];
        d.efc_quad_gauss[3 * w + 1] = qg[1];
        d.efc_quad_gauss[3 * w + 2] = qg[2];
      }
    }
    __syncthreads();
  }
};

// One world's solve by the whole CTA; smem: cta_solver_smem_floats(nv, NW) floats
template <int NW, bool PREC>
__device__ void solve_cta(const MjbModel& m, const MjbData& d, int w, float* smem, bool tc) {
  const int nv = m.nv;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  CtaSolver<NW, PREC> s{m, d, w, tid, lane, warp, nv, d.world_efcadr[w], d.world_nefc[w]};
  s.qacc = d.qacc + W(w, nv);
  s.Ma = d.efc_Ma + W(w, nv);
  s.grad = d.efc_grad + W(w, nv);
  s.Mgrad = d.efc_Mgrad + W(w, nv);
  s.search = d.efc_search + W(w, nv);
  s.mv = d.efc_mv + W(w, nv);
  s.qfrc_constraint = d.qfrc_constraint + W(w, nv);
  s.H = d.efc_h + W(w, nv * nv);
  s.qM = d.qM + (m.is_sparse ? W(w, m.nM) : W(w, nv * nv));
  s.qfrc_smooth = d.qfrc_smooth + W(w, nv);
  s.qacc_smooth = d.qacc_smooth + W(w, nv);
  s.red = smem;
  s.T = smem + 32 * NW;
  s.nz = smem + 32 * NW + 32 * 36 + 32 + warp * 2 * round4i(nv);
  s.zv = smem + 32 * NW + 32 * 36 + 32 + NW * 2 * round4i(nv);
  s.Ld = PREC ? reinterpret_cast<double*>(smem + cta_solver_smem_base(nv, NW)) : nullptr;
  s.vd = PREC ? s.Ld + tri(nv) : nullptr;
  s.rdg = PREC ? s.vd + nv : nullptr;
  s.tc = tc;
  s.run();
}

}  // namespace mjb
