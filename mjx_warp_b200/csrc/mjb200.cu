// libmjb200.so: kernels and the C ABI declared in include/mjb200.h.
//
// Three launch forms share the per-world device stages of mjb_world.cuh / mjb_collide.cuh /
// mjb_solver.cuh (one warp per world everywhere):
//  - plain (MJB_FORM_PLAIN): one kernel per reference stage function (mjb_kinematics,
//    mjb_com_pos, ...), data passed between stages through the Data arrays in HBM, the Newton
//    Hessian refactored in every iteration: the reference's launch sequence and algorithm;
//  - chosen (MJB_FORM_CHOSEN, the default): the plain form's stage kernels up to
//    fwd_acceleration (fusing them into one kernel measured slower: the fused collision and
//    constraint stages cost more than the launches they save), then k_solve (the solver, keeping
//    the Hessian factor while the active set is unchanged) and k_integrate (Euler / implicitfast
//    and the finiteness check in one kernel);
//  - single (MJB_FORM_SINGLE): every stage of a world inside one warp of one kernel.
// No entry point allocates memory or synchronises the stream (except mjb_world_status, which
// copies results to the host).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "mjb_deriv.cuh"
#include "mjb_solver.cuh"
#include "mjb_solver_cta.cuh"

// minimum resident CTAs per SM requested for the solver kernels (caps registers per thread at
// 65536 / (128 * MJB_MINB)); with the staged / unstaged solver paths compiled apart, 4 (128
// registers) measured 2 % faster than 5 (96 registers, spilling) on the humanoid at 8192 worlds
#ifndef MJB_MINB
#define MJB_MINB 4
#endif
// the default for the chosen form's FP32 persistent solver (k_solve_queue<false, false, *>),
// which is compiled for 4 and for 5 (MjbTune.solver_ctas_per_sm): on the humanoid at 8192 worlds
// 5 CTAs per SM (96 registers, with spills) measured 0.256 against 0.241 ms early in a run and
// 0.381 against 0.352 ms once the worlds lie on the floor; the plain form's solver and the
// precision solver were slower at 5
#ifndef MJB_MINB_QUEUE
#define MJB_MINB_QUEUE 5
#endif
// minimum resident CTAs per SM of the other stage kernels and of the integrator (64 registers)
#ifndef MJB_MINB_STAGE
#define MJB_MINB_STAGE 8
#endif
#ifndef MJB_MINB_INT
#define MJB_MINB_INT 8
#endif
// lanes per world in the chosen form's tree-recursion stage kernels (8, 16 or 32; 16 measured
// fastest for the humanoid: phase 0 290 us vs 306 at 8 and 323 at 32)
#ifndef MJB_TREE_LANES
#define MJB_TREE_LANES 16
#endif

namespace mjb {

enum Stage {
  S_KINEMATICS, S_COM_POS, S_CRB, S_FACTOR_M, S_TRANSMISSION, S_COM_VEL, S_PASSIVE, S_RNE,
  S_FWD_VELOCITY, S_FWD_ACTUATION, S_FWD_ACCELERATION, S_NXN, S_NARROW, S_MAKE_CONSTRAINT,
  S_SOLVE, S_EULER, S_IMPLICIT, S_QACC_SMOOTH_COPY, S_CHECK, S_SAP
};

constexpr int kDefaultWarps = 4;


// Kernels take the Model / Data views by value as __grid_constant__ parameters: the stages receive
// them by reference, and without the qualifier every thread would copy both structs (~1.6 KB)
// into its local memory whenever a reference reaches a function that is not inlined.

// NaN / Inf check of the integrated state (sets MJB_WS_NONFINITE)
__device__ void check_finite(const MjbModel& m, const MjbData& d, int w, int lane) {
  bool bad = false;
  for (int i = lane; i < m.nq; i += 32) bad |= !isfinite(d.qpos[W(w, m.nq) + i]);
  for (int i = lane; i < m.nv; i += 32) {
    bad |= !isfinite(d.qvel[W(w, m.nv) + i]);
    bad |= !isfinite(d.qacc[W(w, m.nv) + i]);
  }
  if (__any_sync(WARP_FULL, bad) && lane == 0 && d.world_status) atomicOr(d.world_status + w, MJB_WS_NONFINITE);
}

__device__ __forceinline__ void copy_qacc_smooth(const MjbModel& m, const MjbData& d, int w, int lane) {
  for (int i = lane; i < m.nv; i += 32) d.qacc[W(w, m.nv) + i] = d.qacc_smooth[W(w, m.nv) + i];
  __syncwarp();
}

// the solver needs up to 128 registers; every other stage is held to 64 for occupancy
template <int STAGE>
__global__ void __launch_bounds__(128, STAGE == S_SOLVE ? MJB_MINB : MJB_MINB_STAGE)
    k_stage(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, int smem_per_warp) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  float* sm = smem_per_warp ? smem + size_t(threadIdx.x >> 5) * smem_per_warp : nullptr;
  switch (STAGE) {
    case S_KINEMATICS: kinematics(m, d, w, lane); break;
    case S_COM_POS: com_pos(m, d, w, lane); break;
    case S_CRB: crb(m, d, w, lane); break;
    case S_FACTOR_M: factor_m(m, d, w, lane, sm); break;
    case S_TRANSMISSION: transmission(m, d, w, lane); break;
    case S_COM_VEL: com_vel(m, d, w, lane); break;
    case S_PASSIVE: passive(m, d, w, lane); break;
    case S_RNE: rne(m, d, w, lane); break;
    case S_FWD_VELOCITY: fwd_velocity(m, d, w, lane); break;
    case S_FWD_ACTUATION: fwd_actuation(m, d, w, lane); break;
    case S_FWD_ACCELERATION: fwd_acceleration(m, d, w, lane, sm); break;
    case S_NXN: nxn_broadphase(m, d, w, lane); break;
    case S_SAP: sap_broadphase(m, d, w, lane, sm); break;
    case S_NARROW: primitive_narrowphase(m, d, w, lane); break;
    case S_MAKE_CONSTRAINT: make_constraint(m, d, w, lane); break;
    case S_SOLVE: solve(m, d, w, lane, sm, d.efc_h + W(w, m.nv * m.nv)); break;
    case S_EULER: euler(m, d, w, lane, sm); break;
    case S_IMPLICIT: implicit(m, d, w, lane, sm); break;
    case S_QACC_SMOOTH_COPY: copy_qacc_smooth(m, d, w, lane); break;
    case S_CHECK: check_finite(m, d, w, lane); break;
  }
}

// The chosen form's tree-recursion stages (kinematics, com_pos, crb, transmission, fwd_velocity,
// fwd_actuation) with L lanes per world, 32 / L worlds per warp: a BFS level of a few bodies
// keeps the world's lanes busy instead of leaving most of a warp idle, so the warp instructions
// per world drop by up to 32 / L.  The stages' arithmetic does not depend on L.
template <int STAGE, int L>
__global__ void __launch_bounds__(128, MJB_MINB_STAGE)
    k_stage_lanes(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int w = int(t / L), lane = int(t % L);
  if (w >= d.nworld) return;
  switch (STAGE) {
    case S_KINEMATICS: kinematics<L>(m, d, w, lane); break;
    case S_COM_POS: com_pos<L>(m, d, w, lane); break;
    case S_CRB: crb<L>(m, d, w, lane); break;
    case S_TRANSMISSION: transmission<L>(m, d, w, lane); break;
    case S_FWD_VELOCITY: fwd_velocity<L>(m, d, w, lane); break;
    case S_FWD_ACTUATION: fwd_actuation<L>(m, d, w, lane); break;
  }
}

// whole forward (+ integration) of one world per warp; each warp's slice of dynamic shared memory
// holds the solver's workspace, whose leading factor tile also serves the mass-matrix
// factorisations (factor_m, then the integrator)
__global__ void __launch_bounds__(128, MJB_MINB) k_step_fused(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, int integrate,
                                                    int smem_per_warp) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int w = blockIdx.x * (blockDim.x >> 5) + wib;
  if (w >= d.nworld) return;
  const int nv = m.nv;
  float* sm = smem_per_warp ? smem + size_t(wib) * smem_per_warp : nullptr;
  float* hs = d.efc_h + W(w, nv * nv);
  kinematics(m, d, w, lane);
  com_pos(m, d, w, lane);
  crb(m, d, w, lane);
  factor_m(m, d, w, lane, sm);
  collision(m, d, w, lane, sm);
  make_constraint(m, d, w, lane);
  transmission(m, d, w, lane);
  fwd_velocity(m, d, w, lane);
  fwd_actuation(m, d, w, lane);
  fwd_acceleration(m, d, w, lane, sm, true);  // the tile still holds factor_m's factor
  if (d.njmax == 0) copy_qacc_smooth(m, d, w, lane);
  else solve(m, d, w, lane, sm, hs, true);
  if (integrate) {
    if (m.integrator == 0) euler(m, d, w, lane, sm);
    else implicit(m, d, w, lane, sm);
    check_finite(m, d, w, lane);
  }
}

// chosen form: the constraint solver with the Hessian factor kept across iterations; TC: the
// Newton Hessian of up to 32 staged rows assembled on the tensor pipe in split TF32 (hessian_tc;
// always in the precision form, an autotuner choice in the chosen form)
template <bool PREC, bool TC>
__global__ void __launch_bounds__(128, MJB_MINB) k_solve(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, int smem_per_warp) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  float* sm = smem_per_warp ? smem + size_t(threadIdx.x >> 5) * smem_per_warp : nullptr;
  solve<PREC, TC>(m, d, w, lane, sm, d.efc_h + W(w, m.nv * m.nv), true);
}

// The chosen form's solver schedule.  k_order_worlds sorts the worlds by their constraint row
// count, largest first (a counting sort over buckets min(nefc, 255) in one CTA), and resets the
// work queue; k_solve_queue is persistent — as many CTAs as fit on the GPU at once — and each of
// its warps takes the next world in that order from the queue until none is left, so the longest
// solves start first and the last ones to finish are short (longest-processing-time-first).
// Each world's result does not depend on which warp solves it or when.
constexpr int kOrderBuckets = 256;
// Worlds with the same bucket in a warp are counted and placed with one shared-memory atomic per
// bucket (the lanes of a bucket found by __match_any_sync), so the few buckets a model's row
// counts fall into do not serialise thousands of atomics.
// Each thread loads kOrderLoads of its worlds' row counts before it counts or places any of them
// (one load latency per kOrderLoads worlds), and the descending exclusive scan of the buckets is
// a warp scan over eight buckets per lane.
constexpr int kOrderLoads = 8;
__device__ __forceinline__ int order_bucket(const int* nefc, int w, int nworld) {
  return w < nworld ? min(max(nefc[w], 0), kOrderBuckets - 1) : -1;
}
__global__ void __launch_bounds__(1024) k_order_worlds(const int* nefc, int* order, int* queue,
                                                      int nworld) {
  __shared__ int cnt[kOrderBuckets];
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int chunk = kOrderLoads * blockDim.x;  // worlds per pass of the whole block (warp-uniform)
  for (int b = threadIdx.x; b < kOrderBuckets; b += blockDim.x) cnt[b] = 0;
  __syncthreads();
  for (int w0 = 0; w0 < nworld; w0 += chunk) {
    int bk[kOrderLoads];
#pragma unroll
    for (int j = 0; j < kOrderLoads; j++) bk[j] = order_bucket(nefc, w0 + j * blockDim.x + threadIdx.x, nworld);
#pragma unroll
    for (int j = 0; j < kOrderLoads; j++) {
      const unsigned peers = __match_any_sync(WARP_FULL, bk[j]);
      if (bk[j] >= 0 && (peers & below) == 0) atomicAdd(&cnt[bk[j]], __popc(peers));
    }
  }
  __syncthreads();
  static_assert(kOrderBuckets == 32 * 8, "eight buckets per lane of the scanning warp");
  if (threadIdx.x < 32) {  // lane l: buckets 255 - 8 l .. 248 - 8 l (largest row counts first)
    int c[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      c[j] = cnt[kOrderBuckets - 1 - 8 * lane - j];
      sum += c[j];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(WARP_FULL, incl, o);
      if (lane >= o) incl += t;
    }
    int run = incl - sum;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      cnt[kOrderBuckets - 1 - 8 * lane - j] = run;
      run += c[j];
    }
    if (lane == 0) *queue = 0;
  }
  __syncthreads();
  for (int w0 = 0; w0 < nworld; w0 += chunk) {
    int bk[kOrderLoads];
#pragma unroll
    for (int j = 0; j < kOrderLoads; j++) bk[j] = order_bucket(nefc, w0 + j * blockDim.x + threadIdx.x, nworld);
#pragma unroll
    for (int j = 0; j < kOrderLoads; j++) {
      const int b = bk[j];
      const unsigned peers = __match_any_sync(WARP_FULL, b);
      const int leader = __ffs(peers) - 1;
      int base = 0;
      if (b >= 0 && lane == leader) base = atomicAdd(&cnt[b], __popc(peers));
      base = __shfl_sync(WARP_FULL, base, leader);
      if (b >= 0) order[base + __popc(peers & below)] = w0 + j * blockDim.x + threadIdx.x;
    }
  }
}

template <bool PREC, bool TC, int MINB>
__global__ void __launch_bounds__(128, MINB) k_solve_queue(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, int smem_per_warp) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  float* sm = smem_per_warp ? smem + size_t(threadIdx.x >> 5) * smem_per_warp : nullptr;
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(d.work_queue, 1);
    idx = __shfl_sync(WARP_FULL, idx, 0);
    if (idx >= d.nworld) break;
    const int w = d.world_order[idx];
    solve<PREC, TC>(m, d, w, lane, sm, d.efc_h + W(w, m.nv * m.nv), true);
  }
}

// chosen form, models with nv > 32: one CTA of NW warps per world (mjb_solver_cta.cuh),
// persistent over the work queue in k_order_worlds' order when the Data has the schedule arrays,
// else one CTA per world in index order
template <int NW, bool PREC>
__global__ void __launch_bounds__(NW * 32, NW >= 16 ? 1 : (NW >= 8 ? 2 : (NW >= 4 ? 4 : 8)))
    k_solve_cta(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, int tc) {
  extern __shared__ __align__(16) float smem[];
  __shared__ int s_idx;
  if (!d.work_queue) {
    if (int(blockIdx.x) < d.nworld) solve_cta<NW, PREC>(m, d, blockIdx.x, smem, tc != 0);
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) s_idx = atomicAdd(d.work_queue, 1);
    __syncthreads();
    const int idx = s_idx;
    __syncthreads();
    if (idx >= d.nworld) break;
    solve_cta<NW, PREC>(m, d, d.world_order[idx], smem, tc != 0);
  }
}

// chosen form: integration (forward.py:165-405) and the finiteness check
__global__ void __launch_bounds__(128, MJB_MINB_INT) k_integrate(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, int tile_per_warp) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  float* tile = smem + size_t(threadIdx.x >> 5) * tile_per_warp;
  if (m.integrator == 0) euler(m, d, w, lane, tile);
  else implicit(m, d, w, lane, tile);
  check_finite(m, d, w, lane);
}

// finite-difference transition Jacobians (mjb_deriv.cuh): one warp per perturbed slot
__global__ void k_fd_perturb(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData b,
                             const __grid_constant__ MjbData p, float eps, int flags) {
  const int lane = threadIdx.x & 31;
  const int pw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pw >= p.nworld) return;
  const int centered = flags & kFdCentered;
  const int K = fd_slots(m, flags), w = pw / K, k = pw - w * K;
  const int col = k == 0 ? -1 : (centered ? (k - 1) >> 1 : k - 1);
  const float delta = (centered && ((k - 1) & 1)) ? -eps : eps;
  fd_perturb_world(m, b, p, w, pw, col, delta, lane);
}
// one warp per (base world, column)
__global__ void k_fd_jacobian(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData p,
                              int nworld, float eps, int flags, float* A, float* B) {
  const int lane = threadIdx.x & 31;
  const long long t = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int ncol = fd_ncol(m, flags);
  if (t >= (long long)nworld * ncol) return;
  const int w = int(t / ncol), col = int(t - (long long)w * ncol);
  fd_column(m, p, w, col, flags, eps, A, B, lane);
}
// one warp per world; per_warp floats of dynamic shared memory per warp (step_vjp_floats)
__global__ void __launch_bounds__(128) k_step_vjp(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d,
                                                  const float* lam, const float* qvel_prev,
                                                  float* grad_ctrl, float* grad_qvel,
                                                  float* grad_qpos, int per_warp) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  step_vjp_world(m, d, w, lane, lam, qvel_prev, grad_ctrl, grad_qvel, grad_qpos,
                 smem + size_t(threadIdx.x >> 5) * per_warp);
}
// one warp per world
__global__ void k_transition_vjp(const __grid_constant__ MjbModel m, int nworld, const float* A,
                                 const float* B, const float* lam, float* lam_out, float* grad_ctrl) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= nworld) return;
  transition_vjp_world(m, A, B, lam, lam_out, grad_ctrl, w, lane);
}

// zero the flat-array counters and (optionally) the world status words
__global__ void k_reset(int* a, int* b, int* c, uint32_t* status, int nworld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    if (a) *a = 0;
    if (b) *b = 0;
    if (c) *c = 0;
  }
  if (status && i < nworld) status[i] = 0u;
}

// Rebuild a per-world index (first row, row count) of a flat, worldid-tagged array.
__global__ void k_index_clear(int* adr, int* cnt, int nworld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nworld) {
    adr[i] = 0x7fffffff;
    cnt[i] = 0;
  }
}
__global__ void k_index_rows(const int* worldid, const int* counter, int cap, int* adr, int* cnt,
                             int nworld) {
  const int n = min(*counter, cap);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int w = worldid[r];
    if (w < 0 || w >= nworld) continue;
    atomicMin(adr + w, r);
    atomicAdd(cnt + w, 1);
  }
}
// Checks that each world's rows are contiguous; a split world gets MJB_WS_ROWS_SPLIT and no rows.
__global__ void k_index_fix(const int* worldid, int* adr, int* cnt, uint32_t* status, int nworld) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= nworld) return;
  const int n = cnt[w];
  if (n == 0) {
    if (lane == 0) adr[w] = 0;
    return;
  }
  const int a = adr[w];
  bool bad = false;
  for (int k = lane; k < n; k += 32) bad |= worldid[a + k] != w;
  if (__any_sync(WARP_FULL, bad) && lane == 0) {
    cnt[w] = 0;
    adr[w] = 0;
    if (status) atomicOr(status + w, MJB_WS_ROWS_SPLIT);
  }
}

// support.py:35-137 — res = M vec per world unless skip[w]
__global__ void k_mul_m(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, float* res, const float* vec,
                        const uint8_t* skip) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  if (skip && skip[w]) return;
  if (m.is_sparse) mul_m_sparse(m, d.qM + W(w, m.nM), res + W(w, m.nv), vec + W(w, m.nv), lane);
  else mul_m_world(d.qM + W(w, m.nv * m.nv), m.nv, res + W(w, m.nv), vec + W(w, m.nv), lane);
}
__global__ void k_solve_m(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, float* x, const float* y) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  solve_m_world(m, d, w, x + W(w, m.nv), y + W(w, m.nv), lane);
}
__global__ void k_xfrc(const __grid_constant__ MjbModel m, const __grid_constant__ MjbData d, float* qfrc) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= d.nworld) return;
  xfrc_accumulate(m, d, w, qfrc + W(w, m.nv), lane);
}

}  // namespace mjb

using namespace mjb;

namespace {

inline int grid_for(int nworld, int warps) { return (nworld + warps - 1) / warps; }

inline int finish() {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MJB_OK : MJB_ERR_LAUNCH;
}

// implicitfast needs the dense mass matrix (the reference asserts it, forward.py:268)
inline bool implicit_unsupported(const MjbModel* m) { return m->is_sparse && m->integrator != 0; }

// the precision form: dense mass matrix with tree blocks of up to 32 dofs (the FP64 block
// factor-solves use a 32-row tile); for nv > 32 the Hessian's packed FP64 factor must fit in one
// CTA's shared memory (227 KB: nv up to about 230)
int precision_supported(const MjbModel* m) {
  if (m->is_sparse || m->block_max > 32) return MJB_ERR_UNSUPPORTED;
  if (m->nv > 32 && size_t(cta_solver_smem_floats(m->nv, 16, true)) * sizeof(float) > 227 * 1024)
    return MJB_ERR_SCRATCH;
  return MJB_OK;
}

inline int check(const MjbModel* m, const MjbData* d) {
  if (!m || !d) return MJB_ERR_ARG;
  if (d->nworld <= 0) return d->nworld == 0 ? MJB_OK : MJB_ERR_ARG;
  if (m->cone != 0) return MJB_ERR_UNSUPPORTED;
  return MJB_OK;
}

// The Data fields each stage reads or writes, given the model's sizes and options: a stage
// launched with one of them null returns MJB_ERR_ARG instead of faulting on the device.
// Fields a stage checks for null itself (world_status, the solver's optional per-world outputs,
// contact_solreffriction, world_order / work_queue) are not required.
#define MJB_REQ(cond, field) \
  if ((cond) && !d->field) return MJB_ERR_ARG
int stage_fields(int stage, const MjbModel* m, const MjbData* d) {
  const bool nv = m->nv > 0, nq = m->nq > 0, nj = m->njnt > 0, ng = m->ngeom > 0,
             ns = m->nsite > 0, nu = m->nu > 0, na = m->na > 0;
  const bool con = d->nconmax > 0, efc = d->njmax > 0;
  switch (stage) {
    case S_KINEMATICS:
      MJB_REQ(nq, qpos); MJB_REQ(true, xpos); MJB_REQ(true, xquat); MJB_REQ(true, xmat);
      MJB_REQ(true, xipos); MJB_REQ(true, ximat); MJB_REQ(nj, xanchor); MJB_REQ(nj, xaxis);
      MJB_REQ(ng, geom_xpos); MJB_REQ(ng, geom_xmat); MJB_REQ(ns, site_xpos); MJB_REQ(ns, site_xmat);
      break;
    case S_COM_POS:
      MJB_REQ(true, subtree_com); MJB_REQ(true, cinert); MJB_REQ(nv, cdof); MJB_REQ(true, xipos);
      MJB_REQ(true, ximat); MJB_REQ(true, xmat); MJB_REQ(nj, xanchor); MJB_REQ(nj, xaxis);
      break;
    case S_CRB:
      MJB_REQ(true, crb); MJB_REQ(true, cinert); MJB_REQ(nv, cdof); MJB_REQ(nv, qM);
      break;
    case S_FACTOR_M:
      MJB_REQ(nv, qM); MJB_REQ(nv, qLD); MJB_REQ(nv && m->is_sparse, qLDiagInv);
      break;
    case S_TRANSMISSION:
      MJB_REQ(nu, actuator_length); MJB_REQ(nu, actuator_moment); MJB_REQ(nu && nq, qpos);
      break;
    case S_FWD_VELOCITY:
      MJB_REQ(nu, actuator_velocity); MJB_REQ(nu, actuator_moment);
      [[fallthrough]];
    case S_COM_VEL:
    case S_PASSIVE:
    case S_RNE:
      MJB_REQ(true, cvel); MJB_REQ(nv, cdof_dot); MJB_REQ(nv, cdof); MJB_REQ(nv, qvel);
      MJB_REQ(nq, qpos); MJB_REQ(nv, qfrc_spring); MJB_REQ(nv, qfrc_damper);
      MJB_REQ(nv, qfrc_passive); MJB_REQ(true, rne_cacc); MJB_REQ(true, rne_cfrc);
      MJB_REQ(nv, qfrc_bias); MJB_REQ(true, cinert);
      break;
    case S_FWD_ACTUATION:
      MJB_REQ(nv, qfrc_actuator); MJB_REQ(nu, actuator_force); MJB_REQ(nu, ctrl);
      MJB_REQ(nu, actuator_length); MJB_REQ(nu, actuator_velocity); MJB_REQ(nu, actuator_moment);
      MJB_REQ(na, act); MJB_REQ(na, act_dot);
      break;
    case S_FWD_ACCELERATION:
      MJB_REQ(nv, qfrc_smooth); MJB_REQ(nv, qacc_smooth); MJB_REQ(nv, qfrc_applied);
      MJB_REQ(nv, qfrc_bias); MJB_REQ(nv, qfrc_passive); MJB_REQ(nv, qfrc_actuator);
      MJB_REQ(nv, qM); MJB_REQ(nv, qLD); MJB_REQ(nv && m->is_sparse, qLDiagInv);
      MJB_REQ(true, xfrc_applied);
      break;
    case S_NXN:
    case S_SAP:
      MJB_REQ(con, ncollision); MJB_REQ(con, collision_pair); MJB_REQ(con, collision_worldid);
      MJB_REQ(true, world_pairadr); MJB_REQ(true, world_npair); MJB_REQ(ng, geom_xpos);
      MJB_REQ(ng, geom_xmat);
      break;
    case S_NARROW:
      MJB_REQ(con, collision_pair); MJB_REQ(con, ncon); MJB_REQ(true, world_pairadr);
      MJB_REQ(true, world_npair); MJB_REQ(true, world_conadr); MJB_REQ(true, world_ncon);
      MJB_REQ(con, contact_dist); MJB_REQ(con, contact_pos); MJB_REQ(con, contact_frame);
      MJB_REQ(con, contact_geom); MJB_REQ(con, contact_worldid); MJB_REQ(con, contact_dim);
      MJB_REQ(con, contact_solref); MJB_REQ(con, contact_includemargin);
      MJB_REQ(con, contact_friction); MJB_REQ(con, contact_solimp);
      MJB_REQ(ng, geom_xpos); MJB_REQ(ng, geom_xmat);
      break;
    case S_MAKE_CONSTRAINT:
      MJB_REQ(efc, nefc); MJB_REQ(efc, efc_worldid); MJB_REQ(efc, efc_J); MJB_REQ(efc, efc_pos);
      MJB_REQ(efc, efc_margin); MJB_REQ(efc, efc_D); MJB_REQ(efc, efc_aref);
      MJB_REQ(true, world_efcadr); MJB_REQ(true, world_nefc); MJB_REQ(true, world_conadr);
      MJB_REQ(true, world_ncon); MJB_REQ(con, contact_dist); MJB_REQ(con, contact_pos);
      MJB_REQ(con, contact_frame); MJB_REQ(con, contact_geom); MJB_REQ(con, contact_dim);
      MJB_REQ(con, contact_solref); MJB_REQ(con, contact_includemargin);
      MJB_REQ(con, contact_friction); MJB_REQ(con, contact_solimp); MJB_REQ(nv, cdof);
      MJB_REQ(true, subtree_com); MJB_REQ(nq, qpos); MJB_REQ(nv, qvel);
      break;
    case S_SOLVE: {
      const bool generic = m->nv > 32 || m->is_sparse;
      MJB_REQ(efc, efc_D); MJB_REQ(efc, efc_J); MJB_REQ(efc, efc_Jaref); MJB_REQ(efc, efc_aref);
      MJB_REQ(efc, efc_force); MJB_REQ(efc, efc_active); MJB_REQ(efc, efc_jv);
      MJB_REQ(efc, efc_quad); MJB_REQ(nv, efc_Ma); MJB_REQ(nv, efc_grad); MJB_REQ(nv, efc_Mgrad);
      MJB_REQ(nv, efc_search); MJB_REQ(nv, efc_mv); MJB_REQ(nv, qfrc_constraint); MJB_REQ(nv, qacc);
      MJB_REQ(nv, qacc_warmstart); MJB_REQ(nv, qfrc_smooth); MJB_REQ(nv, qacc_smooth);
      MJB_REQ(nv, qM); MJB_REQ(true, world_efcadr); MJB_REQ(true, world_nefc);
      MJB_REQ(nv && generic && m->solver == 2, efc_h);
      MJB_REQ(nv && generic && m->solver == 1, efc_prev_grad);
      MJB_REQ(nv && generic && m->solver == 1, efc_prev_Mgrad);
      MJB_REQ(nv && m->solver == 1, qLD); MJB_REQ(nv && m->solver == 1 && m->is_sparse, qLDiagInv);
      break;
    }
    case S_EULER: {
      const bool damp = !(m->disableflags & DSBL_EULERDAMP);
      MJB_REQ(nv, qacc); MJB_REQ(nv, qvel); MJB_REQ(nq, qpos);
      MJB_REQ(nv && damp, qacc_integration); MJB_REQ(nv && damp, qfrc_smooth);
      MJB_REQ(nv && damp, qfrc_constraint); MJB_REQ(nv && damp, qM);
      MJB_REQ(nv && damp, qLD_integration);
      break;
    }
    case S_IMPLICIT: {
      const bool act = !(m->disableflags & DSBL_ACTUATION) && m->actuator_affine_bias_gain;
      MJB_REQ(nv, qacc); MJB_REQ(nv, qvel); MJB_REQ(nq, qpos); MJB_REQ(nv, qacc_integration);
      MJB_REQ(nv, qfrc_smooth); MJB_REQ(nv, qfrc_constraint); MJB_REQ(nv, qM);
      MJB_REQ(nv, qM_integration); MJB_REQ(nv, qLD_integration); MJB_REQ(nv, qfrc_integration);
      MJB_REQ(act, act_vel_integration); MJB_REQ(act, actuator_moment); MJB_REQ(act, ctrl);
      break;
    }
    case S_QACC_SMOOTH_COPY:
      MJB_REQ(nv, qacc); MJB_REQ(nv, qacc_smooth);
      break;
    default:
      break;
  }
  return MJB_OK;
}
#undef MJB_REQ

// the fields of the stages of one phase of a step: 0 = fwd_position .. fwd_acceleration,
// 1 = the solver (or the qacc_smooth copy without rows), 2 = the integrator
int phase_fields(const MjbModel* m, const MjbData* d, int phase) {
  static const int kForward[] = {S_KINEMATICS, S_COM_POS, S_CRB, S_FACTOR_M, S_TRANSMISSION,
                                 S_FWD_VELOCITY, S_FWD_ACTUATION, S_FWD_ACCELERATION, S_NXN,
                                 S_NARROW, S_MAKE_CONSTRAINT};
  int rc;
  if (phase == 0) {
    for (int st : kForward)
      if ((rc = stage_fields(st, m, d))) return rc;
    return MJB_OK;
  }
  if (phase == 1) return stage_fields(d->njmax > 0 ? S_SOLVE : S_QACC_SMOOTH_COPY, m, d);
  return stage_fields(m->integrator == 0 ? S_EULER : S_IMPLICIT, m, d);
}

// shared memory per warp (floats) for the solver workspace when nv <= 32, else a factor tile for
// the tree blocks of up to 32 dofs (the generic solver keeps its Hessian in efc_h)
int solver_smem_per_warp(const MjbModel* m) {
  return m->nv <= 32 ? int(solver_smem_floats(m->nv))
                     : std::max(tile_floats(m->nv), generic_nz_floats(m->nv));
}

// the single form's warp slice also serves the sweep-and-prune broadphase (ngeom > 100)
int fused_smem_per_warp(const MjbModel* m) {
  const int spw = solver_smem_per_warp(m);
  return m->ngeom > 100 ? std::max(spw, sap_smem_floats(m->ngeom)) : spw;
}

// dynamic shared memory a CTA of kDefaultWarps warps may use (the opt-in limit of sm_100)
constexpr size_t kMaxSmemPerCta = 227 * 1024;

// opts a kernel in to more than 48 KB of dynamic shared memory (once per kernel, device and size)
constexpr int kSmemDevices = 64;
template <typename K>
void allow_smem(K kernel, size_t bytes, size_t (&configured)[kSmemDevices]) {
  if (bytes <= 48 * 1024) return;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kSmemDevices || bytes > configured[dev]) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (dev >= 0 && dev < kSmemDevices) configured[dev] = bytes;
  }
}

// CTAs of `kernel` resident on the whole GPU at once for blocks of `threads` threads and `smem`
// bytes, queried once per (device, kernel, block size, shared-memory size)
template <typename K>
int resident_ctas(K kernel, int threads, size_t smem) {
  struct Entry {
    int dev;
    const void* fn;
    int threads;
    size_t smem;
    int ctas;
  };
  static Entry cache[64];
  static int used = 0;
  static std::mutex mu;
  int dev = 0;
  cudaGetDevice(&dev);
  const void* fn = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < used; i++)
    if (cache[i].dev == dev && cache[i].fn == fn && cache[i].threads == threads &&
        cache[i].smem == smem)
      return cache[i].ctas;
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  const int n = std::max(1, sms * std::max(1, per_sm));
  if (used < 64) cache[used++] = Entry{dev, fn, threads, smem, n};
  return n;
}

template <int STAGE>
int launch_stage(const MjbModel* m, const MjbData* d, cudaStream_t s) {
  if (int rc = stage_fields(STAGE, m, d)) return rc;
  const int warps = kDefaultWarps;
  int spw = 0;
  size_t bytes = 0;
  if (STAGE == S_SOLVE) spw = m->nv <= 32 ? int(solver_smem_floats(m->nv)) : generic_nz_floats(m->nv);
  if (STAGE == S_FACTOR_M || STAGE == S_FWD_ACCELERATION || STAGE == S_EULER || STAGE == S_IMPLICIT)
    spw = tile_floats(m->nv) + (m->precision ? prec_tile_floats(m->nv) : 0);
  if (STAGE == S_SAP) spw = sap_smem_floats(m->ngeom);
  if (spw) {
    bytes = size_t(spw) * warps * sizeof(float);
    if (bytes > kMaxSmemPerCta) return MJB_ERR_SCRATCH;
    static size_t configured[kSmemDevices];
    allow_smem(k_stage<STAGE>, bytes, configured);
  }
  k_stage<STAGE><<<grid_for(d->nworld, warps), 32 * warps, bytes, s>>>(*m, *d, spw);
  return finish();
}

// the reference's broadphase choice (collision_driver.py:537-540)
int launch_broadphase(const MjbModel* m, const MjbData* d, cudaStream_t s) {
  return m->ngeom > 100 ? launch_stage<S_SAP>(m, d, s) : launch_stage<S_NXN>(m, d, s);
}

// a tree-recursion stage with `lanes` (8, 16 or 32) lanes per world
template <int STAGE, int L>
int launch_lanes_l(const MjbModel* m, const MjbData* d, cudaStream_t s) {
  const long long threads = (long long)d->nworld * L;
  k_stage_lanes<STAGE, L><<<int((threads + 127) / 128), 128, 0, s>>>(*m, *d);
  return finish();
}
template <int STAGE>
int launch_lanes(const MjbModel* m, const MjbData* d, cudaStream_t s, int lanes) {
  if (lanes == 8) return launch_lanes_l<STAGE, 8>(m, d, s);
  if (lanes == 32) return launch_lanes_l<STAGE, 32>(m, d, s);
  return launch_lanes_l<STAGE, 16>(m, d, s);
}

// The chosen form's launch parameters: lanes per world of the tree-recursion stages and warps per
// CTA of the persistent solver.  mjb_autotune measures them per device for a model's nv and a
// Data's rows-per-world capacity (njmax / nworld, the caller's sizing of its contact density);
// without a tuned entry the defaults below apply.
constexpr int kCtaSolverMinNv = 128;
struct ChosenCfg {
  int lanes = MJB_TREE_LANES;
  int warps = kDefaultWarps;
  int cta_warps = 4;  // warps per world of the solver for nv > 32 (0: one warp per world)
  int hessian_tc = 0; // nv <= 32: Newton Hessian on the tensor pipe (split TF32) instead of FMAs
  int solver_ctas = MJB_MINB_QUEUE;  // CTAs per SM of the FP32 FMA-Hessian persistent solver (4, 5)
};
struct TuneEntry {
  int dev, nv, cap;
  ChosenCfg cfg;
};
std::mutex g_tune_mutex;
TuneEntry g_tune[64];
int g_ntune = 0;

inline int rows_capacity(const MjbData* d) { return d->nworld > 0 ? d->njmax / d->nworld : 0; }

ChosenCfg chosen_cfg(const MjbModel* m, const MjbData* d) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int cap = rows_capacity(d);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  for (int i = 0; i < g_ntune; i++)
    if (g_tune[i].dev == dev && g_tune[i].nv == m->nv && g_tune[i].cap == cap) return g_tune[i].cfg;
  ChosenCfg c;
  // untuned: the CTA solver for large trees of dofs (measured faster from the 384-dof bin, slower
  // for the 123-dof humanoid with spheres), one warp per world below
  c.cta_warps = m->nv > kCtaSolverMinNv ? 4 : 0;
  return c;
}

void store_cfg(const MjbModel* m, const MjbData* d, ChosenCfg cfg) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int cap = rows_capacity(d);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  for (int i = 0; i < g_ntune; i++)
    if (g_tune[i].dev == dev && g_tune[i].nv == m->nv && g_tune[i].cap == cap) {
      g_tune[i].cfg = cfg;
      return;
    }
  if (g_ntune < 64) g_tune[g_ntune++] = TuneEntry{dev, m->nv, cap, cfg};
}

void reset_counters(const MjbData* d, bool pairs, bool contacts, bool efc, bool status,
                    cudaStream_t s) {
  const int n = status ? d->nworld : 1;
  k_reset<<<(n + 255) / 256, 256, 0, s>>>(pairs ? d->ncollision : nullptr,
                                            contacts ? d->ncon : nullptr, efc ? d->nefc : nullptr,
                                            status ? d->world_status : nullptr, d->nworld);
}

void rebuild_index(const int* worldid, const int* counter, int cap, int* adr, int* cnt,
                   const MjbData* d, cudaStream_t s) {
  k_index_clear<<<(d->nworld + 255) / 256, 256, 0, s>>>(adr, cnt, d->nworld);
  k_index_rows<<<148 * 4, 256, 0, s>>>(worldid, counter, cap, adr, cnt, d->nworld);
  k_index_fix<<<grid_for(d->nworld, 4), 128, 0, s>>>(worldid, adr, cnt, d->world_status, d->nworld);
}

// the chosen form's world ordering for its persistent solvers (k_order_worlds), launched in
// phase 0 once the rows are made, so that it overlaps the other forward chains' tails
inline void order_worlds(const MjbData* d, cudaStream_t s) {
  if (d->njmax > 0 && d->world_order && d->work_queue && d->world_nefc)
    k_order_worlds<<<1, 1024, 0, s>>>(d->world_nefc, d->world_order, d->work_queue, d->nworld);
}

int run_forward_plain_nosolve(const MjbModel* m, const MjbData* d, cudaStream_t s) {
  int rc;
  if ((rc = launch_stage<S_KINEMATICS>(m, d, s))) return rc;
  if ((rc = launch_stage<S_COM_POS>(m, d, s))) return rc;
  if ((rc = launch_stage<S_CRB>(m, d, s))) return rc;
  if ((rc = launch_stage<S_FACTOR_M>(m, d, s))) return rc;
  reset_counters(d, true, true, true, false, s);
  if ((rc = launch_broadphase(m, d, s))) return rc;
  if ((rc = launch_stage<S_NARROW>(m, d, s))) return rc;
  if ((rc = launch_stage<S_MAKE_CONSTRAINT>(m, d, s))) return rc;
  if ((rc = launch_stage<S_TRANSMISSION>(m, d, s))) return rc;
  if ((rc = launch_stage<S_FWD_VELOCITY>(m, d, s))) return rc;
  if ((rc = launch_stage<S_FWD_ACTUATION>(m, d, s))) return rc;
  if ((rc = launch_stage<S_FWD_ACCELERATION>(m, d, s))) return rc;
  if (d->njmax == 0) return launch_stage<S_QACC_SMOOTH_COPY>(m, d, s);
  return MJB_OK;
}

// The chosen form's fwd_position .. fwd_acceleration as a fork-join over three chains that share
// no outputs: after kinematics and com_pos on the caller's stream, crb -> factor_m and
// transmission -> fwd_velocity -> fwd_actuation run on two auxiliary streams while collision and
// make_constraint continue on the caller's stream; fwd_acceleration joins them.  Each chain's
// kernels fill the tails of the others'.  The auxiliary streams and events are created once per
// device (no memory is allocated) and the enqueue sequence is serialised by a mutex; inside a
// stream capture the fork and join become graph edges.
struct StageFork {
  cudaStream_t aux[2] = {nullptr, nullptr};
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  bool ready = false;
};
std::mutex g_fork_mutex;
StageFork g_fork[kSmemDevices];

int run_forward_fork(const MjbModel* m, const MjbData* d, cudaStream_t s, int lanes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kSmemDevices) {
    const int rc = run_forward_plain_nosolve(m, d, s);
    if (!rc) order_worlds(d, s);
    return rc;
  }
  std::lock_guard<std::mutex> lock(g_fork_mutex);
  StageFork& f = g_fork[dev];
  if (!f.ready) {
    for (auto& a : f.aux)
      if (cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking) != cudaSuccess) return MJB_ERR_LAUNCH;
    for (auto& e : f.ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MJB_ERR_LAUNCH;
    f.ready = true;
  }
  int rc;
  if ((rc = launch_lanes<S_KINEMATICS>(m, d, s, lanes))) return rc;
  if ((rc = launch_lanes<S_COM_POS>(m, d, s, lanes))) return rc;
  if (cudaEventRecord(f.ev[0], s) != cudaSuccess) return MJB_ERR_LAUNCH;
  for (auto& a : f.aux)
    if (cudaStreamWaitEvent(a, f.ev[0], 0) != cudaSuccess) return MJB_ERR_LAUNCH;
  int rc0 = launch_lanes<S_CRB>(m, d, f.aux[0], lanes);
  if (!rc0) rc0 = launch_stage<S_FACTOR_M>(m, d, f.aux[0]);
  int rc1 = launch_lanes<S_TRANSMISSION>(m, d, f.aux[1], lanes);
  if (!rc1) rc1 = launch_lanes<S_FWD_VELOCITY>(m, d, f.aux[1], lanes);
  if (!rc1) rc1 = launch_lanes<S_FWD_ACTUATION>(m, d, f.aux[1], lanes);
  reset_counters(d, true, true, true, false, s);
  int rc2 = launch_broadphase(m, d, s);
  if (!rc2) rc2 = launch_stage<S_NARROW>(m, d, s);
  if (!rc2) rc2 = launch_stage<S_MAKE_CONSTRAINT>(m, d, s);
  if (!rc2) order_worlds(d, s);
  // join even after a failed launch, so a capture is never left with unjoined streams
  if (cudaEventRecord(f.ev[1], f.aux[0]) != cudaSuccess) return MJB_ERR_LAUNCH;
  if (cudaEventRecord(f.ev[2], f.aux[1]) != cudaSuccess) return MJB_ERR_LAUNCH;
  if (cudaStreamWaitEvent(s, f.ev[1], 0) != cudaSuccess) return MJB_ERR_LAUNCH;
  if (cudaStreamWaitEvent(s, f.ev[2], 0) != cudaSuccess) return MJB_ERR_LAUNCH;
  if (rc0 || rc1 || rc2) return rc0 ? rc0 : (rc1 ? rc1 : rc2);
  if ((rc = launch_stage<S_FWD_ACCELERATION>(m, d, s))) return rc;
  if (d->njmax == 0) return launch_stage<S_QACC_SMOOTH_COPY>(m, d, s);
  return MJB_OK;
}

int run_forward_plain(const MjbModel* m, const MjbData* d, cudaStream_t s) {
  int rc;
  if ((rc = run_forward_plain_nosolve(m, d, s))) return rc;
  return d->njmax == 0 ? MJB_OK : launch_stage<S_SOLVE>(m, d, s);
}

// the chosen form's solver launch: k_order_worlds + the persistent k_solve_queue when the Data has
// the schedule arrays, else one warp per world (k_solve); PREC selects the precision form's solver
template <int NW, bool PREC>
void launch_solver_cta(const MjbModel* m, const MjbData* d, int tc, cudaStream_t s) {
  const size_t bytes = size_t(cta_solver_smem_floats(m->nv, NW, PREC)) * sizeof(float);
  static size_t conf[kSmemDevices];
  allow_smem(k_solve_cta<NW, PREC>, bytes, conf);
  if (d->world_order && d->work_queue && d->world_nefc) {
    const int ctas = resident_ctas(k_solve_cta<NW, PREC>, 32 * NW, bytes);  // ordered in phase 0
    k_solve_cta<NW, PREC><<<std::min(ctas, d->nworld), 32 * NW, bytes, s>>>(*m, *d, tc);
  } else {
    MjbData dd = *d;
    dd.work_queue = nullptr;
    k_solve_cta<NW, PREC><<<d->nworld, 32 * NW, bytes, s>>>(*m, dd, tc);
  }
}

template <bool PREC, bool TC, int MINB>
void launch_solver_queue(const MjbModel* m, const MjbData* d, int qw, int spw, cudaStream_t s) {
  const size_t qbytes = size_t(spw) * qw * sizeof(float);
  static size_t conf_queue[kSmemDevices];
  allow_smem(k_solve_queue<PREC, TC, MINB>, size_t(spw) * kDefaultWarps * sizeof(float), conf_queue);
  const int ctas = resident_ctas(k_solve_queue<PREC, TC, MINB>, 32 * qw, qbytes);  // ordered in phase 0
  k_solve_queue<PREC, TC, MINB><<<std::min(ctas, grid_for(d->nworld, qw)), 32 * qw, qbytes, s>>>(*m, *d, spw);
}

template <bool PREC, bool TC>
void launch_solver_warp(const MjbModel* m, const MjbData* d, const ChosenCfg& cfg, int spw,
                        cudaStream_t s) {
  if (d->world_order && d->work_queue && d->world_nefc) {
    if constexpr (PREC || TC) {
      launch_solver_queue<PREC, TC, MJB_MINB>(m, d, cfg.warps, spw, s);
    } else {
      if (cfg.solver_ctas == 4) launch_solver_queue<PREC, TC, 4>(m, d, cfg.warps, spw, s);
      else launch_solver_queue<PREC, TC, 5>(m, d, cfg.warps, spw, s);
    }
  } else {
    const size_t bytes = size_t(spw) * kDefaultWarps * sizeof(float);
    static size_t conf_solve[kSmemDevices];
    allow_smem(k_solve<PREC, TC>, bytes, conf_solve);
    k_solve<PREC, TC><<<grid_for(d->nworld, kDefaultWarps), 32 * kDefaultWarps, bytes, s>>>(*m, *d, spw);
  }
}

template <bool PREC>
void launch_solver(const MjbModel* m, const MjbData* d, const ChosenCfg& cfg, int spw,
                   cudaStream_t s) {
  // nv > 32: the CTA solver (the precision form's FP64 Hessian factor needs it)
  if (m->nv > 32 && (cfg.cta_warps > 0 || PREC)) {
    const int tc = cfg.hessian_tc;
    const int nw = cfg.cta_warps > 0 ? cfg.cta_warps : 4;  // the precision form's default: 4
    if (nw == 2) launch_solver_cta<2, PREC>(m, d, tc, s);
    else if (nw == 4) launch_solver_cta<4, PREC>(m, d, tc, s);
    else if (nw == 16) launch_solver_cta<16, PREC>(m, d, tc, s);
    else launch_solver_cta<8, PREC>(m, d, tc, s);
    return;
  }
  if (PREC) launch_solver_warp<PREC, true>(m, d, cfg, spw, s);
  else if (cfg.hessian_tc) launch_solver_warp<PREC, true>(m, d, cfg, spw, s);
  else launch_solver_warp<PREC, false>(m, d, cfg, spw, s);
}

// the chosen form's phases: 0 = status reset + the stage kernels up to fwd_acceleration,
// 1 = k_solve, 2 = k_integrate
int run_chosen_phase(const MjbModel* m, const MjbData* d, int phase, cudaStream_t s,
                     const ChosenCfg* tuned = nullptr) {
  if (phase >= 0 && phase <= 2)
    if (int rc = phase_fields(m, d, phase)) return rc;
  const ChosenCfg cfg = tuned ? *tuned : chosen_cfg(m, d);
  const int warps = kDefaultWarps;
  const int grid = grid_for(d->nworld, warps);
  const int tpw = tile_floats(m->nv) + (m->precision ? prec_tile_floats(m->nv) : 0);
  const size_t tile_bytes = size_t(tpw) * warps * sizeof(float);
  static size_t conf_int[kSmemDevices];
  if (phase == 0) {
    reset_counters(d, false, false, false, true, s);
    int rc = run_forward_fork(m, d, s, cfg.lanes);
    if (rc) return rc;
  } else if (phase == 1) {
    if (d->njmax > 0) {
      const int spw = m->nv <= 32 ? int(solver_smem_floats(m->nv)) +
                                        (m->precision ? prec_tile_floats(m->nv) : 0)
                                  : generic_nz_floats(m->nv);
      if (m->precision) launch_solver<true>(m, d, cfg, spw, s);
      else launch_solver<false>(m, d, cfg, spw, s);
    }
  } else if (phase == 2) {
    allow_smem(k_integrate, tile_bytes, conf_int);
    k_integrate<<<grid, 32 * warps, tile_bytes, s>>>(*m, *d, tpw);
  } else {
    return MJB_ERR_ARG;
  }
  return finish();
}

int run_chosen(const MjbModel* m, const MjbData* d, int integrate, cudaStream_t s) {
  int rc;
  for (int p = 0; p < (integrate ? 3 : 2); p++)  // every phase's fields before the first launch
    if ((rc = phase_fields(m, d, p))) return rc;
  if ((rc = run_chosen_phase(m, d, 0, s))) return rc;
  if ((rc = run_chosen_phase(m, d, 1, s))) return rc;
  return integrate ? run_chosen_phase(m, d, 2, s) : MJB_OK;
}

int run_fused(const MjbModel* m, const MjbData* d, const MjbRunCfg* cfg, int integrate,
              cudaStream_t s) {
  for (int p = 0; p < (integrate ? 3 : 2); p++)
    if (int rc = phase_fields(m, d, p)) return rc;
  const int warps = (cfg && cfg->worlds_per_block > 0) ? cfg->worlds_per_block : kDefaultWarps;
  if (warps > 4) return MJB_ERR_ARG;  // __launch_bounds__(128)
  reset_counters(d, true, true, true, true, s);
  const int spw = fused_smem_per_warp(m);
  const size_t smem = size_t(spw) * warps * sizeof(float);
  if (smem > kMaxSmemPerCta) return MJB_ERR_SCRATCH;
  static size_t configured[kSmemDevices];
  allow_smem(k_step_fused, smem, configured);
  k_step_fused<<<grid_for(d->nworld, warps), 32 * warps, smem, s>>>(*m, *d, integrate, spw);
  return finish();
}

}  // namespace

extern "C" {

int mjb_abi_version(void) { return MJB_ABI_VERSION; }

const char* mjb_error_string(int status) {
  switch (status) {
    case MJB_OK: return "ok";
    case MJB_ERR_ARG: return "invalid argument";
    case MJB_ERR_UNSUPPORTED: return "unsupported model feature (elliptic cone, implicitfast with the sparse mass matrix, or the precision form with the sparse mass matrix or a tree of over 32 dofs)";
    case MJB_ERR_LAUNCH: return cudaGetErrorString(cudaGetLastError());
    case MJB_ERR_SCRATCH: return "model too large for on-chip scratch";
    default: return "unknown status";
  }
}

int mjb_forward(const MjbModel* m, const MjbData* d, const MjbRunCfg* cfg, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  for (int p = 0; p < 2; p++)
    if ((rc = phase_fields(m, d, p))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int form = cfg ? cfg->fused : MJB_FORM_CHOSEN;
  if (form == MJB_FORM_PLAIN) return run_forward_plain(m, d, s);
  if (form == MJB_FORM_SINGLE) return run_fused(m, d, cfg, 0, s);
  if (form == MJB_FORM_PRECISION) {
    if ((rc = precision_supported(m))) return rc;
    MjbModel mp = *m;
    mp.precision = 1;
    return run_chosen(&mp, d, 0, s);
  }
  if (form != MJB_FORM_CHOSEN) return MJB_ERR_ARG;
  return run_chosen(m, d, 0, s);
}

int mjb_step(const MjbModel* m, const MjbData* d, const MjbRunCfg* cfg, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  for (int p = 0; p < 3; p++)
    if ((rc = phase_fields(m, d, p))) return rc;
  if (implicit_unsupported(m)) return MJB_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  const int form = cfg ? cfg->fused : MJB_FORM_CHOSEN;
  if (form == MJB_FORM_PLAIN) {
    reset_counters(d, false, false, false, true, s);
    if ((rc = run_forward_plain(m, d, s))) return rc;
    if (m->integrator == 0) rc = launch_stage<S_EULER>(m, d, s);
    else rc = launch_stage<S_IMPLICIT>(m, d, s);
    if (rc) return rc;
    return launch_stage<S_CHECK>(m, d, s);
  }
  if (form == MJB_FORM_SINGLE) return run_fused(m, d, cfg, 1, s);
  if (form == MJB_FORM_PRECISION) {
    if ((rc = precision_supported(m))) return rc;
    MjbModel mp = *m;
    mp.precision = 1;
    return run_chosen(&mp, d, 1, s);
  }
  if (form != MJB_FORM_CHOSEN) return MJB_ERR_ARG;
  return run_chosen(m, d, 1, s);
}

int mjb_step_phase(const MjbModel* m, const MjbData* d, int phase, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  return run_chosen_phase(m, d, phase, (cudaStream_t)stream);
}

#define MJB_STAGE_ENTRY(name, STAGE)                                           \
  int name(const MjbModel* m, const MjbData* d, mjbStream stream) {            \
    int rc = check(m, d);                                                      \
    if (rc || d->nworld == 0) return rc;                                       \
    return launch_stage<STAGE>(m, d, (cudaStream_t)stream);                    \
  }

MJB_STAGE_ENTRY(mjb_kinematics, S_KINEMATICS)
MJB_STAGE_ENTRY(mjb_com_pos, S_COM_POS)
MJB_STAGE_ENTRY(mjb_crb, S_CRB)
MJB_STAGE_ENTRY(mjb_factor_m, S_FACTOR_M)
MJB_STAGE_ENTRY(mjb_rne, S_RNE)
MJB_STAGE_ENTRY(mjb_transmission, S_TRANSMISSION)
MJB_STAGE_ENTRY(mjb_com_vel, S_COM_VEL)
MJB_STAGE_ENTRY(mjb_passive, S_PASSIVE)
MJB_STAGE_ENTRY(mjb_fwd_velocity, S_FWD_VELOCITY)
MJB_STAGE_ENTRY(mjb_fwd_actuation, S_FWD_ACTUATION)
MJB_STAGE_ENTRY(mjb_fwd_acceleration, S_FWD_ACCELERATION)
MJB_STAGE_ENTRY(mjb_euler, S_EULER)
int mjb_implicit(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if (m->is_sparse) return MJB_ERR_UNSUPPORTED;
  return launch_stage<S_IMPLICIT>(m, d, (cudaStream_t)stream);
}
MJB_STAGE_ENTRY(mjb_nxn_broadphase, S_NXN)

int mjb_fwd_position(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  for (int st : {S_KINEMATICS, S_COM_POS, S_CRB, S_FACTOR_M, S_NXN, S_NARROW, S_MAKE_CONSTRAINT,
                 S_TRANSMISSION})
    if ((rc = stage_fields(st, m, d))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = launch_stage<S_KINEMATICS>(m, d, s))) return rc;
  if ((rc = launch_stage<S_COM_POS>(m, d, s))) return rc;
  if ((rc = launch_stage<S_CRB>(m, d, s))) return rc;
  if ((rc = launch_stage<S_FACTOR_M>(m, d, s))) return rc;
  if ((rc = mjb_collision(m, d, stream))) return rc;
  if ((rc = mjb_make_constraint(m, d, stream))) return rc;
  return launch_stage<S_TRANSMISSION>(m, d, s);
}

int mjb_collision(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if ((rc = stage_fields(S_NXN, m, d)) || (rc = stage_fields(S_NARROW, m, d))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  reset_counters(d, true, true, false, false, s);  // collision_driver.py:533-534
  if ((rc = launch_broadphase(m, d, s))) return rc;
  return launch_stage<S_NARROW>(m, d, s);
}

MJB_STAGE_ENTRY(mjb_sap_broadphase, S_SAP)

int mjb_primitive_narrowphase(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if ((rc = stage_fields(S_NARROW, m, d))) return rc;
  if (!d->collision_worldid || !d->ncollision) return MJB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  rebuild_index(d->collision_worldid, d->ncollision, d->nconmax, d->world_pairadr, d->world_npair, d, s);
  return launch_stage<S_NARROW>(m, d, s);
}

int mjb_make_constraint(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if ((rc = stage_fields(S_MAKE_CONSTRAINT, m, d))) return rc;
  if (!d->contact_worldid || !d->ncon) return MJB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  rebuild_index(d->contact_worldid, d->ncon, d->nconmax, d->world_conadr, d->world_ncon, d, s);
  reset_counters(d, false, false, true, false, s);
  return launch_stage<S_MAKE_CONSTRAINT>(m, d, s);
}

int mjb_solve(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if ((rc = stage_fields(S_SOLVE, m, d))) return rc;
  if (d->njmax > 0 && (!d->efc_worldid || !d->nefc)) return MJB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  rebuild_index(d->efc_worldid, d->nefc, d->njmax, d->world_efcadr, d->world_nefc, d, s);
  return launch_stage<S_SOLVE>(m, d, s);
}

int mjb_solve_m(const MjbModel* m, const MjbData* d, float* x, const float* y, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if (!x || !y || (m->nv > 0 && !d->qLD) || (m->is_sparse && m->nv > 0 && !d->qLDiagInv))
    return MJB_ERR_ARG;
  k_solve_m<<<grid_for(d->nworld, 4), 128, 0, (cudaStream_t)stream>>>(*m, *d, x, y);
  return finish();
}

int mjb_mul_m(const MjbModel* m, const MjbData* d, float* res, const float* vec, const uint8_t* skip,
              mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if (!res || !vec) return MJB_ERR_ARG;
  k_mul_m<<<grid_for(d->nworld, 4), 128, 0, (cudaStream_t)stream>>>(*m, *d, res, vec, skip);
  return finish();
}

int mjb_xfrc_accumulate(const MjbModel* m, const MjbData* d, float* qfrc, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if (!qfrc) return MJB_ERR_ARG;
  k_xfrc<<<grid_for(d->nworld, 4), 128, 0, (cudaStream_t)stream>>>(*m, *d, qfrc);
  return finish();
}

int mjb_step_io(const MjbModel* m, const MjbData* d, const MjbStepIO* io, int nstep,
                const MjbRunCfg* cfg, mjbStream stream) {
  int rc = check(m, d);
  if (rc) return rc;
  if (!io || nstep < 0) return MJB_ERR_ARG;
  if (d->nworld == 0) return MJB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t W = size_t(d->nworld), f = sizeof(float);
  struct Copy {
    const void* src;
    void* dst;
    size_t bytes;
  };
  const Copy in[4] = {{io->qpos, d->qpos, W * m->nq * f}, {io->qvel, d->qvel, W * m->nv * f},
                      {io->ctrl, d->ctrl, W * m->nu * f},
                      {io->qacc_warmstart, d->qacc_warmstart, W * m->nv * f}};
  const Copy out[8] = {{d->qpos, io->qpos_out, W * m->nq * f},
                       {d->qvel, io->qvel_out, W * m->nv * f},
                       {d->qacc_warmstart, io->qacc_warmstart_out, W * m->nv * f},
                       {d->xpos, io->xpos_out, W * m->nbody * 3 * f},
                       {d->xmat, io->xmat_out, W * m->nbody * 9 * f},
                       {d->subtree_com, io->subtree_com_out, W * m->nbody * 3 * f},
                       {d->cvel, io->cvel_out, W * m->nbody * 6 * f},
                       {d->site_xpos, io->site_xpos_out, W * m->nsite * 3 * f}};
  for (const Copy& c : in)  // a requested copy into a missing Data field is an error
    if (c.src && c.bytes && !c.dst) return MJB_ERR_ARG;
  for (const Copy& c : out)
    if (c.dst && c.bytes && !c.src) return MJB_ERR_ARG;
  for (const Copy& c : in)
    if (c.src && c.bytes &&
        cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return MJB_ERR_LAUNCH;
  for (int k = 0; k < nstep; k++)
    if ((rc = mjb_step(m, d, cfg, stream))) return rc;
  for (const Copy& c : out)
    if (c.dst && c.bytes &&
        cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return MJB_ERR_LAUNCH;
  return MJB_OK;
}

int mjb_world_status(const MjbData* d, uint32_t* host_out, mjbStream stream) {
  if (!d || !host_out || !d->world_status) return MJB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(host_out, d->world_status, sizeof(uint32_t) * d->nworld,
                      cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return MJB_ERR_LAUNCH;
  if (cudaStreamSynchronize(s) != cudaSuccess) return MJB_ERR_LAUNCH;
  return MJB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Allocation-free implicitfast integration.
//
// Some callers cannot allocate device memory at the point where they step the simulation: a
// host framework that hands a plugin nothing but its operand buffers (an XLA / JAX custom call
// without a workspace, for instance), or a real-time control loop that must never pay for
// cudaMalloc's implicit device synchronisation after start-up.  mjb_implicit needs four
// per-world work arrays (the damped mass matrix, its Cholesky factor, the right-hand side and the
// affine actuators' velocity coefficients); this variant takes them from a fixed array that lives
// in the library itself, so the caller only provides the inputs and outputs it already has: qM,
// qfrc_smooth, qfrc_constraint, the actuator moments and controls (read), qpos and qvel (advanced
// in place) and qacc_integration (written).
namespace {

constexpr size_t kNoallocScratchBytes = size_t(64) << 20;  // 64 MiB, held by every GPU that loads
                                                             // the library until the process exits
__device__ __align__(256) float g_noalloc_scratch[kNoallocScratchBytes / sizeof(float)];

constexpr int kMaxDevices = 64;
std::atomic<float*> g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, resolved once per device (the name
// g_noalloc_scratch in host code is only a host-side stand-in and must never be passed to a kernel).
// Host threads that race on the first call store the same address.
int noalloc_scratch(float** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MJB_ERR_LAUNCH;
  float* p = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    void* a = nullptr;
    if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess || !a) return MJB_ERR_LAUNCH;
    p = static_cast<float*>(a);
    g_noalloc_ptr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return MJB_OK;
}

}  // namespace

extern "C" size_t mjb_implicit_noalloc_max_bytes(void) { return kNoallocScratchBytes; }

extern "C" int mjb_implicit_noalloc(const MjbModel* m, const MjbData* d, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if (m->is_sparse) return MJB_ERR_UNSUPPORTED;
  const size_t nv = size_t(m->nv), nu = size_t(m->nu), nw = size_t(d->nworld);
  const size_t need = nw * (2 * nv * nv + nv + nu) * sizeof(float);
  if (need > kNoallocScratchBytes) return MJB_ERR_SCRATCH;
  float* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  MjbData dd = *d;  // same inputs and outputs, work arrays redirected into the static scratch
  dd.qM_integration = scratch;
  dd.qLD_integration = scratch + nw * nv * nv;
  dd.qfrc_integration = scratch + 2 * nw * nv * nv;
  dd.act_vel_integration = scratch + nw * (2 * nv * nv + nv);
  return launch_stage<S_IMPLICIT>(m, &dd, (cudaStream_t)stream);
}

// ------------------------------------------------------------------------------------------
// Autotuner of the chosen form's launch parameters.

extern "C" int mjb_autotune(const MjbModel* m, const MjbData* d, float* warmstart_scratch,
                            MjbTune* out, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  if (!warmstart_scratch || !d->qacc_warmstart) return MJB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t wsb = size_t(d->nworld) * size_t(m->nv) * sizeof(float);
  auto restore = [&]() {
    return cudaMemcpyAsync(d->qacc_warmstart, warmstart_scratch, wsb, cudaMemcpyDeviceToDevice, s);
  };
  if (cudaMemcpyAsync(warmstart_scratch, d->qacc_warmstart, wsb, cudaMemcpyDeviceToDevice, s) !=
      cudaSuccess)
    return MJB_ERR_LAUNCH;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return MJB_ERR_LAUNCH;
  }
  // candidates: tree-stage lanes x the solver's CTA shape (warps per CTA of the persistent
  // one-warp-per-world solver, or, for nv > 32, warps per world of the CTA solver); for
  // nv <= 32 also the Newton Hessian's assembly (FMAs or the tensor pipe), for nv > 32 the
  // tensor-core assembly tried once more on the best CTA shape
  const int lanes[3] = {8, 16, 32}, widths[6] = {1, 2, 4, 1, 2, 4}, cta[4] = {2, 4, 8, 0};
  const bool large = m->nv > 32;
  float best = 0.f;
  ChosenCfg best_cfg;
  bool have = false;
  auto trial = [&](const ChosenCfg& c) -> int {
    auto forward = [&]() -> int {
      if (restore() != cudaSuccess) return MJB_ERR_LAUNCH;
      int r = run_chosen_phase(m, d, 0, s, &c);
      return r ? r : run_chosen_phase(m, d, 1, s, &c);
    };
    int r = forward();  // warm-up
    if (r) return r;
    constexpr int kReps = 3;
    if (cudaEventRecord(e0, s) != cudaSuccess) return MJB_ERR_LAUNCH;
    for (int k = 0; k < kReps && !r; k++) r = forward();
    if (r) return r;
    float ms = 0.f;
    if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return MJB_ERR_LAUNCH;
    ms /= kReps;
    if (!have || ms < best) {
      best = ms;
      best_cfg = c;
      have = true;
    }
    return MJB_OK;
  };
  for (int li = 0; li < 3 && !rc; li++) {
    for (int wi = 0; wi < (large ? 4 : 6) && !rc; wi++) {
      ChosenCfg c;
      c.lanes = lanes[li];
      if (large) {
        c.cta_warps = cta[wi];
      } else {
        c.warps = widths[wi];
        c.hessian_tc = wi >= 3;
      }
      rc = trial(c);
    }
  }
  if (!rc && large && best_cfg.cta_warps > 0) {
    ChosenCfg c = best_cfg;
    c.hessian_tc = 1;
    rc = trial(c);
  }
  if (!rc && !large && !best_cfg.hessian_tc) {  // the persistent solver's other occupancy
    ChosenCfg c = best_cfg;
    c.solver_ctas = best_cfg.solver_ctas == 4 ? 5 : 4;
    rc = trial(c);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int nefc = 0;  // rows of the last trial's forward (the same worlds in every trial)
  if (!rc && d->nefc &&
      cudaMemcpyAsync(&nefc, d->nefc, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = MJB_ERR_LAUNCH;
  if (!rc && restore() != cudaSuccess) rc = MJB_ERR_LAUNCH;
  if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = MJB_ERR_LAUNCH;
  if (rc) return rc;
  store_cfg(m, d, best_cfg);
  if (out) {
    out->tree_lanes = best_cfg.lanes;
    out->solver_warps = best_cfg.warps;
    out->solver_cta_warps = best_cfg.cta_warps;
    out->hessian_tc = best_cfg.hessian_tc;
    out->solver_ctas_per_sm = best_cfg.solver_ctas;
    out->ms_per_forward = best;
    out->rows_per_world = float(std::min(nefc, d->njmax)) / float(d->nworld);
  }
  return MJB_OK;
}

extern "C" int mjb_set_tune(const MjbModel* m, const MjbData* d, const MjbTune* tune) {
  int rc = check(m, d);
  if (rc) return rc;
  if (!tune) return MJB_ERR_ARG;
  const int l = tune->tree_lanes, w = tune->solver_warps, c = tune->solver_cta_warps;
  const int o = tune->solver_ctas_per_sm;
  if ((l != 8 && l != 16 && l != 32) || (w != 1 && w != 2 && w != 4) ||
      (c != 0 && c != 2 && c != 4 && c != 8 && c != 16) ||
      (tune->hessian_tc != 0 && tune->hessian_tc != 1) || (o != 0 && o != 4 && o != 5))
    return MJB_ERR_ARG;
  ChosenCfg cfg;
  cfg.lanes = l;
  cfg.warps = w;
  cfg.cta_warps = c;
  cfg.hessian_tc = tune->hessian_tc;
  if (o) cfg.solver_ctas = o;
  store_cfg(m, d, cfg);
  return MJB_OK;
}

// ------------------------------------------------------------------------------------------
// Finite-difference transition Jacobians (mjb_deriv.cuh).

extern "C" int mjb_fd_perturb(const MjbModel* m, const MjbData* base, const MjbData* pert,
                              float eps, int flags, mjbStream stream) {
  int rc = check(m, base);
  if (rc || base->nworld == 0) return rc;
  if (!pert || !(eps > 0.f) || (flags & ~7)) return MJB_ERR_ARG;
  if ((long long)pert->nworld != (long long)base->nworld * fd_slots(*m, flags)) return MJB_ERR_ARG;
  if (!pert->qpos || !pert->qvel || !base->qpos || !base->qvel) return MJB_ERR_ARG;
  if ((m->na && (!pert->act || !base->act)) || (m->nu && (!pert->ctrl || !base->ctrl)))
    return MJB_ERR_ARG;
  k_fd_perturb<<<grid_for(pert->nworld, 4), 128, 0, (cudaStream_t)stream>>>(*m, *base, *pert, eps,
                                                                            flags);
  return finish();
}

extern "C" int mjb_fd_jacobian(const MjbModel* m, const MjbData* pert, int nworld, float eps,
                               int flags, float* A, float* B, mjbStream stream) {
  int rc = check(m, pert);
  if (rc || nworld == 0) return rc;
  const bool need_b = m->nu && !(flags & (kFdStateOnly | kFdQposOnly));
  if (nworld < 0 || !A || (need_b && !B) || !(eps > 0.f) || (flags & ~7)) return MJB_ERR_ARG;
  if ((long long)pert->nworld != (long long)nworld * fd_slots(*m, flags)) return MJB_ERR_ARG;
  const long long warps = (long long)nworld * fd_ncol(*m, flags);
  k_fd_jacobian<<<int((warps + 3) / 4), 128, 0, (cudaStream_t)stream>>>(*m, *pert, nworld, eps,
                                                                       flags, A, B);
  return finish();
}

static int launch_step_vjp(const MjbModel* m, const MjbData* d, const float* lam,
                           const float* qvel_prev, float* grad_ctrl, float* grad_qvel,
                           float* grad_qpos, mjbStream stream) {
  int rc = check(m, d);
  if (rc || d->nworld == 0) return rc;
  const bool sweep = grad_qvel || grad_qpos;
  if (!lam || (!grad_ctrl && !sweep) || (sweep && !qvel_prev)) return MJB_ERR_ARG;
  const bool act_on = !(m->disableflags & DSBL_ACTUATION) && m->actuator_affine_bias_gain;
  if (m->is_sparse || m->na > 0 || (m->integrator != 0 && act_on)) return MJB_ERR_UNSUPPORTED;
  if (!d->qLD_integration || (m->nu && !d->actuator_moment)) return MJB_ERR_ARG;
  if (m->nv > 32 && !d->efc_h) return MJB_ERR_ARG;
  if (sweep && (!d->cvel || !d->cdof_dot || !d->cinert || !d->cdof)) return MJB_ERR_ARG;
  if (grad_qpos && (!d->rne_cacc || !d->rne_cfrc || !d->xanchor || !d->xaxis || !d->xipos ||
                    !d->ximat || !d->subtree_com || !d->qacc_integration))
    return MJB_ERR_ARG;
  const int per_warp = (step_vjp_floats(*m, grad_qvel != nullptr, grad_qpos != nullptr) + 3) & ~3;
  const size_t warp_bytes = size_t(per_warp) * sizeof(float);
  int warps = 4;
  while (warps > 1 && warps * warp_bytes > 48 * 1024) warps >>= 1;
  const size_t bytes = warps * warp_bytes;
  if (bytes > 227 * 1024) return MJB_ERR_SCRATCH;
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_step_vjp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(bytes));
    if (e != cudaSuccess) return MJB_ERR_LAUNCH;
  }
  k_step_vjp<<<grid_for(d->nworld, warps), 32 * warps, bytes, (cudaStream_t)stream>>>(
      *m, *d, lam, qvel_prev, grad_ctrl, grad_qvel, grad_qpos, per_warp);
  return finish();
}

extern "C" int mjb_ctrl_vjp(const MjbModel* m, const MjbData* d, const float* lam, float* grad_ctrl,
                            mjbStream stream) {
  if (!grad_ctrl) return MJB_ERR_ARG;
  return launch_step_vjp(m, d, lam, nullptr, grad_ctrl, nullptr, nullptr, stream);
}

extern "C" int mjb_step_vjp(const MjbModel* m, const MjbData* d, const float* qvel_prev,
                            const float* lam, float* grad_qpos, float* grad_qvel, float* grad_ctrl,
                            mjbStream stream) {
  return launch_step_vjp(m, d, lam, qvel_prev, grad_ctrl, grad_qvel, grad_qpos, stream);
}

extern "C" int mjb_transition_vjp(const MjbModel* m, int nworld, const float* A, const float* B,
                                  const float* lam, float* lam_out, float* grad_ctrl,
                                  mjbStream stream) {
  if (!m || nworld < 0 || !A || !lam || !lam_out || lam == lam_out) return MJB_ERR_ARG;
  if (nworld == 0) return MJB_OK;
  k_transition_vjp<<<grid_for(nworld, 4), 128, 0, (cudaStream_t)stream>>>(*m, nworld, A, B, lam,
                                                                          lam_out, grad_ctrl);
  return finish();
}

// ------------------------------------------------------------------------------------------
// FMA throughput probe (no counterpart in the reference): the FP32 / FP64 peak that the solver's
// flop-bound roofline is measured against.  Every thread runs 8 independent FMA chains of `iters`
// steps; the caller times the launch with CUDA events: flops = 2 * 8 * iters * threads.
namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(int iters, T* sink) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  T a[8];
#pragma unroll
  for (int c = 0; c < 8; c++) a[c] = T(1) + T(1e-3) * T(c + (t & 7));
  const T b = T(0.9999), k = T(1e-4);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < 8; c++) a[c] = a[c] * b + k;
  }
  T s = T(0);
#pragma unroll
  for (int c = 0; c < 8; c++) s += a[c];
  sink[t] = s;
}

}  // namespace

extern "C" int mjb_fma_probe(int fp64, int blocks, int iters, void* sink, mjbStream stream) {
  if (blocks <= 0 || iters <= 0 || !sink) return MJB_ERR_ARG;
  if (fp64) k_fma_probe<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, static_cast<double*>(sink));
  else k_fma_probe<float><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, static_cast<float*>(sink));
  return finish();
}
