/* mjb200.h — C ABI of the B200-native batched physics step (libmjb200.so).
 *
 * The library evaluates MJWarp's batched forward step (mujoco_warp 3.2.7 alpha) on one B200:
 * every entry point below replaces one function of the reference's Python API
 * (mujoco_warp/__init__.py:18-58) and is what a ctypes / FFI binding of that API calls.  The
 * caller owns all device memory (PyTorch's caching allocator in the bundled Python host); the
 * library allocates nothing on any entry point and never synchronises the stream, so a sequence
 * of calls can be captured in a CUDA graph.
 *
 * Layout: every per-world array is world-major (world w's slice starts at w * <per-world size>),
 * structured element types are flattened (vec3 = 3 floats, quat = 4 (w, x, y, z), mat33 = 9
 * row-major, spatial vector = 6 (angular, linear), vec10 inertia = 10).  Contacts, collision pairs
 * and constraint (efc) rows are flat arrays over nconmax / njmax entries tagged with worldid and
 * counted by a device counter, as in the reference (types.py:615-645, 264-363); each world's
 * entries are contiguous, and the per-world index arrays (world_*adr / world_n*) locate them.
 *
 * Errors: every entry point returns an MjbStatus code; launch failures are reported through
 * cudaGetLastError as MJB_ERR_LAUNCH.  Per-world problems found on the device (capacity overflow,
 * non-finite state) are recorded as bits in MjbData.world_status and read back with
 * mjb_world_status.
 */
#ifndef MJB200_H_
#define MJB200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MJB_ABI_VERSION 7

typedef struct CUstream_st* mjbStream; /* == cudaStream_t */

typedef enum MjbStatus {
  MJB_OK = 0,
  MJB_ERR_ARG = 1,          /* null pointer, bad size or unsupported option */
  MJB_ERR_UNSUPPORTED = 2,  /* model feature the kernels do not implement */
  MJB_ERR_LAUNCH = 3,       /* CUDA launch / runtime error */
  MJB_ERR_SCRATCH = 4,      /* model too large for the kernel's on-chip scratch */
} MjbStatus;

/* per-world status bits (MjbData.world_status) */
#define MJB_WS_CONTACT_OVERFLOW 0x1u  /* contacts beyond nconmax were dropped */
#define MJB_WS_EFC_OVERFLOW 0x2u      /* constraint rows beyond njmax were dropped */
#define MJB_WS_PAIR_OVERFLOW 0x4u     /* broadphase pairs beyond nconmax were dropped */
#define MJB_WS_NONFINITE 0x8u         /* qpos / qvel / qacc not finite after the step */
#define MJB_WS_ROWS_SPLIT 0x10u       /* a world's flat rows were not contiguous */

/* Read-only model, shared by all worlds (types.py:366-612).  Device pointers. */
typedef struct MjbModel {
  int32_t nq, nv, na, nu, nbody, njnt, ngeom, nsite, nmocap, nM;
  int32_t nlimit;      /* len(jnt_limited_slide_hinge_adr) */
  int32_t nlevel;      /* BFS levels of the body tree, world included */
  int32_t nblock;      /* dof tree blocks (one per kinematic tree) */
  int32_t block_max;   /* dofs of the largest tree block (max of block_size) */
  int32_t npair_cand;  /* geom pairs that pass the static filter (broadphase candidates) */
  int32_t nlsp;        /* parallel line-search candidates */
  /* Option (types.py:218-250) */
  int32_t integrator, cone, solver, iterations, ls_iterations, disableflags, is_sparse,
      ls_parallel;
  int32_t actuator_affine_bias_gain;
  int32_t precision;   /* set by MJB_FORM_PRECISION on its own copy; 0 in callers' models */
  float timestep, impratio, tolerance, ls_tolerance, meaninertia;
  float gravity[3];
  /* tree / level tables */
  const int32_t *body_tree, *body_treeadr, *body_childadr, *body_childnum, *body_child,
      *body_subtreeend;
  const int32_t *body_parentid, *body_rootid, *body_weldid, *body_jntnum, *body_jntadr,
      *body_dofnum, *body_dofadr;
  const float *body_pos, *body_quat, *body_ipos, *body_iquat, *body_mass, *subtree_mass,
      *body_inertia, *body_invweight0;
  const int32_t *jnt_type, *jnt_qposadr, *jnt_dofadr, *jnt_bodyid, *jnt_limited,
      *jnt_actfrclimited, *jnt_limited_slide_hinge_adr;
  const float *jnt_solref, *jnt_solimp, *jnt_pos, *jnt_axis, *jnt_stiffness, *jnt_range,
      *jnt_actfrcrange, *jnt_margin;
  const int32_t *dof_bodyid, *dof_jntid, *dof_parentid, *dof_Madr;
  const float *dof_armature, *dof_damping, *dof_invweight0;
  const int32_t *block_adr, *block_size;
  const int32_t *geom_type, *geom_contype, *geom_conaffinity, *geom_condim, *geom_bodyid,
      *geom_priority;
  const float *geom_pos, *geom_quat, *geom_size, *geom_rbound, *geom_solmix, *geom_solref,
      *geom_solimp, *geom_friction, *geom_margin, *geom_gap;
  const int32_t* pair_cand; /* 2 * npair_cand geom ids (g1 < g2), nxn element order */
  const int32_t* site_bodyid;
  const float *site_pos, *site_quat;
  const int32_t *actuator_trntype, *actuator_dyntype, *actuator_gaintype, *actuator_biastype,
      *actuator_trnid, *actuator_actadr, *actuator_ctrllimited, *actuator_forcelimited,
      *actuator_actlimited;
  const float *actuator_dynprm, *actuator_gainprm, *actuator_biasprm, *actuator_ctrlrange,
      *actuator_forcerange, *actuator_actrange, *actuator_gear;
  const float *qpos0, *qpos_spring;
  const float* alpha_candidate;
} MjbModel;

/* Per-world state, intermediates, contacts and constraints (types.py:648-800).  Device
 * pointers; fields a call does not touch may be null. */
typedef struct MjbData {
  int32_t nworld, nconmax, njmax;
  /* state */
  float *qpos, *qvel, *act, *ctrl, *qacc, *qacc_warmstart, *qfrc_applied, *xfrc_applied;
  /* smooth dynamics */
  float *xpos, *xquat, *xmat, *xipos, *ximat, *xanchor, *xaxis, *geom_xpos, *geom_xmat,
      *site_xpos, *site_xmat, *subtree_com, *cinert, *crb, *cdof, *cvel, *cdof_dot, *qM, *qLD,
      *qLDiagInv;
  float *actuator_length, *actuator_velocity, *actuator_force, *actuator_moment;
  float *qfrc_bias, *qfrc_spring, *qfrc_damper, *qfrc_passive, *qfrc_actuator, *qfrc_smooth,
      *qfrc_constraint, *qacc_smooth, *act_dot, *rne_cacc, *rne_cfrc;
  float *qfrc_integration, *qacc_integration, *qM_integration, *qLD_integration,
      *act_vel_integration;
  /* global counters (1 element each) */
  int32_t *ncon, *nefc, *ncollision;
  /* collision pairs and contacts (flat) */
  int32_t *collision_pair, *collision_worldid;
  float *contact_dist, *contact_pos, *contact_frame, *contact_includemargin, *contact_friction,
      *contact_solref, *contact_solreffriction, *contact_solimp;
  int32_t *contact_dim, *contact_geom, *contact_efc_address, *contact_worldid;
  /* constraint rows (flat, njmax) */
  int32_t* efc_worldid;
  float *efc_J, *efc_pos, *efc_margin, *efc_D, *efc_aref, *efc_force, *efc_Jaref, *efc_jv,
      *efc_quad;
  int32_t* efc_active;
  /* solver per world */
  float *efc_Ma, *efc_grad, *efc_grad_dot, *efc_Mgrad, *efc_search, *efc_search_dot,
      *efc_gauss, *efc_cost, *efc_prev_cost, *efc_gtol, *efc_mv, *efc_quad_gauss, *efc_h,
      *efc_alpha, *efc_prev_grad, *efc_prev_Mgrad, *efc_beta;
  int32_t* efc_solver_niter;
  uint8_t* efc_done;
  /* per-world index of the flat arrays and status bits */
  int32_t *world_pairadr, *world_npair, *world_conadr, *world_ncon, *world_efcadr, *world_nefc;
  uint32_t* world_status;
  /* the chosen form's solver schedule (may be null: worlds are then solved in index order):
     world_order (nworld) receives the worlds sorted by constraint rows, largest first, and
     work_queue (1) is the persistent solver's next-world counter */
  int32_t *world_order, *work_queue;
} MjbData;

/* Launch configuration for the step entry points. */
/* Launch forms of mjb_step / mjb_forward (MjbRunCfg.fused; a null cfg selects MJB_FORM_CHOSEN). */
#define MJB_FORM_PLAIN 0  /* one kernel per reference stage; Hessian refactored every iteration */
#define MJB_FORM_CHOSEN 1 /* stage kernels to fwd_acceleration + solver reusing its factor + integrator */
#define MJB_FORM_SINGLE 2 /* the whole step of a world in one warp of one kernel */
/* MJB_FORM_CHOSEN with the Newton Hessian assembled in split TF32 on the tensor pipe (nv <= 32),
   the Hessian and mass-matrix Cholesky factor-solves in FP64 and the line-search polynomial
   coefficients accumulated in FP64.  Dense mass matrix, tree blocks of up to 32 dofs
   (MJB_ERR_UNSUPPORTED otherwise); for nv > 32 the Hessian's FP64 factor lives in shared memory,
   which bounds nv at about 230 (MJB_ERR_SCRATCH beyond). */
#define MJB_FORM_PRECISION 3

typedef struct MjbRunCfg {
  int32_t fused;            /* launch form, MJB_FORM_* */
  int32_t worlds_per_block; /* MJB_FORM_SINGLE: warps (= worlds) per CTA, at most 4; 0 = 4 */
} MjbRunCfg;

int mjb_abi_version(void);
const char* mjb_error_string(int status);

/* step (forward.py:682-695): forward + Euler or implicitfast integration. */
int mjb_step(const MjbModel* m, const MjbData* d, const MjbRunCfg* cfg, mjbStream stream);
/* forward (forward.py:664-679). */
int mjb_forward(const MjbModel* m, const MjbData* d, const MjbRunCfg* cfg, mjbStream stream);
/* One phase of MJB_FORM_CHOSEN's step (no counterpart in the reference, whose step is one call):
   0 = counter reset + fwd_position .. fwd_acceleration (and the ordering of the worlds by their
   constraint rows for phase 1's persistent solver), 1 = the constraint solver, 2 = Euler /
   implicitfast integration + the finiteness check.  Phases 0, 1, 2 in order equal mjb_step; they
   let a caller time the kernels separately or act between forward and integration.  Phase 1
   reads phase 0's ordering: run it once after each phase 0. */
int mjb_step_phase(const MjbModel* m, const MjbData* d, int phase, mjbStream stream);

/* The device buffers of a host framework's step call (the JAX FFI pattern of
 * contrib/jax_unroll.py:40-71 and the notebook's unrolled step): world-major arrays shaped like
 * the matching Data fields.  Inputs are copied into the Data before the first substep (null: the
 * Data's own values are kept); outputs are copied out of it after the last substep (null: not
 * copied). */
typedef struct MjbStepIO {
  const float *qpos, *qvel, *ctrl, *qacc_warmstart;
  float *qpos_out, *qvel_out, *qacc_warmstart_out, *xpos_out, *xmat_out, *subtree_com_out,
      *cvel_out, *site_xpos_out;
} MjbStepIO;
/* Copy in, nstep calls of mjb_step (cfg as there), copy out: every copy is one
 * cudaMemcpyAsync on the stream, so the call allocates nothing, does not synchronise and can be
 * captured in a CUDA graph; no counterpart function in the reference, whose callers write these
 * copies around step themselves. */
int mjb_step_io(const MjbModel* m, const MjbData* d, const MjbStepIO* io, int nstep,
                const MjbRunCfg* cfg, mjbStream stream);

/* Pipeline stages (forward.py:408-661). */
int mjb_fwd_position(const MjbModel* m, const MjbData* d, mjbStream stream);
int mjb_fwd_velocity(const MjbModel* m, const MjbData* d, mjbStream stream);
int mjb_fwd_actuation(const MjbModel* m, const MjbData* d, mjbStream stream);
int mjb_fwd_acceleration(const MjbModel* m, const MjbData* d, mjbStream stream);
int mjb_euler(const MjbModel* m, const MjbData* d, mjbStream stream);    /* forward.py:165 */
int mjb_implicit(const MjbModel* m, const MjbData* d, mjbStream stream); /* forward.py:245 */

/* Smooth dynamics (smooth.py). */
int mjb_kinematics(const MjbModel* m, const MjbData* d, mjbStream stream);   /* :32 */
int mjb_com_pos(const MjbModel* m, const MjbData* d, mjbStream stream);      /* :148 */
int mjb_crb(const MjbModel* m, const MjbData* d, mjbStream stream);          /* :248 */
int mjb_factor_m(const MjbModel* m, const MjbData* d, mjbStream stream);     /* :392 */
int mjb_rne(const MjbModel* m, const MjbData* d, mjbStream stream);          /* :398 */
int mjb_transmission(const MjbModel* m, const MjbData* d, mjbStream stream); /* :469 */
int mjb_com_vel(const MjbModel* m, const MjbData* d, mjbStream stream);      /* :539 */
int mjb_passive(const MjbModel* m, const MjbData* d, mjbStream stream);      /* passive.py:27 */
/* x = qLD^-1 y per world (smooth.py:693-696); x and y are (nworld, nv). */
int mjb_solve_m(const MjbModel* m, const MjbData* d, float* x, const float* y, mjbStream stream);

/* Collision (collision_driver.py, collision_primitive.py). */
int mjb_collision(const MjbModel* m, const MjbData* d, mjbStream stream);      /* :525 */
int mjb_nxn_broadphase(const MjbModel* m, const MjbData* d, mjbStream stream); /* :458 */
int mjb_sap_broadphase(const MjbModel* m, const MjbData* d, mjbStream stream); /* :350 */
int mjb_primitive_narrowphase(const MjbModel* m, const MjbData* d,
                              mjbStream stream); /* collision_primitive.py:271 */

/* Constraints (constraint.py:213) and solver (solver.py:872). */
int mjb_make_constraint(const MjbModel* m, const MjbData* d, mjbStream stream);
int mjb_solve(const MjbModel* m, const MjbData* d, mjbStream stream);

/* Support (support.py). res = M vec per world unless skip[world] (support.py:35-137). */
int mjb_mul_m(const MjbModel* m, const MjbData* d, float* res, const float* vec,
              const uint8_t* skip, mjbStream stream);
/* qfrc += J^T xfrc_applied per world (support.py:140-172). */
int mjb_xfrc_accumulate(const MjbModel* m, const MjbData* d, float* qfrc, mjbStream stream);

/* Copies world_status (nworld words) to host memory; synchronises the stream. */
int mjb_world_status(const MjbData* d, uint32_t* host_out, mjbStream stream);

/* Launch parameters of the chosen form that the autotuner picks (no counterpart in the reference):
 * lanes per world of the tree-recursion stages, warps per CTA of the persistent solver (one warp
 * per world, nv <= 32) and how it assembles the Newton Hessian (FP32 FMAs, or split-TF32
 * tensor-core products, which the precision form always uses), and warps per world of the CTA
 * solver of models with nv > 32. */
typedef struct MjbTune {
  int32_t tree_lanes;        /* 8, 16 or 32 */
  int32_t solver_warps;      /* 1, 2 or 4 */
  int32_t solver_cta_warps;  /* 2, 4, 8 or 16 warps per world; 0 = one warp per world */
  int32_t hessian_tc;        /* nv <= 32: 1 = Newton Hessian in split TF32 on the tensor pipe */
  int32_t solver_ctas_per_sm; /* nv <= 32, FMA Hessian: resident CTAs per SM of the persistent
                                 solver, 4 (128 registers) or 5 (96); 0 in mjb_set_tune = 5 */
  float ms_per_forward;      /* measured chosen-form forward (fwd_position .. solve) at this setting */
  float rows_per_world;      /* mean constraint rows per world of the Data it was measured on */
} MjbTune;

/* Autotuner (no counterpart in the reference): times the chosen form's forward for every
 * tree-lane count and solver CTA width (and, for nv <= 32, the persistent solver's resident CTAs
 * per SM on the best of those) on d's current worlds and keeps the fastest, per device,
 * for models of this nv and Data of this rows-per-world capacity (njmax / nworld); later chosen-
 * form calls with the same key use it (others keep 16 lanes, 4 warps per solver CTA, FMA
 * Hessians, and 4 warps per world when nv > 128, one warp per world below).  out->rows_per_world reports the mean
 * constraint rows per world of d's worlds (the key cannot hold it: the host does not see the row
 * counts of a step without synchronising).  warmstart_scratch:
 * nworld * nv floats of caller memory; qacc_warmstart is saved there and restored before every
 * trial and at the end, so d is left as after one chosen-form forward.  Synchronises the stream;
 * out may be null. */
int mjb_autotune(const MjbModel* m, const MjbData* d, float* warmstart_scratch, MjbTune* out,
                 mjbStream stream);
/* Sets the chosen form's launch parameters for the same key as mjb_autotune (device, nv, rows-
 * per-world capacity) without measuring: tree_lanes, solver_warps, solver_cta_warps, hessian_tc
 * and solver_ctas_per_sm as in MjbTune (the timing fields are ignored).  MJB_ERR_ARG for a value outside
 * those sets. */
int mjb_set_tune(const MjbModel* m, const MjbData* d, const MjbTune* tune);

/* Finite-difference transition Jacobians, no counterpart in the reference (whose API has no
 * derivatives); the scheme is MuJoCo's mjd_transitionFD, batched over worlds.  State
 * x = (qpos in the tangent space, qvel, act), nx = 2 nv + na; input u = ctrl.  `pert` is a Data
 * of nworld * K worlds, K = 1 + ncol (forward differences) or 1 + 2 ncol (centered),
 * ncol = nx + nu (nx with MJB_FD_STATE_ONLY, nv with MJB_FD_QPOS_ONLY).  mjb_fd_perturb copies
 * every base world's state into its K slots and perturbs one column per slot by eps
 * (tangent-space rotations for quaternions); the caller then steps `pert` (mjb_step);
 * mjb_fd_jacobian differences the next states into A (nworld x nx x nx) and B (nworld x nx x nu),
 * row-major per world: A[w][i][j] = d x'_i / d x_j.  eps > 0; in FP32 a value near 1e-3 balances
 * truncation and rounding. */
int mjb_fd_perturb(const MjbModel* m, const MjbData* base, const MjbData* pert, float eps,
                   int flags, mjbStream stream);
int mjb_fd_jacobian(const MjbModel* m, const MjbData* pert, int nworld, float eps, int flags,
                    float* A, float* B, mjbStream stream);
/* `flags`: MJB_FD_CENTERED for centered differences; MJB_FD_STATE_ONLY to perturb the state
 * columns only (ncol = nx; B is not written and may be null); MJB_FD_QPOS_ONLY to perturb the
 * nv qpos columns only (ncol = nv; only A's first nv columns are written).  Both calls take the
 * same flags. */
#define MJB_FD_CENTERED 1
#define MJB_FD_STATE_ONLY 2
#define MJB_FD_QPOS_ONLY 4

/* Adjoint of one step by implicit differentiation at the constraint solver's final active set
 * (no counterpart in the reference): for lam (nworld x nx) the adjoint of the step's next state
 * (qpos tangent, qvel), writes grad_qpos (nworld x nv, qpos tangent: free / ball rotations about
 * local axes) = (d x' / d qpos)^T lam, grad_qvel (nworld x nv) and grad_ctrl (nworld x nu); any
 * of the three may be null.  d must hold that step's results (call it right after mjb_step): its
 * qM, constraint rows and active flags, contacts, qLD_integration, qacc_integration, kinematics,
 * com / rne and actuator arrays and the new qvel; qvel_prev is the qvel the step started from
 * (not needed for grad_ctrl alone).  Exact at a converged Newton solution (the active set and the
 * contacts held fixed).  Needs the dense mass matrix and na = 0, and for implicitfast no
 * affine actuator gains or biases (else MJB_ERR_UNSUPPORTED); grad_qpos further assumes: ball
 * joints alone on their body, no stiffness on free / ball joints, actuators on hinge / slide
 * joints, planes on bodies welded to the world, zero xfrc_applied.  For nv > 32 with the Newton
 * solver the factor of the Hessian that the step left in d->efc_h is reused (with CG the Hessian
 * and its factor are written there). */
int mjb_step_vjp(const MjbModel* m, const MjbData* d, const float* qvel_prev, const float* lam,
                 float* grad_qpos, float* grad_qvel, float* grad_ctrl, mjbStream stream);
/* mjb_step_vjp for grad_ctrl alone */
int mjb_ctrl_vjp(const MjbModel* m, const MjbData* d, const float* lam, float* grad_ctrl,
                 mjbStream stream);

/* Reverse step of a rollout adjoint, per world: lam_out = A^T lam, grad_ctrl = B^T lam
 * (B / grad_ctrl may be null); lam and lam_out are nworld x nx and must not alias. */
int mjb_transition_vjp(const MjbModel* m, int nworld, const float* A, const float* B,
                       const float* lam, float* lam_out, float* grad_ctrl, mjbStream stream);

/* FMA throughput probe (no counterpart in the reference; a measurement aid for the solver's
 * flop-bound roofline): `blocks` CTAs of 256 threads, each thread running 8 independent FP32
 * (fp64 = 0) or FP64 FMA chains of `iters` steps, writing one value per thread to sink
 * (blocks * 256 floats or doubles).  The caller times it: flops = 2 * 8 * iters * blocks * 256. */
int mjb_fma_probe(int fp64, int blocks, int iters, void* sink, mjbStream stream);

/* Allocation-free variant of mjb_implicit, with no counterpart in the reference.  For callers
 * that may not allocate device memory when they step (a plugin that receives only its operand
 * buffers, a control loop that cannot afford cudaMalloc's synchronisation): the integrator's
 * four per-world work arrays (qM_integration, qLD_integration, qfrc_integration and
 * act_vel_integration) come from a 64 MiB array compiled into the library instead of from
 * MjbData, so those four fields may be null.  Inputs and outputs are as for mjb_implicit: qM,
 * qfrc_smooth, qfrc_constraint, actuator_moment, ctrl / act are read; qpos, qvel are advanced;
 * qacc_integration is written.
 * Limit: nworld * (2 * nv * nv + nv + nu) * 4 bytes <= mjb_implicit_noalloc_max_bytes() (64 MiB,
 * e.g. 11140 humanoid worlds at nv = 27, nu = 21); larger requests return MJB_ERR_SCRATCH.  The
 * first call on each device resolves the array's device address (cudaGetSymbolAddress), so make
 * one call per device before capturing a CUDA graph.  All calls share the one array: calls that
 * overlap on the GPU (different streams, or graphs replayed concurrently) race on it.  Nothing in
 * it needs to start at zero: every call writes each element before reading it. */
int mjb_implicit_noalloc(const MjbModel* m, const MjbData* d, mjbStream stream);
size_t mjb_implicit_noalloc_max_bytes(void);

#ifdef __cplusplus
}
#endif

#endif /* MJB200_H_ */
