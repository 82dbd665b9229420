/*
 * pyroffi_b200 -- C-ABI of the B200 (sm_100a) kinematics hot path.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*, a cudaStream_t), launches on that stream and returns an
 * int status (PK_OK or a PK_ERR_* code; pk_last_error() gives the message of
 * the calling thread's last failure).  No entry point keeps a caller's
 * pointer after it returns, synchronises the stream, or allocates device
 * memory.  All arrays are row-major, float32 / int32, device-resident.
 *
 * The drop-in entry points mirror, argument for argument and in the same
 * order, the XLA FFI handlers of the reference (CoMMALab/pyroffi,
 * src/pyroffi/cuda_kernels/); the extents that an XLA buffer carries are
 * passed explicitly after the buffers.
 */
#ifndef PYROFFI_B200_H_
#define PYROFFI_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PK_OK 0
#define PK_ERR_INVALID 1   /* bad shape / index / argument (reference: kInvalidArgument) */
#define PK_ERR_CAPACITY 2  /* exceeds a compile-time capacity (joints, DOF, EEs, smem) */
#define PK_ERR_CUDA 3      /* a CUDA runtime call failed (reference: kInternal) */
#define PK_ERR_TIMEOUT 4   /* a bounded device-side wait ran out */

/* capacities */
#define PK_MAX_JOINTS_ABI 64
#define PK_MAX_ACT_ABI 32
#define PK_MAX_EE_ABI 4

/* Library version string; the calling thread's last error message; the text
 * of a status code (no reference counterpart: the reference's handlers return
 * an ffi::Error carrying the message). */
const char* pk_version(void);
const char* pk_last_error(void);
const char* pk_status_string(int status);

/*
 * Forward kinematics: world pose of every joint, out[B, n_joints, 7] wxyz_xyz.
 * Replaces the XLA FFI target "fk_cuda" (FkCudaFfi,
 * src/pyroffi/cuda_kernels/_fk_cuda_kernel.cu:236-471); argument order as in
 * its Bind() (:456-471): cfg[B,n_act], twists[n_j,6], parent_tf[n_j,7],
 * parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx, topo_inv [n_j],
 * fk_level_starts[n_levels+1], fk_level_joints[n_j].
 */
int pk_fk_cuda(void* stream, const float* cfg, const float* twists, const float* parent_tf,
               const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
               const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
               const int32_t* fk_level_starts, const int32_t* fk_level_joints, float* out,
               int64_t batch, int32_t n_act, int32_t n_joints, int32_t n_levels);

/*
 * World distances of robot spheres, out[B, K, M], M = Ms+Mc+Mb+Mh (spheres,
 * capsules, boxes, halfspaces in that order); spheres with radius < 0 give
 * 1e9.  Replaces "collision_world_sphere" (CollisionWorldSphereFfi,
 * src/pyroffi/cuda_kernels/_collision_cuda_kernel.cu:507-671).
 * centers[3,B,K] SoA, radii[B,K], ws[Ms,4], wc[Mc,7], wb[Mb,15], wh[Mh,6].
 */
int pk_collision_world_sphere(void* stream, const float* centers, const float* radii,
                              const float* world_spheres, const float* world_capsules,
                              const float* world_boxes, const float* world_halfspaces, float* out,
                              int64_t B, int32_t K, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * Per-link minimum over its S spheres (sphere k = s*N + n), out[B, N, M].
 * Replaces "collision_world_sphere_reduced" (CollisionWorldSphereReducedFfi,
 * _collision_cuda_kernel.cu:673-839); n = the int64 attribute "n".
 */
int pk_collision_world_sphere_reduced(void* stream, const float* centers, const float* radii,
                                      const float* world_spheres, const float* world_capsules,
                                      const float* world_boxes, const float* world_halfspaces,
                                      float* out, int64_t B, int32_t K, int32_t Ms, int32_t Mc,
                                      int32_t Mb, int32_t Mh, int64_t n);

/*
 * Capsule robot vs world, out[B, N, M]; caps[7,B,N] SoA (p1, p2, r).
 * Replaces "collision_world_capsule" (CollisionWorldCapsuleFfi,
 * _collision_cuda_kernel.cu:843-1004).
 */
int pk_collision_world_capsule(void* stream, const float* caps, const float* world_spheres,
                               const float* world_capsules, const float* world_boxes,
                               const float* world_halfspaces, float* out, int64_t B, int32_t N,
                               int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * Self distances, out[B, P] = min over all S x S sphere pairs of links
 * (pair_i[p], pair_j[p]); centers[B,S,N,3] AoS, radii[B,S,N]; padding
 * (radius < 0) skipped.  Replaces "collision_self_sphere"
 * (CollisionSelfSphereFfi, _collision_cuda_kernel.cu:1006-1111).
 */
int pk_collision_self_sphere(void* stream, const float* centers, const float* radii,
                             const int32_t* pair_i, const int32_t* pair_j, float* out, int64_t B,
                             int32_t S, int32_t N, int32_t P);

/*
 * Capsule self distances, out[B, P]; caps[B,N,7] AoS.  Replaces
 * "collision_self_capsule" (CollisionSelfCapsuleFfi,
 * _collision_cuda_kernel.cu:1114-1214).
 */
int pk_collision_self_capsule(void* stream, const float* caps, const int32_t* pair_i,
                              const int32_t* pair_j, float* out, int64_t B, int32_t N, int32_t P);

/*
 * Multi-seed Levenberg-Marquardt IK, out_cfg[P, Sd, n_act] (best config per
 * seed) and out_err[P, Sd] (its weighted squared error incl. the collision
 * penalty).  Replaces "ls_ik_cuda" (LsIkCudaFfi,
 * src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:400-529): arguments in the
 * order of its Bind() (:493-529), attributes max_iter .. collision_margin
 * after the buffers, then the extents.  Damping factors are the reference's
 * x0.5 on accept, x3 on reject.
 */
int pk_ls_ik_cuda(void* stream, const float* seeds, const float* twists, const float* parent_tf,
                  const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                  const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                  const int32_t* target_jnts, const int32_t* ancestor_masks, const float* target_Ts,
                  const float* robot_spheres_local, const int32_t* robot_sphere_joint_idx,
                  const float* world_spheres, const float* world_capsules, const float* world_boxes,
                  const float* world_halfspaces, const float* lower, const float* upper,
                  const int32_t* fixed_mask, int64_t max_iter, float pos_weight, float ori_weight,
                  float lambda_init, float eps_pos, float eps_ori, int64_t enable_collision,
                  float collision_weight, float collision_margin, float* out_cfg, float* out_err,
                  int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints,
                  int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc, int32_t Mb,
                  int32_t Mh);

/* Options of the extended LM entry point (no reference counterpart). */
typedef struct pk_lm_options {
  int32_t max_iter;
  float pos_weight;
  float ori_weight;
  float lambda_init;
  float lambda_down;      /* multiply lambda on accept (reference 0.5) */
  float lambda_up;        /* multiply lambda on reject (reference 3.0) */
  float eps_pos;
  float eps_ori;
  int32_t enable_collision;
  float collision_weight;
  float collision_margin;
  int32_t threads_per_seed; /* 0 = default (1 lane; 128 seeds per block up to 8 DOF / 1 EE, 96 up to 16 DOF /
                              2 EEs); 1, 2, 4, 8 = lanes sharing one seed; 5 = one lane per line-search
                              trial; 16, 32 = warp-per-seed body with that many lanes per seed */
  int32_t seeds_per_block;  /* 0 = choose automatically */
  int32_t lanes_per_wide_seed; /* warp-per-seed body: lanes per seed, 16 (0 = default) or 32 */
  int32_t fp64_solve;       /* the damped step is solved through its 6 n_ee x 6 n_ee dual system
                              (Js Js^T + lambda I) y = fw, p = -Js^T y.  0 = FP32 system and Cholesky, with one
                              FP64 iterative-refinement step when the squared ratio of the largest to the
                              smallest pivot exceeds 1e6 (default); 1 = FP64, the precision of the reference's
                              normal equations (seed-group kernel: n_act <= 16, n_ee <= 2, threads_per_seed 0 or
                              1; PK_ERR_INVALID elsewhere, pk_ik_batch included).  With fewer free columns than
                              6 n_ee rows (fixed joints) the n_act x n_act primal system is solved instead, in the
                              same precision.  The warp-per-seed body (more than 16 DOF or 2 EEs) always takes
                              the FP32 form */
  int32_t obstacle_grid;    /* the LM kernels' obstacle tile: the world spheres are binned into a uniform grid of
                              this many cells per axis, built per block in shared memory, and each joint's
                              bounding sphere tests only its cell's list; 0 = default (14 for up to 160 world
                              spheres, 12 for up to 1024, else 8; the launch keeps 8 where the finer grid's
                              shared memory would lower the blocks or seeds resident per SM), 1..16 = that many,
                              -1 = no grid (every obstacle takes the bounding test).  A grid finer than 8 whose
                              lists overflow their capacity falls back to 8 cells per axis.  With one
                              lane per seed the results do not depend on it (each joint's hinge terms are summed
                              in increasing obstacle order); lanes sharing a seed and the warp-per-seed body take
                              the candidates by list position, so their sums may round differently */
} pk_lm_options;

/*
 * Extended LM IK (a new target, not a drop-in; it extends ls_ik_cuda,
 * src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:493-529): as pk_ls_ik_cuda plus
 * explicit robot-sphere self-collision pairs (self_i, self_j index
 * robot_spheres_local, hinge-squared with the same margin and weight),
 * configurable damping factors and launch shape.  target_Ts[P, n_ee, 7].
 */
int pk_ls_ik_ex(void* stream, const pk_lm_options* opt, const float* seeds, const float* twists,
                const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                const int32_t* topo_inv, const int32_t* target_jnts, const int32_t* ancestor_masks,
                const float* target_Ts, const float* robot_spheres_local,
                const int32_t* robot_sphere_joint_idx, const float* world_spheres,
                const float* world_capsules, const float* world_boxes,
                const float* world_halfspaces, const int32_t* self_i, const int32_t* self_j,
                const float* lower, const float* upper, const int32_t* fixed_mask, float* out_cfg,
                float* out_err, int32_t n_problems, int32_t n_seeds, int32_t n_act,
                int32_t n_joints, int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc,
                int32_t Mb, int32_t Mh, int32_t n_self_pairs);

/*
 * One robot class of a batched IK call (no reference counterpart).  The
 * model, target and sphere arrays are those of pk_ls_ik_ex for this robot;
 * seeds and outputs are laid out [n_problems, seed_stride, n_act] and
 * [n_problems, seed_stride], so problems may use fewer seeds than the
 * stride (unused slots are neither read nor written).
 *   body 0: seed-group kernel (n_act <= 8, n_ee == 1; lanes per seed and
 *           seeds per block from pk_lm_options);
 *   body 1: one warp per seed with its state in shared memory
 *           (n_act <= 32, n_ee <= 4);
 *   body 2: seed-group kernel, one lane per seed, 96 seeds per block
 *           (n_act <= 16, n_ee <= 2).
 */
typedef struct pk_ik_class {
  const float* twists;
  const float* parent_tf;
  const int32_t* parent_idx;
  const int32_t* act_idx;
  const float* mimic_mul;
  const float* mimic_off;
  const int32_t* mimic_act_idx;
  const int32_t* topo_inv;
  int32_t n_joints;
  int32_t n_act;
  const int32_t* target_jnts;     /* [n_ee] */
  const int32_t* ancestor_masks;  /* [n_ee, n_joints] */
  const float* target_Ts;         /* [n_problems, n_ee, 7] */
  int32_t n_ee;
  const float* robot_spheres_local;       /* [n_robot_spheres, 4] */
  const int32_t* robot_sphere_joint_idx;  /* [n_robot_spheres] */
  int32_t n_robot_spheres;
  const int32_t* self_i;          /* [n_self] robot-sphere index pairs, or null */
  const int32_t* self_j;
  int32_t n_self;
  const float* lower;             /* [n_act] */
  const float* upper;
  const int32_t* fixed_mask;
  const float* seeds;             /* [n_problems, seed_stride, n_act] */
  float* out_cfg;                 /* [n_problems, seed_stride, n_act] */
  float* out_err;                 /* [n_problems, seed_stride] */
  int32_t n_problems;
  int32_t seed_stride;
  int32_t body;
} pk_ik_class;

/*
 * Batched LM IK over several robot classes sharing one world (no reference
 * counterpart): the persistent form of pk_ls_ik_ex.  items[n_items][4] =
 * (class, problem, first seed, seed count) in device memory, in the order
 * blocks should take them (longest first balances the tail); a body-0 item
 * holds at most seeds_per_block seeds (128 when that is 0 and
 * threads_per_seed is 0 or 1), a body-2 item at most 96.  Each body runs
 * one persistent kernel whose blocks take items from a device counter in
 * queue[2] (caller-owned device memory; cleared here with async memsets on
 * `stream` before the launches, so one queue serves one call in flight at
 * a time; bodies 0 and 2 use queue[0] one after the other).  blocks = 0
 * sizes each grid to one full wave on the current device.  Same per-seed
 * iteration and outputs as pk_ls_ik_ex with opt.
 */
int pk_ik_batch(void* stream, const pk_lm_options* opt, const pk_ik_class* classes, int32_t n_classes,
                const float* world_spheres, const float* world_capsules, const float* world_boxes,
                const float* world_halfspaces, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh,
                const int32_t* items, int32_t n_items, int32_t* queue, int32_t blocks);

/*
 * pk_ik_batch for callers that cannot allocate device memory when they
 * solve (a handler inside a runtime that owns the device memory and gives
 * this call no workspace, a real-time loop that must not allocate once it
 * runs).  No counterpart in the reference.  Same arguments and results as
 * pk_ik_batch without `queue`: the two work-queue counters live in a
 * 256-byte array compiled into the library (it stays on every GPU that
 * loaded the library until the process exits).  Every call looks up that
 * array's device address in the current context (cudaGetSymbolAddress; the
 * address is per context, so it is not cached), and the first call in a
 * context loads the library's device code, so make that first call before
 * any stream capture.  Every call shares the array and clears the counters
 * on `stream` before it starts: calls whose kernels overlap on the GPU
 * (different streams, or different host threads) race on the counters and
 * must be serialised by the caller.  Allocates nothing.
 */
int pk_ik_batch_static(void* stream, const pk_lm_options* opt, const pk_ik_class* classes, int32_t n_classes,
                       const float* world_spheres, const float* world_capsules, const float* world_boxes,
                       const float* world_halfspaces, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh,
                       const int32_t* items, int32_t n_items, int32_t blocks);

/*
 * FP64 re-verification and winner selection (no reference counterpart; it
 * replaces the argmin of _ls_ik_solve_cuda_batch_jit,
 * src/pyroffi/optimization_engines/_ls_ik.py:974-999, and the FP64 check of
 * tests/bench_ik.py:341-353).  For every problem p: the winner seed is
 * argmin_s err[p,s] + continuity_weight * ||cfg[p,s] - prev[p]||^2 (prev may
 * be NULL); its configuration goes to winner_cfg[P, n_act]; FK of the
 * winner's configuration in FP64 gives, for EE 0, pos_err[P] (m) and
 * rot_err[P] (rad, ||log(R_tgt^-1 R)||), and success[P] = pos_err < pos_tol
 * && rot_err < rot_tol.  Any of pos_err / rot_err / success may be NULL.
 */
int pk_ik_verify_select(void* stream, const float* cfgs, const float* errs, const float* prev,
                        float continuity_weight, const float* twists, const float* parent_tf,
                        const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                        const float* mimic_off, const int32_t* mimic_act_idx,
                        const int32_t* topo_inv, const int32_t* target_jnts,
                        const float* target_Ts, float pos_tol, float rot_tol, float* winner_cfg,
                        double* pos_err, double* rot_err, int32_t* success, int32_t n_problems,
                        int32_t n_seeds, int32_t n_act, int32_t n_joints, int32_t n_ee);

/*
 * Fused FK -> link poses -> sphere world centres -> world distances (no
 * reference counterpart; it fuses Robot.forward_kinematics,
 * src/pyroffi/_robot.py:66-109, RobotCollisionSpherized.at_config,
 * src/pyroffi/collision/_robot_collision.py:744-794, and the world-distance
 * kernels).  Spheres are given per link in link frames: link_spheres[N, S, 4]
 * (x, y, z, r; r < 0 = padding), parent_joint_indices[N] (-1 = base link,
 * identity pose).  Outputs (each may be NULL):
 *   min_dist[B]          min over all spheres and obstacles (1e9 if none),
 *   link_poses[B, N, 7]  link poses,
 *   dist_bkm[B, K, M]    per-sphere distances with K = S*N, k = s*N + n, in
 *                        the layout of pk_collision_world_sphere,
 *   dist_bnm[B, N, M]    per-link minimum over the link's spheres, in the
 *                        layout of pk_collision_world_sphere_reduced,
 *   sphere_centers[B, K, 4]  each sphere's world centre and radius (the
 *                        output of at_config), k = s*N + n as in dist_bkm,
 *                        16-byte aligned; padded spheres keep r < 0.
 */
int pk_fk_sphere_collision(void* stream, const float* cfg, const float* twists,
                           const float* parent_tf, const int32_t* parent_idx,
                           const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                           const int32_t* mimic_act_idx, const int32_t* topo_inv,
                           const int32_t* parent_joint_indices, const float* link_spheres,
                           const float* world_spheres, const float* world_capsules,
                           const float* world_boxes, const float* world_halfspaces,
                           float* min_dist, float* link_poses, float* dist_bkm, float* dist_bnm,
                           float* sphere_centers, int64_t batch,
                           int32_t n_act, int32_t n_joints, int32_t n_links, int32_t S, int32_t Ms,
                           int32_t Mc, int32_t Mb, int32_t Mh);

/* Weights of the trajectory cost (no reference counterpart; the defaults of
 * ChompTrajOptConfig, src/pyroffi/optimization_engines/_chomp_optimization.py:31-91,
 * are margin 0.01, w_smooth 1, w_acc 0.5, w_jerk 0.1, w_limits 1, w_coll 3). */
typedef struct pk_traj_options {
  float margin;
  float w_smooth;
  float w_acc;
  float w_jerk;
  float w_limits;
  float w_coll;
  const uint8_t* active;   /* optional (NULL: every trajectory): trajectory b is evaluated only when
                              active[b % active_period] != 0, and its outputs are left as they were otherwise
                              (an optimiser's finished trajectories, its trial copies included) */
  int64_t active_period;
} pk_traj_options;

/*
 * CHOMP trajectory cost and its gradient (hand-written adjoint; no
 * reference counterpart -- it replaces jax.value_and_grad of cost_fn,
 * _chomp_optimization.py:243-263, and the finite-difference gradients of
 * _chomp_trajopt_cuda_kernel.cu:719-784).  traj[B, T, n_act]; robot
 * spheres per link in link frames link_spheres[N, S, 4] (r < 0 padding),
 * parent_joint_indices[N]; active self link pairs (pair_i, pair_j)[P];
 * world obstacles as elsewhere; lower/upper[n_act].  Outputs (each may be
 * NULL, not all): cost[B]; grad[B, T, n_act] = dJ/dtraj (the collision
 * part recomputes the link poses, nothing is kept from a forward call);
 * wp_coll[B, T] the unweighted collision hinge per waypoint.
 */
int pk_traj_cost_grad(void* stream, const pk_traj_options* opt, const float* traj, const float* twists,
                      const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                      const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                      const int32_t* topo_inv, const int32_t* parent_joint_indices,
                      const float* link_spheres, const int32_t* pair_i, const int32_t* pair_j,
                      const float* world_spheres, const float* world_capsules, const float* world_boxes,
                      const float* world_halfspaces, const float* lower, const float* upper, float* cost,
                      float* grad, float* wp_coll, int64_t B, int32_t T, int32_t n_act, int32_t n_joints,
                      int32_t n_links, int32_t S, int32_t P, int32_t Ms, int32_t Mc, int32_t Mb,
                      int32_t Mh);

/*
 * CHOMP descent direction (no reference counterpart; it replaces the
 * clipping and covariant-update steps of chomp_trajopt,
 * src/pyroffi/optimization_engines/_chomp_optimization.py:155-241, 297-318):
 * per trajectory of grad[B, T, n_act], g * min(1, clip / |g|) (no clip when
 * grad_clip_norm <= 0), ends set to 0, then dir = -M^-1 g on every joint's
 * interior timeline by n_cg_iters truncated FP64 CG steps (relative
 * tolerance cg_tol) on M x = 6x + reg x - 4(x[t-1] + x[t+1]) + x[t-2] + x[t+2];
 * covariant = 0 gives dir = -g.  At most 128 interior waypoints.  active[B]
 * (optional, NULL = all): trajectories with active[b] == 0 are skipped and
 * their dir rows left as they were.
 */
int pk_chomp_direction(void* stream, const float* grad, float* dir, int64_t B, int32_t T, int32_t n_act,
                       int32_t n_cg_iters, float grad_clip_norm, float smoothness_reg, float cg_tol,
                       int32_t covariant, const uint8_t* active);

/*
 * CHOMP line search, trial trajectories (no reference counterpart; it fuses
 * the trial update of chomp_trajopt,
 * src/pyroffi/optimization_engines/_chomp_optimization.py:282-291):
 * trials[k, b] = traj[b] + clamp(alphas[k] * dir[b], -max_delta, max_delta)
 * for k < n_alphas, waypoint 0 set to start[n_act] and waypoint T-1 to goal.
 * trials is [n_alphas, B, T, n_act]; alphas is a device array.  active[B]
 * (optional, NULL = all): the trials of trajectories with active[b] == 0
 * are not written.
 */
int pk_chomp_line_trials(void* stream, const float* traj, const float* dir, const float* alphas, int32_t n_alphas,
                         float max_delta, const float* start, const float* goal, float* trials, int64_t B,
                         int32_t T, int32_t n_act, const uint8_t* active);

/*
 * CHOMP line search, selection (no reference counterpart; it fuses the
 * selection and early stop of chomp_trajopt,
 * src/pyroffi/optimization_engines/_chomp_optimization.py:293-304): per
 * trajectory, the first minimum over trial_costs[n_alphas, B] and cost[B]
 * (the zero step); when active[b] and that minimum is below
 * cost[b] - min_cost_improve, traj[b] takes the winning trial.  An active
 * trajectory's stall counter resets on improvement and counts otherwise,
 * and it stays active while stall < early_stop_patience.  traj, active and
 * stall are updated in place.
 */
int pk_chomp_line_select(void* stream, const float* trial_costs, const float* cost, const float* trials, float* traj,
                         uint8_t* active, int32_t* stall, int32_t n_alphas, float min_cost_improve,
                         int32_t early_stop_patience, int64_t B, int32_t T, int32_t n_act);

/*
 * Health check (no reference counterpart; the reference's kernels do not wait
 * on the copy engine).  *count = the number of thread blocks, since the
 * library was loaded or since pk_stage_wait_reset, whose bounded wait for the
 * TMA copy of the obstacle arrays into shared memory ran out of time, on the
 * current device.  Returns PK_OK when that number is 0 and PK_ERR_TIMEOUT
 * otherwise.  Such a block counts itself, waits once more and copies the
 * arrays with plain loads, so its own results stay right; if that second
 * wait runs out too, the block finishes with the copy possibly in flight,
 * the copy may land in a later block's shared memory, and pk_last_error()
 * then says that outputs since then are untrusted.  Each wait is limited by
 * the GPU's global timer (1 s unless pk_stage_wait_configure says otherwise).
 * The counters are read with synchronous copies, so call this between
 * workloads, not inside one.
 */
int pk_stage_wait_timeouts(uint64_t* count);

/* Zeroes the counters behind pk_stage_wait_timeouts on the current device
 * (synchronous; no reference counterpart). */
int pk_stage_wait_reset(void);

/*
 * Test hook and time limit of the bounded wait (no reference counterpart).
 * force_timeout = 1 makes every block of the kernels that stage the obstacle
 * arrays skip the TMA copy, wait out the limit and take the plain-load path
 * (nothing is then in flight, so results equal the normal path's bit for
 * bit); 0 restores the copy.  limit_ns bounds each wait by the GPU's global
 * timer (<= 0: 1 s).  Synchronous; affects later launches on the current
 * device, in every thread.
 */
int pk_stage_wait_configure(int32_t force_timeout, int64_t limit_ns);

/* SCO trajectory optimisation settings: the fields of ScoTrajOptConfig
 * (src/pyroffi/optimization_engines/_sco_optimization.py:52-104, defaults in
 * brackets) and the reference kernel's fd_eps attribute
 * (src/pyroffi/cuda_kernels/_sco_trajopt_cuda.py:152-163). */
typedef struct pk_sco_options {
  int32_t n_outer_iters;         /* [10] linearise-and-solve iterations */
  int32_t n_inner_iters;         /* [30] L-BFGS steps per outer iteration */
  int32_t m_lbfgs;               /* [6] L-BFGS history, 1..16 */
  float w_smooth;                /* [1.0] */
  float w_acc;                   /* [0.5] */
  float w_jerk;                  /* [0.1] */
  float w_limits;                /* [1.0] */
  float w_trust;                 /* [0.5] */
  float w_collision;             /* [1.0] first outer iteration's collision weight */
  float w_collision_max;         /* [100.0] cap of the continuation and weight of the final ranking */
  float penalty_scale;           /* [3.0] */
  float collision_margin;        /* [0.01] */
  float smooth_min_temperature;  /* [0.05] */
  float fd_eps;                  /* 0: analytic Jacobians; > 0: central differences with this step
                                    (the reference kernel uses 1e-4) */
  int32_t self_all_pairs;        /* 1: a self pair's distance is the minimum over all sphere pairs
                                    (the reference kernel); 0: over equal sphere indices (the JAX
                                    compute_self_collision_distance) */
  int32_t inner_threads;         /* threads per trajectory in the inner solve; 0 = automatic */
} pk_sco_options;

/*
 * SCO linearisation (replaces _compute_coll_dists_and_jacs,
 * _sco_optimization.py:258-289, and the finite differences of
 * _sco_trajopt_cuda_kernel.cu:700-757).  For each of C configurations
 * cfg[C, n_act]: dist[C, 5] the smooth-min distances of the groups (self,
 * world spheres, capsules, boxes, halfspaces; 1e10 for a group without
 * pairs), jac[C, 5, n_act] their analytic Jacobians, coll[C] the sum of
 * -colldist_from_sdf(d, margin) over every self pair and (link, obstacle)
 * pair distance.  Any output may be NULL (not all).  Link and world arrays as
 * for pk_traj_cost_grad.
 */
int pk_sco_linearize(void* stream, const pk_sco_options* opt, const float* cfg, const float* twists,
                     const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                     const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                     const int32_t* topo_inv, const int32_t* parent_joint_indices, const float* link_spheres,
                     const int32_t* pair_i, const int32_t* pair_j, const float* world_spheres,
                     const float* world_capsules, const float* world_boxes, const float* world_halfspaces,
                     float* dist, float* jac, float* coll, int64_t C, int32_t n_act, int32_t n_joints,
                     int32_t n_links, int32_t S, int32_t P, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * SCO inner solve (replaces _lbfgs_inner_solve, _sco_optimization.py:296-448,
 * and _sco_trajopt_cuda_kernel.cu:759-888): for each trajectory traj[B, T,
 * n_act] (the linearisation point), n_inner_iters L-BFGS steps on the convex
 * model with dist[B, T, 5], jac[B, T, 5, n_act] and collision weight w_coll;
 * traj is overwritten with the best iterate, endpoints set to start / goal.
 * hist[B, 2, m_lbfgs, T, n_act] holds the L-BFGS history when it does not fit
 * in shared memory (NULL otherwise; PK_ERR_INVALID when it is needed).
 */
int pk_sco_inner(void* stream, const pk_sco_options* opt, float* traj, const float* dist, const float* jac,
                 const float* lower, const float* upper, const float* start, const float* goal, float* hist,
                 float w_coll, int64_t B, int32_t T, int32_t n_act);

/* Nonlinear ranking cost (replaces _eval_cost, _sco_optimization.py:455-474):
 * cost[b] = w_smooth (w_acc acc^2 + w_jerk jerk^2) + w_limits limits +
 * w_collision_max sum_t coll[b, t], with coll from pk_sco_linearize. */
int pk_sco_final_cost(void* stream, const pk_sco_options* opt, const float* traj, const float* coll,
                      const float* lower, const float* upper, float* cost, int64_t B, int32_t T, int32_t n_act);

/* Bytes of device workspace pk_sco_trajopt needs for (B, T, n_act) (no
 * reference counterpart: the reference's XLA call allocates its own). */
int pk_sco_workspace_bytes(const pk_sco_options* opt, int64_t B, int32_t T, int32_t n_act, size_t* bytes);

/*
 * Whole SCO optimisation (replaces the ScoTrajoptCudaFfi custom call,
 * src/pyroffi/cuda_kernels/_sco_trajopt_cuda_kernel.cu:1094-1307, bound by
 * _sco_trajopt_cuda.py:152-300): pins init_trajs[B, T, n_act] to start /
 * goal, runs n_outer_iters x (linearise, inner solve, weight continuation)
 * and writes out_trajs[B, T, n_act] and the ranking costs out_costs[B]; the
 * caller takes argmin(out_costs) as the best trajectory, as the reference
 * wrapper does.  workspace: pk_sco_workspace_bytes bytes, 256-byte aligned.
 * All launches go to `stream` and nothing allocates, so the call can be
 * captured in a CUDA graph.
 */
int pk_sco_trajopt(void* stream, const pk_sco_options* opt, const float* init_trajs, const float* start,
                   const float* goal, const float* twists, const float* parent_tf, const int32_t* parent_idx,
                   const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                   const int32_t* mimic_act_idx, const int32_t* topo_inv, const int32_t* parent_joint_indices,
                   const float* link_spheres, const int32_t* pair_i, const int32_t* pair_j,
                   const float* world_spheres, const float* world_capsules, const float* world_boxes,
                   const float* world_halfspaces, const float* lower, const float* upper, float* out_trajs,
                   float* out_costs, void* workspace, size_t workspace_bytes, int64_t B, int32_t T,
                   int32_t n_act, int32_t n_joints, int32_t n_links, int32_t S, int32_t P, int32_t Ms,
                   int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * HJCD-IK coarse phase: greedy coordinate descent on every seed.  Replaces
 * "hjcd_ik_coarse_cuda" (HjcdIkCoarseCudaFfi,
 * src/pyroffi/cuda_kernels/_hjcd_ik_cuda_kernel.cu:91-321, handler :697-764):
 * buffers and attributes in the order of its Bind(), then the extents.
 * seeds[P, S, n_act], target_jnts[n_ee], ancestor_masks[n_ee, n_joints],
 * target_Ts[P, n_ee, 7], robot_spheres_local[n_rs, 4] with
 * robot_sphere_joint_idx[n_rs], fixed_mask[n_act] (int32, may be NULL).
 * Outputs out[P, S, n_act] and out_err[P, S] (unweighted squared error plus
 * collision_weight * sum (d - margin)^2 over sphere/obstacle pairs closer
 * than the margin).  At most 16 actuated joints and 4 EEs.
 */
int pk_hjcd_ik_coarse_cuda(void* stream, const float* seeds, const float* twists, const float* parent_tf,
                           const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                           const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                           const int32_t* target_jnts, const int32_t* ancestor_masks, const float* target_Ts,
                           const float* robot_spheres_local, const int32_t* robot_sphere_joint_idx,
                           const float* world_spheres, const float* world_capsules, const float* world_boxes,
                           const float* world_halfspaces, const float* lower, const float* upper,
                           const int32_t* fixed_mask, int64_t k_max, int64_t enable_collision,
                           float collision_weight, float collision_margin, float* out, float* out_err,
                           int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints, int32_t n_ee,
                           int32_t n_robot_spheres, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * HJCD-IK refinement: Levenberg-Marquardt with adaptive row weights, a soft
 * joint-limit prior, stall kicks from noise[P, S, max_iter, n_act] and
 * best-iterate tracking.  Replaces "hjcd_ik_lm_cuda" (HjcdIkLmCudaFfi,
 * _hjcd_ik_cuda_kernel.cu:324-695, handler :766-850): buffers and attributes
 * in the order of its Bind().  Outputs out[P, S, n_act] (best configuration
 * per seed), out_err[P, S] and stop_flag[P] (1 when a seed of the problem met
 * eps_pos / eps_ori; every seed of that problem then stops at the next
 * iteration).  At most 16 actuated joints and 4 EEs.
 */
int pk_hjcd_ik_lm_cuda(void* stream, const float* seeds, const float* noise, const float* twists,
                       const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                       const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                       const int32_t* topo_inv, const int32_t* target_jnts, const int32_t* ancestor_masks,
                       const float* target_Ts, const float* robot_spheres_local,
                       const int32_t* robot_sphere_joint_idx, const float* world_spheres,
                       const float* world_capsules, const float* world_boxes, const float* world_halfspaces,
                       const float* lower, const float* upper, const int32_t* fixed_mask, int64_t max_iter,
                       int64_t stall_patience, float lambda_init, float limit_prior_weight, float kick_scale,
                       float eps_pos, float eps_ori, int64_t enable_collision, float collision_weight,
                       float collision_margin, float* out, float* out_err, int32_t* stop_flag,
                       int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints, int32_t n_ee,
                       int32_t n_robot_spheres, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * SQP-IK: multi-seed sequential quadratic programming IK with the joint
 * limits as hard bounds on each step (box QP: Newton step, clamp,
 * n_inner_iters active-set re-solves), fixed row weights, 5-point line search,
 * best-iterate tracking.  Replaces "sqp_ik_cuda" (SqpIkCudaFfi,
 * src/pyroffi/cuda_kernels/_sqp_ik_cuda_kernel.cu:70-591): buffers and
 * attributes in the order of its Bind(), then the extents.  Outputs
 * out[P, S, n_act] and out_err[P, S] (weighted squared error plus the
 * collision penalty).  At most 16 actuated joints and 4 EEs.
 */
int pk_sqp_ik_cuda(void* stream, const float* seeds, const float* twists, const float* parent_tf,
                   const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                   const int32_t* mimic_act_idx, const int32_t* topo_inv, const int32_t* target_jnts,
                   const int32_t* ancestor_masks, const float* target_Ts, const float* robot_spheres_local,
                   const int32_t* robot_sphere_joint_idx, const float* world_spheres, const float* world_capsules,
                   const float* world_boxes, const float* world_halfspaces, const float* lower, const float* upper,
                   const int32_t* fixed_mask, int64_t max_iter, int64_t n_inner_iters, float pos_weight,
                   float ori_weight, float lambda_init, float eps_pos, float eps_ori, int64_t enable_collision,
                   float collision_weight, float collision_margin, float* out, float* out_err, int32_t n_problems,
                   int32_t n_seeds, int32_t n_act, int32_t n_joints, int32_t n_ee, int32_t n_robot_spheres,
                   int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh);

/*
 * FP32 FMA-pipe microbenchmark (no reference counterpart): `blocks` blocks of
 * 256 threads, each thread 8 independent FMA chains of `iters` steps, i.e.
 * 4096 * iters * blocks FLOPs.  Time it with events on `stream`; it gives
 * the measured SIMT roof the kinematics kernels are compared against.
 * `out` must hold `blocks` floats (normally left untouched).
 */
int pk_fp32_fma_peak(void* stream, float* out, int32_t iters, int32_t blocks);

#ifdef __cplusplus
}
#endif

#endif /* PYROFFI_B200_H_ */
