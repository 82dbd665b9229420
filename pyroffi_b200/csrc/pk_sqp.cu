// SQP-IK on the GPU: multi-seed sequential quadratic programming IK with
// joint limits as hard bounds on the step -- the drop-in for the sqp_ik_cuda
// custom call (src/pyroffi/cuda_kernels/_sqp_ik_cuda_kernel.cu:70-460,
// handler :462-591).
//
// Per seed, max_iter iterations: residual and Jacobian of every EE; exit when
// all EEs are within (eps_pos, eps_ori); rows weighted by (pos_weight,
// ori_weight); Jacobi column scaling; H = Js^T Js + lambda I and g = Js^T f
// (FP64 in the reference); the step's box in scaled space,
// ((lower - q) s, (upper - q) s) (0 for fixed joints); the unconstrained
// Newton step by Cholesky, clamped to the box; n_inner active-set re-solves
// (joints at a bound are held there and the free ones re-solved against
// g + H p_bound); unscaling; the trust-region
// clip; a 5-point line search on the weighted error plus the collision
// penalty (first minimum); accept with lambda x0.5 / reject x3; all-time
// best tracking.
//
// The reference kernel's FK takes no mimic or topological-order arrays; the
// FK here is the general one, which agrees with it on robots without mimic
// joints whose joints are listed parent first.
//
// B200 mapping: 32 seeds of one problem per block of 128 threads, 4 lanes
// per seed.  The lanes of a seed hold the same state and compute the same
// step; they split the collision penalty over the obstacles (robot spheres
// grouped by joint, with exact bounding-sphere culling at the margin).  Each
// solve of the step is FP32 with one conditional FP64 refinement step
// (damped_step_f32: the 6 n_ee x 6 n_ee dual system for one or two EEs, the
// normal equations for more).
#include "pk_damped_step.cuh"
#include "pk_seed_ik.cuh"

namespace pk {

constexpr int kSqpThreads = 128;
constexpr int kSqpTps = 4;

// Weighted squared error plus collision penalty at the joint poses in `ps`.
template <int MAXEE, int TPS>
__device__ __forceinline__ float sqp_error(const SeedIkArgs& a, const SeedIkShared& sh, const PoseSlots& ps,
                                           const RobotSpheresS& R, const ObsView& ob, int gl, unsigned gmask,
                                           float (&r)[6 * MAXEE], float (&pee)[3 * MAXEE]) {
  seed_ik_residual<MAXEE>(sh, ps, a.n_ee, 0, r, pee);
  float err = 0.f;
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k) {
    const float rw = r[k] * (k % 6 < 3 ? a.pos_weight : a.ori_weight);
    err += rw * rw;
  }
  return err + seed_ik_penalty<TPS>(a, ps, R, ob, gl, gmask);
}

// Box-constrained step of the current point (see the file comment).
template <int MAXA, int MAXEE>
__device__ __forceinline__ void sqp_direction(const SeedIkArgs& a, const SeedIkShared& sh, const PoseSlots& ps,
                                              const float (&r)[6 * MAXEE], const float (&pee)[3 * MAXEE],
                                              const float (&cfg)[MAXA], float lam, float (&delta)[MAXA]) {
  float J[6 * MAXEE][MAXA];
  seed_ik_jacobian<MAXA, MAXEE>(sh, ps, a.n_ee, pee, J);
  float fw[6 * MAXEE];
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k) {
    const float wk = k % 6 < 3 ? a.pos_weight : a.ori_weight;
    fw[k] = r[k] * wk;
#pragma unroll
    for (int c = 0; c < MAXA; ++c) J[k][c] *= wk;
  }
  float cs[MAXA];
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    float sq = 0.f;
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k) sq += J[k][c] * J[k][c];
    cs[c] = sqrtf(sq) + 1e-8f;
  }
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k)
#pragma unroll
    for (int c = 0; c < MAXA; ++c) J[k][c] = J[k][c] / cs[c];
  float lb[MAXA], ub[MAXA];
  bool fr[MAXA];
  float zero[MAXA], xn[MAXA], x[MAXA];
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    const bool fx = sh.fixed[c];
    lb[c] = fx ? 0.f : (sh.lo[c] - cfg[c]) * cs[c];
    ub[c] = fx ? 0.f : (sh.hi[c] - cfg[c]) * cs[c];
    zero[c] = 0.f;
  }
  // it = -1: the unconstrained Newton step (fixed joints masked), clamped to
  // the box; then n_inner active-set re-solves: joints at a bound stay there,
  // the rest re-solve against g + H p_bound, i.e. with the held joints as
  // fixed columns at p_bound.  One call site for all of them.
  constexpr int R = 6 * MAXEE;
  const int rows = 6 * a.n_ee;
  float p[MAXA];
  for (int it = -1; it < a.n_inner; ++it) {
    bool act[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) {
      act[c] = it < 0 ? (bool)sh.fixed[c] : (p[c] <= lb[c] + 1e-8f || p[c] >= ub[c] - 1e-8f);
      xn[c] = (it >= 0 && act[c]) ? clampf(p[c], lb[c], ub[c]) : 0.f;
      fr[c] = !act[c];
    }
    damped_step_f32<R, MAXA>(J, fw, rows, lam, zero, fr, xn, zero, x);
#pragma unroll
    for (int c = 0; c < MAXA; ++c) p[c] = act[c] ? xn[c] : clampf(x[c], lb[c], ub[c]);
  }
  float dn2 = 0.f, max_p = 0.f, max_o = 0.f;
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    delta[c] = p[c] / cs[c];
    dn2 += delta[c] * delta[c];
  }
#pragma unroll
  for (int e = 0; e < MAXEE; ++e) {
    if (e >= a.n_ee) continue;
    max_p = fmaxf(max_p, sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]));
    max_o = fmaxf(max_o,
                  sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]));
  }
  float Rt;
  if (max_p > 1e-2f || max_o > 0.6f) Rt = 0.38f;
  else if (max_p > 1e-3f || max_o > 0.25f) Rt = 0.22f;
  else if (max_p > 2e-4f || max_o > 0.08f) Rt = 0.12f;
  else Rt = 0.05f;
  const float dn = sqrtf(dn2);
  if (dn > Rt) {
    const float sc = Rt / (dn + 1e-18f);
#pragma unroll
    for (int c = 0; c < MAXA; ++c) delta[c] *= sc;
  }
}

template <int MAXA, int MAXEE, int TPS>
__global__ void __launch_bounds__(kSqpThreads) sqp_kernel(SeedIkArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SeedIkShared& sh = *reinterpret_cast<SeedIkShared*>(smem_raw);
  RobotSpheresS R = seed_ik_spheres_at(smem_raw + sizeof(SeedIkShared), a.n_rs, a.m.n_joints);
  float* world = reinterpret_cast<float*>(smem_raw + seed_ik_world_offset(a));
  float* slots = reinterpret_cast<float*>(smem_raw + seed_ik_slots_offset(a));
  const int tid = threadIdx.x, n = a.m.n_act, p = blockIdx.y;
  const int G = blockDim.x / TPS, grp = tid / TPS, gl = tid % TPS;
  const unsigned gmask = ((1u << TPS) - 1u) << ((tid & 31) & ~(TPS - 1));
  ObsView ob;
  seed_ik_stage(a, sh, R, world, ob, p, 1);
  const int s = blockIdx.x * G + grp;
  if (s >= a.S) return;  // the whole seed group
  const size_t gs = (size_t)p * a.S + s;
  const PoseSlots ps{slots + tid, (int)blockDim.x};
  const float alphas[5] = {1.f, 0.5f, 0.25f, 0.1f, 0.025f};
  float cfg[MAXA], best_cfg[MAXA];
#pragma unroll
  for (int c = 0; c < MAXA; ++c) cfg[c] = best_cfg[c] = c < n ? a.seeds[gs * n + c] : 0.f;
  auto cur_at = [&](int i) { return reg_at(cfg, i); };
  float r[6 * MAXEE], pee[3 * MAXEE];
  fk_thread(sh.jt, cur_at, ps);
  float best_err = sqp_error<MAXEE, TPS>(a, sh, ps, R, ob, gl, gmask, r, pee);
  float lam = a.lambda_init;
  for (int it = 0; it < a.iters; ++it) {
    fk_thread(sh.jt, cur_at, ps);
    seed_ik_residual<MAXEE>(sh, ps, a.n_ee, 0, r, pee);
    bool conv = true;
#pragma unroll
    for (int e = 0; e < MAXEE; ++e) {
      if (e >= a.n_ee) continue;
      const float pn = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
      const float on = sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
      if (pn >= a.eps_pos || on >= a.eps_ori) conv = false;
    }
    if (conv) break;
    const float curr = sqp_error<MAXEE, TPS>(a, sh, ps, R, ob, gl, gmask, r, pee);
    float delta[MAXA];
    sqp_direction<MAXA, MAXEE>(a, sh, ps, r, pee, cfg, lam, delta);
    float best_a_err = 1e30f;
    int best_ai = 0;
#pragma unroll 1
    for (int ai = 0; ai < 5; ++ai) {
      float trial[MAXA];
#pragma unroll
      for (int c = 0; c < MAXA; ++c) trial[c] = clampf(cfg[c] + alphas[ai] * delta[c], sh.lo[c], sh.hi[c]);
      fk_thread(sh.jt, [&](int i) { return reg_at(trial, i); }, ps);
      float rt[6 * MAXEE], pt[3 * MAXEE];
      const float et = sqp_error<MAXEE, TPS>(a, sh, ps, R, ob, gl, gmask, rt, pt);
      if (et < best_a_err) { best_a_err = et; best_ai = ai; }
    }
    float trial[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) trial[c] = clampf(cfg[c] + alphas[best_ai] * delta[c], sh.lo[c], sh.hi[c]);
    if (best_a_err < curr * (1.f - 1e-4f)) {
#pragma unroll
      for (int c = 0; c < MAXA; ++c) cfg[c] = trial[c];
      lam = fmaxf(lam * 0.5f, 1e-10f);
    } else {
      lam = fminf(lam * 3.f, 1e6f);
    }
    if (best_a_err < best_err) {
      best_err = best_a_err;
#pragma unroll
      for (int c = 0; c < MAXA; ++c) best_cfg[c] = trial[c];
    }
  }
  if (gl == 0) {
    for (int c = 0; c < n; ++c) a.out[gs * n + c] = reg_at(best_cfg, c);
    a.out_err[gs] = best_err;
  }
}

}  // namespace pk

using namespace pk;

namespace {

template <int MAXA, int MAXEE>
int launch_sqp(const SeedIkArgs& a, size_t smem, cudaStream_t st) {
  auto k = sqp_kernel<MAXA, MAXEE, kSqpTps>;
  if (int s = set_smem_limit((const void*)k, smem)) return s;
  constexpr int G = kSqpThreads / kSqpTps;
  const dim3 grid((unsigned)((a.S + G - 1) / G), (unsigned)a.P);
  k<<<grid, kSqpThreads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "sqp_kernel launch");
}

}  // namespace

extern "C" int pk_sqp_ik_cuda(void* stream, const float* seeds, const float* twists, const float* parent_tf,
                              const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                              const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                              const int32_t* target_jnts, const int32_t* ancestor_masks, const float* target_Ts,
                              const float* robot_spheres_local, const int32_t* robot_sphere_joint_idx,
                              const float* world_spheres, const float* world_capsules, const float* world_boxes,
                              const float* world_halfspaces, const float* lower, const float* upper,
                              const int32_t* fixed_mask, int64_t max_iter, int64_t n_inner_iters, float pos_weight,
                              float ori_weight, float lambda_init, float eps_pos, float eps_ori,
                              int64_t enable_collision, float collision_weight, float collision_margin, float* out,
                              float* out_err, int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints,
                              int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh) {
  SeedIkArgs a = seed_ik_args(seeds, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
                              topo_inv, target_jnts, ancestor_masks, target_Ts, robot_spheres_local,
                              robot_sphere_joint_idx, world_spheres, world_capsules, world_boxes, world_halfspaces,
                              lower, upper, fixed_mask, out, out_err, n_problems, n_seeds, n_act, n_joints, n_ee,
                              n_robot_spheres, Ms, Mc, Mb, Mh);
  PK_CHECK_ARG(max_iter >= 0 && max_iter < (1LL << 31), "bad max_iter");
  PK_CHECK_ARG(n_inner_iters >= 0 && n_inner_iters < (1LL << 31), "bad n_inner_iters");
  a.iters = (int)max_iter;
  a.n_inner = (int)n_inner_iters;
  a.pos_weight = pos_weight;
  a.ori_weight = ori_weight;
  a.lambda_init = lambda_init;
  a.eps_pos = eps_pos;
  a.eps_ori = eps_ori;
  a.enable_collision = enable_collision ? 1 : 0;
  a.collision_weight = collision_weight;
  a.collision_margin = collision_margin;
  size_t smem = 0;
  if (int s = seed_ik_common(a, n_act, n_joints, n_ee, kSqpThreads, &smem, true)) return s;
  if (n_problems == 0 || n_seeds == 0) return PK_OK;
  if (int s = seed_ik_check_buffers(a)) return s;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_act <= 8 && n_ee == 1) return launch_sqp<8, 1>(a, smem, st);
  if (n_ee <= 2) return launch_sqp<16, 2>(a, smem, st);
  return launch_sqp<16, 4>(a, smem, st);
}
