// HJCD-IK on the GPU: greedy coordinate-descent coarse search followed by
// Levenberg-Marquardt refinement with a joint-limit prior and stall kicks --
// the drop-in for the hjcd_ik_coarse_cuda / hjcd_ik_lm_cuda custom calls
// (src/pyroffi/cuda_kernels/_hjcd_ik_cuda_kernel.cu:91-695, bound by
// src/pyroffi/cuda_kernels/_hjcd_ik_cuda.py).
//
// Coarse phase (:91-321), per seed, k_max steps: stacked residual and
// Jacobian of every EE; row weights 1 (position) and
// clamp(|r_pos| / |r_ori|, 0.05, 1) (orientation, set to 0 while the EE is
// 1 mm or more away); of the free joints, the one with the largest predicted
// decrease (J_a^T f)^2 / |J_a|^2 takes the step -J_a^T f / |J_a|^2, clamped to
// the limits.  The score is the unweighted squared error plus the collision
// penalty.
//
// Refinement (:324-695), per seed, max_iter iterations: the same adaptive row
// weights (without gating), Jacobi column scaling, normal equations (FP64 in
// the reference) with LM damping and the soft joint-limit prior
// lpw / h^2 (q - mid), fixed joints masked, Cholesky (a non-positive pivot
// gives a zero step), the trust-region
// clip, a 5-point line search on the unweighted error (the first trial that
// is a new minimum and a sufficient decrease ends it), accept with lambda
// x0.5 / reject x3, all-time best tracking, and a Gaussian kick from the
// caller's noise after stall_patience rejections.  A seed whose EEs are all
// within (eps_pos, eps_ori) stops, and so do the other seeds of its problem
// from the next iteration on.
//
// B200 mapping.  Coarse: one thread per seed, grid (seed blocks, problems),
// robot, limits, world and robot spheres in shared memory, joint poses in
// per-thread shared slots.  Refinement: one 128-thread block per problem,
// four lanes per refinement seed (32 seeds at a time; the four lanes split
// the collision penalty); the problem's stop flag is a block vote
// (__syncthreads_or), so every seed of a problem stops at the same iteration
// and results do not depend on scheduling (the reference polls a global flag
// across blocks).
#include "pk_damped_step.cuh"
#include "pk_seed_ik.cuh"

namespace pk {

constexpr int kHjcdThreads = 128;  // refinement: one block per problem
constexpr int kHjcdTps = 4;        // refinement: lanes per seed (they split the collision penalty)

// ---------------------------------------------------------------------------
// coarse phase: one thread per seed
// ---------------------------------------------------------------------------

template <int MAXA, int MAXEE>
__global__ void __launch_bounds__(128) hjcd_coarse_kernel(SeedIkArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SeedIkShared& sh = *reinterpret_cast<SeedIkShared*>(smem_raw);
  RobotSpheresS R = seed_ik_spheres_at(smem_raw + sizeof(SeedIkShared), a.n_rs, a.m.n_joints);
  float* world = reinterpret_cast<float*>(smem_raw + seed_ik_world_offset(a));
  float* slots = reinterpret_cast<float*>(smem_raw + seed_ik_slots_offset(a));
  const int p = blockIdx.y, tid = threadIdx.x, n = a.m.n_act;
  ObsView ob;
  seed_ik_stage(a, sh, R, world, ob, p, 1);
  const int s = blockIdx.x * blockDim.x + tid;
  if (s >= a.S) return;
  const size_t gs = (size_t)p * a.S + s;
  const PoseSlots ps{slots + tid, (int)blockDim.x};
  float cfg[MAXA];
#pragma unroll
  for (int c = 0; c < MAXA; ++c) cfg[c] = c < n ? a.seeds[gs * n + c] : 0.f;
  auto cfg_at = [&](int i) { return reg_at(cfg, i); };
  float r[6 * MAXEE], pee[3 * MAXEE];
  float J[6 * MAXEE][MAXA];
  for (int it = 0; it < a.iters; ++it) {
    fk_thread(sh.jt, cfg_at, ps);
    seed_ik_residual<MAXEE>(sh, ps, a.n_ee, 0, r, pee);
    seed_ik_jacobian<MAXA, MAXEE>(sh, ps, a.n_ee, pee, J);
    // adaptive row weights, orientation gated off 1 mm or more from the target
    float fw[6 * MAXEE];
#pragma unroll
    for (int e = 0; e < MAXEE; ++e) {
      const float pn = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
      const float on = sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
      float wo = clampf((pn + 1e-8f) / (on + 1e-8f), 0.05f, 1.f);
      if (pn >= 1e-3f) wo = 0.f;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const float wk = k < 3 ? 1.f : wo;
        fw[6 * e + k] = r[6 * e + k] * wk;
#pragma unroll
        for (int c = 0; c < MAXA; ++c) J[6 * e + k][c] *= wk;
      }
    }
    int best = -1;
    float best_impr = -1.f, best_step = 0.f;
#pragma unroll
    for (int c = 0; c < MAXA; ++c) {
      float dot = 0.f, sq = 0.f;
#pragma unroll
      for (int k = 0; k < 6 * MAXEE; ++k) {
        dot += J[k][c] * fw[k];
        sq += J[k][c] * J[k][c];
      }
      sq += 1e-8f;
      const float impr = dot * dot / sq;
      if (!sh.fixed[c] && impr > best_impr) { best_impr = impr; best = c; best_step = -dot / sq; }
    }
    if (best < 0) break;
#pragma unroll
    for (int c = 0; c < MAXA; ++c)
      if (c == best) cfg[c] = clampf(cfg[c] + best_step, sh.lo[c], sh.hi[c]);
  }
  fk_thread(sh.jt, cfg_at, ps);
  seed_ik_residual<MAXEE>(sh, ps, a.n_ee, 0, r, pee);
  float err = 0.f;
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k) err += r[k] * r[k];
  err += seed_ik_penalty<1>(a, ps, R, ob, 0, 0u);
  a.out_err[gs] = err;
  for (int c = 0; c < n; ++c) a.out[gs * n + c] = reg_at(cfg, c);
}

// ---------------------------------------------------------------------------
// refinement: one warp per problem, one lane per seed
// ---------------------------------------------------------------------------

// Unweighted squared error plus penalty at the joint poses in `ps`.
template <int MAXEE, int TPS>
__device__ __forceinline__ float hjcd_error(const SeedIkArgs& a, const SeedIkShared& sh, const PoseSlots& ps,
                                            const RobotSpheresS& R, const ObsView& ob, int gl, unsigned gmask,
                                            float (&r)[6 * MAXEE], float (&pee)[3 * MAXEE]) {
  seed_ik_residual<MAXEE>(sh, ps, a.n_ee, 0, r, pee);
  float err = 0.f;
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k) err += r[k] * r[k];
  return err + seed_ik_penalty<TPS>(a, ps, R, ob, gl, gmask);
}

// LM step of the current point: adaptive row weights, Jacobi column scaling,
// the damped system with the joint-limit prior, fixed and padding columns
// masked, solved in FP32 with one conditional FP64 refinement step
// (damped_step_f32: its dual form for one or two EEs; zero step on a
// non-positive pivot), unscaling and the trust-region clip.
template <int MAXA, int MAXEE>
__device__ __forceinline__ void hjcd_direction(const SeedIkArgs& a, const SeedIkShared& sh, const PoseSlots& ps,
                                               const float (&r)[6 * MAXEE], const float (&pee)[3 * MAXEE],
                                               const float (&cfg)[MAXA], float lam, float (&delta)[MAXA]) {
  const int n_ee = a.n_ee;
  float J[6 * MAXEE][MAXA];
  seed_ik_jacobian<MAXA, MAXEE>(sh, ps, n_ee, pee, J);
  float fw[6 * MAXEE];
  float max_p = 0.f, max_o = 0.f;
#pragma unroll
  for (int e = 0; e < MAXEE; ++e) {
    const float pn = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
    const float on = sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
    if (e < n_ee) { max_p = fmaxf(max_p, pn); max_o = fmaxf(max_o, on); }
    const float wo = clampf((pn + 1e-8f) / (on + 1e-8f), 0.05f, 1.f);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float wk = k < 3 ? 1.f : wo;
      fw[6 * e + k] = r[6 * e + k] * wk;
#pragma unroll
      for (int c = 0; c < MAXA; ++c) J[6 * e + k][c] *= wk;
    }
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
  // the joint-limit prior w / h^2 (q - mid) in scaled columns: diagonal
  // w / (h^2 s^2), right-hand side w (q - mid) / (h^2 s)
  bool fr[MAXA];
  float pd[MAXA], v[MAXA], zero[MAXA], x[MAXA];
#pragma unroll
  for (int i = 0; i < MAXA; ++i) {
    fr[i] = !sh.fixed[i];
    zero[i] = 0.f;
    const float hr = (sh.hi[i] - sh.lo[i]) * 0.5f + 1e-8f;
    const float mid = (sh.lo[i] + sh.hi[i]) * 0.5f;
    const float dpr = a.limit_prior_weight / (hr * hr);
    pd[i] = fr[i] ? dpr / (cs[i] * cs[i]) : 0.f;
    v[i] = fr[i] ? dpr * (cfg[i] - mid) / cs[i] : 0.f;
  }
  const bool ok = damped_step_f32<6 * MAXEE, MAXA>(J, fw, 6 * n_ee, lam, pd, fr, zero, v, x);
  float dn2 = 0.f;
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    delta[c] = ok ? x[c] / cs[c] : 0.f;
    dn2 += delta[c] * delta[c];
  }
  float R;
  if (max_p > 1e-2f || max_o > 0.6f) R = 0.38f;
  else if (max_p > 1e-3f || max_o > 0.25f) R = 0.22f;
  else if (max_p > 2e-4f || max_o > 0.08f) R = 0.12f;
  else R = 0.05f;
  const float dn = sqrtf(dn2);
  if (dn > R) {
    const float sc = R / (dn + 1e-18f);
#pragma unroll
    for (int c = 0; c < MAXA; ++c) delta[c] *= sc;
  }
}

template <int MAXA, int MAXEE, int TPS>
__global__ void __launch_bounds__(kHjcdThreads) hjcd_lm_kernel(SeedIkArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SeedIkShared& sh = *reinterpret_cast<SeedIkShared*>(smem_raw);
  RobotSpheresS R = seed_ik_spheres_at(smem_raw + sizeof(SeedIkShared), a.n_rs, a.m.n_joints);
  float* world = reinterpret_cast<float*>(smem_raw + seed_ik_world_offset(a));
  float* slots = reinterpret_cast<float*>(smem_raw + seed_ik_slots_offset(a));
  const int tid = threadIdx.x, n = a.m.n_act, p = blockIdx.x;
  const int G = blockDim.x / TPS, grp = tid / TPS, gl = tid % TPS;
  const unsigned gmask = (TPS == 32 ? 0xffffffffu : ((1u << TPS) - 1u)) << ((tid & 31) & ~(TPS - 1));
  ObsView ob;
  seed_ik_stage(a, sh, R, world, ob, p, 1);
  const PoseSlots ps{slots + tid, (int)blockDim.x};
  const float alphas[5] = {1.f, 0.5f, 0.25f, 0.1f, 0.025f};
  bool stop = false;  // block-uniform: a seed of this problem has converged
  for (int s0 = 0; s0 < a.S; s0 += G) {
    const int s = s0 + grp;
    const bool live = s < a.S;
    const size_t gs = (size_t)p * a.S + (live ? s : 0);
    float cfg[MAXA], best_cfg[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) cfg[c] = best_cfg[c] = (live && c < n) ? a.seeds[gs * n + c] : 0.f;
    auto cur_at = [&](int i) { return reg_at(cfg, i); };
    float r[6 * MAXEE], pee[3 * MAXEE];
    float best_err = 0.f;
    if (live) {
      fk_thread(sh.jt, cur_at, ps);
      best_err = hjcd_error<MAXEE, TPS>(a, sh, ps, R, ob, gl, gmask, r, pee);
    }
    float lam = a.lambda_init;
    int stall = 0;
    bool done = !live || stop;
    for (int it = 0; it < a.iters; ++it) {
      if (stop) done = true;
      if (__syncthreads_and(done)) break;
      bool conv = false;
      float curr = 0.f;
      if (!done) {
        fk_thread(sh.jt, cur_at, ps);
        curr = hjcd_error<MAXEE, TPS>(a, sh, ps, R, ob, gl, gmask, r, pee);
        conv = true;
#pragma unroll
        for (int e = 0; e < MAXEE; ++e) {
          if (e >= a.n_ee) continue;
          const float pn = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
          const float on =
              sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
          if (pn >= a.eps_pos || on >= a.eps_ori) conv = false;
        }
      }
      if (__syncthreads_or(!done && conv)) stop = true;
      if (conv) done = true;
      if (done) continue;
      // the TPS lanes of a group hold the same state and compute the same step
      float delta[MAXA];
      hjcd_direction<MAXA, MAXEE>(a, sh, ps, r, pee, cfg, lam, delta);
      float best_a_err = 1e30f;
      int best_ai = 0;
      for (int ai = 0; ai < 5; ++ai) {
        float trial[MAXA];
#pragma unroll
        for (int c = 0; c < MAXA; ++c) trial[c] = clampf(cfg[c] + alphas[ai] * delta[c], sh.lo[c], sh.hi[c]);
        fk_thread(sh.jt, [&](int i) { return reg_at(trial, i); }, ps);
        float rt[6 * MAXEE], pt[3 * MAXEE];
        const float et = hjcd_error<MAXEE, TPS>(a, sh, ps, R, ob, gl, gmask, rt, pt);
        if (et < best_a_err) {
          best_a_err = et;
          best_ai = ai;
          if (et < curr * (1.f - 1e-4f)) break;
        }
      }
      float trial[MAXA];
#pragma unroll
      for (int c = 0; c < MAXA; ++c) trial[c] = clampf(cfg[c] + alphas[best_ai] * delta[c], sh.lo[c], sh.hi[c]);
      if (best_a_err < curr * (1.f - 1e-4f)) {
#pragma unroll
        for (int c = 0; c < MAXA; ++c) cfg[c] = trial[c];
        lam = fmaxf(lam * 0.5f, 1e-10f);
        stall = 0;
      } else {
        lam = fminf(lam * 3.f, 1e6f);
        ++stall;
      }
      if (best_a_err < best_err) {
        best_err = best_a_err;
#pragma unroll
        for (int c = 0; c < MAXA; ++c) best_cfg[c] = trial[c];
      }
      if (stall >= a.stall_patience) {
        const float* kn = a.noise + (gs * a.iters + it) * n;
#pragma unroll
        for (int c = 0; c < MAXA; ++c)
          if (c < n && !sh.fixed[c]) cfg[c] = clampf(cfg[c] + kn[c] * a.kick_scale, sh.lo[c], sh.hi[c]);
        lam = a.lambda_init;
        stall = 0;
      }
    }
    if (live && gl == 0) {
      for (int c = 0; c < n; ++c) a.out[gs * n + c] = reg_at(best_cfg, c);
      a.out_err[gs] = best_err;
    }
  }
  if (tid == 0 && a.stop_flag) a.stop_flag[p] = stop ? 1 : 0;
}

}  // namespace pk

using namespace pk;

namespace {

template <int MAXA, int MAXEE>
int launch_coarse(const SeedIkArgs& a, int nth, size_t smem, cudaStream_t st) {
  auto k = hjcd_coarse_kernel<MAXA, MAXEE>;
  if (int s = set_smem_limit((const void*)k, smem)) return s;
  const dim3 grid((unsigned)((a.S + nth - 1) / nth), (unsigned)a.P);
  k<<<grid, nth, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "hjcd_coarse_kernel launch");
}

template <int MAXA, int MAXEE>
int launch_lm(const SeedIkArgs& a, size_t smem, cudaStream_t st) {
  auto k = hjcd_lm_kernel<MAXA, MAXEE, kHjcdTps>;
  if (int s = set_smem_limit((const void*)k, smem)) return s;
  k<<<(unsigned)a.P, kHjcdThreads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "hjcd_lm_kernel launch");
}

}  // namespace

extern "C" int pk_hjcd_ik_coarse_cuda(void* stream, const float* seeds, const float* twists, const float* parent_tf,
                                      const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                                      const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                                      const int32_t* target_jnts, const int32_t* ancestor_masks,
                                      const float* target_Ts, const float* robot_spheres_local,
                                      const int32_t* robot_sphere_joint_idx, const float* world_spheres,
                                      const float* world_capsules, const float* world_boxes,
                                      const float* world_halfspaces, const float* lower, const float* upper,
                                      const int32_t* fixed_mask, int64_t k_max, int64_t enable_collision,
                                      float collision_weight, float collision_margin, float* out, float* out_err,
                                      int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints,
                                      int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc, int32_t Mb,
                                      int32_t Mh) {
  SeedIkArgs a = seed_ik_args(seeds, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
                         topo_inv, target_jnts, ancestor_masks, target_Ts, robot_spheres_local,
                         robot_sphere_joint_idx, world_spheres, world_capsules, world_boxes, world_halfspaces, lower,
                         upper, fixed_mask, out, out_err, n_problems, n_seeds, n_act, n_joints, n_ee,
                         n_robot_spheres, Ms, Mc, Mb, Mh);
  PK_CHECK_ARG(k_max >= 0 && k_max < (1LL << 31), "bad k_max");
  a.iters = (int)k_max;
  a.enable_collision = enable_collision ? 1 : 0;
  a.collision_weight = collision_weight;
  a.collision_margin = collision_margin;
  const int nth = n_seeds < 128 ? ((n_seeds + 31) / 32) * 32 : 128;
  size_t smem = 0;
  if (int s = seed_ik_common(a, n_act, n_joints, n_ee, nth < 32 ? 32 : nth, &smem)) return s;
  if (n_problems == 0 || n_seeds == 0) return PK_OK;
  if (int s = seed_ik_check_buffers(a)) return s;
  cudaStream_t st = (cudaStream_t)stream;
  const int t = nth < 32 ? 32 : nth;
  if (n_act <= 8 && n_ee == 1) return launch_coarse<8, 1>(a, t, smem, st);
  if (n_ee <= 2) return launch_coarse<16, 2>(a, t, smem, st);
  return launch_coarse<16, 4>(a, t, smem, st);
}

extern "C" int pk_hjcd_ik_lm_cuda(void* stream, const float* seeds, const float* noise, const float* twists,
                                  const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                                  const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                                  const int32_t* topo_inv, const int32_t* target_jnts, const int32_t* ancestor_masks,
                                  const float* target_Ts, const float* robot_spheres_local,
                                  const int32_t* robot_sphere_joint_idx, const float* world_spheres,
                                  const float* world_capsules, const float* world_boxes,
                                  const float* world_halfspaces, const float* lower, const float* upper,
                                  const int32_t* fixed_mask, int64_t max_iter, int64_t stall_patience,
                                  float lambda_init, float limit_prior_weight, float kick_scale, float eps_pos,
                                  float eps_ori, int64_t enable_collision, float collision_weight,
                                  float collision_margin, float* out, float* out_err, int32_t* stop_flag,
                                  int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints,
                                  int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc, int32_t Mb,
                                  int32_t Mh) {
  SeedIkArgs a = seed_ik_args(seeds, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
                         topo_inv, target_jnts, ancestor_masks, target_Ts, robot_spheres_local,
                         robot_sphere_joint_idx, world_spheres, world_capsules, world_boxes, world_halfspaces, lower,
                         upper, fixed_mask, out, out_err, n_problems, n_seeds, n_act, n_joints, n_ee,
                         n_robot_spheres, Ms, Mc, Mb, Mh);
  PK_CHECK_ARG(max_iter >= 0 && max_iter < (1LL << 31), "bad max_iter");
  PK_CHECK_ARG(stall_patience >= 1 && stall_patience < (1LL << 31), "stall_patience must be >= 1");
  a.noise = noise;
  a.stop_flag = stop_flag;
  a.iters = (int)max_iter;
  a.stall_patience = (int)stall_patience;
  a.lambda_init = lambda_init;
  a.limit_prior_weight = limit_prior_weight;
  a.kick_scale = kick_scale;
  a.eps_pos = eps_pos;
  a.eps_ori = eps_ori;
  a.enable_collision = enable_collision ? 1 : 0;
  a.collision_weight = collision_weight;
  a.collision_margin = collision_margin;
  size_t smem = 0;
  if (int s = seed_ik_common(a, n_act, n_joints, n_ee, kHjcdThreads, &smem, true)) return s;
  if (n_problems == 0) return PK_OK;
  PK_CHECK_ARG(n_seeds == 0 || max_iter == 0 || noise, "null noise");
  if (int s = seed_ik_check_buffers(a)) return s;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_seeds == 0) {
    if (stop_flag) return cuda_status(cudaMemsetAsync(stop_flag, 0, sizeof(int32_t) * n_problems, st), "memset");
    return PK_OK;
  }
  if (n_act <= 8 && n_ee == 1) return launch_lm<8, 1>(a, smem, st);
  if (n_ee <= 2) return launch_lm<16, 2>(a, smem, st);
  return launch_lm<16, 4>(a, smem, st);
}
