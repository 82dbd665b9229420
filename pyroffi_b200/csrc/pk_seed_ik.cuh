// Per-seed IK machinery shared by the HJCD and SQP kernels: arguments,
// block staging (robot, targets, limits, robot spheres grouped by joint with
// bounding spheres, world), EE residual, stacked Jacobian and the collision
// penalty with bounding-sphere culling, split over the lanes of a seed.
#pragma once

#include <float.h>

#include <algorithm>

#include "pk_obstacle_grid.cuh"
#include "pk_obstacles.cuh"

namespace pk {

struct SeedIkArgs {
  ModelArgs m;
  WorldArgs w;
  const float* seeds;          // [P, S, n]
  const float* noise;          // [P, S, iters, n] (refinement kicks)
  const int* target_jnts;      // [n_ee]
  const int* ancestor_masks;   // [n_ee, n_joints]
  const float* target_Ts;      // [P, n_ee, 7]
  const float* rs_local;       // [n_rs, 4] robot spheres in their joint frames
  const int* rs_joint;         // [n_rs]
  const float* lower;
  const float* upper;
  const int* fixed_mask;       // [n]
  float* out;                  // [P, S, n]
  float* out_err;              // [P, S]
  int* stop_flag;              // [P] or null
  int P, S, n_ee, n_rs, iters, stall_patience, enable_collision, stage_world;
  float collision_weight, collision_margin, lambda_init, limit_prior_weight, kick_scale, eps_pos, eps_ori;
  int n_inner;                 // SQP: active-set re-solves per step
  float pos_weight, ori_weight;  // SQP: fixed row weights
  int grid_entries;            // capacity of the sphere-obstacle grid's lists (0: no grid)
  int grid_n;                  // cells per axis the grid is allocated for
};

struct SeedIkShared {
  JointTable jt;
  float tgt[1][PK_MAX_EE][7];
  unsigned long long anc[PK_MAX_EE];  // ancestor joints of each EE (original indices)
  int tsorted[PK_MAX_EE];             // sorted position of each EE's joint
  float lo[PK_MAX_ACT], hi[PK_MAX_ACT];
  int fixed[PK_MAX_ACT];              // fixed or padding
  int n_groups;                       // joint groups of the robot spheres
  int grid_on;                        // the sphere-obstacle grid is built
  int grid_n;                         // its cells per axis
  float3 glo, ginv;                   // its origin and inverse cell size
};

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fmaxf(lo, fminf(hi, x)); }

// Robot spheres in shared memory, grouped by the joint that carries them,
// and the grid of world spheres within reach of a group's bounding sphere.
struct RobotSpheresS {
  float4* sph;     // [n_rs] joint-frame centre, radius; group k is gstart[k] .. gstart[k + 1]
  float4* bound;   // [nj] bounding sphere of each group (joint frame)
  int* start;      // [nj + 1] staging scratch
  int* gstart;     // [nj + 1]
  int* joint;      // [nj] sorted joint of each group
  int ng;
  const int* cell_start;            // obstacle grid (null: scan every world sphere)
  const unsigned short* cell_obs;
  float3 glo, ginv;
  int gn;                           // cells per axis
};

__host__ __device__ __forceinline__ size_t seed_ik_spheres_bytes(int n_rs, int nj) {
  return sizeof(float4) * ((size_t)n_rs + nj) + sizeof(int) * (3 * (size_t)nj + 2);
}

// Dynamic shared memory: SeedIkShared, robot spheres, the world (when staged),
// the obstacle grid (cell offsets, lists, scratch), then the pose slots.
__host__ __device__ inline size_t seed_ik_align16(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline size_t seed_ik_world_offset(const SeedIkArgs& a) {
  return seed_ik_align16(sizeof(SeedIkShared) + seed_ik_spheres_bytes(a.n_rs, a.m.n_joints));
}
__host__ __device__ inline size_t seed_ik_grid_offset(const SeedIkArgs& a) {
  return seed_ik_world_offset(a) + (a.stage_world ? sizeof(float) * a.w.smem_floats() : 0);
}
__host__ __device__ inline size_t seed_ik_grid_bytes(const SeedIkArgs& a) {
  if (!a.grid_entries) return 0;
  return seed_ik_align16(sizeof(int) * (obstacle_grid_cells(a.grid_n) + 1)) + seed_ik_align16(2 * (size_t)a.grid_entries) +
         seed_ik_align16(sizeof(int) * (size_t)a.w.Ms);
}
__host__ __device__ inline size_t seed_ik_slots_offset(const SeedIkArgs& a) {
  return seed_ik_grid_offset(a) + seed_ik_grid_bytes(a);
}

__device__ __forceinline__ RobotSpheresS seed_ik_spheres_at(unsigned char* p, int n_rs, int nj) {
  RobotSpheresS R;
  R.sph = reinterpret_cast<float4*>(p);
  R.bound = R.sph + n_rs;
  R.start = reinterpret_cast<int*>(R.bound + nj);
  R.gstart = R.start + nj + 1;
  R.joint = R.gstart + nj + 1;
  R.ng = 0;
  return R;
}

// Robot description, EE targets of `p0 + i` for i < n_tgt in slot i, limits,
// robot spheres (joint-frame centre and radius, sorted joint position) and
// optionally the world.  Ends with __syncthreads().
__device__ inline void seed_ik_stage(const SeedIkArgs& a, SeedIkShared& sh, RobotSpheresS& R, float* world_dst, ObsView& ob,
                           int p0, int n_tgt) {
  load_joint_table(sh.jt, a.m);
  const int n = a.m.n_act, nj = a.m.n_joints, tid = threadIdx.x, nth = blockDim.x;
  for (int e = tid; e < a.n_ee; e += nth) {
    unsigned long long m = 0ull;
    for (int j = 0; j < nj && j < 64; ++j)
      if (a.ancestor_masks[e * nj + j]) m |= 1ull << j;
    sh.anc[e] = m;
    const int tj = a.target_jnts[e];
    sh.tsorted[e] = (tj >= 0 && tj < nj) ? sh.jt.sorted_of[tj] : 0;
  }
  for (int i = tid; i < n_tgt * a.n_ee * 7; i += nth) {
    const int w = i / (a.n_ee * 7), r = i - w * a.n_ee * 7;
    const int p = p0 + w;
    sh.tgt[w][r / 7][r % 7] = p < a.P ? a.target_Ts[(size_t)p * a.n_ee * 7 + r] : 0.f;
  }
  for (int c = tid; c < PK_MAX_ACT; c += nth) {
    const bool live = c < n;
    sh.lo[c] = live ? a.lower[c] : 0.f;
    sh.hi[c] = live ? a.upper[c] : 0.f;
    sh.fixed[c] = live ? (a.fixed_mask ? a.fixed_mask[c] != 0 : 0) : 1;
  }
  __syncthreads();  // sorted_of is complete
  if (tid == 0) {
    // robot spheres grouped by (sorted) joint, in sphere order within a group;
    // spheres on an out-of-range joint are dropped
    for (int j = 0; j <= nj; ++j) R.start[j] = 0;
    for (int i = 0; i < a.n_rs; ++i) {
      const int j = a.rs_joint[i];
      if (j >= 0 && j < nj) ++R.start[sh.jt.sorted_of[j] + 1];
    }
    int ng = 0, off = 0;
    for (int j = 0; j < nj; ++j) {
      const int c = R.start[j + 1];
      if (c) { R.joint[ng] = j; R.gstart[ng] = off; ++ng; off += c; }
      R.start[j + 1] = off;  // fill cursor base: start[j] .. start[j + 1]
    }
    R.gstart[ng] = off;
    sh.n_groups = ng;
    // start[j] now holds where joint j's spheres begin: the fill cursor
    for (int i = 0; i < a.n_rs; ++i) {
      const int j = a.rs_joint[i];
      if (j < 0 || j >= nj) continue;
      const float* q = a.rs_local + 4 * i;
      R.sph[R.start[sh.jt.sorted_of[j]]++] = make_float4(q[0], q[1], q[2], q[3]);
    }
  }
  __syncthreads();
  R.ng = sh.n_groups;
  for (int k = tid; k < R.ng; k += nth) {
    // bounding sphere of group k in its joint frame; the slack keeps it
    // conservative under rounding
    float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
    for (int i = R.gstart[k]; i < R.gstart[k + 1]; ++i) {
      const float4 q = R.sph[i];
      lo[0] = fminf(lo[0], q.x); hi[0] = fmaxf(hi[0], q.x);
      lo[1] = fminf(lo[1], q.y); hi[1] = fmaxf(hi[1], q.y);
      lo[2] = fminf(lo[2], q.z); hi[2] = fmaxf(hi[2], q.z);
    }
    const float bx = 0.5f * (lo[0] + hi[0]), by = 0.5f * (lo[1] + hi[1]), bz = 0.5f * (lo[2] + hi[2]);
    float rad = 0.f;
    for (int i = R.gstart[k]; i < R.gstart[k + 1]; ++i) {
      const float4 q = R.sph[i];
      rad = fmaxf(rad, sqrtf((q.x - bx) * (q.x - bx) + (q.y - by) * (q.y - by) + (q.z - bz) * (q.z - bz)) + q.w);
    }
    R.bound[k] = make_float4(bx, by, bz, rad + 1e-4f + 1e-5f * fabsf(rad));
  }
  if (a.stage_world) {
    ob = stage_world(a.w, world_dst);
  } else {
    ob.sph = reinterpret_cast<const float4*>(a.w.spheres);
    ob.cap = a.w.capsules;
    ob.box = a.w.boxes;
    ob.hs = a.w.halfspaces;
    ob.Ms = a.w.Ms; ob.Mc = a.w.Mc; ob.Mb = a.w.Mb; ob.Mh = a.w.Mh;
  }
  __syncthreads();
  // world-sphere grid for queries by group bounding spheres: reach = the
  // largest bounding radius + the margin
  R.cell_start = nullptr;
  R.cell_obs = nullptr;
  if (a.grid_entries && R.ng > 0) {
    unsigned char* g = reinterpret_cast<unsigned char*>(world_dst) + (seed_ik_grid_offset(a) - seed_ik_world_offset(a));
    int* cell_start = reinterpret_cast<int*>(g);
    unsigned short* cell_obs =
        reinterpret_cast<unsigned short*>(g + seed_ik_align16(sizeof(int) * (obstacle_grid_cells(a.grid_n) + 1)));
    int* obox = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(cell_obs) +
                                       seed_ik_align16(2 * (size_t)a.grid_entries));
    float reach = 0.f;
    for (int k = 0; k < R.ng; ++k) reach = fmaxf(reach, R.bound[k].w);
    reach += a.collision_margin;
    if (tid == 0) {
      sh.grid_n = a.grid_n;
      obstacle_grid_bounds(ob.sph, ob.Ms, reach, sh.grid_n, sh.glo, sh.ginv);
      sh.grid_on = 1;
    }
    __syncthreads();
    obstacle_grid_build(ob.sph, ob.Ms, reach, sh.grid_n, sh.glo, sh.ginv, obox, cell_start, cell_obs, a.grid_entries,
                        sh.grid_on);
    // a fine grid whose lists overflow the capacity falls back to the default resolution
    if (!sh.grid_on && sh.grid_n > kObsGridDefault) {
      __syncthreads();
      if (tid == 0) {
        sh.grid_n = kObsGridDefault;
        obstacle_grid_bounds(ob.sph, ob.Ms, reach, sh.grid_n, sh.glo, sh.ginv);
        sh.grid_on = 1;
      }
      __syncthreads();
      obstacle_grid_build(ob.sph, ob.Ms, reach, sh.grid_n, sh.glo, sh.ginv, obox, cell_start, cell_obs,
                          a.grid_entries, sh.grid_on);
    }
    if (sh.grid_on) {
      R.cell_start = cell_start;
      R.cell_obs = cell_obs;
      R.glo = sh.glo;
      R.ginv = sh.ginv;
      R.gn = sh.grid_n;
    }
  }
}

// Residual of every EE against target slot `w`: world position difference and
// the rotation vector of q_ee conj(q_tgt) (w >= 0; 2 v below |v| = 1e-6).
template <int MAXEE>
__device__ __forceinline__ void seed_ik_residual(const SeedIkShared& sh, const PoseSlots& ps, int n_ee, int w,
                                              float (&r)[6 * MAXEE], float (&pee)[3 * MAXEE]) {
#pragma unroll
  for (int e = 0; e < MAXEE; ++e) {
    if (e >= n_ee) {
#pragma unroll
      for (int c = 0; c < 6; ++c) r[6 * e + c] = 0.f;
      pee[3 * e] = pee[3 * e + 1] = pee[3 * e + 2] = 0.f;
      continue;
    }
    const Pose T = ps.load(sh.tsorted[e]);
    const float* g = sh.tgt[w][e];
    r[6 * e + 0] = T.tx - g[4];
    r[6 * e + 1] = T.ty - g[5];
    r[6 * e + 2] = T.tz - g[6];
    const float bw = g[0], bx = -g[1], by = -g[2], bz = -g[3];
    float qw = T.w * bw - T.x * bx - T.y * by - T.z * bz;
    float qx = T.w * bx + T.x * bw + T.y * bz - T.z * by;
    float qy = T.w * by - T.x * bz + T.y * bw + T.z * bx;
    float qz = T.w * bz + T.x * by - T.y * bx + T.z * bw;
    if (qw < 0.f) { qw = -qw; qx = -qx; qy = -qy; qz = -qz; }
    const float s = sqrtf(qx * qx + qy * qy + qz * qz);
    const float f = s > 1e-6f ? 2.f * atan2f(s, qw) / s : 2.f;
    r[6 * e + 3] = qx * f;
    r[6 * e + 4] = qy * f;
    r[6 * e + 5] = qz * f;
    pee[3 * e] = T.tx; pee[3 * e + 1] = T.ty; pee[3 * e + 2] = T.tz;
  }
}

// Stacked geometric Jacobian J[k][c] (revolute z x (p_ee - p_j) / z,
// prismatic z / 0, times the mimic multiplier, restricted to each EE's
// ancestors).
template <int MAXA, int MAXEE>
__device__ __forceinline__ void seed_ik_jacobian(const SeedIkShared& sh, const PoseSlots& ps, int n_ee,
                                              const float (&pee)[3 * MAXEE], float (&J)[6 * MAXEE][MAXA]) {
  const JointTable& jt = sh.jt;
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k)
#pragma unroll
    for (int c = 0; c < MAXA; ++c) J[k][c] = 0.f;
  for (int i = 0; i < jt.n; ++i) {
    const int jk = jt.jkind[i];
    const int a1 = jt.a1[i], a2 = jt.a2[i];
    if (jk == 0 || (a1 < 0 && a2 < 0)) continue;
    const Pose Tj = ps.load(i);
    const float3 z = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z, make_float3(jt.axis[i][0], jt.axis[i][1], jt.axis[i][2]));
    const float sm = jt.mul[i];
    const int orig = jt.orig[i];
#pragma unroll
    for (int e = 0; e < MAXEE; ++e) {
      if (e >= n_ee || orig >= 64 || !((sh.anc[e] >> orig) & 1ull)) continue;
      float col[6];
      if (jk == 1) {
        const float ax = pee[3 * e] - Tj.tx, ay = pee[3 * e + 1] - Tj.ty, az = pee[3 * e + 2] - Tj.tz;
        col[0] = z.y * az - z.z * ay; col[1] = z.z * ax - z.x * az; col[2] = z.x * ay - z.y * ax;
        col[3] = z.x; col[4] = z.y; col[5] = z.z;
      } else {
        col[0] = z.x; col[1] = z.y; col[2] = z.z; col[3] = col[4] = col[5] = 0.f;
      }
#pragma unroll
      for (int c = 0; c < MAXA; ++c) {
        const float wsel = ((c == a1) ? sm : 0.f) + ((c == a2) ? sm : 0.f);
#pragma unroll
        for (int k = 0; k < 6; ++k) J[6 * e + k][c] += wsel * col[k];
      }
    }
  }
}

// Collision penalty weight * sum over (robot sphere, obstacle) with d < margin
// of (d - margin)^2, from the joint poses in `ps`.  The TPS lanes of a seed
// group split the obstacles and every lane returns the group's total.  An
// obstacle at least the margin from a joint group's bounding sphere adds
// exactly 0 for every sphere of the group and is skipped; with the grid, the
// world spheres tested are those listed in the cell of the group's bounding
// centre.  A world sphere that passes is moved into the joint's frame once
// and tested against the group's spheres there on squared distances (a
// square root only for a hit); the other kinds are tested in the world frame.
template <int TPS>
__device__ __forceinline__ float seed_ik_penalty(const SeedIkArgs& a, const PoseSlots& ps, const RobotSpheresS& R,
                                              const ObsView& ob, int gl, unsigned gmask) {
  if (!a.enable_collision || R.ng == 0) return 0.f;
  const int M = ob.Ms + ob.Mc + ob.Mb + ob.Mh;
  const float margin = a.collision_margin;
  float pen = 0.f;
  for (int k = 0; k < R.ng; ++k) {
    const Pose Tj = ps.load(R.joint[k]);
    const float4 jb = R.bound[k];
    const float3 B = pose_apply(Tj, make_float3(jb.x, jb.y, jb.z));
    // KIND: the obstacle's kind, or -1 to dispatch on m
    auto narrow = [&](int m, auto kind) {
      constexpr int KIND = decltype(kind)::value;
      for (int i = R.gstart[k]; i < R.gstart[k + 1]; ++i) {
        const float4 q = R.sph[i];
        const float d = obstacle_dist<KIND>(ob, m, pose_apply(Tj, make_float3(q.x, q.y, q.z)), q.w);
        if (d < margin) {
          const float e = d - margin;
          pen += e * e;
        }
      }
    };
    // world sphere m against the group's spheres, in the joint's frame
    auto narrow_sphere = [&](int m) {
      const float4 O = ob.sph[m];
      const float3 o = pose_apply_inv(Tj, make_float3(O.x, O.y, O.z));
      for (int i = R.gstart[k]; i < R.gstart[k + 1]; ++i) {
        const float4 q = R.sph[i];
        const float dx = q.x - o.x, dy = q.y - o.y, dz = q.z - o.z;
        const float d2 = dx * dx + dy * dy + dz * dz;
        const float rr = q.w + O.w + margin;
        if (d2 < rr * fabsf(rr)) {
          const float e = sqrtf(d2) - rr;
          pen += e * e;
        }
      }
    };
    if (R.cell_start) {
      const int cell = obstacle_grid_cell(R.glo, R.ginv, R.gn, B);
      if (cell >= 0) {
        const int e1 = R.cell_start[cell + 1];
        for (int e = R.cell_start[cell] + gl; e < e1; e += TPS) {
          const int m = R.cell_obs[e];
          if (obstacle_near<0>(ob, m, B, jb.w, margin)) narrow_sphere(m);
        }
      }
    } else {
      for (int m = gl; m < ob.Ms; m += TPS)
        if (obstacle_near<0>(ob, m, B, jb.w, margin)) narrow_sphere(m);
    }
    for (int m = ob.Ms + gl; m < M; m += TPS)
      if (obstacle_near(ob, m, B, jb.w, margin)) narrow(m, ObsKind<-1>());
  }
#pragma unroll
  for (int o = 1; o < TPS; o <<= 1) pen += __shfl_xor_sync(gmask, pen, o);
  return a.collision_weight * pen;
}

template <int MAXA>
__device__ __forceinline__ float reg_at(const float (&v)[MAXA], int i) {
  float r = 0.f;
#pragma unroll
  for (int c = 0; c < MAXA; ++c)
    if (c == i) r = v[c];
  return r;
}

static inline size_t seed_ik_smem(const SeedIkArgs& a, int nth) {
  return seed_ik_slots_offset(a) + sizeof(float) * (size_t)a.m.n_joints * 7 * nth;
}

// Host side: extents and capacity checks and the shared-memory size (the
// world is staged when it fits; with `grid`, a staged world of 32 or more
// spheres gets the obstacle grid), argument packing, null-buffer checks.
static inline int seed_ik_common(SeedIkArgs& a, int n_act, int n_joints, int n_ee, int nth, size_t* smem_out,
                                 bool grid = false) {
  PK_CHECK_ARG(a.P >= 0 && a.S >= 0 && n_act >= 0 && n_joints >= 0 && n_ee >= 0 && a.n_rs >= 0, "negative extent");
  PK_CHECK_CAP(n_joints <= PK_MAX_JOINTS, "n_joints=%d exceeds %d", n_joints, PK_MAX_JOINTS);
  PK_CHECK_CAP(n_act <= 16, "at most 16 actuated joints (got %d)", n_act);
  PK_CHECK_CAP(n_ee >= 1 && n_ee <= PK_MAX_EE, "n_ee=%d must be in [1, %d]", n_ee, PK_MAX_EE);
  PK_CHECK_ARG(a.iters >= 0, "negative iteration count");
  a.stage_world = a.w.smem_floats() * sizeof(float) <= 48 * 1024;
  const bool want_grid = grid && a.enable_collision && a.stage_world && a.w.Ms >= 32 && a.w.Ms <= 65535;
  // the LM kernels' default resolution (lm_grid_option) and list capacity
  a.grid_n = want_grid ? lm_grid_option(0, a.w.Ms) : 0;
  a.grid_entries = want_grid ? obstacle_grid_capacity(a.grid_n, a.w.Ms) : 0;
  size_t smem = seed_ik_smem(a, nth);
  if (smem > 200 * 1024 && a.grid_entries) {
    a.grid_entries = 0;
    smem = seed_ik_smem(a, nth);
  }
  if (smem > 200 * 1024 && a.stage_world) {
    a.stage_world = 0;
    smem = seed_ik_smem(a, nth);
  }
  PK_CHECK_CAP(smem <= 200 * 1024, "IK working set (%zu B of shared memory) too large", smem);
  *smem_out = smem;
  return PK_OK;
}

static inline SeedIkArgs seed_ik_args(const float* seeds, const float* twists, const float* parent_tf, const int32_t* parent_idx,
                   const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                   const int32_t* mimic_act_idx, const int32_t* topo_inv, const int32_t* target_jnts,
                   const int32_t* ancestor_masks, const float* target_Ts, const float* rs_local,
                   const int32_t* rs_joint, const float* ws, const float* wc, const float* wb, const float* wh,
                   const float* lower, const float* upper, const int32_t* fixed_mask, float* out, float* out_err,
                   int32_t P, int32_t S, int32_t n_act, int32_t n_joints, int32_t n_ee, int32_t n_rs, int32_t Ms,
                   int32_t Mc, int32_t Mb, int32_t Mh) {
  SeedIkArgs a{};
  a.m = ModelArgs{twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx, topo_inv, n_joints,
                  n_act};
  a.w = WorldArgs{ws, wc, wb, wh, Ms, Mc, Mb, Mh};
  a.seeds = seeds; a.target_jnts = target_jnts; a.ancestor_masks = ancestor_masks; a.target_Ts = target_Ts;
  a.rs_local = rs_local; a.rs_joint = rs_joint; a.lower = lower; a.upper = upper; a.fixed_mask = fixed_mask;
  a.out = out; a.out_err = out_err;
  a.P = P; a.S = S; a.n_ee = n_ee; a.n_rs = n_rs;
  return a;
}

static inline int seed_ik_check_buffers(const SeedIkArgs& a) {
  PK_CHECK_ARG(a.seeds && a.m.twists && a.m.parent_tf && a.m.parent_idx && a.m.act_idx && a.m.mimic_mul &&
                   a.m.mimic_off && a.m.mimic_act_idx && a.m.topo_inv && a.target_jnts && a.ancestor_masks &&
                   a.target_Ts && a.lower && a.upper && a.out && a.out_err,
               "null buffer");
  PK_CHECK_ARG(a.n_rs == 0 || (a.rs_local && a.rs_joint), "null robot spheres");
  PK_CHECK_ARG((a.w.Ms == 0 || a.w.spheres) && (a.w.Mc == 0 || a.w.capsules) && (a.w.Mb == 0 || a.w.boxes) &&
                   (a.w.Mh == 0 || a.w.halfspaces),
               "null world buffer");
  return PK_OK;
}


}  // namespace pk
