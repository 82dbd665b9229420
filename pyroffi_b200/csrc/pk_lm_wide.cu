// Warp-per-seed Levenberg-Marquardt IK: the body for wide robots (trees,
// up to 32 actuated DOF, up to 4 end effectors), the grid launch that
// pk_ls_ik_ex uses for them, and its persistent work-queue kernel for
// pk_ik_batch.
//
// The per-seed iteration is the one of the seed-group kernel (pk_lm.cu),
// which restates ls_ik_lm_kernel (src/pyroffi/cuda_kernels/
// _ls_ik_cuda_kernel.cu:65-394): residual, weighted stacked Jacobian, Jacobi
// column scaling, damped normal equations (FP64 in the reference), Cholesky
// (step 0 on a non-positive pivot), trust-region clip, 5-point line search
// on clamped trials, accept/reject of the damping, all-time best.
//
// B200 mapping: one warp owns one seed and keeps the seed's state in
// shared memory, so no per-thread array grows with the DOF count:
//  * FK runs level by level over the joint tree (joints of one depth level
//    on different lanes);
//  * lane c builds Jacobian column c.  Only the active columns are formed:
//    an actuated joint that is fixed, or moves no end effector, has an
//    all-zero column whose damped step is exactly 0, so dropping it changes
//    nothing but the size of the solve;
//  * the damped system (its rows x rows dual form when the residual rows are
//    fewer than the active columns) is formed in FP32 by packed entries,
//    factored by a left-looking Cholesky parallel over the rows below the
//    pivot, and solved column by column, with one FP64 refinement step when
//    the squared pivot ratio exceeds 1e6;
//  * the collision penalty is split over the lanes: sphere transforms by
//    sphere, world spheres by sphere-carrying joint (bounding-sphere cull
//    and a per-block obstacle grid, as in the seed-group kernel), other
//    obstacle types by sphere, self pairs by pair, then a warp sum.
// The robot class, world and grid are staged per block in shared memory and
// re-staged only when a block moves to another class (targets: another
// problem).
#include <float.h>

#include <algorithm>

#include "pk_batch.cuh"
#include "pk_obstacle_grid.cuh"

namespace pk {

constexpr int W_MAXROWS = 6 * PK_MAX_EE;

struct WideArgs {
  ModelArgs m;
  const float* seeds;
  const int* target_jnts;
  const int* ancestor_masks;
  const float* target_Ts;
  const float* spheres_local;
  const int* sphere_joint;
  const int* self_i;
  const int* self_j;
  const float* lower;
  const float* upper;
  const int* fixed_mask;
  float* out_cfg;
  float* out_err;
  int n_act, n_ee, n_rs, n_self, seed_stride, n_problems;
};

// Byte offsets of the dynamic shared memory, sized for the largest class.
struct WideLayout {
  size_t rs, rsj, rsk, pairs, ws, wc, wb, wh, cells, cell_obs, obox, warps, warp_bytes, total;
  size_t w_cfg, w_best, w_dact, w_trial, w_dcol, w_cs, w_r, w_fw, w_pee, w_T, w_J, w_A, w_y, w_b, w_d, w_t, w_pos,
      w_slot;
  int max_rs, max_self, max_joints, max_act, max_rows, max_entries, nwarps;
  int grid_n;  // obstacle grid cells per axis (0: no grid)
};

struct WideLaunch {
  WideArgs cls[PK_MAX_CLASSES];
  int body[PK_MAX_CLASSES];
  int n_classes;
  WorldArgs w;
  int max_iter;
  float pos_w, ori_w, lam0, lam_down, lam_up, eps_pos, eps_ori;
  int coll;
  float coll_w, margin;
  const int4* items;  // persistent: the item list
  int n_items;
  int* queue;         // persistent: item counter; null: grid launch (problem blockIdx.y, seed block blockIdx.x)
  int grid_chunk;     // grid launch: seeds per block
  int grid_n;         // obstacle grid cells per axis (0: no grid)
  int grid_auto;      // grid_n is the default resolution (the launch may coarsen it)
  WideLayout L;
};

struct WideShared {
  JointTable jt;
  unsigned long long anc[PK_MAX_EE];
  float tgt[PK_MAX_EE][7];
  int tsorted[PK_MAX_EE];
  float lo[PK_MAX_ACT], hi[PK_MAX_ACT];
  int ncol;
  int col_act[PK_MAX_ACT];
  int col_start[PK_MAX_ACT + 1];
  int col_joint[2 * PK_MAX_JOINTS];
  float col_w[2 * PK_MAX_JOINTS];
  int n_lvl;
  int lvl_start[PK_MAX_JOINTS + 1];
  int lvl_joint[PK_MAX_JOINTS];
  int n_js;
  int js_joint[PK_MAX_JOINTS];     // sorted joint of each sphere-carrying slot
  int jstart[PK_MAX_JOINTS + 1];   // grouped sphere range per slot
  float4 jb[PK_MAX_JOINTS];        // bounding sphere per slot (joint frame)
  int n_rs, n_pairs;
  int grid_on;
  int grid_n;                      // cells per axis of the grid in use
  float3 glo, ginv;
  float rmax;
};

__host__ __device__ inline size_t w_align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ inline WideLayout wide_layout(int max_rs, int max_self, int max_joints, int max_act, int max_ee,
                                       const WorldArgs& w, int nwarps, int grid_n) {
  WideLayout L{};
  L.max_rs = max_rs; L.max_self = max_self; L.max_joints = max_joints; L.max_act = max_act;
  L.max_rows = 6 * max_ee; L.nwarps = nwarps;
  L.grid_n = grid_n;
  L.max_entries = (grid_n > 0 && w.Ms >= 32 && w.Ms <= 65535) ? obstacle_grid_capacity(grid_n, w.Ms) : 0;
  size_t o = w_align16(sizeof(WideShared));
  L.rs = o; o = w_align16(o + 16 * (size_t)max_rs);
  L.rsj = o; o = w_align16(o + 4 * (size_t)max_rs);
  L.rsk = o; o = w_align16(o + 4 * (size_t)max_rs);
  L.pairs = o; o = w_align16(o + 8 * (size_t)max_self);
  L.ws = o; o = w_align16(o + 16 * (size_t)w.Ms);
  L.wc = o; o = w_align16(o + 28 * (size_t)w.Mc);
  L.wb = o; o = w_align16(o + 60 * (size_t)w.Mb);
  L.wh = o; o = w_align16(o + 24 * (size_t)w.Mh);
  L.cells = o; o = w_align16(o + (L.max_entries ? 4 * (size_t)(obstacle_grid_cells(grid_n) + 1) : 0));
  L.cell_obs = o; o = w_align16(o + 2 * (size_t)L.max_entries);
  L.obox = o; o = w_align16(o + (L.max_entries ? 4 * (size_t)w.Ms : 0));
  // one warp's area
  size_t q = 0;
  L.w_cfg = q; q += 4 * PK_MAX_ACT;
  L.w_best = q; q += 4 * PK_MAX_ACT;
  L.w_dact = q; q += 4 * PK_MAX_ACT;
  L.w_trial = q; q += 4 * PK_MAX_ACT;
  L.w_dcol = q; q += 4 * PK_MAX_ACT;
  L.w_cs = q; q += 4 * PK_MAX_ACT;
  L.w_r = q; q += 4 * W_MAXROWS;
  L.w_fw = q; q += 4 * W_MAXROWS;
  L.w_pee = q; q += 4 * 3 * PK_MAX_EE;
  q = w_align16(q);
  L.w_T = q; q = w_align16(q + 28 * (size_t)max_joints);
  // The Jacobian (direction step) and the per-joint slot data (penalty) are
  // never live together, nor are the normal equations and the sphere
  // positions: each pair shares one region.
  L.w_J = q;
  L.w_slot = q;  // per sphere-carrying joint: B, R (float4); list range, offset (int4)
  q = w_align16(q + std::max(4 * (size_t)L.max_rows * max_act, 32 * (size_t)max_joints));
  L.w_A = q;
  L.w_y = w_align16(q + 4 * (size_t)max_act * (max_act + 1) / 2);
  L.w_b = L.w_y + 4 * (size_t)PK_MAX_ACT;  // the system has at most PK_MAX_ACT rows
  L.w_d = L.w_b + 4 * (size_t)PK_MAX_ACT;
  L.w_t = L.w_d + 4 * (size_t)PK_MAX_ACT;  // ncol or rows doubles, both <= PK_MAX_ACT
  L.w_pos = q;
  q = w_align16(std::max(L.w_t + 8 * (size_t)PK_MAX_ACT, q + 16 * (size_t)max_rs));
  L.warp_bytes = q;
  L.warps = o;
  L.total = o + q * nwarps;
  return L;
}

// ---------------------------------------------------------------------------
// staging
// ---------------------------------------------------------------------------

// Robot class c and the world, by all threads of the block; ends with __syncthreads().
__device__ void wide_stage_class(const WideLaunch& P, const WideArgs& A, unsigned char* smem) {
  const WideLayout& L = P.L;
  WideShared& sh = *reinterpret_cast<WideShared*>(smem);
  float4* rs4 = reinterpret_cast<float4*>(smem + L.rs);
  int* rsj = reinterpret_cast<int*>(smem + L.rsj);
  int* rsk = reinterpret_cast<int*>(smem + L.rsk);
  int2* pairs = reinterpret_cast<int2*>(smem + L.pairs);
  float4* ws4 = reinterpret_cast<float4*>(smem + L.ws);
  float* wc = reinterpret_cast<float*>(smem + L.wc);
  float* wb = reinterpret_cast<float*>(smem + L.wb);
  float* wh = reinterpret_cast<float*>(smem + L.wh);
  int* cell_start = reinterpret_cast<int*>(smem + L.cells);
  unsigned short* cell_obs = reinterpret_cast<unsigned short*>(smem + L.cell_obs);
  int* obox = reinterpret_cast<int*>(smem + L.obox);
  const int tid = threadIdx.x;
  const WorldArgs& w = P.w;

  load_joint_table(sh.jt, A.m);  // ends with __syncthreads()
  const int nj = A.m.n_joints;
  if (tid < A.n_ee) {
    unsigned long long bits = 0ull;
    for (int j = 0; j < nj; ++j)
      if (A.ancestor_masks[tid * nj + j]) bits |= 1ull << j;
    sh.anc[tid] = bits;
    const int tj = A.target_jnts[tid];
    sh.tsorted[tid] = (tj >= 0 && tj < nj) ? sh.jt.sorted_of[tj] : 0;
  }
  for (int i = tid; i < PK_MAX_ACT; i += blockDim.x) {
    const bool real = i < A.n_act;
    sh.lo[i] = real ? A.lower[i] : 0.f;
    sh.hi[i] = real ? A.upper[i] : 0.f;
  }
  // the world by the TMA bulk-copy engine (stage_world: bounded wait,
  // plain-load fallback; its layout is this one's), then the margin folded
  // into the sphere radii in place
  (void)wc; (void)wb; (void)wh;
  stage_world(w, reinterpret_cast<float*>(ws4));
  __syncthreads();
  for (int i = tid; i < w.Ms; i += blockDim.x) ws4[i].w = ws4[i].w + P.margin;
  __syncthreads();

  // Thread 0: active columns and their joint lists, FK levels, spheres
  // grouped by joint (invalid joint indices dropped, as the reference skips
  // them), bounding spheres, self pairs in grouped indices, grid bounds.
  if (tid == 0) {
    const JointTable& jt = sh.jt;
    const int n = jt.n;
    // active columns
    int ncol = 0, t = 0;
    for (int act = 0; act < A.n_act; ++act) {
      if (A.fixed_mask[act] != 0) continue;
      const int t0 = t;
      for (int i = 0; i < n; ++i) {
        if (jt.jkind[i] == 0) continue;
        const int hits = (jt.a1[i] == act) + (jt.a2[i] == act);
        if (hits == 0) continue;
        bool moves = false;
        for (int e = 0; e < A.n_ee; ++e) moves |= ((sh.anc[e] >> jt.orig[i]) & 1ull) != 0;
        if (!moves) continue;
        sh.col_joint[t] = i;
        sh.col_w[t] = jt.mul[i] * (float)hits;
        ++t;
      }
      if (t == t0) continue;
      sh.col_act[ncol] = act;
      sh.col_start[ncol] = t0;
      ++ncol;
    }
    sh.col_start[ncol] = t;
    sh.ncol = ncol;
    // levels
    int lvl[PK_MAX_JOINTS], cnt[PK_MAX_JOINTS + 1];
    int n_lvl = 0;
    for (int i = 0; i < n; ++i) {
      const int p = jt.psorted[i];
      lvl[i] = (p < 0 || p >= i) ? 0 : lvl[p] + 1;
      n_lvl = max(n_lvl, lvl[i] + 1);
    }
    for (int l = 0; l <= n_lvl; ++l) cnt[l] = 0;
    for (int i = 0; i < n; ++i) cnt[lvl[i]]++;
    int run = 0;
    for (int l = 0; l < n_lvl; ++l) { sh.lvl_start[l] = run; run += cnt[l]; cnt[l] = sh.lvl_start[l]; }
    sh.lvl_start[n_lvl] = run;
    for (int i = 0; i < n; ++i) sh.lvl_joint[cnt[lvl[i]]++] = i;
    sh.n_lvl = n_lvl;
    // spheres grouped by sphere-carrying joint, in sorted joint order
    int scnt[PK_MAX_JOINTS], slot_of[PK_MAX_JOINTS];
    for (int j = 0; j < n; ++j) scnt[j] = 0;
    for (int k = 0; k < A.n_rs; ++k) {
      const int j = A.sphere_joint[k];
      if (j >= 0 && j < nj) scnt[jt.sorted_of[j]]++;
    }
    int n_js = 0, total = 0;
    for (int js = 0; js < n; ++js) {
      slot_of[js] = -1;
      if (scnt[js] == 0) continue;
      slot_of[js] = n_js;
      sh.js_joint[n_js] = js;
      sh.jstart[n_js] = total;
      total += scnt[js];
      scnt[js] = sh.jstart[n_js];
      ++n_js;
    }
    sh.jstart[n_js] = total;
    sh.n_js = n_js;
    sh.n_rs = total;
    for (int k = 0; k < A.n_rs; ++k) {
      const int j = A.sphere_joint[k];
      if (j < 0 || j >= nj) { rsk[k] = -1; continue; }
      const int js = jt.sorted_of[j];
      const int at = scnt[js]++;
      rsk[k] = at;
      rs4[at] = make_float4(A.spheres_local[4 * k], A.spheres_local[4 * k + 1], A.spheres_local[4 * k + 2],
                            A.spheres_local[4 * k + 3]);
      rsj[at] = slot_of[js];
    }
    float rmax = 0.f;
    for (int q = 0; q < n_js; ++q) {
      float lo3[3] = {3e38f, 3e38f, 3e38f}, hi3[3] = {-3e38f, -3e38f, -3e38f};
      for (int k = sh.jstart[q]; k < sh.jstart[q + 1]; ++k) {
        const float v[3] = {rs4[k].x, rs4[k].y, rs4[k].z};
        for (int d = 0; d < 3; ++d) { lo3[d] = fminf(lo3[d], v[d]); hi3[d] = fmaxf(hi3[d], v[d]); }
      }
      const float cx = 0.5f * (lo3[0] + hi3[0]), cy = 0.5f * (lo3[1] + hi3[1]), cz = 0.5f * (lo3[2] + hi3[2]);
      float R = -3e38f;
      for (int k = sh.jstart[q]; k < sh.jstart[q + 1]; ++k) {
        const float dx = rs4[k].x - cx, dy = rs4[k].y - cy, dz = rs4[k].z - cz;
        R = fmaxf(R, sqrtf(dx * dx + dy * dy + dz * dz) + rs4[k].w);
      }
      R = R + 1e-4f + 1e-5f * fabsf(R);  // slack keeps the cull conservative under FP32 rounding
      sh.jb[q] = make_float4(cx, cy, cz, R);
      rmax = fmaxf(rmax, R);
    }
    sh.rmax = rmax;
    // self pairs in grouped sphere positions (pairs with an invalid sphere are dropped)
    int n_pairs = 0;
    if (P.coll && A.n_self > 0) {
      for (int q = 0; q < A.n_self; ++q) {
        const int x = A.self_i[q], y = A.self_j[q];
        if (x < 0 || y < 0 || x >= A.n_rs || y >= A.n_rs) continue;
        if (rsk[x] < 0 || rsk[y] < 0) continue;
        pairs[n_pairs++] = make_int2(rsk[x], rsk[y]);
      }
    }
    sh.n_pairs = n_pairs;
    // obstacle-grid bounds (world radii already carry the margin)
    sh.grid_on = 0;
    sh.grid_n = L.grid_n;
    if (L.max_entries > 0 && n_js > 0 && P.coll) {
      obstacle_grid_bounds(ws4, w.Ms, rmax, sh.grid_n, sh.glo, sh.ginv);
      sh.grid_on = 1;
    }
  }
  __syncthreads();

  if (sh.grid_on) {
    obstacle_grid_build(ws4, w.Ms, sh.rmax, sh.grid_n, sh.glo, sh.ginv, obox, cell_start, cell_obs, L.max_entries,
                        sh.grid_on);
    // a fine grid whose lists overflow the capacity falls back to the default resolution
    if (!sh.grid_on && sh.grid_n > kObsGridDefault) {
      __syncthreads();
      if (threadIdx.x == 0) {
        sh.grid_n = kObsGridDefault;
        obstacle_grid_bounds(ws4, w.Ms, sh.rmax, sh.grid_n, sh.glo, sh.ginv);
        sh.grid_on = 1;
      }
      __syncthreads();
      obstacle_grid_build(ws4, w.Ms, sh.rmax, sh.grid_n, sh.glo, sh.ginv, obox, cell_start, cell_obs,
                          L.max_entries, sh.grid_on);
    }
  }
}

// Targets of problem pb (threads < n_ee); the caller synchronises.
__device__ inline void wide_stage_targets(const WideArgs& A, int pb, WideShared& sh) {
  const int t = threadIdx.x;
  if (t < A.n_ee)
    for (int c = 0; c < 7; ++c) sh.tgt[t][c] = A.target_Ts[((size_t)pb * A.n_ee + t) * 7 + c];
}

// ---------------------------------------------------------------------------
// per-seed body: a group of G lanes (G = 16: two seeds per warp; G = 32:
// one) owns one seed; gl is the lane within the group, gm the group's mask.
// ---------------------------------------------------------------------------

template <int G>
__device__ __forceinline__ float w_group_sum(float v, unsigned gm) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o);
  return v;
}

__device__ __forceinline__ void w_hinge(float d2, float rr, float& pen) {
  if (d2 < rr * fabsf(rr)) {
    const float e = sqrtf(d2) - rr;
    pen += e * e;
  }
}

struct WideWarp {
  float *cfg, *best, *dact, *trial, *dcol, *cs, *r, *fw, *pee, *T, *J;
  float *A, *y, *b, *d;  // damped system: factor, solution, right-hand side, correction
  double* t;             // refinement scratch
  float4* pos;
  float4* slotB;  // per slot: bounding centre (world) and radius
  int4* slotL;    // per slot: first list entry, candidate count, offset in the flattened candidates, -
};

__device__ __forceinline__ Pose w_load(const float* T, int i) {
  const float* p = T + 7 * i;
  return Pose{p[0], p[1], p[2], p[3], p[4], p[5], p[6]};
}
__device__ __forceinline__ void w_store(float* T, int i, const Pose& P) {
  float* p = T + 7 * i;
  p[0] = P.w; p[1] = P.x; p[2] = P.y; p[3] = P.z; p[4] = P.tx; p[5] = P.ty; p[6] = P.tz;
}

// FK of configuration q (shared, n_act floats) into W.T: every joint's local
// transform in parallel, then the compositions level by level in place
// (a joint's parent is final before its level runs).
template <int G>
__device__ __forceinline__ void w_fk(const WideShared& sh, const float* q, const WideWarp& W, int gl, unsigned gm) {
  const JointTable& jt = sh.jt;
  for (int i = gl; i < jt.n; i += G) {
    const int src = jt.src[i];
    w_store(W.T, i, joint_local(jt, i, ((src < 0) ? 0.f : q[src]) * jt.mul[i] + jt.off[i]));
  }
  __syncwarp(gm);
  for (int lv = 1; lv < sh.n_lvl; ++lv) {
    for (int idx = sh.lvl_start[lv] + gl; idx < sh.lvl_start[lv + 1]; idx += G) {
      const int i = sh.lvl_joint[idx];
      const int p = jt.psorted[i];
      if (p >= 0) w_store(W.T, i, pose_compose(w_load(W.T, p), w_load(W.T, i)));
    }
    __syncwarp(gm);
  }
}

// Residual of every EE into W.r / W.pee (lane e), as the seed-group kernel's ee_residual.
__device__ __forceinline__ void w_residual(const WideShared& sh, int n_ee, const WideWarp& W, int gl, unsigned gm) {
  if (gl < n_ee) {
    const int e = gl;
    const Pose T = w_load(W.T, sh.tsorted[e]);
    const float* g = sh.tgt[e];
    float* r = W.r + 6 * e;
    r[0] = T.tx - g[4];
    r[1] = T.ty - g[5];
    r[2] = T.tz - g[6];
    const float bw = g[0], bx = -g[1], by = -g[2], bz = -g[3];
    float qw = T.w * bw - T.x * bx - T.y * by - T.z * bz;
    float qx = T.w * bx + T.x * bw + T.y * bz - T.z * by;
    float qy = T.w * by - T.x * bz + T.y * bw + T.z * bx;
    float qz = T.w * bz + T.x * by - T.y * bx + T.z * bw;
    if (qw < 0.f) { qw = -qw; qx = -qx; qy = -qy; qz = -qz; }
    const float s = sqrtf(qx * qx + qy * qy + qz * qz);
    const float f = (s > 1e-6f) ? 2.f * atan2f(s, qw) / s : 2.f;
    r[3] = qx * f;
    r[4] = qy * f;
    r[5] = qz * f;
    W.pee[3 * e] = T.tx; W.pee[3 * e + 1] = T.ty; W.pee[3 * e + 2] = T.tz;
  }
  __syncwarp(gm);
}

// Collision penalty (before the weight) of the configuration whose poses are in W.T.
template <int G>
__device__ __noinline__ float w_penalty(const WideLaunch& P, const WideShared& sh, const unsigned char* smem,
                                        const WideWarp& W, int gl, unsigned gm) {
  const WideLayout& L = P.L;
  const float4* rs4 = reinterpret_cast<const float4*>(smem + L.rs);
  const int* rsj = reinterpret_cast<const int*>(smem + L.rsj);
  const int2* pairs = reinterpret_cast<const int2*>(smem + L.pairs);
  const float4* ws4 = reinterpret_cast<const float4*>(smem + L.ws);
  const float* wc = reinterpret_cast<const float*>(smem + L.wc);
  const float* wb = reinterpret_cast<const float*>(smem + L.wb);
  const float* wh = reinterpret_cast<const float*>(smem + L.wh);
  const int* cell_start = reinterpret_cast<const int*>(smem + L.cells);
  const unsigned short* cell_obs = reinterpret_cast<const unsigned short*>(smem + L.cell_obs);
  const int n_rs = sh.n_rs;
  // sphere world positions: for the self pairs and the capsule / box /
  // halfspace tests (world spheres are tested in the joint's frame)
  if (sh.n_pairs > 0 || P.w.Mc + P.w.Mb + P.w.Mh > 0) {
    for (int k = gl; k < n_rs; k += G) {
      const float4 s = rs4[k];
      const float3 p = pose_apply(w_load(W.T, sh.js_joint[rsj[k]]), make_float3(s.x, s.y, s.z));
      W.pos[k] = make_float4(p.x, p.y, p.z, s.w);
    }
  }
  __syncwarp(gm);
  float pen = 0.f;
  const int Ms = P.w.Ms;
  if (Ms > 0) {
    // per sphere-carrying joint: bounding centre and its candidate obstacles
    for (int j = gl; j < sh.n_js; j += G) {
      const float4 bl = sh.jb[j];
      const float3 B = pose_apply(w_load(W.T, sh.js_joint[j]), make_float3(bl.x, bl.y, bl.z));
      int e0 = 0, n = Ms;
      if (sh.grid_on) {
        const int cell = obstacle_grid_cell(sh.glo, sh.ginv, sh.grid_n, B);
        // outside the grid no obstacle is within reach of this joint
        if (cell < 0) {
          n = 0;
        } else {
          e0 = cell_start[cell];
          n = cell_start[cell + 1] - e0;
        }
      }
      W.slotB[j] = make_float4(B.x, B.y, B.z, bl.w);
      W.slotL[j] = make_int4(e0, n, 0, 0);
    }
    __syncwarp(gm);
    // offsets of each joint's candidates in the flattened list (serial: at most 64 joints)
    int total = 0;
    for (int j = 0; j < sh.n_js; ++j) total += W.slotL[j].y;
    if (gl == 0) {
      int run = 0;
      for (int j = 0; j < sh.n_js; ++j) { W.slotL[j].z = run; run += W.slotL[j].y; }
    }
    __syncwarp(gm);
    // lanes take (joint, candidate) pairs in turn: bounding-sphere test, then
    // the joint's spheres against the candidate
    int j = 0;
    for (int it = gl; it < total; it += G) {
      while (j + 1 < sh.n_js && W.slotL[j + 1].z <= it) ++j;
      while (W.slotL[j].z > it) --j;
      const int4 sl = W.slotL[j];
      const int e = sl.x + (it - sl.z);
      const float4 O = ws4[sh.grid_on ? (int)cell_obs[e] : e];
      const float4 Bj = W.slotB[j];
      const float rr = Bj.w + O.w;
      const float dx = Bj.x - O.x, dy = Bj.y - O.y, dz = Bj.z - O.z;
      if (dx * dx + dy * dy + dz * dz < rr * fabsf(rr)) {
        // the obstacle in the joint's frame, against the joint's spheres there
        const float3 o = pose_apply_inv(w_load(W.T, sh.js_joint[j]), make_float3(O.x, O.y, O.z));
        for (int k = sh.jstart[j]; k < sh.jstart[j + 1]; ++k) {
          const float4 q = rs4[k];
          const float ex = q.x - o.x, ey = q.y - o.y, ez = q.z - o.z;
          w_hinge(ex * ex + ey * ey + ez * ez, q.w + O.w, pen);
        }
      }
    }
  }
  const float margin = P.margin;
  if (P.w.Mc + P.w.Mb + P.w.Mh > 0) {
    for (int k = gl; k < n_rs; k += G) {
      const float4 q = W.pos[k];
      const float3 p = make_float3(q.x, q.y, q.z);
      for (int m = 0; m < P.w.Mc; ++m) {
        const float d = d_sphere_capsule(p, q.w, wc + 7 * m);
        if (d < margin) { const float e = d - margin; pen += e * e; }
      }
      for (int m = 0; m < P.w.Mb; ++m) {
        const float d = d_sphere_box(p, q.w, wb + 15 * m);
        if (d < margin) { const float e = d - margin; pen += e * e; }
      }
      for (int m = 0; m < P.w.Mh; ++m) {
        const float d = d_sphere_halfspace(p, q.w, wh + 6 * m);
        if (d < margin) { const float e = d - margin; pen += e * e; }
      }
    }
  }
  for (int q = gl; q < sh.n_pairs; q += G) {
    const int2 pr = pairs[q];
    const float4 a = W.pos[pr.x], b = W.pos[pr.y];
    const float ex = a.x - b.x, ey = a.y - b.y, ez = a.z - b.z;
    w_hinge(ex * ex + ey * ey + ez * ez, a.w + b.w + margin, pen);
  }
  pen = w_group_sum<G>(pen, gm);
  __syncwarp(gm);
  return pen;
}

// Weighted squared residual sum, the same on every lane (sequential order).
__device__ __forceinline__ float w_weighted_sq(const WideWarp& W, int n_ee, const float (&Wt)[6]) {
  float e = 0.f;
  for (int k = 0; k < 6 * n_ee; ++k) {
    const float rw = W.r[k] * Wt[k % 6];
    e += rw * rw;
  }
  return e;
}

// Damped step of the current point into W.dact (all actuated entries);
// returns ||fw||^2.  Poses of the current point are in W.T, its residual in W.r.
template <int G, int MAXEE>
__device__ __noinline__ float w_direction(const WideShared& sh, int n_act, int n_ee, const float (&Wt)[6], float lam,
                                          float max_p, float max_o, const WideWarp& W, int gl, unsigned gm) {
  const JointTable& jt = sh.jt;
  const int ncol = sh.ncol, rows = 6 * n_ee;
  // Jacobian columns c = gl, gl + G, ...: weighted, Jacobi-scaled, column-major
  for (int c = gl; c < ncol; c += G) {
    float Jc[6 * MAXEE];
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k) Jc[k] = 0.f;
    for (int t = sh.col_start[c]; t < sh.col_start[c + 1]; ++t) {
      const int i = sh.col_joint[t];
      const float wt = sh.col_w[t];
      const Pose Tj = w_load(W.T, i);
      const float3 z = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z, make_float3(jt.axis[i][0], jt.axis[i][1], jt.axis[i][2]));
      const int orig = jt.orig[i];
      const bool rev = jt.jkind[i] == 1;
#pragma unroll
      for (int e = 0; e < MAXEE; ++e) {
        if (e >= n_ee || !((sh.anc[e] >> orig) & 1ull)) continue;
        float col[6];
        if (rev) {
          const float ax = W.pee[3 * e] - Tj.tx, ay = W.pee[3 * e + 1] - Tj.ty, az = W.pee[3 * e + 2] - Tj.tz;
          col[0] = z.y * az - z.z * ay; col[1] = z.z * ax - z.x * az; col[2] = z.x * ay - z.y * ax;
          col[3] = z.x; col[4] = z.y; col[5] = z.z;
        } else {
          col[0] = z.x; col[1] = z.y; col[2] = z.z; col[3] = col[4] = col[5] = 0.f;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) Jc[6 * e + k] += wt * col[k];
      }
    }
    float sq = 0.f;
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k) {
      if (k < rows) {
        Jc[k] *= Wt[k % 6];
        sq += Jc[k] * Jc[k];
      }
    }
    const float s = sqrtf(sq) + 1e-8f;
    W.cs[c] = s;
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k)
      if (k < rows) W.J[c * rows + k] = Jc[k] / s;
  }
  for (int k = gl; k < rows; k += G) W.fw[k] = W.r[k] * Wt[k % 6];
  __syncwarp(gm);
  float fw2 = 0.f;
  for (int k = 0; k < rows; ++k) fw2 += W.fw[k] * W.fw[k];

  // FP32 damped system, packed lower triangle: lanes take the entries
  // e = i (i + 1) / 2 + j in turn.  With fewer residual rows than active
  // columns it is the dual form (Js Js^T + lam I) y = fw, p = -Js^T y (the
  // push-through identity: the same step as (Js^T Js + lam I) p = -Js^T fw,
  // on a rows x rows system); otherwise the normal equations themselves,
  // then of full column rank.  When the squared ratio of the largest to the
  // smallest Cholesky pivot exceeds 1e6, one step of iterative refinement
  // follows: the residual in FP64 from the FP32 entries (which FP64 holds
  // exactly), the correction solved with the FP32 factor.
  const bool dual = rows < ncol;
  const int n = dual ? rows : ncol;
  {
    const int ne = n * (n + 1) / 2;
    int i = 0, j = gl;
    while (i < n && j > i) { j -= i + 1; ++i; }
    for (int e = gl; e < ne; e += G) {
      float acc = (i == j) ? lam : 0.f;
      if (dual) {
        for (int c = 0; c < ncol; ++c) acc = fmaf(W.J[c * rows + i], W.J[c * rows + j], acc);
      } else {
        for (int k = 0; k < rows; ++k) acc = fmaf(W.J[i * rows + k], W.J[j * rows + k], acc);
      }
      W.A[e] = acc;
      j += G;
      while (i < n && j > i) { j -= i + 1; ++i; }
    }
  }
  if (dual) {
    for (int i = gl; i < rows; i += G) W.b[i] = W.y[i] = W.fw[i];
  } else {
    for (int i = gl; i < ncol; i += G) {
      float rb = 0.f;
      for (int k = 0; k < rows; ++k) rb = fmaf(W.J[i * rows + k], W.fw[k], rb);
      W.b[i] = W.y[i] = -rb;
    }
  }
  __syncwarp(gm);

  // Cholesky A = L L^T, left-looking; a non-positive pivot zeroes the step.
  // The diagonal keeps 1 / L[k][k] (every later use multiplies by it).
  bool ok = true;
  float pmax = 0.f, pmin = 3.4e38f;
  for (int k = 0; k < n; ++k) {
    const int kk = k * (k + 1) / 2;
    float s2 = W.A[kk + k];
    for (int q = 0; q < k; ++q) s2 = fmaf(-W.A[kk + q], W.A[kk + q], s2);
    if (!(s2 > 0.f)) ok = false;
    pmax = fmaxf(pmax, s2);
    pmin = fminf(pmin, s2);
    const float inv = 1.f / sqrtf(ok ? s2 : 1.f);
    for (int i = k + 1 + gl; i < n; i += G) {
      const int ii = i * (i + 1) / 2;
      float tt = W.A[ii + k];
      for (int q = 0; q < k; ++q) tt = fmaf(-W.A[ii + q], W.A[kk + q], tt);
      W.A[ii + k] = tt * inv;
    }
    __syncwarp(gm);
    if (gl == 0) W.A[kk + k] = inv;
    __syncwarp(gm);
  }
  // L y = b, then L^T x = y (column by column; x overwrites v)
  auto tri_solve = [&](float* v) {
    for (int i = 0; i < n; ++i) {
      const float yi = v[i] * W.A[i * (i + 1) / 2 + i];
      for (int j = i + 1 + gl; j < n; j += G) v[j] = fmaf(-W.A[j * (j + 1) / 2 + i], yi, v[j]);
      __syncwarp(gm);
      if (gl == 0) v[i] = yi;
      __syncwarp(gm);
    }
    for (int i = n - 1; i >= 0; --i) {
      const int ii = i * (i + 1) / 2;
      const float xi = v[i] * W.A[ii + i];
      for (int j = gl; j < i; j += G) v[j] = fmaf(-W.A[ii + j], xi, v[j]);
      __syncwarp(gm);
      if (gl == 0) v[i] = xi;
      __syncwarp(gm);
    }
  };
  tri_solve(W.y);
  if (ok && pmax > 1e6f * pmin) {
    // the residual b - A y in FP64: t = Js y (dual: per column) or Js x
    // (primal: per row) first, then per row of the system
    const int nt = dual ? ncol : rows;
    for (int c = gl; c < nt; c += G) {
      double acc = 0.0;
      if (dual) {
        for (int k = 0; k < rows; ++k) acc = fma((double)W.J[c * rows + k], (double)W.y[k], acc);
      } else {
        for (int q = 0; q < ncol; ++q) acc = fma((double)W.J[q * rows + c], (double)W.y[q], acc);
      }
      W.t[c] = acc;
    }
    __syncwarp(gm);
    for (int i = gl; i < n; i += G) {
      double acc = (double)lam * (double)W.y[i];
      if (dual) {
        for (int c = 0; c < ncol; ++c) acc = fma((double)W.J[c * rows + i], W.t[c], acc);
      } else {
        for (int k = 0; k < rows; ++k) acc = fma((double)W.J[i * rows + k], W.t[k], acc);
      }
      W.d[i] = (float)((double)W.b[i] - acc);
    }
    __syncwarp(gm);
    tri_solve(W.d);
    for (int i = gl; i < n; i += G) W.y[i] = (float)((double)W.y[i] + (double)W.d[i]);
    __syncwarp(gm);
  }
  if (dual) {
    for (int c = gl; c < ncol; c += G) {
      float pc = 0.f;
      for (int k = 0; k < rows; ++k) pc = fmaf(W.J[c * rows + k], W.y[k], pc);
      W.dcol[c] = ok ? -pc / W.cs[c] : 0.f;
    }
  } else {
    for (int c = gl; c < ncol; c += G) W.dcol[c] = ok ? W.y[c] / W.cs[c] : 0.f;
  }
  __syncwarp(gm);
  float dn2 = 0.f;
  for (int c = 0; c < ncol; ++c) dn2 += W.dcol[c] * W.dcol[c];
  float R;
  if (max_p > 1e-2f || max_o > 0.6f) R = 0.38f;
  else if (max_p > 1e-3f || max_o > 0.25f) R = 0.22f;
  else if (max_p > 2e-4f || max_o > 0.08f) R = 0.12f;
  else R = 0.05f;
  const float dn = sqrtf(dn2);
  const float sc = (dn > R) ? R / (dn + 1e-18f) : 1.f;
  for (int a = gl; a < n_act; a += G) W.dact[a] = 0.f;
  __syncwarp(gm);
  for (int c = gl; c < ncol; c += G) W.dact[sh.col_act[c]] = (dn > R) ? W.dcol[c] * sc : W.dcol[c];
  __syncwarp(gm);
  return fw2;
}

__device__ __forceinline__ float w_alpha(int i) {
  return i == 0 ? 1.0f : i == 1 ? 0.5f : i == 2 ? 0.25f : i == 3 ? 0.1f : 0.025f;
}

// LM for flat seed index gs of class A (targets of its problem staged).
template <int G, int MAXEE>
__device__ void w_seed(const WideLaunch& P, const WideArgs& A, const WideShared& sh, const unsigned char* smem,
                       const WideWarp& W, size_t gs, int gl, unsigned gm) {
  const int n_act = A.n_act, n_ee = A.n_ee;
  const float Wt[6] = {P.pos_w, P.pos_w, P.pos_w, P.ori_w, P.ori_w, P.ori_w};
  const bool use_coll = P.coll && sh.n_rs > 0;
  for (int a = gl; a < n_act; a += G) {
    const float v = A.seeds[gs * n_act + a];
    W.cfg[a] = v;
    W.best[a] = v;
    W.dact[a] = 0.f;
  }
  __syncwarp(gm);
  auto evaluate = [&](const float* q, float& pen) {
    w_fk<G>(sh, q, W, gl, gm);
    w_residual(sh, n_ee, W, gl, gm);
    pen = use_coll ? P.coll_w * w_penalty<G>(P, sh, smem, W, gl, gm) : 0.f;
    return w_weighted_sq(W, n_ee, Wt) + pen;
  };
  float pen_cur;
  float best_err = evaluate(W.cfg, pen_cur);
  float lam = P.lam0;
  for (int it = 0; it < P.max_iter; ++it) {
    // current point: poses and residual (its penalty is carried), convergence, damped step
    w_fk<G>(sh, W.cfg, W, gl, gm);
    w_residual(sh, n_ee, W, gl, gm);
    bool all_conv = true;
    float max_p = 0.f, max_o = 0.f;
    for (int e = 0; e < n_ee; ++e) {
      const float* r = W.r + 6 * e;
      const float np = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const float no = sqrtf(r[3] * r[3] + r[4] * r[4] + r[5] * r[5]);
      if (np >= P.eps_pos || no >= P.eps_ori) all_conv = false;
      max_p = fmaxf(max_p, np);
      max_o = fmaxf(max_o, no);
    }
    if (all_conv) break;
    const float curr = w_direction<G, MAXEE>(sh, n_act, n_ee, Wt, lam, max_p, max_o, W, gl, gm) + pen_cur;
    // line search: first minimum over the 5 step sizes
    float best_a_err = 1e30f, best_a_pen = pen_cur;
    int best_a = 0;
    for (int t = 0; t < 5; ++t) {
      const float al = w_alpha(t);
      for (int a = gl; a < n_act; a += G)
        W.trial[a] = fmaxf(sh.lo[a], fminf(sh.hi[a], W.cfg[a] + al * W.dact[a]));
      __syncwarp(gm);
      // a trial whose pose error alone cannot beat the best trial skips its
      // penalty (>= 0), which changes no decision or output
      w_fk<G>(sh, W.trial, W, gl, gm);
      w_residual(sh, n_ee, W, gl, gm);
      const float wsq = w_weighted_sq(W, n_ee, Wt);
      if (!(wsq < best_a_err)) continue;
      const float pen = use_coll ? P.coll_w * w_penalty<G>(P, sh, smem, W, gl, gm) : 0.f;
      const float err = wsq + pen;
      if (err < best_a_err) { best_a_err = err; best_a = t; best_a_pen = pen; }
    }
    const float al = w_alpha(best_a);
    const bool accept = best_a_err < curr * (1.0f - 1e-4f);
    const bool improve = best_a_err < best_err;
    for (int a = gl; a < n_act; a += G) {
      const float tv = fmaxf(sh.lo[a], fminf(sh.hi[a], W.cfg[a] + al * W.dact[a]));
      if (improve) W.best[a] = tv;
      if (accept) W.cfg[a] = tv;
    }
    __syncwarp(gm);
    if (accept) {
      pen_cur = best_a_pen;
      lam = fmaxf(lam * P.lam_down, 1e-10f);
    } else {
      lam = fminf(lam * P.lam_up, 1e6f);
    }
    if (improve) best_err = best_a_err;
  }
  for (int a = gl; a < n_act; a += G) A.out_cfg[gs * n_act + a] = W.best[a];
  if (gl == 0) A.out_err[gs] = best_err;
  __syncwarp(gm);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

__device__ __forceinline__ WideWarp w_group_area(const WideLayout& L, unsigned char* smem, int group) {
  unsigned char* b = smem + L.warps + L.warp_bytes * group;
  WideWarp W;
  W.cfg = reinterpret_cast<float*>(b + L.w_cfg);
  W.best = reinterpret_cast<float*>(b + L.w_best);
  W.dact = reinterpret_cast<float*>(b + L.w_dact);
  W.trial = reinterpret_cast<float*>(b + L.w_trial);
  W.dcol = reinterpret_cast<float*>(b + L.w_dcol);
  W.cs = reinterpret_cast<float*>(b + L.w_cs);
  W.r = reinterpret_cast<float*>(b + L.w_r);
  W.fw = reinterpret_cast<float*>(b + L.w_fw);
  W.pee = reinterpret_cast<float*>(b + L.w_pee);
  W.T = reinterpret_cast<float*>(b + L.w_T);
  W.J = reinterpret_cast<float*>(b + L.w_J);
  W.A = reinterpret_cast<float*>(b + L.w_A);
  W.y = reinterpret_cast<float*>(b + L.w_y);
  W.b = reinterpret_cast<float*>(b + L.w_b);
  W.d = reinterpret_cast<float*>(b + L.w_d);
  W.t = reinterpret_cast<double*>(b + L.w_t);
  W.pos = reinterpret_cast<float4*>(b + L.w_pos);
  W.slotB = reinterpret_cast<float4*>(b + L.w_slot);
  W.slotL = reinterpret_cast<int4*>(b + L.w_slot + 16 * (size_t)L.max_joints);
  return W;
}

// Grid launch (P.queue == null): block (x, y) runs seeds [x * chunk, ...) of
// problem y of class 0.  Persistent launch: blocks take items from the list
// through the counter P.queue[0] until it runs out, skipping items of
// classes that use the other body.  Groups of G lanes take the item's seeds
// in turn.
template <int G, int MAXEE>
__global__ void __launch_bounds__(256, 2) lm_warp_kernel(const __grid_constant__ WideLaunch P) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  __shared__ WideArgs s_args;
  WideShared& sh = *reinterpret_cast<WideShared*>(smem);
  const int group = threadIdx.x / G, gl = threadIdx.x % G, ngroups = blockDim.x / G;
  const unsigned gm = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  const WideWarp W = w_group_area(P.L, smem, group);
  int staged_cls = -1, staged_pb = -1;
  for (int round = 0;; ++round) {
    int4 item;
    if (P.queue) {
      if (threadIdx.x == 0) s_item = atomicAdd(P.queue, 1);
      __syncthreads();
      const int it = s_item;
      __syncthreads();
      if (it >= P.n_items) break;
      item = P.items[it];
      if (item.x < 0 || item.x >= P.n_classes) continue;
      int body;
      pick_class(P.body, item.x, body);
      if (body != kBodyWarp) continue;
    } else {
      if (round > 0) break;
      const int first = blockIdx.x * P.grid_chunk;
      item = make_int4(0, blockIdx.y, first, min(P.grid_chunk, P.cls[0].seed_stride - first));
    }
    if (item.x != staged_cls) {
      if (threadIdx.x == 0) pick_class(P.cls, item.x, s_args);
      __syncthreads();
    }
    const WideArgs& A = s_args;
    if (item.y < 0 || item.y >= A.n_problems || item.z < 0 || item.w <= 0 || item.z + item.w > A.seed_stride) {
      staged_cls = -1;  // malformed item: nothing is read or written for it
      __syncthreads();
      continue;
    }
    if (item.x != staged_cls) {
      wide_stage_class(P, A, smem);
      staged_cls = item.x;
      staged_pb = -1;
    }
    if (item.y != staged_pb) {
      wide_stage_targets(A, item.y, sh);
      __syncthreads();
      staged_pb = item.y;
    }
    for (int s = group; s < item.w; s += ngroups)
      w_seed<G, MAXEE>(P, A, sh, smem, W, (size_t)item.y * A.seed_stride + item.z + s, gl, gm);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

static WideArgs wide_args(const pk_ik_class& c) {
  WideArgs a{};
  a.m = ModelArgs{c.twists, c.parent_tf, c.parent_idx, c.act_idx, c.mimic_mul, c.mimic_off, c.mimic_act_idx,
                  c.topo_inv, c.n_joints, c.n_act};
  a.seeds = c.seeds; a.target_jnts = c.target_jnts; a.ancestor_masks = c.ancestor_masks;
  a.target_Ts = c.target_Ts; a.spheres_local = c.robot_spheres_local; a.sphere_joint = c.robot_sphere_joint_idx;
  a.self_i = c.self_i; a.self_j = c.self_j; a.lower = c.lower; a.upper = c.upper; a.fixed_mask = c.fixed_mask;
  a.out_cfg = c.out_cfg; a.out_err = c.out_err;
  a.n_act = c.n_act; a.n_ee = c.n_ee; a.n_rs = c.n_robot_spheres; a.n_self = c.n_self;
  a.seed_stride = c.seed_stride; a.n_problems = c.n_problems;
  return a;
}

static void wide_options(WideLaunch& P, const pk_lm_options& o) {
  P.max_iter = o.max_iter; P.pos_w = o.pos_weight; P.ori_w = o.ori_weight; P.lam0 = o.lambda_init;
  P.lam_down = o.lambda_down; P.lam_up = o.lambda_up; P.eps_pos = o.eps_pos; P.eps_ori = o.eps_ori;
  P.coll = o.enable_collision ? 1 : 0; P.coll_w = o.collision_weight; P.margin = o.collision_margin;
  P.grid_n = lm_grid_option(o.obstacle_grid, P.w.Ms);
  P.grid_auto = o.obstacle_grid == 0;
}

static int wide_group(const pk_lm_options& o) { return o.lanes_per_wide_seed == 32 ? 32 : 16; }

struct WideMax {
  int rs, self, joints, act, ee;
};

// Largest per-class extents over the warp-body classes of P.
static WideMax wide_max(const WideLaunch& P) {
  WideMax m{0, 0, 1, 1, 1};
  for (int c = 0; c < P.n_classes; ++c) {
    if (P.body[c] != kBodyWarp) continue;
    const WideArgs& a = P.cls[c];
    m.rs = std::max(m.rs, a.n_rs);
    m.self = std::max(m.self, P.coll ? a.n_self : 0);
    m.joints = std::max(m.joints, a.m.n_joints);
    m.act = std::max(m.act, a.n_act);
    m.ee = std::max(m.ee, a.n_ee);
  }
  return m;
}

// Chooses the block size (256, 128 or 64 threads) that keeps the most seeds
// resident per SM within the shared-memory limit, sets P.L for it and
// launches: a (problem, seed block) grid, or one persistent wave.
template <int G, int MAXEE>
static int run_warp_t(WideLaunch& P, const WideMax& mx, int grid_seeds, int grid_problems, bool persistent,
                      int blocks, cudaStream_t st, int* launched) {
  auto kern = lm_warp_kernel<G, MAXEE>;
  int dev = 0, max_smem = 0, sms = 0;
  if (int s = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return s;
  if (int s = cuda_status(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "attribute"))
    return s;
  if (int s = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute")) return s;
  int best_threads = 0, best_per_sm = 0, best_groups = -1;
  WideLayout best{};
  // the default grid resolution, and the coarser 8 cells when it keeps more
  // seeds resident (its lists and cells take less shared memory)
  const int grids[2] = {P.grid_n, (P.grid_auto && P.grid_n > kObsGridDefault) ? kObsGridDefault : -1};
  for (int gi = 0; gi < 2; ++gi) {
    if (grids[gi] < 0) continue;
    for (int threads = 256; threads >= 64 && threads >= G; threads >>= 1) {
      const WideLayout L = wide_layout(mx.rs, mx.self, mx.joints, mx.act, mx.ee, P.w, threads / G, grids[gi]);
      if (L.total > (size_t)max_smem) continue;
      if (int s = set_smem_limit((const void*)kern, L.total)) return s;
      int per_sm = 0;
      if (int s = cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, L.total),
                              "occupancy"))
        return s;
      const int groups = per_sm * (threads / G);
      if (groups > best_groups) { best_groups = groups; best_threads = threads; best_per_sm = per_sm; best = L; }
    }
  }
  PK_CHECK_CAP(best_threads > 0 && best_per_sm > 0,
               "warp-body LM working set does not fit in %d B of shared memory even for one seed group per block",
               max_smem);
  P.L = best;
  if (int s = set_smem_limit((const void*)kern, best.total)) return s;
  dim3 grid;
  if (persistent) {
    grid = dim3(blocks > 0 ? blocks : std::max(1, sms * best_per_sm));
  } else {
    P.grid_chunk = 2 * (best_threads / G);
    grid = dim3((grid_seeds + P.grid_chunk - 1) / P.grid_chunk, grid_problems);
  }
  kern<<<grid, best_threads, best.total, st>>>(P);
  if (launched) ++*launched;
  return cuda_status(cudaGetLastError(), "lm_warp_kernel launch");
}

static int run_warp(WideLaunch& P, int G, int grid_seeds, int grid_problems, bool persistent, int blocks,
                    cudaStream_t st, int* launched) {
  const WideMax mx = wide_max(P);
  if (G == 32)
    return mx.ee <= 2 ? run_warp_t<32, 2>(P, mx, grid_seeds, grid_problems, persistent, blocks, st, launched)
                      : run_warp_t<32, 4>(P, mx, grid_seeds, grid_problems, persistent, blocks, st, launched);
  return mx.ee <= 2 ? run_warp_t<16, 2>(P, mx, grid_seeds, grid_problems, persistent, blocks, st, launched)
                    : run_warp_t<16, 4>(P, mx, grid_seeds, grid_problems, persistent, blocks, st, launched);
}

static int validate_wide_class(const pk_ik_class& c, bool coll) {
  PK_CHECK_ARG(c.n_problems >= 0 && c.seed_stride >= 0 && c.n_act >= 0 && c.n_joints >= 0 && c.n_ee >= 1 &&
                   c.n_robot_spheres >= 0 && c.n_self >= 0,
               "bad class extents");
  PK_CHECK_CAP(c.n_joints <= PK_MAX_JOINTS, "n_joints=%d exceeds %d", c.n_joints, PK_MAX_JOINTS);
  PK_CHECK_CAP(c.n_act <= PK_MAX_ACT, "n_act=%d exceeds %d", c.n_act, PK_MAX_ACT);
  PK_CHECK_CAP(c.n_ee <= PK_MAX_EE, "n_ee=%d exceeds %d", c.n_ee, PK_MAX_EE);
  PK_CHECK_ARG(c.twists && c.parent_tf && c.parent_idx && c.act_idx && c.mimic_mul && c.mimic_off &&
                   c.mimic_act_idx && c.topo_inv && c.target_jnts && c.ancestor_masks && c.target_Ts &&
                   c.lower && c.upper && c.fixed_mask && c.seeds && c.out_cfg && c.out_err,
               "null buffer in class");
  PK_CHECK_ARG(c.n_robot_spheres == 0 || (c.robot_spheres_local && c.robot_sphere_joint_idx),
               "null robot spheres");
  PK_CHECK_ARG(!coll || c.n_self == 0 || (c.self_i && c.self_j), "null self pairs");
  return PK_OK;
}


int launch_warp_grid(const pk_ik_class& c, const WorldArgs& w, const pk_lm_options& opt, cudaStream_t st) {
  if (int s = validate_wide_class(c, opt.enable_collision != 0)) return s;
  if (c.n_problems == 0 || c.seed_stride == 0) return PK_OK;
  PK_CHECK_CAP(c.n_problems <= 65535, "n_problems=%d exceeds the grid limit 65535", c.n_problems);
  WideLaunch P{};
  P.cls[0] = wide_args(c);
  P.body[0] = kBodyWarp;
  P.n_classes = 1;
  P.w = w;
  wide_options(P, opt);
  P.queue = nullptr;
  return run_warp(P, wide_group(opt), c.seed_stride, c.n_problems, false, 0, st, nullptr);
}

int launch_warp_batch(const BatchCall& b, cudaStream_t st, int* launched) {
  WideLaunch P{};
  bool any = false;
  for (int c = 0; c < b.n_classes; ++c) {
    P.cls[c] = wide_args(b.cls[c]);
    P.body[c] = b.cls[c].body;
    if (b.cls[c].body == kBodyWarp) {
      if (int s = validate_wide_class(b.cls[c], b.opt.enable_collision != 0)) return s;
      any = true;
    }
  }
  if (!any || b.n_items == 0) return PK_OK;
  P.n_classes = b.n_classes;
  P.w = b.w;
  wide_options(P, b.opt);
  P.items = b.items;
  P.n_items = b.n_items;
  P.queue = b.queue + 1;
  return run_warp(P, wide_group(b.opt), 0, 0, true, b.blocks, st, launched);
}

}  // namespace pk
