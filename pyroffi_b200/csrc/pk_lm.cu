// Multi-seed Levenberg-Marquardt IK with a collision hinge penalty, FP64
// winner re-verification.
//
// pk_ls_ik_cuda replaces the reference's "ls_ik_cuda" XLA FFI target
// (src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:65-529).  The iteration is
// the reference's: residual = world position difference + rotation vector of
// q_ee * conj(q_tgt); stacked geometric Jacobian; row weights; Jacobi column
// scaling; damped normal equations with fixed-joint masking and a Cholesky
// solve (FP64 in the reference; here the FP32 dual system with one
// conditional FP64 refinement, lm_solve_f32); trust-region clip; 5-point
// line search on clamped trials; accept/reject of the damping step;
// all-time best tracking.
//
// B200 mapping:
//  * a group of TPS adjacent lanes owns one seed (TPS = 1 by default: one
//    lane per seed, 128 seeds per block).  Every lane of a group runs the
//    (cheap) FK / Jacobian / damped-step math redundantly, so the group's
//    decisions are bit-identical without broadcasts; with TPS > 1 the
//    (dominant) collision penalty is split over the group's lanes and the
//    partial sums meet in a butterfly shuffle; with one lane per seed the
//    self pairs are drained by the whole warp (self_warp).
//  * robot description, obstacle set, sphere list, limits and this block's
//    targets are staged once per block in shared memory; joint poses of
//    each lane live in a bank-strided shared slot array; configuration,
//    Jacobian and damping state stay in registers (all loops over the DOF
//    are unrolled to the compile-time bucket MAXA, padded dimensions are
//    masked like fixed joints).
//  * the collision penalty never touches most (sphere, obstacle) pairs:
//    every sphere-carrying joint gets a bounding sphere; a per-block
//    uniform grid over the world spheres hands each joint only the obstacles
//    whose (inflated) ball covers the joint's cell; self pairs are grouped
//    by joint pair and a group is skipped when the two bounding spheres are
//    margin apart.  All culls are conservative (exact in real arithmetic,
//    with slack for FP32), so the penalty equals the brute-force sum.
//  * hinge terms are tested on squared distance first:
//    d - margin < 0  <=>  |c - o|^2 < (r_s + r_o + margin)^2 for a positive
//    sum, so the square root runs only for the rare active pairs.
//  * the penalty at the current configuration is carried from the accepted
//    trial instead of being recomputed (it is the same value).
#include <float.h>

#include <algorithm>

#include "pk_batch.cuh"
#include "pk_damped_step.cuh"
#include "pk_obstacle_grid.cuh"

namespace pk {

struct LmArgs {
  ModelArgs m;
  WorldArgs w;
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
  int P, Sd, n_act, n_ee, n_rs, n_self;
  int max_iter;
  float pos_w, ori_w, lam0, lam_down, lam_up, eps_pos, eps_ori;
  int coll;
  float coll_w, margin;
  int spb;
  int f64_solve;  // the damped step's system in FP64 (seed-group kernel, one lane per seed); else FP32
  int grid_n;     // obstacle grid cells per axis (0: no grid, every obstacle takes the bounding test)
  int grid_auto;  // grid_n is the default resolution (the launch may coarsen it; see lm_fit_grid)
};

// Shared-memory layout of one LM block.
struct LmShared {
  JointTable jt;
  unsigned long long anc[PK_MAX_EE];  // ancestor bits by original joint index
  float tgt[PK_MAX_EE][7];
  int tsorted[PK_MAX_EE];
  float lo[PK_MAX_ACT], hi[PK_MAX_ACT];
  int fixed[PK_MAX_ACT];
  float4 jb[PK_MAX_JOINTS];        // bounding sphere of each sphere-carrying joint (joint frame)
  int jstart[PK_MAX_JOINTS + 1];   // sphere range per sphere-carrying joint
  int pjstart[PK_MAX_JOINTS + 1];  // range of sphere pairs (the paired table) per sphere-carrying joint
  int jlist[PK_MAX_JOINTS];        // sorted joint position per sphere-carrying joint
  int n_js;
  int n_rs;                        // valid robot spheres after staging
  int n_groups;                    // self-pair groups
  int grid_on;
  int grid_n;                      // cells per axis of the grid in use
  float3 glo, ginv;                // obstacle grid origin, inverse cell size
  float rmax;                      // largest joint bounding radius
};

template <int N>
__device__ __forceinline__ float reg_get(const float (&a)[N], int i) {
  float v = 0.f;
#pragma unroll
  for (int k = 0; k < N; ++k) v = (k == i) ? a[k] : v;
  return v;
}

// Line-search step sizes {1, 0.5, 0.25, 0.1, 0.025} (_ls_ik_cuda_kernel.cu:339).
__device__ __forceinline__ float line_alpha(int i) {
  return i == 0 ? 1.0f : i == 1 ? 0.5f : i == 2 ? 0.25f : i == 3 ? 0.1f : 0.025f;
}

// World spheres are padded to whole 32*TPS chunks so the culling loop needs no bounds test.
__host__ __device__ __forceinline__ int lm_ms_pad(int Ms, int tps) {
  const int chunk = 32 * tps;
  return ((Ms + chunk - 1) / chunk) * chunk;
}

// Self-pair groups per chunk of the warp item list (one lane per seed).
constexpr int kSelfChunk = 16;

// Seeds per block of the 16-wide one-lane kernel by default: the 16-DOF /
// 2-EE register state takes the whole register file at 2 blocks of 128
// threads, and a 128-seed block's per-seed pose slots push a 500-obstacle
// world's block past half of the SM's shared memory; 96 keeps 2 blocks.
constexpr int kSeedsPerBlock16 = 96;

// Trial-lane kernel: float4 positions per seed, padded by one float4 so the
// 6 seeds of a warp reading the same sphere use different bank groups.
__host__ __device__ __forceinline__ int lm_pos4_stride(int n_rs) { return n_rs + 1; }

// Byte offsets of the LM block's dynamic shared memory.
struct LmLayout {
  size_t rs, rsp, ws, pairs, pair4, prec, pgstart, wscr, gjoint, gstart, rsj, rsk, cells, cell_obs, wc, wb, wh, slots, cen, pos, scratch,
      total;
  int ms_pad, grid, max_entries, scratch_ints, recs;
};

__host__ __device__ inline size_t lm_align16(size_t x) { return (x + 15) & ~size_t(15); }

// threads == 0: seed-group kernel.  Per seed, the joint pose slots and the
// bounding-sphere centres, both laid out item-major ([item][spb]: component
// c of item i of seed g at (i * K + c) * spb + g), so seeds reading the same
// item hit distinct banks.  Sphere world positions are never stored: world
// obstacles are moved into joint frames and self pairs go through one
// relative transform per joint pair.  Both run on packed FP32x2 arithmetic,
// two spheres or two pairs per operation, from paired tables: each joint's
// spheres in pairs (float4 (x0, x1, y0, y1), (z0, z1, r0, r1); an odd joint
// padded with a sphere of radius -1e9), and each self-pair group's pairs in
// pairs (float4 (-ax0, -ax1, -ay0, -ay1), (-az0, -az1, rr0, rr1),
// (bx0, bx1, by0, by1), (bz0, bz1, rr0|rr0|, rr1|rr1|) with rr = r_a + r_b +
// margin; an odd group padded with a pair that never hits).  The staging
// scratch (self-pair key counts, obstacle boxes) overlays the per-seed area
// before the seeds run.
// threads > 0: trial-lane kernel (per-lane pose slots for `threads` lanes,
// per-seed sphere positions).
__host__ __device__ inline LmLayout lm_layout(const LmArgs& a, int tps, int threads = 0) {
  LmLayout L;
  size_t o = lm_align16(sizeof(LmShared));
  const int n_rs = a.n_rs, n_self = a.coll ? a.n_self : 0;
  L.ms_pad = lm_ms_pad(a.w.Ms, tps);
  if (threads == 0) {
    L.scratch_ints = a.coll ? max(a.m.n_joints * a.m.n_joints, a.w.Ms) : 0;
  } else {
    L.scratch_ints = 7 * a.m.n_joints * threads;  // the pose slots double as staging scratch
  }
  L.grid = (a.grid_n > 0 && a.coll && a.w.Ms >= 32 && a.w.Ms <= 65535 && a.w.Ms <= L.scratch_ints) ? 1 : 0;
  // list capacity: a finer grid lists each obstacle in more cells
  L.max_entries = L.grid ? obstacle_grid_capacity(a.grid_n, a.w.Ms) : 0;
  L.rs = o; o = lm_align16(o + 16 * (size_t)n_rs);
  L.rsp = o; o = lm_align16(o + (threads == 0 ? 16 * (size_t)(n_rs + a.m.n_joints) : 0));
  // the world, in stage_world's layout: spheres in ms_pad float4 slots, then
  // capsules, boxes, halfspaces, each on a 16-byte boundary
  L.ws = o; o = lm_align16(o + 16 * (size_t)L.ms_pad);
  L.wc = o; o = lm_align16(o + 28 * (size_t)a.w.Mc);
  L.wb = o; o = lm_align16(o + 60 * (size_t)a.w.Mb);
  L.wh = o; o = lm_align16(o + 24 * (size_t)a.w.Mh);
  L.pairs = o; o = lm_align16(o + 8 * (size_t)n_self);
  L.pair4 = o; o = lm_align16(o + (threads > 0 ? 16 * (size_t)n_self : 0));
  L.prec = o; o = lm_align16(o + (threads == 0 ? 64 * (size_t)n_self : 0));
  L.pgstart = o; o = lm_align16(o + (threads == 0 ? 4 * (size_t)(n_self + 2) : 0));
  // one lane per seed: per warp, the self-pair item list (kSelfChunk * 32 u16)
  // and the item sums (kSelfChunk * 32 floats)
  L.wscr = o; o = lm_align16(o + ((threads == 0 && tps == 1 && n_self > 0) ? (size_t)(a.spb / 32) * kSelfChunk * 32 * 6 : 0));
  L.recs = threads == 0 ? 1 : 0;
  L.gjoint = o; o = lm_align16(o + 8 * (size_t)(n_self + 1));
  L.gstart = o; o = lm_align16(o + 4 * (size_t)(n_self + 2));
  L.rsj = o; o = lm_align16(o + 4 * (size_t)n_rs);
  L.rsk = o; o = lm_align16(o + 4 * (size_t)n_rs);
  L.cells = o; o = lm_align16(o + (L.grid ? 4 * (size_t)(obstacle_grid_cells(a.grid_n) + 1) : 0));
  L.cell_obs = o; o = lm_align16(o + 2 * (size_t)L.max_entries);
  if (threads == 0) {
    L.slots = o; o = lm_align16(o + 28 * (size_t)a.m.n_joints * a.spb);
    // bounding centres are kept per seed only where other lanes read them:
    // lanes sharing a seed (tps > 1) or the warp-shared self-pair items
    L.cen = o; o = lm_align16(o + ((a.coll && (tps > 1 || n_self > 0)) ? 12 * (size_t)a.m.n_joints * a.spb : 0));
    L.scratch = L.slots;
    L.pos = o;
    o = max(o, lm_align16(L.scratch + 4 * (size_t)L.scratch_ints));
  } else {
    L.slots = o; o = lm_align16(o + 28 * (size_t)a.m.n_joints * threads);
    L.pos = o; o = lm_align16(o + 16 * (size_t)lm_pos4_stride(n_rs) * a.spb);
    L.scratch = L.slots;
    L.cen = L.pos;
  }
  L.total = o;
  return L;
}

// FK of one configuration computed by every lane of a seed group (identical
// values) and stored by the leader only.  A non-chain parent is read back
// from the shared slots, so a tree needs the group to sync after each store.
template <typename CfgFn>
__device__ __forceinline__ void fk_group(const JointTable& jt, CfgFn cfg_at, const PoseSlots& out, bool leader,
                                         unsigned gmask) {
  Pose prev = pose_identity();
  const int n = jt.n;
  const bool chain = jt.chain != 0;
  for (int i = 0; i < n; ++i) {
    const int src = jt.src[i];
    const float qref = (src < 0) ? 0.f : cfg_at(src);
    const float q = qref * jt.mul[i] + jt.off[i];
    const Pose Tpc = joint_local(jt, i, q);
    const int ps = jt.psorted[i];
    Pose Tw;
    if (ps < 0) Tw = Tpc;
    else if (ps == i - 1) Tw = pose_compose(prev, Tpc);
    else Tw = pose_compose(out.load(ps), Tpc);
    if (leader) out.store(i, Tw);
    if (!chain) __syncwarp(gmask);
    prev = Tw;
  }
}

template <int TPS>
__device__ __forceinline__ float group_sum(float v, unsigned gmask) {
#pragma unroll
  for (int o = TPS / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
  return v;
}

struct PenaltyCtx {
  const float4* rs;      // robot spheres (x, y, z, r) in their joint frame, grouped by joint slot
  const float4* jb;      // per sphere-carrying joint slot: bounding sphere (x, y, z, R) in its frame
  const int* jstart;     // [n_js + 1] sphere range of each joint slot
  const int* jlist;      // [n_js] sorted joint position of each joint slot
  const float4* ws;      // world spheres (x, y, z, r + margin), padded to a multiple of 32*TPS
  const float* wc;
  const float* wb;
  const float* wh;
  const float4* rsp;     // robot spheres in pairs, 2 float4 per pair (the layout's paired sphere table)
  const int* pjstart;    // [n_js + 1] sphere-pair range of each joint slot
  const float4* prec;    // self pairs in pairs, 4 float4 per pair of pairs (the layout's paired pair table)
  const int2* gjoint;    // [n_groups] joint slots (x, y) of each self-pair group
  const int* pgstart;    // [n_groups + 1] padded pair range of each group (even)
  const int* cell_start; // [G^3 + 1] obstacle grid (null: no grid, scan every obstacle)
  const unsigned short* cell_obs;
  float* cen;            // this seed's bounding centres: component c of slot j at cen[(3 j + c) * cs]
                         // (null: not kept; each lane computes its seed's centres where it needs them)
  int cs;
  float3 glo, ginv;      // grid origin and inverse cell size
  int gn;                // grid cells per axis
  int n_rs, n_js, n_groups, Ms_pad, Mc, Mb, Mh;
  float margin;
};

// Hinge term of a sphere pair given squared centre distance d2 and
// rr = r_a + r_b + margin: (d - margin)^2 when d < margin.  Tested on d2
// first (for rr > 0, d < margin <=> d2 < rr^2; rr <= 0 never hits).
__device__ __forceinline__ void hinge_sq(float d2, float rr, float& pen) {
  if (d2 < rr * fabsf(rr)) {
    const float e = sqrtf(d2) - rr;
    pen += e * e;
  }
}

// Exact hinge terms of the sphere pairs [p0, p1) of a joint against world
// sphere O (radius already + margin), with the obstacle centre moved into
// the joint's frame (T) once: |R c_k + t - o| = |c_k - R^T (o - t)|; two
// spheres per packed FP32x2 operation, terms added in sphere order.
__device__ __forceinline__ void narrow_world(const PenaltyCtx& c, const Pose& T, int p0, int p1, float4 O,
                                             float& pen) {
  const float3 o = pose_apply_inv(T, make_float3(O.x, O.y, O.z));
  const float2 nx = make_float2(-o.x, -o.x), ny = make_float2(-o.y, -o.y), nz = make_float2(-o.z, -o.z);
  const float2 ow = make_float2(O.w, O.w);
  for (int p = p0; p < p1; ++p) {
    const float4 s0 = c.rsp[2 * p], s1 = c.rsp[2 * p + 1];
    const float2 dx = __fadd2_rn(make_float2(s0.x, s0.y), nx);
    const float2 dy = __fadd2_rn(make_float2(s0.z, s0.w), ny);
    const float2 dz = __fadd2_rn(make_float2(s1.x, s1.y), nz);
    float2 d2 = __fmul2_rn(dx, dx);
    d2 = __ffma2_rn(dy, dy, d2);
    d2 = __ffma2_rn(dz, dz, d2);
    const float2 rr = __fadd2_rn(make_float2(s1.z, s1.w), ow);
    hinge_sq(d2.x, rr.x, pen);
    hinge_sq(d2.y, rr.y, pen);
  }
}

// Hinge terms of the pairs of self-pair group gi of one seed (poses in ps),
// added to pen in pair order: one relative transform T_x^-1 T_y (rotation
// conj(q_x) q_y as a matrix M, translation u = R_x^T (t_y - t_x)), then per
// pair |c_a - (M c_b + u)| from the joint-frame records, two pairs per
// packed FP32x2 operation.
__device__ __forceinline__ void group_pairs(const PenaltyCtx& c, const PoseSlots& ps, int gi, float& pen) {
  const int2 ja = c.gjoint[gi];
  const Pose A = ps.load(c.jlist[ja.x]);
  const Pose Bp = ps.load(c.jlist[ja.y]);
  const float qw = A.w * Bp.w + A.x * Bp.x + A.y * Bp.y + A.z * Bp.z;
  const float qx = A.w * Bp.x - A.x * Bp.w - A.y * Bp.z + A.z * Bp.y;
  const float qy = A.w * Bp.y + A.x * Bp.z - A.y * Bp.w - A.z * Bp.x;
  const float qz = A.w * Bp.z - A.x * Bp.y + A.y * Bp.x - A.z * Bp.w;
  const float3 u = pose_apply_inv(A, make_float3(Bp.tx, Bp.ty, Bp.tz));
  auto dup = [](float v) { return make_float2(v, v); };
  const float2 m00 = dup(1.f - 2.f * (qy * qy + qz * qz)), m01 = dup(2.f * (qx * qy - qw * qz)),
               m02 = dup(2.f * (qx * qz + qw * qy));
  const float2 m10 = dup(2.f * (qx * qy + qw * qz)), m11 = dup(1.f - 2.f * (qx * qx + qz * qz)),
               m12 = dup(2.f * (qy * qz - qw * qx));
  const float2 m20 = dup(2.f * (qx * qz - qw * qy)), m21 = dup(2.f * (qy * qz + qw * qx)),
               m22 = dup(1.f - 2.f * (qx * qx + qy * qy));
  const float2 ux = dup(u.x), uy = dup(u.y), uz = dup(u.z);
  // two pairs per packed FP32x2 operation: e = M c_b + u - c_a
  const int q1 = c.pgstart[gi + 1];
  for (int q = c.pgstart[gi]; q < q1; q += 2) {
    const float4 r0 = c.prec[2 * q], r1 = c.prec[2 * q + 1], r2 = c.prec[2 * q + 2], r3 = c.prec[2 * q + 3];
    const float2 bx = make_float2(r2.x, r2.y), by = make_float2(r2.z, r2.w), bz = make_float2(r3.x, r3.y);
    const float2 ex = __ffma2_rn(m00, bx, __ffma2_rn(m01, by, __ffma2_rn(m02, bz, __fadd2_rn(ux, make_float2(r0.x, r0.y)))));
    const float2 ey = __ffma2_rn(m10, bx, __ffma2_rn(m11, by, __ffma2_rn(m12, bz, __fadd2_rn(uy, make_float2(r0.z, r0.w)))));
    const float2 ez = __ffma2_rn(m20, bx, __ffma2_rn(m21, by, __ffma2_rn(m22, bz, __fadd2_rn(uz, make_float2(r1.x, r1.y)))));
    float2 d2 = __fmul2_rn(ex, ex);
    d2 = __ffma2_rn(ey, ey, d2);
    d2 = __ffma2_rn(ez, ez, d2);
    if (d2.x < r3.z) { const float e = sqrtf(d2.x) - r1.z; pen += e * e; }
    if (d2.y < r3.w) { const float e = sqrtf(d2.y) - r1.w; pen += e * e; }
  }
}

// Self pairs of one seed, split over its TPS lanes (TPS > 1): the
// bounding-sphere culls of the joint-slot groups into a mask of this lane's
// surviving groups (survivors go round-robin to the seed's lanes), then the
// pairs of those groups in increasing group order.
template <int TPS>
__device__ __forceinline__ void self_share(const PenaltyCtx& c, const PoseSlots& ps, int t, float& pen) {
  const float* const cen = c.cen;
  const int cs = c.cs;
  int turn = 0;  // surviving groups seen so far (the same count on every lane of the seed)
  for (int g0 = 0; g0 < c.n_groups; g0 += 32) {
    unsigned mask = 0u;
    for (int i = 0; i < 32 && g0 + i < c.n_groups; ++i) {
      const int2 ja = c.gjoint[g0 + i];
      const float dx = cen[(3 * ja.x) * cs] - cen[(3 * ja.y) * cs];
      const float dy = cen[(3 * ja.x + 1) * cs] - cen[(3 * ja.y + 1) * cs];
      const float dz = cen[(3 * ja.x + 2) * cs] - cen[(3 * ja.y + 2) * cs];
      const float rr = c.jb[ja.x].w + c.jb[ja.y].w + c.margin;
      if (!(dx * dx + dy * dy + dz * dz < rr * fabsf(rr))) continue;
      if ((turn++ & (TPS - 1)) == t) mask |= 1u << i;
    }
    while (mask) {
      const int gi = g0 + __ffs(mask) - 1;
      mask &= mask - 1u;
      group_pairs(c, ps, gi, pen);
    }
  }
}

// Self pairs of the 32 seeds of a warp (TPS == 1), all 32 lanes together.
// Per chunk of kSelfChunk groups, each lane culls the groups for its own
// seed (none when !need); the surviving (seed, group) items go into the
// warp's list in (group, lane) order; lane l takes items l, l + 32, ... and
// writes each item's sum (its pairs in pair order) to res[group][seed]; then
// each lane adds its own surviving groups' sums in group order.  The result
// does not depend on which lane took which item, and the work of a chunk is
// spread over the warp instead of following the seed with the most
// surviving groups.  slots_w: the pose slots of the warp's first seed; b4:
// the culls four groups per step.
__device__ __forceinline__ void self_warp(const PenaltyCtx& c, float* slots_w, int spb, bool need, bool b4,
                                          float& pen, unsigned short* list, float* res) {
  const int lane = threadIdx.x & 31;
  const float* const cen = c.cen;
  const int cs = c.cs;
  for (int g0 = 0; g0 < c.n_groups; g0 += kSelfChunk) {
    const int nc = min(kSelfChunk, c.n_groups - g0);
    unsigned mine = 0u;
    int n_items = 0;
    // this lane's surviving groups of the chunk (B4: four groups' loads at a time)
    if (need && !b4) {
      for (int i = 0; i < nc; ++i) {
        const int2 ja = c.gjoint[g0 + i];
        const float dx = cen[(3 * ja.x) * cs] - cen[(3 * ja.y) * cs];
        const float dy = cen[(3 * ja.x + 1) * cs] - cen[(3 * ja.y + 1) * cs];
        const float dz = cen[(3 * ja.x + 2) * cs] - cen[(3 * ja.y + 2) * cs];
        const float rr = c.jb[ja.x].w + c.jb[ja.y].w + c.margin;
        if (dx * dx + dy * dy + dz * dz < rr * fabsf(rr)) mine |= 1u << i;
      }
    } else if (need) {
      for (int i0 = 0; i0 < nc; i0 += 4) {
        float d2[4], rr[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int2 ja = c.gjoint[g0 + min(i0 + u, nc - 1)];
          const float dx = cen[(3 * ja.x) * cs] - cen[(3 * ja.y) * cs];
          const float dy = cen[(3 * ja.x + 1) * cs] - cen[(3 * ja.y + 1) * cs];
          const float dz = cen[(3 * ja.x + 2) * cs] - cen[(3 * ja.y + 2) * cs];
          rr[u] = c.jb[ja.x].w + c.jb[ja.y].w + c.margin;
          d2[u] = dx * dx + dy * dy + dz * dz;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (i0 + u < nc && d2[u] < rr[u] * fabsf(rr[u])) mine |= 1u << (i0 + u);
      }
    }
    for (int i = 0; i < nc; ++i) {
      const bool sv = (mine >> i) & 1u;
      const unsigned m = __ballot_sync(0xffffffffu, sv);
      if (sv) list[n_items + __popc(m & ((1u << lane) - 1u))] = (unsigned short)((lane << 8) | i);
      n_items += __popc(m);
    }
    __syncwarp();
    for (int k = lane; k < n_items; k += 32) {
      const int item = list[k];
      const int o = item >> 8, i = item & 255;
      float part = 0.f;
      group_pairs(c, PoseSlots{slots_w + o, spb}, g0 + i, part);
      res[i * 32 + o] = part;
    }
    __syncwarp();
    while (mine) {
      const int i = __ffs(mine) - 1;
      mine &= mine - 1u;
      pen += res[i * 32 + lane];
    }
    __syncwarp();  // the next chunk reuses list and res
  }
}

// Partial hinge penalty of lane t of a TPS-group (not weighted, not summed).
//  1. lane t puts the bounding-sphere centres of joint slots t, t+TPS, ...
//     (world frame) into this seed's shared slots;
//  2. world spheres: conservative culls before any sphere-level test.  The
//     joint's bounding sphere (centre B, radius R) can only reach obstacle o
//     if |B - o| < R + r_o + margin.  With the obstacle grid, only the
//     obstacles registered in B's cell (every obstacle whose ball of radius
//     r_o + margin + max R covers part of that cell) are candidates; lane t
//     takes candidates t, t+TPS, ...  Without it, lane t scans obstacles
//     t, t+TPS, ... into a 32-bit survivor mask.  A surviving obstacle is
//     moved into the joint's frame and tested against the joint's spheres;
//  3. capsules / boxes / halfspaces: lane t takes joint slots t, t+TPS, ...;
//     a joint whose bounding ball is margin clear of a capsule or box (both
//     distances are 1-Lipschitz in the point, so no sphere inside the ball
//     is closer) is skipped for it, else its spheres are tested in the world
//     frame;
//  4. self pairs by joint-slot group: a group is skipped when the two
//     joints' bounding spheres are margin apart; the surviving groups go
//     round-robin to the group's lanes, and a lane takes each of its groups
//     whole: one relative transform T_x^-1 T_y (as a rotation matrix), then
//     per pair |c_a - (M c_b + u)| from the joint-frame records.
//
// TPS == 1: every lane of the warp calls it (need == false: the lane adds
// nothing but takes part in the warp's self-pair items, self_warp); TPS > 1:
// the seed's lanes call it when the seed needs it.
//
// B4: the grid candidates and the self-pair group culls four per step (their
// loads in flight together).  The launch takes it for the one-lane 8-DOF
// kernel on a grid of 14 or more cells per axis (short lists): on longer
// lists, and in the 16-DOF kernels (registers), it measured slower.  The
// survivors are the same, but the compiler may contract a distance or a
// hinge sum differently in the two forms (one ulp in about 1 of 2,000
// outputs was seen).
template <int TPS, bool B4>
__device__ float penalty_share(const PenaltyCtx& c, const PoseSlots& ps, int t, unsigned gmask, bool need,
                               float* slots_w, int spb, unsigned short* wlist, float* wres) {
  float pen = 0.f;
  float* const cen = c.cen;
  const int cs = c.cs;
  const bool b4 = B4;
  // bounding centre of joint slot j: kept per seed, or computed here
  auto centre = [&](int j) {
    if (cen) return make_float3(cen[(3 * j) * cs], cen[(3 * j + 1) * cs], cen[(3 * j + 2) * cs]);
    const float4 bl = c.jb[j];
    return pose_apply(ps.load(c.jlist[j]), make_float3(bl.x, bl.y, bl.z));
  };
  if (need) {
    if (cen) {
      for (int j = t; j < c.n_js; j += TPS) {
        const Pose T = ps.load(c.jlist[j]);
        const float4 bl = c.jb[j];
        const float3 B = pose_apply(T, make_float3(bl.x, bl.y, bl.z));
        cen[(3 * j) * cs] = B.x; cen[(3 * j + 1) * cs] = B.y; cen[(3 * j + 2) * cs] = B.z;
      }
      if (TPS > 1) __syncwarp(gmask);
    }

    for (int j = 0; j < c.n_js && c.Ms_pad > 0; ++j) {
      const float R = c.jb[j].w;
      const float3 Bj = centre(j);
      const float Bx = Bj.x, By = Bj.y, Bz = Bj.z;
      const int p0 = c.pjstart[j], p1 = c.pjstart[j + 1];
      if (c.cell_start) {
        const int cell = obstacle_grid_cell(c.glo, c.ginv, c.gn, make_float3(Bx, By, Bz));
        if (cell < 0) continue;  // outside the grid no obstacle is within reach of this joint
        const int e1 = c.cell_start[cell + 1];
        // the lane's candidates in chunks of 32: bounding tests into a survivor
        // mask first, then the narrow tests of the survivors, so a warp runs
        // the narrow loop max-over-lanes times per chunk instead of once per
        // candidate slot in which any lane has a survivor
        for (int e0 = c.cell_start[cell] + t; e0 < e1; e0 += 32 * TPS) {
          unsigned mask = 0u;
          if (!b4) {
            for (int i = 0; i < 32 && e0 + i * TPS < e1; ++i) {
              const float4 O = c.ws[c.cell_obs[e0 + i * TPS]];
              const float rr = R + O.w;
              const float dx = Bx - O.x, dy = By - O.y, dz = Bz - O.z;
              if (dx * dx + dy * dy + dz * dz < rr * fabsf(rr)) mask |= 1u << i;
            }
          } else {
            // four candidates per step, their index and obstacle loads issued
            // together (independent shared-memory loads in flight instead of
            // one dependent pair per candidate); past the list end a step reads
            // obstacle 0 and tests nothing
            for (int i0 = 0; i0 < 32 && e0 + i0 * TPS < e1; i0 += 4) {
              int idx[4];
              bool in[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int e = e0 + (i0 + u) * TPS;
                in[u] = e < e1;
                idx[u] = in[u] ? (int)c.cell_obs[e] : 0;
              }
              float4 O[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) O[u] = c.ws[idx[u]];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const float rr = R + O[u].w;
                const float dx = Bx - O[u].x, dy = By - O[u].y, dz = Bz - O[u].z;
                if (in[u] && dx * dx + dy * dy + dz * dz < rr * fabsf(rr)) mask |= 1u << (i0 + u);
              }
            }
          }
          if (mask) {
            const Pose T = ps.load(c.jlist[j]);
            while (mask) {
              const int i = __ffs(mask) - 1;
              mask &= mask - 1u;
              narrow_world(c, T, p0, p1, c.ws[c.cell_obs[e0 + i * TPS]], pen);
            }
          }
        }
      } else {
        for (int ob = t; ob < c.Ms_pad; ob += 32 * TPS) {
          unsigned mask = 0u;
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float4 O = c.ws[ob + i * TPS];
            const float rr = R + O.w;
            const float dx = Bx - O.x, dy = By - O.y, dz = Bz - O.z;
            if (dx * dx + dy * dy + dz * dz < rr * fabsf(rr)) mask |= 1u << i;
          }
          if (mask) {
            const Pose T = ps.load(c.jlist[j]);
            while (mask) {
              const int i = __ffs(mask) - 1;
              mask &= mask - 1u;
              narrow_world(c, T, p0, p1, c.ws[ob + i * TPS], pen);
            }
          }
        }
      }
    }

    if (c.Mc + c.Mb + c.Mh > 0) {
      for (int j = t; j < c.n_js; j += TPS) {
        const float3 B = centre(j);
        const float R = c.jb[j].w;
        const int k0 = c.jstart[j], k1 = c.jstart[j + 1];
        const Pose T = ps.load(c.jlist[j]);
        for (int m = 0; m < c.Mc; ++m) {
          if (!(d_sphere_capsule(B, R, c.wc + 7 * m) < c.margin)) continue;
          for (int k = k0; k < k1; ++k) {
            const float4 s = c.rs[k];
            const float d = d_sphere_capsule(pose_apply(T, make_float3(s.x, s.y, s.z)), s.w, c.wc + 7 * m);
            if (d < c.margin) { const float e = d - c.margin; pen += e * e; }
          }
        }
        for (int m = 0; m < c.Mb; ++m) {
          if (!(d_sphere_box(B, R, c.wb + 15 * m) < c.margin)) continue;
          for (int k = k0; k < k1; ++k) {
            const float4 s = c.rs[k];
            const float d = d_sphere_box(pose_apply(T, make_float3(s.x, s.y, s.z)), s.w, c.wb + 15 * m);
            if (d < c.margin) { const float e = d - c.margin; pen += e * e; }
          }
        }
        for (int m = 0; m < c.Mh; ++m) {  // no cull: a normal need not be unit length
          for (int k = k0; k < k1; ++k) {
            const float4 s = c.rs[k];
            const float d = d_sphere_halfspace(pose_apply(T, make_float3(s.x, s.y, s.z)), s.w, c.wh + 6 * m);
            if (d < c.margin) { const float e = d - c.margin; pen += e * e; }
          }
        }
      }
    }

    if (TPS > 1) self_share<TPS>(c, ps, t, pen);
  }
  if (TPS == 1 && c.n_groups > 0) self_warp(c, slots_w, spb, need, b4, pen, wlist, wres);
  __syncwarp(gmask);
  return pen;
}

// Residual of every EE (reference helper _ik_cuda_helpers.cuh:472-499).
template <int MAXEE>
__device__ __forceinline__ void ee_residual(const LmShared& sh, const PoseSlots& ps, int n_ee,
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
    const float* g = sh.tgt[e];
    r[6 * e + 0] = T.tx - g[4];
    r[6 * e + 1] = T.ty - g[5];
    r[6 * e + 2] = T.tz - g[6];
    // q_err = q_ee * conj(q_tgt)
    const float bw = g[0], bx = -g[1], by = -g[2], bz = -g[3];
    float qw = T.w * bw - T.x * bx - T.y * by - T.z * bz;
    float qx = T.w * bx + T.x * bw + T.y * bz - T.z * by;
    float qy = T.w * by - T.x * bz + T.y * bw + T.z * bx;
    float qz = T.w * bz + T.x * by - T.y * bx + T.z * bw;
    if (qw < 0.f) { qw = -qw; qx = -qx; qy = -qy; qz = -qz; }
    const float s = sqrtf(qx * qx + qy * qy + qz * qz);
    float f;
    if (s > 1e-6f) f = 2.f * atan2f(s, qw) / s;
    else f = 2.f;
    r[6 * e + 3] = qx * f;
    r[6 * e + 4] = qy * f;
    r[6 * e + 5] = qz * f;
    pee[3 * e] = T.tx; pee[3 * e + 1] = T.ty; pee[3 * e + 2] = T.tz;
  }
}

// FP32 damped step with one conditional FP64 refinement step (the default
// form of lm_direction), on the same R x R dual system as the FP64 form:
// (Js Js^T + lam I) y = fw, p = -Js^T y (R = 6 MAXEE), fixed and padded
// joints as zero columns.  Its eigenvalues are sigma_i(Js)^2 + lam: unlike
// the MAXA x MAXA normal equations of a redundant arm, whose null space puts
// an eigenvalue at lam itself, it is only ill-conditioned near singular
// configurations.  The system and its Cholesky are FP32; when the squared
// ratio of the largest to the smallest pivot (over the live rows) exceeds
// 1e6, one step of iterative refinement follows: the residual
// fw - (Js Js^T + lam I) y in FP64 (from the FP32 Jacobian entries, which
// FP64 holds exactly), the correction solved with the FP32 factor.  With
// fewer free columns than live rows the primal system is solved instead, in
// the same way (damped_step_primal).  J is the column-scaled weighted
// Jacobian, fw the weighted residual; writes the unscaled step into delta
// (zero on a non-positive pivot).
template <int MAXA, int MAXEE>
__device__ __forceinline__ void lm_solve_f32(const LmShared& sh, const float (&J)[6 * MAXEE][MAXA],
                                             const float (&fw)[6 * MAXEE], int rows, float lam,
                                             const float (&col_s)[MAXA], float (&delta)[MAXA]) {
  constexpr int R = 6 * MAXEE;
  {
    // fewer free columns than live rows (fixed joints): the dual system
    // would carry the null space of Js^T as eigenvalues lam, so the primal
    // system (of full column rank then) is solved instead; block-uniform
    bool fr[MAXA];
    float zero[MAXA], x[MAXA];
    int nf = 0;
#pragma unroll
    for (int c = 0; c < MAXA; ++c) {
      fr[c] = !sh.fixed[c];
      zero[c] = 0.f;
      nf += fr[c] ? 1 : 0;
    }
    if (nf < rows) {
      bool ok;
      if constexpr (MAXA <= 8) ok = damped_step_primal<R, MAXA>(J, fw, lam, zero, fr, zero, zero, x);
      else ok = damped_step_primal_ool<R, MAXA>(J, fw, lam, zero, fr, zero, zero, x);
#pragma unroll
      for (int c = 0; c < MAXA; ++c) delta[c] = (ok && fr[c]) ? x[c] / col_s[c] : 0.f;
      return;
    }
  }
  float A[R * (R + 1) / 2];
#pragma unroll
  for (int i = 0; i < R; ++i) {
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      float acc = (i == j) ? lam : 0.f;
#pragma unroll
      for (int c = 0; c < MAXA; ++c)
        if (!sh.fixed[c]) acc = fmaf(J[i][c], J[j][c], acc);
      A[i * (i + 1) / 2 + j] = acc;
    }
  }
  // Cholesky A = L L^T in place, diagonal kept as its reciprocal
  bool ok = true;
  float pmax = 0.f, pmin = 3.4e38f;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    float s2 = A[k * (k + 1) / 2 + k];
#pragma unroll
    for (int q = 0; q < k; ++q) s2 = fmaf(-A[k * (k + 1) / 2 + q], A[k * (k + 1) / 2 + q], s2);
    if (!(s2 > 0.f)) ok = false;
    if (k < rows) {  // padding rows of absent EEs hold lam alone
      pmax = fmaxf(pmax, s2);
      pmin = fminf(pmin, s2);
    }
    const float inv = 1.f / sqrtf(ok ? s2 : 1.f);
    A[k * (k + 1) / 2 + k] = inv;
#pragma unroll
    for (int i = k + 1; i < R; ++i) {
      float tt = A[i * (i + 1) / 2 + k];
#pragma unroll
      for (int q = 0; q < k; ++q) tt = fmaf(-A[i * (i + 1) / 2 + q], A[k * (k + 1) / 2 + q], tt);
      A[i * (i + 1) / 2 + k] = tt * inv;
    }
  }
  auto solve = [&](float (&v)[R]) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      float s2 = v[i];
#pragma unroll
      for (int q = 0; q < i; ++q) s2 = fmaf(-A[i * (i + 1) / 2 + q], v[q], s2);
      v[i] = s2 * A[i * (i + 1) / 2 + i];
    }
#pragma unroll
    for (int i = R - 1; i >= 0; --i) {
      float s2 = v[i];
#pragma unroll
      for (int q = i + 1; q < R; ++q) s2 = fmaf(-A[q * (q + 1) / 2 + i], v[q], s2);
      v[i] = s2 * A[i * (i + 1) / 2 + i];
    }
  };
  float y[R];
#pragma unroll
  for (int i = 0; i < R; ++i) y[i] = fw[i];
  solve(y);
  if (ok && pmax > 1e6f * pmin) {
    // r = fw - (Js Js^T + lam I) y in FP64 over the free columns
    double u[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < R; ++k) acc = fma((double)J[k][c], (double)y[k], acc);
      u[c] = sh.fixed[c] ? 0.0 : acc;
    }
    float d[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      double acc = (double)lam * (double)y[i];
#pragma unroll
      for (int c = 0; c < MAXA; ++c) acc = fma((double)J[i][c], u[c], acc);
      d[i] = (float)((double)fw[i] - acc);
    }
    solve(d);
#pragma unroll
    for (int i = 0; i < R; ++i) y[i] = (float)((double)y[i] + (double)d[i]);
  }
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    float pc = 0.f;
#pragma unroll
    for (int k = 0; k < R; ++k) pc = fmaf(J[k][c], y[k], pc);
    delta[c] = (ok && !sh.fixed[c]) ? -pc / col_s[c] : 0.f;
  }
}

// Damped Gauss-Newton step of the current point (_ls_ik_cuda_kernel.cu:257-335):
// weighted stacked Jacobian from the joint poses in `ps`, Jacobi column
// scaling, normal equations (Js^T Js + lam I) p = -Js^T fw with fixed and
// padded joints masked, Cholesky solve (p = 0 on a non-positive pivot),
// unscaling and the trust-region clip.  Writes `delta`, returns ||fw||^2.
// The damped system is solved through its R x R dual form (R = 6 MAXEE
// residual rows; the reference solves the MAXA x MAXA normal equations in
// FP64, the same step in exact arithmetic).  F64S false (the default): the
// dual system and its Cholesky in FP32, with one FP64 refinement step when
// the squared pivot ratio exceeds 1e6 (lm_solve_f32).  F64S true: in FP64.
template <int MAXA, int MAXEE, bool F64S = false>
__device__ __forceinline__ float lm_direction(const LmShared& sh, const PoseSlots& ps, int n_ee, const float (&W)[6],
                                              const float (&r)[6 * MAXEE], const float (&pee)[3 * MAXEE],
                                              float lam, float max_p, float max_o, float (&delta)[MAXA]) {
  const JointTable& jt = sh.jt;
  // weighted stacked Jacobian J[k][c]
  float J[6 * MAXEE][MAXA];
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k)
#pragma unroll
    for (int c = 0; c < MAXA; ++c) J[k][c] = 0.f;
  for (int i = 0; i < jt.n; ++i) {
    const int jk = jt.jkind[i];
    const int a1 = jt.a1[i], a2 = jt.a2[i];
    if (jk == 0 || (a1 < 0 && a2 < 0)) continue;
    const Pose Tj = ps.load(i);
    const float3 z = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z,
                                 make_float3(jt.axis[i][0], jt.axis[i][1], jt.axis[i][2]));
    const float sm = jt.mul[i];
    const int orig = jt.orig[i];
#pragma unroll
    for (int e = 0; e < MAXEE; ++e) {
      if (e >= n_ee || !((sh.anc[e] >> orig) & 1ull)) continue;
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
  float fw[6 * MAXEE];
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k) {
    fw[k] = r[k] * W[k % 6];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) J[k][c] *= W[k % 6];
  }
  float fw2 = 0.f;
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k) fw2 += fw[k] * fw[k];

  // Jacobi column scaling
  float col_s[MAXA];
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    float sq = 0.f;
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k) sq += J[k][c] * J[k][c];
    col_s[c] = sqrtf(sq) + 1e-8f;
  }
#pragma unroll
  for (int k = 0; k < 6 * MAXEE; ++k)
#pragma unroll
    for (int c = 0; c < MAXA; ++c) J[k][c] = J[k][c] / col_s[c];

  if constexpr (!F64S) {
    lm_solve_f32<MAXA, MAXEE>(sh, J, fw, 6 * n_ee, lam, col_s, delta);
  } else {
  // FP64, through the push-through identity
  //   (Js^T Js + lam I)^-1 Js^T = Js^T (Js Js^T + lam I)^-1,
  // so p = -Js^T y with (Js Js^T + lam I) y = fw: an R x R system (R = 6
  // MAXEE rows) instead of MAXA x MAXA, the same step in exact arithmetic.
  // Fixed and padded joints enter as zero columns of Js, which gives them a
  // zero step and the other joints the step of the reduced system, as the
  // masked MAXA x MAXA system does (lam > 0 keeps both positive definite).
  constexpr int R = 6 * MAXEE;
  double A[R * (R + 1) / 2];
  double y[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      double acc = (i == j) ? (double)lam : 0.0;
#pragma unroll
      for (int c = 0; c < MAXA; ++c)
        if (!sh.fixed[c]) acc = fma((double)J[i][c], (double)J[j][c], acc);
      A[i * (i + 1) / 2 + j] = acc;
    }
    y[i] = (double)fw[i];
  }
  // Cholesky A = L L^T in place; a non-positive pivot zeroes the step
  bool ok = true;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    double s2 = A[k * (k + 1) / 2 + k];
#pragma unroll
    for (int q = 0; q < k; ++q) s2 -= A[k * (k + 1) / 2 + q] * A[k * (k + 1) / 2 + q];
    if (!(s2 > 0.0)) ok = false;
    const double lkk = sqrt(ok ? s2 : 1.0);
    const double inv = 1.0 / lkk;
    A[k * (k + 1) / 2 + k] = inv;
#pragma unroll
    for (int i = k + 1; i < R; ++i) {
      double tt = A[i * (i + 1) / 2 + k];
#pragma unroll
      for (int q = 0; q < k; ++q) tt -= A[i * (i + 1) / 2 + q] * A[k * (k + 1) / 2 + q];
      A[i * (i + 1) / 2 + k] = tt * inv;
    }
  }
  // forward / backward substitution (the diagonal holds reciprocals)
#pragma unroll
  for (int i = 0; i < R; ++i) {
    double s2 = y[i];
#pragma unroll
    for (int q = 0; q < i; ++q) s2 -= A[i * (i + 1) / 2 + q] * y[q];
    y[i] = s2 * A[i * (i + 1) / 2 + i];
  }
#pragma unroll
  for (int i = R - 1; i >= 0; --i) {
    double s2 = y[i];
#pragma unroll
    for (int q = i + 1; q < R; ++q) s2 -= A[q * (q + 1) / 2 + i] * y[q];
    y[i] = s2 * A[i * (i + 1) / 2 + i];
  }
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    double pc = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k) pc = fma((double)J[k][c], y[k], pc);
    delta[c] = (ok && !sh.fixed[c]) ? (float)(-pc) / col_s[c] : 0.f;
  }
  }
  float dn2 = 0.f;
#pragma unroll
  for (int c = 0; c < MAXA; ++c) dn2 += delta[c] * delta[c];
  // trust region
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

  return fw2;
}

// Block prologue shared by both LM kernels: robot description, targets of
// problem blockIdx.y, limits, world, grouped robot spheres and joint bounding
// spheres, grouped self pairs and the obstacle grid, all in shared memory.
// Ends with __syncthreads().
template <int MAXA>
__device__ void lm_stage(const LmArgs& a, unsigned char* smem_raw, const LmLayout& L, int pb) {
  LmShared& sh = *reinterpret_cast<LmShared*>(smem_raw);
  float4* rs4 = reinterpret_cast<float4*>(smem_raw + L.rs);
  float4* ws4 = reinterpret_cast<float4*>(smem_raw + L.ws);
  int2* pairs = reinterpret_cast<int2*>(smem_raw + L.pairs);
  float4* prec = reinterpret_cast<float4*>(smem_raw + L.prec);
  int2* gjoint = reinterpret_cast<int2*>(smem_raw + L.gjoint);
  int* gstart = reinterpret_cast<int*>(smem_raw + L.gstart);
  int* rsj = reinterpret_cast<int*>(smem_raw + L.rsj);
  int* rsk = reinterpret_cast<int*>(smem_raw + L.rsk);
  int* cell_start = reinterpret_cast<int*>(smem_raw + L.cells);
  unsigned short* cell_obs = reinterpret_cast<unsigned short*>(smem_raw + L.cell_obs);
  float* wc = reinterpret_cast<float*>(smem_raw + L.wc);
  float* wb = reinterpret_cast<float*>(smem_raw + L.wb);
  float* wh = reinterpret_cast<float*>(smem_raw + L.wh);
  int* scratch = reinterpret_cast<int*>(smem_raw + L.scratch);  // reused by the kernel after staging

  load_joint_table(sh.jt, a.m);
  const int tid = threadIdx.x;
  if (tid < a.n_ee) {
    const int tj = a.target_jnts[tid];
    sh.tsorted[tid] = (tj >= 0 && tj < a.m.n_joints) ? sh.jt.sorted_of[tj] : 0;
    unsigned long long bits = 0ull;
    for (int j = 0; j < a.m.n_joints; ++j)
      if (a.ancestor_masks[tid * a.m.n_joints + j]) bits |= 1ull << j;
    sh.anc[tid] = bits;
    for (int c = 0; c < 7; ++c) sh.tgt[tid][c] = a.target_Ts[((size_t)pb * a.n_ee + tid) * 7 + c];
  }
  for (int i = tid; i < MAXA; i += blockDim.x) {
    const bool real = i < a.n_act;
    sh.lo[i] = real ? a.lower[i] : 0.f;
    sh.hi[i] = real ? a.upper[i] : 0.f;
    sh.fixed[i] = real ? (a.fixed_mask[i] != 0) : 1;
  }
  // the world by the TMA bulk-copy engine (stage_world: bounded wait,
  // plain-load fallback), then the margin folded into the sphere radii and
  // the padding slots set, in place
  (void)wc; (void)wb; (void)wh;
  stage_world(a.w, reinterpret_cast<float*>(ws4), L.ms_pad);
  __syncthreads();
  for (int i = tid; i < L.ms_pad; i += blockDim.x) {
    if (i < a.w.Ms) ws4[i].w = ws4[i].w + a.margin;
    else ws4[i] = make_float4(1e18f, 1e18f, 1e18f, 0.f);  // padding: never within reach
  }
  __syncthreads();

  // Thread 0 (a few hundred serial steps, once per block): robot spheres
  // grouped by joint in topological order (invalid joint indices dropped, as
  // the reference skips them, _ls_ik_cuda_kernel.cu:171); one bounding sphere
  // per sphere-carrying joint; self pairs remapped to grouped sphere slots
  // and grouped by joint-slot pair; the obstacle-grid bounds.
  if (tid == 0) {
    const int nj = a.m.n_joints;
    int cnt[PK_MAX_JOINTS], slot_of[PK_MAX_JOINTS];
    for (int j = 0; j < nj; ++j) cnt[j] = 0;
    for (int k = 0; k < a.n_rs; ++k) {
      const int j = a.sphere_joint[k];
      if (j >= 0 && j < nj) cnt[sh.jt.sorted_of[j]]++;
    }
    int n_js = 0, total = 0;
    for (int js = 0; js < nj; ++js) {
      slot_of[js] = -1;
      if (cnt[js] == 0) continue;
      slot_of[js] = n_js;
      sh.jlist[n_js] = js;
      sh.jstart[n_js] = total;
      total += cnt[js];
      cnt[js] = sh.jstart[n_js];  // running insert position
      ++n_js;
    }
    sh.jstart[n_js] = total;
    sh.n_js = n_js;
    sh.n_rs = total;
    for (int k = 0; k < a.n_rs; ++k) {
      const int j = a.sphere_joint[k];
      if (j < 0 || j >= nj) { rsk[k] = -1; continue; }
      const int js = sh.jt.sorted_of[j];
      const int at = cnt[js]++;
      rsk[k] = at;
      rs4[at] = make_float4(a.spheres_local[4 * k], a.spheres_local[4 * k + 1], a.spheres_local[4 * k + 2],
                            a.spheres_local[4 * k + 3]);
      rsj[at] = slot_of[js];
    }
    float rmax = 0.f;
    for (int q = 0; q < n_js; ++q) {
      float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
      for (int k = sh.jstart[q]; k < sh.jstart[q + 1]; ++k) {
        const float v[3] = {rs4[k].x, rs4[k].y, rs4[k].z};
        for (int d = 0; d < 3; ++d) { lo[d] = fminf(lo[d], v[d]); hi[d] = fmaxf(hi[d], v[d]); }
      }
      const float cx = 0.5f * (lo[0] + hi[0]), cy = 0.5f * (lo[1] + hi[1]), cz = 0.5f * (lo[2] + hi[2]);
      float R = -3e38f;
      for (int k = sh.jstart[q]; k < sh.jstart[q + 1]; ++k) {
        const float dx = rs4[k].x - cx, dy = rs4[k].y - cy, dz = rs4[k].z - cz;
        R = fmaxf(R, sqrtf(dx * dx + dy * dy + dz * dz) + rs4[k].w);
      }
      // slack keeps the culls conservative under FP32 rounding
      R = R + 1e-4f + 1e-5f * fabsf(R);
      sh.jb[q] = make_float4(cx, cy, cz, R);
      rmax = fmaxf(rmax, R);
    }
    if (L.recs) {
      // the paired sphere table: joint slot q's spheres from pair pjstart[q]
      float* rf = reinterpret_cast<float*>(smem_raw + L.rsp);
      int run = 0;
      for (int q = 0; q < n_js; ++q) {
        sh.pjstart[q] = run;
        const int k0 = sh.jstart[q], n = sh.jstart[q + 1] - k0;
        for (int i = 0; i < n + (n & 1); ++i) {
          const int h = i & 1;
          float* f = rf + 8 * (run + (i >> 1));
          const float4 v = (i < n) ? rs4[k0 + i] : make_float4(0.f, 0.f, 0.f, -1e9f);
          f[h] = v.x; f[2 + h] = v.y; f[4 + h] = v.z; f[6 + h] = v.w;
        }
        run += (n + 1) >> 1;
      }
      sh.pjstart[n_js] = run;
    }
    // self pairs in grouped sphere slots, grouped by (joint slot, joint slot)
    // with a counting sort on the key x_slot * n_js + y_slot; the layout
    // sizes the scratch for n_joints^2 >= n_js^2 keys, so every group holds
    // the pairs of one joint pair (x_slot <= y_slot).  The seed-group layout
    // also gets each pair as a joint-frame record: (c_a, r_a + r_b + margin)
    // in slot x's frame, (c_b, 0) in slot y's frame.
    int n_groups = 0;
    if (a.coll && a.n_self > 0 && n_js > 0) {
      const int NK = n_js * n_js;
      int* kc = scratch;
      for (int i = 0; i < NK; ++i) kc[i] = 0;
      for (int pass = 0; pass < 2; ++pass) {
        for (int q = 0; q < a.n_self; ++q) {
          int x = a.self_i[q], y = a.self_j[q];
          if (x < 0 || y < 0 || x >= a.n_rs || y >= a.n_rs) continue;
          x = rsk[x]; y = rsk[y];
          if (x < 0 || y < 0) continue;
          if (rsj[x] > rsj[y]) { const int tmp = x; x = y; y = tmp; }
          const int key = rsj[x] * n_js + rsj[y];
          if (pass == 0) {
            kc[key]++;
          } else {
            pairs[kc[key]++] = make_int2(x, y);
          }
        }
        if (pass == 0) {
          int run = 0;
          for (int key = 0; key < NK; ++key) {
            if (kc[key] == 0) continue;
            gjoint[n_groups] = make_int2(key / n_js, key % n_js);
            gstart[n_groups] = run;
            const int c0 = kc[key];
            kc[key] = run;
            run += c0;
            ++n_groups;
          }
          gstart[n_groups] = run;
        }
      }
      if (L.recs) {
        // the paired pair table: group g's pairs from padded index pgstart[g]
        int* pgstart = reinterpret_cast<int*>(smem_raw + L.pgstart);
        float* pf = reinterpret_cast<float*>(prec);
        int run = 0;
        for (int g = 0; g < n_groups; ++g) {
          pgstart[g] = run;
          const int n = gstart[g + 1] - gstart[g];
          for (int i = 0; i < n + (n & 1); ++i) {
            const int pq = run + i, h = pq & 1;
            float* f = pf + 16 * (pq >> 1);
            if (i < n) {
              const int2 pr = pairs[gstart[g] + i];
              const float4 A = rs4[pr.x], Bs = rs4[pr.y];
              const float rr = A.w + Bs.w + a.margin;
              f[h] = -A.x; f[2 + h] = -A.y; f[4 + h] = -A.z; f[6 + h] = rr;
              f[8 + h] = Bs.x; f[10 + h] = Bs.y; f[12 + h] = Bs.z; f[14 + h] = rr * fabsf(rr);
            } else {  // padding: |u|^2 >= 0 is never below -1
              f[h] = 0.f; f[2 + h] = 0.f; f[4 + h] = 0.f; f[6 + h] = -1.f;
              f[8 + h] = 0.f; f[10 + h] = 0.f; f[12 + h] = 0.f; f[14 + h] = -1.f;
            }
          }
          run += n + (n & 1);
        }
        pgstart[n_groups] = run;
      }
    }
    sh.n_groups = n_groups;
    // obstacle-grid bounds (world radii already carry the margin)
    sh.grid_on = 0;
    sh.grid_n = a.grid_n;
    if (L.grid && n_js > 0) {
      obstacle_grid_bounds(ws4, a.w.Ms, rmax, a.grid_n, sh.glo, sh.ginv);
      sh.rmax = rmax;
      sh.grid_on = 1;
    }
  }
  __syncthreads();

  if (sh.grid_on) {
    obstacle_grid_build(ws4, a.w.Ms, sh.rmax, sh.grid_n, sh.glo, sh.ginv, scratch, cell_start, cell_obs,
                        L.max_entries, sh.grid_on);
    // a fine grid whose lists overflow the capacity falls back to the default
    // resolution (fewer, longer lists) before going without a grid
    if (!sh.grid_on && sh.grid_n > kObsGridDefault) {
      __syncthreads();
      if (tid == 0) {
        sh.grid_n = kObsGridDefault;
        obstacle_grid_bounds(ws4, a.w.Ms, sh.rmax, sh.grid_n, sh.glo, sh.ginv);
        sh.grid_on = 1;
      }
      __syncthreads();
      obstacle_grid_build(ws4, a.w.Ms, sh.rmax, sh.grid_n, sh.glo, sh.ginv, scratch, cell_start, cell_obs,
                          L.max_entries, sh.grid_on);
    }
  }
}

// `count` seeds of problem pb, with the block's shared memory already
// staged for (a, pb) by lm_stage; seed group g reads and writes flat seed
// index gs_base + g.  Every lane of the warp stays in the iteration loop
// until all of the warp's seeds are done (converged, out of iterations, or
// past `count`, which reads and writes nothing): a done seed's lanes run
// along without changing its state, so the warp's collective steps
// (self_warp) always see all 32 lanes.  No block-wide barrier.
template <int MAXA, int MAXEE, int TPS, bool F64S = false, bool B4 = false>
__device__ __forceinline__ void lm_seed_groups(const LmArgs& a, unsigned char* smem_raw, const LmLayout& L, int pb,
                                               int count, size_t gs_base) {
  LmShared& sh = *reinterpret_cast<LmShared*>(smem_raw);
  float4* rs4 = reinterpret_cast<float4*>(smem_raw + L.rs);
  float4* ws4 = reinterpret_cast<float4*>(smem_raw + L.ws);
  int2* gjoint = reinterpret_cast<int2*>(smem_raw + L.gjoint);
  int* gstart = reinterpret_cast<int*>(smem_raw + L.gstart);
  int* cell_start = reinterpret_cast<int*>(smem_raw + L.cells);
  unsigned short* cell_obs = reinterpret_cast<unsigned short*>(smem_raw + L.cell_obs);
  float* wc = reinterpret_cast<float*>(smem_raw + L.wc);
  float* wb = reinterpret_cast<float*>(smem_raw + L.wb);
  float* wh = reinterpret_cast<float*>(smem_raw + L.wh);
  float* slots = reinterpret_cast<float*>(smem_raw + L.slots);
  float* cen = reinterpret_cast<float*>(smem_raw + L.cen);
  const float4* prec = reinterpret_cast<const float4*>(smem_raw + L.prec);
  const int tid = threadIdx.x;
  const int g = tid / TPS, t = tid - g * TPS;
  const int lane = tid & 31;
  const unsigned gmask = (TPS == 32) ? 0xffffffffu : (((1u << TPS) - 1u) << (lane & ~(TPS - 1)));
  const bool valid = g < count;
  const size_t gs = gs_base + (valid ? g : 0);
  (void)pb;

  const JointTable& jt = sh.jt;
  // one pose-slot set per seed (written by lane 0 of the group, read by all)
  const PoseSlots ps{slots + g, a.spb};
  const bool leader = (t == 0);
  const bool use_coll = a.coll && (sh.n_rs > 0);
  PenaltyCtx pc;
  pc.rs = rs4; pc.jb = sh.jb; pc.jstart = sh.jstart; pc.jlist = sh.jlist;
  pc.rsp = reinterpret_cast<const float4*>(smem_raw + L.rsp); pc.pjstart = sh.pjstart;
  pc.ws = ws4; pc.wc = wc; pc.wb = wb; pc.wh = wh; pc.prec = prec; pc.gjoint = gjoint;
  pc.pgstart = reinterpret_cast<const int*>(smem_raw + L.pgstart);
  pc.cell_start = sh.grid_on ? cell_start : nullptr; pc.cell_obs = cell_obs;
  pc.cen = (TPS > 1 || (a.coll && a.n_self > 0)) ? cen + g : nullptr; pc.cs = a.spb; pc.glo = sh.glo; pc.ginv = sh.ginv; pc.gn = sh.grid_n;
  pc.n_rs = sh.n_rs; pc.n_js = sh.n_js; pc.n_groups = sh.n_groups; pc.Ms_pad = L.ms_pad;
  pc.Mc = a.w.Mc; pc.Mb = a.w.Mb; pc.Mh = a.w.Mh; pc.margin = a.margin;

  float W[6] = {a.pos_w, a.pos_w, a.pos_w, a.ori_w, a.ori_w, a.ori_w};

  float cfg[MAXA], best[MAXA];
#pragma unroll
  for (int i = 0; i < MAXA; ++i) {
    cfg[i] = (valid && i < a.n_act) ? a.seeds[gs * a.n_act + i] : 0.f;
    best[i] = cfg[i];
  }
  float* const slots_w = slots + (g & ~31);  // one lane per seed: the pose slots of the warp's first seed
  unsigned short* const wlist =
      reinterpret_cast<unsigned short*>(smem_raw + L.wscr) + (size_t)(tid >> 5) * kSelfChunk * 32 * 3;
  float* const wres = reinterpret_cast<float*>(wlist + kSelfChunk * 32);

  // TPS == 1: called by every lane (collective); TPS > 1: by the lanes of
  // seeds that need it
  auto penalty = [&](bool need) -> float {
    if (!use_coll) return 0.f;
    if (TPS > 1 && !need) return 0.f;
    const float share = penalty_share<TPS, B4>(pc, ps, t, gmask, need, slots_w, a.spb, wlist, wres);
    return a.coll_w * group_sum<TPS>(share, gmask);
  };
  // Every lane of the group computes the FK (same values); lane 0 stores it.
  // The syncs keep lane 0 from overwriting poses another lane still reads.
  auto run_fk = [&](const float (&q)[MAXA]) {
    __syncwarp(gmask);
    fk_group(jt, [&](int i) { return reg_get<MAXA>(q, i); }, ps, leader, gmask);
    __syncwarp(gmask);
  };
  auto weighted_sq = [&](const float (&r)[6 * MAXEE]) {
    float e = 0.f;
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k) {
      const float rw = r[k] * W[k % 6];
      e += rw * rw;
    }
    return e;
  };

  // Evaluation schedule: ev = -1 the initial point, then per iteration ev = 0
  // (current point: residual, Jacobian, damped step) and ev = 1..5 (the
  // line-search trials).  A single call site each for FK, residual and
  // penalty keeps the kernel small enough for the instruction cache.
  float r[6 * MAXEE], pee[3 * MAXEE];
  float delta[MAXA];
  float lam = a.lam0;
  float pen_cur = 0.f, best_err = 0.f, curr = 0.f;
  float best_a_err = 1e30f, best_a_pen = 0.f;
  int best_a = 0;
  int it = 0, ev = -1;
  bool done = !valid;
#pragma unroll
  for (int c = 0; c < MAXA; ++c) delta[c] = 0.f;
  // ev runs the same schedule on every lane of the warp; `done` only stops
  // a seed's state from changing
  while (!__all_sync(0xffffffffu, done)) {
    float q[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c)
      q[c] = (ev <= 0) ? cfg[c] : fmaxf(sh.lo[c], fminf(sh.hi[c], cfg[c] + line_alpha(ev - 1) * delta[c]));
    run_fk(q);
    ee_residual<MAXEE>(sh, ps, a.n_ee, r, pee);

    if (ev == 0) {
      if (!done) {
        bool all_conv = true;
        float max_p = 0.f, max_o = 0.f;
#pragma unroll
        for (int e = 0; e < MAXEE; ++e) {
          if (e < a.n_ee) {
            const float np = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
            const float no = sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
            if (np >= a.eps_pos || no >= a.eps_ori) all_conv = false;
            max_p = fmaxf(max_p, np);
            max_o = fmaxf(max_o, no);
          }
        }
        if (all_conv) {
          done = true;
        } else {
          curr = lm_direction<MAXA, MAXEE, F64S>(sh, ps, a.n_ee, W, r, pee, lam, max_p, max_o, delta) + pen_cur;
          best_a_err = 1e30f;
          best_a_pen = pen_cur;
          best_a = 0;
        }
      }
      ev = 1;
      continue;
    }

    // The penalty is >= 0, so a trial whose pose error alone is not below
    // the best trial so far cannot win (wsq + pen >= wsq in FP32 too): its
    // penalty is skipped, which leaves every decision and output unchanged.
    // (The test is uniform across the seed's lanes.)
    const float wsq = weighted_sq(r);
    const float pen = penalty(!done && (ev < 0 || wsq < best_a_err));
    if (!done) {
      const float err = wsq + pen;
      if (ev < 0) {
        pen_cur = pen;
        best_err = err;
        if (a.max_iter <= 0) done = true;
      } else {
        if (err < best_a_err) { best_a_err = err; best_a = ev - 1; best_a_pen = pen; }
        if (ev == 5) {
          // accept / reject the damped step, track the all-time best
          const float alpha = line_alpha(best_a);
          float trial[MAXA];
#pragma unroll
          for (int c = 0; c < MAXA; ++c) trial[c] = fmaxf(sh.lo[c], fminf(sh.hi[c], cfg[c] + alpha * delta[c]));
          if (best_a_err < curr * (1.0f - 1e-4f)) {
#pragma unroll
            for (int c = 0; c < MAXA; ++c) cfg[c] = trial[c];
            pen_cur = best_a_pen;
            lam = fmaxf(lam * a.lam_down, 1e-10f);
          } else {
            lam = fminf(lam * a.lam_up, 1e6f);
          }
          if (best_a_err < best_err) {
            best_err = best_a_err;
#pragma unroll
            for (int c = 0; c < MAXA; ++c) best[c] = trial[c];
          }
          if (++it >= a.max_iter) done = true;
        }
      }
    }
    ev = (ev < 0 || ev == 5) ? 0 : ev + 1;
  }

  if (t == 0 && valid) {
#pragma unroll
    for (int c = 0; c < MAXA; ++c)
      if (c < a.n_act) a.out_cfg[gs * a.n_act + c] = best[c];
    a.out_err[gs] = best_err;
  }
}

// MINB: resident blocks per SM the register budget is sized for.  4 caps a
// thread at 128 registers (a few hundred bytes of spills at MAXA = 8); 2
// leaves room for the whole seed state, for launches whose shared memory
// admits only 2 blocks per SM anyway.
template <int MAXA, int MAXEE, int TPS, int MINB, bool F64S = false, bool B4 = false>
__global__ void __launch_bounds__(128, MINB) lm_kernel(LmArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LmLayout L = lm_layout(a, TPS);
  const int pb = blockIdx.y;
  lm_stage<MAXA>(a, smem_raw, L, pb);
  const int s_first = blockIdx.x * a.spb;
  const int count = min(a.spb, a.Sd - s_first);
  lm_seed_groups<MAXA, MAXEE, TPS, F64S, B4>(a, smem_raw, L, pb, count, (size_t)pb * a.Sd + s_first);
}

// Persistent seed-group kernel of pk_ik_batch: blocks take items (class,
// problem, first seed, count) from the list through the counter queue[0]
// until it runs out, skipping items of classes that use the warp body, and
// stage each item's class and problem before running its seeds.
struct SeedGroupBatch {
  LmArgs cls[PK_MAX_CLASSES];
  int body[PK_MAX_CLASSES];
  int n_classes;
  const int4* items;
  int n_items;
  int* queue;
};

// MINB as for lm_kernel.  MAXA / MAXEE select the body: <8, 1> serves the
// classes of body kBodySeedGroup, <16, 2> (one lane per seed) those of
// kBodySeedGroup16; items of other bodies are skipped.
template <int MAXA, int MAXEE, int TPS, int MINB>
__global__ void __launch_bounds__(128, MINB) lm_batch_kernel(const __grid_constant__ SeedGroupBatch B) {
  constexpr int kMyBody = (MAXA <= 8 && MAXEE == 1) ? kBodySeedGroup : kBodySeedGroup16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ LmArgs s_args;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(B.queue, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= B.n_items) break;
    const int4 item = B.items[it];
    if (item.x < 0 || item.x >= B.n_classes) continue;
    int body;
    pick_class(B.body, item.x, body);
    if (body != kMyBody) continue;
    if (threadIdx.x == 0) pick_class(B.cls, item.x, s_args);
    __syncthreads();
    const LmArgs& a = s_args;
    if (item.y < 0 || item.y >= a.P || item.z < 0 || item.w <= 0 || item.z + item.w > a.Sd || item.w > a.spb)
      continue;  // malformed item: nothing is read or written for it
    const LmLayout L = lm_layout(a, TPS);
    lm_stage<MAXA>(a, smem_raw, L, item.y);
    lm_seed_groups<MAXA, MAXEE, TPS>(a, smem_raw, L, item.y, item.w, (size_t)item.y * a.Sd + item.z);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Trial-lane LM kernel: a group of 5 lanes owns one seed; per iteration all 5
// compute the current point's residual, Jacobian and damped step (identical
// values), lane t computes the FK and residual of line-search trial t, then
// the 5 lanes evaluate the collision penalty of each trial together and the
// 5 errors meet by shuffle.  FK, the step computation and the penalty all
// run with one instruction stream per warp of 6 seeds.
// ---------------------------------------------------------------------------

// Cooperative penalty of one configuration by the 5 lanes of a seed group.
// Work items are striped over the lanes (lane t takes items t, t+5, ...):
// sphere transforms into the seed's float4 position buffer (x, y, z, r),
// then per-joint grid queries (bounding-sphere cull, exact tests of the
// joint's spheres against the surviving obstacles), capsule / box /
// halfspace tests and the self pairs (pre-resolved to byte offsets into the
// position buffer and r_a + r_b + margin).  Every lane runs the same loops,
// so a warp (6 seeds) does not diverge on the culling outcome of one seed.
// Returns lane t's partial sum.
struct CoopCtx {
  const float4* rs;      // robot spheres grouped by joint slot (joint frame)
  const float4* jb;      // bounding sphere per joint slot
  const int* jstart;
  const int* jlist;
  const float4* ws;      // world spheres (x, y, z, r + margin)
  const float* wc;
  const float* wb;
  const float* wh;
  const int4* pair4;     // self pairs: (byte offset a, byte offset b, rr bits, 0)
  int n_pairs;
  const int* cell_start; // null: scan every obstacle
  const unsigned short* cell_obs;
  float4* pos;           // this seed's sphere world positions and radii [n_rs]
  float3 glo, ginv;
  int gn;
  int n_rs, n_js, Ms, Mc, Mb, Mh;
  float margin;
};

__device__ float coop_penalty(const CoopCtx& c, const PoseSlots& psk, int t, unsigned gmask) {
  constexpr int GL = 5;
  float part = 0.f;
  float4* const px = c.pos;
  for (int j = 0; j < c.n_js; ++j) {
    const int k0 = c.jstart[j], k1 = c.jstart[j + 1];
    int k = k0 + ((t - k0) % GL + GL) % GL;  // first grouped sphere of this joint with k % 5 == t
    if (k >= k1) continue;
    const Pose T = psk.load(c.jlist[j]);
    for (; k < k1; k += GL) {
      const float4 s = c.rs[k];
      const float3 w = pose_apply(T, make_float3(s.x, s.y, s.z));
      px[k] = make_float4(w.x, w.y, w.z, s.w);
    }
  }
  __syncwarp(gmask);

  for (int j = t; j < c.n_js && c.Ms > 0; j += GL) {
    const float4 bl = c.jb[j];
    const float3 B = pose_apply(psk.load(c.jlist[j]), make_float3(bl.x, bl.y, bl.z));
    int e0 = 0, e1 = c.Ms;
    const unsigned short* list = nullptr;
    if (c.cell_start) {
      const int cell = obstacle_grid_cell(c.glo, c.ginv, c.gn, B);
      if (cell < 0) continue;
      e0 = c.cell_start[cell];
      e1 = c.cell_start[cell + 1];
      list = c.cell_obs;
    }
    const int k0 = c.jstart[j], k1 = c.jstart[j + 1];
    for (int e = e0; e < e1; ++e) {
      const float4 O = c.ws[list ? (int)list[e] : e];
      const float rr = bl.w + O.w;
      const float dx = B.x - O.x, dy = B.y - O.y, dz = B.z - O.z;
      if (dx * dx + dy * dy + dz * dz < rr * fabsf(rr)) {
        for (int k = k0; k < k1; ++k) {
          const float4 P = px[k];
          const float ex = P.x - O.x, ey = P.y - O.y, ez = P.z - O.z;
          hinge_sq(ex * ex + ey * ey + ez * ez, P.w + O.w, part);
        }
      }
    }
  }

  if (c.Mc + c.Mb + c.Mh > 0) {
    for (int k = t; k < c.n_rs; k += GL) {
      const float4 P = px[k];
      const float3 p = make_float3(P.x, P.y, P.z);
      for (int m = 0; m < c.Mc; ++m) {
        const float d = d_sphere_capsule(p, P.w, c.wc + 7 * m);
        if (d < c.margin) { const float e = d - c.margin; part += e * e; }
      }
      for (int m = 0; m < c.Mb; ++m) {
        const float d = d_sphere_box(p, P.w, c.wb + 15 * m);
        if (d < c.margin) { const float e = d - c.margin; part += e * e; }
      }
      for (int m = 0; m < c.Mh; ++m) {
        const float d = d_sphere_halfspace(p, P.w, c.wh + 6 * m);
        if (d < c.margin) { const float e = d - c.margin; part += e * e; }
      }
    }
  }

  const char* const pbytes = reinterpret_cast<const char*>(px);
#pragma unroll 4
  for (int q = t; q < c.n_pairs; q += GL) {
    const int4 pr = c.pair4[q];
    const float4 A = *reinterpret_cast<const float4*>(pbytes + pr.x);
    const float4 Bq = *reinterpret_cast<const float4*>(pbytes + pr.y);
    const float dx = A.x - Bq.x, dy = A.y - Bq.y, dz = A.z - Bq.z;
    hinge_sq(dx * dx + dy * dy + dz * dz, __int_as_float(pr.z), part);
  }
  __syncwarp(gmask);
  return part;
}

// Sum of the group's 5 partial sums in lane order (the same value, bit for
// bit, on every lane of the group).
__device__ __forceinline__ float group5_sum(float v, unsigned gmask, int base) {
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 5; ++k) s += __shfl_sync(gmask, v, base + k);
  return s;
}

template <int MAXA, int MAXEE>
__global__ void __launch_bounds__(128, 4) lm_trial_kernel(LmArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LmLayout L = lm_layout(a, 1, blockDim.x);
  lm_stage<MAXA>(a, smem_raw, L, blockIdx.y);
  LmShared& sh = *reinterpret_cast<LmShared*>(smem_raw);
  const int tid = threadIdx.x;
  const int pb = blockIdx.y;
  {
    // self pairs as byte offsets into a seed's float4 position buffer plus
    // r_a + r_b + margin, so a pair test is three shared loads and a compare
    const int2* pairs = reinterpret_cast<const int2*>(smem_raw + L.pairs);
    const float4* rs4 = reinterpret_cast<const float4*>(smem_raw + L.rs);
    int4* pair4 = reinterpret_cast<int4*>(smem_raw + L.pair4);
    const int np = sh.n_groups > 0 ? reinterpret_cast<const int*>(smem_raw + L.gstart)[sh.n_groups] : 0;
    for (int q = tid; q < np; q += blockDim.x) {
      const int2 pr = pairs[q];
      pair4[q] = make_int4(16 * pr.x, 16 * pr.y, __float_as_int(rs4[pr.x].w + rs4[pr.y].w + a.margin), 0);
    }
    __syncthreads();
  }
  const int lane = tid & 31, wid = tid >> 5;
  const int gw = lane / 5, t = lane - 5 * gw;
  if (gw >= 6) return;  // lanes 30, 31
  const int s = blockIdx.x * a.spb + wid * 6 + gw;
  if (s >= a.Sd) return;
  const size_t gs = (size_t)pb * a.Sd + s;
  const unsigned gmask = 0x1Fu << (5 * gw);
  const int base = 5 * gw;

  CoopCtx cc;
  cc.rs = reinterpret_cast<const float4*>(smem_raw + L.rs);
  cc.jb = sh.jb; cc.jstart = sh.jstart; cc.jlist = sh.jlist;
  cc.ws = reinterpret_cast<const float4*>(smem_raw + L.ws);
  cc.wc = reinterpret_cast<const float*>(smem_raw + L.wc);
  cc.wb = reinterpret_cast<const float*>(smem_raw + L.wb);
  cc.wh = reinterpret_cast<const float*>(smem_raw + L.wh);
  cc.pair4 = reinterpret_cast<const int4*>(smem_raw + L.pair4);
  cc.n_pairs = sh.n_groups > 0 ? reinterpret_cast<const int*>(smem_raw + L.gstart)[sh.n_groups] : 0;
  cc.cell_start = sh.grid_on ? reinterpret_cast<const int*>(smem_raw + L.cells) : nullptr;
  cc.cell_obs = reinterpret_cast<const unsigned short*>(smem_raw + L.cell_obs);
  cc.pos = reinterpret_cast<float4*>(smem_raw + L.pos) + (size_t)(wid * 6 + gw) * lm_pos4_stride(a.n_rs);
  cc.glo = sh.glo; cc.ginv = sh.ginv; cc.gn = sh.grid_n;
  cc.n_rs = sh.n_rs; cc.n_js = sh.n_js; cc.Ms = a.w.Ms;
  cc.Mc = a.w.Mc; cc.Mb = a.w.Mb; cc.Mh = a.w.Mh; cc.margin = a.margin;
  const bool use_coll = a.coll && (sh.n_rs > 0);

  const JointTable& jt = sh.jt;
  const PoseSlots ps{reinterpret_cast<float*>(smem_raw + L.slots) + tid, (int)blockDim.x};
  float W[6] = {a.pos_w, a.pos_w, a.pos_w, a.ori_w, a.ori_w, a.ori_w};
  float cfg[MAXA], best[MAXA], delta[MAXA];
#pragma unroll
  for (int i = 0; i < MAXA; ++i) {
    cfg[i] = (i < a.n_act) ? a.seeds[gs * a.n_act + i] : 0.f;
    best[i] = cfg[i];
    delta[i] = 0.f;
  }
  auto run_fk = [&](const float (&q)[MAXA]) { fk_thread(jt, [&](int i) { return reg_get<MAXA>(q, i); }, ps); };
  auto weighted_sq = [&](const float (&r)[6 * MAXEE]) {
    float e = 0.f;
#pragma unroll
    for (int k = 0; k < 6 * MAXEE; ++k) {
      const float rw = r[k] * W[k % 6];
      e += rw * rw;
    }
    return e;
  };

  float r[6 * MAXEE], pee[3 * MAXEE];
  // ev = -1: the initial point; ev = 0: current point (step); ev = 1: this lane's trial
  float lam = a.lam0, pen_cur = 0.f, best_err = 0.f, curr = 0.f;
  int it = 0, ev = -1;
  while (true) {
    float q[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c)
      q[c] = (ev <= 0) ? cfg[c] : fmaxf(sh.lo[c], fminf(sh.hi[c], cfg[c] + line_alpha(t) * delta[c]));
    run_fk(q);
    ee_residual<MAXEE>(sh, ps, a.n_ee, r, pee);
    if (ev == 0) {
      bool all_conv = true;
      float max_p = 0.f, max_o = 0.f;
#pragma unroll
      for (int e = 0; e < MAXEE; ++e) {
        if (e < a.n_ee) {
          const float np = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
          const float no = sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
          if (np >= a.eps_pos || no >= a.eps_ori) all_conv = false;
          max_p = fmaxf(max_p, np);
          max_o = fmaxf(max_o, no);
        }
      }
      if (all_conv) break;
      curr = lm_direction<MAXA, MAXEE>(sh, ps, a.n_ee, W, r, pee, lam, max_p, max_o, delta) + pen_cur;
      ev = 1;
      continue;
    }
    // penalty of every trial (lane k's poses), the 5 lanes together
    __syncwarp(gmask);
    float pen = 0.f;
    if (use_coll) {
      float* const slot_base = reinterpret_cast<float*>(smem_raw + L.slots) + (tid - t);
      for (int k = 0; k < (ev < 0 ? 1 : 5); ++k) {
        const PoseSlots psk{slot_base + k, (int)blockDim.x};
        const float pk = a.coll_w * group5_sum(coop_penalty(cc, psk, t, gmask), gmask, base);
        if (k == t || ev < 0) pen = pk;
      }
    }
    const float err = weighted_sq(r) + pen;
    if (ev < 0) {
      pen_cur = pen;
      best_err = err;
      if (a.max_iter <= 0) break;
      ev = 0;
      continue;
    }
    // the 5 trial errors meet; the first minimum wins (_ls_ik_cuda_kernel.cu:361-366)
    float best_a_err = 1e30f, best_a_pen = pen_cur;
    int best_a = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const float ek = __shfl_sync(gmask, err, base + k);
      const float pk = __shfl_sync(gmask, pen, base + k);
      if (ek < best_a_err) { best_a_err = ek; best_a = k; best_a_pen = pk; }
    }
    const float alpha = line_alpha(best_a);
    float trial[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) trial[c] = fmaxf(sh.lo[c], fminf(sh.hi[c], cfg[c] + alpha * delta[c]));
    if (best_a_err < curr * (1.0f - 1e-4f)) {
#pragma unroll
      for (int c = 0; c < MAXA; ++c) cfg[c] = trial[c];
      pen_cur = best_a_pen;
      lam = fmaxf(lam * a.lam_down, 1e-10f);
    } else {
      lam = fminf(lam * a.lam_up, 1e6f);
    }
    if (best_a_err < best_err) {
      best_err = best_a_err;
#pragma unroll
      for (int c = 0; c < MAXA; ++c) best[c] = trial[c];
    }
    if (++it >= a.max_iter) break;
    ev = 0;
  }
  if (t == 0) {
#pragma unroll
    for (int c = 0; c < MAXA; ++c)
      if (c < a.n_act) a.out_cfg[gs * a.n_act + c] = best[c];
    a.out_err[gs] = best_err;
  }
}

// ---------------------------------------------------------------------------
// FP64 re-verification + winner selection, one block per problem
// ---------------------------------------------------------------------------

struct PoseD {
  double w, x, y, z, tx, ty, tz;
};

__device__ __forceinline__ void qrot_d(double w, double x, double y, double z, double vx, double vy,
                                       double vz, double& ox, double& oy, double& oz) {
  const double tx = 2.0 * (y * vz - z * vy), ty = 2.0 * (z * vx - x * vz), tz = 2.0 * (x * vy - y * vx);
  ox = vx + w * tx + (y * tz - z * ty);
  oy = vy + w * ty + (z * tx - x * tz);
  oz = vz + w * tz + (x * ty - y * tx);
}

__device__ __forceinline__ PoseD compose_d(const PoseD& a, const PoseD& b) {
  PoseD o;
  o.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  o.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  o.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
  o.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
  double rx, ry, rz;
  qrot_d(a.w, a.x, a.y, a.z, b.tx, b.ty, b.tz, rx, ry, rz);
  o.tx = rx + a.tx; o.ty = ry + a.ty; o.tz = rz + a.tz;
  return o;
}

// exp(twist * q) in FP64 (full SE(3) exponential; series below 1e-8 rad^2).
__device__ PoseD motion_d(const float* tw, double q) {
  const double vx = tw[0] * q, vy = tw[1] * q, vz = tw[2] * q;
  const double ox = tw[3] * q, oy = tw[4] * q, oz = tw[5] * q;
  const double t2 = ox * ox + oy * oy + oz * oz;
  double sh_t, ch, B, C;
  if (t2 < 1e-8) {
    sh_t = 0.5 - t2 / 48.0;
    ch = 1.0 - t2 / 8.0;
    B = 0.5 - t2 / 24.0;
    C = 1.0 / 6.0 - t2 / 120.0;
  } else {
    const double th = sqrt(t2);
    double sh, st, ct;
    sincos(0.5 * th, &sh, &ch);
    sincos(th, &st, &ct);
    sh_t = sh / th;
    B = (1.0 - ct) / t2;
    C = (th - st) / (t2 * th);
  }
  PoseD d;
  d.w = ch; d.x = sh_t * ox; d.y = sh_t * oy; d.z = sh_t * oz;
  const double cx = oy * vz - oz * vy, cy = oz * vx - ox * vz, cz = ox * vy - oy * vx;
  const double ccx = oy * cz - oz * cy, ccy = oz * cx - ox * cz, ccz = ox * cy - oy * cx;
  d.tx = vx + B * cx + C * ccx;
  d.ty = vy + B * cy + C * ccy;
  d.tz = vz + B * cz + C * ccz;
  return d;
}

struct VerifyArgs {
  ModelArgs m;
  const float* cfgs;
  const float* errs;
  const float* prev;
  float cw;
  const int* target_jnts;
  const float* target_Ts;
  float pos_tol, rot_tol;
  float* winner_cfg;
  double* pos_err;
  double* rot_err;
  int* success;
  int P, Sd, n_act, n_ee;
};

__global__ void __launch_bounds__(128) verify_select_kernel(VerifyArgs a) {
  __shared__ JointTable jt;
  __shared__ double Tw[PK_MAX_JOINTS][7];
  __shared__ float sbest[32];
  __shared__ int sidx[32];
  __shared__ int winner;
  load_joint_table(jt, a.m);
  const int p = blockIdx.x;
  float bv = FLT_MAX;
  int bi = 0x7fffffff;
  for (int s = threadIdx.x; s < a.Sd; s += blockDim.x) {
    const size_t gs = (size_t)p * a.Sd + s;
    float v = a.errs[gs];
    if (a.prev && a.cw != 0.f) {
      float d2 = 0.f;
      for (int c = 0; c < a.n_act; ++c) {
        const float d = a.cfgs[gs * a.n_act + c] - a.prev[(size_t)p * a.n_act + c];
        d2 += d * d;
      }
      v += a.cw * d2;
    }
    if (v < bv || (v == bv && s < bi) || (bi == 0x7fffffff && !(v == v))) { bv = v; bi = s; }
  }
  // block argmin, ties -> smallest seed index
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov < bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { sbest[wid] = bv; sidx[wid] = bi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float v = sbest[0];
    int i = sidx[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (sbest[w] < v || (sbest[w] == v && sidx[w] < i)) { v = sbest[w]; i = sidx[w]; }
    winner = (i == 0x7fffffff) ? 0 : i;
  }
  __syncthreads();
  const size_t gw = (size_t)p * a.Sd + winner;
  for (int c = threadIdx.x; c < a.n_act; c += blockDim.x)
    a.winner_cfg[(size_t)p * a.n_act + c] = a.cfgs[gw * a.n_act + c];
  if (threadIdx.x != 0) return;
  // FP64 FK of the winner
  const float* q = a.cfgs + gw * a.n_act;
  for (int i = 0; i < jt.n; ++i) {
    const int src = jt.src[i];
    const double qv = ((src < 0) ? 0.0 : (double)q[src]) * (double)jt.mul[i] + (double)jt.off[i];
    PoseD Tpc{jt.ptf[i][0], jt.ptf[i][1], jt.ptf[i][2], jt.ptf[i][3], jt.ptf[i][4], jt.ptf[i][5], jt.ptf[i][6]};
    if (jt.kind[i] != kFixed) Tpc = compose_d(Tpc, motion_d(jt.tw[i], qv));
    const int ps = jt.psorted[i];
    PoseD T = Tpc;
    if (ps >= 0) {
      const PoseD Pp{Tw[ps][0], Tw[ps][1], Tw[ps][2], Tw[ps][3], Tw[ps][4], Tw[ps][5], Tw[ps][6]};
      T = compose_d(Pp, Tpc);
    }
    Tw[i][0] = T.w; Tw[i][1] = T.x; Tw[i][2] = T.y; Tw[i][3] = T.z;
    Tw[i][4] = T.tx; Tw[i][5] = T.ty; Tw[i][6] = T.tz;
  }
  double pe = 0.0, re = 0.0;
  for (int e = 0; e < a.n_ee; ++e) {
    const int tj = a.target_jnts[e];
    const int i = (tj >= 0 && tj < jt.n) ? jt.sorted_of[tj] : 0;
    const float* g = a.target_Ts + ((size_t)p * a.n_ee + e) * 7;
    const double dx = Tw[i][4] - g[4], dy = Tw[i][5] - g[5], dz = Tw[i][6] - g[6];
    pe = fmax(pe, sqrt(dx * dx + dy * dy + dz * dz));
    // conj(q_tgt) * q
    const double aw = g[0], ax = -g[1], ay = -g[2], az = -g[3];
    const double bw = Tw[i][0], bx = Tw[i][1], by = Tw[i][2], bz = Tw[i][3];
    const double rw = aw * bw - ax * bx - ay * by - az * bz;
    const double rx = aw * bx + ax * bw + ay * bz - az * by;
    const double ry = aw * by - ax * bz + ay * bw + az * bx;
    const double rz = aw * bz + ax * by - ay * bx + az * bw;
    const double nv = sqrt(rx * rx + ry * ry + rz * rz);
    re = fmax(re, 2.0 * atan2(nv, fabs(rw)));
  }
  if (a.pos_err) a.pos_err[p] = pe;
  if (a.rot_err) a.rot_err[p] = re;
  if (a.success) a.success[p] = (pe < (double)a.pos_tol && re < (double)a.rot_tol) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static size_t lm_smem_bytes(const LmArgs& a, int tps) { return lm_layout(a, tps).total; }

// Blocks per SM that shared memory admits (at most the 4 of the small
// register budget).
static int lm_blocks_per_sm(size_t smem) { return (int)std::min<size_t>(4, (228 * 1024) / (smem + 1024)); }

// The fine default grid (lm_grid_option) only where its larger cell lists
// keep the blocks per SM that the default resolution admits; else the
// default resolution.  `threads` as for lm_layout.
static void lm_fit_grid(LmArgs& a, int tps, int threads = 0) {
  if (!a.grid_auto || a.grid_n <= kObsGridDefault) return;
  LmArgs b = a;
  b.grid_n = kObsGridDefault;
  if (lm_blocks_per_sm(lm_layout(a, tps, threads).total) < lm_blocks_per_sm(lm_layout(b, tps, threads).total))
    a.grid_n = kObsGridDefault;
}

template <int MAXA, int MAXEE, int TPS, bool F64S = false>
static int launch_lm_t(const LmArgs& a0, cudaStream_t st) {
  LmArgs a = a0;
  lm_fit_grid(a, TPS);
  const int threads = a.spb * TPS;
  const size_t smem = lm_smem_bytes(a, TPS);
  PK_CHECK_CAP(smem <= 220 * 1024, "LM working set (%zu B of shared memory) too large", smem);
  dim3 grid((a.Sd + a.spb - 1) / a.spb, a.P);
  // The 4-block register budget (spills) only where shared memory admits 3
  // or more blocks per SM and the grid needs more than 2 blocks per SM.
  auto kern = lm_kernel<MAXA, MAXEE, TPS, 2, F64S>;
  if constexpr (MAXA <= 8) {
    int dev = 0, sms = 0;
    if (int s = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return s;
    if (int s = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute")) return s;
    const bool four = (228 * 1024) / (smem + 1024) >= 3 && (long long)grid.x * grid.y > 2LL * sms;
    if (four) kern = lm_kernel<MAXA, MAXEE, TPS, 4, F64S>;
    // one lane per seed on the finest default grid (short lists): the
    // four-per-step candidate loads
    if constexpr (TPS == 1 && !F64S) {
      if (a.coll && a.grid_n >= kObsGridFine)
        kern = four ? lm_kernel<MAXA, MAXEE, 1, 4, false, true> : lm_kernel<MAXA, MAXEE, 1, 2, false, true>;
    }
  }
  if (int s = set_smem_limit((const void*)kern, smem)) return s;
  kern<<<grid, threads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "lm_kernel launch");
}

template <int MAXA, int MAXEE>
static int launch_lm_tps(const LmArgs& a, int tps, cudaStream_t st) {
  if (a.f64_solve) return launch_lm_t<MAXA, MAXEE, 1, true>(a, st);
  switch (tps) {
    case 1: return launch_lm_t<MAXA, MAXEE, 1>(a, st);
    case 2: return launch_lm_t<MAXA, MAXEE, 2>(a, st);
    case 4: return launch_lm_t<MAXA, MAXEE, 4>(a, st);
    default: return launch_lm_t<MAXA, MAXEE, 8>(a, st);
  }
}

template <int MAXA, int MAXEE>
static int launch_lm_trial(LmArgs a, cudaStream_t st) {
  const int threads = 128;
  a.spb = 6 * (threads / 32);  // 6 groups of 5 lanes per warp
  lm_fit_grid(a, 1, threads);
  const size_t smem = lm_layout(a, 1, threads).total;
  PK_CHECK_CAP(smem <= 220 * 1024, "LM working set (%zu B of shared memory) too large", smem);
  auto kern = lm_trial_kernel<MAXA, MAXEE>;
  if (int s = set_smem_limit((const void*)kern, smem)) return s;
  dim3 grid((a.Sd + a.spb - 1) / a.spb, a.P);
  kern<<<grid, threads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "lm_trial_kernel launch");
}

static pk_ik_class class_of(const LmArgs& a) {
  pk_ik_class c{};
  c.twists = a.m.twists; c.parent_tf = a.m.parent_tf; c.parent_idx = a.m.parent_idx; c.act_idx = a.m.act_idx;
  c.mimic_mul = a.m.mimic_mul; c.mimic_off = a.m.mimic_off; c.mimic_act_idx = a.m.mimic_act_idx;
  c.topo_inv = a.m.topo_inv; c.n_joints = a.m.n_joints; c.n_act = a.n_act;
  c.target_jnts = a.target_jnts; c.ancestor_masks = a.ancestor_masks; c.target_Ts = a.target_Ts; c.n_ee = a.n_ee;
  c.robot_spheres_local = a.spheres_local; c.robot_sphere_joint_idx = a.sphere_joint; c.n_robot_spheres = a.n_rs;
  c.self_i = a.self_i; c.self_j = a.self_j; c.n_self = a.n_self;
  c.lower = a.lower; c.upper = a.upper; c.fixed_mask = a.fixed_mask;
  c.seeds = a.seeds; c.out_cfg = a.out_cfg; c.out_err = a.out_err;
  c.n_problems = a.P; c.seed_stride = a.Sd; c.body = kBodyWarp;
  return c;
}

static int launch_lm(LmArgs a, int tps, int spb, cudaStream_t st) {
  // threads_per_seed 5: the trial-lane kernel (5 lanes per seed, one
  // line-search trial each); 1, 2, 4, 8: the seed-group kernel with the
  // collision penalty split across that many lanes; 0: the fastest measured
  // default, 1 lane x 128 seeds per block.  (16 and 32, the warp-per-seed
  // body, are routed by lm_common.)
  if (tps <= 0) {
    tps = 1;
    if (spb <= 0) spb = (a.n_act <= 8 && a.n_ee <= 1) ? 128 : kSeedsPerBlock16;
  }
  if (tps == 5) {
    PK_CHECK_ARG(!a.f64_solve, "fp64_solve runs with threads_per_seed 0 or 1");
    if (a.n_act <= 8 && a.n_ee <= 1) return launch_lm_trial<8, 1>(a, st);
    if (a.n_act <= 16 && a.n_ee <= 2) return launch_lm_trial<16, 2>(a, st);
    set_error("the LM kernel supports n_act <= 16 with n_ee <= 2 (got n_act=%d, n_ee=%d)", a.n_act, a.n_ee);
    return PK_ERR_CAPACITY;
  }
  PK_CHECK_ARG(tps == 1 || tps == 2 || tps == 4 || tps == 8, "threads_per_seed must be 0, 1, 2, 4, 5, 8, 16 or 32");
  PK_CHECK_ARG(!a.f64_solve || tps == 1, "fp64_solve runs with threads_per_seed 0 or 1");
  if (spb <= 0) spb = 128 / tps;
  PK_CHECK_ARG(spb * tps <= 128 && (spb * tps) % 32 == 0,
               "seeds_per_block * threads_per_seed must be a multiple of 32 and at most 128");
  a.spb = spb;
  if (a.n_act <= 8 && a.n_ee <= 1) return launch_lm_tps<8, 1>(a, tps, st);
  if (a.n_act <= 16 && a.n_ee <= 2) return launch_lm_tps<16, 2>(a, tps, st);
  set_error("the LM kernel supports n_act <= 16 with n_ee <= 2 (got n_act=%d, n_ee=%d)", a.n_act, a.n_ee);
  return PK_ERR_CAPACITY;
}

static int validate_lm(const LmArgs& a) {
  PK_CHECK_ARG(a.P >= 0 && a.Sd >= 0 && a.n_act >= 0 && a.n_ee >= 0 && a.n_rs >= 0 && a.n_self >= 0,
               "negative extent");
  PK_CHECK_CAP(a.m.n_joints <= PK_MAX_JOINTS, "n_joints=%d exceeds %d", a.m.n_joints, PK_MAX_JOINTS);
  PK_CHECK_CAP(a.n_act <= PK_MAX_ACT, "n_act=%d exceeds %d (the reference kernel silently overflows "
               "its per-thread arrays here)", a.n_act, PK_MAX_ACT);
  PK_CHECK_CAP(a.n_ee <= PK_MAX_EE, "n_ee=%d exceeds %d", a.n_ee, PK_MAX_EE);
  PK_CHECK_ARG(a.n_ee >= 1, "at least one end-effector target is required");
  PK_CHECK_ARG(a.max_iter >= 0 && a.max_iter <= 1000000, "max_iter out of range");
  return PK_OK;
}

}  // namespace pk

using namespace pk;

static int lm_common(void* stream, const pk_lm_options& o, const float* seeds, const float* twists,
                     const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                     const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                     const int32_t* topo_inv, const int32_t* target_jnts,
                     const int32_t* ancestor_masks, const float* target_Ts,
                     const float* robot_spheres_local, const int32_t* robot_sphere_joint_idx,
                     const float* ws, const float* wc, const float* wb, const float* wh,
                     const int32_t* self_i, const int32_t* self_j, const float* lower,
                     const float* upper, const int32_t* fixed_mask, float* out_cfg,
                     float* out_err, int32_t P, int32_t Sd, int32_t n_act, int32_t n_joints,
                     int32_t n_ee, int32_t n_rs, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh,
                     int32_t n_self) {
  LmArgs a{};
  a.m = ModelArgs{twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
                  topo_inv, n_joints, n_act};
  a.w = WorldArgs{ws, wc, wb, wh, Ms, Mc, Mb, Mh};
  a.seeds = seeds; a.target_jnts = target_jnts; a.ancestor_masks = ancestor_masks;
  a.target_Ts = target_Ts; a.spheres_local = robot_spheres_local;
  a.sphere_joint = robot_sphere_joint_idx; a.self_i = self_i; a.self_j = self_j;
  a.lower = lower; a.upper = upper; a.fixed_mask = fixed_mask;
  a.out_cfg = out_cfg; a.out_err = out_err;
  a.P = P; a.Sd = Sd; a.n_act = n_act; a.n_ee = n_ee; a.n_rs = n_rs; a.n_self = n_self;
  a.max_iter = o.max_iter; a.pos_w = o.pos_weight; a.ori_w = o.ori_weight;
  a.lam0 = o.lambda_init; a.lam_down = o.lambda_down; a.lam_up = o.lambda_up;
  a.eps_pos = o.eps_pos; a.eps_ori = o.eps_ori;
  a.coll = o.enable_collision ? 1 : 0; a.coll_w = o.collision_weight; a.margin = o.collision_margin;
  a.f64_solve = o.fp64_solve ? 1 : 0;
  PK_CHECK_ARG(o.obstacle_grid >= -1 && o.obstacle_grid <= kObsGridMax,
               "obstacle_grid must be -1 (none), 0 (default) or 1..%d cells per axis", kObsGridMax);
  a.grid_n = lm_grid_option(o.obstacle_grid, Ms);
  a.grid_auto = o.obstacle_grid == 0;
  if (int s = validate_lm(a)) return s;
  if (P == 0 || Sd == 0) return PK_OK;
  PK_CHECK_ARG(seeds && twists && parent_tf && parent_idx && act_idx && mimic_mul && mimic_off &&
                   mimic_act_idx && topo_inv && target_jnts && ancestor_masks && target_Ts &&
                   lower && upper && fixed_mask && out_cfg && out_err,
               "null buffer");
  PK_CHECK_ARG(n_rs == 0 || (robot_spheres_local && robot_sphere_joint_idx), "null robot spheres");
  PK_CHECK_ARG((Ms == 0 || ws) && (Mc == 0 || wc) && (Mb == 0 || wb) && (Mh == 0 || wh),
               "null world buffer");
  PK_CHECK_ARG(n_self == 0 || (self_i && self_j), "null self pairs");
  if (!a.coll) { a.n_self = 0; }
  // threads_per_seed 16 or 32: the warp-per-seed body (pk_lm_wide.cu) with
  // that many lanes per seed; robots beyond the seed-group kernel's buckets
  // (n_act > 16 or n_ee > 2) take it too
  if (o.threads_per_seed == 16 || o.threads_per_seed == 32 || a.n_act > 16 || a.n_ee > 2) {
    PK_CHECK_ARG(!a.f64_solve, "fp64_solve runs in the seed-group kernel (n_act <= 16, n_ee <= 2, "
                 "threads_per_seed 0 or 1)");
    pk_lm_options ow = o;
    if (o.threads_per_seed == 16 || o.threads_per_seed == 32) ow.lanes_per_wide_seed = o.threads_per_seed;
    return launch_warp_grid(class_of(a), a.w, ow, (cudaStream_t)stream);
  }
  return launch_lm(a, o.threads_per_seed, o.seeds_per_block, (cudaStream_t)stream);
}

extern "C" int pk_ls_ik_cuda(void* stream, const float* seeds, const float* twists,
                             const float* parent_tf, const int32_t* parent_idx,
                             const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                             const int32_t* mimic_act_idx, const int32_t* topo_inv,
                             const int32_t* target_jnts, const int32_t* ancestor_masks,
                             const float* target_Ts, const float* robot_spheres_local,
                             const int32_t* robot_sphere_joint_idx, const float* world_spheres,
                             const float* world_capsules, const float* world_boxes,
                             const float* world_halfspaces, const float* lower, const float* upper,
                             const int32_t* fixed_mask, int64_t max_iter, float pos_weight,
                             float ori_weight, float lambda_init, float eps_pos, float eps_ori,
                             int64_t enable_collision, float collision_weight,
                             float collision_margin, float* out_cfg, float* out_err,
                             int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints,
                             int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc,
                             int32_t Mb, int32_t Mh) {
  PK_CHECK_ARG(max_iter >= 0 && max_iter <= 1000000, "max_iter out of range");
  pk_lm_options o{};
  o.max_iter = (int32_t)max_iter;
  o.pos_weight = pos_weight;
  o.ori_weight = ori_weight;
  o.lambda_init = lambda_init;
  o.lambda_down = 0.5f;
  o.lambda_up = 3.0f;
  o.eps_pos = eps_pos;
  o.eps_ori = eps_ori;
  o.enable_collision = enable_collision ? 1 : 0;
  o.collision_weight = collision_weight;
  o.collision_margin = collision_margin;
  return lm_common(stream, o, seeds, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off,
                   mimic_act_idx, topo_inv, target_jnts, ancestor_masks, target_Ts,
                   robot_spheres_local, robot_sphere_joint_idx, world_spheres, world_capsules,
                   world_boxes, world_halfspaces, nullptr, nullptr, lower, upper, fixed_mask,
                   out_cfg, out_err, n_problems, n_seeds, n_act, n_joints, n_ee, n_robot_spheres,
                   Ms, Mc, Mb, Mh, 0);
}

extern "C" int pk_ls_ik_ex(void* stream, const pk_lm_options* opt, const float* seeds,
                           const float* twists, const float* parent_tf, const int32_t* parent_idx,
                           const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                           const int32_t* mimic_act_idx, const int32_t* topo_inv,
                           const int32_t* target_jnts, const int32_t* ancestor_masks,
                           const float* target_Ts, const float* robot_spheres_local,
                           const int32_t* robot_sphere_joint_idx, const float* world_spheres,
                           const float* world_capsules, const float* world_boxes,
                           const float* world_halfspaces, const int32_t* self_i,
                           const int32_t* self_j, const float* lower, const float* upper,
                           const int32_t* fixed_mask, float* out_cfg, float* out_err,
                           int32_t n_problems, int32_t n_seeds, int32_t n_act, int32_t n_joints,
                           int32_t n_ee, int32_t n_robot_spheres, int32_t Ms, int32_t Mc,
                           int32_t Mb, int32_t Mh, int32_t n_self_pairs) {
  PK_CHECK_ARG(opt != nullptr, "null options");
  return lm_common(stream, *opt, seeds, twists, parent_tf, parent_idx, act_idx, mimic_mul,
                   mimic_off, mimic_act_idx, topo_inv, target_jnts, ancestor_masks, target_Ts,
                   robot_spheres_local, robot_sphere_joint_idx, world_spheres, world_capsules,
                   world_boxes, world_halfspaces, self_i, self_j, lower, upper, fixed_mask,
                   out_cfg, out_err, n_problems, n_seeds, n_act, n_joints, n_ee, n_robot_spheres,
                   Ms, Mc, Mb, Mh, n_self_pairs);
}

extern "C" int pk_ik_verify_select(void* stream, const float* cfgs, const float* errs,
                                   const float* prev, float continuity_weight,
                                   const float* twists, const float* parent_tf,
                                   const int32_t* parent_idx, const int32_t* act_idx,
                                   const float* mimic_mul, const float* mimic_off,
                                   const int32_t* mimic_act_idx, const int32_t* topo_inv,
                                   const int32_t* target_jnts, const float* target_Ts,
                                   float pos_tol, float rot_tol, float* winner_cfg,
                                   double* pos_err, double* rot_err, int32_t* success,
                                   int32_t n_problems, int32_t n_seeds, int32_t n_act,
                                   int32_t n_joints, int32_t n_ee) {
  PK_CHECK_ARG(n_problems >= 0 && n_seeds >= 0 && n_act >= 0 && n_ee >= 1, "bad extent");
  PK_CHECK_CAP(n_joints <= PK_MAX_JOINTS, "n_joints=%d exceeds %d", n_joints, PK_MAX_JOINTS);
  if (n_problems == 0) return PK_OK;
  PK_CHECK_ARG(n_seeds >= 1, "need at least one seed per problem");
  PK_CHECK_ARG(cfgs && errs && twists && parent_tf && parent_idx && act_idx && mimic_mul &&
                   mimic_off && mimic_act_idx && topo_inv && target_jnts && target_Ts && winner_cfg,
               "null buffer");
  VerifyArgs a{};
  a.m = ModelArgs{twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
                  topo_inv, n_joints, n_act};
  a.cfgs = cfgs; a.errs = errs; a.prev = prev; a.cw = continuity_weight;
  a.target_jnts = target_jnts; a.target_Ts = target_Ts; a.pos_tol = pos_tol; a.rot_tol = rot_tol;
  a.winner_cfg = winner_cfg; a.pos_err = pos_err; a.rot_err = rot_err; a.success = success;
  a.P = n_problems; a.Sd = n_seeds; a.n_act = n_act; a.n_ee = n_ee;
  verify_select_kernel<<<n_problems, 128, 0, (cudaStream_t)stream>>>(a);
  return cuda_status(cudaGetLastError(), "verify_select_kernel launch");
}

namespace pk {

template <int MAXA, int MAXEE, int TPS>
static int launch_batch_t(const SeedGroupBatch& B, size_t smem, int threads, int blocks, cudaStream_t st) {
  // the 4-block register budget only where shared memory admits 3 or more blocks per SM (8-wide body)
  auto kern = lm_batch_kernel<MAXA, MAXEE, TPS, 2>;
  if constexpr (MAXA <= 8)
    if ((228 * 1024) / (smem + 1024) >= 3) kern = lm_batch_kernel<MAXA, MAXEE, TPS, 4>;
  if (int s = set_smem_limit((const void*)kern, smem)) return s;
  if (blocks <= 0) {
    int dev = 0, sms = 0, per_sm = 0;
    if (int s = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return s;
    if (int s = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute")) return s;
    if (int s = cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem), "occupancy"))
      return s;
    blocks = std::max(1, sms * std::max(per_sm, 1));
  }
  kern<<<blocks, threads, smem, st>>>(B);
  return cuda_status(cudaGetLastError(), "lm_batch_kernel launch");
}

// One persistent launch over the items of the classes of `body`
// (kBodySeedGroup: 8-wide, lanes and seeds per block from the options;
// kBodySeedGroup16: 16-wide, one lane per seed, kSeedsPerBlock16 seeds per block).
static int launch_seed_group_body(const BatchCall& b, int body, cudaStream_t st, bool& queue_used, int& count) {
  int tps = b.opt.threads_per_seed, spb = b.opt.seeds_per_block;
  if (body == kBodySeedGroup16) {
    tps = 1;
    spb = kSeedsPerBlock16;
  }
  if (tps <= 0) { tps = 1; if (spb <= 0) spb = 128; }
  if (spb <= 0) spb = 128 / tps;
  SeedGroupBatch B{};
  bool any = false;
  size_t smem = 0;
  for (int c = 0; c < b.n_classes; ++c) {
    const pk_ik_class& k = b.cls[c];
    B.body[c] = k.body;
    if (k.body != body) continue;
    PK_CHECK_ARG(tps == 1 || tps == 2 || tps == 4 || tps == 8,
                 "seed-group classes take threads_per_seed 0, 1, 2, 4 or 8 (got %d)", tps);
    PK_CHECK_ARG(spb * tps <= 128 && (spb * tps) % 32 == 0,
                 "seeds_per_block * threads_per_seed must be a multiple of 32 and at most 128");
    if (body == kBodySeedGroup)
      PK_CHECK_CAP(k.n_act <= 8 && k.n_ee == 1, "body-0 classes need n_act <= 8 and one EE (class %d: %d, %d)",
                   c, k.n_act, k.n_ee);
    else
      PK_CHECK_CAP(k.n_act <= 16 && k.n_ee <= 2, "body-2 classes need n_act <= 16 and n_ee <= 2 (class %d: %d, %d)",
                   c, k.n_act, k.n_ee);
    LmArgs a{};
    a.m = ModelArgs{k.twists, k.parent_tf, k.parent_idx, k.act_idx, k.mimic_mul, k.mimic_off, k.mimic_act_idx,
                    k.topo_inv, k.n_joints, k.n_act};
    a.w = b.w;
    a.seeds = k.seeds; a.target_jnts = k.target_jnts; a.ancestor_masks = k.ancestor_masks; a.target_Ts = k.target_Ts;
    a.spheres_local = k.robot_spheres_local; a.sphere_joint = k.robot_sphere_joint_idx;
    a.self_i = k.self_i; a.self_j = k.self_j; a.lower = k.lower; a.upper = k.upper; a.fixed_mask = k.fixed_mask;
    a.out_cfg = k.out_cfg; a.out_err = k.out_err;
    a.P = k.n_problems; a.Sd = k.seed_stride; a.n_act = k.n_act; a.n_ee = k.n_ee; a.n_rs = k.n_robot_spheres;
    a.n_self = k.n_self;
    const pk_lm_options& o = b.opt;
    a.max_iter = o.max_iter; a.pos_w = o.pos_weight; a.ori_w = o.ori_weight; a.lam0 = o.lambda_init;
    a.lam_down = o.lambda_down; a.lam_up = o.lambda_up; a.eps_pos = o.eps_pos; a.eps_ori = o.eps_ori;
    a.coll = o.enable_collision ? 1 : 0; a.coll_w = o.collision_weight; a.margin = o.collision_margin;
    if (!a.coll) a.n_self = 0;
    a.spb = spb;
    a.grid_n = lm_grid_option(o.obstacle_grid, a.w.Ms);
    a.grid_auto = o.obstacle_grid == 0;
    if (int s = validate_lm(a)) return s;
    PK_CHECK_ARG(k.seeds && k.out_cfg && k.out_err && k.target_Ts && k.lower && k.upper && k.fixed_mask,
                 "null buffer in class %d", c);
    B.cls[c] = a;
    smem = std::max(smem, lm_layout(a, tps).total);
    any = true;
  }
  {
    // the fine default grid only where it keeps the blocks per SM (lm_fit_grid), over all classes
    size_t smem_def = 0;
    bool fine = false;
    for (int c = 0; c < b.n_classes; ++c) {
      if (b.cls[c].body != body) continue;
      LmArgs d = B.cls[c];
      if (d.grid_auto && d.grid_n > kObsGridDefault) {
        d.grid_n = kObsGridDefault;
        fine = true;
      }
      smem_def = std::max(smem_def, lm_layout(d, tps).total);
    }
    if (fine && lm_blocks_per_sm(smem) < lm_blocks_per_sm(smem_def)) {
      for (int c = 0; c < b.n_classes; ++c)
        if (b.cls[c].body == body && B.cls[c].grid_auto && B.cls[c].grid_n > kObsGridDefault)
          B.cls[c].grid_n = kObsGridDefault;
      smem = smem_def;
    }
  }
  if (!any || b.n_items == 0) return PK_OK;
  PK_CHECK_CAP(smem <= 220 * 1024, "LM working set (%zu B of shared memory) too large", smem);
  B.n_classes = b.n_classes;
  B.items = b.items;
  B.n_items = b.n_items;
  B.queue = b.queue;
  const int threads = spb * tps;
  // the item counter queue[0] serves both seed-group launches: the second
  // one starts from a counter cleared on the stream after the first
  if (queue_used) {
    if (int s = cuda_status(cudaMemsetAsync(b.queue, 0, sizeof(int32_t), st), "queue reset")) return s;
  }
  int s;
  if (body == kBodySeedGroup16) {
    s = launch_batch_t<16, 2, 1>(B, smem, threads, b.blocks, st);
  } else {
    switch (tps) {
      case 1: s = launch_batch_t<8, 1, 1>(B, smem, threads, b.blocks, st); break;
      case 2: s = launch_batch_t<8, 1, 2>(B, smem, threads, b.blocks, st); break;
      case 4: s = launch_batch_t<8, 1, 4>(B, smem, threads, b.blocks, st); break;
      default: s = launch_batch_t<8, 1, 8>(B, smem, threads, b.blocks, st); break;
    }
  }
  if (s == PK_OK) {
    queue_used = true;
    ++count;
  }
  return s;
}

int launch_seed_group_batch(const BatchCall& b, cudaStream_t st, int* launched) {
  bool queue_used = false;
  int n = 0;
  if (int s = launch_seed_group_body(b, kBodySeedGroup, st, queue_used, n)) return s;
  if (int s = launch_seed_group_body(b, kBodySeedGroup16, st, queue_used, n)) return s;
  if (launched) *launched += n;
  return PK_OK;
}

}  // namespace pk

extern "C" int pk_ik_batch(void* stream, const pk_lm_options* opt, const pk_ik_class* classes, int32_t n_classes,
                           const float* world_spheres, const float* world_capsules, const float* world_boxes,
                           const float* world_halfspaces, int32_t Ms, int32_t Mc, int32_t Mb, int32_t Mh,
                           const int32_t* items, int32_t n_items, int32_t* queue, int32_t blocks) {
  PK_CHECK_ARG(opt != nullptr && classes != nullptr, "null options or classes");
  PK_CHECK_ARG(!opt->fp64_solve, "fp64_solve is not offered by the batched kernels");
  PK_CHECK_ARG(opt->obstacle_grid >= -1 && opt->obstacle_grid <= kObsGridMax,
               "obstacle_grid must be -1 (none), 0 (default) or 1..%d cells per axis", kObsGridMax);
  PK_CHECK_ARG(n_classes >= 1, "at least one class is required");
  PK_CHECK_CAP(n_classes <= PK_MAX_CLASSES, "n_classes=%d exceeds %d", n_classes, PK_MAX_CLASSES);
  PK_CHECK_ARG(n_items >= 0 && Ms >= 0 && Mc >= 0 && Mb >= 0 && Mh >= 0, "negative extent");
  PK_CHECK_ARG((Ms == 0 || world_spheres) && (Mc == 0 || world_capsules) && (Mb == 0 || world_boxes) &&
                   (Mh == 0 || world_halfspaces),
               "null world buffer");
  if (n_items == 0) return PK_OK;
  PK_CHECK_ARG(items && queue, "null items or queue");
  PK_CHECK_ARG((reinterpret_cast<uintptr_t>(items) & 15) == 0, "items must be 16-byte aligned");
  for (int c = 0; c < n_classes; ++c)
    PK_CHECK_ARG(classes[c].body == kBodySeedGroup || classes[c].body == kBodyWarp ||
                     classes[c].body == kBodySeedGroup16,
                 "class %d: body must be 0, 1 or 2", c);
  const cudaStream_t st = (cudaStream_t)stream;
  if (int s = cuda_status(cudaMemsetAsync(queue, 0, 2 * sizeof(int32_t), st), "queue reset")) return s;
  BatchCall b{classes, n_classes, WorldArgs{world_spheres, world_capsules, world_boxes, world_halfspaces, Ms, Mc, Mb, Mh},
              *opt, reinterpret_cast<const int4*>(items), n_items, queue, blocks};
  int launched = 0;
  if (int s = launch_warp_batch(b, st, &launched)) return s;
  return launch_seed_group_batch(b, st, &launched);
}

// ---------------------------------------------------------------------------
// pk_ik_batch_static: pk_ik_batch without caller-provided device memory.
//
// Some callers cannot allocate device memory at the time they solve: a
// handler inside a runtime that owns all device memory and offers this call
// no workspace, or a real-time control loop that must not allocate once it
// runs.  This entry keeps the persistent kernels' only scratch -- the two
// work-queue counters -- in a fixed array that is part of the library
// image, so the call needs no allocation at all.
// ---------------------------------------------------------------------------

#define PK_STATIC_QUEUE_INTS 64  // 256 bytes; one call needs 2

namespace {

// Loaded with the library on every GPU that runs it and kept until exit.
static __device__ __align__(256) int32_t g_static_queue[PK_STATIC_QUEUE_INTS];

constexpr int kStaticQueueNeeded = 2;  // item counters of the two persistent kernels
static_assert(kStaticQueueNeeded <= PK_STATIC_QUEUE_INTS, "the static queue area is too small");

// Device address of g_static_queue in the current context.  Host code only
// sees a stand-in for the symbol, so the address is looked up with
// cudaGetSymbolAddress, which allocates nothing.  It is looked up on every
// call rather than cached: the module is loaded once per context, so after
// cudaDeviceReset, or in another context on the same device, the array sits
// at another address.  The first call in a context loads the module, which
// is why that call should come before any stream capture.
int static_queue_address(int32_t** out) {
  void* p = nullptr;
  if (int s = cuda_status(cudaGetSymbolAddress(&p, g_static_queue), "cudaGetSymbolAddress")) return s;
  *out = static_cast<int32_t*>(p);
  return PK_OK;
}

}  // namespace

extern "C" int pk_ik_batch_static(void* stream, const pk_lm_options* opt, const pk_ik_class* classes,
                                  int32_t n_classes, const float* world_spheres, const float* world_capsules,
                                  const float* world_boxes, const float* world_halfspaces, int32_t Ms, int32_t Mc,
                                  int32_t Mb, int32_t Mh, const int32_t* items, int32_t n_items, int32_t blocks) {
  int32_t* queue = nullptr;
  if (int s = static_queue_address(&queue)) return s;
  // pk_ik_batch clears the counters with an async memset on `stream` before its launches
  return pk_ik_batch(stream, opt, classes, n_classes, world_spheres, world_capsules, world_boxes, world_halfspaces,
                     Ms, Mc, Mb, Mh, items, n_items, queue, blocks);
}
