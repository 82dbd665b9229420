// SCO trajectory optimisation (sequential convex optimisation, Schulman et
// al. 2013) on the GPU -- the drop-in for sco_trajopt(..., use_cuda=True)
// (src/pyroffi/optimization_engines/_sco_optimization.py:505-551, run by
// src/pyroffi/cuda_kernels/_sco_trajopt_cuda_kernel.cu:584-1080).
//
// Outer iteration (n_outer_iters times), all trajectories at once:
//   1. linearise: at every waypoint q, five group distances d_g (self, world
//      spheres, capsules, boxes, halfspaces), each the smooth minimum
//      -tau log sum_p exp(-d_p / tau) of the group's pair distances (a pair's
//      distance is the hard minimum over its spheres; a group without pairs
//      reads 1e10), and their Jacobians J_g = dd_g/dq (:193-327, :700-757);
//   2. inner solve, per trajectory: n_inner_iters L-BFGS steps (history m,
//      Shanno-Kettler scaling, 5-point line search {1, .5, .25, .1, .025},
//      first sufficient decrease else first minimum) on the convex model
//        w_smooth (w_acc |acc|^2 + w_jerk |jerk|^2) + w_limits |limit excess|^2
//        + w_coll sum_{t,g} max(0, margin - d_lin)^2 + w_trust |q - q_k|^2,
//      d_lin = d_g + J_g (q_t - q_k,t), endpoints pinned; the best iterate is
//      kept and the endpoints are re-pinned (:333-582, :759-888);
//   3. w_coll <- min(w_coll * penalty_scale, w_collision_max).
// Finally each trajectory is ranked by its nonlinear cost at w_collision_max:
// smoothness + limits + w_collision_max * sum of -colldist_from_sdf over every
// self pair and (link, obstacle) pair distance (:893-1072).
//
// B200 mapping.  Linearisation runs over all B*T waypoints in one launch,
// TG lanes per waypoint.  The Jacobian is analytic and takes one pass: each
// (group, link) keeps an online-softmax accumulator -- the running maximum of
// e = -d/tau, the sum of exp(e - max) and the exp-weighted force
// F = sum w grad_c d and moment M = sum w (c x grad_c d) at the sphere that
// attains the pair's minimum -- which merges across lanes and links like a
// log-sum-exp; then dd_g/dq_j = omega_j . (M - p_j x F) + v_j . F summed over
// the links below joint j (rescaled by exp(max - lse)).  The reference takes
// central differences instead (2 n + 1 distance passes per waypoint); that
// form is kept as an option (fd_eps > 0).  The inner solve is one block per
// trajectory with the iterate, model, Jacobians and (when it fits) the L-BFGS
// history in shared memory and block reductions for the dot products.
#include <float.h>
#include <math.h>

#include "pk_obstacles.cuh"

namespace pk {

constexpr int kScoG = 5;      // self, spheres, capsules, boxes, halfspaces
constexpr int kScoMaxHist = 16;

struct ScoLinArgs {
  ModelArgs m;
  WorldArgs w;
  const float* cfg;           // [C, n]
  const int* parent_joint;    // [N]
  const float* link_spheres;  // [N, S, 4]
  const int* pair_i;          // [P]
  const int* pair_j;
  float* dist;                // [C, 5] or null
  float* jac;                 // [C, 5, n] or null
  float* coll;                // [C] or null: sum of -colldist_from_sdf over all pair distances
  long long C;
  int N, S, P, self_all;
  float tau, margin;
};

__device__ __forceinline__ float colldist(float d, float margin) {
  // colldist_from_sdf (src/pyroffi/collision/_collision.py:136-166)
  d = fminf(d, margin);
  float v;
  if (d < 0.f) {
    v = d - 0.5f * margin;
  } else {
    const float e = d - margin;
    v = -0.5f / (margin + 1e-6f) * e * e;
  }
  return fminf(v, 0.f);
}

// Online softmax over e = -d/tau with the exp-weighted force and moment.
struct SoftAcc {
  float ref, s;
  float3 F, M;
  __device__ __forceinline__ void init() {
    ref = -INFINITY;
    s = 0.f;
    F = make_float3(0.f, 0.f, 0.f);
    M = F;
  }
  __device__ __forceinline__ void scale(float k) {
    s *= k;
    F.x *= k; F.y *= k; F.z *= k;
    M.x *= k; M.y *= k; M.z *= k;
  }
  // `count`: the term enters the sum (a self pair is counted by one of its links only)
  __device__ __forceinline__ void add(float e, bool count, bool want_force, float3 g, float3 c) {
    if (e > ref) {
      scale(ref == -INFINITY ? 0.f : __expf(ref - e));
      ref = e;
    }
    const float w = __expf(e - ref);
    if (count) s += w;
    if (want_force) {
      F.x += w * g.x; F.y += w * g.y; F.z += w * g.z;
      const float3 cm = cross3(c, g);
      M.x += w * cm.x; M.y += w * cm.y; M.z += w * cm.z;
    }
  }
  // butterfly merge over the TG lanes of a group (every lane ends with the total)
  template <int TG>
  __device__ __forceinline__ void merge(unsigned gm) {
#pragma unroll
    for (int o = 1; o < TG; o <<= 1) {
      const float r2 = __shfl_xor_sync(gm, ref, o), s2 = __shfl_xor_sync(gm, s, o);
      const float fx = __shfl_xor_sync(gm, F.x, o), fy = __shfl_xor_sync(gm, F.y, o),
                  fz = __shfl_xor_sync(gm, F.z, o);
      const float mx = __shfl_xor_sync(gm, M.x, o), my = __shfl_xor_sync(gm, M.y, o),
                  mz = __shfl_xor_sync(gm, M.z, o);
      const float r = fmaxf(ref, r2);
      const float k1 = (ref == -INFINITY) ? 0.f : __expf(ref - r);
      const float k2 = (r2 == -INFINITY) ? 0.f : __expf(r2 - r);
      s = s * k1 + s2 * k2;
      F = make_float3(F.x * k1 + fx * k2, F.y * k1 + fy * k2, F.z * k1 + fz * k2);
      M = make_float3(M.x * k1 + mx * k2, M.y * k1 + my * k2, M.z * k1 + mz * k2);
      ref = r;
    }
  }
  __device__ __forceinline__ void store(float* q) const {
    q[0] = ref; q[1] = s; q[2] = F.x; q[3] = F.y; q[4] = F.z; q[5] = M.x; q[6] = M.y; q[7] = M.z;
  }
};

template <int TG>
__device__ __forceinline__ float group_sum(float v, unsigned gm) {
#pragma unroll
  for (int o = 1; o < TG; o <<= 1) v += __shfl_xor_sync(gm, v, o);
  return v;
}

// One world obstacle of a known kind in registers (1 sphere, 2 capsule, 3
// box, 4 halfspace) and its signed distance to a sphere (c, r).
template <int KIND>
struct ScoObs;

template <>
struct ScoObs<1> {
  float x, y, z, r;
  __device__ __forceinline__ void load(const ObsView& ob, int k) {
    const float4 s = ob.sph[k];
    x = s.x; y = s.y; z = s.z; r = s.w;
  }
  __device__ __forceinline__ float dist(float cx, float cy, float cz, float cr) const {
    const float dx = cx - x, dy = cy - y, dz = cz - z;
    return sqrt_fast(dx * dx + dy * dy + dz * dz) - (cr + r);
  }
};

template <>
struct ScoObs<2> {
  float ax, ay, az, vx, vy, vz, r, il2;  // p1, p2 - p1, radius, 1 / |p2 - p1|^2 (0 when degenerate)
  __device__ __forceinline__ void load(const ObsView& ob, int k) {
    const float* p = ob.cap + 7 * k;
    ax = p[0]; ay = p[1]; az = p[2];
    vx = p[3] - p[0]; vy = p[4] - p[1]; vz = p[5] - p[2];
    r = p[6];
    const float l2 = vx * vx + vy * vy + vz * vz;
    il2 = l2 > 1e-12f ? 1.f / l2 : 0.f;
  }
  __device__ __forceinline__ float dist(float cx, float cy, float cz, float cr) const {
    float t = ((cx - ax) * vx + (cy - ay) * vy + (cz - az) * vz) * il2;
    t = fmaxf(0.f, fminf(1.f, t));
    const float px = fmaf(t, vx, ax) - cx, py = fmaf(t, vy, ay) - cy, pz = fmaf(t, vz, az) - cz;
    return sqrt_fast(px * px + py * py + pz * pz) - (cr + r);
  }
};

template <>
struct ScoObs<3> {
  float p[15];  // centre, axis columns, half-lengths
  __device__ __forceinline__ void load(const ObsView& ob, int k) {
#pragma unroll
    for (int i = 0; i < 15; ++i) p[i] = ob.box[15 * k + i];
  }
  __device__ __forceinline__ float dist(float cx, float cy, float cz, float cr) const {
    const float dx = cx - p[0], dy = cy - p[1], dz = cz - p[2];
    const float q1 = fabsf(dx * p[3] + dy * p[4] + dz * p[5]) - p[12];
    const float q2 = fabsf(dx * p[6] + dy * p[7] + dz * p[8]) - p[13];
    const float q3 = fabsf(dx * p[9] + dy * p[10] + dz * p[11]) - p[14];
    const float m1 = fmaxf(q1, 0.f), m2 = fmaxf(q2, 0.f), m3 = fmaxf(q3, 0.f);
    return sqrt_fast(m1 * m1 + m2 * m2 + m3 * m3) + fminf(fmaxf(fmaxf(q1, q2), q3), 0.f) - cr;
  }
};

template <>
struct ScoObs<4> {
  float nx, ny, nz, off;  // normal, normal . point
  __device__ __forceinline__ void load(const ObsView& ob, int k) {
    const float* h = ob.hs + 6 * k;
    nx = h[0]; ny = h[1]; nz = h[2];
    off = h[3] * h[0] + h[4] * h[1] + h[5] * h[2];
  }
  __device__ __forceinline__ float dist(float cx, float cy, float cz, float cr) const {
    return cx * nx + cy * ny + cz * nz - off - cr;
  }
};

// Terms whose softmax weight is below exp(-kScoSkip) of the running maximum
// (2e-9; an FP32 sum that already holds the maximum term, >= 1, absorbs
// anything below 6e-8) are left out of the accumulators.
constexpr float kScoSkip = 20.f;

// One world group of one link: lane gl takes obstacles gl, gl + TG, ... of the
// kind's `count` (global obstacle index base + k); returns the accumulator
// merged over the group's lanes.  `gref`: the group's running maximum over
// the links done so far.  An obstacle is skipped whole when the link's
// bounding sphere (B, R) bounds its weight below the skip level (and, with
// the collision sum wanted, its distance at or above the margin).
template <int KIND, int MAXS, int TG>
__device__ __forceinline__ SoftAcc world_group(const ScoLinArgs& a, const ObsView& ob, int base, int count, int gl,
                                               unsigned gm, const LinkSpheres<MAXS>& L, float3 B, float R,
                                               bool want_soft, bool want_j, float inv_tau, float gref,
                                               float& csum) {
  SoftAcc acc;
  acc.init();
  for (int k = gl; k < count; k += TG) {
    ScoObs<KIND> o;
    o.load(ob, k);
    const float lb = o.dist(B.x, B.y, B.z, R);  // <= every sphere distance of the link
    if (want_soft) {
      if (-lb * inv_tau < fmaxf(acc.ref, gref) - kScoSkip && (!a.coll || lb >= a.margin)) continue;
    } else if (lb >= a.margin) {
      continue;  // adds exactly 0 to the collision sum
    }
    float dmin = FLT_MAX;
    int arg = 0;
    if constexpr (KIND == 1) {
      const float2 nx = make_float2(-o.x, -o.x), ny = make_float2(-o.y, -o.y), nz = make_float2(-o.z, -o.z);
      const float2 ro = make_float2(o.r, o.r);
#pragma unroll
      for (int q = 0; q < MAXS / 2; ++q) {  // padded spheres carry radius -1e30 and never win
        const float2 d = L.sphere_dist2_fast(q, nx, ny, nz, ro);
        if (d.x < dmin) { dmin = d.x; arg = 2 * q; }
        if (d.y < dmin) { dmin = d.y; arg = 2 * q + 1; }
      }
    } else {
#pragma unroll
      for (int s = 0; s < MAXS; ++s) {
        const float d = o.dist(L.X(s), L.Y(s), L.Z(s), L.R(s));
        if (d < dmin) { dmin = d; arg = s; }
      }
    }
    if (a.coll) csum -= colldist(dmin, a.margin);
    if (!want_soft) continue;
    const float e = -dmin * inv_tau;
    if (e < fmaxf(acc.ref, gref) - kScoSkip) continue;
    float3 cc = make_float3(0.f, 0.f, 0.f), gg = cc;
    if (want_j) {
      float rr = 0.f;
#pragma unroll
      for (int s = 0; s < MAXS; ++s)
        if (s == arg) { cc = make_float3(L.X(s), L.Y(s), L.Z(s)); rr = L.R(s); }
      obstacle_dist_grad<KIND - 1>(ob, base + k, cc, rr, gg);
    }
    acc.add(e, true, want_j, gg, cc);
  }
  if (want_soft) acc.merge<TG>(gm);
  return acc;
}

// Linearisation: group distances, their analytic Jacobians and/or the
// nonlinear collision sum, TG lanes per configuration.
template <int MAXS, int TG>
__global__ void __launch_bounds__(128, MAXS <= 8 ? 4 : (MAXS <= 16 ? 3 : 2)) sco_linearize_kernel(ScoLinArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  JointTable& jt = *reinterpret_cast<JointTable*>(smem_raw);
  unsigned char* p = smem_raw + sizeof(JointTable);
  const int N = a.N, S = a.S, n = a.m.n_act, nj = a.m.n_joints, P = a.P;
  const int nth = blockDim.x, tid = threadIdx.x;
  const int ng = nth / TG, grp = tid / TG, gl = tid % TG;
  const unsigned gm = ((1u << TG) - 1u) << ((tid & 31) & ~(TG - 1));
  float4* lsph = reinterpret_cast<float4*>(p); p += sizeof(float4) * N * S;
  float4* lbnd = reinterpret_cast<float4*>(p); p += sizeof(float4) * N;  // link bounding spheres
  int* lpj = reinterpret_cast<int*>(p); p += sizeof(int) * N;    // parent joint (sorted), -1 base
  int* lcnt = reinterpret_cast<int*>(p); p += sizeof(int) * N;   // valid spheres of the link
  int* lcur = reinterpret_cast<int*>(p); p += sizeof(int) * N;   // CSR fill cursor
  int* lps = reinterpret_cast<int*>(p); p += sizeof(int) * (N + 1);  // CSR start of each link's self pairs
  int* lpl = reinterpret_cast<int*>(p); p += sizeof(int) * 2 * P;    // entries 2 * pair + role
  p = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
  float* slots = reinterpret_cast<float*>(p); p += sizeof(float) * nj * 7 * ng;
  float* gjs = reinterpret_cast<float*>(p); p += sizeof(float) * nj * nth;
  p = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));

  load_joint_table(jt, a.m);
  const ObsView ob = stage_world(a.w, reinterpret_cast<float*>(p));
  for (int i = tid; i < N * S; i += nth) {
    const float* s = a.link_spheres + 4 * i;
    lsph[i] = make_float4(s[0], s[1], s[2], s[3]);
  }
  for (int l = tid; l < N; l += nth) {
    const int pj = a.parent_joint[l];
    lpj[l] = (pj < 0 || pj >= nj) ? -1 : jt.sorted_of[pj];
    int c = 0;
    for (int s = 0; s < S; ++s) c += a.link_spheres[4 * (l * S + s) + 3] >= 0.f;
    lcnt[l] = c;
    // bounding sphere of the link's spheres (link frame); the slack keeps
    // it conservative under rounding
    float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
    for (int s = 0; s < S; ++s) {
      const float* q = a.link_spheres + 4 * (l * S + s);
      if (q[3] < 0.f) continue;
      for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], q[k]); hi[k] = fmaxf(hi[k], q[k]); }
    }
    const float bx = 0.5f * (lo[0] + hi[0]), by = 0.5f * (lo[1] + hi[1]), bz = 0.5f * (lo[2] + hi[2]);
    float R = 0.f;
    for (int s = 0; s < S; ++s) {
      const float* q = a.link_spheres + 4 * (l * S + s);
      if (q[3] < 0.f) continue;
      R = fmaxf(R, sqrtf((q[0] - bx) * (q[0] - bx) + (q[1] - by) * (q[1] - by) + (q[2] - bz) * (q[2] - bz)) + q[3]);
    }
    lbnd[l] = c ? make_float4(bx, by, bz, R + 1e-4f + 1e-5f * R) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  if (tid == 0) {
    // self pairs per link (both links of a pair list it, in pair order); a
    // pair with an out-of-range or sphere-less link, or i == j, is skipped
    for (int l = 0; l <= N; ++l) lps[l] = 0;
    for (int q = 0; q < P; ++q) {
      const int li = a.pair_i[q], lj = a.pair_j[q];
      if (li < 0 || lj < 0 || li >= N || lj >= N || li == lj || !lcnt[li] || !lcnt[lj]) continue;
      ++lps[li + 1];
      ++lps[lj + 1];
    }
    for (int l = 0; l < N; ++l) { lps[l + 1] += lps[l]; lcur[l] = lps[l]; }
    for (int q = 0; q < P; ++q) {
      const int li = a.pair_i[q], lj = a.pair_j[q];
      if (li < 0 || lj < 0 || li >= N || lj >= N || li == lj || !lcnt[li] || !lcnt[lj]) continue;
      lpl[lcur[li]++] = 2 * q;
      lpl[lcur[lj]++] = 2 * q + 1;
    }
  }
  __syncthreads();

  const bool want_soft = a.dist != nullptr || a.jac != nullptr;
  const bool want_j = a.jac != nullptr;
  const float inv_tau = 1.f / a.tau;
  const int Ms = a.w.Ms, Mc = a.w.Mc, Mb = a.w.Mb;
  float* G = gjs + tid * nj;  // lane g < 5: group g's joint gradient, relative to its running maximum
  const PoseSlots ps{slots + grp, ng};
  static_assert(TG >= kScoG, "one lane per group");

  for (long long c = (long long)blockIdx.x * ng + grp; c < a.C; c += (long long)gridDim.x * ng) {
    const float* q = a.cfg + c * n;
    if (gl == 0) fk_thread(jt, [&](int i) { return q[i]; }, ps);
    // lane g < 5 owns group g: running maximum rg of -d/tau, sum sg of exp(-d/tau - rg), G
    float rg = -INFINITY, sg = 0.f;
    float gref[kScoG];  // every group's running maximum, known to all lanes
#pragma unroll
    for (int g = 0; g < kScoG; ++g) gref[g] = -INFINITY;
    if (want_j && gl < kScoG)
      for (int j = 0; j < nj; ++j) G[j] = 0.f;
    __syncwarp(gm);
    float csum = 0.f;
    for (int l = 0; l < N; ++l) {
      if (lcnt[l] == 0) continue;
      const Pose Tl = lpj[l] < 0 ? pose_identity() : ps.load(lpj[l]);
      LinkSpheres<MAXS> ls;
#pragma unroll
      for (int q = 0; q < MAXS / 2; ++q) {
        const float4 w0 = (2 * q < S) ? lsph[l * S + 2 * q] : make_float4(0.f, 0.f, 0.f, -1.f);
        const float4 w1 = (2 * q + 1 < S) ? lsph[l * S + 2 * q + 1] : make_float4(0.f, 0.f, 0.f, -1.f);
        const float3 v0 = pose_apply(Tl, make_float3(w0.x, w0.y, w0.z));
        const float3 v1 = pose_apply(Tl, make_float3(w1.x, w1.y, w1.z));
        ls.x[q] = make_float2(v0.x, v1.x); ls.y[q] = make_float2(v0.y, v1.y); ls.z[q] = make_float2(v0.z, v1.z);
        // a padded sphere's distances read 1e30
        ls.r[q] = make_float2(w0.w < 0.f ? -1e30f : w0.w, w1.w < 0.f ? -1e30f : w1.w);
      }
      const float4 bl = lbnd[l];
      const float3 Bw = pose_apply(Tl, make_float3(bl.x, bl.y, bl.z));
      // world groups: (link, obstacle) pairs, lane gl takes obstacles gl, gl + TG, ...
      SoftAcc mine, t;
      mine.init();
      t = world_group<1, MAXS, TG>(a, ob, 0, Ms, gl, gm, ls, Bw, bl.w, want_soft, want_j, inv_tau,
                                   gref[1], csum);
      if (gl == 1) mine = t;
      t = world_group<2, MAXS, TG>(a, ob, Ms, Mc, gl, gm, ls, Bw, bl.w, want_soft, want_j, inv_tau,
                                   gref[2], csum);
      if (gl == 2) mine = t;
      t = world_group<3, MAXS, TG>(a, ob, Ms + Mc, Mb, gl, gm, ls, Bw, bl.w, want_soft, want_j,
                                   inv_tau, gref[3], csum);
      if (gl == 3) mine = t;
      t = world_group<4, MAXS, TG>(a, ob, Ms + Mc + Mb, a.w.Mh, gl, gm, ls, Bw, bl.w, want_soft,
                                   want_j, inv_tau, gref[4], csum);
      if (gl == 4) mine = t;
      // self group: the pairs listing link l; lane gl takes entries gl, gl + TG, ...
      SoftAcc acc;
      acc.init();
      for (int k = lps[l] + gl; k < lps[l + 1]; k += TG) {
        const int e = lpl[k], pq = e >> 1, role = e & 1;
        const int o = role ? a.pair_i[pq] : a.pair_j[pq];
        if (!want_soft && role) continue;  // the collision sum takes each pair once
        const Pose To = lpj[o] < 0 ? pose_identity() : ps.load(lpj[o]);
        {
          // bounding spheres: skip a pair whose weight is bounded below the skip
          // level (or, for the collision sum alone, that is at least the margin apart)
          const float4 bo = lbnd[o];
          const float3 Bo = pose_apply(To, make_float3(bo.x, bo.y, bo.z));
          const float dx = Bw.x - Bo.x, dy = Bw.y - Bo.y, dz = Bw.z - Bo.z;
          const float lb = sqrt_fast(dx * dx + dy * dy + dz * dz) - (bl.w + bo.w);
          if (want_soft) {
            if (-lb * inv_tau < fmaxf(acc.ref, gref[0]) - kScoSkip && (!a.coll || lb >= a.margin)) continue;
          } else if (lb >= a.margin) {
            continue;
          }
        }
        float dmin = FLT_MAX;
        int arga = 0;
        float3 cb = make_float3(0.f, 0.f, 0.f);
        if (a.self_all) {
          // minimum over every (sphere of l, sphere of o)
          for (int sb = 0; sb < S; ++sb) {
            const float4 qb = lsph[o * S + sb];
            if (qb.w < 0.f) continue;
            const float3 pb = pose_apply(To, make_float3(qb.x, qb.y, qb.z));
            const float2 nx = make_float2(-pb.x, -pb.x), ny = make_float2(-pb.y, -pb.y), nz = make_float2(-pb.z, -pb.z);
#pragma unroll
            for (int q = 0; q < MAXS / 2; ++q) {
              const float2 d = ls.sphere_dist2_fast(q, nx, ny, nz, make_float2(qb.w, qb.w));
              if (d.x < dmin) { dmin = d.x; arga = 2 * q; cb = pb; }
              if (d.y < dmin) { dmin = d.y; arga = 2 * q + 1; cb = pb; }
            }
          }
        } else {
          // minimum over equal sphere indices
#pragma unroll
          for (int s = 0; s < MAXS; ++s) {
            if (s >= S || ls.R(s) < 0.f) continue;
            const float4 qb = lsph[o * S + s];
            if (qb.w < 0.f) continue;
            const float3 pb = pose_apply(To, make_float3(qb.x, qb.y, qb.z));
            const float dx = ls.X(s) - pb.x, dy = ls.Y(s) - pb.y, dz = ls.Z(s) - pb.z;
            const float d = sqrt_fast(dx * dx + dy * dy + dz * dz) - (ls.R(s) + qb.w);
            if (d < dmin) { dmin = d; arga = s; cb = pb; }
          }
        }
        if (!(dmin < 1e29f)) continue;  // no valid sphere pair (no common sphere index)
        if (a.coll && role == 0) csum -= colldist(dmin, a.margin);
        if (!want_soft) continue;
        const float ev = -dmin * inv_tau;
        if (ev < fmaxf(acc.ref, gref[0]) - kScoSkip) continue;
        float3 ca = make_float3(0.f, 0.f, 0.f);
#pragma unroll
        for (int s = 0; s < MAXS; ++s)
          if (s == arga) ca = make_float3(ls.X(s), ls.Y(s), ls.Z(s));
        float3 nrm = make_float3(0.f, 0.f, 0.f);
        if (want_j) {
          const float dx = ca.x - cb.x, dy = ca.y - cb.y, dz = ca.z - cb.z;
          const float len = sqrtf(dx * dx + dy * dy + dz * dz);
          const float inv = len > 0.f ? 1.f / len : 0.f;
          nrm = make_float3(dx * inv, dy * inv, dz * inv);
        }
        acc.add(ev, role == 0, want_j, nrm, ca);
      }
      if (want_soft) {
        acc.merge<TG>(gm);
        if (gl == 0) mine = acc;
        // lane g folds link l into group g
        if (gl < kScoG && mine.ref != -INFINITY) {
          if (mine.ref > rg) {
            const float k = (rg == -INFINITY) ? 0.f : __expf(rg - mine.ref);
            sg *= k;
            if (want_j)
              for (int j = 0; j < nj; ++j) G[j] *= k;
            rg = mine.ref;
          }
          const float k = __expf(mine.ref - rg);
          sg += k * mine.s;
          if (want_j) {
            const float3 F = make_float3(k * mine.F.x, k * mine.F.y, k * mine.F.z);
            const float3 Mo = make_float3(k * mine.M.x, k * mine.M.y, k * mine.M.z);
            if (F.x != 0.f || F.y != 0.f || F.z != 0.f || Mo.x != 0.f || Mo.y != 0.f || Mo.z != 0.f) {
              // every joint from the link's parent joint to the root moves the link
              for (int j = lpj[l]; j >= 0; j = jt.psorted[j]) {
                if (jt.kind[j] == kFixed) continue;
                const Pose Tj = ps.load(j);
                const float* tw = jt.tw[j];
                const float3 w = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z, make_float3(tw[3], tw[4], tw[5]));
                const float3 vv = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z, make_float3(tw[0], tw[1], tw[2]));
                const float3 pxF = cross3(make_float3(Tj.tx, Tj.ty, Tj.tz), F);
                G[j] += w.x * (Mo.x - pxF.x) + w.y * (Mo.y - pxF.y) + w.z * (Mo.z - pxF.z) + vv.x * F.x +
                        vv.y * F.y + vv.z * F.z;
              }
            }
          }
        }
        const int lane0 = (tid & 31) & ~(TG - 1);
#pragma unroll
        for (int g = 0; g < kScoG; ++g) gref[g] = __shfl_sync(gm, rg, lane0 + g);
      }
    }
    if (a.coll) {
      csum = group_sum<TG>(csum, gm);
      if (gl == 0) a.coll[c] = csum;
    }
    if (want_soft && gl < kScoG) {
      const bool has = sg > 0.f;
      const float lse = has ? logf(sg) + rg : 0.f;
      if (a.dist) a.dist[c * kScoG + gl] = has ? -a.tau * lse : 1e10f;
      if (want_j) {
        // softmax weights exp(-d/tau - lse) = exp(-d/tau - rg) / sg
        const float inv = has ? 1.f / sg : 0.f;
        float* out = a.jac + (c * kScoG + gl) * n;
        for (int col = 0; col < n; ++col) {
          float v = 0.f;
          for (int j = 0; j < nj; ++j)
            if (jt.src[j] == col) v += jt.mul[j] * G[j];
          out[col] = v * inv;
        }
      }
    }
    __syncwarp(gm);
  }
}

// ---------------------------------------------------------------------------
// inner L-BFGS solve, one block per trajectory
// ---------------------------------------------------------------------------

struct ScoInnerArgs {
  float* traj;          // [B, T, n]: the linearisation point in, the best iterate out (endpoints re-pinned)
  const float* dist;    // [B, T, 5]
  const float* jac;     // [B, T, 5, n]
  const float* lower;   // [n]
  const float* upper;
  const float* start;   // [n]
  const float* goal;
  float* hist;          // [B, 2, m, T, n] L-BFGS history when it is not kept in shared memory
  int B, T, n, m, iters;
  float w_smooth, w_acc, w_jerk, w_limits, w_trust, w_coll, margin;
};

__device__ __constant__ float kSt[5] = {-1.f / 12.f, 16.f / 12.f, -30.f / 12.f, 16.f / 12.f, -1.f / 12.f};
__device__ __constant__ float kLsAlpha[5] = {1.f, 0.5f, 0.25f, 0.1f, 0.025f};

// Sum of K values over the block; every thread returns the same totals.
template <int K>
__device__ __forceinline__ void block_sum(float (&v)[K], float* red) {
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();  // the previous reduction has been read
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * 32 + w] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    float s = 0.f;
    for (int i = 0; i < nw; ++i) s += red[k * 32 + i];  // fixed order
    v[k] = s;
  }
}

struct InnerView {
  float *x, *qk, *g, *gp, *dir, *bx, *acc, *gacc, *J, *dk, *dl, *gc, *lo, *hi, *rho, *syv, *yyv, *alph, *red, *Sb, *Yb;
};

// A thread's walk over a row-major [rows, n] element space, i = tid, tid +
// nth, ...: its (row, column) advance without a division per step.
struct Walk {
  int t0, d0, dt, dd, n;
  __device__ __forceinline__ void step(int& t, int& d) const {
    t += dt;
    d += dd;
    if (d >= n) { d -= n; ++t; }
  }
};

// Cost and gradient of the convex model at v.x; leaves acc(x) in v.acc and
// d_lin in v.dl.  Row k of acc is the stencil over rows k..k+4 of x, so the
// element loops index acc and x by i +- q n.
__device__ float inner_cost_grad(const ScoInnerArgs& a, const InnerView& v, const Walk& W) {
  const int T = a.T, n = a.n, Tn = T * n, K = T > 4 ? T - 4 : 0, Kn = K * n, tid = threadIdx.x,
            nth = blockDim.x;
  float part = 0.f;
  __syncthreads();  // x is complete
  for (int i = tid; i < Kn; i += nth) {
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q) s += kSt[q] * v.x[i + q * n];
    v.acc[i] = s;
  }
  for (int i = tid; i < T * kScoG; i += nth) {
    const int t = i / kScoG;
    float dl = v.dk[i];
    const float* Jr = v.J + i * n;
    const float* xr = v.x + t * n;
    const float* qr = v.qk + t * n;
    for (int d = 0; d < n; ++d) dl += Jr[d] * (xr[d] - qr[d]);
    v.dl[i] = dl;
    const float viol = fmaxf(0.f, a.margin - dl);
    part += a.w_coll * viol * viol;
    v.gc[i] = -2.f * a.w_coll * viol;
  }
  __syncthreads();
  for (int i = tid; i < Kn; i += nth) {
    const float c = v.acc[i];
    part += a.w_smooth * a.w_acc * c * c;
    float ga = 2.f * a.w_acc * c;
    if (i + n < Kn) {
      const float j = v.acc[i + n] - c;
      part += a.w_smooth * a.w_jerk * j * j;
      ga -= 2.f * a.w_jerk * j;
    }
    if (i >= n) ga += 2.f * a.w_jerk * (c - v.acc[i - n]);
    v.gacc[i] = ga;
  }
  __syncthreads();
  for (int i = tid, t = W.t0, d = W.d0; i < Tn; i += nth, W.step(t, d)) {
    float gs = 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int k = i - q * n;
      if (k >= 0 && k < Kn) gs += kSt[q] * v.gacc[k];
    }
    const float xv = v.x[i], lo = v.lo[d], hi = v.hi[d];
    const float viol = fmaxf(0.f, xv - hi) + fmaxf(0.f, lo - xv);
    part += a.w_limits * viol * viol;
    const float sgn = xv > hi ? 1.f : (xv < lo ? -1.f : 0.f);
    const float delta = xv - v.qk[i];
    part += a.w_trust * delta * delta;
    float gcol = 0.f;
    const float* gct = v.gc + t * kScoG;
    const float* Jt = v.J + t * kScoG * n + d;
#pragma unroll
    for (int g = 0; g < kScoG; ++g) gcol += gct[g] * Jt[g * n];
    float gi = a.w_smooth * gs + 2.f * a.w_limits * viol * sgn + gcol + 2.f * a.w_trust * delta;
    if (t == 0 || t == T - 1) gi = 0.f;
    v.g[i] = gi;
  }
  float r[1] = {part};
  block_sum<1>(r, v.red);
  return r[0];
}

template <bool SMEM_HIST>
__global__ void __launch_bounds__(256, 2) sco_inner_kernel(ScoInnerArgs a) {
  extern __shared__ __align__(16) float sm[];
  const int T = a.T, n = a.n, Tn = T * n, K = T > 4 ? T - 4 : 0, m = a.m;
  const int tid = threadIdx.x, nth = blockDim.x;
  const long long b = blockIdx.x;
  InnerView v;
  float* p = sm;
  v.x = p; p += Tn;
  v.qk = p; p += Tn;
  v.g = p; p += Tn;
  v.gp = p; p += Tn;
  v.dir = p; p += Tn;
  v.bx = p; p += Tn;
  v.acc = p; p += K * n;
  v.gacc = p; p += K * n;
  v.J = p; p += kScoG * Tn;
  v.dk = p; p += kScoG * T;
  v.dl = p; p += kScoG * T;
  v.gc = p; p += kScoG * T;
  v.lo = p; p += n;
  v.hi = p; p += n;
  v.rho = p; p += m;
  v.syv = p; p += m;
  v.yyv = p; p += m;
  v.alph = p; p += m;
  v.red = p; p += 5 * 32;
  if (SMEM_HIST) {
    v.Sb = p;
    v.Yb = p + (size_t)m * Tn;
  } else {
    v.Sb = a.hist + (size_t)b * 2 * m * Tn;
    v.Yb = v.Sb + (size_t)m * Tn;
  }
  const float* tr = a.traj + b * Tn;
  for (int i = tid; i < Tn; i += nth) v.x[i] = v.qk[i] = v.bx[i] = tr[i];
  for (int i = tid; i < kScoG * Tn; i += nth) v.J[i] = a.jac[b * kScoG * Tn + i];
  for (int i = tid; i < kScoG * T; i += nth) v.dk[i] = a.dist[b * kScoG * T + i];
  for (int i = tid; i < n; i += nth) { v.lo[i] = a.lower[i]; v.hi[i] = a.upper[i]; }

  const Walk W{tid / n, tid % n, nth / n, nth % n, n};
  float cost = inner_cost_grad(a, v, W);
  float best_cost = cost;
  int m_used = 0, newest = 0;
  for (int it = 0; it < a.iters; ++it) {
    if (it > 0) {
      cost = inner_cost_grad(a, v, W);
      // curvature pair (s, y) = (last step, gradient change)
      float r[2] = {0.f, 0.f};
      for (int i = tid; i < Tn; i += nth) {
        const float y = v.g[i] - v.gp[i];
        r[0] += v.dir[i] * y;
        r[1] += y * y;
      }
      block_sum<2>(r, v.red);
      if (r[0] > 1e-10f * r[1] + 1e-30f) {
        const int nn = (newest + 1) % m;
        for (int i = tid; i < Tn; i += nth) {
          v.Sb[(size_t)nn * Tn + i] = v.dir[i];
          v.Yb[(size_t)nn * Tn + i] = v.g[i] - v.gp[i];
        }
        if (tid == 0) { v.rho[nn] = 1.f / (r[0] + 1e-30f); v.syv[nn] = r[0]; v.yyv[nn] = r[1]; }
        newest = nn;
        if (m_used < m) ++m_used;
        __syncthreads();
      }
    }
    for (int i = tid; i < Tn; i += nth) v.gp[i] = v.g[i];
    // direction -H g by the two-loop recursion (own elements only between reductions)
    if (m_used == 0) {
      float r[1] = {0.f};
      for (int i = tid; i < Tn; i += nth) r[0] += v.g[i] * v.g[i];
      block_sum<1>(r, v.red);
      const float inv = 1.f / (sqrtf(r[0]) + 1e-18f);
      for (int i = tid; i < Tn; i += nth) v.dir[i] = -v.g[i] * inv;
    } else {
      for (int i = tid; i < Tn; i += nth) v.dir[i] = v.g[i];
      for (int k = 0; k < m_used; ++k) {
        const int idx = (newest - k + m) % m;
        const float* Si = v.Sb + (size_t)idx * Tn;
        const float* Yi = v.Yb + (size_t)idx * Tn;
        float r[1] = {0.f};
        for (int i = tid; i < Tn; i += nth) r[0] += Si[i] * v.dir[i];
        block_sum<1>(r, v.red);
        const float al = v.rho[idx] * r[0];
        if (tid == 0) v.alph[k] = al;
        for (int i = tid; i < Tn; i += nth) v.dir[i] -= al * Yi[i];
      }
      const float gamma = v.syv[newest] / (v.yyv[newest] + 1e-18f);
      for (int i = tid; i < Tn; i += nth) v.dir[i] *= gamma;
      for (int k = m_used - 1; k >= 0; --k) {
        const int idx = (newest - k + m) % m;
        const float* Si = v.Sb + (size_t)idx * Tn;
        const float* Yi = v.Yb + (size_t)idx * Tn;
        float r[1] = {0.f};
        for (int i = tid; i < Tn; i += nth) r[0] += Yi[i] * v.dir[i];
        block_sum<1>(r, v.red);  // also publishes alph[] written by thread 0
        const float c = v.alph[k] - v.rho[idx] * r[0];
        for (int i = tid; i < Tn; i += nth) v.dir[i] += c * Si[i];
      }
      for (int i = tid; i < Tn; i += nth) v.dir[i] = -v.dir[i];
    }
    for (int i = tid; i < Tn; i += nth)
      if (i < n || i >= Tn - n) v.dir[i] = 0.f;  // pinned endpoints
    __syncthreads();
    // 5-point line search: acc and d_lin are linear in the step, so the trial
    // costs take acc(x) + a acc(dir) and d_lin(x) + a J dir
    const int Kn = K * n;
    for (int i = tid; i < Kn; i += nth) {
      float s = 0.f;
#pragma unroll
      for (int q = 0; q < 5; ++q) s += kSt[q] * v.dir[i + q * n];
      v.gacc[i] = s;
    }
    for (int i = tid; i < T * kScoG; i += nth) {
      const int t = i / kScoG;
      float s = 0.f;
      const float* Jr = v.J + i * n;
      const float* dr = v.dir + t * n;
      for (int d = 0; d < n; ++d) s += Jr[d] * dr[d];
      v.gc[i] = s;
    }
    __syncthreads();
    float tc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = tid; i < Kn; i += nth) {
      const float c = v.acc[i], cd = v.gacc[i];
      const bool jerk = i + n < Kn;
      const float c1 = jerk ? v.acc[i + n] : 0.f, cd1 = jerk ? v.gacc[i + n] : 0.f;
#pragma unroll
      for (int ai = 0; ai < 5; ++ai) {
        const float al = kLsAlpha[ai];
        const float c0 = c + al * cd;
        tc[ai] += a.w_smooth * a.w_acc * c0 * c0;
        if (jerk) {
          const float j = (c1 + al * cd1) - c0;
          tc[ai] += a.w_smooth * a.w_jerk * j * j;
        }
      }
    }
    for (int i = tid, t = W.t0, d = W.d0; i < Tn; i += nth, W.step(t, d)) {
      const float x0 = v.x[i], p0 = v.dir[i], q0 = v.qk[i], lo = v.lo[d], hi = v.hi[d];
#pragma unroll
      for (int ai = 0; ai < 5; ++ai) {
        const float xv = x0 + kLsAlpha[ai] * p0;
        const float viol = fmaxf(0.f, xv - hi) + fmaxf(0.f, lo - xv);
        const float delta = xv - q0;
        tc[ai] += a.w_limits * viol * viol + a.w_trust * delta * delta;
      }
    }
    for (int i = tid; i < T * kScoG; i += nth) {
      const float dl = v.dl[i], gd = v.gc[i];
#pragma unroll
      for (int ai = 0; ai < 5; ++ai) {
        const float viol = fmaxf(0.f, a.margin - (dl + kLsAlpha[ai] * gd));
        tc[ai] += a.w_coll * viol * viol;
      }
    }
    block_sum<5>(tc, v.red);
    int best = 0;
    for (int ai = 1; ai < 5; ++ai)
      if (tc[ai] < tc[best]) best = ai;
    const float suff = cost * (1.f - 1e-4f);
    for (int ai = 0; ai < 5; ++ai)
      if (tc[ai] < suff) { best = ai; break; }
    const float al = kLsAlpha[best];
    const bool better = tc[best] < best_cost;
    for (int i = tid; i < Tn; i += nth) {
      const float st = al * v.dir[i];
      v.x[i] += st;
      v.dir[i] = st;
      if (better) v.bx[i] = v.x[i];
    }
    if (better) best_cost = tc[best];
  }
  __syncthreads();
  float* out = a.traj + b * Tn;
  for (int i = tid, t = W.t0, d = W.d0; i < Tn; i += nth, W.step(t, d))
    out[i] = t == 0 ? a.start[d] : (t == T - 1 ? a.goal[d] : v.bx[i]);
}

// Nonlinear ranking cost per trajectory: smoothness + limits + w * sum_t coll[t].
__global__ void __launch_bounds__(128) sco_final_kernel(const float* traj, const float* coll, const float* lower,
                                                        const float* upper, float* cost, int T, int n,
                                                        float w_smooth, float w_acc, float w_jerk,
                                                        float w_limits, float w_coll) {
  __shared__ float red[32];
  const long long b = blockIdx.x;
  const float* x = traj + b * T * n;
  const int K = T > 4 ? T - 4 : 0;
  float part = 0.f;
  for (int i = threadIdx.x; i < K * n; i += blockDim.x) {
    const int k = i / n, d = i - k * n;
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q) a0 += kSt[q] * x[(k + q) * n + d];
    part += w_smooth * w_acc * a0 * a0;
    if (k + 1 < K) {
#pragma unroll
      for (int q = 0; q < 5; ++q) a1 += kSt[q] * x[(k + 1 + q) * n + d];
      const float j = a1 - a0;
      part += w_smooth * w_jerk * j * j;
    }
  }
  for (int i = threadIdx.x; i < T * n; i += blockDim.x) {
    const int d = i % n;
    const float viol = fmaxf(0.f, x[i] - upper[d]) + fmaxf(0.f, lower[d] - x[i]);
    part += w_limits * viol * viol;
  }
  for (int t = threadIdx.x; t < T; t += blockDim.x) part += w_coll * coll[b * T + t];
  float r[1] = {part};
  block_sum<1>(r, red);
  if (threadIdx.x == 0) cost[b] = r[0];
}

// out[b, t] = start / goal at the ends, else init[b, t]
__global__ void sco_pin_kernel(const float* init, const float* start, const float* goal, float* out, long long B,
                               int T, int n) {
  const long long total = B * T * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % n), t = (int)((i / n) % T);
    out[i] = t == 0 ? start[d] : (t == T - 1 ? goal[d] : init[i]);
  }
}

// central-difference configurations: row c (2n + 1) is q_c, row c (2n + 1) + 2d + 1 adds eps to
// coordinate d and row c (2n + 1) + 2d + 2 subtracts it
__global__ void sco_fd_configs_kernel(const float* cfg, float* out, long long C, int n, float eps) {
  const int R = 2 * n + 1;
  const long long total = C * R * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i % n);
    const long long row = i / n;
    const long long c = row / R;
    const int r = (int)(row - c * R);
    float v = cfg[c * n + d];
    if (r > 0 && (r - 1) / 2 == d) v = ((r - 1) % 2 == 0) ? v + eps : v - eps;
    out[i] = v;
  }
}

__global__ void sco_fd_jac_kernel(const float* dfd, float* dist, float* jac, long long C, int n, float eps) {
  const int R = 2 * n + 1;
  const long long total = C * kScoG;
  const float inv2e = 1.f / (2.f * eps);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / kScoG;
    const int g = (int)(i - c * kScoG);
    const float* base = dfd + c * R * kScoG;
    dist[i] = base[g];
    for (int d = 0; d < n; ++d)
      jac[i * n + d] = (base[(2 * d + 1) * kScoG + g] - base[(2 * d + 2) * kScoG + g]) * inv2e;
  }
}

static size_t lin_smem(const ScoLinArgs& a, int nth, int TG) {
  const int ng = nth / TG, nj = a.m.n_joints;
  size_t s = sizeof(JointTable) + sizeof(float4) * a.N * (a.S + 1) + sizeof(int) * (3 * a.N + a.N + 1 + 2 * a.P);
  s = (s + 15) & ~size_t(15);
  s += sizeof(float) * ((size_t)nj * 7 * ng + (size_t)nj * nth);
  s = (s + 15) & ~size_t(15);
  return s + sizeof(float) * a.w.smem_floats();
}

static int launch_linearize(const ScoLinArgs& a, cudaStream_t st) {
  if (a.C == 0) return PK_OK;
  constexpr int TG = 8, nth = 128;
  const size_t smem = lin_smem(a, nth, TG);
  PK_CHECK_CAP(smem <= 220 * 1024, "SCO linearisation working set (%zu B of shared memory) too large", smem);
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long ng = nth / TG;
  long long blocks = (a.C + ng - 1) / ng;
  if (blocks > 64LL * sms) blocks = 64LL * sms;  // grid-stride beyond that
  auto kern = a.S <= 4    ? sco_linearize_kernel<4, TG>
              : a.S <= 8  ? sco_linearize_kernel<8, TG>
              : a.S <= 16 ? sco_linearize_kernel<16, TG>
                          : sco_linearize_kernel<32, TG>;
  if (int s = set_smem_limit((const void*)kern, smem)) return s;
  kern<<<(unsigned)blocks, nth, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "sco_linearize_kernel launch");
}

static int inner_threads(const pk_sco_options* o, int Tn) {
  if (o->inner_threads > 0) return o->inner_threads;
  return Tn <= 1536 ? 128 : 256;
}

static size_t inner_smem_bytes(int T, int n, int m, bool hist) {
  const size_t Tn = (size_t)T * n, Kn = (size_t)(T > 4 ? T - 4 : 0) * n;
  return sizeof(float) * (6 * Tn + 2 * Kn + (size_t)kScoG * Tn + 3 * (size_t)kScoG * T + 2 * (size_t)n +
                          4 * (size_t)m + 5 * 32 + (hist ? 2 * (size_t)m * Tn : 0));
}

constexpr size_t kInnerSmemMax = 200 * 1024;

static bool hist_in_smem(int T, int n, int m) { return inner_smem_bytes(T, n, m, true) <= kInnerSmemMax; }

static int launch_inner(const ScoInnerArgs& a, int nth, cudaStream_t st) {
  if (a.B == 0) return PK_OK;
  const bool sh = hist_in_smem(a.T, a.n, a.m);
  const size_t smem = inner_smem_bytes(a.T, a.n, a.m, sh);
  PK_CHECK_CAP(smem <= kInnerSmemMax, "SCO inner-solve working set (%zu B of shared memory) too large", smem);
  PK_CHECK_ARG(sh || a.hist, "the L-BFGS history does not fit in shared memory: a history buffer is required");
  auto kern = sh ? sco_inner_kernel<true> : sco_inner_kernel<false>;
  if (int s = set_smem_limit((const void*)kern, smem)) return s;
  kern<<<(unsigned)a.B, nth, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "sco_inner_kernel launch");
}

static unsigned ew_blocks(long long total) {
  long long b = (total + 255) / 256;
  if (b > 4096) b = 4096;
  return (unsigned)(b < 1 ? 1 : b);
}

static int check_options(const pk_sco_options* o) {
  PK_CHECK_ARG(o != nullptr, "null options");
  PK_CHECK_ARG(o->n_outer_iters >= 0 && o->n_inner_iters >= 0, "negative iteration count");
  PK_CHECK_ARG(o->m_lbfgs >= 1 && o->m_lbfgs <= kScoMaxHist, "m_lbfgs must be in [1, %d] (got %d)", kScoMaxHist,
               o->m_lbfgs);
  PK_CHECK_ARG(o->smooth_min_temperature > 0.f, "smooth_min_temperature must be positive");
  PK_CHECK_ARG(o->fd_eps >= 0.f, "fd_eps must be >= 0");
  PK_CHECK_ARG(o->inner_threads == 0 || (o->inner_threads % 32 == 0 && o->inner_threads <= 256 &&
                                         o->inner_threads >= 32),
               "inner_threads must be 0 or a multiple of 32 in [32, 256]");
  return PK_OK;
}

}  // namespace pk

using namespace pk;

namespace {

struct WsLayout {
  size_t dist, jac, coll, hist, fd_cfg, fd_dist, total;
};

WsLayout ws_layout(const pk_sco_options* o, long long B, int T, int n) {
  auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t C = (size_t)B * T;
  WsLayout w;
  size_t off = 0;
  w.dist = off; off += up(sizeof(float) * C * kScoG);
  w.jac = off; off += up(sizeof(float) * C * kScoG * n);
  w.coll = off; off += up(sizeof(float) * C);
  w.hist = off; off += hist_in_smem(T, n, o->m_lbfgs) ? 0 : up(sizeof(float) * (size_t)B * 2 * o->m_lbfgs * T * n);
  const size_t R = 2 * (size_t)n + 1;
  w.fd_cfg = off; off += o->fd_eps > 0.f ? up(sizeof(float) * C * R * n) : 0;
  w.fd_dist = off; off += o->fd_eps > 0.f ? up(sizeof(float) * C * R * kScoG) : 0;
  w.total = off;
  return w;
}

int check_robot(int64_t n_act, int32_t n_joints, int32_t n_links, int32_t S, int32_t P) {
  PK_CHECK_ARG(n_act >= 0 && n_links >= 0 && S >= 0 && P >= 0 && n_joints >= 0, "negative extent");
  PK_CHECK_CAP(n_joints <= PK_MAX_JOINTS, "n_joints=%d exceeds %d", n_joints, PK_MAX_JOINTS);
  PK_CHECK_CAP(S <= 32, "at most 32 spheres per link (got %d)", S);
  return PK_OK;
}

ScoLinArgs lin_args(const pk_sco_options* o, const float* cfg, const float* twists, const float* parent_tf,
                    const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                    const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                    const int32_t* parent_joint_indices, const float* link_spheres, const int32_t* pair_i,
                    const int32_t* pair_j, const float* ws, const float* wc, const float* wb, const float* wh,
                    long long C, int n_act, int n_joints, int N, int S, int P, int Ms, int Mc, int Mb, int Mh) {
  ScoLinArgs a;
  a.m = ModelArgs{twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx, topo_inv,
                  n_joints, n_act};
  a.w = WorldArgs{ws, wc, wb, wh, Ms, Mc, Mb, Mh};
  a.cfg = cfg; a.parent_joint = parent_joint_indices; a.link_spheres = link_spheres;
  a.pair_i = pair_i; a.pair_j = pair_j;
  a.dist = a.jac = a.coll = nullptr;
  a.C = C; a.N = N; a.S = S; a.P = P;
  a.self_all = o->self_all_pairs ? 1 : 0;
  a.tau = o->smooth_min_temperature;
  a.margin = o->collision_margin;
  return a;
}

ScoInnerArgs inner_args(const pk_sco_options* o, float* traj, const float* dist, const float* jac,
                        const float* lower, const float* upper, const float* start, const float* goal, float* hist,
                        float w_coll, long long B, int T, int n) {
  ScoInnerArgs a;
  a.traj = traj; a.dist = dist; a.jac = jac; a.lower = lower; a.upper = upper; a.start = start; a.goal = goal;
  a.hist = hist;
  a.B = (int)B; a.T = T; a.n = n; a.m = o->m_lbfgs; a.iters = o->n_inner_iters;
  a.w_smooth = o->w_smooth; a.w_acc = o->w_acc; a.w_jerk = o->w_jerk; a.w_limits = o->w_limits;
  a.w_trust = o->w_trust; a.w_coll = w_coll; a.margin = o->collision_margin;
  return a;
}

}  // namespace

extern "C" int pk_sco_linearize(void* stream, const pk_sco_options* opt, const float* cfg, const float* twists,
                                const float* parent_tf, const int32_t* parent_idx, const int32_t* act_idx,
                                const float* mimic_mul, const float* mimic_off, const int32_t* mimic_act_idx,
                                const int32_t* topo_inv, const int32_t* parent_joint_indices,
                                const float* link_spheres, const int32_t* pair_i, const int32_t* pair_j,
                                const float* world_spheres, const float* world_capsules, const float* world_boxes,
                                const float* world_halfspaces, float* dist, float* jac, float* coll, int64_t C,
                                int32_t n_act, int32_t n_joints, int32_t n_links, int32_t S, int32_t P, int32_t Ms,
                                int32_t Mc, int32_t Mb, int32_t Mh) {
  if (int s = check_options(opt)) return s;
  if (int s = check_robot(n_act, n_joints, n_links, S, P)) return s;
  PK_CHECK_ARG(C >= 0 && Ms >= 0 && Mc >= 0 && Mb >= 0 && Mh >= 0, "negative extent");
  PK_CHECK_ARG(dist || jac || coll, "no output requested");
  if (C == 0) return PK_OK;
  PK_CHECK_ARG(cfg && twists && parent_tf && parent_idx && act_idx && mimic_mul && mimic_off && mimic_act_idx &&
                   topo_inv && parent_joint_indices,
               "null buffer");
  PK_CHECK_ARG(n_links * S == 0 || link_spheres, "null link_spheres");
  PK_CHECK_ARG(P == 0 || (pair_i && pair_j), "null pairs");
  PK_CHECK_ARG((Ms == 0 || world_spheres) && (Mc == 0 || world_capsules) && (Mb == 0 || world_boxes) &&
                   (Mh == 0 || world_halfspaces),
               "null world buffer");
  ScoLinArgs a = lin_args(opt, cfg, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
                          topo_inv, parent_joint_indices, link_spheres, pair_i, pair_j, world_spheres,
                          world_capsules, world_boxes, world_halfspaces, C, n_act, n_joints, n_links, S, P, Ms, Mc,
                          Mb, Mh);
  a.dist = dist; a.jac = jac; a.coll = coll;
  return launch_linearize(a, (cudaStream_t)stream);
}

extern "C" int pk_sco_inner(void* stream, const pk_sco_options* opt, float* traj, const float* dist,
                            const float* jac, const float* lower, const float* upper, const float* start,
                            const float* goal, float* hist, float w_coll, int64_t B, int32_t T, int32_t n_act) {
  if (int s = check_options(opt)) return s;
  PK_CHECK_ARG(B >= 0 && T >= 2 && n_act >= 1, "need B >= 0, T >= 2, n_act >= 1");
  PK_CHECK_CAP(B < (1LL << 31), "batch too large");
  if (B == 0) return PK_OK;
  PK_CHECK_ARG(traj && dist && jac && lower && upper && start && goal, "null buffer");
  return launch_inner(inner_args(opt, traj, dist, jac, lower, upper, start, goal, hist, w_coll, B, T, n_act),
                      inner_threads(opt, T * n_act), (cudaStream_t)stream);
}

extern "C" int pk_sco_final_cost(void* stream, const pk_sco_options* opt, const float* traj, const float* coll,
                                 const float* lower, const float* upper, float* cost, int64_t B, int32_t T,
                                 int32_t n_act) {
  if (int s = check_options(opt)) return s;
  PK_CHECK_ARG(B >= 0 && T >= 1 && n_act >= 1, "need B >= 0, T >= 1, n_act >= 1");
  if (B == 0) return PK_OK;
  PK_CHECK_ARG(traj && coll && lower && upper && cost, "null buffer");
  PK_CHECK_CAP(B < (1LL << 31), "batch too large");
  sco_final_kernel<<<(unsigned)B, 128, 0, (cudaStream_t)stream>>>(traj, coll, lower, upper, cost, T, n_act,
                                                                  opt->w_smooth, opt->w_acc, opt->w_jerk,
                                                                  opt->w_limits, opt->w_collision_max);
  return cuda_status(cudaGetLastError(), "sco_final_kernel launch");
}

extern "C" int pk_sco_workspace_bytes(const pk_sco_options* opt, int64_t B, int32_t T, int32_t n_act,
                                      size_t* bytes) {
  if (int s = check_options(opt)) return s;
  PK_CHECK_ARG(bytes != nullptr, "null output");
  PK_CHECK_ARG(B >= 0 && T >= 0 && n_act >= 0, "negative extent");
  *bytes = ws_layout(opt, B, T, n_act).total;
  return PK_OK;
}

extern "C" int pk_sco_trajopt(void* stream, const pk_sco_options* opt, const float* init_trajs, const float* start,
                              const float* goal, const float* twists, const float* parent_tf,
                              const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                              const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                              const int32_t* parent_joint_indices, const float* link_spheres, const int32_t* pair_i,
                              const int32_t* pair_j, const float* world_spheres, const float* world_capsules,
                              const float* world_boxes, const float* world_halfspaces, const float* lower,
                              const float* upper, float* out_trajs, float* out_costs, void* workspace,
                              size_t workspace_bytes, int64_t B, int32_t T, int32_t n_act, int32_t n_joints,
                              int32_t n_links, int32_t S, int32_t P, int32_t Ms, int32_t Mc, int32_t Mb,
                              int32_t Mh) {
  if (int s = check_options(opt)) return s;
  if (int s = check_robot(n_act, n_joints, n_links, S, P)) return s;
  PK_CHECK_ARG(B >= 0 && T >= 2 && n_act >= 1, "need B >= 0, T >= 2, n_act >= 1");
  PK_CHECK_ARG(Ms >= 0 && Mc >= 0 && Mb >= 0 && Mh >= 0, "negative extent");
  PK_CHECK_CAP(B < (1LL << 31), "batch too large");
  if (B == 0) return PK_OK;
  PK_CHECK_ARG(init_trajs && start && goal && twists && parent_tf && parent_idx && act_idx && mimic_mul &&
                   mimic_off && mimic_act_idx && topo_inv && parent_joint_indices && lower && upper && out_trajs &&
                   out_costs,
               "null buffer");
  PK_CHECK_ARG(n_links * S == 0 || link_spheres, "null link_spheres");
  PK_CHECK_ARG(P == 0 || (pair_i && pair_j), "null pairs");
  PK_CHECK_ARG((Ms == 0 || world_spheres) && (Mc == 0 || world_capsules) && (Mb == 0 || world_boxes) &&
                   (Mh == 0 || world_halfspaces),
               "null world buffer");
  const WsLayout L = ws_layout(opt, B, T, n_act);
  PK_CHECK_ARG(workspace && workspace_bytes >= L.total, "workspace of %zu bytes needed (got %zu)", L.total,
               workspace_bytes);
  PK_CHECK_ARG((reinterpret_cast<uintptr_t>(workspace) & 255) == 0, "workspace must be 256-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  float* dist = reinterpret_cast<float*>(w + L.dist);
  float* jac = reinterpret_cast<float*>(w + L.jac);
  float* coll = reinterpret_cast<float*>(w + L.coll);
  float* hist = hist_in_smem(T, n_act, opt->m_lbfgs) ? nullptr : reinterpret_cast<float*>(w + L.hist);
  float* fd_cfg = opt->fd_eps > 0.f ? reinterpret_cast<float*>(w + L.fd_cfg) : nullptr;
  float* fd_dist = opt->fd_eps > 0.f ? reinterpret_cast<float*>(w + L.fd_dist) : nullptr;
  const long long C = B * (long long)T;

  sco_pin_kernel<<<ew_blocks(C * n_act), 256, 0, st>>>(init_trajs, start, goal, out_trajs, B, T, n_act);
  if (int s = cuda_status(cudaGetLastError(), "sco_pin_kernel launch")) return s;
  ScoLinArgs la = lin_args(opt, out_trajs, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off,
                           mimic_act_idx, topo_inv, parent_joint_indices, link_spheres, pair_i, pair_j,
                           world_spheres, world_capsules, world_boxes, world_halfspaces, C, n_act, n_joints,
                           n_links, S, P, Ms, Mc, Mb, Mh);
  const int nth = inner_threads(opt, T * n_act);
  float w_coll = opt->w_collision;
  for (int outer = 0; outer < opt->n_outer_iters; ++outer) {
    if (opt->fd_eps > 0.f) {
      sco_fd_configs_kernel<<<ew_blocks(C * (2 * n_act + 1) * n_act), 256, 0, st>>>(out_trajs, fd_cfg, C, n_act,
                                                                                    opt->fd_eps);
      if (int s = cuda_status(cudaGetLastError(), "sco_fd_configs_kernel launch")) return s;
      ScoLinArgs fa = la;
      fa.cfg = fd_cfg;
      fa.C = C * (2 * n_act + 1);
      fa.dist = fd_dist;
      if (int s = launch_linearize(fa, st)) return s;
      sco_fd_jac_kernel<<<ew_blocks(C * kScoG), 256, 0, st>>>(fd_dist, dist, jac, C, n_act, opt->fd_eps);
      if (int s = cuda_status(cudaGetLastError(), "sco_fd_jac_kernel launch")) return s;
    } else {
      ScoLinArgs a = la;
      a.dist = dist;
      a.jac = jac;
      if (int s = launch_linearize(a, st)) return s;
    }
    if (int s = launch_inner(inner_args(opt, out_trajs, dist, jac, lower, upper, start, goal, hist, w_coll, B, T,
                                        n_act),
                             nth, st))
      return s;
    w_coll = fminf(w_coll * opt->penalty_scale, opt->w_collision_max);
  }
  ScoLinArgs ca = la;
  ca.coll = coll;
  if (int s = launch_linearize(ca, st)) return s;
  sco_final_kernel<<<(unsigned)B, 128, 0, st>>>(out_trajs, coll, lower, upper, out_costs, T, n_act, opt->w_smooth,
                                                opt->w_acc, opt->w_jerk, opt->w_limits, opt->w_collision_max);
  return cuda_status(cudaGetLastError(), "sco_final_kernel launch");
}
