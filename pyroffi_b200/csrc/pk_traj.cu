// CHOMP trajectory cost and its hand-written adjoint (forward + backward).
//
// Cost of trajectory b (the reference's cost_fn,
// src/pyroffi/optimization_engines/_chomp_optimization.py:243-249):
//   J_b = w_smooth * smooth + w_limits * limits + w_coll * sum_t coll(q_bt)
// with the 4th-order acceleration / jerk smoothness (:93-110), squared limit
// violations (:113-121) and the collision hinge (:140-153): per waypoint,
// over the active self link pairs (min over the same sphere index s,
// src/pyroffi/collision/_robot_collision.py:796-828) and over every
// (link, obstacle) pair (min over the link's spheres, :830-895), the sum of
// max(0, margin - d)^2.
//
// B200 mapping: one block per trajectory, one thread per waypoint.  The
// backward pass recomputes the link poses (nothing is stored between the
// passes); a hinge term only sends force through the sphere that attains
// its minimum (the derivative of min), which is summed per link as a force
// F and a moment M = sum c x F; the joint gradient is then
// dJ/dq_a = z_a . (M - p_a x F) (revolute, z_a = R_a omega) or z_a . F
// (prismatic, z_a = R_a v) over the links below joint a, mapped to the
// actuated coordinates through the mimic multipliers.  A link's bounding
// sphere (centre B, radius R) gives the lower bound sdf_o(B) - R of every
// sphere-to-obstacle distance of the link, so (link, obstacle) pairs with
// bound >= margin are skipped exactly.  Smoothness and limit terms are
// computed by the same block from the trajectory tile in shared memory.
#include <float.h>

#include "pk_obstacles.cuh"

namespace pk {

struct TrajArgs {
  ModelArgs m;
  WorldArgs w;
  const float* traj;      // [B, T, n]
  const int* parent_joint;  // [N]
  const float* link_spheres;  // [N, S, 4]
  const int* pair_i;      // [P] active self link pairs
  const int* pair_j;
  const float* lower;
  const float* upper;
  float* cost;            // [B] or null
  float* grad;            // [B, T, n] or null
  float* wp_coll;         // [B, T] or null (unweighted collision cost per waypoint)
  long long B;
  int T, N, S, P;
  float margin, w_smooth, w_acc, w_jerk, w_limits, w_coll;
  const unsigned char* active;  // null, or trajectory b runs only when active[b % active_period]
  long long active_period;
};

// Lanes per waypoint: the world (link, obstacle) pairs and the self pairs of
// one waypoint are split over a group of TG lanes (TG = 2 or 4); its FK,
// force totals and joint gradient live once per waypoint in shared memory.
template <int MAXS, int TG>
__global__ void __launch_bounds__(64 * TG, 8 / TG) traj_cost_kernel(TrajArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (a.active && !a.active[blockIdx.x % a.active_period]) return;  // block-uniform: nothing is written
  JointTable& jt = *reinterpret_cast<JointTable*>(smem_raw);
  unsigned char* p = smem_raw + sizeof(JointTable);
  const int N = a.N, S = a.S, T = a.T, n = a.m.n_act, nj = a.m.n_joints;
  const int nth = blockDim.x, tid = threadIdx.x;
  const int ng = nth / TG, grp = tid / TG, gl = tid % TG;
  const unsigned gm = ((1u << TG) - 1u) << ((tid & 31) & ~(TG - 1));
  float4* lsph = reinterpret_cast<float4*>(p); p += sizeof(float4) * N * S;       // link spheres
  float4* lbnd = reinterpret_cast<float4*>(p); p += sizeof(float4) * N;           // link bounding spheres
  int* lpj = reinterpret_cast<int*>(p); p += sizeof(int) * ((N + 3) & ~3);        // parent joint (sorted), -1 base
  float* xs = reinterpret_cast<float*>(p); p += sizeof(float) * ((T * n + 3) & ~3);  // trajectory tile
  float* acc = reinterpret_cast<float*>(p); p += sizeof(float) * ((T * n + 3) & ~3);  // acc, then its adjoint
  float* red = reinterpret_cast<float*>(p); p += sizeof(float) * ((nth + 3) & ~3);
  float* wpc = reinterpret_cast<float*>(p); p += sizeof(float) * ((T + 3) & ~3);
  float* slots = reinterpret_cast<float*>(p); p += sizeof(float) * nj * 7 * ng;   // per waypoint group
  float* lt = reinterpret_cast<float*>(p); p += sizeof(float) * N * 6 * ng;       // link force / moment totals
  float* gq = reinterpret_cast<float*>(p); p += sizeof(float) * nj * ng;          // gradient per joint
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
  }
  const long long b = blockIdx.x;
  for (int i = tid; i < T * n; i += nth) xs[i] = a.traj[b * T * n + i];
  __syncthreads();
  for (int l = tid; l < N; l += nth) {
    float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
    int cnt = 0;
    for (int s = 0; s < S; ++s) {
      const float4 q = lsph[l * S + s];
      if (q.w < 0.f) continue;
      ++cnt;
      lo[0] = fminf(lo[0], q.x); hi[0] = fmaxf(hi[0], q.x);
      lo[1] = fminf(lo[1], q.y); hi[1] = fmaxf(hi[1], q.y);
      lo[2] = fminf(lo[2], q.z); hi[2] = fmaxf(hi[2], q.z);
    }
    const float cx = 0.5f * (lo[0] + hi[0]), cy = 0.5f * (lo[1] + hi[1]), cz = 0.5f * (lo[2] + hi[2]);
    float R = -1.f;
    for (int s = 0; s < S; ++s) {
      const float4 q = lsph[l * S + s];
      if (q.w < 0.f) continue;
      R = fmaxf(R, sqrtf((q.x - cx) * (q.x - cx) + (q.y - cy) * (q.y - cy) + (q.z - cz) * (q.z - cz)) + q.w);
    }
    // R < 0 marks a link without spheres; the slack keeps the cull conservative
    lbnd[l] = cnt ? make_float4(cx, cy, cz, R + 1e-4f + 1e-5f * fabsf(R)) : make_float4(0.f, 0.f, 0.f, -1.f);
  }
  __syncthreads();

  const bool want_grad = a.grad != nullptr;
  const float margin = a.margin;
  for (int t0 = 0; t0 < T; t0 += ng) {
    const int t = t0 + grp;
    if (t >= T) continue;  // the whole group skips
    const PoseSlots ps{slots + grp, ng};
    if (gl == 0) fk_thread(jt, [&](int i) { return xs[t * n + i]; }, ps);
    float* L = lt + grp;
    for (int i = gl; i < N * 6; i += TG) L[i * ng] = 0.f;
    __syncwarp(gm);
    float cw = 0.f;
    // world: (link, obstacle) hinge on the link's minimum sphere distance;
    // lane gl takes obstacles gl, gl + TG, ... of each kind
    for (int l = 0; l < N; ++l) {
      const float4 bl = lbnd[l];
      if (bl.w < 0.f) continue;
      const Pose Tl = lpj[l] < 0 ? pose_identity() : ps.load(lpj[l]);
      const float3 B = pose_apply(Tl, make_float3(bl.x, bl.y, bl.z));
      LinkSpheres<MAXS> ls;
      bool have = false;
      float3 F = make_float3(0.f, 0.f, 0.f), Mo = make_float3(0.f, 0.f, 0.f);
      // narrow phase of obstacle m: the link's minimum sphere distance, its
      // hinge and the force at the sphere that attains it
      auto narrow = [&](int m, auto kind) {
        constexpr int K = decltype(kind)::value;
        if (!have) {
#pragma unroll
          for (int q = 0; q < MAXS / 2; ++q) {
            const float4 a0 = (2 * q < S) ? lsph[l * S + 2 * q] : make_float4(0.f, 0.f, 0.f, -1.f);
            const float4 a1 = (2 * q + 1 < S) ? lsph[l * S + 2 * q + 1] : make_float4(0.f, 0.f, 0.f, -1.f);
            const float3 w0 = pose_apply(Tl, make_float3(a0.x, a0.y, a0.z));
            const float3 w1 = pose_apply(Tl, make_float3(a1.x, a1.y, a1.z));
            ls.x[q] = make_float2(w0.x, w1.x); ls.y[q] = make_float2(w0.y, w1.y); ls.z[q] = make_float2(w0.z, w1.z);
            ls.r[q] = make_float2(a0.w < 0.f ? -1e30f : a0.w, a1.w < 0.f ? -1e30f : a1.w);
          }
          have = true;
        }
        float dmin = FLT_MAX;
        int arg = -1;
#pragma unroll
        for (int q = 0; q < MAXS / 2; ++q) {
          float2 d;
          if constexpr (K == 0) {
            d = ls.sphere_dist2(q, ob.sph[m]);
          } else if constexpr (K == 2) {
            d = ls.box_dist2(q, ob.box + 15 * (m - ob.Ms - ob.Mc));
          } else {
            d.x = obstacle_dist<K>(ob, m, make_float3(ls.x[q].x, ls.y[q].x, ls.z[q].x), ls.r[q].x);
            d.y = obstacle_dist<K>(ob, m, make_float3(ls.x[q].y, ls.y[q].y, ls.z[q].y), ls.r[q].y);
          }
          if (d.x < dmin) { dmin = d.x; arg = 2 * q; }
          if (d.y < dmin) { dmin = d.y; arg = 2 * q + 1; }
        }
        // padded spheres read about 1e30: a link of padding only has no hit
        if (!(dmin < margin)) return;
        const float v = margin - dmin;
        cw += v * v;
        if (want_grad) {
          float3 c = make_float3(0.f, 0.f, 0.f), g;
          float rr = 0.f;
#pragma unroll
          for (int s = 0; s < MAXS; ++s)
            if (s == arg) { c = make_float3(ls.X(s), ls.Y(s), ls.Z(s)); rr = ls.R(s); }
          obstacle_dist_grad<K>(ob, m, c, rr, g);
          const float k = -2.f * v;  // d(v^2)/dd
          const float3 f = make_float3(k * g.x, k * g.y, k * g.z);
          F.x += f.x; F.y += f.y; F.z += f.z;
          const float3 cm = cross3(c, f);
          Mo.x += cm.x; Mo.y += cm.y; Mo.z += cm.z;
        }
      };
      for_each_near_obstacle(ob, B, bl.w, margin, gl, TG, narrow);
      if (want_grad) {
#pragma unroll
        for (int o = 1; o < TG; o <<= 1) {
          F.x += __shfl_xor_sync(gm, F.x, o); F.y += __shfl_xor_sync(gm, F.y, o); F.z += __shfl_xor_sync(gm, F.z, o);
          Mo.x += __shfl_xor_sync(gm, Mo.x, o); Mo.y += __shfl_xor_sync(gm, Mo.y, o); Mo.z += __shfl_xor_sync(gm, Mo.z, o);
        }
        if (gl == 0) {
          L[(l * 6 + 0) * ng] += F.x; L[(l * 6 + 1) * ng] += F.y; L[(l * 6 + 2) * ng] += F.z;
          L[(l * 6 + 3) * ng] += Mo.x; L[(l * 6 + 4) * ng] += Mo.y; L[(l * 6 + 5) * ng] += Mo.z;
        }
      }
    }
    __syncwarp(gm);
    // self: active link pairs, min over the same sphere index s; lane gl takes
    // pairs gl, gl + TG, ... and the lanes write their forces in turn
    for (int p0 = 0; p0 < a.P; p0 += TG) {
      const int pi = p0 + gl;
      bool hit = false;
      int li = 0, lj = 0;
      float3 f = make_float3(0.f, 0.f, 0.f), ma = f, mb = f;
      if (pi < a.P) {
        li = a.pair_i[pi];
        lj = a.pair_j[pi];
        const bool ok = !(li < 0 || lj < 0 || li >= N || lj >= N) && lbnd[li].w >= 0.f && lbnd[lj].w >= 0.f;
        if (ok) {
          const float4 bi = lbnd[li], bj = lbnd[lj];
          const Pose Ti = lpj[li] < 0 ? pose_identity() : ps.load(lpj[li]);
          const Pose Tj = lpj[lj] < 0 ? pose_identity() : ps.load(lpj[lj]);
          const float3 Bi = pose_apply(Ti, make_float3(bi.x, bi.y, bi.z));
          const float3 Bj = pose_apply(Tj, make_float3(bj.x, bj.y, bj.z));
          const float bx = Bi.x - Bj.x, by = Bi.y - Bj.y, bz = Bi.z - Bj.z;
          const float rb = bi.w + bj.w + margin;
          if (bx * bx + by * by + bz * bz < rb * fabsf(rb)) {
            float dmin = FLT_MAX;
            float3 ca = make_float3(0.f, 0.f, 0.f), cb = ca;
            for (int s = 0; s < S; ++s) {
              const float4 qa = lsph[li * S + s], qb = lsph[lj * S + s];
              if (qa.w < 0.f || qb.w < 0.f) continue;
              const float3 pa = pose_apply(Ti, make_float3(qa.x, qa.y, qa.z));
              const float3 pb = pose_apply(Tj, make_float3(qb.x, qb.y, qb.z));
              const float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
              const float d = sqrtf(dx * dx + dy * dy + dz * dz) - (qa.w + qb.w);
              if (d < dmin) { dmin = d; ca = pa; cb = pb; }
            }
            if (dmin < margin) {
              const float v = margin - dmin;
              cw += v * v;
              hit = true;
              const float dx = ca.x - cb.x, dy = ca.y - cb.y, dz = ca.z - cb.z;
              const float nrm = sqrtf(dx * dx + dy * dy + dz * dz);
              const float k = nrm > 0.f ? -2.f * v / nrm : 0.f;
              f = make_float3(k * dx, k * dy, k * dz);  // force on sphere a; -f on sphere b
              ma = cross3(ca, f);
              mb = cross3(cb, f);
            }
          }
        }
      }
      if (want_grad) {
        for (int r = 0; r < TG; ++r) {
          if (gl == r && hit) {
            L[(li * 6 + 0) * ng] += f.x; L[(li * 6 + 1) * ng] += f.y; L[(li * 6 + 2) * ng] += f.z;
            L[(li * 6 + 3) * ng] += ma.x; L[(li * 6 + 4) * ng] += ma.y; L[(li * 6 + 5) * ng] += ma.z;
            L[(lj * 6 + 0) * ng] -= f.x; L[(lj * 6 + 1) * ng] -= f.y; L[(lj * 6 + 2) * ng] -= f.z;
            L[(lj * 6 + 3) * ng] -= mb.x; L[(lj * 6 + 4) * ng] -= mb.y; L[(lj * 6 + 5) * ng] -= mb.z;
          }
          __syncwarp(gm);
        }
      }
    }
#pragma unroll
    for (int o = 1; o < TG; o <<= 1) cw += __shfl_xor_sync(gm, cw, o);
    if (gl == 0) {
      wpc[t] = cw;
      if (a.wp_coll) a.wp_coll[b * T + t] = cw;
      if (want_grad) {
        float* G = gq + grp;
        for (int j = 0; j < nj; ++j) G[j * ng] = 0.f;
        // every link's (F, M) acts on all joints from its parent joint to the root
        for (int l = 0; l < N; ++l) {
          const float3 F = make_float3(L[(l * 6 + 0) * ng], L[(l * 6 + 1) * ng], L[(l * 6 + 2) * ng]);
          const float3 Mo = make_float3(L[(l * 6 + 3) * ng], L[(l * 6 + 4) * ng], L[(l * 6 + 5) * ng]);
          if (F.x == 0.f && F.y == 0.f && F.z == 0.f && Mo.x == 0.f && Mo.y == 0.f && Mo.z == 0.f) continue;
          for (int j = lpj[l]; j >= 0; j = jt.psorted[j]) {
            const int kind = jt.kind[j];
            if (kind == kFixed) continue;
            const Pose Tj = ps.load(j);
            const float* tw = jt.tw[j];
            const float3 w = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z, make_float3(tw[3], tw[4], tw[5]));
            const float3 vv = quat_rotate(Tj.w, Tj.x, Tj.y, Tj.z, make_float3(tw[0], tw[1], tw[2]));
            // point velocity under dq_j: w x (c - p_j) + (R v); dJ/dq_j = sum F . that
            const float3 pxF = cross3(make_float3(Tj.tx, Tj.ty, Tj.tz), F);
            G[j * ng] += w.x * (Mo.x - pxF.x) + w.y * (Mo.y - pxF.y) + w.z * (Mo.z - pxF.z) +
                         vv.x * F.x + vv.y * F.y + vv.z * F.z;
          }
        }
        float* grow = a.grad + (b * T + t) * n;
        for (int c = 0; c < n; ++c) grow[c] = 0.f;
        for (int j = 0; j < nj; ++j) {
          const int src = jt.src[j];
          if (src >= 0) grow[src] += a.w_coll * jt.mul[j] * G[j * ng];
        }
      }
    }
    __syncwarp(gm);
  }
  __syncthreads();

  // smoothness: acc_k = sum_i c_i x_{k+i} / 12,  jerk_k = acc_{k+1} - acc_k
  const int K = T - 4;
  const float cst[5] = {-1.f / 12.f, 16.f / 12.f, -30.f / 12.f, 16.f / 12.f, -1.f / 12.f};
  for (int i = tid; i < K * n; i += nth) {
    const int k = i / n, d = i - k * n;
    float v = 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q) v += cst[q] * xs[(k + q) * n + d];
    acc[i] = v;
  }
  __syncthreads();
  float part = 0.f;
  for (int i = tid; i < K * n; i += nth) {
    const int k = i / n;
    const float v = acc[i];
    part += a.w_smooth * a.w_acc * v * v;
    if (k + 1 < K) {
      const float j = acc[i + n] - v;
      part += a.w_smooth * a.w_jerk * j * j;
    }
  }
  for (int i = tid; i < T * n; i += nth) {
    const int d = i % n;
    const float x = xs[i];
    const float vv = fmaxf(0.f, x - a.upper[d]) + fmaxf(0.f, a.lower[d] - x);
    part += a.w_limits * vv * vv;
  }
  for (int t = tid; t < T; t += nth) part += a.w_coll * wpc[t];
  red[tid] = part;
  __syncthreads();
  if (tid == 0 && a.cost) {
    float s = 0.f;
    for (int i = 0; i < nth; ++i) s += red[i];  // fixed order: deterministic
    a.cost[b] = s;
  }
  if (!want_grad) return;
  // adjoint of the smoothness: g_acc_k = 2 w_acc acc_k + 2 w_jerk (jerk_{k-1} - jerk_k)
  __syncthreads();
  float ga[8];
  int cnt = 0;
  for (int i = tid; i < K * n && cnt < 8; i += nth, ++cnt) {
    const int k = i / n;
    float g = 2.f * a.w_acc * acc[i];
    if (k + 1 < K) g -= 2.f * a.w_jerk * (acc[i + n] - acc[i]);
    if (k >= 1) g += 2.f * a.w_jerk * (acc[i] - acc[i - n]);
    ga[cnt] = g;
  }
  __syncthreads();
  cnt = 0;
  for (int i = tid; i < K * n && cnt < 8; i += nth, ++cnt) acc[i] = ga[cnt];
  __syncthreads();
  for (int i = tid; i < T * n; i += nth) {
    const int t = i / n, d = i - t * n;
    float g = 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int k = t - q;
      if (k >= 0 && k < K) g += cst[q] * acc[k * n + d];
    }
    const float x = xs[i];
    const float gl = 2.f * fmaxf(0.f, x - a.upper[d]) - 2.f * fmaxf(0.f, a.lower[d] - x);
    a.grad[b * T * n + i] += a.w_smooth * g + a.w_limits * gl;
  }
}

static size_t traj_smem(const TrajArgs& a, int nth, int TG) {
  size_t s = sizeof(JointTable) + sizeof(float4) * a.N * a.S + sizeof(float4) * a.N + sizeof(int) * ((a.N + 3) & ~3) +
             2 * sizeof(float) * ((a.T * a.m.n_act + 3) & ~3) + sizeof(float) * ((nth + 3) & ~3) +
             sizeof(float) * ((a.T + 3) & ~3) +
             sizeof(float) * (size_t)(nth / TG) * (a.m.n_joints * 7 + a.N * 6 + a.m.n_joints);
  s = (s + 15) & ~size_t(15);
  return s + sizeof(float) * a.w.smem_floats();
}

}  // namespace pk

using namespace pk;

extern "C" int pk_traj_cost_grad(void* stream, const pk_traj_options* opt, const float* traj,
                                 const float* twists, const float* parent_tf, const int32_t* parent_idx,
                                 const int32_t* act_idx, const float* mimic_mul, const float* mimic_off,
                                 const int32_t* mimic_act_idx, const int32_t* topo_inv,
                                 const int32_t* parent_joint_indices, const float* link_spheres,
                                 const int32_t* pair_i, const int32_t* pair_j, const float* world_spheres,
                                 const float* world_capsules, const float* world_boxes,
                                 const float* world_halfspaces, const float* lower, const float* upper,
                                 float* cost, float* grad, float* wp_coll, int64_t B, int32_t T, int32_t n_act,
                                 int32_t n_joints, int32_t n_links, int32_t S, int32_t P, int32_t Ms, int32_t Mc,
                                 int32_t Mb, int32_t Mh) {
  PK_CHECK_ARG(opt != nullptr, "null options");
  PK_CHECK_ARG(B >= 0 && T >= 0 && n_act >= 0 && n_links >= 0 && S >= 0 && P >= 0, "negative extent");
  PK_CHECK_CAP(n_joints <= PK_MAX_JOINTS, "n_joints=%d exceeds %d", n_joints, PK_MAX_JOINTS);
  PK_CHECK_CAP(S <= 32, "at most 32 spheres per link (got %d)", S);
  PK_CHECK_ARG(T >= 5, "the 4th-order smoothness stencil needs T >= 5 waypoints (got %d)", T);
  if (B == 0) return PK_OK;
  PK_CHECK_ARG(traj && twists && parent_tf && parent_idx && act_idx && mimic_mul && mimic_off && mimic_act_idx &&
                   topo_inv && parent_joint_indices && lower && upper,
               "null buffer");
  PK_CHECK_ARG(n_links * S == 0 || link_spheres, "null link_spheres");
  PK_CHECK_ARG(P == 0 || (pair_i && pair_j), "null pairs");
  PK_CHECK_ARG((Ms == 0 || world_spheres) && (Mc == 0 || world_capsules) && (Mb == 0 || world_boxes) &&
                   (Mh == 0 || world_halfspaces),
               "null world buffer");
  PK_CHECK_ARG(cost || grad || wp_coll, "no output requested");
  TrajArgs a;
  a.m = ModelArgs{twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx, topo_inv,
                  n_joints, n_act};
  a.w = WorldArgs{world_spheres, world_capsules, world_boxes, world_halfspaces, Ms, Mc, Mb, Mh};
  a.traj = traj; a.parent_joint = parent_joint_indices; a.link_spheres = link_spheres;
  a.pair_i = pair_i; a.pair_j = pair_j; a.lower = lower; a.upper = upper;
  a.cost = cost; a.grad = grad; a.wp_coll = wp_coll;
  a.B = B; a.T = T; a.N = n_links; a.S = S; a.P = P;
  a.margin = opt->margin; a.w_smooth = opt->w_smooth; a.w_acc = opt->w_acc; a.w_jerk = opt->w_jerk;
  a.w_limits = opt->w_limits; a.w_coll = opt->w_coll;
  PK_CHECK_ARG(opt->active == nullptr || opt->active_period > 0, "active_period must be positive with an active mask");
  a.active = opt->active;
  a.active_period = opt->active ? opt->active_period : 1;
  // lanes per waypoint: 4 when a waypoint has much world to test or the
  // batch is too small to fill the GPU with 2-lane blocks, else 2
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int TG = (Ms + Mc + Mb + Mh >= 1024 || B <= 2LL * sms) ? 4 : 2;
  int ng = 8;  // waypoint groups per block (TG lanes each)
  while (ng < T && ng < 64) ng *= 2;
  const int nth = ng * TG;
  PK_CHECK_CAP((size_t)(T - 4) * n_act <= (size_t)8 * nth, "trajectory too long for one block (T*n_act=%d)", T * n_act);
  const size_t smem = traj_smem(a, nth, TG);
  PK_CHECK_CAP(smem <= 200 * 1024, "trajectory working set (%zu B of shared memory) too large", smem);
  PK_CHECK_CAP(B < (1LL << 31), "batch too large");
  auto kern = (S <= 8)    ? (TG == 4 ? traj_cost_kernel<8, 4> : traj_cost_kernel<8, 2>)
              : (S <= 16) ? (TG == 4 ? traj_cost_kernel<16, 4> : traj_cost_kernel<16, 2>)
                          : (TG == 4 ? traj_cost_kernel<32, 4> : traj_cost_kernel<32, 2>);
  if (int s = set_smem_limit((const void*)kern, smem)) return s;
  kern<<<(unsigned)B, nth, smem, (cudaStream_t)stream>>>(a);
  return cuda_status(cudaGetLastError(), "traj_cost_kernel launch");
}
