// World-obstacle staging and per-obstacle signed distance dispatch.
//
// Obstacle arrays use the reference's world layout
// (src/pyroffi/collision/_cuda_collision.py:98-168): spheres [Ms,4]
// (x,y,z,r), capsules [Mc,7] (p1,p2,r), boxes [Mb,15] (centre, axis
// columns, half-lengths), halfspaces [Mh,6] (normal, point).  The obstacle
// index m runs over spheres, capsules, boxes, halfspaces in that order.
#pragma once

#include "pk_common.cuh"

namespace pk {

// 1/sqrt(x) by the PTX approximate reciprocal square root (MUFU; a few ulp).
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// sqrt(x) for x >= 0 as x * rsqrt(x + 1e-30): the 1e-30 keeps x = 0 finite
// (giving 0) and is below FP32 resolution for any x above 1e-23.
__device__ __forceinline__ float sqrt_fast(float x) { return x * rsqrt_approx(x + 1e-30f); }

struct WorldArgs {
  const float* spheres;
  const float* capsules;
  const float* boxes;
  const float* halfspaces;
  int Ms, Mc, Mb, Mh;
  __host__ __device__ int total() const { return Ms + Mc + Mb + Mh; }
  // floats needed to stage everything in shared memory: spheres, capsules,
  // boxes, halfspaces, each array starting on a 16-byte boundary
  __host__ __device__ size_t smem_floats() const {
    return (size_t)Ms * 4 + round4((size_t)Mc * 7) + round4((size_t)Mb * 15) + round4((size_t)Mh * 6);
  }
  __host__ __device__ static size_t round4(size_t v) { return (v + 3) & ~size_t(3); }
};

struct ObsView {
  const float4* sph;
  const float* cap;
  const float* box;
  const float* hs;
  int Ms, Mc, Mb, Mh;
};

// State of the bounded wait of stage_world in the kernels of this source
// file (one copy per file; the pk_stage_wait_* entry points visit them all):
//   gave_up    blocks whose first wait for the TMA copy ran out of time;
//   abandoned  of those, blocks whose second wait ran out too, so that they
//              finished with a copy possibly still in flight;
//   force      test hook: when set, no copy is issued and every wait runs out;
//   limit_ns   the time limit of each wait, by %globaltimer (default 1 s).
struct StageWaitState {
  unsigned int gave_up;
  unsigned int abandoned;
  unsigned int force;
  unsigned int pad;
  unsigned long long limit_ns;
};
static __device__ StageWaitState g_stage_wait = {0u, 0u, 0u, 0u, 1000000000ull};

// Host side: this file's hooks (StageWaitHooks) for its own g_stage_wait.
namespace {
int stage_wait_read(unsigned long long* gave_up, unsigned long long* abandoned) {
  StageWaitState v{};
  if (int s = cuda_status(cudaMemcpyFromSymbol(&v, g_stage_wait, sizeof(v)), "stage wait state")) return s;
  *gave_up += v.gave_up;
  *abandoned += v.abandoned;
  return PK_OK;
}
int stage_wait_reset() {
  const unsigned int z[2] = {0u, 0u};
  return cuda_status(cudaMemcpyToSymbol(g_stage_wait, z, sizeof(z)), "stage wait reset");
}
int stage_wait_set(unsigned int force, unsigned long long limit_ns) {
  if (int s = cuda_status(cudaMemcpyToSymbol(g_stage_wait, &force, sizeof(force),
                                             offsetof(StageWaitState, force)), "stage wait force"))
    return s;
  return cuda_status(cudaMemcpyToSymbol(g_stage_wait, &limit_ns, sizeof(limit_ns),
                                        offsetof(StageWaitState, limit_ns)), "stage wait limit");
}
[[maybe_unused]] const int kStageWaitHooks =
    register_stage_wait_hooks(StageWaitHooks{stage_wait_read, stage_wait_reset, stage_wait_set});
}  // namespace

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Copies the obstacle arrays into shared memory at `dst` (16-byte aligned),
// each array starting on a 16-byte boundary; called by every thread of the
// block, and the caller synchronises afterwards.  The 16-byte-aligned bulk of
// each array goes through the TMA bulk-copy engine: one thread issues
// cp.async.bulk global -> shared with the completion counted in bytes on an
// mbarrier, and every thread waits on that barrier for at most
// g_stage_wait.limit_ns.  A thread whose wait runs out counts the block in
// gave_up (thread 0 does), waits once more with the same limit, and then
// loads the bulk with plain loads itself, so this block's data is right
// either way (a copy that lands late writes the same bytes).  If the second
// wait runs out too, the block counts itself in `abandoned` and finishes
// with the copy possibly still in flight, which may then land in the shared
// memory of a later block: pk_stage_wait_timeouts reports PK_ERR_TIMEOUT,
// and the outputs of that launch and of later ones on the device are not to
// be trusted.  With g_stage_wait.force set, no copy is issued (nothing is in
// flight), the first wait runs out, and the block takes the plain-load path
// without the second wait.  An array whose source is not 16-byte aligned,
// and the bytes past the last 16-byte multiple, are copied with plain loads.
// sphere_slots (>= Ms; -1: Ms) float4 slots are reserved for the spheres,
// so a caller can pad them; the other arrays follow the reserved slots.
__device__ inline ObsView stage_world(const WorldArgs& w, float* dst, int sphere_slots = -1) {
  __shared__ __align__(8) unsigned long long s_bar;
  const float* src[4] = {w.spheres, w.capsules, w.boxes, w.halfspaces};
  const int nf[4] = {w.Ms * 4, w.Mc * 7, w.Mb * 15, w.Mh * 6};
  float* d[4];
  unsigned bulk[4];
  unsigned total = 0;
  float* q = dst;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d[k] = q;
    q += (k == 0 && sphere_slots > w.Ms) ? 4 * (size_t)sphere_slots : WorldArgs::round4((size_t)nf[k]);
    const bool aligned = nf[k] > 0 && (reinterpret_cast<uintptr_t>(src[k]) & 15) == 0;
    bulk[k] = aligned ? ((unsigned)nf[k] * 4u) & ~15u : 0u;
    total += bulk[k];
  }
  const int tid = threadIdx.x, nth = blockDim.x;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    for (int i = (int)(bulk[k] / 4) + tid; i < nf[k]; i += nth) d[k][i] = src[k][i];
  if (total > 0) {
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&s_bar);
    const bool force = *(volatile const unsigned int*)&g_stage_wait.force != 0u;
    const unsigned long long limit = *(volatile const unsigned long long*)&g_stage_wait.limit_ns;
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0 && !force) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total) : "memory");
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (bulk[k])
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  (unsigned)__cvta_generic_to_shared(d[k])),
              "l"(src[k]), "r"(bulk[k]), "r"(bar)
              : "memory");
    }
    auto wait = [&]() {
      unsigned done = 0;
      const unsigned long long t0 = global_ns();
      for (;;) {
        asm volatile(
            "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], 0;\n selp.u32 %0, 1, 0, P;\n}"
            : "=r"(done)
            : "r"(bar)
            : "memory");
        if (done || global_ns() - t0 > limit) break;
      }
      return done != 0;
    };
    if (!wait()) {
      if (tid == 0) atomicAdd(&g_stage_wait.gave_up, 1u);
      if (!force && !wait() && tid == 0) atomicAdd(&g_stage_wait.abandoned, 1u);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        for (int i = tid; i < (int)(bulk[k] / 4); i += nth) d[k][i] = src[k][i];
    }
  }
  ObsView v;
  v.sph = reinterpret_cast<const float4*>(d[0]);
  v.cap = d[1];
  v.box = d[2];
  v.hs = d[3];
  v.Ms = w.Ms; v.Mc = w.Mc; v.Mb = w.Mb; v.Mh = w.Mh;
  return v;
}

// A link's spheres in the world frame, held in register pairs (spheres 2q,
// 2q + 1) so the sphere-obstacle loops run on packed FP32x2 arithmetic.
// Padded spheres carry radius -1e30: their distances read about 1e30 and
// never win a minimum.  Each pair method computes, element by element, the
// same operations as its scalar counterpart.
template <int MAXS>
struct LinkSpheres {
  static_assert(MAXS % 2 == 0, "spheres come in pairs");
  float2 x[MAXS / 2], y[MAXS / 2], z[MAXS / 2], r[MAXS / 2];
  __device__ __forceinline__ float X(int s) const { return (s & 1) ? x[s >> 1].y : x[s >> 1].x; }
  __device__ __forceinline__ float Y(int s) const { return (s & 1) ? y[s >> 1].y : y[s >> 1].x; }
  __device__ __forceinline__ float Z(int s) const { return (s & 1) ? z[s >> 1].y : z[s >> 1].x; }
  __device__ __forceinline__ float R(int s) const { return (s & 1) ? r[s >> 1].y : r[s >> 1].x; }
  // squared distance of spheres 2q, 2q + 1 to the point -(npx, npy, npz)
  __device__ __forceinline__ float2 sq_dist2(int q, float2 npx, float2 npy, float2 npz) const {
    const float2 dx = __fadd2_rn(x[q], npx), dy = __fadd2_rn(y[q], npy), dz = __fadd2_rn(z[q], npz);
    float2 d2 = __fmul2_rn(dx, dx);
    d2 = __ffma2_rn(dy, dy, d2);
    return __ffma2_rn(dz, dz, d2);
  }
  // |c_s - p| - (r_s + rp) with sqrt_fast
  __device__ __forceinline__ float2 sphere_dist2_fast(int q, float2 npx, float2 npy, float2 npz, float2 rp) const {
    const float2 d2 = sq_dist2(q, npx, npy, npz);
    const float2 e = __fadd2_rn(d2, make_float2(1e-30f, 1e-30f));
    const float2 len = __fmul2_rn(d2, make_float2(rsqrt_approx(e.x), rsqrt_approx(e.y)));
    return __ffma2_rn(__fadd2_rn(r[q], rp), make_float2(-1.f, -1.f), len);
  }
  // d_sphere_sphere against world sphere o (IEEE sqrt)
  __device__ __forceinline__ float2 sphere_dist2(int q, float4 o) const {
    const float2 d2 = sq_dist2(q, make_float2(-o.x, -o.x), make_float2(-o.y, -o.y), make_float2(-o.z, -o.z));
    const float2 len = make_float2(sqrtf(d2.x), sqrtf(d2.y));
    return __ffma2_rn(__fadd2_rn(r[q], make_float2(o.w, o.w)), make_float2(-1.f, -1.f), len);
  }
  // d_sphere_box against box b (centre, axis columns, half-lengths; IEEE sqrt)
  __device__ __forceinline__ float2 box_dist2(int q, const float* b) const {
    const float2 dx = __fadd2_rn(x[q], make_float2(-b[0], -b[0]));
    const float2 dy = __fadd2_rn(y[q], make_float2(-b[1], -b[1]));
    const float2 dz = __fadd2_rn(z[q], make_float2(-b[2], -b[2]));
    float2 qv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float2 p = __fmul2_rn(dx, make_float2(b[3 + 3 * i], b[3 + 3 * i]));
      p = __ffma2_rn(dy, make_float2(b[4 + 3 * i], b[4 + 3 * i]), p);
      p = __ffma2_rn(dz, make_float2(b[5 + 3 * i], b[5 + 3 * i]), p);
      qv[i] = make_float2(fabsf(p.x) - b[12 + i], fabsf(p.y) - b[12 + i]);
    }
    const float2 m1 = make_float2(fmaxf(qv[0].x, 0.f), fmaxf(qv[0].y, 0.f));
    const float2 m2 = make_float2(fmaxf(qv[1].x, 0.f), fmaxf(qv[1].y, 0.f));
    const float2 m3 = make_float2(fmaxf(qv[2].x, 0.f), fmaxf(qv[2].y, 0.f));
    float2 s2 = __fmul2_rn(m1, m1);
    s2 = __ffma2_rn(m2, m2, s2);
    s2 = __ffma2_rn(m3, m3, s2);
    const float2 out = make_float2(sqrtf(s2.x), sqrtf(s2.y));
    const float2 in = make_float2(fminf(fmaxf(fmaxf(qv[0].x, qv[1].x), qv[2].x), 0.f),
                                  fminf(fmaxf(fmaxf(qv[0].y, qv[1].y), qv[2].y), 0.f));
    return __ffma2_rn(r[q], make_float2(-1.f, -1.f), __fadd2_rn(out, in));
  }
};

// Obstacle kind as a type (0 sphere, 1 capsule, 2 box, 3 halfspace), for
// callers that know it at compile time.
template <int K>
struct ObsKind {
  static constexpr int value = K;
};

// Signed distance from sphere (c, r) to obstacle m (exact IEEE sqrt).  KIND
// is m's kind when the caller knows it, -1 to dispatch on m.
template <int KIND = -1>
__device__ __forceinline__ float obstacle_dist(const ObsView& o, int m, float3 c, float r) {
  if (KIND == 0 || (KIND < 0 && m < o.Ms)) {
    const float4 s = o.sph[m];
    return d_sphere_sphere(c, r, s.x, s.y, s.z, s.w);
  }
  m -= o.Ms;
  if (KIND == 1 || (KIND < 0 && m < o.Mc)) return d_sphere_capsule(c, r, o.cap + 7 * m);
  m -= o.Mc;
  if (KIND == 2 || (KIND < 0 && m < o.Mb)) return d_sphere_box(c, r, o.box + 15 * m);
  m -= o.Mb;
  return d_sphere_halfspace(c, r, o.hs + 6 * m);
}

// Signed distance from sphere (c, r) to obstacle m and its gradient w.r.t. c
// (KIND as for obstacle_dist).
template <int KIND = -1>
__device__ inline float obstacle_dist_grad(const ObsView& o, int m, float3 c, float r, float3& g) {
  if (KIND == 0 || (KIND < 0 && m < o.Ms)) {
    const float4 s = o.sph[m];
    const float dx = c.x - s.x, dy = c.y - s.y, dz = c.z - s.z;
    const float n = sqrtf(dx * dx + dy * dy + dz * dz);
    const float inv = n > 0.f ? 1.f / n : 0.f;
    g = make_float3(dx * inv, dy * inv, dz * inv);
    return n - (r + s.w);
  }
  m -= o.Ms;
  if (KIND == 1 || (KIND < 0 && m < o.Mc)) {
    const float* cp = o.cap + 7 * m;
    const float vx = cp[3] - cp[0], vy = cp[4] - cp[1], vz = cp[5] - cp[2];
    const float len2 = vx * vx + vy * vy + vz * vz;
    float t = 0.f;
    if (len2 > 1e-12f) t = fmaxf(0.f, fminf(1.f, ((c.x - cp[0]) * vx + (c.y - cp[1]) * vy + (c.z - cp[2]) * vz) / len2));
    const float dx = c.x - (cp[0] + t * vx), dy = c.y - (cp[1] + t * vy), dz = c.z - (cp[2] + t * vz);
    const float n = sqrtf(dx * dx + dy * dy + dz * dz);
    const float inv = n > 0.f ? 1.f / n : 0.f;
    g = make_float3(dx * inv, dy * inv, dz * inv);
    return n - (r + cp[6]);
  }
  m -= o.Mc;
  if (KIND == 2 || (KIND < 0 && m < o.Mb)) {
    const float* b = o.box + 15 * m;
    const float dx = c.x - b[0], dy = c.y - b[1], dz = c.z - b[2];
    const float l[3] = {dx * b[3] + dy * b[4] + dz * b[5], dx * b[6] + dy * b[7] + dz * b[8],
                        dx * b[9] + dy * b[10] + dz * b[11]};
    float q[3], gl[3];
    for (int i = 0; i < 3; ++i) q[i] = fabsf(l[i]) - b[12 + i];
    const float m0 = fmaxf(q[0], 0.f), m1 = fmaxf(q[1], 0.f), m2 = fmaxf(q[2], 0.f);
    const float out = sqrtf(m0 * m0 + m1 * m1 + m2 * m2);
    const float qmax = fmaxf(fmaxf(q[0], q[1]), q[2]);
    if (out > 0.f) {
      gl[0] = copysignf(m0 / out, l[0]); gl[1] = copysignf(m1 / out, l[1]); gl[2] = copysignf(m2 / out, l[2]);
    } else {
      const int im = (q[0] >= q[1] && q[0] >= q[2]) ? 0 : (q[1] >= q[2] ? 1 : 2);
      gl[0] = gl[1] = gl[2] = 0.f;
      gl[im] = copysignf(1.f, l[im]);
    }
    g = make_float3(gl[0] * b[3] + gl[1] * b[6] + gl[2] * b[9], gl[0] * b[4] + gl[1] * b[7] + gl[2] * b[10],
                    gl[0] * b[5] + gl[1] * b[8] + gl[2] * b[11]);
    return out + fminf(qmax, 0.f) - r;
  }
  m -= o.Mb;
  const float* h = o.hs + 6 * m;
  g = make_float3(h[0], h[1], h[2]);
  return (c.x - h[3]) * h[0] + (c.y - h[4]) * h[1] + (c.z - h[5]) * h[2] - r;
}

// Broad phase: may the ball (B, R) come within `margin` of obstacle m (index
// over spheres, capsules, boxes, halfspaces in that order)?  The ball bounds a
// group of spheres, so its distance bounds theirs from below and a `false`
// means every one of them is at least `margin` from the obstacle.  Squared
// lengths instead of square roots; the caller's ball carries the slack that
// covers the rounding.  KIND is the obstacle's kind (0-3) when the caller
// knows it, -1 to dispatch on m.
template <int KIND = -1>
__device__ __forceinline__ bool obstacle_near(const ObsView& ob, int m, float3 B, float R, float margin) {
  const float Rm = R + margin;
  if (KIND == 0 || (KIND < 0 && m < ob.Ms)) {
    const float4 o = ob.sph[m];
    const float dx = B.x - o.x, dy = B.y - o.y, dz = B.z - o.z;
    const float rr = Rm + o.w;
    return dx * dx + dy * dy + dz * dz < rr * fabsf(rr);
  }
  m -= ob.Ms;
  if (KIND == 1 || (KIND < 0 && m < ob.Mc)) {
    const float* cp = ob.cap + 7 * m;
    const float vx = cp[3] - cp[0], vy = cp[4] - cp[1], vz = cp[5] - cp[2];
    const float len2 = vx * vx + vy * vy + vz * vz;
    float t = 0.f;
    if (len2 > 1e-12f)
      t = fmaxf(0.f, fminf(1.f, ((B.x - cp[0]) * vx + (B.y - cp[1]) * vy + (B.z - cp[2]) * vz) / len2));
    const float dx = B.x - (cp[0] + t * vx), dy = B.y - (cp[1] + t * vy), dz = B.z - (cp[2] + t * vz);
    const float rr = Rm + cp[6];
    return dx * dx + dy * dy + dz * dz < rr * fabsf(rr);
  }
  m -= ob.Mc;
  if (KIND == 2 || (KIND < 0 && m < ob.Mb)) {
    const float* b = ob.box + 15 * m;
    const float dx = B.x - b[0], dy = B.y - b[1], dz = B.z - b[2];
    const float q1 = fmaxf(fabsf(dx * b[3] + dy * b[4] + dz * b[5]) - b[12], 0.f);
    const float q2 = fmaxf(fabsf(dx * b[6] + dy * b[7] + dz * b[8]) - b[13], 0.f);
    const float q3 = fmaxf(fabsf(dx * b[9] + dy * b[10] + dz * b[11]) - b[14], 0.f);
    // a centre inside the box has a bound <= -R, below any margin > -R
    return q1 * q1 + q2 * q2 + q3 * q3 < Rm * fabsf(Rm) || Rm <= 0.f;
  }
  m -= ob.Mb;
  const float* h = ob.hs + 6 * m;
  return (B.x - h[3]) * h[0] + (B.y - h[4]) * h[1] + (B.z - h[5]) * h[2] - R < margin;
}

// Calls f(m, ObsKind<kind>()) for each obstacle m of this lane's share --
// every stride-th obstacle of each kind from `lane` -- that obstacle_near
// keeps: one loop per kind, so neither the test nor f needs to dispatch.
template <class F>
__device__ __forceinline__ void for_each_near_obstacle(const ObsView& ob, float3 B, float R, float margin, int lane,
                                                       int stride, F&& f) {
  int base = 0;
  for (int k = lane; k < ob.Ms; k += stride)
    if (obstacle_near<0>(ob, base + k, B, R, margin)) f(base + k, ObsKind<0>());
  base += ob.Ms;
  for (int k = lane; k < ob.Mc; k += stride)
    if (obstacle_near<1>(ob, base + k, B, R, margin)) f(base + k, ObsKind<1>());
  base += ob.Mc;
  for (int k = lane; k < ob.Mb; k += stride)
    if (obstacle_near<2>(ob, base + k, B, R, margin)) f(base + k, ObsKind<2>());
  base += ob.Mb;
  for (int k = lane; k < ob.Mh; k += stride)
    if (obstacle_near<3>(ob, base + k, B, R, margin)) f(base + k, ObsKind<3>());
}

__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// Order-preserving float <-> int map for atomic min on signed floats.
__device__ __forceinline__ int float_to_ordered(float f) {
  const int i = __float_as_int(f);
  return (i >= 0) ? i : (i ^ 0x7fffffff);
}
__device__ __forceinline__ float ordered_to_float(int i) {
  return __int_as_float((i >= 0) ? i : (i ^ 0x7fffffff));
}

__device__ __forceinline__ float warp_min(float v, unsigned mask = 0xffffffffu) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(mask, v, o));
  return v;
}

}  // namespace pk
