// Shared device code for the pyroffi_b200 kernels (sm_100a).
//
// Conventions follow the reference (jaxlie SE(3), src/pyroffi/_robot.py and
// src/pyroffi/cuda_kernels/_fk_cuda_helpers.cuh): poses are wxyz_xyz, joint
// motions are exp(twist * q) with twist = [v, omega], T_parent_child =
// parent_tf o exp(twist * q), T_world[j] = T_world[parent(j)] o T_parent_child.
//
// The robot description is staged per block into shared memory in
// topological order (JointTable), so a kernel never keeps device pointers
// from a previous call: every launch reads the caller's buffers afresh.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pyroffi_b200.h"

#define PK_MAX_JOINTS 64
#define PK_MAX_ACT 32
#define PK_MAX_EE 4

namespace pk {

// ---------------------------------------------------------------------------
// small vector / SE(3) math (float)
// ---------------------------------------------------------------------------

struct Pose {
  float w, x, y, z;     // rotation (unit quaternion)
  float tx, ty, tz;     // translation
};

__device__ __forceinline__ Pose pose_identity() { return Pose{1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}; }

__device__ __forceinline__ float3 quat_rotate(float w, float x, float y, float z, float3 v) {
  // v' = v + w * t + u x t,  t = 2 u x v
  const float tx = 2.f * (y * v.z - z * v.y);
  const float ty = 2.f * (z * v.x - x * v.z);
  const float tz = 2.f * (x * v.y - y * v.x);
  return make_float3(v.x + w * tx + (y * tz - z * ty),
                     v.y + w * ty + (z * tx - x * tz),
                     v.z + w * tz + (x * ty - y * tx));
}

__device__ __forceinline__ float3 pose_apply(const Pose& T, float3 p) {
  float3 r = quat_rotate(T.w, T.x, T.y, T.z, p);
  return make_float3(r.x + T.tx, r.y + T.ty, r.z + T.tz);
}

// p expressed in the frame of pose T: R^T (p - t).
__device__ __forceinline__ float3 pose_apply_inv(const Pose& T, float3 p) {
  return quat_rotate(T.w, -T.x, -T.y, -T.z, make_float3(p.x - T.tx, p.y - T.ty, p.z - T.tz));
}

__device__ __forceinline__ Pose pose_compose(const Pose& a, const Pose& b) {
  Pose o;
  o.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  o.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  o.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
  o.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
  float3 t = quat_rotate(a.w, a.x, a.y, a.z, make_float3(b.tx, b.ty, b.tz));
  o.tx = t.x + a.tx;
  o.ty = t.y + a.ty;
  o.tz = t.z + a.tz;
  return o;
}

// Joint kinds of the motion exp(twist * q).
enum JointKind : int { kFixed = 0, kRevolute = 1, kPrismatic = 2, kScrew = 3 };

// exp(twist * q) for a joint of the given kind.  Revolute joints (v = 0) take
// the closed form q_rot = (cos(t/2), sin(t/2)/t * omega q), translation 0;
// prismatic joints (omega = 0) a pure translation v q; any other twist uses
// the full SE(3) exponential (B = (1-cos t)/t^2, C = (t - sin t)/t^3), with
// the reference's identity-rotation cut-off for theta^2 < 1e-12.
__device__ __forceinline__ Pose joint_motion(int kind, const float* tw, float q) {
  Pose d = pose_identity();
  if (kind == kPrismatic) {
    d.tx = tw[0] * q; d.ty = tw[1] * q; d.tz = tw[2] * q;
    return d;
  }
  const float ox = tw[3] * q, oy = tw[4] * q, oz = tw[5] * q;
  const float th2 = ox * ox + oy * oy + oz * oz;
  if (kind == kRevolute) {
    if (th2 < 1e-12f) return d;
    const float th = sqrtf(th2);
    float sh, ch;
    sincosf(0.5f * th, &sh, &ch);
    const float s = sh / th;
    d.w = ch; d.x = s * ox; d.y = s * oy; d.z = s * oz;
    return d;
  }
  // screw / general
  const float vx = tw[0] * q, vy = tw[1] * q, vz = tw[2] * q;
  if (th2 < 1e-12f) { d.tx = vx; d.ty = vy; d.tz = vz; return d; }
  const float th = sqrtf(th2);
  float sh, ch, st, ct;
  sincosf(0.5f * th, &sh, &ch);
  sincosf(th, &st, &ct);
  const float s = sh / th;
  d.w = ch; d.x = s * ox; d.y = s * oy; d.z = s * oz;
  // t = V v,  V = I + B [w]x + C [w]x^2  (jaxlie SE3.exp; the reference's
  // CUDA helper adds (sin t / t - 1) v here, which only screw twists reach)
  const float B = (1.f - ct) / th2, C = (th - st) / (th2 * th);
  const float cx = oy * vz - oz * vy, cy = oz * vx - ox * vz, cz = ox * vy - oy * vx;
  const float od = ox * vx + oy * vy + oz * vz;
  d.tx = vx + B * cx + C * (ox * od - th2 * vx);
  d.ty = vy + B * cy + C * (oy * od - th2 * vy);
  d.tz = vz + B * cz + C * (oz * od - th2 * vz);
  return d;
}

// ---------------------------------------------------------------------------
// Robot description staged in shared memory, in topological order.
// ---------------------------------------------------------------------------

struct ModelArgs {
  const float* twists;       // [n_j, 6]
  const float* parent_tf;    // [n_j, 7]
  const int* parent_idx;     // [n_j]
  const int* act_idx;        // [n_j]
  const float* mimic_mul;    // [n_j]
  const float* mimic_off;    // [n_j]
  const int* mimic_act_idx;  // [n_j]
  const int* topo_inv;       // [n_j] sorted position -> original joint index
  int n_joints;
  int n_act;
};

// 16-byte aligned so float4 arrays can follow it in shared memory.
struct __align__(16) JointTable {
  float ptf[PK_MAX_JOINTS][7];  // parent_tf, by sorted position
  float tw[PK_MAX_JOINTS][6];   // twist
  float mul[PK_MAX_JOINTS];
  float off[PK_MAX_JOINTS];
  float axis[PK_MAX_JOINTS][3]; // unit Jacobian axis in the joint frame
  float ru[PK_MAX_JOINTS][4];   // revolute motion: unit omega axis and |omega|
  int src[PK_MAX_JOINTS];       // actuated source index (-1: none)
  int psorted[PK_MAX_JOINTS];   // sorted position of the parent (-1: root)
  int orig[PK_MAX_JOINTS];      // original joint index
  int kind[PK_MAX_JOINTS];      // JointKind of the motion
  int jkind[PK_MAX_JOINTS];     // Jacobian kind: 0 none, 1 revolute, 2 prismatic
  int a1[PK_MAX_JOINTS];        // act_idx[j]
  int a2[PK_MAX_JOINTS];        // mimic_act_idx[j]
  int sorted_of[PK_MAX_JOINTS]; // original joint index -> sorted position
  int n;
  int chain;                    // 1 when psorted[i] == i-1 for every i > 0 and psorted[0] == -1
};

// Cooperative staging by all threads of a block; ends with __syncthreads().
__device__ inline void load_joint_table(JointTable& jt, const ModelArgs& m) {
  // Out-of-range indices in the caller's arrays are clamped so no shared or
  // global access leaves its buffer (the results are then meaningless, as
  // with the reference, but nothing faults).
  const int n = m.n_joints;
  for (int i = threadIdx.x; i < n; i += blockDim.x) jt.sorted_of[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int j = m.topo_inv[i];
    j = (j >= 0 && j < n) ? j : 0;
    jt.orig[i] = j;
    jt.sorted_of[j] = i;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int j = jt.orig[i];
    for (int c = 0; c < 7; ++c) jt.ptf[i][c] = m.parent_tf[j * 7 + c];
    float tw[6];
    for (int c = 0; c < 6; ++c) tw[c] = jt.tw[i][c] = m.twists[j * 6 + c];
    int ma = m.mimic_act_idx[j], aa = m.act_idx[j];
    ma = (ma >= 0 && ma < m.n_act) ? ma : -1;
    aa = (aa >= 0 && aa < m.n_act) ? aa : -1;
    const int src = (ma != -1) ? ma : aa;
    jt.src[i] = src;
    jt.mul[i] = m.mimic_mul[j];
    jt.off[i] = m.mimic_off[j];
    jt.a1[i] = aa;
    jt.a2[i] = ma;
    const int p = m.parent_idx[j];
    // a parent must precede its child in topological order
    const int pp = (p < 0 || p >= n) ? -1 : jt.sorted_of[p];
    jt.psorted[i] = (pp >= 0 && pp < i) ? pp : -1;
    const float lin2 = tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2];
    const float ang2 = tw[3] * tw[3] + tw[4] * tw[4] + tw[5] * tw[5];
    int kind;
    if (src == -1 && jt.off[i] == 0.f) kind = kFixed;
    else if (lin2 == 0.f && ang2 == 0.f) kind = kFixed;
    else if (lin2 == 0.f) kind = kRevolute;
    else if (ang2 == 0.f) kind = kPrismatic;
    else kind = kScrew;
    jt.kind[i] = kind;
    {
      const float n_w = sqrtf(ang2);
      const float inv = (n_w > 0.f) ? 1.f / n_w : 0.f;
      jt.ru[i][0] = tw[3] * inv; jt.ru[i][1] = tw[4] * inv; jt.ru[i][2] = tw[5] * inv; jt.ru[i][3] = n_w;
    }
    // Jacobian column kind as in the reference helper: revolute when
    // |omega|^2 > 1e-6, else prismatic when |v|^2 > 1e-6.
    if (ang2 > 1e-6f) {
      const float inv = rsqrtf(ang2);
      jt.jkind[i] = 1;
      jt.axis[i][0] = tw[3] * inv; jt.axis[i][1] = tw[4] * inv; jt.axis[i][2] = tw[5] * inv;
    } else if (lin2 > 1e-6f) {
      const float inv = rsqrtf(lin2);
      jt.jkind[i] = 2;
      jt.axis[i][0] = tw[0] * inv; jt.axis[i][1] = tw[1] * inv; jt.axis[i][2] = tw[2] * inv;
    } else {
      jt.jkind[i] = 0;
      jt.axis[i][0] = jt.axis[i][1] = jt.axis[i][2] = 0.f;
    }
  }
  if (threadIdx.x == 0) jt.n = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    int chain = 1;
    for (int i = 0; i < n; ++i)
      if (jt.psorted[i] != i - 1) { chain = 0; break; }
    jt.chain = chain;
  }
  __syncthreads();
}

__device__ __forceinline__ Pose load_ptf(const JointTable& jt, int i) {
  return Pose{jt.ptf[i][0], jt.ptf[i][1], jt.ptf[i][2], jt.ptf[i][3],
              jt.ptf[i][4], jt.ptf[i][5], jt.ptf[i][6]};
}

// T_parent_child = parent_tf o exp(twist * q) of sorted joint i.  For a
// revolute twist (0, w) with w = n u, |u| = 1, exp is the pure rotation
// (cos(q n / 2), sin(q n / 2) u) -- the same quaternion as
// (cos(t/2), sin(t/2)/t * w q) with t = |q| n, without the square root and
// division -- so T_pc keeps parent_tf's translation.
__device__ __forceinline__ Pose joint_local(const JointTable& jt, int i, float q) {
  Pose P = load_ptf(jt, i);
  const int kind = jt.kind[i];
  if (kind == kFixed) return P;
  if (kind == kRevolute) {
    float s, c;
    sincosf(0.5f * q * jt.ru[i][3], &s, &c);
    const float bx = s * jt.ru[i][0], by = s * jt.ru[i][1], bz = s * jt.ru[i][2];
    Pose o;
    o.w = P.w * c - P.x * bx - P.y * by - P.z * bz;
    o.x = P.w * bx + P.x * c + P.y * bz - P.z * by;
    o.y = P.w * by - P.x * bz + P.y * c + P.z * bx;
    o.z = P.w * bz + P.x * by - P.y * bx + P.z * c;
    o.tx = P.tx; o.ty = P.ty; o.tz = P.tz;
    return o;
  }
  return pose_compose(P, joint_motion(kind, jt.tw[i], q));
}

// Per-thread pose storage in shared memory, strided by `stride` floats
// between consecutive components so consecutive threads hit consecutive
// banks.  Component c of sorted joint i lives at base[(i*7+c)*stride].
struct PoseSlots {
  float* base;
  int stride;
  __device__ __forceinline__ void store(int i, const Pose& T) const {
    float* p = base + (i * 7) * stride;
    p[0] = T.w; p[stride] = T.x; p[2 * stride] = T.y; p[3 * stride] = T.z;
    p[4 * stride] = T.tx; p[5 * stride] = T.ty; p[6 * stride] = T.tz;
  }
  __device__ __forceinline__ Pose load(int i) const {
    const float* p = base + (i * 7) * stride;
    return Pose{p[0], p[stride], p[2 * stride], p[3 * stride], p[4 * stride], p[5 * stride], p[6 * stride]};
  }
};

// Forward kinematics of one configuration (cfg: pointer to n_act floats,
// any address space).  World poses are stored by sorted position.
template <typename CfgFn>
__device__ __forceinline__ void fk_thread(const JointTable& jt, CfgFn cfg_at, const PoseSlots& out) {
  Pose prev = pose_identity();
  const int n = jt.n;
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
    out.store(i, Tw);
    prev = Tw;
  }
}

// ---------------------------------------------------------------------------
// distance primitives (positive = separated)
// ---------------------------------------------------------------------------

__device__ __forceinline__ float d_sphere_sphere(float3 a, float ar, float bx, float by, float bz, float br) {
  const float dx = a.x - bx, dy = a.y - by, dz = a.z - bz;
  return sqrtf(dx * dx + dy * dy + dz * dz) - (ar + br);
}

__device__ __forceinline__ float d_sphere_capsule(float3 s, float sr, const float* c) {
  const float vx = c[3] - c[0], vy = c[4] - c[1], vz = c[5] - c[2];
  const float len2 = vx * vx + vy * vy + vz * vz;
  float t = 0.f;
  if (len2 > 1e-12f) {
    t = ((s.x - c[0]) * vx + (s.y - c[1]) * vy + (s.z - c[2]) * vz) / len2;
    t = fmaxf(0.f, fminf(1.f, t));
  }
  const float px = c[0] + t * vx - s.x, py = c[1] + t * vy - s.y, pz = c[2] + t * vz - s.z;
  return sqrtf(px * px + py * py + pz * pz) - (sr + c[6]);
}

__device__ __forceinline__ float box_sdf_local(float p1, float p2, float p3, float h1, float h2, float h3) {
  const float q1 = fabsf(p1) - h1, q2 = fabsf(p2) - h2, q3 = fabsf(p3) - h3;
  const float m1 = fmaxf(q1, 0.f), m2 = fmaxf(q2, 0.f), m3 = fmaxf(q3, 0.f);
  return sqrtf(m1 * m1 + m2 * m2 + m3 * m3) + fminf(fmaxf(fmaxf(q1, q2), q3), 0.f);
}

__device__ __forceinline__ float d_sphere_box(float3 s, float sr, const float* b) {
  const float dx = s.x - b[0], dy = s.y - b[1], dz = s.z - b[2];
  return box_sdf_local(dx * b[3] + dy * b[4] + dz * b[5],
                       dx * b[6] + dy * b[7] + dz * b[8],
                       dx * b[9] + dy * b[10] + dz * b[11], b[12], b[13], b[14]) - sr;
}

__device__ __forceinline__ float d_sphere_halfspace(float3 s, float sr, const float* h) {
  return (s.x - h[3]) * h[0] + (s.y - h[4]) * h[1] + (s.z - h[5]) * h[2] - sr;
}

__device__ __forceinline__ float d_capsule_capsule(const float* A, const float* Bc) {
  const float d1x = A[3] - A[0], d1y = A[4] - A[1], d1z = A[5] - A[2];
  const float d2x = Bc[3] - Bc[0], d2y = Bc[4] - Bc[1], d2z = Bc[5] - Bc[2];
  const float rx = A[0] - Bc[0], ry = A[1] - Bc[1], rz = A[2] - Bc[2];
  const float a = d1x * d1x + d1y * d1y + d1z * d1z;
  const float e = d2x * d2x + d2y * d2y + d2z * d2z;
  const float f = d2x * rx + d2y * ry + d2z * rz;
  const float eps = 1e-10f;
  float s, t;
  if (a <= eps && e <= eps) {
    s = t = 0.f;
  } else if (a <= eps) {
    s = 0.f;
    t = fmaxf(0.f, fminf(1.f, f / e));
  } else {
    const float c = d1x * rx + d1y * ry + d1z * rz;
    if (e <= eps) {
      t = 0.f;
      s = fmaxf(0.f, fminf(1.f, -c / a));
    } else {
      const float b = d1x * d2x + d1y * d2y + d1z * d2z;
      const float den = a * e - b * b;
      s = (fabsf(den) > eps) ? fmaxf(0.f, fminf(1.f, (b * f - c * e) / den)) : 0.f;
      t = (b * s + f) / e;
      if (t < 0.f) { t = 0.f; s = fmaxf(0.f, fminf(1.f, -c / a)); }
      else if (t > 1.f) { t = 1.f; s = fmaxf(0.f, fminf(1.f, (b - c) / a)); }
    }
  }
  const float px = A[0] + s * d1x - (Bc[0] + t * d2x);
  const float py = A[1] + s * d1y - (Bc[1] + t * d2y);
  const float pz = A[2] + s * d1z - (Bc[2] + t * d2z);
  return sqrtf(px * px + py * py + pz * pz) - (A[6] + Bc[6]);
}

__device__ __forceinline__ float d_capsule_box(const float* c, const float* b) {
  const float d1x = c[0] - b[0], d1y = c[1] - b[1], d1z = c[2] - b[2];
  const float al1 = d1x * b[3] + d1y * b[4] + d1z * b[5];
  const float al2 = d1x * b[6] + d1y * b[7] + d1z * b[8];
  const float al3 = d1x * b[9] + d1y * b[10] + d1z * b[11];
  const float d2x = c[3] - b[0], d2y = c[4] - b[1], d2z = c[5] - b[2];
  const float ab1 = d2x * b[3] + d2y * b[4] + d2z * b[5] - al1;
  const float ab2 = d2x * b[6] + d2y * b[7] + d2z * b[8] - al2;
  const float ab3 = d2x * b[9] + d2y * b[10] + d2z * b[11] - al3;
  const float l2 = ab1 * ab1 + ab2 * ab2 + ab3 * ab3;
  float t = 0.f;
  if (l2 > 1e-12f) t = fmaxf(0.f, fminf(1.f, (-al1 * ab1 - al2 * ab2 - al3 * ab3) / l2));
  return box_sdf_local(al1 + t * ab1, al2 + t * ab2, al3 + t * ab3, b[12], b[13], b[14]) - c[6];
}

__device__ __forceinline__ float d_capsule_halfspace(const float* c, const float* h) {
  const float d1 = (c[0] - h[3]) * h[0] + (c[1] - h[4]) * h[1] + (c[2] - h[5]) * h[2];
  const float d2 = (c[3] - h[3]) * h[0] + (c[4] - h[4]) * h[1] + (c[5] - h[5]) * h[2];
  return fminf(d1, d2) - c[6];
}

}  // namespace pk

// ---------------------------------------------------------------------------
// host-side status helpers shared by the C-ABI translation units
// ---------------------------------------------------------------------------
namespace pk {
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* where);
// Raises the kernel's dynamic shared-memory limit when `bytes` exceeds the
// 48 KB default (on the current device).
int set_smem_limit(const void* kernel, size_t bytes);
// Host hooks of the bounded wait in the obstacle staging of one source file
// (pk_obstacles.cuh): read its counters (adding to the sums), zero them, set
// the test hook and the time limit; each on the current device.
struct StageWaitHooks {
  int (*read)(unsigned long long* gave_up, unsigned long long* abandoned);
  int (*reset)();
  int (*set)(unsigned int force, unsigned long long limit_ns);
};
int register_stage_wait_hooks(StageWaitHooks h);
}  // namespace pk

#define PK_CHECK_ARG(cond, ...)                 \
  do {                                          \
    if (!(cond)) {                              \
      pk::set_error(__VA_ARGS__);               \
      return PK_ERR_INVALID;                    \
    }                                           \
  } while (0)

#define PK_CHECK_CAP(cond, ...)                 \
  do {                                          \
    if (!(cond)) {                              \
      pk::set_error(__VA_ARGS__);               \
      return PK_ERR_CAPACITY;                   \
    }                                           \
  } while (0)
