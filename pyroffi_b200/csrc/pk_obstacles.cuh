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

struct WorldArgs {
  const float* spheres;
  const float* capsules;
  const float* boxes;
  const float* halfspaces;
  int Ms, Mc, Mb, Mh;
  __host__ __device__ int total() const { return Ms + Mc + Mb + Mh; }
  // floats needed to stage everything in shared memory (spheres first, 16-byte aligned)
  __host__ __device__ size_t smem_floats() const {
    return (size_t)Ms * 4 + (size_t)Mc * 7 + (size_t)Mb * 15 + (size_t)Mh * 6;
  }
};

struct ObsView {
  const float4* sph;
  const float* cap;
  const float* box;
  const float* hs;
  int Ms, Mc, Mb, Mh;
};

// Copies the obstacle arrays into shared memory at `dst` (16-byte aligned)
// with all threads of the block; the caller synchronises afterwards.
__device__ inline ObsView stage_world(const WorldArgs& w, float* dst) {
  ObsView v;
  float* p = dst;
  for (int i = threadIdx.x; i < w.Ms * 4; i += blockDim.x) p[i] = w.spheres[i];
  v.sph = reinterpret_cast<const float4*>(p);
  p += w.Ms * 4;
  for (int i = threadIdx.x; i < w.Mc * 7; i += blockDim.x) p[i] = w.capsules[i];
  v.cap = p;
  p += w.Mc * 7;
  for (int i = threadIdx.x; i < w.Mb * 15; i += blockDim.x) p[i] = w.boxes[i];
  v.box = p;
  p += w.Mb * 15;
  for (int i = threadIdx.x; i < w.Mh * 6; i += blockDim.x) p[i] = w.halfspaces[i];
  v.hs = p;
  v.Ms = w.Ms; v.Mc = w.Mc; v.Mb = w.Mb; v.Mh = w.Mh;
  return v;
}

// Signed distance from sphere (c, r) to obstacle m (exact IEEE sqrt).
__device__ __forceinline__ float obstacle_dist(const ObsView& o, int m, float3 c, float r) {
  if (m < o.Ms) {
    const float4 s = o.sph[m];
    return d_sphere_sphere(c, r, s.x, s.y, s.z, s.w);
  }
  m -= o.Ms;
  if (m < o.Mc) return d_sphere_capsule(c, r, o.cap + 7 * m);
  m -= o.Mc;
  if (m < o.Mb) return d_sphere_box(c, r, o.box + 15 * m);
  m -= o.Mb;
  return d_sphere_halfspace(c, r, o.hs + 6 * m);
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
