// Collision-distance drop-ins: world sphere ([B,K,M] and per-link reduced
// [B,N,M]), world capsule, self sphere and self capsule.
//
// Replaces the handlers of src/pyroffi/cuda_kernels/_collision_cuda_kernel.cu
// (CollisionWorldSphereFfi :507, ...ReducedFfi :673, CollisionWorldCapsuleFfi
// :843, CollisionSelfSphereFfi :1006, CollisionSelfCapsuleFfi :1114).
//
// B200 layout: every obstacle type is staged once per block into shared
// memory and handled by one kernel (no per-type launches, no graph cache).
// Output rows [.., M] are written by groups of lanes running over m, so each
// warp store covers contiguous 16-byte chunks of one row; the reduced
// kernel keeps the running min over s in registers.  Self kernels stage each
// configuration's spheres (AoS in HBM) in shared memory once and evaluate
// pairs from there.
#include "pk_obstacles.cuh"

namespace pk {

// lanes that share one output row: enough to cover M with 4 columns each
static int lanes_per_row(int M) {
  int l = 1;
  while (l < 32 && l * 4 < M) l <<= 1;
  return l;
}

struct RowArgs {
  WorldArgs w;
  const float* centers;  // [3, B, K] SoA (sphere robot) or caps [7, B, N] (capsule robot)
  const float* radii;    // [B, K] (sphere robot)
  float* out;
  long long B;
  int K;                 // robot elements per configuration (spheres K, or links N)
  int N;                 // links (reduced kernel)
  int S;                 // spheres per link (reduced kernel)
  int lpr;               // lanes per row
  int stage;
};

__device__ __forceinline__ ObsView world_view(const RowArgs& a, float* smem) {
  if (a.stage) return stage_world(a.w, smem);
  ObsView ob;
  ob.sph = reinterpret_cast<const float4*>(a.w.spheres);
  ob.cap = a.w.capsules; ob.box = a.w.boxes; ob.hs = a.w.halfspaces;
  ob.Ms = a.w.Ms; ob.Mc = a.w.Mc; ob.Mb = a.w.Mb; ob.Mh = a.w.Mh;
  return ob;
}

// MODE 0: per-sphere rows [B,K,M]; MODE 1: per-link min over s [B,N,M];
// MODE 2: capsule robot rows [B,N,M].
template <int MODE>
__global__ void __launch_bounds__(256) world_rows_kernel(RowArgs a) {
  extern __shared__ __align__(16) float smem_f[];
  const ObsView ob = world_view(a, smem_f);
  __syncthreads();
  const int M = a.w.total();
  const int lpr = a.lpr;
  const int rows_per_block = blockDim.x / lpr;
  const int sub = threadIdx.x / lpr, sl = threadIdx.x - sub * lpr;
  const long long R = a.B * (long long)a.K;  // rows (b, k) or (b, n)
  const long long row = (long long)blockIdx.x * rows_per_block + sub;
  if (row >= R) return;
  const long long b = row / a.K;
  const int k = (int)(row - b * a.K);
  float* orow = a.out + row * (long long)M;
  const bool vec4 = ((M & 3) == 0) && ((reinterpret_cast<uintptr_t>(a.out) & 15) == 0);

  if (MODE == 0) {
    const long long BK = a.B * (long long)a.K;
    const float r = __ldg(a.radii + row);
    const float3 c = make_float3(__ldg(a.centers + row), __ldg(a.centers + BK + row),
                                 __ldg(a.centers + 2 * BK + row));
    if (vec4) {
      for (int m0 = sl * 4; m0 < M; m0 += lpr * 4) {
        float4 d;
        if (r < 0.f) {
          d = make_float4(1e9f, 1e9f, 1e9f, 1e9f);
        } else {
          d.x = obstacle_dist(ob, m0, c, r);
          d.y = obstacle_dist(ob, m0 + 1, c, r);
          d.z = obstacle_dist(ob, m0 + 2, c, r);
          d.w = obstacle_dist(ob, m0 + 3, c, r);
        }
        __stcs(reinterpret_cast<float4*>(orow + m0), d);
      }
    } else {
      for (int m0 = sl; m0 < M; m0 += lpr) orow[m0] = (r < 0.f) ? 1e9f : obstacle_dist(ob, m0, c, r);
    }
  } else if (MODE == 1) {
    // row = (b, n); sphere k = s*N + n
    const long long BK = a.B * (long long)a.S * a.N;
    const long long kb = b * (long long)a.S * a.N + k;
    for (int m0 = sl * 4; m0 < M; m0 += lpr * 4) {
      float d0 = 1e9f, d1 = 1e9f, d2 = 1e9f, d3 = 1e9f;
      for (int s = 0; s < a.S; ++s) {
        const long long q = kb + (long long)s * a.N;
        const float r = __ldg(a.radii + q);
        if (r < 0.f) continue;
        const float3 c = make_float3(__ldg(a.centers + q), __ldg(a.centers + BK + q),
                                     __ldg(a.centers + 2 * BK + q));
        d0 = fminf(d0, obstacle_dist(ob, m0, c, r));
        if (m0 + 1 < M) d1 = fminf(d1, obstacle_dist(ob, m0 + 1, c, r));
        if (m0 + 2 < M) d2 = fminf(d2, obstacle_dist(ob, m0 + 2, c, r));
        if (m0 + 3 < M) d3 = fminf(d3, obstacle_dist(ob, m0 + 3, c, r));
      }
      if (vec4) {
        __stcs(reinterpret_cast<float4*>(orow + m0), make_float4(d0, d1, d2, d3));
      } else {
        orow[m0] = d0;
        if (m0 + 1 < M) orow[m0 + 1] = d1;
        if (m0 + 2 < M) orow[m0 + 2] = d2;
        if (m0 + 3 < M) orow[m0 + 3] = d3;
      }
    }
  } else {
    // capsule robot: caps [7, B, N] SoA; row = (b, n)
    float cap[7];
#pragma unroll
    for (int c = 0; c < 7; ++c) cap[c] = __ldg(a.centers + (long long)c * R + row);
    for (int m0 = sl; m0 < M; m0 += lpr) {
      int m = m0;
      float d;
      if (m < ob.Ms) {
        // sphere-capsule with the world sphere as the sphere argument
        const float4 s = ob.sph[m];
        d = d_sphere_capsule(make_float3(s.x, s.y, s.z), s.w, cap);
      } else if ((m -= ob.Ms) < ob.Mc) {
        d = d_capsule_capsule(cap, ob.cap + 7 * m);
      } else if ((m -= ob.Mc) < ob.Mb) {
        d = d_capsule_box(cap, ob.box + 15 * m);
      } else {
        m -= ob.Mb;
        d = d_capsule_halfspace(cap, ob.hs + 6 * m);
      }
      orow[m0] = d;
    }
  }
}

// Self-collision, sphere robot: centers [B,S,N,3], radii [B,S,N]; one
// thread per (b, p), configurations staged in shared memory per block.
__global__ void __launch_bounds__(256) self_sphere_kernel(const float* __restrict__ centers,
                                                          const float* __restrict__ radii,
                                                          const int* __restrict__ pair_i,
                                                          const int* __restrict__ pair_j,
                                                          float* __restrict__ out, long long B, int S,
                                                          int N, int P, int cpb) {
  extern __shared__ __align__(16) float4 sph[];  // [cpb][S*N] (x,y,z,r)
  const int SN = S * N;
  const long long b0 = (long long)blockIdx.x * cpb;
  const int nc = (int)min((long long)cpb, B - b0);
  for (int g = threadIdx.x; g < nc * SN; g += blockDim.x) {
    const long long e = b0 * SN + g;
    sph[g] = make_float4(__ldg(centers + 3 * e), __ldg(centers + 3 * e + 1), __ldg(centers + 3 * e + 2),
                         __ldg(radii + e));
  }
  __syncthreads();
  for (int g = threadIdx.x; g < nc * P; g += blockDim.x) {
    const int c = g / P, p = g - c * P;
    const int li = __ldg(pair_i + p), lj = __ldg(pair_j + p);
    const float4* base = sph + c * SN;
    float dmin = 1e9f;
    if (li < 0 || li >= N || lj < 0 || lj >= N) {  // invalid link index: no pair
      out[(b0 + c) * P + p] = dmin;
      continue;
    }
    for (int si = 0; si < S; ++si) {
      const float4 A = base[si * N + li];
      if (A.w < 0.f) continue;
      for (int sj = 0; sj < S; ++sj) {
        const float4 Bq = base[sj * N + lj];
        if (Bq.w < 0.f) continue;
        dmin = fminf(dmin, d_sphere_sphere(make_float3(A.x, A.y, A.z), A.w, Bq.x, Bq.y, Bq.z, Bq.w));
      }
    }
    out[(b0 + c) * P + p] = dmin;
  }
}

__global__ void __launch_bounds__(256) self_capsule_kernel(const float* __restrict__ caps,
                                                           const int* __restrict__ pair_i,
                                                           const int* __restrict__ pair_j,
                                                           float* __restrict__ out, long long B, int N,
                                                           int P) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * P) return;
  const long long b = idx / P;
  const int p = (int)(idx - b * P);
  const int li = __ldg(pair_i + p), lj = __ldg(pair_j + p);
  if (li < 0 || li >= N || lj < 0 || lj >= N) {  // invalid link index: no pair
    out[idx] = 1e9f;
    return;
  }
  float A[7], Bc[7];
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    A[c] = __ldg(caps + (b * N + li) * 7 + c);
    Bc[c] = __ldg(caps + (b * N + lj) * 7 + c);
  }
  out[idx] = d_capsule_capsule(A, Bc);
}

static const size_t kWorldSmemLimit = 128 * 1024;

static int check_world(const WorldArgs& w) {
  PK_CHECK_ARG(w.Ms >= 0 && w.Mc >= 0 && w.Mb >= 0 && w.Mh >= 0, "negative obstacle count");
  PK_CHECK_ARG((w.Ms == 0 || w.spheres) && (w.Mc == 0 || w.capsules) && (w.Mb == 0 || w.boxes) &&
                   (w.Mh == 0 || w.halfspaces),
               "null world buffer");
  return PK_OK;
}

template <int MODE>
static int launch_rows(cudaStream_t stream, RowArgs a) {
  const int M = a.w.total();
  a.lpr = lanes_per_row(M);
  const size_t wbytes = sizeof(float) * a.w.smem_floats();
  a.stage = wbytes <= kWorldSmemLimit ? 1 : 0;
  PK_CHECK_ARG(a.stage || a.w.spheres == nullptr ||
                   (reinterpret_cast<uintptr_t>(a.w.spheres) & 15) == 0,
               "world_spheres must be 16-byte aligned when the world exceeds shared memory");
  const int threads = 256;
  const int rpb = threads / a.lpr;
  const long long rows = a.B * (long long)a.K;
  const long long blocks = (rows + rpb - 1) / rpb;
  PK_CHECK_CAP(blocks < (1LL << 31), "batch too large");
  const size_t smem = a.stage ? wbytes : 0;
  if (int st = set_smem_limit((const void*)world_rows_kernel<MODE>, smem)) return st;
  world_rows_kernel<MODE><<<(unsigned)blocks, threads, smem, stream>>>(a);
  return cuda_status(cudaGetLastError(), "world_rows_kernel launch");
}

}  // namespace pk

using namespace pk;

extern "C" int pk_collision_world_sphere(void* stream, const float* centers, const float* radii,
                                         const float* world_spheres, const float* world_capsules,
                                         const float* world_boxes, const float* world_halfspaces,
                                         float* out, int64_t B, int32_t K, int32_t Ms, int32_t Mc,
                                         int32_t Mb, int32_t Mh) {
  PK_CHECK_ARG(B >= 0 && K >= 0, "negative extent");
  WorldArgs w{world_spheres, world_capsules, world_boxes, world_halfspaces, Ms, Mc, Mb, Mh};
  if (int st = check_world(w)) return st;
  if (B == 0 || K == 0 || w.total() == 0) return PK_OK;
  PK_CHECK_ARG(centers && radii && out, "null buffer");
  RowArgs a{};
  a.w = w; a.centers = centers; a.radii = radii; a.out = out; a.B = B; a.K = K;
  return launch_rows<0>((cudaStream_t)stream, a);
}

extern "C" int pk_collision_world_sphere_reduced(void* stream, const float* centers,
                                                 const float* radii, const float* world_spheres,
                                                 const float* world_capsules,
                                                 const float* world_boxes,
                                                 const float* world_halfspaces, float* out,
                                                 int64_t B, int32_t K, int32_t Ms, int32_t Mc,
                                                 int32_t Mb, int32_t Mh, int64_t n) {
  PK_CHECK_ARG(B >= 0 && K >= 0 && n >= 0, "negative extent");
  WorldArgs w{world_spheres, world_capsules, world_boxes, world_halfspaces, Ms, Mc, Mb, Mh};
  if (int st = check_world(w)) return st;
  if (B == 0 || n == 0 || w.total() == 0) return PK_OK;
  PK_CHECK_ARG(n <= K || K == 0, "n=%lld exceeds K=%d", (long long)n, K);
  PK_CHECK_ARG(centers && radii && out, "null buffer");
  RowArgs a{};
  a.w = w; a.centers = centers; a.radii = radii; a.out = out; a.B = B;
  a.N = (int)n; a.S = (int)(K / n); a.K = (int)n;
  // centers are [3, B, K]: the SoA plane stride is B*K even when K != S*N.
  // Sphere (b, s, n) sits at b*K + s*N + n; the kernel addresses b*S*N, so
  // require K == S*N as the reference does (its K / N truncation).
  PK_CHECK_ARG((long long)a.S * n == K, "K=%d is not a multiple of n=%lld", K, (long long)n);
  return launch_rows<1>((cudaStream_t)stream, a);
}

extern "C" int pk_collision_world_capsule(void* stream, const float* caps,
                                          const float* world_spheres, const float* world_capsules,
                                          const float* world_boxes, const float* world_halfspaces,
                                          float* out, int64_t B, int32_t N, int32_t Ms, int32_t Mc,
                                          int32_t Mb, int32_t Mh) {
  PK_CHECK_ARG(B >= 0 && N >= 0, "negative extent");
  WorldArgs w{world_spheres, world_capsules, world_boxes, world_halfspaces, Ms, Mc, Mb, Mh};
  if (int st = check_world(w)) return st;
  if (B == 0 || N == 0 || w.total() == 0) return PK_OK;
  PK_CHECK_ARG(caps && out, "null buffer");
  RowArgs a{};
  a.w = w; a.centers = caps; a.out = out; a.B = B; a.K = N;
  return launch_rows<2>((cudaStream_t)stream, a);
}

extern "C" int pk_collision_self_sphere(void* stream, const float* centers, const float* radii,
                                        const int32_t* pair_i, const int32_t* pair_j, float* out,
                                        int64_t B, int32_t S, int32_t N, int32_t P) {
  PK_CHECK_ARG(B >= 0 && S >= 0 && N >= 0 && P >= 0, "negative extent");
  if (B == 0 || P == 0) return PK_OK;
  PK_CHECK_ARG(centers && radii && pair_i && pair_j && out, "null buffer");
  const int SN = S * N;
  int cpb = 64;
  while (cpb > 1 && (size_t)cpb * SN * sizeof(float4) > 96 * 1024) cpb >>= 1;
  PK_CHECK_CAP((size_t)cpb * SN * sizeof(float4) <= 96 * 1024, "S*N=%d too large", SN);
  const size_t smem = (size_t)cpb * SN * sizeof(float4);
  const long long blocks = (B + cpb - 1) / cpb;
  PK_CHECK_CAP(blocks < (1LL << 31), "batch too large");
  if (int st = set_smem_limit((const void*)self_sphere_kernel, smem)) return st;
  self_sphere_kernel<<<(unsigned)blocks, 256, smem, (cudaStream_t)stream>>>(centers, radii, pair_i,
                                                                             pair_j, out, B, S, N, P, cpb);
  return cuda_status(cudaGetLastError(), "self_sphere_kernel launch");
}

extern "C" int pk_collision_self_capsule(void* stream, const float* caps, const int32_t* pair_i,
                                         const int32_t* pair_j, float* out, int64_t B, int32_t N,
                                         int32_t P) {
  PK_CHECK_ARG(B >= 0 && N >= 0 && P >= 0, "negative extent");
  if (B == 0 || P == 0) return PK_OK;
  PK_CHECK_ARG(caps && pair_i && pair_j && out, "null buffer");
  const long long total = B * (long long)P;
  const long long blocks = (total + 255) / 256;
  PK_CHECK_CAP(blocks < (1LL << 31), "batch too large");
  self_capsule_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(caps, pair_i, pair_j, out, B,
                                                                            N, P);
  return cuda_status(cudaGetLastError(), "self_capsule_kernel launch");
}
