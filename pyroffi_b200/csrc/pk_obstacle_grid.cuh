// Uniform grid over the sphere obstacles, built per block in shared memory:
// a query ball of radius at most `reach` whose centre lies in cell c can only
// reach obstacles listed in c.  Shared by the LM kernels and the per-seed IK
// (HJCD, SQP) kernels.
//
// Obstacle o (centre x_o, radius r_o) is listed in every cell that the
// bounding box of the ball of radius r_o + reach + 1e-3 around x_o touches,
// in increasing o; the grid spans the union of those boxes, so a centre
// outside it is out of reach of every obstacle.  If |B - x_o| < R + r_o with
// R <= reach then B lies in that box and the cell of B lists o: cell indices
// are monotone in the coordinate, and the 1e-3 covers the rounding of the
// caller's test.
#pragma once

namespace pk {

// Cells per axis G: a launch option (the obstacle tile of the IK kernels),
// 8 by default, at most 16 (cell indices are packed in 4 bits).
constexpr int kObsGridDefault = 8;
constexpr int kObsGridMax = 16;
__host__ __device__ __forceinline__ int obstacle_grid_cells(int G) { return G * G * G; }
// pk_lm_options.obstacle_grid -> cells per axis: 0 the default, -1 no grid (0 here)
__host__ __device__ __forceinline__ int obstacle_grid_option(int v) { return v == 0 ? kObsGridDefault : (v < 0 ? 0 : v); }
// The IK kernels' default: 14 cells per axis for up to 160 obstacle
// spheres, 12 for up to 1024, 8 above, with lists of up to 80 entries per
// sphere (16384 in all) for the finer grids; a grid whose lists overflow
// falls back to 8 cells (obstacle_grid_capacity).  On the 100-sphere IK
// benchmark world the 14-cell grid lists 34 candidates per query against 57
// at 8 (the same 5.5 survive the bounding test); on the 500-sphere mixed
// batch world 12 cells list 47-92 candidates per evaluation against 122-150.
constexpr int kObsGridFine = 14;
constexpr int kObsGridFineMaxSpheres = 160;
constexpr int kObsGridMid = 12;
constexpr int kObsGridMidMaxSpheres = 1024;
__host__ __device__ __forceinline__ int lm_grid_option(int v, int Ms) {
  if (v == 0)
    return Ms <= kObsGridFineMaxSpheres ? kObsGridFine : (Ms <= kObsGridMidMaxSpheres ? kObsGridMid : kObsGridDefault);
  return obstacle_grid_option(v);
}
// List capacity of a grid of G cells per axis over Ms spheres.
__host__ __device__ __forceinline__ int obstacle_grid_capacity(int G, int Ms) {
  const int per = G > kObsGridDefault ? 80 : 48;
  const int c = per * Ms;
  return c < 1024 ? 1024 : (c > 16384 ? 16384 : c);
}

// Origin and inverse cell size of the grid (one thread).
__device__ inline void obstacle_grid_bounds(const float4* ws, int Ms, float reach, int G, float3& lo, float3& inv) {
  float l[3] = {3e38f, 3e38f, 3e38f}, h[3] = {-3e38f, -3e38f, -3e38f};
  for (int o = 0; o < Ms; ++o) {
    const float4 O = ws[o];
    const float rho = O.w + reach + 1e-3f;
    l[0] = fminf(l[0], O.x - rho); h[0] = fmaxf(h[0], O.x + rho);
    l[1] = fminf(l[1], O.y - rho); h[1] = fmaxf(h[1], O.y + rho);
    l[2] = fminf(l[2], O.z - rho); h[2] = fmaxf(h[2], O.z + rho);
  }
  lo = make_float3(l[0], l[1], l[2]);
  inv = make_float3(G / fmaxf(h[0] - l[0], 1e-6f), G / fmaxf(h[1] - l[1], 1e-6f), G / fmaxf(h[2] - l[2], 1e-6f));
}

// Cell lists: cell_start[G^3 + 1] offsets into cell_obs; obox[Ms]
// is scratch.  Called by every thread of the block with block-uniform
// arguments; `on` (shared) is cleared when the lists would exceed
// max_entries, and the caller then scans every obstacle instead.  Each
// obstacle adds itself to the cells of its box (shared-memory atomics), and
// every cell's list is then sorted, so the lists hold increasing obstacle
// indices whatever the order of the atomics.
__device__ inline void obstacle_grid_build(const float4* ws, int Ms, float reach, int G, float3 lo, float3 inv,
                                           int* obox, int* cell_start, unsigned short* cell_obs, int max_entries,
                                           int& on) {
  const int NC = obstacle_grid_cells(G);
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int c = tid; c <= NC; c += nth) cell_start[c] = 0;
  for (int o = tid; o < Ms; o += nth) {
    const float4 O = ws[o];
    const float rho = O.w + reach + 1e-3f;
    const float c3[3] = {O.x, O.y, O.z}, l3[3] = {lo.x, lo.y, lo.z}, i3[3] = {inv.x, inv.y, inv.z};
    int packed = 0;
    for (int d = 0; d < 3; ++d) {
      const int i0 = min(max(__float2int_rd((c3[d] - rho - l3[d]) * i3[d]), 0), G - 1);
      const int i1 = min(max(__float2int_rd((c3[d] + rho - l3[d]) * i3[d]), 0), G - 1);
      packed |= (i0 | (i1 << 4)) << (8 * d);
    }
    obox[o] = packed;
  }
  __syncthreads();
  // calls f(cell) for every cell of obstacle o's box
  auto cells_of = [&](int o, auto&& f) {
    const int b = obox[o];
    for (int ix = b & 15; ix <= ((b >> 4) & 15); ++ix)
      for (int iy = (b >> 8) & 15; iy <= ((b >> 12) & 15); ++iy)
        for (int iz = (b >> 16) & 15; iz <= ((b >> 20) & 15); ++iz) f((ix * G + iy) * G + iz);
  };
  for (int o = tid; o < Ms; o += nth) cells_of(o, [&](int c) { atomicAdd(&cell_start[c], 1); });
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int c = 0; c < NC; ++c) {
      const int n = cell_start[c];
      cell_start[c] = run;
      run += n;
    }
    cell_start[NC] = run;
    if (run > max_entries) on = 0;
  }
  __syncthreads();
  if (on) {
    // fill: cell_start[c] advances to the end of cell c, i.e. the start of c + 1
    for (int o = tid; o < Ms; o += nth)
      cells_of(o, [&](int c) { cell_obs[atomicAdd(&cell_start[c], 1)] = (unsigned short)o; });
    __syncthreads();
    if (tid == 0) {
      for (int c = NC - 1; c > 0; --c) cell_start[c] = cell_start[c - 1];
      cell_start[0] = 0;
    }
    __syncthreads();
    for (int c = tid; c < NC; c += nth) {
      const int e0 = cell_start[c], e1 = cell_start[c + 1];
      for (int i = e0 + 1; i < e1; ++i) {
        const unsigned short v = cell_obs[i];
        int j = i - 1;
        while (j >= e0 && cell_obs[j] > v) {
          cell_obs[j + 1] = cell_obs[j];
          --j;
        }
        cell_obs[j + 1] = v;
      }
    }
  }
  __syncthreads();
}

// Cell of point B, or -1 outside the grid (no obstacle within reach).
__device__ __forceinline__ int obstacle_grid_cell(float3 lo, float3 inv, int G, float3 B) {
  const int ix = __float2int_rd((B.x - lo.x) * inv.x);
  const int iy = __float2int_rd((B.y - lo.y) * inv.y);
  const int iz = __float2int_rd((B.z - lo.z) * inv.z);
  if ((unsigned)ix >= (unsigned)G || (unsigned)iy >= (unsigned)G || (unsigned)iz >= (unsigned)G) return -1;
  return (ix * G + iy) * G + iz;
}

}  // namespace pk
