// CHOMP covariant direction in one launch: per trajectory, global-norm
// gradient clipping and pinned endpoints, then the truncated conjugate
// gradient solve of the smoothness metric on every joint's interior timeline
// (the reference's _cg_solve / covariant update,
// src/pyroffi/optimization_engines/_chomp_optimization.py:155-241,
// 297-318):
//
//   g <- g * min(1, clip / |g|)          (per trajectory; no clip when clip <= 0)
//   g[0] = g[T-1] = 0
//   M x = g_int,  (M x)_i = 6 x_i + reg x_i - 4 (x_{i-1} + x_{i+1}) + (x_{i-2} + x_{i+2})
//   d = -x on the interior, 0 at the ends
//
// CG: x = 0, r = p = b, rr = r.r, tol2 = (tol |b| + 1e-12)^2 with
// |b| = sqrt(b.b + 1e-18); per step alpha = rr / (p.Ap + 1e-9),
// beta = rr' / (rr + 1e-9), and a timeline stops updating once rr' <= tol2.
// The solve runs in FP64: truncated CG on this ill-conditioned metric is
// rounding-sensitive.
//
// B200 mapping: one block per trajectory, one warp per joint timeline (the
// warps loop over the joints); p lives in shared memory for the stencil, the
// dot products are warp shuffles.
#include <algorithm>

#include "pk_common.cuh"

namespace pk {

struct ChompDirArgs {
  const float* grad;   // [B, T, n]
  float* dir;          // [B, T, n]
  int T, n, iters;
  float clip, reg, tol;
  int covariant;
  const unsigned char* active;  // null, or only trajectories with active[b] != 0 are processed
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(256) chomp_direction_kernel(ChompDirArgs a) {
  extern __shared__ __align__(16) double shp[];   // [warps][Tin + 4]: p with two zeros on each side
  __shared__ float red[8];
  __shared__ float s_scale;
  const int T = a.T, n = a.n, Tn = T * n, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nw = blockDim.x >> 5;
  const long long b = blockIdx.x;
  if (a.active && !a.active[b]) return;  // block-uniform
  const float* g = a.grad + b * Tn;
  float* d = a.dir + b * Tn;
  // global-norm clip (FP32, as the reference's jnp.linalg.norm of the gradient)
  float part = 0.f;
  for (int i = tid; i < Tn; i += blockDim.x) part += g[i] * g[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) red[wid] = part;
  __syncthreads();
  if (tid == 0) {
    float s = 0.f;
    for (int w = 0; w < nw; ++w) s += red[w];
    const float gn = sqrtf(s);
    s_scale = (a.clip > 0.f && gn > a.clip) ? a.clip / (gn + 1e-12f) : 1.f;
  }
  __syncthreads();
  const float scale = s_scale;
  if (!a.covariant || T <= 2) {
    for (int i = tid; i < Tn; i += blockDim.x) {
      const int t = i / n;
      d[i] = (t == 0 || t == T - 1) ? 0.f : -(g[i] * scale);
    }
    return;
  }
  const int Tin = T - 2;
  double* P = shp + (size_t)wid * (Tin + 4) + 2;   // P[-2 .. Tin+1]
  if (lane < 2) { P[-2 + lane] = 0.0; P[Tin + lane] = 0.0; }
  const double reg = (double)a.reg, six = 6.0;
  for (int j = wid; j < n; j += nw) {
    // b = clipped gradient of joint j on the interior
    double bb = 0.0;
    for (int i = lane; i < Tin; i += 32) {
      const double v = (double)(g[(i + 1) * n + j] * scale);
      P[i] = v;
      bb += v * v;
    }
    bb = warp_sum_d(bb);
    const double bnorm = sqrt(bb + 1e-18);
    const double tol2 = ((double)a.tol * bnorm + 1e-12) * ((double)a.tol * bnorm + 1e-12);
    double rr = bb;
    bool active = true;
    // x and r per lane (elements lane, lane + 32, ...): up to 4 per lane held
    // in registers when Tin <= 128, else re-read from the direction buffer
    constexpr int KMAX = 4;
    double x[KMAX], r[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      const int i = lane + 32 * k;
      x[k] = 0.0;
      r[k] = i < Tin ? P[i] : 0.0;
    }
    __syncwarp();
    for (int it = 0; it < a.iters; ++it) {
      // Ap and p.Ap
      double pAp = 0.0, Ap[KMAX], pv[KMAX];
#pragma unroll
      for (int k = 0; k < KMAX; ++k) {
        const int i = lane + 32 * k;
        if (i < Tin) {
          const double pi = P[i];
          double y = six * pi + reg * pi;
          y -= 4.0 * P[i - 1];
          y -= 4.0 * P[i + 1];
          y += P[i - 2];
          y += P[i + 2];
          Ap[k] = y;
          pv[k] = pi;
          pAp += pi * y;
        } else {
          Ap[k] = 0.0;
          pv[k] = 0.0;
        }
      }
      pAp = warp_sum_d(pAp);
      const double alpha = rr / (pAp + 1e-9);
      double rrn = 0.0, rn[KMAX];
#pragma unroll
      for (int k = 0; k < KMAX; ++k) {
        rn[k] = r[k] - alpha * Ap[k];
        rrn += rn[k] * rn[k];
      }
      rrn = warp_sum_d(rrn);
      const double beta = rrn / (rr + 1e-9);
      __syncwarp();  // every lane has read P
      if (active) {
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
          const int i = lane + 32 * k;
          x[k] += alpha * pv[k];
          r[k] = rn[k];
          if (i < Tin) P[i] = rn[k] + beta * pv[k];
        }
        rr = rrn;
      }
      active = active && (rrn > tol2);
      __syncwarp();
      if (!active) break;  // warp-uniform: nothing changes any more
    }
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      const int i = lane + 32 * k;
      if (i < Tin) d[(i + 1) * n + j] = -(float)x[k];
    }
    if (lane == 0) { d[j] = 0.f; d[(T - 1) * n + j] = 0.f; }
    __syncwarp();
  }
}

// Line-search trials: trials[k, b] = traj[b] + clamp(alpha_k dir[b], -max_delta,
// max_delta) with the ends pinned to start / goal (the reference's trial
// update, _chomp_optimization.py:282-291, for K step sizes at once).  NaN
// passes through the clamp, as in torch.clamp.
__global__ void chomp_trials_kernel(const float* __restrict__ traj, const float* __restrict__ dir,
                                    const float* __restrict__ alphas, float max_delta, const float* __restrict__ start,
                                    const float* __restrict__ goal, float* __restrict__ trials, long long per, int T,
                                    int n, int K, const unsigned char* __restrict__ active) {
  const long long total = per * K;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / per);
    const long long e = i - (long long)k * per;
    const int c = (int)(e % n);
    const int t = (int)((e / n) % T);
    if (active && !active[e / ((long long)T * n)]) continue;  // a finished trajectory: its trials are not read
    float v;
    if (t == 0) {
      v = start[c];
    } else if (t == T - 1) {
      v = goal[c];
    } else {
      const float step = alphas[k] * dir[e];
      v = traj[e] + (step != step ? step : fminf(fmaxf(step, -max_delta), max_delta));
    }
    trials[i] = v;
  }
}

// Line-search selection, one block per trajectory: the first minimum over
// the K trial costs and the current cost (as torch.min: a NaN wins), the
// step taken when the trajectory is active and the minimum improves the
// current cost by min_improve, the stall counter and the early stop
// (_chomp_optimization.py:293-304).
__global__ void chomp_select_kernel(const float* __restrict__ tc, const float* __restrict__ cur,
                                    const float* __restrict__ trials, float* __restrict__ traj,
                                    unsigned char* __restrict__ active, int* __restrict__ stall, float min_improve,
                                    int patience, long long B, long long per_traj, int K) {
  const long long b = blockIdx.x;
  __shared__ int take;
  if (threadIdx.x == 0) {
    float best = tc[b];
    int idx = 0;
    for (int k = 1; k <= K; ++k) {
      if (best != best) break;
      const float v = (k < K) ? tc[(long long)k * B + b] : cur[b];
      if (v != v || v < best) { best = v; idx = k; }
    }
    const bool improved = best < cur[b] - min_improve;
    const bool act = active[b] != 0;
    take = (act && improved && idx < K) ? idx : -1;
    int st = stall[b];
    if (act) st = improved ? 0 : st + 1;
    stall[b] = st;
    active[b] = (act && st < patience) ? 1 : 0;
  }
  __syncthreads();
  if (take < 0) return;
  const float* src = trials + ((long long)take * B + b) * per_traj;
  float* dst = traj + b * per_traj;
  for (long long i = threadIdx.x; i < per_traj; i += blockDim.x) dst[i] = src[i];
}

}  // namespace pk

using namespace pk;

extern "C" int pk_chomp_direction(void* stream, const float* grad, float* dir, int64_t B, int32_t T, int32_t n_act,
                                  int32_t n_cg_iters, float grad_clip_norm, float smoothness_reg, float cg_tol,
                                  int32_t covariant, const uint8_t* active) {
  PK_CHECK_ARG(B >= 0 && T >= 0 && n_act >= 0 && n_cg_iters >= 0, "negative extent");
  PK_CHECK_CAP(T <= 130, "the CG solve takes at most 128 interior waypoints (T=%d)", T);
  PK_CHECK_CAP(B < (1LL << 31), "batch too large");
  if (B == 0 || T == 0 || n_act == 0) return PK_OK;
  PK_CHECK_ARG(grad && dir, "null buffer");
  ChompDirArgs a{grad, dir, T, n_act, n_cg_iters, grad_clip_norm, smoothness_reg, cg_tol, covariant ? 1 : 0, active};
  int warps = n_act < 8 ? n_act : 8;
  const size_t smem = sizeof(double) * (size_t)warps * ((T > 2 ? T - 2 : 0) + 4);
  chomp_direction_kernel<<<(unsigned)B, 32 * warps, smem, (cudaStream_t)stream>>>(a);
  return cuda_status(cudaGetLastError(), "chomp_direction_kernel launch");
}

extern "C" int pk_chomp_line_trials(void* stream, const float* traj, const float* dir, const float* alphas,
                                    int32_t n_alphas, float max_delta, const float* start, const float* goal,
                                    float* trials, int64_t B, int32_t T, int32_t n_act, const uint8_t* active) {
  PK_CHECK_ARG(B >= 0 && T >= 0 && n_act >= 0 && n_alphas >= 0, "negative extent");
  const long long per = (long long)B * T * n_act;
  if (per == 0 || n_alphas == 0) return PK_OK;
  PK_CHECK_ARG(traj && dir && alphas && start && goal && trials, "null buffer");
  const long long total = per * n_alphas;
  const long long blocks = std::min<long long>((total + 255) / 256, 148LL * 32);
  chomp_trials_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(traj, dir, alphas, max_delta, start, goal,
                                                                           trials, per, T, n_act, n_alphas, active);
  return cuda_status(cudaGetLastError(), "chomp_trials_kernel launch");
}

extern "C" int pk_chomp_line_select(void* stream, const float* trial_costs, const float* cost, const float* trials,
                                    float* traj, uint8_t* active, int32_t* stall, int32_t n_alphas,
                                    float min_cost_improve, int32_t early_stop_patience, int64_t B, int32_t T,
                                    int32_t n_act) {
  PK_CHECK_ARG(B >= 0 && T >= 0 && n_act >= 0 && n_alphas >= 1, "bad extent");
  PK_CHECK_CAP(B < (1LL << 31), "batch too large");
  if (B == 0) return PK_OK;
  PK_CHECK_ARG(trial_costs && cost && trials && traj && active && stall, "null buffer");
  chomp_select_kernel<<<(unsigned)B, 128, 0, (cudaStream_t)stream>>>(trial_costs, cost, trials, traj, active, stall,
                                                                      min_cost_improve, early_stop_patience, B,
                                                                      (long long)T * n_act, n_alphas);
  return cuda_status(cudaGetLastError(), "chomp_select_kernel launch");
}
