// FP32 damped least-squares step with one conditional FP64 refinement step,
// shared by the HJCD and SQP refinement kernels.
//
// Over the free columns F (free[c]), with the other columns N held at
// x_N = xn_N, it solves
//
//   (Js_F^T Js_F + diag(lam + pd_F)) x_F = -(Js_F^T (fw + Js_N xn_N) + v_F)
//
// for a column-scaled Jacobian Js (R rows, MAXA columns), a residual fw, the
// damping lam > 0, an extra diagonal pd >= 0 and an extra right-hand side v
// (HJCD's joint-limit prior: pd = w / (h^2 s^2), v = w (q - mid) / (h^2 s)).
// Masked columns of the reference kernels' MAXA x MAXA systems (an identity
// row with right-hand side 0, _sqp_ik_cuda_kernel.cu and
// _hjcd_ik_cuda_kernel.cu) are the N columns here: fixed joints with
// xn = 0, and SQP's active-set re-solves with the bound-holding joints at
// xn = p_bound, whose coupling g_F + H_FN p_N = Js_F^T (fw + Js_N p_N)
// enters through the right-hand side as above.
//
// R < MAXA and at least as many free columns as live rows (one or two EEs of
// a redundant arm): the R x R dual form.  With
// W_c = lam / (lam + pd_c) and u_c = v_c / (lam + pd_c) on F, W_c = 0 and
// u_c = -xn_c on N, the same step is
//
//   (Js W Js^T + lam I) z = fw - Js u,   x = -u - W Js^T z
//
// (the Woodbury form of the primal system, multiplied through by lam; with
// pd = v = 0 it is the push-through identity (Js^T Js + lam I)^-1 Js^T =
// Js^T (Js Js^T + lam I)^-1).  Its eigenvalues are sigma_i(Js W^1/2)^2 + lam:
// a redundant arm's null space, which puts an eigenvalue at lam itself into
// the MAXA x MAXA system, does not appear.  Otherwise the primal system,
// whose free columns then number at most the rows: with fewer free columns
// than rows (fixed joints, or joints held at a bound) the dual system would
// carry the null space of Js_F^T as eigenvalues lam instead.
//
// Either system and its Cholesky are FP32; when the squared ratio of the
// largest to the smallest pivot (over the first `rows` rows of the dual, or
// the free rows of the primal) exceeds 1e6, one step of iterative refinement
// follows: the residual in FP64 from the FP32 entries (which FP64 holds
// exactly), the correction solved with the FP32 factor.  A non-positive
// pivot gives x = 0 and returns false, as the reference's Cholesky does.
#pragma once

namespace pk {

// squared pivot ratio above which one FP64 refinement step follows
constexpr float kDampedRefineRatio = 1e6f;

template <int N>
struct PackedChol {
  float L[N * (N + 1) / 2];  // lower triangle, diagonal as its reciprocal

  // In-place factor of the packed matrix already in L; pivots of rows with
  // use[k] feed the ratio test.  Returns false on a non-positive pivot.
  template <typename Use>
  __device__ __forceinline__ bool factor(Use use, float& pmax, float& pmin) {
    bool ok = true;
    pmax = 0.f;
    pmin = 3.4e38f;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      float s2 = L[k * (k + 1) / 2 + k];
#pragma unroll
      for (int q = 0; q < k; ++q) s2 = fmaf(-L[k * (k + 1) / 2 + q], L[k * (k + 1) / 2 + q], s2);
      if (!(s2 > 0.f)) ok = false;
      if (use(k)) {
        pmax = fmaxf(pmax, s2);
        pmin = fminf(pmin, s2);
      }
      const float inv = 1.f / sqrtf(ok ? s2 : 1.f);
      L[k * (k + 1) / 2 + k] = inv;
#pragma unroll
      for (int i = k + 1; i < N; ++i) {
        float tt = L[i * (i + 1) / 2 + k];
#pragma unroll
        for (int q = 0; q < k; ++q) tt = fmaf(-L[i * (i + 1) / 2 + q], L[k * (k + 1) / 2 + q], tt);
        L[i * (i + 1) / 2 + k] = tt * inv;
      }
    }
    return ok;
  }

  __device__ __forceinline__ void solve(float (&b)[N]) const {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      float s2 = b[i];
#pragma unroll
      for (int q = 0; q < i; ++q) s2 = fmaf(-L[i * (i + 1) / 2 + q], b[q], s2);
      b[i] = s2 * L[i * (i + 1) / 2 + i];
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
      float s2 = b[i];
#pragma unroll
      for (int q = i + 1; q < N; ++q) s2 = fmaf(-L[q * (q + 1) / 2 + i], b[q], s2);
      b[i] = s2 * L[i * (i + 1) / 2 + i];
    }
  }
};

// Dual form (see above); `rows` <= R residual rows are live (the rest are
// zero padding).
template <int R, int MAXA>
__device__ __forceinline__ bool damped_step_dual(const float (&J)[R][MAXA], const float (&fw)[R], int rows, float lam,
                                                 const float (&pd)[MAXA], const bool (&fr)[MAXA],
                                                 const float (&xn)[MAXA], const float (&v)[MAXA], float (&x)[MAXA]) {
  float w[MAXA], u[MAXA];
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    const float d = lam + pd[c];
    w[c] = fr[c] ? lam / d : 0.f;
    u[c] = fr[c] ? v[c] / d : -xn[c];
  }
  PackedChol<R> M;
  float z[R], rhs[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      float acc = (i == j) ? lam : 0.f;
#pragma unroll
      for (int c = 0; c < MAXA; ++c)
        if (fr[c]) acc = fmaf(J[i][c] * w[c], J[j][c], acc);
      M.L[i * (i + 1) / 2 + j] = acc;
    }
    float b = fw[i];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) b = fmaf(-J[i][c], u[c], b);
    rhs[i] = z[i] = b;
  }
  float pmax, pmin;
  const bool ok = M.factor([&](int k) { return k < rows; }, pmax, pmin);
  M.solve(z);
  if (ok && pmax > kDampedRefineRatio * pmin) {
    double t[MAXA];
#pragma unroll
    for (int c = 0; c < MAXA; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < R; ++k) acc = fma((double)J[k][c], (double)z[k], acc);
      t[c] = fr[c] ? acc * (double)w[c] : 0.0;
    }
    float d[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      double acc = (double)lam * (double)z[i];
#pragma unroll
      for (int c = 0; c < MAXA; ++c) acc = fma((double)J[i][c], t[c], acc);
      d[i] = (float)((double)rhs[i] - acc);
    }
    M.solve(d);
#pragma unroll
    for (int i = 0; i < R; ++i) z[i] = (float)((double)z[i] + (double)d[i]);
  }
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    float pc = 0.f;
#pragma unroll
    for (int k = 0; k < R; ++k) pc = fmaf(J[k][c], z[k], pc);
    x[c] = ok ? (fr[c] ? -u[c] - w[c] * pc : xn[c]) : 0.f;
  }
  return ok;
}

// Primal form: the free rows of (Js^T Js + diag(lam + pd)), identity rows
// (right-hand side xn) elsewhere.
template <int R, int MAXA>
__device__ __forceinline__ bool damped_step_primal(const float (&J)[R][MAXA], const float (&fw)[R], float lam,
                                                   const float (&pd)[MAXA], const bool (&fr)[MAXA],
                                                   const float (&xn)[MAXA], const float (&v)[MAXA],
                                                   float (&x)[MAXA]) {
  float f2[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    float b = fw[k];
#pragma unroll
    for (int c = 0; c < MAXA; ++c)
      if (!fr[c]) b = fmaf(J[k][c], xn[c], b);
    f2[k] = b;
  }
  PackedChol<MAXA> A;
  float rhs[MAXA];
#pragma unroll
  for (int i = 0; i < MAXA; ++i) {
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < R; ++k) acc = fmaf(J[k][i], J[k][j], acc);
      if (i == j) acc += lam + pd[i];
      A.L[i * (i + 1) / 2 + j] = (fr[i] && fr[j]) ? acc : (i == j ? 1.f : 0.f);
    }
    float g = v[i];
#pragma unroll
    for (int k = 0; k < R; ++k) g = fmaf(J[k][i], f2[k], g);
    rhs[i] = x[i] = fr[i] ? -g : xn[i];
  }
  float pmax, pmin;
  const bool ok = A.factor([&](int k) { return fr[k]; }, pmax, pmin);
  A.solve(x);
  if (ok && pmax > kDampedRefineRatio * pmin) {
    double s[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      double acc = 0.0;
#pragma unroll
      for (int c = 0; c < MAXA; ++c)
        if (fr[c]) acc = fma((double)J[k][c], (double)x[c], acc);
      s[k] = acc;
    }
    float d[MAXA];
#pragma unroll
    for (int i = 0; i < MAXA; ++i) {
      double acc = ((double)lam + (double)pd[i]) * (double)x[i];
#pragma unroll
      for (int k = 0; k < R; ++k) acc = fma((double)J[k][i], s[k], acc);
      d[i] = fr[i] ? (float)((double)rhs[i] - acc) : 0.f;
    }
    A.solve(d);
#pragma unroll
    for (int i = 0; i < MAXA; ++i) x[i] = (float)((double)x[i] + (double)d[i]);
  }
#pragma unroll
  for (int c = 0; c < MAXA; ++c) x[c] = ok ? (fr[c] ? x[c] : xn[c]) : 0.f;
  return ok;
}

// The primal form out of line, for the rare case of a dual-form caller with
// fewer free columns than live rows: its MAXA x MAXA factor then takes no
// registers from the caller's hot path (the system goes through local memory).
template <int R, int MAXA>
struct DampedSystem {
  float J[R][MAXA];
  float fw[R];
  float pd[MAXA], xn[MAXA], v[MAXA];
  bool fr[MAXA];
  float lam;
};

template <int R, int MAXA>
__device__ __noinline__ bool damped_step_primal_cold(const DampedSystem<R, MAXA>* s, float* x) {
  float xr[MAXA];
  const bool ok = damped_step_primal<R, MAXA>(s->J, s->fw, s->lam, s->pd, s->fr, s->xn, s->v, xr);
#pragma unroll
  for (int c = 0; c < MAXA; ++c) x[c] = xr[c];
  return ok;
}

template <int R, int MAXA>
__device__ __forceinline__ bool damped_step_primal_ool(const float (&J)[R][MAXA], const float (&fw)[R], float lam,
                                                       const float (&pd)[MAXA], const bool (&fr)[MAXA],
                                                       const float (&xn)[MAXA], const float (&v)[MAXA],
                                                       float (&x)[MAXA]) {
  DampedSystem<R, MAXA> s;
#pragma unroll
  for (int k = 0; k < R; ++k) {
#pragma unroll
    for (int c = 0; c < MAXA; ++c) s.J[k][c] = J[k][c];
    s.fw[k] = fw[k];
  }
#pragma unroll
  for (int c = 0; c < MAXA; ++c) {
    s.pd[c] = pd[c];
    s.xn[c] = xn[c];
    s.v[c] = v[c];
    s.fr[c] = fr[c];
  }
  s.lam = lam;
  float xo[MAXA];
  const bool ok = damped_step_primal_cold<R, MAXA>(&s, xo);
#pragma unroll
  for (int c = 0; c < MAXA; ++c) x[c] = xo[c];
  return ok;
}

// The step described above: the dual form when R < MAXA and the free
// columns are at least the `rows` live residual rows, else the primal form
// (the smaller of the two systems that is not rank-deficient; out of line
// when the dual form is the usual one).  Writes x on every column; returns
// false (x = 0) on a non-positive pivot.
template <int R, int MAXA>
__device__ __forceinline__ bool damped_step_f32(const float (&J)[R][MAXA], const float (&fw)[R], int rows, float lam,
                                                const float (&pd)[MAXA], const bool (&fr)[MAXA],
                                                const float (&xn)[MAXA], const float (&v)[MAXA], float (&x)[MAXA]) {
  if constexpr (R < MAXA) {
    int nf = 0;
#pragma unroll
    for (int c = 0; c < MAXA; ++c) nf += fr[c] ? 1 : 0;
    if (nf >= rows) return damped_step_dual<R, MAXA>(J, fw, rows, lam, pd, fr, xn, v, x);
    if constexpr (MAXA <= 8) return damped_step_primal<R, MAXA>(J, fw, lam, pd, fr, xn, v, x);
    else return damped_step_primal_ool<R, MAXA>(J, fw, lam, pd, fr, xn, v, x);
  } else {
    return damped_step_primal<R, MAXA>(J, fw, lam, pd, fr, xn, v, x);
  }
}

}  // namespace pk
