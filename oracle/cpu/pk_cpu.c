/*
 * CPU port of the hot path (FP32, OpenMP) -- test / baseline infrastructure only.
 *
 * This is the oracle's C form, used as the timed CPU baseline ("port"): the
 * reference's own CPU path is JAX (jax, jaxlie), which this image does not
 * have.  It restates, per configuration / seed and in FP32 like the
 * reference's CUDA kernels:
 *   - fk_single (src/pyroffi/cuda_kernels/_fk_cuda_helpers.cuh:158-208),
 *   - compute_multi_ee_residual_and_jacobian (_ik_cuda_helpers.cuh:433-551),
 *   - ls_ik_lm_kernel (src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:65-394)
 *     with FP64 normal equations and Cholesky, plus optional explicit
 *     robot-sphere self pairs and configurable damping factors,
 *   - FK + sphere transform + min signed distance vs world spheres.
 * Parallel over seeds / configurations with OpenMP.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#define CMAXJ 64
#define CMAXA 32
#define CMAXE 4

typedef struct {
  const float *twists, *parent_tf, *mimic_mul, *mimic_off;
  const int32_t *parent_idx, *act_idx, *mimic_act_idx, *topo_inv;
  int n_joints, n_act;
} cmodel;

static void qmul(const float* a, const float* b, float* o) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

static void qrot(const float* q, const float* v, float* o) {
  const float w = q[0], x = q[1], y = q[2], z = q[3];
  const float cx = y * v[2] - z * v[1], cy = z * v[0] - x * v[2], cz = x * v[1] - y * v[0];
  const float ccx = y * cz - z * cy, ccy = z * cx - x * cz, ccz = x * cy - y * cx;
  o[0] = v[0] + 2.f * w * cx + 2.f * ccx;
  o[1] = v[1] + 2.f * w * cy + 2.f * ccy;
  o[2] = v[2] + 2.f * w * cz + 2.f * ccz;
}

static void compose(const float* a, const float* b, float* o) {
  float r[3];
  qmul(a, b, o);
  qrot(a, b + 4, r);
  o[4] = r[0] + a[4];
  o[5] = r[1] + a[5];
  o[6] = r[2] + a[6];
}

static void se3exp(const float* t, float* o) {
  const float vx = t[0], vy = t[1], vz = t[2], ox = t[3], oy = t[4], oz = t[5];
  const float th2 = ox * ox + oy * oy + oz * oz;
  if (th2 < 1e-12f) {
    o[0] = 1.f; o[1] = o[2] = o[3] = 0.f;
    o[4] = vx; o[5] = vy; o[6] = vz;
    return;
  }
  const float th = sqrtf(th2);
  const float sh = sinf(0.5f * th), ch = cosf(0.5f * th);
  const float s = sh / th;
  o[0] = ch; o[1] = s * ox; o[2] = s * oy; o[3] = s * oz;
  /* t = (I + B [w]x + C [w]x^2) v as jaxlie SE3.exp */
  const float st = sinf(th), ct = cosf(th);
  const float B = (1.f - ct) / th2, C = (th - st) / (th2 * th);
  const float cx = oy * vz - oz * vy, cy = oz * vx - ox * vz, cz = ox * vy - oy * vx;
  const float od = ox * vx + oy * vy + oz * vz;
  o[4] = vx + B * cx + C * (ox * od - th2 * vx);
  o[5] = vy + B * cy + C * (oy * od - th2 * vy);
  o[6] = vz + B * cz + C * (oz * od - th2 * vz);
}

static void fk(const cmodel* m, const float* cfg, float* Tw) {
  for (int i = 0; i < m->n_joints; ++i) {
    const int j = m->topo_inv[i];
    const int src = (m->mimic_act_idx[j] != -1) ? m->mimic_act_idx[j] : m->act_idx[j];
    const float q = ((src == -1) ? 0.f : cfg[src]) * m->mimic_mul[j] + m->mimic_off[j];
    float Tpc[7];
    if (src == -1 && m->mimic_off[j] == 0.f) {
      memcpy(Tpc, m->parent_tf + 7 * j, sizeof(Tpc));
    } else {
      float tg[6], d[7];
      for (int k = 0; k < 6; ++k) tg[k] = m->twists[6 * j + k] * q;
      se3exp(tg, d);
      compose(m->parent_tf + 7 * j, d, Tpc);
    }
    const int p = m->parent_idx[j];
    if (p == -1) memcpy(Tw + 7 * j, Tpc, sizeof(Tpc));
    else compose(Tw + 7 * p, Tpc, Tw + 7 * j);
  }
}

static void residual(const float* Tw, const int32_t* tj, const float* tgt, int n_ee, float* r) {
  for (int e = 0; e < n_ee; ++e) {
    const float* T = Tw + 7 * tj[e];
    const float* g = tgt + 7 * e;
    float* re = r + 6 * e;
    re[0] = T[4] - g[4]; re[1] = T[5] - g[5]; re[2] = T[6] - g[6];
    const float gi[4] = {g[0], -g[1], -g[2], -g[3]};
    float q[4];
    qmul(T, gi, q);
    if (q[0] < 0.f) { q[0] = -q[0]; q[1] = -q[1]; q[2] = -q[2]; q[3] = -q[3]; }
    const float sh = sqrtf(q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const float f = (sh > 1e-6f) ? 2.f * atan2f(sh, q[0]) / sh : 2.f;
    re[3] = q[1] * f; re[4] = q[2] * f; re[5] = q[3] * f;
  }
}

static void jacobian(const cmodel* m, const float* Tw, const int32_t* tj, const int32_t* anc,
                     int n_ee, float* J) {
  const int na = m->n_act;
  memset(J, 0, sizeof(float) * 6 * n_ee * na);
  for (int j = 0; j < m->n_joints; ++j) {
    const int a1 = m->act_idx[j], a2 = m->mimic_act_idx[j];
    if (a1 < 0 && a2 < 0) continue;
    const float* tw = m->twists + 6 * j;
    const float ang2 = tw[3] * tw[3] + tw[4] * tw[4] + tw[5] * tw[5];
    const float lin2 = tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2];
    float ax[3], z[3];
    int rev;
    if (ang2 > 1e-6f) {
      const float inv = 1.f / sqrtf(ang2);
      ax[0] = tw[3] * inv; ax[1] = tw[4] * inv; ax[2] = tw[5] * inv; rev = 1;
    } else if (lin2 > 1e-6f) {
      const float inv = 1.f / sqrtf(lin2);
      ax[0] = tw[0] * inv; ax[1] = tw[1] * inv; ax[2] = tw[2] * inv; rev = 0;
    } else {
      continue;
    }
    qrot(Tw + 7 * j, ax, z);
    const float* pj = Tw + 7 * j + 4;
    for (int e = 0; e < n_ee; ++e) {
      if (!anc[e * m->n_joints + j]) continue;
      const float* pe = Tw + 7 * tj[e] + 4;
      float c[6];
      if (rev) {
        const float d0 = pe[0] - pj[0], d1 = pe[1] - pj[1], d2 = pe[2] - pj[2];
        c[0] = z[1] * d2 - z[2] * d1; c[1] = z[2] * d0 - z[0] * d2; c[2] = z[0] * d1 - z[1] * d0;
        c[3] = z[0]; c[4] = z[1]; c[5] = z[2];
      } else {
        c[0] = z[0]; c[1] = z[1]; c[2] = z[2]; c[3] = c[4] = c[5] = 0.f;
      }
      const float s = m->mimic_mul[j];
      for (int k = 0; k < 6; ++k) {
        if (a1 >= 0) J[(6 * e + k) * na + a1] += s * c[k];
        if (a2 >= 0) J[(6 * e + k) * na + a2] += s * c[k];
      }
    }
  }
}

typedef struct {
  const float* rs; const int32_t* rsj; int n_rs;
  const float* ws; int Ms;
  const int32_t* si; const int32_t* sj; int n_self;
  float margin, weight;
  int enable;
} cpen;

static float penalty(const cmodel* m, const cpen* c, const float* Tw) {
  if (!c->enable || c->n_rs <= 0) return 0.f;
  float pos[3 * 1024];
  float pen = 0.f;
  for (int i = 0; i < c->n_rs && i < 1024; ++i) {
    const int j = c->rsj[i];
    if (j < 0 || j >= m->n_joints) continue;
    float w[3];
    qrot(Tw + 7 * j, c->rs + 4 * i, w);
    w[0] += Tw[7 * j + 4]; w[1] += Tw[7 * j + 5]; w[2] += Tw[7 * j + 6];
    pos[3 * i] = w[0]; pos[3 * i + 1] = w[1]; pos[3 * i + 2] = w[2];
    const float r = c->rs[4 * i + 3];
    for (int k = 0; k < c->Ms; ++k) {
      const float* o = c->ws + 4 * k;
      const float dx = w[0] - o[0], dy = w[1] - o[1], dz = w[2] - o[2];
      const float d = sqrtf(dx * dx + dy * dy + dz * dz) - (r + o[3]);
      if (d < c->margin) { const float e = d - c->margin; pen += e * e; }
    }
  }
  for (int q = 0; q < c->n_self; ++q) {
    const int a = c->si[q], b = c->sj[q];
    if (a < 0 || b < 0 || a >= c->n_rs || b >= c->n_rs || a >= 1024 || b >= 1024) continue;
    const float dx = pos[3 * a] - pos[3 * b], dy = pos[3 * a + 1] - pos[3 * b + 1], dz = pos[3 * a + 2] - pos[3 * b + 2];
    const float d = sqrtf(dx * dx + dy * dy + dz * dz) - (c->rs[4 * a + 3] + c->rs[4 * b + 3]);
    if (d < c->margin) { const float e = d - c->margin; pen += e * e; }
  }
  return c->weight * pen;
}

static int chol(double* A, double* b, int n) {
  double y[CMAXA];
  for (int k = 0; k < n; ++k) {
    double s = A[k * n + k];
    for (int p = 0; p < k; ++p) s -= A[k * n + p] * A[k * n + p];
    if (s <= 0.0) { for (int i = 0; i < n; ++i) b[i] = 0.0; return 0; }
    const double l = sqrt(s);
    A[k * n + k] = l;
    for (int i = k + 1; i < n; ++i) {
      double t = A[i * n + k];
      for (int p = 0; p < k; ++p) t -= A[i * n + p] * A[k * n + p];
      A[i * n + k] = t / l;
    }
  }
  for (int i = 0; i < n; ++i) {
    double s = b[i];
    for (int p = 0; p < i; ++p) s -= A[i * n + p] * y[p];
    y[i] = s / A[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (int p = i + 1; p < n; ++p) s -= A[p * n + i] * b[p];
    b[i] = s / A[i * n + i];
  }
  return 1;
}

static inline float clampf(float x, float lo, float hi) { return fmaxf(lo, fminf(hi, x)); }

static float weighted(const float* r, int n_ee, float pw, float ow) {
  float e = 0.f;
  for (int k = 0; k < 6 * n_ee; ++k) {
    const float w = (k % 6) < 3 ? pw : ow;
    e += (r[k] * w) * (r[k] * w);
  }
  return e;
}

int pk_cpu_ls_ik(const float* seeds, const float* twists, const float* parent_tf,
                 const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                 const float* mimic_off, const int32_t* mimic_act_idx, const int32_t* topo_inv,
                 const int32_t* target_jnts, const int32_t* ancestor_masks, const float* target_Ts,
                 const float* rs, const int32_t* rsj, const float* ws, const int32_t* self_i,
                 const int32_t* self_j, const float* lower, const float* upper,
                 const int32_t* fixed, float* out_cfg, float* out_err, int P, int Sd, int n_act,
                 int n_joints, int n_ee, int n_rs, int Ms, int n_self, int max_iter, float pw,
                 float ow, float lam0, float lam_down, float lam_up, float eps_pos, float eps_ori,
                 int enable_coll, float coll_w, float margin, int n_threads) {
  if (n_joints > CMAXJ || n_act > CMAXA || n_ee > CMAXE || n_rs > 1024) return 2;
  cmodel m = {twists, parent_tf, mimic_mul, mimic_off, parent_idx, act_idx, mimic_act_idx, topo_inv, n_joints, n_act};
  cpen pc = {rs, rsj, n_rs, ws, Ms, self_i, self_j, n_self, margin, coll_w, enable_coll};
  if (n_threads > 0) omp_set_num_threads(n_threads);
  const long long total = (long long)P * Sd;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long gs = 0; gs < total; ++gs) {
    const int p = (int)(gs / Sd);
    const float* tgt = target_Ts + (size_t)p * n_ee * 7;
    float cfg[CMAXA], best[CMAXA], Tw[CMAXJ * 7], r[6 * CMAXE], J[6 * CMAXE * CMAXA];
    for (int a = 0; a < n_act; ++a) best[a] = cfg[a] = seeds[gs * n_act + a];
    fk(&m, cfg, Tw);
    residual(Tw, target_jnts, tgt, n_ee, r);
    float best_err = weighted(r, n_ee, pw, ow) + penalty(&m, &pc, Tw);
    float lam = lam0;
    for (int it = 0; it < max_iter; ++it) {
      fk(&m, cfg, Tw);
      residual(Tw, target_jnts, tgt, n_ee, r);
      int conv = 1;
      float max_p = 0.f, max_o = 0.f;
      for (int e = 0; e < n_ee; ++e) {
        const float np = sqrtf(r[6 * e] * r[6 * e] + r[6 * e + 1] * r[6 * e + 1] + r[6 * e + 2] * r[6 * e + 2]);
        const float no = sqrtf(r[6 * e + 3] * r[6 * e + 3] + r[6 * e + 4] * r[6 * e + 4] + r[6 * e + 5] * r[6 * e + 5]);
        if (np >= eps_pos || no >= eps_ori) conv = 0;
        max_p = fmaxf(max_p, np);
        max_o = fmaxf(max_o, no);
      }
      if (conv) break;
      jacobian(&m, Tw, target_jnts, ancestor_masks, n_ee, J);
      float fw[6 * CMAXE];
      float curr = 0.f;
      for (int k = 0; k < 6 * n_ee; ++k) {
        const float w = (k % 6) < 3 ? pw : ow;
        fw[k] = r[k] * w;
        curr += fw[k] * fw[k];
        for (int a = 0; a < n_act; ++a) J[k * n_act + a] *= w;
      }
      curr += penalty(&m, &pc, Tw);
      float cs[CMAXA];
      for (int a = 0; a < n_act; ++a) {
        float sq = 0.f;
        for (int k = 0; k < 6 * n_ee; ++k) sq += J[k * n_act + a] * J[k * n_act + a];
        cs[a] = sqrtf(sq) + 1e-8f;
      }
      for (int k = 0; k < 6 * n_ee; ++k)
        for (int a = 0; a < n_act; ++a) J[k * n_act + a] /= cs[a];
      double A[CMAXA * CMAXA], rhs[CMAXA];
      for (int i = 0; i < n_act; ++i) {
        for (int j = 0; j < n_act; ++j) {
          double acc = 0.0;
          for (int k = 0; k < 6 * n_ee; ++k) acc += (double)J[k * n_act + i] * (double)J[k * n_act + j];
          A[i * n_act + j] = acc;
        }
        double rb = 0.0;
        for (int k = 0; k < 6 * n_ee; ++k) rb += (double)J[k * n_act + i] * (double)fw[k];
        rhs[i] = -rb;
        A[i * n_act + i] += (double)lam;
      }
      for (int a = 0; a < n_act; ++a) {
        if (!fixed[a]) continue;
        for (int j = 0; j < n_act; ++j) A[a * n_act + j] = A[j * n_act + a] = 0.0;
        A[a * n_act + a] = 1.0;
        rhs[a] = 0.0;
      }
      chol(A, rhs, n_act);
      float delta[CMAXA], dn = 0.f;
      for (int a = 0; a < n_act; ++a) { delta[a] = (float)rhs[a] / cs[a]; dn += delta[a] * delta[a]; }
      float R;
      if (max_p > 1e-2f || max_o > 0.6f) R = 0.38f;
      else if (max_p > 1e-3f || max_o > 0.25f) R = 0.22f;
      else if (max_p > 2e-4f || max_o > 0.08f) R = 0.12f;
      else R = 0.05f;
      dn = sqrtf(dn);
      if (dn > R) { const float sc = R / (dn + 1e-18f); for (int a = 0; a < n_act; ++a) delta[a] *= sc; }
      static const float alphas[5] = {1.0f, 0.5f, 0.25f, 0.1f, 0.025f};
      float bae = 1e30f;
      int bai = 0;
      for (int ai = 0; ai < 5; ++ai) {
        float tr[CMAXA], rt[6 * CMAXE];
        for (int a = 0; a < n_act; ++a) tr[a] = clampf(cfg[a] + alphas[ai] * delta[a], lower[a], upper[a]);
        fk(&m, tr, Tw);
        residual(Tw, target_jnts, tgt, n_ee, rt);
        const float et = weighted(rt, n_ee, pw, ow) + penalty(&m, &pc, Tw);
        if (et < bae) { bae = et; bai = ai; }
      }
      float tr[CMAXA];
      for (int a = 0; a < n_act; ++a) tr[a] = clampf(cfg[a] + alphas[bai] * delta[a], lower[a], upper[a]);
      if (bae < curr * (1.0f - 1e-4f)) {
        memcpy(cfg, tr, sizeof(float) * n_act);
        lam = fmaxf(lam * lam_down, 1e-10f);
      } else {
        lam = fminf(lam * lam_up, 1e6f);
      }
      if (bae < best_err) { best_err = bae; memcpy(best, tr, sizeof(float) * n_act); }
    }
    memcpy(out_cfg + gs * n_act, best, sizeof(float) * n_act);
    out_err[gs] = best_err;
  }
  return 0;
}

/* FK + link poses + min signed distance of all link spheres vs world spheres. */
int pk_cpu_fk_collision(const float* cfg, const float* twists, const float* parent_tf,
                        const int32_t* parent_idx, const int32_t* act_idx, const float* mimic_mul,
                        const float* mimic_off, const int32_t* mimic_act_idx,
                        const int32_t* topo_inv, const int32_t* parent_joint,
                        const float* link_spheres, const float* ws, float* out_min,
                        float* out_poses, long long B, int n_act, int n_joints, int N, int S,
                        int Ms, int n_threads) {
  if (n_joints > CMAXJ) return 2;
  cmodel m = {twists, parent_tf, mimic_mul, mimic_off, parent_idx, act_idx, mimic_act_idx, topo_inv, n_joints, n_act};
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < B; ++b) {
    float Tw[CMAXJ * 7];
    fk(&m, cfg + b * n_act, Tw);
    float dmin = 1e9f;
    for (int n = 0; n < N; ++n) {
      const int pj = parent_joint[n];
      float T[7] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (pj >= 0) memcpy(T, Tw + 7 * pj, sizeof(T));
      if (out_poses) memcpy(out_poses + (b * N + n) * 7, T, sizeof(T));
      for (int s = 0; s < S; ++s) {
        const float* ls = link_spheres + ((size_t)n * S + s) * 4;
        if (ls[3] < 0.f) continue;
        float w[3];
        qrot(T, ls, w);
        w[0] += T[4]; w[1] += T[5]; w[2] += T[6];
        for (int k = 0; k < Ms; ++k) {
          const float* o = ws + 4 * k;
          const float dx = w[0] - o[0], dy = w[1] - o[1], dz = w[2] - o[2];
          const float d = sqrtf(dx * dx + dy * dy + dz * dz) - (ls[3] + o[3]);
          dmin = fminf(dmin, d);
        }
      }
    }
    out_min[b] = dmin;
  }
  return 0;
}

int pk_cpu_max_threads(void) { return omp_get_max_threads(); }
