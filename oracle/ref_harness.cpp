// Host build of the reference's own CUDA helper functions -- test infrastructure only.
//
// The reference's device helpers (src/pyroffi/cuda_kernels/_fk_cuda_helpers.cuh,
// _ik_cuda_helpers.cuh, _collision_cuda_helpers.cuh) depend on nothing but
// <cuda_runtime.h> and <cmath>, so g++ compiles them for the CPU straight
// from the reference tree (see oracle/Makefile).  This file only forwards
// them through extern "C" symbols so tests/golden/make_golden.py can call them
// with ctypes and record golden vectors.  No reference source is copied here.
#include "_ik_cuda_helpers.cuh"
#include "_collision_cuda_helpers.cuh"

extern "C" {

void ref_se3_exp(const float* tangent, float* out) { se3_exp(tangent, out); }

void ref_se3_compose(const float* a, const float* b, float* out) { se3_compose(a, b, out); }

void ref_fk_single(const float* cfg, const float* twists, const float* parent_tf,
                   const int* parent_idx, const int* act_idx, const float* mimic_mul,
                   const float* mimic_off, const int* mimic_act_idx, const int* topo_inv,
                   float* T_world, int n_joints, int n_act) {
  fk_single(cfg, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
            topo_inv, T_world, n_joints, n_act);
}

void ref_multi_ee_residual_and_jacobian(const float* cfg, float* T_world, const float* twists,
                                        const float* parent_tf, const int* parent_idx,
                                        const int* act_idx, const float* mimic_mul,
                                        const float* mimic_off, const int* mimic_act_idx,
                                        const int* topo_inv, const int* target_jnts,
                                        const int* ancestor_masks, const float* target_Ts,
                                        int n_joints, int n_act, int n_ee, float* r, float* J) {
  compute_multi_ee_residual_and_jacobian(cfg, T_world, twists, parent_tf, parent_idx, act_idx,
                                         mimic_mul, mimic_off, mimic_act_idx, topo_inv,
                                         target_jnts, ancestor_masks, target_Ts, n_joints, n_act,
                                         n_ee, r, J);
}

int ref_chol_solve_f64(double* A, double* b, int n) { return chol_solve(A, b, n) ? 1 : 0; }

float ref_sphere_sphere(const float* a, const float* b) {
  return sphere_sphere_dist(a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3]);
}
float ref_sphere_capsule(const float* s, const float* c) {
  return sphere_capsule_dist(s[0], s[1], s[2], s[3], c[0], c[1], c[2], c[3], c[4], c[5], c[6]);
}
float ref_sphere_box(const float* s, const float* b) {
  return sphere_box_dist(s[0], s[1], s[2], s[3], b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7],
                         b[8], b[9], b[10], b[11], b[12], b[13], b[14]);
}
float ref_sphere_halfspace(const float* s, const float* h) {
  return sphere_halfspace_dist(s[0], s[1], s[2], s[3], h[0], h[1], h[2], h[3], h[4], h[5]);
}
float ref_capsule_capsule(const float* a, const float* b) {
  return capsule_capsule_dist(a[0], a[1], a[2], a[3], a[4], a[5], a[6], b[0], b[1], b[2], b[3],
                              b[4], b[5], b[6]);
}
float ref_capsule_box(const float* c, const float* b) {
  return capsule_box_dist(c[0], c[1], c[2], c[3], c[4], c[5], c[6], b[0], b[1], b[2], b[3], b[4],
                          b[5], b[6], b[7], b[8], b[9], b[10], b[11], b[12], b[13], b[14]);
}
float ref_capsule_halfspace(const float* c, const float* h) {
  return capsule_halfspace_dist(c[0], c[1], c[2], c[3], c[4], c[5], c[6], h[0], h[1], h[2], h[3],
                                h[4], h[5]);
}
void ref_apply_se3_point(const float* T, const float* p, float* out) { apply_se3_point(T, p, out); }
float ref_colldist_from_sdf(float d, float margin) { return colldist_from_sdf(d, margin); }

}  // extern "C"
