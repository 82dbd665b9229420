// Internal interface of the batched (work-queue) IK launchers: the two
// seed-group bodies (pk_lm.cu) and the warp-per-seed body (pk_lm_wide.cu)
// each run one persistent kernel over the items of their robot classes.
#pragma once

#include "pk_obstacles.cuh"
#include "pyroffi_b200.h"

namespace pk {

constexpr int PK_MAX_CLASSES = 8;

// body selector of a class (pk_ik_class.body)
constexpr int kBodySeedGroup = 0;    // TPS lanes per seed, registers (n_act <= 8, one EE)
constexpr int kBodyWarp = 1;         // one warp per seed, shared-memory state (n_act <= 32)
constexpr int kBodySeedGroup16 = 2;  // one lane per seed, registers (n_act <= 16, n_ee <= 2)

struct BatchCall {
  const pk_ik_class* cls;  // host array, n_classes entries
  int n_classes;
  WorldArgs w;
  pk_lm_options opt;
  const int4* items;       // device [n_items] (class, problem, first seed, seed count)
  int n_items;
  int* queue;              // device [2] item counters (cleared by the launcher)
  int blocks;              // persistent grid per kernel; 0 = one full wave
};

// The launch's class table is indexed at run time; reading it with constant
// indices (one case per class) keeps it in parameter space instead of a
// local-memory copy.
template <typename T, typename Table>
__device__ __forceinline__ void pick_class(const Table& tab, int c, T& dst) {
  switch (c) {
    case 0: dst = tab[0]; break;
    case 1: dst = tab[1]; break;
    case 2: dst = tab[2]; break;
    case 3: dst = tab[3]; break;
    case 4: dst = tab[4]; break;
    case 5: dst = tab[5]; break;
    case 6: dst = tab[6]; break;
    default: dst = tab[7]; break;
  }
}
static_assert(PK_MAX_CLASSES == 8, "pick_class covers 8 classes");

// Each launches its persistent kernel when some class uses its body and
// adds the number of kernels launched to *launched.
int launch_seed_group_batch(const BatchCall& b, cudaStream_t st, int* launched);
int launch_warp_batch(const BatchCall& b, cudaStream_t st, int* launched);

// Warp-per-seed LM over a plain (problems x seed blocks) grid, the route of
// pk_ls_ik_ex for robots beyond the seed-group kernel's buckets.
int launch_warp_grid(const pk_ik_class& c, const WorldArgs& w, const pk_lm_options& opt, cudaStream_t st);

}  // namespace pk
