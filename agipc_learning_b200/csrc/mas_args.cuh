// mas_args.cuh -- what the MAS apply kernels read about the hierarchy and
// the stored inverses, and the prolongation of the coarse levels to a fine
// slot (shared by the apply kernels and the fused PCG iteration kernel).
#pragma once
#include "maspcg_internal.cuh"

namespace maspcg {

struct ApplyArgs {
  const int* cmap1;
  const int* cmap[kMaxLevels];  // fine slot -> level-l local node (-1 padding), l >= 1
  const int* pmr;               // part_map_real: -1 marks a padding slot
  const int* going_next;
  float* coarse_r;
  float* coarse_z;
  const void* inv;
  const float* scale;
  int* chain_count;             // per coarse domain: arrivals so far (zero between launches)
  const int* chain_target;      // per coarse domain: arrivals that complete it
  double* chain_dot;            // per coarse domain: R.Z
  int* err;
  int fem_off, c0;
  LevelInfo lv;
};

// Coarse correction of a level-0 slot: the sum over the coarse levels of the
// level's z at the slot's ancestor (the prolongation, CollectFinalZ).  Returns
// false for a padding slot, whose z is zero.  The ancestors are loaded
// together with the padding mark (none depends on another), so the
// correction costs two dependent loads, not three.
__device__ __forceinline__ bool coarse_correction(const ApplyArgs& a, int slot, float c[3])
{
  c[0] = c[1] = c[2] = 0.f;
  int node[kMaxLevels];
#pragma unroll
  for (int l = 1; l < kMaxLevels; ++l) node[l] = l < a.lv.levelnum ? __ldg(a.cmap[l] + slot) : -1;
  if (a.pmr[slot] < 0) return false;
#pragma unroll
  for (int l = 1; l < kMaxLevels; ++l) {
    if (l < a.lv.levelnum) {
      const float* q = a.coarse_z + 3 * (size_t)(a.lv.begin[l] - a.c0 + node[l]);
      c[0] += q[0];
      c[1] += q[1];
      c[2] += q[2];
    }
  }
  return true;
}

ApplyArgs mas_apply_args(maspcg_handle* h);

}  // namespace maspcg
