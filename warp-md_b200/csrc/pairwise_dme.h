// pairwise_dme.h -- all-pairs distance-matrix error (PairwiseRmsdPlan metric "dme").
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wmd {

// out[i][j] = sqrt(sum_k (d_i[k] - d_j[k])^2 / n_pairs) over the atom pairs
// k = (a < b) of the selection, zero diagonal, symmetric; all zeros when
// n_sel < 2.  coords, sel, box and out are device pointers; box holds
// per-frame orthorhombic lengths [n_frames][3] or is null (no PBC).
cudaError_t launch_pair_dme(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                            int64_t n_sel, const float* box, float* out, int* status, cudaStream_t s);

}  // namespace wmd
