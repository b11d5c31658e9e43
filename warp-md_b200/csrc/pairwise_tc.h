// pairwise_tc.h -- tensor-core (tcgen05) forms of the pairwise RMSD matrix.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "device_util.cuh"
#include "pairwise.h"

namespace wmd {

// limbs = 3 (24-bit fixed point) or 2 (16-bit); see pairwise_tc.cu.
int pairwise_tc_run(PairwiseWorkspace& w, int sm_count, const float* coords, int64_t n_frames, int64_t n_atoms,
                    int stride, const uint32_t* sel, int64_t n_sel, int metric, int limbs, float* out, int* status,
                    const WaitCfg& wait, cudaStream_t s, std::string* msg);

}  // namespace wmd
