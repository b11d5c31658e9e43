// pairwise.h -- all-pairs frame x frame RMSD matrix (internal interface).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "device_util.cuh"

namespace wmd {

struct PairwiseWorkspace {
  void* centred = nullptr;  // per-frame centred coordinates (layout per mode)
  size_t centred_bytes = 0;
  double* gsum = nullptr;   // [F] sum |x - cx|^2 of the stored coordinates
  double* cen = nullptr;    // [F][3] centroids
  size_t frames_cap = 0;
  void* extra = nullptr;    // mode-specific scratch
  size_t extra_bytes = 0;
  WaitCfg wait;             // limits of the tensor-core kernel's bounded waits
  // Partition of the upper triangle over `parts` callers (one per GPU): a
  // launch computes only the tiles whose tile row is part (mod parts), and
  // leaves every other entry zero, so the parts sum to the whole matrix.
  int part = 0, parts = 1;
};

void pairwise_workspace_free(PairwiseWorkspace& w);

// Fills out[n_frames][n_frames] (device, row-major float32).  Returns 0 or a
// WMD_ERR_* code with a message in *msg.
int pairwise_run(PairwiseWorkspace& w, int sm_count, const float* coords, int64_t n_frames, int64_t n_atoms,
                 int stride, const uint32_t* sel, int64_t n_sel, int metric, int mode, float* out, int* status,
                 cudaStream_t s, std::string* msg);

}  // namespace wmd
