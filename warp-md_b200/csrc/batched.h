// batched.h -- batched per-frame RMSD over many trajectories (internal).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wmd {

// One trajectory of the batch, as the kernels see it (device-resident table).
struct BatchSeg {
  const float* coords;  // [n_frames][n_atoms][3], 16-byte aligned
  const float* ref;     // [n_atoms][3]
  double* rmsd;         // [n_frames]
  float* grad;          // [n_frames][n_atoms][3] or null
  double* yc;           // centred reference [n_atoms][3] (workspace)
  int64_t n_atoms;
  int64_t n_frames;
  int64_t item0;        // first global work item (items: n_tiles x n_frames)
  int64_t frame0;       // first global frame
  int n_tiles;
  int pad;
  double sum_c[3];      // sum of y_c, written on the device each call
  double gy;            // G_y, written on the device each call
};

struct BatchLaunch {
  const BatchSeg* segs = nullptr;
  int n_segs = 0;
  int64_t total_items = 0;
  int64_t total_frames = 0;
  double* partial = nullptr;         // [total_items][16]
  double* stats = nullptr;           // [total_frames][16] (with gradients)
  double* rot = nullptr;             // [total_frames][16] (with gradients)
  double* refine = nullptr;          // [total_frames][16]
  unsigned* refine_count = nullptr;
  int* status = nullptr;
};

struct BatchPlan {
  BatchLaunch launch;
  BatchSeg* segs_dev = nullptr;
  int n_segs = 0;
  int apt = 8;       // atoms per thread: 4 (512-atom tiles) or 8 (1024-atom tiles)
  int grid_fwd = 0;
  int grid_bwd = 0;
};

int batched_tile_atoms(int apt);
int batched_grid(int apt, bool backward, int sm_count, int64_t items);
// Enqueues the whole batched pipeline on s (no allocation, no host sync).
cudaError_t batched_enqueue(const BatchPlan& P, bool with_grad, cudaStream_t s);

}  // namespace wmd
