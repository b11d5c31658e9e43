// batched.h -- batched per-frame RMSD over many trajectories (internal).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

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
  int64_t group0;       // frame-major layout: first global frame group
  int64_t n_groups;     //   groups of this trajectory (m_group frames each, the last may be short)
  int64_t cost0;        //   estimated cost of all groups before this trajectory's
  int64_t group_cost;   //   estimated cost of one full group
  int64_t lane_unit_cost;  // lanes layout: estimated cost of a (tile, 32-frame group) unit of a whole tile
  int64_t lane_last_cost;  //   ... and of a unit of the last tile (the only one when n_atoms <= tile)
  int64_t lane_full_units; //   units of the whole tiles, (n_tiles - 1) x ceil(n_frames / 32); tile-major
  int64_t lane_units;      //   units of this trajectory (n_tiles x ceil(n_frames / 32))
  int64_t lane_cost0;      //   estimated cost of all units before this trajectory's
  int n_tiles;
  int m_group;          //   frames per group
  int tma;              // lanes layout forward: 0 per-lane bulk copies, 1 frame rows, 2 quad rows (tensor map)
  double sum_c[3];      // sum of y_c, written on the device each call
  double gy;            // G_y, written on the device each call
  double mean_y[3];     // mean of the reference, written on the device each call
};

struct BatchLaunch {
  const BatchSeg* segs = nullptr;
  const CUtensorMap* maps = nullptr;  // [n_segs] lanes layout: each trajectory's frames as a 2-D tensor map
  int n_segs = 0;
  int64_t total_items = 0;
  int64_t total_frames = 0;
  int64_t total_groups = 0;          // frame-major layout
  int64_t total_cost = 0;
  int64_t total_lane_cost = 0;       // lanes layout
  double* partial = nullptr;         // [total_items][16]
  double* rot = nullptr;             // [total_frames][16] (with gradients): R, xbar, 1/(n rmsd)
  double* refine = nullptr;          // [total_frames][16]
  unsigned* refine_count = nullptr;
  int* status = nullptr;
};

struct BatchPlan {
  BatchLaunch launch;
  BatchSeg* segs_dev = nullptr;
  int n_segs = 0;
  int apt = 8;       // atoms per thread: 4 (512-atom tiles) or 8 (1024-atom tiles)
  int variant = 0;   // kBatchTiles, kBatchFrames or kBatchLanes
  int grid_fwd = 0;
  int grid_bwd = 0;
};

// Tile-major: work items (atom tile, frame) spread over persistent CTAs, frame
// statistics finished by a second kernel, gradients by a second streaming pass
// (36 B per atom-frame with gradients).  Frame-major: each CTA owns whole
// frames, finishes QCP in-kernel and re-reads the frame from L2 for the
// gradient (24 B per atom-frame from HBM).
// Lanes: the tile-major pipeline with its forward statistics computed frames
// across lanes (a lane per frame of a 32-frame group, no cross-lane
// reduction), the same per-item partials, finisher and gradient pass.
enum BatchVariant : int { kBatchTiles = 0, kBatchFrames = 1, kBatchLanes = 2 };

// Frame-major grouping: up to kGroupFrames consecutive frames of one
// trajectory with at most kGroupBytes of coordinates form a group, whose QCP
// runs on one warp, a lane per frame.  CTAs take runs of groups of equal
// estimated cost: kCostItem per chunk streamed (each pass) + kCostFinish per
// group (QCP and rotation, about six chunk-times of latency).
constexpr int kGroupFrames = 16;
constexpr int kGroupBytes = 64 * 1024;
constexpr int64_t kCostItem = 4;
constexpr int64_t kCostFinish = 24;

// Tensor maps of the lanes layout's forward pass, one per trajectory (64-byte
// aligned host array): frame rows [n_frames][3 n_atoms] floats in 32-row x
// 32-float boxes with 128-byte swizzle when a frame is a multiple of 16 bytes
// (tma = 1), else quad rows [n_frames / 4][12 n_atoms] in 8-row x 100-float
// boxes (tma = 2; the last n_frames mod 4 frames are read with plain loads).
// Trajectories with fewer than 4 frames, no atoms, or with
// WARPMD_BATCHED_TMA=0, keep per-lane bulk copies (tma = 0).  Returns false
// with *msg set when the driver's encoder is unavailable or refuses a map.
bool batched_encode_maps(std::vector<BatchSeg>& segs, CUtensorMap* maps, std::string* msg);

int batched_tile_atoms(int apt);
int batched_grid(int apt, bool backward, int sm_count, int64_t items);
int batched_frame_grid(int apt, bool with_grad, int sm_count, int64_t groups);
int batched_lanes_grid(int sm_count, int64_t units);
// Enqueues the whole batched pipeline on s (no allocation, no host sync).
cudaError_t batched_enqueue(const BatchPlan& P, bool with_grad, cudaStream_t s);

}  // namespace wmd
