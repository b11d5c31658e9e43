// wmd_internal.h -- launch parameters shared between the host API
// (wmd_api.cu) and the kernel files.  Not part of the public C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_util.cuh"

namespace wmd {

// Per-frame kernel geometry: 4 warps per CTA (thread 0 also issues the bulk
// copies); each thread owns 8 atoms of a 1024-atom tile, whose reference
// coordinates it keeps in registers (FP64, centred) while frames stream past.
constexpr int kConsumerWarps = 4;
constexpr int kConsumerThreads = kConsumerWarps * 32;
constexpr int kThreads = kConsumerThreads;
constexpr int kStatDoubles = 16;  // per-frame / per-tile partial record

// Which outputs a per-frame forward launch writes.
struct FrameOutputs {
  double* rmsd = nullptr;   // [n_frames]
  double* stats = nullptr;  // [n_frames][16]
  float* cov = nullptr;     // [n_frames][9]
  float* sum_x2 = nullptr;  // [n_frames]
  float* sum_y2 = nullptr;  // [n_frames]
};

struct RefInfo {
  const double* yc = nullptr;  // device [n_sel][3]: y - mean(y) in FP64 (weighted: w (y - mean_w(y)))
  const float* w = nullptr;    // device [n_sel] per-atom weights (masses), or null
  int64_t n_sel = 0;
  double sum_c[3] = {0, 0, 0};  // sum of yc (round-off residue of the centring)
  double gy = 0;                // sum |yc - mean(yc)|^2
  double mean[3] = {0, 0, 0};   // mean(y), for the no-fit RMSD
  double sumsq = 0;             // sum |y|^2, for the no-fit RMSD
  double wsum = 0;              // sum of the weights (n_sel when unweighted)
};

struct FrameLaunch {
  const float* coords = nullptr;  // device, frames of this launch
  int64_t n_frames = 0;
  int64_t n_atoms = 0;            // frame stride in atoms
  int stride = 3;                 // floats per atom (3 or 4)
  const uint32_t* sel = nullptr;  // device indices, or null (dense 0..n_sel-1)
  bool gather = false;            // plain loads (selection or unaligned base)
  int tile_atoms = 2048;          // atoms per tile (kConsumerThreads * atoms/thread, or kLaneTile)
  bool lanes = false;             // frames-across-lanes forward kernel (rmsd_lanes.cu)
  int lane_warps = 0;             // its active warps (set at launch)
  int64_t lane_atom0 = 0;         // its atoms: [lane_atom0, lane_atom0 + lane_atoms) of every frame
  int64_t lane_atoms = 0;
  const double* lane_y = nullptr; // reference values over those atoms (centred, weighted), +32 zero atoms
  const float* lane_w = nullptr;  // per-atom weights over those atoms, or null (all 1)
  int align = 1;
  RefInfo ref;
  FrameOutputs out;
  // backward
  const double* rot = nullptr;  // [n_frames][16] from the backward prologue
  float* grad = nullptr;        // [n_frames][n_atoms][3]
  // scratch
  double* partial = nullptr;    // [n_frames][n_tiles][16] per-tile sums
  double* refine = nullptr;     // [n_frames][16] records of frames needing the residual pass
  unsigned* refine_count = nullptr;  // number of records, zeroed before each forward
  int* status = nullptr;        // device-visible status word (mapped host)
  WaitCfg wait;                 // limits of the bounded waits
  int grid = 0;                 // CTAs (persistent)
};

// A frame whose RMSD is below kRefineScale * (G_x + G_y) / n (A^-1 * A^2) is
// recomputed from explicit residuals: there the one-pass G_x + G_y - 2 lambda
// route would leave cancellation noise of ~1e-14 (G_x + G_y) / n in the MSD.
constexpr double kRefineScale = 1e-7;

// Records the message wmd_last_error(NULL) returns on this thread.
void set_thread_error(const char* msg);

int frame_tiles(const FrameLaunch& L);
// Picks the forward kernel for a launch (sets lanes and tile_atoms); call
// before sizing the partials with frame_tiles.
void frame_plan(FrameLaunch& L, int sm_count);
// frames-across-lanes forward (rmsd_lanes.cu): at most 2,048 atoms per
// partial record
constexpr int kLaneTile = 2048;
bool lanes_eligible(const FrameLaunch& L);
bool lanes_worthwhile(const FrameLaunch& L, int sm_count);
int lanes_tile(const FrameLaunch& L, int sm_count);
int lanes_grid(const FrameLaunch& L, int sm_count);
cudaError_t launch_lanes_forward(const FrameLaunch& L, bool raw, cudaStream_t s);
// Expands a strictly increasing device selection's reference values (yc
// [n_sel][3]) and weights (w, or all 1 when null) onto the atom span starting
// at a0, into zeroed buffers.
cudaError_t launch_lanes_expand(const uint32_t* sel, int64_t n_sel, int64_t a0, const double* yc, const float* w,
                                double* y_exp, float* w_exp, cudaStream_t s);
size_t frame_smem_bytes(int stride, int tile_atoms);
// Forward: zeroes L.refine_count, runs the fused kernel, then the residual pass
// over the frames it flagged.
cudaError_t launch_rmsd_forward(const FrameLaunch& L, cudaStream_t s);
// Only the streaming kernel of the aligned forward (tile partials into
// L.partial); the caller finishes the frames itself.
cudaError_t launch_rmsd_stream(const FrameLaunch& L, cudaStream_t s);
// Only the streaming kernel, weighted statistics: per tile sum w x (3),
// sum w x_a^2 (3) and sum x (w y_c)^T (9) into L.partial (needs L.ref.w).
cudaError_t launch_rmsd_stream_weighted(const FrameLaunch& L, cudaStream_t s);
// Per-frame dL/drmsd: grad_f64[f * grad_stride] when grad_f64 is set, else
// grad_rmsd[f], else 1.
cudaError_t launch_rmsd_backward(const FrameLaunch& L, const double* stats, const float* grad_rmsd,
                                 const double* grad_f64, int64_t grad_stride, double* rot_scratch, cudaStream_t s);
// occupancy-derived persistent grid for a launch
int frame_grid(const FrameLaunch& L, int sm_count, bool backward);
// The gathered kernel's (tile, frame) partials for L's frames with tiles of
// L.tile_atoms over a dense selection: the frames-across-lanes kernel's layout,
// for frames it leaves to others (raw: the no-fit record).
cudaError_t launch_gather_partials(const FrameLaunch& L, bool raw, int sm_count, cudaStream_t s);

// Whole-frame kernels for many frames of up to kVgMaxAtoms atoms
// (rmsd_vg.cu): forward (rmsd and the 16-double records of
// wmd_rmsd_forward), backward (gradient from those records) and both in one
// launch.  Dense selections of packed xyz only.
constexpr int64_t kVgMaxAtoms = 16384;
enum VgMode : int { kVgFwd = 0, kVgBwd = 1, kVgBoth = 2 };
struct VgLaunch {
  const float* coords = nullptr;  // device [n_frames][n_atoms][3], 16-byte aligned
  int64_t n_frames = 0, n_atoms = 0;
  RefInfo ref;                    // dense reference (n_sel == n_atoms)
  double* rmsd = nullptr;         // [n_frames] or null
  double* stats = nullptr;        // [n_frames][16]: written (forward), read (backward), or null (both)
  const void* w = nullptr;        // per-frame dL/drmsd (backward, both), null = 1
  int w_f64 = 0;                  // w holds doubles (else floats)
  int64_t w_stride = 1;           // elements between frames' weights (0: one shared weight)
  float* grad = nullptr;          // [n_frames][n_atoms][3], 16-byte aligned (backward, both)
  int* status = nullptr;
  WaitCfg wait;
};
bool vg_usable(const float* coords, const float* grad, int64_t n_frames, int64_t n_atoms, int stride, int sm_count);
// On failure *why (when given) names the step: a tensor map or the launch.
cudaError_t launch_vg(int mode, const VgLaunch& V, int sm_count, cudaStream_t s, const char** why = nullptr);

}  // namespace wmd
