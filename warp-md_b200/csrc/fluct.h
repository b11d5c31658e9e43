// fluct.h -- per-atom fluctuations and per-group RMSD (internal; the C ABI is
// in include/warpmd_rmsd.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wmd {

// FP64 moments per selected atom: sum d (3), sum d_c^2 (3), sum d_x d_y,
// d_x d_z, d_y d_z (3), with d = x - (the atom's position in the first frame).
constexpr int kFluctMoments = 9;

// Frame groups of the partial pass for this many atoms and frames.
int fluct_groups(int64_t n_sel, int64_t n_frames, int sm_count);
// shift[n_sel][3] = the selected atoms of the frame at coords; a device-side
// selection index >= n_atoms sets the bad-index bit in *status.
cudaError_t launch_fluct_shift(const float* coords, int64_t n_atoms, int stride, const uint32_t* sel, int64_t n_sel,
                               float* shift, int* status, cudaStream_t s);
// Moments of a run of frames into part[groups][n_sel][9], then added in group
// order into acc[n_sel][9].
cudaError_t launch_fluct_chunk(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                               int64_t n_sel, const float* shift, int groups, double* part, double* acc,
                               cudaStream_t s);
// RMSF [n_sel] and ADP [n_sel][6] (either may be null) from acc over n_frames.
cudaError_t launch_fluct_finalize(const double* acc, int64_t n_sel, int64_t n_frames, float* rmsf, float* adp,
                                  cudaStream_t s);
// Group blocks for launch_group_rmsd: blocks[0..n] (n returned) are group
// indices; block b holds groups [blocks[b], blocks[b+1]).  blocks needs
// n_groups + 1 entries.
int group_blocks(const uint32_t* goff, int64_t n_groups, uint32_t* blocks);
// out[f][g] = sqrt(mean over the group's atoms of |R_f x + t_f - y|^2); xf
// null means R = I, t = 0.  goff [n_groups + 1] indexes gatoms (validated
// atom indices); contig_base >= 0 says gatoms[q] == contig_base + q for every
// q (gatoms is then not read); blocks from group_blocks.
cudaError_t launch_group_rmsd(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const double* xf,
                              const uint32_t* goff, const uint32_t* gatoms, int64_t contig_base,
                              const uint32_t* blocks, int64_t n_blocks, int64_t n_groups, const float* ref_all,
                              float* out, int sm_count, cudaStream_t s);

}  // namespace wmd
