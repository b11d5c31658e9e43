// superpose.h -- per-frame superposition transforms and their application
// (internal; the C ABI is in include/warpmd_rmsd.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "wmd_internal.h"

namespace wmd {

// From the tile partials in L.partial (weighted or plain statistics): per
// frame R and t = c_y - R c_x into xf64 [n_frames][16] (R row-major in 0..8,
// t in 9..11) and, when xf32 is not null, float32 [n_frames][12].
// norotate: R = I (translation only).
cudaError_t launch_superpose_finalize(const FrameLaunch& L, int norotate, double* xf64, float* xf32, cudaStream_t s);

// out[f][a] = R_f coords[f][a] + t_f for every atom, float32 packed xyz.
// Packed input with 16-byte aligned coords and out takes the shared-memory
// staged kernel (bulk copies in and out); anything else the plain one.
// status: device-visible word the staged kernel reports bounded-wait timeouts into.
cudaError_t launch_superpose_apply(const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                   const double* xf64, float* out, int sm_count, int* status, cudaStream_t s);

}  // namespace wmd
