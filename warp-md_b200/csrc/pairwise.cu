// pairwise.cu -- all-pairs frame x frame RMSD matrix.
//
// Reference behaviour: PairwiseRmsdPlan::finalize
// (crates/traj-engine/src/plans/rmsd/plan.rs:593-674) -- CPU only, FP64, one
// Kabsch SVD per pair (rmsd_aligned, plan.rs:1112-1159) or a raw RMSD
// (rmsd_raw, plan.rs:1081-1091); symmetric fill, zero diagonal, all zeros when
// fewer than two atoms are selected.
//
// Here every frame is centred once (FP64 centroid, coordinates stored in the
// mode's precision, G_i = sum |x_i - c_i|^2 of the stored values in FP64), the
// nine covariance entries of all pairs are the 3N x 3N Gram matrix of the
// centred frames, and a per-pair FP64 epilogue turns each 3x3 block into an
// RMSD (QCP for "rms"; G_i + G_j - 2 tr H + n |c_i - c_j|^2 for "nofit").
//
// This file holds the SIMT forms (FP32 and FP64 accumulation); the
// tensor-core forms live in pairwise_tc.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/warpmd_rmsd.h"
#include "pairwise.h"
#include "pairwise_tc.h"
#include "device_util.cuh"
#include "qcp.cuh"

namespace wmd {

constexpr int kPairKc = 32;  // atoms per K step of the SIMT tiles

// Centres each selected frame.  One CTA per frame.  Output layout
// xc[f][c][n_pad] (atoms contiguous per component, zero padded).
template <typename T>
__global__ void __launch_bounds__(256) pair_prep(const float* __restrict__ coords, int64_t n_atoms, int stride,
                                                 const uint32_t* __restrict__ sel, int64_t n_sel, int64_t n_pad,
                                                 T* __restrict__ xc, double* __restrict__ gsum,
                                                 double* __restrict__ cen, int* status) {
  __shared__ double red[8][4];
  const int64_t f = blockIdx.x;
  const float* fr = coords + (size_t)f * n_atoms * stride;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
    int64_t idx = sel ? (int64_t)sel[k] : k;
    if (idx >= n_atoms) {  // bad device-side selection: report, read atom 0
      atomicOr(status, kStatusBadIndex);
      idx = 0;
    }
    const float* p = fr + idx * stride;
    s0 += p[0]; s1 += p[1]; s2 += p[2];
  }
  for (int o = 16; o; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) { red[warp][0] = s0; red[warp][1] = s1; red[warp][2] = s2; }
  __syncthreads();
  double c[3] = {0, 0, 0};
  for (int w = 0; w < 8; ++w) { c[0] += red[w][0]; c[1] += red[w][1]; c[2] += red[w][2]; }
  const double inv = n_sel > 0 ? 1.0 / (double)n_sel : 0.0;
  c[0] *= inv; c[1] *= inv; c[2] *= inv;
  __syncthreads();
  T* row = xc + (size_t)f * 3 * n_pad;
  double g = 0;
  for (int64_t k = threadIdx.x; k < n_pad; k += blockDim.x) {
    if (k < n_sel) {
      int64_t idx = sel ? (int64_t)sel[k] : k;
      if (idx >= n_atoms) idx = 0;
      const float* p = fr + idx * stride;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const T v = (T)((double)p[q] - c[q]);
        row[q * n_pad + k] = v;
        g += (double)v * (double)v;
      }
    } else {
      row[k] = T(0); row[n_pad + k] = T(0); row[2 * n_pad + k] = T(0);
    }
  }
  for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
  if (lane == 0) red[warp][3] = g;
  __syncthreads();
  if (threadIdx.x == 0) {
    double gt = 0;
    for (int w = 0; w < 8; ++w) gt += red[w][3];
    gsum[f] = gt;
    cen[f * 3 + 0] = c[0]; cen[f * 3 + 1] = c[1]; cen[f * 3 + 2] = c[2];
  }
}

// Per-pair epilogue shared by every pairwise form: h = covariance block of
// frames (i, j), returns the RMSD.
__device__ __forceinline__ double pair_rmsd(const double h[9], double gi, double gj, const double* ci,
                                            const double* cj, double n, int metric) {
  if (metric == WMD_PAIR_NOFIT) {
    const double d0 = ci[0] - cj[0], d1 = ci[1] - cj[1], d2 = ci[2] - cj[2];
    const double s = gi + gj - 2.0 * (h[0] + h[4] + h[8]) + n * (d0 * d0 + d1 * d1 + d2 * d2);
    return s > 0.0 ? sqrt(s / n) : 0.0;
  }
  const QcpOut q = qcp_lambda(h, 0.5 * (gi + gj));
  return sqrt(msd_from(gi, gj, q.lambda, n));
}

// SIMT tile: 16x16 threads, each owning FA x FB frame pairs (full 3x3 blocks in
// registers).  Block covers frames [I0, I0 + 16 FA) x [J0, J0 + 16 FB); only
// pairs i < j are computed and written to both (i, j) and (j, i).
template <typename T, int FA, int FB>
__global__ void __launch_bounds__(256) pair_tile_simt(const T* __restrict__ xc, const double* __restrict__ gsum,
                                                      const double* __restrict__ cen, int64_t F, int64_t n_pad,
                                                      double n, int metric, float* __restrict__ out) {
  constexpr int BI = 16 * FA, BJ = 16 * FB;
  constexpr int RA = 3 * BI, RB = 3 * BJ;
  constexpr int LD = kPairKc + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);
  T* Bs = As + RA * LD;
  const int64_t I0 = (int64_t)blockIdx.y * BI, J0 = (int64_t)blockIdx.x * BJ;
  if (I0 >= J0 + BJ - 1 || I0 >= F || J0 >= F) return;  // no pair with i < j in this block
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[FA][FB][9];
#pragma unroll
  for (int a = 0; a < FA; ++a)
#pragma unroll
    for (int b = 0; b < FB; ++b)
#pragma unroll
      for (int e = 0; e < 9; ++e) acc[a][b][e] = T(0);

  for (int64_t k0 = 0; k0 < n_pad; k0 += kPairKc) {
    // stage rows (frame, component) x kPairKc atoms
    for (int idx = threadIdx.x; idx < (RA + RB) * kPairKc; idx += 256) {
      const int r = idx / kPairKc, kk = idx % kPairKc;
      T v = T(0);
      if (r < RA) {
        const int64_t fr = I0 + r / 3;
        if (fr < F) v = xc[((size_t)fr * 3 + (r % 3)) * n_pad + k0 + kk];
        As[r * LD + kk] = v;
      } else {
        const int rb = r - RA;
        const int64_t fr = J0 + rb / 3;
        if (fr < F) v = xc[((size_t)fr * 3 + (rb % 3)) * n_pad + k0 + kk];
        Bs[rb * LD + kk] = v;
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kPairKc; ++kk) {
      T xa[FA][3], xb[FB][3];
#pragma unroll
      for (int a = 0; a < FA; ++a)
#pragma unroll
        for (int q = 0; q < 3; ++q) xa[a][q] = As[((ty * FA + a) * 3 + q) * LD + kk];
#pragma unroll
      for (int b = 0; b < FB; ++b)
#pragma unroll
        for (int q = 0; q < 3; ++q) xb[b][q] = Bs[((tx * FB + b) * 3 + q) * LD + kk];
#pragma unroll
      for (int a = 0; a < FA; ++a)
#pragma unroll
        for (int b = 0; b < FB; ++b)
#pragma unroll
          for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int q = 0; q < 3; ++q) acc[a][b][p * 3 + q] = fma(xa[a][p], xb[b][q], acc[a][b][p * 3 + q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < FA; ++a) {
    const int64_t i = I0 + ty * FA + a;
#pragma unroll
    for (int b = 0; b < FB; ++b) {
      const int64_t j = J0 + tx * FB + b;
      if (i < j && j < F) {
        double h[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) h[e] = (double)acc[a][b][e];
        const float v = (float)pair_rmsd(h, gsum[i], gsum[j], cen + i * 3, cen + j * 3, n, metric);
        out[(size_t)i * F + j] = v;
        out[(size_t)j * F + i] = v;
      }
    }
  }
}

void pairwise_workspace_free(PairwiseWorkspace& w) {
  if (w.centred) cudaFree(w.centred);
  if (w.gsum) cudaFree(w.gsum);
  if (w.cen) cudaFree(w.cen);
  if (w.extra) cudaFree(w.extra);
  w = PairwiseWorkspace();
}

static int grow(void** p, size_t* have, size_t want, std::string* msg) {
  if (*p && *have >= want) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(p, std::max<size_t>(want, 256));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    *msg = std::string("cuda driver error: pairwise workspace allocation failed: ") + cudaGetErrorString(e);
    return WMD_ERR_OOM;
  }
  *have = std::max<size_t>(want, 256);
  return 0;
}

template <typename T, int FA, int FB>
static cudaError_t run_simt(PairwiseWorkspace& w, int64_t F, int64_t n_pad, int64_t n_sel, int metric, float* out,
                            cudaStream_t s) {
  constexpr int BI = 16 * FA, BJ = 16 * FB;
  const size_t smem = (size_t)(3 * BI + 3 * BJ) * (kPairKc + 1) * sizeof(T);
  auto kern = pair_tile_simt<T, FA, FB>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((F + BJ - 1) / BJ), (unsigned)((F + BI - 1) / BI));
  kern<<<grid, 256, smem, s>>>(static_cast<const T*>(w.centred), w.gsum, w.cen, F, n_pad, (double)n_sel, metric,
                               out);
  return cudaGetLastError();
}

int pairwise_run(PairwiseWorkspace& w, int sm_count, const float* coords, int64_t n_frames, int64_t n_atoms,
                 int stride, const uint32_t* sel, int64_t n_sel, int metric, int mode, float* out, int* status,
                 cudaStream_t s, std::string* msg) {
  const size_t out_bytes = (size_t)n_frames * n_frames * sizeof(float);
  cudaError_t e = cudaMemsetAsync(out, 0, out_bytes, s);
  if (e != cudaSuccess) {
    *msg = std::string("cuda driver error: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  if (n_sel < 2 || n_frames < 2) return 0;  // all zeros (plan.rs:604-610)

  if (mode == WMD_MODE_I8X3 || mode == WMD_MODE_I8X2)
    return pairwise_tc_run(w, sm_count, coords, n_frames, n_atoms, stride, sel, n_sel, metric,
                           mode == WMD_MODE_I8X3 ? 3 : 2, out, status, s, msg);

  const bool f64 = mode == WMD_MODE_FP64;
  const int64_t n_pad = (n_sel + kPairKc - 1) / kPairKc * kPairKc;
  const size_t elem = f64 ? sizeof(double) : sizeof(float);
  int rc = grow(&w.centred, &w.centred_bytes, (size_t)n_frames * 3 * n_pad * elem, msg);
  if (rc) return rc;
  if (w.frames_cap < (size_t)n_frames) {
    if (w.gsum) cudaFree(w.gsum);
    if (w.cen) cudaFree(w.cen);
    w.gsum = nullptr;
    w.cen = nullptr;
    w.frames_cap = 0;
    if ((e = cudaMalloc(&w.gsum, n_frames * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&w.cen, n_frames * 3 * sizeof(double))) != cudaSuccess) {
      cudaGetLastError();
      *msg = std::string("cuda driver error: pairwise workspace allocation failed: ") + cudaGetErrorString(e);
      return WMD_ERR_OOM;
    }
    w.frames_cap = n_frames;
  }
  if (f64)
    pair_prep<double><<<(unsigned)n_frames, 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, n_pad,
                                                         static_cast<double*>(w.centred), w.gsum, w.cen, status);
  else
    pair_prep<float><<<(unsigned)n_frames, 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, n_pad,
                                                        static_cast<float*>(w.centred), w.gsum, w.cen, status);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = f64 ? run_simt<double, 2, 2>(w, n_frames, n_pad, n_sel, metric, out, s)
                                : run_simt<float, 4, 2>(w, n_frames, n_pad, n_sel, metric, out, s);
  if (e != cudaSuccess) {
    *msg = std::string("cuda driver error: pairwise launch: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  return 0;
}

}  // namespace wmd
