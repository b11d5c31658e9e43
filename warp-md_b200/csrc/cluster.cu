// cluster.cu -- DBSCAN over the all-pairs RMSD matrix (TrajectoryClusterPlan,
// method "dbscan": crates/traj-engine/src/plans/analysis/clustering.rs:160-190,
// 269-383).
//
// The reference runs the textbook sequential DBSCAN over the triangular f32
// matrix.  Its result is a function of the matrix alone, which this file
// computes in parallel:
//   * a point is core when at least min_samples points (itself included) lie
//     within eps;
//   * clusters are the connected components of core points under d <= eps,
//     numbered in increasing order of their smallest core index (the order in
//     which the sequential outer loop starts them);
//   * a non-core point takes the smallest cluster id among its core neighbours
//     (the first cluster whose expansion reaches it), or -1 (noise);
//   * a cluster's centroid is the member with the smallest FP64 sum of
//     distances to all members, summed in index order, ties to the lowest
//     index (clustering.rs:347-373).
// Kernels: row degrees; union-find over core-core edges (lock-free, larger
// root hooked under the smaller, so each root is its component's minimum);
// root ranking; labels; sizes; medoid sums and the two-pass argmin.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "cluster.h"

namespace wmd {
namespace {

constexpr int kRowThreads = 256;

__device__ __forceinline__ bool within(float d, double eps) { return (double)d <= eps; }

// deg[i] = #{j : d(i, j) <= eps}, the diagonal counted as 0.
__global__ void __launch_bounds__(kRowThreads) degree_kernel(const float* __restrict__ D, int64_t n, double eps,
                                                             int64_t min_samples, uint8_t* __restrict__ core) {
  __shared__ int red[kRowThreads / 32];
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const float* row = D + (size_t)i * n;
    int c = 0;
    for (int64_t j = threadIdx.x; j < n; j += kRowThreads) c += (j == i || within(row[j], eps)) ? 1 : 0;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kRowThreads / 32; ++w) t += red[w];
      core[i] = (int64_t)t >= min_samples ? 1 : 0;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int find_root(const int* parent, int x) {
  // parents only ever point to smaller indices, so this takes at most x steps
  // (loads bypass L1, so links made by other SMs are seen)
  int p = __ldcg(parent + x);
  while (p != x) {
    x = p;
    p = __ldcg(parent + x);
  }
  return x;
}

// Scratch layout (dbscan_scratch_bytes): parent, root, cluster_of_root as int
// [n] each, sum as double [n], core as byte [n].
struct DbLayout {
  int* parent;
  int* root;
  int* cluster_of_root;
  double* sum;
  uint8_t* core;
  __host__ __device__ DbLayout(void* scratch, int64_t n) {
    char* p = static_cast<char*>(scratch);
    parent = reinterpret_cast<int*>(p);
    root = parent + n;
    cluster_of_root = root + n;
    sum = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(cluster_of_root + n) + 7) & ~uintptr_t(7));
    core = reinterpret_cast<uint8_t*>(sum + n);
  }
};

__global__ void init_parent_kernel(int* parent, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parent[i] = (int)i;
}

// Union of every core-core pair within eps, i < j: a block per row i.
__global__ void __launch_bounds__(kRowThreads) union_kernel(const float* __restrict__ D, int64_t n, double eps,
                                                            const uint8_t* __restrict__ core, int* parent,
                                                            int* status) {
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    if (!core[i]) continue;
    const float* row = D + (size_t)i * n;
    for (int64_t j = i + 1 + threadIdx.x; j < n; j += kRowThreads) {
      if (!core[j] || !within(row[j], eps)) continue;
      int a = (int)i, b = (int)j;
      // lock-free union: hook the larger root under the smaller; a failed CAS
      // means another thread linked that root (at most n - 1 links happen in
      // all), so look again -- with a cap that reports instead of spinning on
      int tries = 0;
      for (;; ++tries) {
        if (tries > (1 << 24)) {
          atomicOr(status, kClusterStatusRetries);
          break;
        }
        a = find_root(parent, a);
        b = find_root(parent, b);
        if (a == b) break;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) break;
        a = lo;
        b = old;
      }
    }
  }
}

// root[i] = component root of core point i (-1 for non-core); is_root flags.
__global__ void roots_kernel(const int* parent, const uint8_t* core, int64_t n, int* root) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) root[i] = core[i] ? find_root(parent, (int)i) : -1;
}

// cluster_of_root[i] = rank of root i among all roots (one block, in order).
__global__ void __launch_bounds__(1024) rank_roots_kernel(const int* root, int64_t n, int* cluster_of_root,
                                                          int* n_clusters) {
  __shared__ int carry;
  __shared__ int warp_sums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const int flag = (i < n && root[i] == (int)i) ? 1 : 0;
    // block-wide exclusive scan of flag
    int v = flag;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
      int w = warp_sums[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += u;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const int incl = v + (warp > 0 ? warp_sums[warp - 1] : 0);
    if (i < n) cluster_of_root[i] = flag ? carry + incl - 1 : -1;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_clusters = carry;
}

// Labels: core -> its component's cluster; non-core -> the smallest cluster of
// a core neighbour within eps, or -1.  A block per point.
__global__ void __launch_bounds__(kRowThreads) label_kernel(const float* __restrict__ D, int64_t n, double eps,
                                                            const uint8_t* __restrict__ core,
                                                            const int* __restrict__ root,
                                                            const int* __restrict__ cluster_of_root,
                                                            int* __restrict__ labels) {
  __shared__ int red[kRowThreads / 32];
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    if (core[i]) {
      if (threadIdx.x == 0) labels[i] = cluster_of_root[root[i]];
      continue;
    }
    const float* row = D + (size_t)i * n;
    int best = 0x7fffffff;
    for (int64_t j = threadIdx.x; j < n; j += kRowThreads)
      if (j != i && core[j] && within(row[j], eps)) best = min(best, cluster_of_root[root[j]]);
    for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      int b = 0x7fffffff;
      for (int w = 0; w < kRowThreads / 32; ++w) b = min(b, red[w]);
      labels[i] = b == 0x7fffffff ? -1 : b;
    }
    __syncthreads();
  }
}

__global__ void sizes_kernel(const int* labels, int64_t n, unsigned* sizes) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && labels[i] >= 0) atomicAdd(sizes + labels[i], 1u);
}

// sum[i] = sum over members j of i's cluster, in index order, of d(i, j), FP64
// (a thread per point, sequential like the reference's loop).
__global__ void __launch_bounds__(256) medoid_sum_kernel(const float* __restrict__ D, int64_t n,
                                                         const int* __restrict__ labels, double* __restrict__ sum,
                                                         unsigned long long* __restrict__ best_bits) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = labels[i];
  if (c < 0) return;
  const float* row = D + (size_t)i * n;
  double s = 0.0;
  for (int64_t j = 0; j < n; ++j)
    if (labels[j] == c) s += j == i ? 0.0 : (double)row[j];
  sum[i] = s;
  // non-negative doubles order like their bit patterns
  atomicMin(best_bits + c, (unsigned long long)__double_as_longlong(s));
}

__global__ void medoid_pick_kernel(int64_t n, const int* labels, const double* sum,
                                   const unsigned long long* best_bits, unsigned* centroid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = labels[i];
  if (c < 0) return;
  if ((unsigned long long)__double_as_longlong(sum[i]) == best_bits[c]) atomicMin(centroid + c, (unsigned)i);
}

// ---------------------------------------------------------------------------
// k-means (TrajectoryClusterPlan, method "kmeans": clustering.rs:191-205,
// 376-548).  Features are the selection's coordinates after superposition
// onto frame 0, in FP64; every distance and every sum runs in the reference's
// order (features in order, samples in index order), so assignments are the
// reference's up to exact FP64 ties.
// ---------------------------------------------------------------------------

constexpr int kKmChunk = 16;  // centers per pass of the assignment kernel

// feat[i][3a + c] = (R_i x_ia + t_i)_c
template <int STRIDE>
__global__ void kmeans_features_kernel(const float* __restrict__ coords, int64_t n_frames, int64_t n_atoms,
                                       const uint32_t* __restrict__ sel, int64_t n_sel,
                                       const double* __restrict__ xf, double* __restrict__ feat) {
  const int64_t total = n_frames * n_sel;
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < total; it += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = it / n_sel, a = it - f * n_sel;
    const int64_t atom = sel ? (int64_t)sel[a] : a;
    const float* p = coords + ((size_t)f * n_atoms + atom) * STRIDE;
    const double* x = xf + f * 16;
    const double p0 = p[0], p1 = p[1], p2 = p[2];
    double* o = feat + (size_t)f * n_sel * 3 + a * 3;
    o[0] = x[0] * p0 + x[1] * p1 + x[2] * p2 + x[9];
    o[1] = x[3] * p0 + x[4] * p1 + x[5] * p2 + x[10];
    o[2] = x[6] * p0 + x[7] * p1 + x[8] * p2 + x[11];
  }
}

// labels[i] = argmin_c sum_k (feat[i][k] - centers[c][k])^2, first minimum;
// dist_own[i] (optional) = the distance to the chosen center.
__global__ void __launch_bounds__(128) kmeans_assign_kernel(const double* __restrict__ feat, int64_t n, int64_t nf,
                                                            const double* __restrict__ centers, int k,
                                                            int* __restrict__ labels, double* __restrict__ dist_own) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* row = feat + (size_t)i * nf;
  int best = 0;
  double best_d = __longlong_as_double(0x7ff0000000000000ll);  // +inf
  for (int c0 = 0; c0 < k; c0 += kKmChunk) {
    const int cn = min(kKmChunk, k - c0);
    double d[kKmChunk];
#pragma unroll
    for (int c = 0; c < kKmChunk; ++c) d[c] = 0.0;
    for (int64_t j = 0; j < nf; ++j) {
      const double v = row[j];
#pragma unroll
      for (int c = 0; c < kKmChunk; ++c)
        if (c < cn) {
          const double e = v - __ldg(centers + (size_t)(c0 + c) * nf + j);
          d[c] = __dadd_rn(d[c], __dmul_rn(e, e));  // d*d then +, unfused, as sq_dist
        }
    }
#pragma unroll
    for (int c = 0; c < kKmChunk; ++c)
      if (c < cn && d[c] < best_d) {
        best_d = d[c];
        best = c0 + c;
      }
  }
  labels[i] = best;
  if (dist_own) dist_own[i] = best_d;
}

// Per feature column j: sums[c][j] over the samples of cluster c, in index
// order (threads own columns, so loads are coalesced), and counts.
__global__ void __launch_bounds__(128) kmeans_sums_kernel(const double* __restrict__ feat, int64_t n, int64_t nf,
                                                          const int* __restrict__ labels, int k,
                                                          double* __restrict__ sums, int* __restrict__ counts) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int c0 = blockIdx.y * kKmChunk;
  const int cn = min(kKmChunk, k - c0);
  if (j >= nf) return;
  double acc[kKmChunk];
  int cnt[kKmChunk];
#pragma unroll
  for (int c = 0; c < kKmChunk; ++c) { acc[c] = 0.0; cnt[c] = 0; }
  for (int64_t i = 0; i < n; ++i) {
    const int c = labels[i] - c0;
    if (c < 0 || c >= cn) continue;
    const double v = feat[(size_t)i * nf + j];
#pragma unroll
    for (int q = 0; q < kKmChunk; ++q)
      if (q == c) {
        acc[q] += v;
        ++cnt[q];
      }
  }
  for (int q = 0; q < cn; ++q) sums[(size_t)(c0 + q) * nf + j] = acc[q];
  if (j == 0)
    for (int q = 0; q < cn; ++q) counts[c0 + q] = cnt[q];
}

// New centers: sums / count, or the sample reseed[c] for an empty cluster;
// shift[c] = |old - new| (features in order).  A block per cluster, thread 0
// keeps the sequential shift sum.
__global__ void __launch_bounds__(256) kmeans_centers_kernel(const double* __restrict__ feat, int64_t nf,
                                                             const double* __restrict__ sums,
                                                             const int* __restrict__ counts,
                                                             const int64_t* __restrict__ reseed,
                                                             const double* __restrict__ old_c,
                                                             double* __restrict__ new_c, double* __restrict__ shift) {
  const int c = blockIdx.x;
  const int64_t src = reseed[c];
  const double inv = counts[c] > 0 ? 1.0 / (double)counts[c] : 0.0;
  for (int64_t j = threadIdx.x; j < nf; j += blockDim.x)
    new_c[(size_t)c * nf + j] = src >= 0 ? feat[(size_t)src * nf + j] : sums[(size_t)c * nf + j] * inv;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int64_t j = 0; j < nf; ++j) {
      const double e = old_c[(size_t)c * nf + j] - new_c[(size_t)c * nf + j];
      s = __dadd_rn(s, __dmul_rn(e, e));
    }
    shift[c] = sqrt(s);
  }
}

// Distance of each sample to its own cluster's center (features in order) and
// the per-cluster minimum as ordered bits (non-negative doubles).
__global__ void __launch_bounds__(128) kmeans_own_dist_kernel(const double* __restrict__ feat, int64_t n, int64_t nf,
                                                              const double* __restrict__ centers,
                                                              const int* __restrict__ labels, double* __restrict__ d,
                                                              unsigned long long* __restrict__ best_bits) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = labels[i];
  const double* row = feat + (size_t)i * nf;
  const double* ctr = centers + (size_t)c * nf;
  double s = 0.0;
  for (int64_t j = 0; j < nf; ++j) {
    const double e = row[j] - ctr[j];
    s = __dadd_rn(s, __dmul_rn(e, e));
  }
  d[i] = s;
  atomicMin(best_bits + c, (unsigned long long)__double_as_longlong(s));
}

__global__ void kmeans_gather_kernel(const double* __restrict__ feat, int64_t nf, const int64_t* __restrict__ idx,
                                     double* __restrict__ centers) {
  const int c = blockIdx.x;
  for (int64_t j = threadIdx.x; j < nf; j += blockDim.x) centers[(size_t)c * nf + j] = feat[(size_t)idx[c] * nf + j];
}

}  // namespace

size_t dbscan_scratch_bytes(int64_t n) { return (size_t)n * (3 * sizeof(int) + sizeof(double) + 1) + 64; }

cudaError_t dbscan_run(const float* D, int64_t n, double eps, int64_t min_samples, void* scratch, int* labels,
                       int* n_clusters_dev, int* status, int sm_count, cudaStream_t s) {
  DbLayout L(scratch, n);
  const unsigned rows = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n, (int64_t)sm_count * 16));
  const unsigned lin = (unsigned)((n + 255) / 256);
  degree_kernel<<<rows, kRowThreads, 0, s>>>(D, n, eps, min_samples, L.core);
  init_parent_kernel<<<lin, 256, 0, s>>>(L.parent, n);
  union_kernel<<<rows, kRowThreads, 0, s>>>(D, n, eps, L.core, L.parent, status);
  roots_kernel<<<lin, 256, 0, s>>>(L.parent, L.core, n, L.root);
  rank_roots_kernel<<<1, 1024, 0, s>>>(L.root, n, L.cluster_of_root, n_clusters_dev);
  label_kernel<<<rows, kRowThreads, 0, s>>>(D, n, eps, L.core, L.root, L.cluster_of_root, labels);
  return cudaGetLastError();
}

cudaError_t dbscan_summary(const float* D, int64_t n, const int* labels, int64_t n_clusters, void* scratch,
                           unsigned* sizes, unsigned* centroids, unsigned long long* best_bits, cudaStream_t s) {
  DbLayout L(scratch, n);
  cudaError_t e;
  if (n_clusters == 0) return cudaSuccess;
  if ((e = cudaMemsetAsync(sizes, 0, (size_t)n_clusters * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(centroids, 0xff, (size_t)n_clusters * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(best_bits, 0xff, (size_t)n_clusters * sizeof(unsigned long long), s)) != cudaSuccess)
    return e;
  const unsigned lin = (unsigned)((n + 255) / 256);
  sizes_kernel<<<lin, 256, 0, s>>>(labels, n, sizes);
  medoid_sum_kernel<<<lin, 256, 0, s>>>(D, n, labels, L.sum, best_bits);
  medoid_pick_kernel<<<lin, 256, 0, s>>>(n, labels, L.sum, best_bits, centroids);
  return cudaGetLastError();
}

}  // namespace wmd

namespace wmd {

cudaError_t kmeans_features(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                            int64_t n_sel, const double* xf, double* feat, int sm_count, cudaStream_t s) {
  const int64_t total = n_frames * n_sel;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count * 16));
  if (stride == 4) kmeans_features_kernel<4><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, sel, n_sel, xf, feat);
  else kmeans_features_kernel<3><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, sel, n_sel, xf, feat);
  return cudaGetLastError();
}

cudaError_t kmeans_gather(const double* feat, int64_t nf, const int64_t* idx, int k, double* centers, cudaStream_t s) {
  kmeans_gather_kernel<<<k, 256, 0, s>>>(feat, nf, idx, centers);
  return cudaGetLastError();
}

cudaError_t kmeans_assign(const double* feat, int64_t n, int64_t nf, const double* centers, int k, int* labels,
                          double* dist_own, cudaStream_t s) {
  kmeans_assign_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(feat, n, nf, centers, k, labels, dist_own);
  return cudaGetLastError();
}

cudaError_t kmeans_sums(const double* feat, int64_t n, int64_t nf, const int* labels, int k, double* sums, int* counts,
                        cudaStream_t s) {
  const dim3 grid((unsigned)((nf + 127) / 128), (unsigned)((k + kKmChunk - 1) / kKmChunk));
  kmeans_sums_kernel<<<grid, 128, 0, s>>>(feat, n, nf, labels, k, sums, counts);
  return cudaGetLastError();
}

cudaError_t kmeans_centers(const double* feat, int64_t nf, const double* sums, const int* counts, const int64_t* reseed,
                           int k, const double* old_c, double* new_c, double* shift, cudaStream_t s) {
  kmeans_centers_kernel<<<k, 256, 0, s>>>(feat, nf, sums, counts, reseed, old_c, new_c, shift);
  return cudaGetLastError();
}

cudaError_t kmeans_finish(const double* feat, int64_t n, int64_t nf, const double* centers, const int* labels, int k,
                          double* dist, unsigned long long* best_bits, unsigned* sizes, unsigned* centroids,
                          cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(sizes, 0, (size_t)k * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(centroids, 0xff, (size_t)k * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(best_bits, 0xff, (size_t)k * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  const unsigned lin = (unsigned)((n + 127) / 128);
  sizes_kernel<<<lin, 128, 0, s>>>(labels, n, sizes);
  kmeans_own_dist_kernel<<<lin, 128, 0, s>>>(feat, n, nf, centers, labels, dist, best_bits);
  medoid_pick_kernel<<<lin, 128, 0, s>>>(n, labels, dist, best_bits, centroids);
  return cudaGetLastError();
}

}  // namespace wmd
