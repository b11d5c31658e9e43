// cluster.h -- DBSCAN over a device-resident all-pairs matrix (internal; the C
// ABI is in include/warpmd_rmsd.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wmd {

// Status bit: a union retried more often than any valid run can need.
constexpr int kClusterStatusRetries = 32;

size_t dbscan_scratch_bytes(int64_t n);
// D: device [n][n] float32 distances (diagonal 0).  Writes labels [n] and the
// cluster count (device int).
cudaError_t dbscan_run(const float* D, int64_t n, double eps, int64_t min_samples, void* scratch, int* labels,
                       int* n_clusters_dev, int* status, int sm_count, cudaStream_t s);
// Cluster sizes and medoids (the same scratch); best_bits: n_clusters words.
cudaError_t dbscan_summary(const float* D, int64_t n, const int* labels, int64_t n_clusters, void* scratch,
                           unsigned* sizes, unsigned* centroids, unsigned long long* best_bits, cudaStream_t s);

// k-means pieces, each in the reference's summation order.
cudaError_t kmeans_features(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                            int64_t n_sel, const double* xf, double* feat, int sm_count, cudaStream_t s);
cudaError_t kmeans_gather(const double* feat, int64_t nf, const int64_t* idx, int k, double* centers, cudaStream_t s);
cudaError_t kmeans_assign(const double* feat, int64_t n, int64_t nf, const double* centers, int k, int* labels,
                          double* dist_own, cudaStream_t s);
cudaError_t kmeans_sums(const double* feat, int64_t n, int64_t nf, const int* labels, int k, double* sums, int* counts,
                        cudaStream_t s);
cudaError_t kmeans_centers(const double* feat, int64_t nf, const double* sums, const int* counts, const int64_t* reseed,
                           int k, const double* old_c, double* new_c, double* shift, cudaStream_t s);
// Final sizes (from labels) and per-cluster nearest member to the final center
// (first index on ties); centroids of empty clusters are left as 0xffffffff.
cudaError_t kmeans_finish(const double* feat, int64_t n, int64_t nf, const double* centers, const int* labels, int k,
                          double* dist, unsigned long long* best_bits, unsigned* sizes, unsigned* centroids,
                          cudaStream_t s);

}  // namespace wmd
