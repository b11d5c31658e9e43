/*
 * warpmd_rmsd.h -- C ABI of the B200 (sm_100a) RMSD library libwarpmd_rmsd.so.
 *
 * Scope: the RMSD hot path of warp-md 0.4.30 -- per-frame optimal-superposition
 * RMSD against a reference (RmsdPlan), the all-pairs frame x frame RMSD matrix
 * (PairwiseRmsdPlan, metrics "rms" and "nofit"), the gradient dRMSD/dx, and a
 * batched launch over many trajectories of uneven size.
 *
 * Conventions
 *   - Every entry point returns an int status: WMD_OK (0) or a negative WMD_ERR_*
 *     code; wmd_last_error(ctx) gives the message of the last failure on ctx.
 *     This mirrors TrajResult<T> / TrajError (crates/traj-core/src/error.rs:3-34):
 *     WMD_ERR_MISMATCH <-> TrajError::Mismatch, WMD_ERR_UNSUPPORTED and
 *     WMD_ERR_CUDA <-> TrajError::Unsupported("cuda driver error: ...")
 *     (crates/traj-gpu/src/cuda.rs:384-390).
 *   - Coordinates are float32, frame-major: coords[frame][atom][stride] with
 *     stride 3 (packed xyz) or 4 (xyzw, the reference's FrameChunk/Float4 layout,
 *     crates/traj-core/src/frame.rs:10-20; w is ignored).
 *   - Pointers may be host or device memory where a function says so; the
 *     library detects which with cudaPointerGetAttributes.  Host inputs are
 *     streamed to the device in chunks inside the call (copies overlap the
 *     kernels), host outputs are written before the call returns.
 *   - `stream` is a cudaStream_t (NULL = the legacy default stream).  Calls with
 *     only device pointers are asynchronous on that stream; calls with any host
 *     pointer synchronize before returning.
 *   - A wmd_ctx owns its scratch memory and is not thread-safe: use one context
 *     per host thread / stream.  The caller owns every input and output buffer.
 */
#ifndef WARPMD_RMSD_H
#define WARPMD_RMSD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WMD_OK 0
#define WMD_ERR_INVALID_ARG (-1) /* null pointer, bad stride/size/mode       */
#define WMD_ERR_CUDA (-2)        /* CUDA runtime error (message has details) */
#define WMD_ERR_OOM (-3)         /* device or pinned-host allocation failed  */
#define WMD_ERR_MISMATCH (-4)    /* shapes disagree (TrajError::Mismatch)    */
#define WMD_ERR_UNSUPPORTED (-5) /* mode/metric not provided on this build   */
#define WMD_ERR_TIMEOUT (-6)     /* a bounded device-side wait ran out       */
#define WMD_ERR_NO_DEVICE (-7)   /* no CUDA device / not an sm_100 device     */
#define WMD_ERR_IO (-8)          /* file missing or shorter than its records  */
                                 /* say (TrajError::Io)                       */
#define WMD_ERR_PARSE (-9)       /* malformed trajectory file (TrajError::Parse) */

#define WMD_PAIR_RMS 0   /* optimal-superposition RMSD (metric "rms")  */
#define WMD_PAIR_NOFIT 1 /* plain coordinate RMSD (metric "nofit")     */
#define WMD_PAIR_DME 2   /* distance-matrix error (metric "dme")        */

#define WMD_MODE_FP32 0  /* plain FP32 SIMT covariance tiles, FP64 QCP epilogue       */
#define WMD_MODE_I8X3 1  /* tcgen05 int8 tensor cores, 3 limbs (24-bit fixed point):   */
                         /* the 8 limb products other than lo x lo in exact int32     */
                         /* accumulation, self-sums truncated alike; pairs below      */
                         /* 0.01 A recomputed exactly in FP64; error <= 1e-4 A        */
#define WMD_MODE_I8X2 2  /* 2 limbs (16-bit fixed point), all 4 products, exact Gram  */
                         /* matrix of the quantised frames; error ~2e-4 A             */
#define WMD_MODE_FP64 3  /* FP64 SIMT covariance tiles (accuracy reference on GPU)    */

/* Per-frame statistics written by wmd_rmsd_forward and read by
 * wmd_rmsd_backward: 16 doubles per frame
 *   [0..2]  frame centroid        [3..11] H = sum (x - cx)(y - cy)^T (row-major)
 *   [12]    lambda_max (QCP)      [13]    rmsd
 *   [14]    n_sel                 [15]    G_x + G_y                            */
#define WMD_FRAME_STATS 16

typedef struct wmd_ctx wmd_ctx;
typedef struct wmd_ref wmd_ref;

/* Creates a context on CUDA device `device` (replaces GpuContext::new,
 * crates/traj-gpu/src/cuda/runtime_core.rs:4-17; no runtime compilation). */
int wmd_create(int device, wmd_ctx** out);
int wmd_destroy(wmd_ctx* ctx);
/* Message of the last failing call on ctx (never NULL; "" when none).  With
 * ctx == NULL, the message of the last failing wmd_create or
 * wmd_rmsd_frames_noalloc on this thread. */
const char* wmd_last_error(const wmd_ctx* ctx);
/* Library version string, e.g. "0.4.30+b200.1". */
const char* wmd_version(void);

/* Uploads a reference structure of n_sel atoms (host or device pointer,
 * stride 3 or 4) and precomputes, in FP64, its centroid, the centred
 * coordinates and G_y.  Replaces GpuContext::reference
 * (crates/traj-gpu/src/cuda/runtime_core.rs:127-137). */
int wmd_reference_upload(wmd_ctx* ctx, const float* ref, int64_t n_sel, int stride, wmd_ref** out);
int wmd_reference_free(wmd_ctx* ctx, wmd_ref* ref);

/* Error-path diagnostics (no counterpart in the reference, whose CUDA failures
 * surface as TrajError::Unsupported, crates/traj-gpu/src/cuda.rs:384-390).
 * Every device-side wait of this library is bounded: a wait that runs out
 * stops the kernel, lets its copies in flight land, and the call (or the next
 * call on the context) returns WMD_ERR_TIMEOUT.  For the per-frame streaming
 * forward kernels and the tensor-core pairwise kernel launched on `ctx` from
 * now on, the consumers' waits give up after wait_limit_ns (0 restores the
 * default of 4 s), and withhold_first_stage != 0 leaves the first pipeline
 * stage of their first CTA unfilled, so that its wait must run out.  For tests
 * of that path; the results of such calls are not valid. */
int wmd_set_wait_test(wmd_ctx* ctx, uint64_t wait_limit_ns, int withhold_first_stage);

/* Per-frame RMSD of n_frames frames against `ref` (RmsdPlan, plan.rs:323-404
 * and rmsd_aligned_selected plan.rs:1161-1248 when align != 0; rmsd_raw_selected
 * plan.rs:1093-1110 when align == 0).
 *   coords : host or device, [n_frames][n_atoms][stride]
 *   sel    : NULL for the dense selection 0..n_sel-1 (requires n_atoms == n_sel),
 *            else n_sel uint32 atom indices < n_atoms (host or device)
 *   out    : host or device, n_frames doubles
 * FP64 accumulation of the frame statistics, QCP in FP64. */
int wmd_rmsd_frames(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                    const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int align, double* out,
                    void* stream);

/* Same as wmd_rmsd_frames (align = 1) but device pointers only, and also
 * writes WMD_FRAME_STATS doubles per frame to `stats` (device) for
 * wmd_rmsd_backward. */
int wmd_rmsd_forward(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                     const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, double* out, double* stats,
                     void* stream);

/* Gradient of the aligned RMSD (no counterpart in the reference, which has no
 * derivative): grad[f][sel[i]][:] = grad_rmsd[f] * (x_i - cx - R^T (y_i - cy))
 * / (n_sel * rmsd_f), R re-derived from the QCP eigenvector of the H stored in
 * `stats`.  Device pointers only.  grad_rmsd may be NULL (all ones).  grad is
 * [n_frames][n_atoms][3] float32; rows of unselected atoms are not written. */
int wmd_rmsd_backward(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                      const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const double* stats,
                      const float* grad_rmsd, float* grad, void* stream);

/* wmd_rmsd_backward with the per-frame weights dL/drmsd as doubles at
 * grad_rmsd[f * grad_stride] (grad_stride 0: one weight for every frame, as a
 * broadcast tensor has), or all 1 when grad_rmsd is NULL.  Device pointers. */
int wmd_rmsd_backward_f64(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                          const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const double* stats,
                          const double* grad_rmsd, int64_t grad_stride, float* grad, void* stream);

/* Per-frame aligned RMSD and the gradient of L = sum_f w_f rmsd_f in one call
 * (no counterpart in the reference, which has no derivative): rmsd[f] as
 * wmd_rmsd_forward (NULL to skip), grad as wmd_rmsd_backward with weights
 * w_f = weights[f * weight_stride] (NULL: all 1).  For a dense selection of
 * packed xyz frames (n_atoms % 4 == 0, at most 16,384 atoms, at least 16
 * frames per SM) one launch reads every frame from DRAM once and writes its
 * gradient: 24 bytes per atom-frame; other shapes run the forward and the
 * backward.  Device pointers only. */
int wmd_rmsd_value_and_grad(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                            const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const double* weights,
                            int64_t weight_stride, double* rmsd, float* grad, void* stream);

/* Shape drop-in for GpuContext::rmsd_covariance
 * (crates/traj-gpu/src/cuda/runtime_core.rs:375-472): per frame the 3x3
 * covariance cov[f*9 + 3*a + b] = sum (x_a - cx_a)(y_b - cy_b) and the centred
 * sums of squares sum_x2[f], sum_y2[f], as float32 (accumulated in FP64).
 * Host or device outputs. */
int wmd_rmsd_covariance(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                        const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, float* cov, float* sum_x2,
                        float* sum_y2, void* stream);

/* All-pairs RMSD matrix (PairwiseRmsdPlan::finalize, plan.rs:593-674): out is
 * row-major n_frames x n_frames float32, symmetric, zero diagonal, all zeros
 * when n_sel < 2.  coords/sel/out host or device.  metric WMD_PAIR_*,
 * mode WMD_MODE_* (ignored for WMD_PAIR_DME, which is wmd_pairwise_dme
 * without a box). */
int wmd_pairwise_rmsd(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                      const uint32_t* sel, int64_t n_sel, int metric, int mode, float* out, void* stream);

/* One part of the all-pairs matrix for a computation split over `parts` GPUs
 * (the tile partition of PairwiseRmsdPlan::finalize's i < j loop,
 * plan.rs:593-674, which the reference runs as one loop).  Every caller holds
 * all frames; part `part` computes the pairs i < j whose tile row (40 frames
 * in the tensor-core modes, 32 in the SIMT modes) is part (mod parts), writes
 * each at (i, j) and (j, i), and leaves every other entry 0.  The parts for
 * part = 0..parts-1 are disjoint and their sum is wmd_pairwise_rmsd's matrix
 * exactly (the tensor-core modes quantise every frame with the same
 * trajectory-wide scale in every part).  WMD_PAIR_DME only with parts = 1. */
int wmd_pairwise_rmsd_part(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                           const uint32_t* sel, int64_t n_sel, int metric, int mode, int part, int parts,
                           float* out, void* stream);

/* All-pairs distance-matrix error (PairwiseRmsdPlan metric "dme",
 * plan.rs:612-645 with pair_distances_compact, plan.rs:1279-1302): per frame the
 * distances of every selected atom pair a < b (difference in f32, distance in
 * FP64; with `box`, the minimum image per axis of length > 0 as apply_pbc,
 * crates/traj-core/src/pbc_math.rs:17-27), then out[i][j] =
 * sqrt(sum_k (d_i[k] - d_j[k])^2 / n_pairs) in FP64, summed in pair order and
 * rounded to float32: the reference's numbers.  Symmetric, zero diagonal, all
 * zeros when n_sel < 2.  box: per-frame orthorhombic lengths [n_frames][3]
 * float32 (pbc "orthorhombic") or NULL (pbc "none").  coords/sel/box/out host
 * or device. */
int wmd_pairwise_dme(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                     const uint32_t* sel, int64_t n_sel, const float* box, float* out, void* stream);

/* One trajectory of a batched launch.  All pointers are device pointers. */
typedef struct wmd_batch_desc {
  const float* coords; /* [n_frames][n_atoms][3] packed xyz             */
  const float* ref;    /* [n_atoms][3] reference structure               */
  int64_t n_atoms;
  int64_t n_frames;
  double* rmsd;        /* [n_frames] output                              */
  float* grad;         /* [n_frames][n_atoms][3] output, or NULL         */
} wmd_batch_desc;

/* Per-frame aligned RMSD (+ dRMSD/dx when with_grad != 0 and grad != NULL) of
 * n_traj independent trajectories of uneven size, each against its own
 * reference, in one persistent launch sequence.  No counterpart in the
 * reference, which runs one RmsdPlan per trajectory (plan.rs:164-418); the
 * values are those of wmd_rmsd_forward per trajectory (align = 1, all atoms),
 * and grad[f] is d rmsd[f] / d coords[f] (the reference's gradient with an
 * upstream gradient of 1).
 *
 * wmd_batched_prepare validates the descriptors (device memory; coords and grad
 * 16-byte aligned; a trajectory with n_frames == 0 is skipped, one with n_atoms == 0
 * gets RMSD 0), sizes the context's workspace, uploads the trajectory table
 * and picks the layout and tile shape by timing the batch once per candidate
 * (frame-major or tile-major, 512- or 1024-atom tiles) -- it runs
 * the batch, so the coordinates must be valid, and it synchronizes.
 * wmd_batched_rmsd then takes the same descriptors (checked bytewise; anything
 * else is WMD_ERR_INVALID_ARG) and only enqueues kernels on `stream`: no
 * allocation and no host synchronization, so it can be captured in a CUDA
 * graph.  with_grad on wmd_batched_rmsd needs with_grad on the prepare. */
int wmd_batched_prepare(wmd_ctx* ctx, const wmd_batch_desc* descs, int n_traj, int with_grad);
int wmd_batched_rmsd(wmd_ctx* ctx, const wmd_batch_desc* descs, int n_traj, int with_grad, void* stream);
/* Layout the prepare step chose: atoms per tile (512 or 1024) and the layout
 * in *frame_major: 1 frame-major (each CTA owns whole frames, QCP in-kernel,
 * the gradient pass re-reads the frame from L2), 0 tile-major (tiles of all
 * frames spread over CTAs, separate finishing kernels), 2 tile-major with
 * the forward statistics computed frames across lanes (a lane per frame of
 * a 32-frame group).  Either pointer may be NULL.  WMD_ERR_INVALID_ARG when
 * no batch is prepared. */
int wmd_batched_layout(const wmd_ctx* ctx, int* tile_atoms, int* frame_major);

/* ---- Optimal superposition (AlignPlan, RotationMatrixPlan, SuperposePlan,
 *      SuperposeTrajectoryPlan: crates/traj-engine/src/plans/geometry/align/
 *      plan_exec.rs:76-523, align_matrix.rs:16-70) ---- */

/* Reference with per-atom weights (the reference's `mass=True`: the masses of
 * the selected atoms).  weights: n_sel floats, host or device, or NULL (all
 * weights 1, the same as wmd_reference_upload).  A weighted reference serves
 * only wmd_superpose_transforms and wmd_superpose; the RMSD entry points
 * reject it with WMD_ERR_INVALID_ARG. */
int wmd_reference_upload_weighted(wmd_ctx* ctx, const float* ref, int64_t n_sel, int stride, const float* weights,
                                  wmd_ref** out);

/* Per frame, the weighted Kabsch superposition of the selection onto the
 * reference (kabsch_rotation_weighted, geometry_math.rs:235-300): R (3x3,
 * row-major, R (x - c_x) ~ y - c_y) and t = c_y - R c_x, written as 12 floats
 * per frame [n_frames][12] = R00..R22, t0..t2 -- AlignPlan's rows
 * (plan_exec.rs:225-238); RotationMatrixPlan keeps the first 9.  norotate:
 * R = I, t = c_y - c_x.  An empty selection or zero total weight gives R = I,
 * t = 0 (centroid_weighted returns 0 then).  coords and transforms may be host
 * or device memory; with any host pointer the call synchronizes. */
int wmd_superpose_transforms(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                             const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int norotate, float* transforms,
                             void* stream);

/* SuperposePlan: every atom of every frame moved by its frame's transform,
 * out[f][a] = R_f coords[f][a] + t_f in FP64 rounded to float32, packed xyz
 * [n_frames][n_atoms][3] (plan_exec.rs:431-444).  transforms, if not NULL,
 * also receives the [n_frames][12] rows.  Host or device pointers as above. */
int wmd_superpose(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                  const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int norotate, float* out,
                  float* transforms, void* stream);

/* ---- Fluctuations and per-residue RMSD (RmsfPlan, AtomicFluctPlan,
 *      BfactorsPlan, AtomicAdpPlan, RmsdPerResPlan:
 *      crates/traj-engine/src/plans/geometry/rms.rs:17-430, 431-686) ---- */

/* Per selected atom, over all frames, without superposition:
 *   rmsf[i]  = sqrt(var_x + var_y + var_z)            (RmsfPlan, rms.rs:193-218)
 *   adp[i]   = (uxx, uyy, uzz, uxy, uxz, uyz), the covariance of the position
 *              with the diagonal clamped at 0         (AtomicAdpPlan, rms.rs:378-411)
 * Either output may be NULL.  Moments are taken in FP64 about each atom's
 * position in the first frame.  n_frames == 0 gives RMSF 0 and writes no ADP
 * rows.  BfactorsPlan is 8 pi^2 / 3 * rmsf^2 and AtomicFluctPlan is rmsf: the
 * caller derives them.  coords and the outputs may be host or device memory;
 * with any host pointer the call synchronizes. */
int wmd_rmsf(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
             int64_t n_sel, float* rmsf, float* adp, void* stream);

/* Groups of atoms (RmsdPerResPlan's residues) with the reference coordinates
 * of every atom, uploaded once: group g is group_atoms[group_offsets[g] ..
 * group_offsets[g + 1]) (atom indices into the frame), ref_all is
 * [n_atoms][stride] (3 or 4).  All may be host or device memory; the indices
 * are validated here.  Free with wmd_group_ref_free. */
typedef struct wmd_group_ref wmd_group_ref;
int wmd_group_ref_upload(wmd_ctx* ctx, const float* ref_all, int64_t n_atoms, int stride,
                         const uint32_t* group_offsets, const uint32_t* group_atoms, int64_t n_groups,
                         wmd_group_ref** out);
int wmd_group_ref_free(wmd_ctx* ctx, wmd_group_ref* groups);

/* RmsdPerResPlan: per frame, the selection is superposed onto `ref` (the
 * selected reference atoms, unweighted Kabsch) when align != 0, and for every
 * group g out[f][g] = sqrt(mean over the group's atoms a of
 * |R x_a + t - ref_all[a]|^2); align == 0 compares raw coordinates (`ref` may
 * then be NULL).  An empty group gives 0.  out is float32 [n_frames][n_groups],
 * host or device; coords host or device. */
int wmd_rmsd_per_group(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                       const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const wmd_group_ref* groups, int align,
                       float* out, void* stream);

/* ---- Clustering (TrajectoryClusterPlan, method "dbscan":
 *      crates/traj-engine/src/plans/analysis/clustering.rs:160-190, 269-383) ---- */

/* DBSCAN over the all-pairs RMSD matrix of the frames (wmd_pairwise_rmsd with
 * metric rms and the given mode; WMD_MODE_FP64 reproduces the reference's
 * matrix to the last float32 bit in practice).  The result is the reference's
 * sequential DBSCAN:
 *   labels[f]   cluster id, or -1 for noise (int32 [n_frames]);
 *   sizes[c], centroids[c]  members per cluster and the member with the
 *               smallest summed distance to its cluster (ties: lowest index);
 *               both need room for n_frames entries, *n_clusters are written.
 * eps <= 0 is WMD_ERR_INVALID_ARG, an empty selection WMD_ERR_MISMATCH; a
 * min_samples below 1 counts as 1.  The matrix (n_frames^2 float32) lives in
 * the context.  Outputs may be host or device memory; the call synchronizes. */
int wmd_cluster_dbscan(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                       const uint32_t* sel, int64_t n_sel, int mode, float eps, int64_t min_samples, int32_t* labels,
                       uint32_t* centroids, uint32_t* sizes, int64_t* n_clusters, void* stream);

/* k-means (TrajectoryClusterPlan, method "kmeans": clustering.rs:191-205,
 * 376-548): every frame's selection superposed onto frame 0's (unweighted
 * Kabsch) gives an FP64 feature vector; centers start at the first n_clusters
 * of a xorshift64 Fisher-Yates shuffle seeded with `seed` (0 -> a fixed
 * constant), Lloyd iterations stop after max_iter (at least 1) or once no
 * center moves more than tol; empty clusters are reseeded from the same
 * generator.  Outputs: labels int32 [n_frames]; sizes and centroids (the
 * member nearest its center) for *n_out = min(max(n_clusters, 1), n_frames)
 * clusters.  Distances and sums follow the reference's order, so labels are
 * the reference's up to exact FP64 ties.  Synchronizes. */
int wmd_cluster_kmeans(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                       const uint32_t* sel, int64_t n_sel, int64_t n_clusters, int64_t max_iter, float tol,
                       uint64_t seed, int32_t* labels, uint32_t* centroids, uint32_t* sizes, int64_t* n_out,
                       void* stream);

/* ---- DCD trajectories (DcdReader, crates/traj-io/src/dcd.rs:45-570;
 *      PyTrajectory.open_dcd / read_chunk, crates/traj-py/src/io.rs:687-708,
 *      1335-1560) ----
 * The file is parsed on the host at open; frames are read as raw bytes
 * (threaded pread into pinned buffers), copied to the device asynchronously
 * and decoded there (record markers checked, byte order, selection, length
 * scale), overlapping the read of the next batch.  Errors follow the
 * reference's: WMD_ERR_IO, WMD_ERR_PARSE, WMD_ERR_UNSUPPORTED (unknown record
 * marker), WMD_ERR_MISMATCH (selection index out of bounds). */
typedef struct wmd_dcd wmd_dcd;
int wmd_dcd_open(wmd_ctx* ctx, const char* path, float length_scale, wmd_dcd** out);
int wmd_dcd_close(wmd_ctx* ctx, wmd_dcd* dcd);
/* n_atoms; n_frames = whole frames the file holds; header_frames = the
 * header's count when positive, else 0 (n_frames_hint). */
int wmd_dcd_info(const wmd_dcd* dcd, int64_t* n_atoms, int64_t* n_frames, int64_t* header_frames);
/* read_chunk / read_chunk_selected from frame `first`: up to max_frames
 * frames into coords [n][n_out][3] float32 (host or device), n_out = n_sel
 * when sel is not NULL (atoms in selection order, repeats allowed) else
 * n_atoms.  box_kind [n] (0 none, 1 orthorhombic, 2 triclinic) and box [n][9]
 * (box vectors a, b, c as rows), host, may be NULL.  *n_read = frames read
 * (fewer than max_frames at the end of the file).  A read that reaches a
 * damaged end of file fails as the reference's chunk does and reads nothing. */
int wmd_dcd_read(wmd_ctx* ctx, wmd_dcd* dcd, int64_t first, int64_t max_frames, const uint32_t* sel, int64_t n_sel,
                 float* coords, int32_t* box_kind, float* box, int64_t* n_read, void* stream);
/* RmsdPlan over frames [first, first + max_frames) of the file: the selected
 * atoms of every frame against `ref` (align as in wmd_rmsd_frames); out [n]
 * doubles, host or device; *n_read as in wmd_dcd_read.  The file read, the
 * host->device copy, the decode and the RMSD kernels of successive batches
 * overlap. */
int wmd_dcd_rmsd(wmd_ctx* ctx, wmd_dcd* dcd, int64_t first, int64_t max_frames, const uint32_t* sel, int64_t n_sel,
                 const wmd_ref* ref, int align, double* out, int64_t* n_read, void* stream);

/* Per-frame aligned RMSD for callers that cannot allocate memory.  No
 * counterpart in the reference.  Everything else in this header needs a
 * wmd_ctx and a wmd_ref, which allocate device and pinned memory; this call
 * allocates nothing, for code that runs where allocation is forbidden or
 * unsafe (inside a host callback or a real-time loop, in a plugin whose host
 * program owns all GPU memory, or without a context to keep workspaces in).
 *   coords : device, [n_frames][n_atoms][stride]; the first n_sel atoms of each
 *            frame are used (dense selection)
 *   ref    : device, [n_sel][ref_stride] reference structure
 *   out    : device, n_frames doubles -- the same values as wmd_rmsd_frames
 *            with align = 1 (FP64 statistics and QCP)
 * Runs asynchronously on `stream` on the current CUDA device.  Its scratch is
 * one fixed 16 MiB array inside the library (held by every GPU that loads the
 * library until exit), so n_sel is limited to 65,536 atoms; larger selections
 * are rejected with WMD_ERR_INVALID_ARG (message via wmd_last_error(NULL)).
 * The first call on a device looks up that array's device address; make it
 * before any stream capture.  All calls on a device share the array: calls
 * that may overlap on the GPU race and must be serialised by the caller. */
int wmd_rmsd_frames_noalloc(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const float* ref,
                            int64_t n_sel, int ref_stride, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WARPMD_RMSD_H */
