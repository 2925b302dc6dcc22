/*
 * lig_b200 — C ABI of the B200-native gsplat2d hot path.
 *
 * Plain pointers, sizes and a CUDA stream (passed as void*); no torch types.
 * Every buffer is allocated by the caller.  Every entry point is asynchronous
 * on `stream`, returns LIG_OK or a LIG_ERR_* code, and never synchronises the
 * host.  Device pointers typed `void*` hold float (dtype LIG_F32) or double
 * (dtype LIG_F64) arrays; the FP64 instantiation exists for checking against
 * an FP64 oracle.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root; csrc/ = gsplat2d/gsplat2d/cuda/csrc/).  The
 * reference bound these through pybind11 (csrc/ext.cpp:4-17); here they are
 * bound through ctypes by lig_b200/_lib.py.
 */
#ifndef LIG_B200_H
#define LIG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LIG_OK 0
#define LIG_ERR_INVALID 1     /* bad argument (size, dtype, block width, null) */
#define LIG_ERR_CAPACITY 2    /* intersection count exceeds the given capacity */
#define LIG_ERR_LAUNCH 3      /* a kernel launch failed (cudaGetLastError) */
#define LIG_ERR_WORKSPACE 4   /* workspace smaller than the *_workspace_bytes query */
#define LIG_ERR_TOO_LARGE 5   /* num_points above LIG_STATIC_MAX_POINTS (allocation-free entry) */

#define LIG_F32 0
#define LIG_F64 1

/* Device status word bits written by lig_bin (int32 at `status`). */
#define LIG_STATUS_OVERFLOW 1 /* num_intersects > capacity: outputs incomplete */
#define LIG_STATUS_BADBOX 2   /* a tile bbox disagreed with num_tiles_hit */

/* ABI version (bumped on any signature change). */
int lig_abi_version(void);

/* Number of CUDA kernels this library has launched in this process (all
 * devices, all threads) — for launch accounting by benchmarks. */
int64_t lig_kernel_launches(void);

/* ------------------------------------------------------------ projection */

/* Projection forward: conic, SnugBox extent, tile bbox and tile-hit count per
 * Gaussian.  cholesky=0: in3 = cov2d [N,3] (upper triangle a,b,c);
 * cholesky=1: in3 = [l11, l21, l22].  opacities may be NULL (1.0).
 * Every output element is written (zeros where the reference leaves its
 * torch::zeros initialisation).
 * Replaces project_gaussians_forward_tensor (csrc/bindings.cu:68-117) and
 * project_gaussians_forward_cholesky_tensor (csrc/bindings.cu:153-202). */
int lig_project_fwd(int dtype, int num_points, int cholesky, const void *in3,
                    const void *means2d, const void *opacities, int img_h, int img_w,
                    int block_width, void *xys, void *extents, void *conics,
                    int32_t *num_tiles_hit, void *stream);

/* Projection backward that recomputes conic and extent from the inputs
 * instead of reading saved ones.  v_xy / v_conic rows may be strided
 * (row stride in elements, unit inner stride).
 * Replaces the saved-tensor path of project_gaussians.py:77-104 and
 * project_gaussians_cholesky.py:84-112. */
int lig_project_bwd(int dtype, int num_points, int cholesky, const void *in3,
                    const void *means2d, const void *opacities, int img_h, int img_w,
                    int block_width, const void *v_xy, int64_t v_xy_stride,
                    const void *v_conic, int64_t v_conic_stride, void *v_in3,
                    void *v_mean2d, void *stream);

/* Projection backward from saved extents and conics (reference-shaped).
 * in3 is only read when cholesky=1.
 * Replaces project_gaussians_backward_tensor (csrc/bindings.cu:119-151) and
 * project_gaussians_backward_cholesky_tensor (csrc/bindings.cu:204-237). */
int lig_project_bwd_saved(int dtype, int num_points, int cholesky, const void *extents,
                          const void *in3, const void *conics, const void *v_xy,
                          const void *v_conic, void *v_in3, void *v_mean2d, void *stream);

/* Conic and extent only.  Where det == 0 the outputs are zeros.
 * Replaces compute_cov2d_bounds_tensor (csrc/bindings.cu:41-66). */
int lig_cov2d_bounds(int dtype, int num_points, const void *cov2d, const void *opacities,
                     void *conics, void *extents, void *stream);

/* --------------------------------------------------------------- binning */

/* Workspace bytes needed by lig_cumsum_tiles. */
size_t lig_cumsum_workspace_bytes(int num_points);

/* Inclusive int32 prefix sum of num_tiles_hit; the total (num_intersects) is
 * written to the device word *num_intersects, with no host synchronisation.
 * One kernel (a single-pass scan with decoupled look-back); num_tiles_hit and
 * cum_tiles_hit must not overlap and the workspace must be 8-byte aligned
 * (LIG_ERR_INVALID otherwise).
 * Replaces compute_cumulative_intersects (gsplat2d/gsplat2d/utils.py:61-67). */
int lig_cumsum_tiles(int num_points, const int32_t *num_tiles_hit, int32_t *cum_tiles_hit,
                     int32_t *num_intersects, void *workspace, size_t workspace_bytes,
                     void *stream);

/* Workspace bytes needed by lig_bin for `capacity` intersections over
 * num_tiles tiles (per-tile counters and cursors, the scan state). */
size_t lig_bin_workspace_bytes(int num_points, int capacity, int num_tiles);

/* Binning by tile in one call: per-tile counts of the emitted (Gaussian,
 * tile) slots, their prefix sum, a scatter of every slot into its tile's
 * range and a per-tile sort by Gaussian index, which gives the order of the
 * reference's stable sort of the emitted keys.  Reads the intersection count from the device word *num_intersects and
 * handles at most `capacity` of them; if more exist it sets
 * LIG_STATUS_OVERFLOW in *status (device int32, zeroed by the call) and the
 * outputs are incomplete.  Outputs: gaussian_ids_sorted [capacity],
 * tile_bins [T,2] ((0,0) for empty tiles); optional (may be NULL):
 * isect_ids / gaussian_ids (unsorted, int64 keys tile<<32) and
 * isect_ids_sorted.
 * Replaces bin_and_sort_gaussians (gsplat2d/gsplat2d/utils.py:70-100):
 * map_gaussian_to_intersects (csrc/bindings.cu:239-281), torch.sort +
 * torch.gather (utils.py:97-98) and get_tile_bin_edges (csrc/bindings.cu:283-301). */
int lig_bin(int dtype, int num_points, const void *xys, const void *extents,
            const int32_t *cum_tiles_hit, const int32_t *num_intersects, int img_h, int img_w,
            int block_width, int capacity, void *workspace, size_t workspace_bytes,
            int32_t *gaussian_ids_sorted, int32_t *tile_bins, int64_t *isect_ids,
            int32_t *gaussian_ids, int64_t *isect_ids_sorted, int32_t *status, void *stream);

/* Key emission only, reference-shaped (num_intersects given by the host).
 * Replaces map_gaussian_to_intersects_tensor (csrc/bindings.cu:239-281). */
int lig_map_intersects(int dtype, int num_points, int num_intersects, const void *xys,
                       const void *extents, const int32_t *cum_tiles_hit, int tiles_x,
                       int tiles_y, int block_width, int64_t *isect_ids, int32_t *gaussian_ids,
                       void *stream);

/* Tile ranges from sorted int64 keys; empty tiles get (0,0).
 * Replaces get_tile_bin_edges_tensor (csrc/bindings.cu:283-301). */
int lig_tile_bin_edges(int num_intersects, const int64_t *isect_ids_sorted, int num_tiles,
                       int32_t *tile_bins, void *stream);

/* ---------------------------------------------------------- rasterization */

/* Workspace bytes for lig_raster_fwd / lig_raster_bwd (packed records; the
 * workspace must be 16-byte aligned, LIG_ERR_INVALID otherwise). */
size_t lig_raster_workspace_bytes(int dtype, int num_points);

/* Weighted-sum rasterizer forward.  out_dx/out_dy/out_dxy == NULL selects the
 * plain sum; non-NULL selects the gradient-aware variant.  colors are [N,3].
 * When *num_intersects == 0 the image is all ones and the other outputs zero
 * (the reference's empty-list branch, rasterize.py:80-90).
 * Replaces rasterize_forward_tensor (csrc/bindings.cu:303-401). */
int lig_raster_fwd(int dtype, int img_h, int img_w, int block_width, int num_points,
                   const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                   const int32_t *num_intersects, const void *xys, const void *conics,
                   const void *colors, const void *opacities, void *workspace,
                   size_t workspace_bytes, void *out_img, void *out_wsum, void *out_dx,
                   void *out_dy, void *out_dxy, int32_t *final_idx, void *stream);

/* Rasterizer backward.  v_dx == NULL selects the sum variant (reference alpha
 * clamp 0.99), non-NULL the gradient-aware one (reference clamp 0.999);
 * alpha_clamp overrides the clamp when > 0.  v_wsum and v_opacity may be NULL
 * (v_wsum NULL = zero cotangent, an unused wsum output).  All outputs are
 * fully written.
 * Replaces rasterize_backward_tensor (csrc/bindings.cu:403-506). */
int lig_raster_bwd(int dtype, int img_h, int img_w, int block_width, int num_points,
                   const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                   const int32_t *num_intersects, const void *xys, const void *conics,
                   const void *colors, const void *opacities, const int32_t *final_idx,
                   const void *v_img, const void *v_wsum, const void *v_dx, const void *v_dy,
                   const void *v_dxy, double alpha_clamp, void *workspace,
                   size_t workspace_bytes, void *v_xy, void *v_xy_abs, void *v_conic,
                   void *v_rgb, void *v_opacity, void *stream);

/* Sum-rasterizer backward fused with the L2 fit loss: the pixel cotangent is
 * the gradient of mean((clamp(img, 0, 1) - target)^2) times the device scalar
 * *grad_loss, computed per pixel from img and target (both [H,W,3]) instead
 * of read from a materialised dL/dimg; wsum cotangent zero.  Otherwise as
 * lig_raster_bwd, except that with opacities == NULL v_xy_abs is written as
 * zeros (the fit uses neither it nor an opacity gradient, so the kernel
 * skips both).  Replaces, in the fit loop, the clamp + F.mse_loss backward
 * of gaussianlig.py:95-103 feeding rasterize_backward_tensor
 * (csrc/bindings.cu:403-506). */
int lig_raster_bwd_l2(int dtype, int img_h, int img_w, int block_width, int num_points,
                      const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                      const int32_t *num_intersects, const void *xys, const void *conics,
                      const void *colors, const void *opacities, const int32_t *final_idx,
                      const void *img, const void *target, const void *grad_loss,
                      double alpha_clamp, void *workspace, size_t workspace_bytes, void *v_xy,
                      void *v_xy_abs, void *v_conic, void *v_rgb, void *v_opacity,
                      void *stream);

/* Bytes of the per-tile loss partials of lig_raster_fwd_l2 (num_tiles
 * doubles; for the batched entry the batch's total tile count). */
size_t lig_l2_tile_partials_bytes(int num_tiles);

/* Fit-loop forward with the clamped-L2 loss fused in: the tile lists are
 * rendered as lig_raster_fwd, but per pixel `diff` [H,W,3] receives
 * (0 <= x <= 1) ? clamp(x, 0, 1) - target : 0 instead of the image x, and
 * *loss = mean((clamp(x, 0, 1) - target)^2) (gaussianlig.py:95-102) is reduced
 * deterministically from per-tile fp64 partials.  final_idx as
 * lig_raster_fwd, or NULL: the fit loop's backward without opacities never
 * reads it, and without it the forward neither tracks nor writes the
 * per-pixel last index (4 bytes a pixel).  The same holds for the _u8 and
 * batched forms below.  Workspace: lig_raster_workspace_bytes. */
int lig_raster_fwd_l2(int dtype, int img_h, int img_w, int block_width, int num_points,
                      const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                      const int32_t *num_intersects, const void *xys, const void *conics,
                      const void *colors, const void *opacities, const void *target,
                      void *workspace, size_t workspace_bytes, double *tile_partials,
                      void *diff, int32_t *final_idx, void *loss, void *stream);

/* Sum backward of that loss from the forward's diff: pixel cotangent
 * diff * 2 / (3 H W) * grad_loss (equal to lig_raster_bwd_l2's).  As in
 * lig_raster_bwd_l2, with opacities == NULL the fit needs neither |v_xy| nor
 * an opacity gradient: v_xy_abs is written as zeros and not accumulated;
 * final_idx is then not read and may be NULL (also in the batched form). */
int lig_raster_bwd_diff(int dtype, int img_h, int img_w, int block_width, int num_points,
                        const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                        const int32_t *num_intersects, const void *xys, const void *conics,
                        const void *colors, const void *opacities, const int32_t *final_idx,
                        const void *diff, const void *grad_loss, double alpha_clamp,
                        void *workspace, size_t workspace_bytes, void *v_xy, void *v_xy_abs,
                        void *v_conic, void *v_colors, void *v_opacity, void *stream);

/* Workspace bytes of lig_l2_clamped_loss. */
size_t lig_l2_workspace_bytes(void);

/* mean((clamp(img, 0, 1) - target)^2) over n elements into the device scalar
 * *loss, deterministic.  Replaces torch.clamp + F.mse_loss of the fit loop
 * (gaussianlig.py:95-102, utils.py:17-21). */
int lig_l2_clamped_loss(int dtype, int64_t n, const void *img, const void *target, void *loss,
                        void *workspace, size_t workspace_bytes, void *stream);

/* Bounded device-side waits that gave up on the current device since the
 * library loaded (the backward's optional bulk-copy staging polls an
 * mbarrier with an iteration limit and abandons the tile rather than hang);
 * 0 in normal operation, -1 if the query itself failed.  No counterpart in
 * the reference (its kernels have no device-side waits). */
int lig_wait_timeouts(void);

/* Check of the alpha cut (no counterpart in the reference).  The fused-loss
 * forward decides a pixel's alpha >= 1/255 test (the reference's
 * `sigma < 0 || alpha < 1/255` rejection, csrc/forward.cu:255-258) for
 * Gaussians with culling data by one unsigned compare of sigma's bit pattern
 * with a cut that the pack step finds on the device.  This entry
 * point writes into out[0..2] (device memory, three uint32, on `stream`): the
 * cut found by that search, and the first failing and last passing bit
 * pattern of a scan of the decision over every non-negative float up to
 * +inf (about a millisecond).  out[0] == out[1] == out[2] + 1 shows the
 * decision is a step at the cut. */
int lig_alpha_cut(uint32_t *out, void *stream);

/* Sum rasterizer forward that allocates nothing.  No counterpart in the
 * reference.  For callers that cannot allocate device memory when they render
 * (e.g. a plugin running inside a framework that has reserved nearly all GPU
 * memory for its own pool, or a real-time loop that forbids allocations after
 * start-up): the scratch lig_raster_fwd takes as `workspace` comes from a
 * fixed array inside the library (LIG_STATIC_MAX_POINTS records, 6 MiB per
 * GPU, held until the process exits).  float32 only; otherwise identical to
 * lig_raster_fwd with out_dx/out_dy/out_dxy = NULL.  Returns
 * LIG_ERR_TOO_LARGE when num_points > LIG_STATIC_MAX_POINTS.  The first call
 * on a device looks up the array's device address, so make it before any
 * stream capture (after a device reset the next call looks it up again).
 * All calls on a device share the array (each call rewrites the records it
 * uses): calls that overlap on that GPU, e.g. on two streams, race. */
#define LIG_STATIC_MAX_POINTS 131072
int lig_raster_fwd_noalloc(int img_h, int img_w, int block_width, int num_points,
                           const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                           const int32_t *num_intersects, const float *xys, const float *conics,
                           const float *colors, const float *opacities, float *out_img,
                           float *out_wsum, int32_t *final_idx, void *stream);

/* ---------------------------------------------------------------- upscale */

/* Gradient-aware Hermite-bicubic upscale of [src_h,src_w,3] value/dx/dy/dxy
 * planes to [dst_h,dst_w,3].  mode 0: half-pixel mapping over the ROI
 * (x1,y1,x2,y2), ROI extent truncated to int — replaces
 * gradient_aware_upscale_forward_tensor (csrc/bindings.cu:508-559);
 * mode 1: align-corners mapping (ROI ignored) — replaces
 * torch_gradient_aware_upscale (upscaler_torch.py:168-183). */
int lig_upscale_fwd(int dtype, int mode, int src_h, int src_w, int dst_h, int dst_w,
                    double roi_x1, double roi_y1, double roi_x2, double roi_y2,
                    const void *render, const void *dx, const void *dy, const void *dxy,
                    void *out, void *stream);

/* Upscale backward as a gather (each source texel written once, no atomics).
 * Replaces gradient_aware_upscale_backward_tensor (csrc/bindings.cu:561-605)
 * and the autograd of upscaler_torch.py. */
int lig_upscale_bwd(int dtype, int mode, int src_h, int src_w, int dst_h, int dst_w,
                    double roi_x1, double roi_y1, double roi_x2, double roi_y2,
                    const void *grad_out, void *grad_render, void *grad_dx, void *grad_dy,
                    void *grad_dxy, void *stream);

/* lig_upscale_fwd / lig_upscale_bwd for HWC planes of `channels` (1 or 3)
 * channels: channels == 1 is the single-channel form,
 * torch_gradient_aware_upscale_single_channel (upscaler_torch.py:91-165),
 * which the reference applies per channel; the 3-channel entries above are
 * these with channels == 3. */
int lig_upscale_fwd_nc(int dtype, int mode, int channels, int src_h, int src_w, int dst_h,
                       int dst_w, double roi_x1, double roi_y1, double roi_x2, double roi_y2,
                       const void *render, const void *dx, const void *dy, const void *dxy,
                       void *out, void *stream);
int lig_upscale_bwd_nc(int dtype, int mode, int channels, int src_h, int src_w, int dst_h,
                       int dst_w, double roi_x1, double roi_y1, double roi_x2, double roi_y2,
                       const void *grad_out, void *grad_render, void *grad_dx, void *grad_dy,
                       void *grad_dxy, void *stream);

/* Forward projection of a view of the Gaussians (region decode at a scale):
 * every Gaussian is first mapped to means' = (means - origin) * (sx, sy) and
 * L' = diag(sx, sy) L (cholesky != 0; the scale_to rule of
 * minimal_trainer_upscale.py:139-157) or cov' = S cov S, then projected as
 * lig_project_fwd onto an img_h x img_w output — a crop / rescaled render
 * without materialising the transformed parameters. */
int lig_project_fwd_view(int dtype, int num_points, int cholesky, const void *in3,
                         const void *means2d, const void *opacities, int img_h, int img_w,
                         int block_width, double origin_x, double origin_y, double scale_x,
                         double scale_y, void *xys, void *extents, void *conics,
                         int32_t *num_tiles_hit, void *stream);

/* ---------------------------------------------------------------- batched */

/* A batch of up to LIG_MAX_BATCH images processed by one launch per stage.
 * Image i has heights[i] x widths[i] pixels and counts[i] Gaussians (host
 * arrays of n_img int32).  Per-Gaussian arrays are the images' arrays
 * concatenated in batch order; [H,W,3] buffers likewise (image i starts at
 * pixel sum_{j<i} H_j W_j); tile lists are flattened image-major, so the
 * global tile of image i's local tile t is sum_{j<i} tiles_j + t.  Each image
 * behaves as if rendered alone: its tile keys, sorted ids (as global ids),
 * tile ranges (shifted), images and final indices are those of the
 * single-image calls, and its empty-list branch applies per image.  No
 * reference counterpart: the reference renders one image per call
 * (gaussianlig.py:88-93 in a per-image loop, train.py:112-158). */
#define LIG_MAX_BATCH 64

/* Projection of every Gaussian of the batch against its own image. */
int lig_project_fwd_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                          const int32_t *counts, int cholesky, const void *in3,
                          const void *means2d, const void *opacities, int block_width,
                          void *xys, void *extents, void *conics, int32_t *num_tiles_hit,
                          void *stream);
int lig_project_bwd_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                          const int32_t *counts, int cholesky, const void *in3,
                          const void *means2d, const void *opacities, int block_width,
                          const void *v_xy, int64_t v_xy_stride, const void *v_conic,
                          int64_t v_conic_stride, void *v_in3, void *v_mean2d, void *stream);

/* lig_bin over the whole batch (one count, scan, scatter and sort);
 * tile_bins has sum_i tiles_i entries.  Workspace: lig_bin_workspace_bytes
 * with the batch's total tile count.  cum / num_intersects as lig_bin (the
 * inclusive prefix sum over the concatenated counts). */
int lig_bin_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                  const int32_t *counts, int block_width, const void *xys, const void *extents,
                  const int32_t *cum, const int32_t *num_intersects, int capacity,
                  void *workspace, size_t workspace_bytes, int32_t *gaussian_ids_sorted,
                  int32_t *tile_bins, int32_t *status, void *stream);

/* Sum / gradient-aware forward over the flattened (image, tile) list.
 * persistent != 0: one CTA per resident slot pulls work items from *work
 * (one int32 of device memory, overwritten); else one CTA per tile.  cum:
 * the inclusive prefix sum of the counts (per-image empty test).
 * Workspace: lig_raster_workspace_bytes(dtype, total points). */
int lig_raster_fwd_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                         const int32_t *counts, int block_width,
                         const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                         const int32_t *num_intersects, const int32_t *cum, const void *xys,
                         const void *conics, const void *colors, const void *opacities,
                         int persistent, int32_t *work, void *workspace, size_t workspace_bytes,
                         void *out_img, void *out_wsum, void *out_dx, void *out_dy,
                         void *out_dxy, int32_t *final_idx, void *stream);

/* Sum backward of loss = sum_i mean((clamp(img_i, 0, 1) - target_i)^2),
 * the pixel cotangent 2/(3 H_i W_i) (clamp - target) * grad_loss formed in
 * the kernel (as lig_raster_bwd_l2 per image). */
int lig_raster_bwd_l2_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                            const int32_t *counts, int block_width,
                            const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                            const int32_t *num_intersects, const int32_t *cum, const void *xys,
                            const void *conics, const void *colors, const void *opacities,
                            const int32_t *final_idx, const void *img, const void *target,
                            const void *grad_loss, double alpha_clamp, int persistent,
                            int32_t *work, void *workspace, size_t workspace_bytes, void *v_xy,
                            void *v_xy_abs, void *v_conic, void *v_colors, void *v_opacity,
                            void *stream);

/* Batched lig_raster_fwd_l2: loss = sum_i mean_i(...), per_image[i] the
 * image's mean (may be NULL); tile_partials holds the batch's total tiles. */
int lig_raster_fwd_l2_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                            const int32_t *counts, int block_width,
                            const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                            const int32_t *num_intersects, const int32_t *cum, const void *xys,
                            const void *conics, const void *colors, const void *opacities,
                            const void *target, int persistent, int32_t *work, void *workspace,
                            size_t workspace_bytes, double *tile_partials, void *diff,
                            int32_t *final_idx, void *loss, void *per_image, void *stream);

/* lig_raster_fwd_l2 with an 8-bit target [H,W,3] (as lig_raster_fwd_l2_u8_batch
 * below: each byte counts as byte / 255 rounded to nearest). */
int lig_raster_fwd_l2_u8(int dtype, int img_h, int img_w, int block_width, int num_points,
                         const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                         const int32_t *num_intersects, const void *xys, const void *conics,
                         const void *colors, const void *opacities, const uint8_t *target,
                         void *workspace, size_t workspace_bytes, double *tile_partials,
                         void *diff, int32_t *final_idx, void *loss, void *stream);

/* lig_raster_fwd_l2_batch with an 8-bit target [sum_i H_i W_i, 3] (RGB
 * images as stored): each byte t counts as t / 255 rounded to nearest — the
 * float torchvision's ToTensor gives, which train.py's image loading uses
 * (train.py:30, 209-214) — so every output equals
 * lig_raster_fwd_l2_batch's with that float target, for a quarter of the
 * target's bytes.  No reference counterpart (the reference keeps the target
 * as fp32 on the device). */
int lig_raster_fwd_l2_u8_batch(int dtype, int n_img, const int32_t *heights,
                               const int32_t *widths, const int32_t *counts, int block_width,
                               const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                               const int32_t *num_intersects, const int32_t *cum,
                               const void *xys, const void *conics, const void *colors,
                               const void *opacities, const uint8_t *target, int persistent,
                               int32_t *work, void *workspace, size_t workspace_bytes,
                               double *tile_partials, void *diff, int32_t *final_idx, void *loss,
                               void *per_image, void *stream);

/* Batched lig_raster_bwd_diff (per-image scale 2 / (3 H_i W_i)). */
int lig_raster_bwd_diff_batch(int dtype, int n_img, const int32_t *heights,
                              const int32_t *widths, const int32_t *counts, int block_width,
                              const int32_t *gaussian_ids_sorted, const int32_t *tile_bins,
                              const int32_t *num_intersects, const int32_t *cum, const void *xys,
                              const void *conics, const void *colors, const void *opacities,
                              const int32_t *final_idx, const void *diff, const void *grad_loss,
                              double alpha_clamp, int persistent, int32_t *work, void *workspace,
                              size_t workspace_bytes, void *v_xy, void *v_xy_abs, void *v_conic,
                              void *v_colors, void *v_opacity, void *stream);

/* Workspace bytes of lig_l2_clamped_loss_batch. */
size_t lig_l2_batch_workspace_bytes(int n_img);

/* loss = sum_i mean((clamp(img_i, 0, 1) - target_i)^2) (0-d), per_image[i] =
 * that image's mean (may be NULL); deterministic; a batch of one gives
 * lig_l2_clamped_loss's value bit for bit. */
int lig_l2_clamped_loss_batch(int dtype, int n_img, const int32_t *heights,
                              const int32_t *widths, const void *img, const void *target,
                              void *loss, void *per_image, void *workspace,
                              size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------- level pipeline */

/* Residual target of the next level (train.py:113-126): with
 * r = gt - up + 0.5 over n floats, out = (r - min r) / (max r - min r) and
 * minmax[0..1] = (min r, max r) (device floats; the level's store_min /
 * store_max).  Bit-identical to the torch expression on NaN-free inputs. */
int lig_level_residual(int64_t n, const float *gt, const float *up, float *out, float *minmax,
                       void *stream);

/* One level of a multi-level decode (train.py:188-200): out[H,W,3] =
 * base + (r * (max - min) - 0.5 + min), r = render (clamped to [0,1] when
 * clamp_render), base = prev [prev_h, prev_w, 3] resized to H x W by
 * bilinear half-pixel sampling (F.interpolate mode='bilinear'), or prev itself
 * when the sizes agree, or 0 when prev is NULL; (min, max) from minmax
 * (device floats) when given, else store_min / store_max; clamp_out clamps
 * the result to [0, 1]. */
int lig_level_compose(int prev_h, int prev_w, const float *prev, int H, int W,
                      const float *render, const float *minmax, double store_min,
                      double store_max, int clamp_render, int clamp_out, float *out,
                      void *stream);

/* -------------------------------------------------------------- optimiser */

/* Scratch bytes of lig_adam_step (device memory, 16 B). */
size_t lig_adam_scratch_bytes(void);

/* One Adam step over a flat fp32 buffer of n parameters (16-byte aligned
 * params / grads / moments), for the fit loops' optimiser
 * (gaussianlig.py:64-68: Adam over every Gaussian parameter).  *step
 * (device int32) counts applied steps and gives the bias corrections.  If
 * status (device int32, may be NULL) has LIG_STATUS_OVERFLOW set — the
 * binning of this step overflowed its capacity — nothing is updated and
 * *skipped (device int32, may be NULL) is incremented. */
int lig_adam_step(int64_t n, float *params, const float *grads, float *exp_avg,
                  float *exp_avg_sq, double lr, double beta1, double beta2, double eps,
                  const int32_t *status, int32_t *step, int32_t *skipped, void *scratch,
                  void *stream);

/* Scratch bytes of lig_adam_step_batch (device memory). */
size_t lig_adam_batch_scratch_bytes(int n_img);

/* Adam over a batch of fits in one flat fp32 buffer laid out
 * [means 2N | cholesky 3N | rgb 3N] (N = sum of counts, image i owning
 * Gaussians [sum_{j<i} counts_j, sum_{j<=i} counts_j)); steps (device
 * int32[n_img]) are per image, so each image follows the updates of its own
 * fit.  status / skipped as lig_adam_step. */
int lig_adam_step_batch(int n_img, const int32_t *counts, float *params, const float *grads,
                        float *exp_avg, float *exp_avg_sq, double lr, double beta1, double beta2,
                        double eps, const int32_t *status, int32_t *steps, int32_t *skipped,
                        void *scratch, size_t scratch_bytes, void *stream);

/* ----------------------------------------------------------------- probes */

/* FP32 FMA throughput probe: blocks x 256 threads, each `iters` x 8
 * independent FMAs (2 FLOP each).  Used to measure the FP32 roofline
 * denominator on the device.  No reference counterpart (measurement aid). */
int lig_probe_fp32(int blocks, int iters, float *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* LIG_B200_H */
