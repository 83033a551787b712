/*
 * filtergs_b200 -- C ABI of the B200 (sm_100a) FilterGS rasterizer.
 *
 * Plain device pointers, sizes and a cudaStream_t passed as void*.  No torch
 * types.  Every entry point returns an FGS_* status.  All pointers named in
 * an argument list are device pointers unless the comment says "host".
 *
 * The reference interface each entry point replaces is cited beside it
 * (paths inside the reference project xenon-w/FilterGS).
 */
#ifndef FILTERGS_B200_H
#define FILTERGS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define FGS_OK 0
#define FGS_ERR_ARG 1          /* invalid argument (shape, null pointer, size)          */
#define FGS_ERR_CUDA 2         /* a CUDA runtime call or launch failed                  */
#define FGS_ERR_TIMEOUT 3      /* a bounded device-side wait gave up                    */
#define FGS_ERR_PREFILTERED 4  /* prefiltered set, yet a Gaussian failed the near test   */
#define FGS_ERR_CAPACITY 5     /* a preallocated capacity was exceeded                  */
#define FGS_ERR_OVERFLOW 6     /* more tile/Gaussian pairs than the binning supports    */

#define FGS_BACKWARD_REF_COMPAT 0 /* reproduce the reference backward (+0.3 dilation)    */
#define FGS_BACKWARD_CONSISTENT 1 /* differentiate exactly what the forward computed     */

#define FGS_STATS_SLOTS 64        /* RenderStats::MAX_KPC_BINS (rasterizer.h:24)        */

/* Human-readable text of a status code (static storage). */
const char *fgs_status_string(int status);
/* Library version string. */
const char *fgs_version(void);

/* ------------------------------------------------------------------ arguments
 * One rasterizer call.  Mirrors the argument list of
 * RasterizeGaussiansCUDA (antialias/rasterize_points.cu:36-62) after the
 * binding resolved its empty tensors to null pointers (:112-135).          */
typedef struct fgs_raster_args {
    int P;                       /* number of Gaussians                                   */
    int D;                       /* active SH degree                                     */
    int M;                       /* SH coefficients per channel (0 when shs is null)      */
    int width, height;           /* image size in pixels                                  */
    const float *background;     /* [3]                                                   */
    const float *means3D;        /* [P,3]                                                 */
    const float *shs;            /* [P,M,3] or null                                       */
    const float *colors_precomp; /* [P,3]  or null (exactly one of shs / colors_precomp)  */
    const float *opacities;      /* [P]                                                   */
    const float *scales;         /* [P,3]  or null                                        */
    float scale_modifier;
    const float *rotations;      /* [P,4] (r,x,y,z) or null                               */
    const float *cov3D_precomp;  /* [P,6]  or null (exactly one of scale+rot / cov3D)     */
    const float *viewmatrix;     /* [16] column-major world->view                         */
    const float *projmatrix;     /* [16] column-major world->clip                         */
    const float *campos;         /* [3]                                                   */
    float tan_fovx, tan_fovy;
    int prefiltered;             /* reference traps on a violation; here FGS_ERR_PREFILTERED */
    int use_filter;              /* 2D dilation: cov2D diagonal = max(., 0.3)             */
    float ogfs_epsilon_scale, ogfs_epsilon_max, ogfs_energy_floor, ogfs_radius_ratio_min;
    int ogfs_enable_stats;       /* compute the KPC/GTC statistics vector                 */
    float filter3d_scale;        /* 3D filter: cov3D += (s * z_view / focal_x)^2 I; 0 = off (no reference counterpart) */
} fgs_raster_args;

/* ------------------------------------------------------------------ workspaces
 * The three opaque byte buffers of the reference forward/backward
 * (geomBuffer / imageBuffer / binningBuffer, rasterizer_impl.cu:211-250).
 * Their layout is private to this library; they only need the returned size
 * and 256-byte alignment, and are passed unchanged from forward to backward. */
size_t fgs_geom_bytes(int P);
size_t fgs_image_bytes(int width, int height);
size_t fgs_binning_bytes(long long num_rendered, int P);

/* ------------------------------------------------------------------ forward
 * CudaRasterizer::Rasterizer::forward (rasterizer.h:49-76,
 * rasterizer_impl.cu:254-563), split at the point where the reference copies
 * num_rendered to the host (rasterizer_impl.cu:367):
 *   1. fgs_forward_preprocess: preprocess + depth ordering; synchronises the
 *      stream once and returns num_rendered (host long long) and writes radii
 *      ([P] int, may be null).
 *   2. the caller allocates fgs_binning_bytes(num_rendered, P);
 *   3. fgs_forward_render: binning, sort, tile ranges, compositing.
 * Outputs are fully written (no zero-initialisation needed):
 *   out_color [3,H,W], out_point_id [H,W], out_point_weight_pixel [H,W],
 *   out_point_weight [P].  When ogfs_enable_stats is set, stats_host (host,
 *   stats_len doubles) receives the reference's statistics vector
 *   (rasterize_points.cu:138-177): 9 + 2*FGS_STATS_SLOTS + 2*tiles values,
 *   and the call synchronises the stream.                                   */
int fgs_forward_preprocess(const fgs_raster_args *a, void *geom, void *image, int *radii,
                           long long *num_rendered, void *stream);
int fgs_forward_render(const fgs_raster_args *a, void *geom, void *image, void *binning, long long num_rendered,
                       const int *radii, float *out_color, int *out_point_id, float *out_point_weight_pixel,
                       float *out_point_weight, double *stats_host, int stats_len, void *stream);

/* ------------------------------------------------------------------ backward
 * CudaRasterizer::Rasterizer::backward (rasterizer.h:82-111,
 * rasterizer_impl.cu:582-676) and RasterizeGaussiansBackwardCUDA
 * (rasterize_points.cu:181-260).  All gradient outputs are fully written:
 *   dL_dmeans2D [P,3], dL_dconic [P,4], dL_dopacity [P], dL_dcolors [P,3],
 *   dL_dmeans3D [P,3], dL_dcov3D [P,6], dL_dsh [P,M,3] (may be null when M==0),
 *   dL_dscales [P,3], dL_drotations [P,4] (both may be null when scales is null).
 * radii: the forward's radii (may be null; not read): the Gaussians with radii > 0
 *   receive gradients, as in the reference (backward.cu:156,367), and geom holds
 *   their list from the forward.
 * backward_mode: FGS_BACKWARD_REF_COMPAT or FGS_BACKWARD_CONSISTENT.        */
int fgs_backward(const fgs_raster_args *a, const void *geom, const void *image, const void *binning,
                 long long num_rendered, const int *radii, const float *dL_dout_color, float *dL_dmeans2D,
                 float *dL_dconic, float *dL_dopacity, float *dL_dcolors, float *dL_dmeans3D, float *dL_dcov3D,
                 float *dL_dsh, float *dL_dscales, float *dL_drotations, int backward_mode, void *stream);

/* Synchronise `stream` and return the first error recorded by device code in
 * `geom` (FGS_OK when none).  The debug flag of the Python API calls this. */
int fgs_check(const void *geom, void *stream);

/* ------------------------------------------------------------------ utilities
 * markVisible (rasterizer_impl.cu:197-209, rasterize_points.cu:299-318): present[P] bytes 0/1. */
int fgs_mark_visible(int P, const float *means3D, const float *viewmatrix, const float *projmatrix,
                     uint8_t *present, void *stream);
/* _C.compute_radius (forward.cu:208-263, rasterize_points.cu:263-296): 3-sigma radius, float[P]. */
int fgs_compute_radius(int P, int height, int width, const float *means3D, const float *scales,
                       const float *rotations, const float *viewmatrix, const float *projmatrix, float tan_fovx,
                       float tan_fovy, float *radii, void *stream);
/* FilterGS compute_radius_v2.compute_radius (compute_radius_kernel_v2.cu:180-229,355-380). */
int fgs_compute_radius_v2(int P, const float *means3D, const float *scales, const float *rotations,
                          const float *projmatrix, const float *viewmatrix, float focal_x, float focal_y,
                          float tan_fovx, float tan_fovy, float *radii, void *stream);
/* FilterGS compute_visibility_radius (compute_radius_kernel_v2.cu:231-353,382-430):
 * mask[P] bytes, radius2d[P], depth[P].  ancestor_path is [P, max_level] int32. */
int fgs_visibility_radius(int P, const float *means3D, const float *log_scales, const float *rotations,
                          const float *projmatrix, const float *viewmatrix, const int32_t *tree_node_index,
                          const int32_t *ancestor_path, int max_level, float focal_x, float focal_y,
                          float tan_fovx, float tan_fovy, float padding, float radius_max,
                          float radius_filter_threshold, uint8_t *mask, float *radius2d, float *depth,
                          void *stream);

/* ------------------------------------------------------------------ batched views
 * No counterpart in the reference (it renders one view per call, with a host
 * synchronisation in each).  Many views of one Gaussian set: per view the
 * front end runs with its pair count kept on the device, and compositing --
 * forward and backward -- is one persistent launch over the tiles of all
 * views.  After fgs_batch_create, forward/backward enqueue work only (no host
 * synchronisation, no allocation), so they can be captured in a CUDA graph.
 * Gradients of all views are summed into the shared dense outputs given at
 * creation.  A view whose pairs exceed pair_capacity is truncated and
 * FGS_ERR_OVERFLOW is reported by fgs_batch_check.                          */
typedef struct fgs_view_args {
    int width, height;
    float tan_fovx, tan_fovy;
    const float *viewmatrix;      /* [16] device */
    const float *projmatrix;      /* [16] device */
    const float *campos;          /* [3] device */
    long long pair_capacity;      /* tile/Gaussian pairs reserved for this view */
    float *out_color;             /* [3,H,W] forward output */
    int *out_radii;               /* [P] or null */
    const float *dL_dout_color;   /* [3,H,W] backward input (read by fgs_batch_backward) */
} fgs_view_args;
/* Workspace bytes for P Gaussians and these views (their sizes and capacities). */
size_t fgs_batch_workspace_bytes(int P, int nviews, const fgs_view_args *views);
/* `shared` carries the Gaussians and global settings (its camera fields are ignored).
 * Shared gradient outputs (dense, summed over views): dL_dmeans3D [P,3], dL_dopacity [P],
 * dL_dsh [P,M,3] (null if no SH), dL_dscales [P,3], dL_drotations [P,4] (null with cov3D_precomp).
 * Returns a handle (null on error, *status set); synchronises `stream` once.            */
void *fgs_batch_create(const fgs_raster_args *shared, int nviews, const fgs_view_args *views, void *workspace,
                       size_t workspace_bytes, int backward_mode, float *dL_dmeans3D, float *dL_dopacity,
                       float *dL_dsh, float *dL_dscales, float *dL_drotations, int *status, void *stream);
int fgs_batch_forward(void *handle, void *stream);
int fgs_batch_backward(void *handle, void *stream);
/* Re-target the image output and upstream-gradient input ([3,H,W] each) of `count`
 * views (view_ids[i] -> out_color[i], dL_dout_color[i]) for the launches that follow on
 * `stream`.  The compositing kernels read these pointers from device memory, so a graph
 * captured from fgs_batch_forward/backward follows the change without re-capture
 * (double-buffered I/O).  dL_dout_color, or an entry of it, may be null (kept).     */
int fgs_batch_set_view_io(void *handle, int count, const int *view_ids, float *const *out_color,
                          const float *const *dL_dout_color, void *stream);
/* Optional per-view forward outputs of the reference's call (rasterize_points.cu:178):
 * out_point_id [H,W] (the strongest contributor of each pixel, -1 for none),
 * out_point_weight_pixel [H,W] (its weight T*alpha) and out_point_weight [P] (each
 * Gaussian's largest weight in the view, zeroed by every forward).  Arrays or entries
 * may be null (that output off).  Like fgs_batch_set_view_io, a captured graph follows
 * the change without re-capture.  No reference counterpart for the batching itself. */
int fgs_batch_set_view_outputs(void *handle, int count, const int *view_ids, int *const *out_point_id,
                               float *const *out_point_weight_pixel, float *const *out_point_weight, void *stream);
/* Pair counts of the last forward per view (host [nviews]); synchronises. */
int fgs_batch_pair_counts(void *handle, long long *counts, void *stream);
/* Synchronise and return the first device-side error of the batch (FGS_OK when none). */
int fgs_batch_check(void *handle, void *stream);
void fgs_batch_destroy(void *handle);
/* Optional training statistics, accumulated by every fgs_batch_backward (views in order):
 * grad_sum[P] += |dL/dmeans2D[:2]| and vis_count[P] += 1 per view that sees the Gaussian,
 * flag[P] = 1 (the caller zeroes the flags between steps).  All null: off.
 * LoG/model/counter.py:36-83 (the two statistics the training step keeps).            */
int fgs_batch_set_densify(void *handle, float *grad_sum, int *vis_count, unsigned char *flag);

/* ------------------------------------------------------------------ training step
 * The loss, optimizer and statistics of LoG's training loop around the rasterizer.   */
/* Scratch bytes of fgs_loss_l1_ssim for one [3,H,W] image (0 if the image is smaller than
 * the 11x11 window). */
size_t fgs_loss_scratch_bytes(int width, int height);
/* LoG/render/loss.py:6-44 + renderer.py:260-273.  For one view: writes
 *   dL_dpred = l1_grad_scale * sign(pred - target) + ssim_grad_scale * d(1 - ssim_sum)/dpred
 * (SSIM: 11x11 Gaussian window, sigma 1.5, no padding) and adds the view's sum |pred - target|
 * to sums[0] and its sum of SSIM map values to sums[1] (doubles on the device, in a fixed
 * order).  For the loss 0.8 L1 + 0.2 (1 - SSIM) over a batch: l1_grad_scale =
 * 0.8 / (batch * 3 * H * W), ssim_grad_scale = 0.2 / (batch * 3 * (H-10) * (W-10)).    */
int fgs_loss_l1_ssim(int width, int height, const float *pred, const float *target, float *dL_dpred,
                     float l1_grad_scale, float ssim_grad_scale, double *sums, void *scratch, void *stream);
/* LoG/model/activation.py: scale = exp(log_scale), rot = normalize(rot_raw), opac = sigmoid(logit). */
int fgs_train_activate(int P, const float *log_scale, const float *rot_raw, const float *opac_logit, float *scale,
                       float *rot, float *opac, void *stream);
/* One view of the plain path: for radii > 0, grad_sum += |dL_dmeans2D[:2]|, vis_count += 1, flag = 1. */
int fgs_densify_dense(int P, const int *radii, const float *dL_dmeans2D, float *grad_sum, int *vis_count,
                      unsigned char *flag, void *stream);
/* LoG/model/sparse_optimizer.py:41-78,163-196: one Adam step (the device step counter is
 * incremented first; bias corrections from it; eps as given) on the rows with flag set.
 * Gradients are w.r.t. the rasterizer's inputs (means, SH, activated opacity / scale,
 * normalised rotation) and are chained through the activations; the activated values of
 * the updated rows are rewritten.  lr: means, SH, opacity, scale, rotation.             */
typedef struct fgs_adam_args {
    int P, M;                     /* Gaussians, SH coefficients per channel (0: no SH) */
    float lr[5];
    double beta1, beta2;          /* as the reference's Python floats: 1 - beta is formed in double */
    float eps;
    float *xyz, *shs, *opac_logit, *log_scale, *rot_raw;      /* raw parameters (updated) */
    float *opac, *scale, *rot;                                /* activated (rewritten) */
    const float *g_xyz, *g_shs, *g_opac, *g_scale, *g_rot;    /* gradients */
    float *m_xyz, *m_shs, *m_opac, *m_scale, *m_rot;          /* first moments */
    float *v_xyz, *v_shs, *v_opac, *v_scale, *v_rot;          /* second moments */
} fgs_adam_args;
int fgs_adam_step(const fgs_adam_args *a, const unsigned char *flag, int *step, void *stream);

/* ------------------------------------------------------------------ LoD selection and gather
 * gather_attributes_cuda (FilterGS/cuda/gather_attributes_kernel.cu:70-145): rows of xyz/scaling [.,3],
 * rotation [.,4] (16-byte aligned), opacity [.,1], colors [.,3] and optional shs [., sh_coeffs, sh_channels]
 * at index[0..N) (int64) into the o_* outputs.                                                       */
int fgs_gather_attributes(long long N, const int64_t *index, const float *xyz, const float *scaling,
                          const float *rotation, const float *opacity, const float *colors, const float *shs,
                          int sh_coeffs, int sh_channels, float *o_xyz, float *o_scaling, float *o_rotation,
                          float *o_opacity, float *o_colors, float *o_shs, void *stream);
/* torch.nonzero(mask) of FilterGS/filtergs.py:64 without the host sync: ordered int64 indices of the
 * nonzero bytes of mask[n]; the count stays on the device (*count, u64).  scratch:
 * fgs_compact_scratch_bytes(n) bytes, 4-byte aligned.                                                 */
size_t fgs_compact_scratch_bytes(int n);
int fgs_compact_mask(int n, const uint8_t *mask, int64_t *out_index, unsigned long long *count, void *scratch,
                     void *stream);
/* FilterGS get_all (FilterGS/filtergs.py:98-134) fused: gather index[0..min(N_cap, *count_dev)) and
 * apply LoG/model/activation.py:36-43 -- exp(scale), sigmoid(opacity), F.normalize(rotation),
 * SH2RGB(features_dc) + eval_sh_wobase(shs_rest, sh_degree) (LoG/model/sh_utils.py:31-74).
 * count_dev may be null (then N_cap rows).                                                           */
int fgs_gather_activate(long long N_cap, const int64_t *index, const unsigned long long *count_dev,
                        const float *xyz, const float *log_scale, const float *rotation, const float *opacity_raw,
                        const float *features_dc, const float *shs_rest, int sh_degree, int rest_coeffs,
                        const float *campos, float *o_xyz, float *o_scaling, float *o_rotation, float *o_opacity,
                        float *o_colors, void *stream);
/* FilterGS.render's guard (FilterGS/filtergs.py:159-172): keep[n] = 1 for the rows whose xyz,
 * scaling, rotation, opacity and colour (the activated rows of fgs_gather_activate) are all
 * finite, with min(scaling) > 0 and opacity > 0; *dropped (device, u64) counts the others.  */
int fgs_rows_valid(long long N, const float *xyz, const float *scaling, const float *rotation, const float *opacity,
                   const float *colors, uint8_t *keep, unsigned long long *dropped, void *stream);
/* The LoG node radius (LoG/model/level_of_gaussian.py:66-88 -> compute_radius_kernel_v2.cu:180-229)
 * from raw parameters: exp(log_scales) and the normalised quaternion are applied in the kernel.        */
int fgs_radius_raw(int P, const float *means3D, const float *log_scales, const float *rotations,
                   const float *viewmatrix, const float *projmatrix, float focal_x, float focal_y, float tan_fovx,
                   float tan_fovy, float *radius, void *stream);
/* TensorTree.traverse (LoG/model/tensor_tree.py:133-187) on the device: node ids of the cut in the
 * reference's order (kept roots, then each level's kept children in frontier order) into out[P]; the
 * count to *out_count_dev (u32, device).  tree: [num_internal, max_child] child ids (-1 = none);
 * levels = the deepest level to expand (the reference stops at 30).  No host synchronisation.
 * scratch: fgs_log_cut_scratch_bytes(...) bytes.                                                     */
size_t fgs_log_cut_scratch_bytes(int P, int num_roots, int max_child, int levels);
int fgs_log_cut(int P, const int32_t *roots, int num_roots, const int32_t *node_index, const int32_t *tree,
                int max_child, const float *radius, float min_resolution_pixel, int levels, int32_t *out,
                uint32_t *out_count_dev, void *scratch, void *stream);
/* Redundancy culling of a node list (no reference counterpart): keep ids[i] (i < *count_dev) with
 * radius >= min_px and sigmoid(opacity_raw) >= 1/255, order preserved, as int64 into out; count to
 * *out_count_dev.  scratch: fgs_compact_scratch_bytes(cap) bytes.                                   */
int fgs_cull(const int32_t *ids, const uint32_t *count_dev, int cap, const float *radius, const float *opacity_raw,
             float min_px, int64_t *out, unsigned long long *out_count_dev, void *scratch, void *stream);
/* ancestor_path of a LoG tree (replaces rebuild_ancestor_path, apps/ancestor.py:21-73, a per-level
 * torch loop): out[i, k] = id of node i's ancestor at depth k, -1 elsewhere, [P, L] int32 row-major,
 * from index_parent [P] and depth [P] (int32).  Same result as the reference's level order, also for
 * trees whose depths disagree with their parents'.  Where the reference raises (a parent id >= P, or a
 * node with a parent at depth > L) the kernel leaves FGS_ERR_ARG in *err_dev (bit 1 << code, zeroed
 * here) and the row unfinished.  No host synchronisation.                                             */
int fgs_ancestor_path(int P, const int32_t *index_parent, const int32_t *depth, int L, int32_t *out,
                      unsigned *err_dev, void *stream);

/* ------------------------------------------------------------------ test accessors
 * Sorted (tile|depth) keys and Gaussian ids of a forward, in the reference's
 * 64-bit key format (rasterizer_impl.cu:139-141).  keys/vals: [num_rendered]. */
int fgs_sorted_pairs(const void *geom, const void *binning, int P, long long num_rendered, uint64_t *keys,
                     uint32_t *vals, void *stream);
/* Per-Gaussian preprocess outputs kept in geom: means2D [P,2], depth [P],
 * conic_opacity [P,4], rgb [P,3], tiles_touched [P] (any may be null). */
int fgs_preprocess_outputs(const void *geom, int P, float *means2D, float *depths, float *conic_opacity,
                           float *rgb, uint32_t *tiles_touched, void *stream);
/* Per-pixel state kept in image: final transmittance [H*W], n_contrib [H*W], ranges [tiles,2]. */
int fgs_image_outputs(const void *image, int width, int height, float *final_T, uint32_t *n_contrib,
                      uint32_t *ranges, void *stream);

/* ------------------------------------------------------------------ forward without allocation
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they render (a render thread that must not pay cudaMalloc's
 * device-wide synchronisation, a plugin inside an application that owns all
 * device memory, a process under a fixed memory budget): the whole forward
 * (preprocess, binning, sort, compositing; no statistics) with its scratch
 * workspaces in one library-owned device array of fgs_noalloc_capacity_bytes()
 * (32 MiB) that every GPU loading this library keeps until exit.  The caller
 * passes the inputs in `a` and the outputs: radii [P] int, out_color [3,H,W],
 * out_point_id [H,W], out_point_weight_pixel [H,W], out_point_weight [P];
 * num_rendered (host) receives the pair count.  Workspaces that do not fit
 * the array are rejected with FGS_ERR_CAPACITY (checked before any work for
 * the per-Gaussian and per-pixel state, after preprocessing for the pairs: a
 * call refused there has already written radii).  ogfs_enable_stats must be 0
 * (FGS_ERR_ARG otherwise).  Each call looks up the array's device address on
 * the current device; the first call on a device loads the library's device
 * code, so it should come before any stream capture.  The call synchronises
 * `stream`; a CUDA error left pending by earlier work on the device is
 * reported as FGS_ERR_CUDA.  Calls share the array: two calls that overlap on
 * the GPU race and must be serialised by the caller.                       */
size_t fgs_noalloc_capacity_bytes(void);
int fgs_forward_noalloc(const fgs_raster_args *a, int *radii, float *out_color, int *out_point_id,
                        float *out_point_weight_pixel, float *out_point_weight, long long *num_rendered,
                        void *stream);

/* ------------------------------------------------------------------ profiling hooks
 * No reference counterpart (the reference times stages with torch CUDA events
 * around whole calls, FilterGS/filtergs.py:26-39).  When enabled, forward and
 * backward record a CUDA event pair around each stage below; fgs_profile_read
 * synchronises on those events and returns the summed milliseconds and call
 * counts per stage.  fgs_launch_count is the number of kernels this library
 * has launched in the process (memsets and copies excluded).               */
#define FGS_STAGE_PREPROCESS 0
#define FGS_STAGE_DEPTH_SORT 1
#define FGS_STAGE_DUPLICATE 2
#define FGS_STAGE_TILE_SORT 3
#define FGS_STAGE_RANGES 4
#define FGS_STAGE_RENDER_FWD 5
#define FGS_STAGE_STATS 6
#define FGS_STAGE_RENDER_BWD 7
#define FGS_STAGE_PREPROCESS_BWD 8
#define FGS_NUM_STAGES 9
int fgs_profile_enable(int on);
/* Render kernel shape used by forward/backward in this process (no reference
 * counterpart; the reference hard-codes one pixel per thread and 256-record
 * batches): pixels per thread 1|2|4 and shared-memory batch 64|128|256 for
 * each of the forward and backward compositing kernels.  Chosen by the
 * autotuner (filtergs_b200/autotune.py).  cfg: int[4] out.             */
int fgs_set_render_config(int fwd_ppt, int fwd_batch, int bwd_ppt, int bwd_batch);
int fgs_get_render_config(int *cfg);
/* Forward: tiles with at least min_records tile/Gaussian pairs are rendered in bands of pixels, one
 * warp per band and four bands per CTA, longest tiles first, before the other tiles (min_records 0,
 * the default: never).
 * band_shape: 0 = 16x2, 1 = 8x4, 2 = 4x4, 3 = 4x2 pixels per band.  The outputs do not change; long
 * tiles stop being the critical path of the forward.  Process-wide, like the above.
 * fgs_get_render_split: cfg int[2] out (min_records, band_shape).                                   */
int fgs_set_render_split(int min_records, int band_shape);
int fgs_get_render_split(int *cfg);
int fgs_profile_read(double *ms, long long *calls, int reset);
long long fgs_launch_count(void);

/* Failure-path test hook (no reference counterpart; the reference has no bounded
 * waits).  From the next forward on, chunk `skip_chunk` of the first depth-sort
 * pass never publishes its look-back counts, so the chunks after it wait until
 * `wait_ns` nanoseconds run out (0: the default one-second limit), record
 * FGS_ERR_TIMEOUT and finish; fgs_forward_preprocess then returns
 * FGS_ERR_TIMEOUT.  skip_chunk = 0xffffffff switches the hook off.  Only the
 * depth sort's keys and ids move in that pass, so the wrong offsets of a timed-out
 * pass stay inside its buffers.  Process-wide; for tests only.               */
int fgs_debug_lookback_fault(unsigned int skip_chunk, unsigned long long wait_ns);

#ifdef __cplusplus
}
#endif
#endif /* FILTERGS_B200_H */
