/*
 * mbirjax_b200 -- C ABI of the B200 (sm_100a) kernels for the MBIR hot path.
 *
 * Every entry point takes raw device pointers, sizes and a cudaStream_t (passed as void*), returns 0 on
 * success or a negative MBX_ERR_* code, never throws and never traps.  The caller owns all buffers;
 * entry points that need scratch memory take a caller-provided workspace whose size the matching
 * *_workspace_bytes query returns.  Nothing synchronises the stream, so every entry point can be
 * captured in a CUDA graph.  Out-of-range pixel or view indices found on the device are skipped and
 * recorded in a device error word that mbx_get_device_error() reads (and clears).
 *
 * Data layout (all float32, C order):
 *   recon / flat recon     (num_recon_rows * num_recon_cols, num_recon_slices)  -- one voxel cylinder per pixel
 *   voxel_values           (num_pixels, num_recon_slices)
 *   sinogram               (num_views, num_det_rows, num_det_channels)
 *   pixel_indices          int32, indices into the flattened (num_recon_rows, num_recon_cols) grid
 *   view_indices           int32 or NULL (NULL = all views in order)
 *
 * Each declaration names the reference (mbirjax v0.6.7) interface it replaces.
 */
#ifndef MBIRJAX_B200_H
#define MBIRJAX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MBX_API __attribute__((visibility("default")))
#else
#define MBX_API
#endif

#define MBX_OK 0
#define MBX_ERR_INVALID_ARG (-1)
#define MBX_ERR_UNSUPPORTED (-2)
#define MBX_ERR_CUDA (-3)
#define MBX_ERR_WORKSPACE (-4)

#define MBX_GEOM_PARALLEL 0
#define MBX_GEOM_CONE 1
#define MBX_GEOM_TRANSLATION 2

/* Largest psf_radius / bp_psf_radius the kernels accept. */
#define MBX_MAX_PSF_RADIUS 4

/* Projector geometry.  Replaces the (sinogram_shape, recon_shape, geometry_params) namedtuple that
 * Projectors.create_projectors closes over (projectors.py:47-54), built from
 * ParallelBeamModel.get_geometry_parameters (parallel_beam.py:94-113),
 * ConeBeamModel.get_geometry_parameters (cone_beam.py:110-136) or
 * TranslationModel.get_geometry_parameters (translation_model.py:83-107).  For MBX_GEOM_TRANSLATION the
 * object moves by a translation vector per view in front of a fixed cone-beam source (no rotation): angles is
 * unused (may be NULL), psf_radius serves both fans, and bp_psf_radius / recon_slice_offset are unused. */
typedef struct mbx_geom {
    int32_t kind;                        /* MBX_GEOM_PARALLEL or MBX_GEOM_CONE */
    int32_t num_views;                   /* sinogram_shape[0]; length of angles */
    int32_t num_det_rows;                /* sinogram_shape[1] */
    int32_t num_det_channels;            /* sinogram_shape[2] */
    int32_t num_recon_rows;              /* recon_shape[0] */
    int32_t num_recon_cols;              /* recon_shape[1] */
    int32_t num_recon_slices;            /* recon_shape[2] (== num_det_rows for parallel beam) */
    int32_t psf_radius;                  /* get_psf_radius() */
    int32_t bp_psf_radius;               /* cone only: ConeBeamModel.bp_psf_radius */
    int32_t entries_per_cylinder_batch;  /* cone only: 128 in the reference */
    float delta_det_channel;
    float delta_det_row;
    float det_channel_offset;
    float det_row_offset;
    float delta_voxel;
    float recon_slice_offset;            /* cone only */
    float source_detector_dist;          /* cone only; +inf allowed */
    float magnification;                 /* cone only; source_detector_dist / source_iso_dist */
    const float *angles;                 /* parallel / cone: device pointer, num_views angles in radians */
    float delta_recon_row;               /* translation only: recon row pitch along the source axis (ALU) */
    const float *translations;           /* translation only: device pointer, num_views x 3 (tx, ty, tz) in ALU */
    float max_magnification;             /* translation only: an upper bound of the pixel magnification over all
                                            pixels and views (0: unknown; the general kernels are used) */
} mbx_geom;

/* qGGMRF prior parameters (b, sigma_x, p, q, T) as TomographyModel.create_vcd_subset_updater builds them
 * (tomography_model.py:1325-1327); b from get_b_from_nbr_wts (qggmrf.py:388-395), order
 * [row+1, row-1, col+1, col-1, slice+1, slice-1]. */
typedef struct mbx_qggmrf_params {
    float b[6];
    float sigma_x;
    float p;
    float q;
    float T;
} mbx_qggmrf_params;

/* Library identification and error reporting. */
MBX_API const char *mbx_version(void);
MBX_API const char *mbx_error_string(int code);
/* The CUDA error code behind the last MBX_ERR_CUDA returned on this host thread. */
MBX_API int mbx_last_cuda_error(void);
/* Reads and clears the device error word of the current device (synchronises the device).
 * Bit 0: a pixel index was out of range; bit 1: a view index was out of range; bit 2: a projector tile
 * exceeded its shared-memory row cache (the geometry check should make this impossible). */
MBX_API int mbx_get_device_error(int *flags_out);
/* Number of kernel launches this library has submitted since it was loaded (host-side count, all devices and
 * streams; launches replayed from a captured CUDA graph are not re-counted). */
MBX_API uint64_t mbx_launch_count(void);
/* Autotuning of the projector plans (no counterpart in the reference, whose XLA compiler picks its own
 * schedule).  The first mbx_sparse_forward_project / mbx_sparse_back_project of a call shape (geometry sizes,
 * views, pixel count rounded up to a power of two) times its candidate plans on the caller's stream,
 * synchronising it, and caches the fastest for the process; a call made while its stream is captured uses the
 * default plan.  Forward candidates: channel-block width, pass size, and the kernel variant compiled for 2 or 3
 * resident CTAs per SM; back-projection candidates: footprints staged in shared memory or computed per thread.
 * mbx_vcd_batched_prepare tunes its two projection stages the same way, cached per batch shape.  Plans differ
 * only in float summation order.  mode: 0 = default plans, 1 = tune (default), k >= 2 = use candidate k-1 (or the
 * last one) everywhere without timing (to check every plan against the default).  Returns the previous mode. */
MBX_API int mbx_set_autotune(int mode);

/* ---- projectors ------------------------------------------------------------------------------- */

/* Workspace the forward projector needs for a call with these sizes (0 when it needs none). */
MBX_API size_t mbx_forward_project_workspace_bytes(const mbx_geom *g, int64_t num_pixels, int32_t num_views_sel);

/* Sparse forward projection: voxel_values (num_pixels, S) at pixel_indices -> sinogram_out
 * (num_views_sel, R, C), every element written.  Output view j uses angle view_indices[j] (or j).
 * Replaces Projectors.sparse_forward_project (projectors.py:61-129) over
 * ParallelBeamModel.forward_project_pixel_batch_to_one_view (parallel_beam.py:138-178) /
 * ConeBeamModel.forward_project_pixel_batch_to_one_view (cone_beam.py:189-377), as called by
 * TomographyModel.sparse_forward_project (tomography_model.py:576-622). */
MBX_API int mbx_sparse_forward_project(const mbx_geom *g, const float *voxel_values, const int32_t *pixel_indices,
                               int64_t num_pixels, const int32_t *view_indices, int32_t num_views_sel,
                               float *sinogram_out, void *workspace, size_t workspace_bytes, void *stream);

/* Workspace the back projector needs for a call with these sizes (0 when it needs none). */
MBX_API size_t mbx_back_project_workspace_bytes(const mbx_geom *g, int64_t num_pixels, int32_t num_views_sel);

/* Sparse back projection of a full sinogram (num_views, R, C) to out (num_pixels, S) (overwritten):
 *   out = scale * sum_views A^coeff_power^T (weights * sinogram)
 * over views view_indices[0..num_views_sel) (or all).  weights may be NULL (all ones); scale is 1 for the
 * reference's sparse_back_project.  coeff_power is 1 (back projection) or 2 (Hessian diagonal).  sinogram may be
 * NULL: the values back-projected are then the weights, or 1 everywhere when weights is NULL too, which gives the
 * Hessian diagonal of unit weights (coeff_power 2) without a sinogram-sized buffer of ones.
 * Replaces Projectors.sparse_back_project (projectors.py:131-209) over
 * ParallelBeamModel.back_project_one_view_to_pixel_batch (parallel_beam.py:180-221) /
 * ConeBeamModel.back_project_one_view_to_pixel_batch (cone_beam.py:379-541), as called by
 * TomographyModel.sparse_back_project (tomography_model.py:624-677) and compute_hessian_diagonal
 * (tomography_model.py:679-708). */
MBX_API int mbx_sparse_back_project(const mbx_geom *g, const float *sinogram, const float *weights,
                            const int32_t *pixel_indices, int64_t num_pixels, const int32_t *view_indices,
                            int32_t num_views_sel, int32_t coeff_power, float scale, float *out,
                            void *workspace, size_t workspace_bytes, void *stream);

/* Size of the static device array behind mbx_sparse_back_project_noalloc (16 MiB). */
#define MBX_NOALLOC_SCRATCH_BYTES (16u << 20)

/* mbx_sparse_back_project without a workspace argument, for callers that cannot allocate GPU memory at call
 * time (for example code running inside JAX, which the mbirjax reference configures to take 98% of the GPU
 * for its own allocator, or pipelines that reserve all device memory up front).  This entry point has no
 * counterpart in the reference.  It calls no cudaMalloc, cudaFree or other allocating routine.  The scratch
 * for the split view sums lives in a static device array of MBX_NOALLOC_SCRATCH_BYTES: every GPU on which the
 * entry point is used holds that array until the process exits.  Its address is looked up on the first call on
 * each device, so make that first call before any stream capture.  All calls on a device share the array, so
 * calls whose GPU work overlaps race and must be serialised by the caller.  A call whose sizes would need more
 * scratch than the array holds returns MBX_ERR_WORKSPACE before any launch. */
MBX_API int mbx_sparse_back_project_noalloc(const mbx_geom *g, const float *sinogram, const float *weights,
                                            const int32_t *pixel_indices, int64_t num_pixels,
                                            const int32_t *view_indices, int32_t num_views_sel, int32_t coeff_power,
                                            float scale, float *out, void *stream);

/* ---- qGGMRF prior ----------------------------------------------------------------------------- */

/* Surrogate gradient and Hessian diagonal at pixel_indices (num_pixels, S) each.
 * Replaces qggmrf_gradient_and_hessian_at_indices (qggmrf.py:118-279). */
MBX_API int mbx_qggmrf_grad_hess(const float *flat_recon, int32_t num_recon_rows, int32_t num_recon_cols,
                         int32_t num_recon_slices, const int32_t *pixel_indices, int64_t num_pixels,
                         const mbx_qggmrf_params *qp, float *grad_out, float *hess_out, void *stream);

/* Workspace for mbx_qggmrf_loss_grad. */
MBX_API size_t mbx_qggmrf_loss_grad_workspace_bytes(int32_t num_recon_rows, int32_t num_recon_cols,
                                            int32_t num_recon_slices);

/* qGGMRF loss (written to *loss_out, a device double) and its gradient grad_out (full recon shape,
 * overwritten; may be NULL).  Replaces qggmrf_loss (qggmrf.py:31-65) and its autodiff gradient. */
MBX_API int mbx_qggmrf_loss_grad(const float *recon, int32_t num_recon_rows, int32_t num_recon_cols,
                         int32_t num_recon_slices, const mbx_qggmrf_params *qp, double *loss_out,
                         float *grad_out, void *workspace, size_t workspace_bytes, void *stream);

/* ---- VCD subset update ------------------------------------------------------------------------ */

/* Workspace for one mbx_vcd_subset_step with these sizes. */
MBX_API size_t mbx_vcd_subset_step_workspace_bytes(const mbx_geom *g, int64_t num_pixels);

/* One VCD subset update, fully on the device (no host synchronisation):
 *   delta = -(g_fwd + g_prior) / (h_fwd + h_prior),  g_fwd = -fm * A^T (w e),  h_fwd = fm * H[idx]
 *   alpha = clip((fm <w e, A delta> - <g_prior, delta>) / (fm <w A delta, A delta> + <h_prior, delta^2>/2
 *           + eps), eps, 1.5)
 *   flat_recon[idx] += alpha delta;  error_sinogram -= alpha A delta
 * weights may be NULL (constant weights 1).  The inner products accumulate in float64.  stats_out (a device
 * double[4]) receives {alpha, sum|alpha delta|, forward_linear - prior_linear, denominator}.
 * Replaces the vcd_subset_updater closure of TomographyModel.create_vcd_subset_updater
 * (tomography_model.py:1310-1544) with get_forward_lin_quad (tomography_model.py:1546-1631) and
 * update_recon (tomography_model.py:1820-1823). */
MBX_API int mbx_vcd_subset_step(const mbx_geom *g, float *flat_recon, float *error_sinogram, const float *weights,
                        const float *fm_hessian, const int32_t *pixel_indices, int64_t num_pixels,
                        float fm_constant, const mbx_qggmrf_params *qp, double *stats_out, void *workspace,
                        size_t workspace_bytes, void *stream);

/* mbx_vcd_subset_step with the two options of the reference's subset updater:
 *   prox_input (flat like flat_recon, or NULL): proximal-map prior instead of qGGMRF, g_prior = (x - v) /
 *     sigma_prox^2 and h_prior = sigma_prox^2 as the reference writes it (tomography_model.py:1388-1391,
 *     prox_gradient_at_indices qggmrf.py:8-28); qp is then unused;
 *   positivity != 0: after alpha is found, delta = max(-x / (alpha + eps), delta) at the subset and the clipped
 *     delta is forward-projected again before the updates (tomography_model.py:1497-1507).
 * Workspace as mbx_vcd_subset_step_workspace_bytes. */
MBX_API int mbx_vcd_subset_step_ex(const mbx_geom *g, float *flat_recon, float *error_sinogram, const float *weights,
                           const float *fm_hessian, const int32_t *pixel_indices, int64_t num_pixels,
                           float fm_constant, const mbx_qggmrf_params *qp, const float *prox_input,
                           float sigma_prox, int32_t positivity, double *stats_out, void *workspace,
                           size_t workspace_bytes, void *stream);

/* ---- qGGMRF denoiser ---------------------------------------------------------------------------- */

/* Workspace for one mbx_qggmrf_denoise_step over num_pixels cylinders of num_slices voxels. */
MBX_API size_t mbx_qggmrf_denoise_step_workspace_bytes(int64_t num_pixels, int32_t num_slices);
/* One subset update of the qGGMRF denoiser (identity forward model), fully on the device:
 *   delta = -(-fm e + g_prior) / (1 + h_prior) with e = flat_error_image[idx] (noisy - current image)
 *   alpha = clip((fm <e, delta> - <g_prior, delta>) / (fm <delta, delta> + <h_prior, delta^2>/1.1 + eps), eps, 1.5)
 *   flat_image[idx] += alpha delta;  flat_error_image[idx] -= alpha delta
 * Images are flat (num_rows * num_cols, num_slices); inner products in float64; stats_out (device double[4], may
 * be NULL) receives {alpha, sum|alpha delta|, numerator, denominator}.  Replaces vcd_subset_denoiser
 * (denoising.py:366-411). */
MBX_API int mbx_qggmrf_denoise_step(float *flat_image, float *flat_error_image, int32_t num_rows, int32_t num_cols,
                            int32_t num_slices, const int32_t *pixel_indices, int64_t num_pixels,
                            float fm_constant, const mbx_qggmrf_params *qp, double *stats_out, void *workspace,
                            size_t workspace_bytes, void *stream);
/* 3x3x3 median filter with edge replication of a (d0, d1, d2) float32 volume into out (not in place).
 * Replaces median_filter3d (denoising.py:414-490). */
MBX_API int mbx_median_filter3d(const float *x, int32_t d0, int32_t d1, int32_t d2, float *out, void *stream);

/* ---- batched VCD over many scans ------------------------------------------------------------- */

/* One scan of a batch: its geometry, device buffers and VCD parameters (the state the reference keeps per
 * TomographyModel in vcd_recon, tomography_model.py:1086-1255). */
typedef struct mbx_scan {
    mbx_geom geom;
    float *flat_recon;              /* (Nr*Nc, S), updated in place */
    float *error_sinogram;          /* (V, R, C), updated in place; 16-byte aligned */
    const float *weights;           /* (V, R, C) or NULL for constant weights 1 */
    const float *fm_hessian;        /* (Nr*Nc, S): back projection of the weights with squared coefficients */
    const int32_t *partition;       /* (num_subsets, subset_size) pixel indices, as gen_pixel_partition */
    const int32_t *partition_order; /* optional (num_subsets, subset_size): a permutation of each subset's
                                       positions giving the order the back projector visits them (locality) */
    int32_t num_subsets;
    int32_t subset_size;
    float fm_constant;              /* 1 / sigma_y^2 */
    mbx_qggmrf_params qp;
    /* Inputs of the batched set-up (mbx_vcd_batched_setup); NULL / 0 when the caller sets the state up itself. */
    const float *sinogram;          /* (V, R, C) measured sinogram y */
    const int32_t *full_indices;    /* the region-of-reconstruction pixels, gen_full_indices (vcd_utils.py:310-318) */
    int32_t num_full_indices;
} mbx_scan;

/* Opaque host-side record of a prepared batch (filled by mbx_vcd_batched_prepare). */
typedef struct mbx_batched_plan {
    uint64_t opaque[128];
} mbx_batched_plan;

/* Workspace for a batch with num_steps subset steps in its schedule (0 if the batch is not supported). */
MBX_API size_t mbx_vcd_batched_workspace_bytes(const mbx_scan *scans, int32_t num_scans, int32_t num_steps);

/* Option of mbx_vcd_batched_prepare2: plan the subset forward projections.  Each subset is projected once per
 * iteration, always onto the same (view, channel block) tiles; with this option mbx_vcd_batched_refresh scans and
 * sorts every tile's pixels once per reconstruction and stores the sorted record passes in the workspace (about
 * 17 bytes per pixel and view, 33 for cone and translation geometry), and every forward-projection stage replays
 * them instead of scanning and sorting again.  Same results as without it. */
#define MBX_BATCHED_PLAN_FORWARD 1

/* mbx_vcd_batched_workspace_bytes / mbx_vcd_batched_prepare with options (MBX_BATCHED_PLAN_FORWARD). */
MBX_API size_t mbx_vcd_batched_workspace_bytes2(const mbx_scan *scans, int32_t num_scans, int32_t num_steps,
                                                int32_t flags);

/* Validates the batch, lays out the workspace and uploads the per-scan argument records, the tile work lists
 * and the subset schedule (schedule[step * num_scans + scan] = subset index that scan updates at that step;
 * the reference draws it with np.random.permutation per iteration, tomography_model.py:1281).  step_stats
 * (device, num_steps * num_scans * 4 doubles) receives per step and scan {alpha, l1 of the update, alpha
 * numerator, alpha denominator}; iter_stats (device, num_iterations * num_scans * 4) receives
 * {sum W e^2, sum |recon|, 0, 0} from mbx_vcd_batched_iteration_stats.  All scans must share one geometry kind
 * and one num_subsets and have psf_radius (and for cone beam bp_psf_radius) 1; otherwise MBX_ERR_UNSUPPORTED.  Synchronises the
 * stream (call it before any stream capture).  Replaces running the reference's vcd_recon once per scan. */
MBX_API int mbx_vcd_batched_prepare(const mbx_scan *scans, int32_t num_scans, const int32_t *schedule,
                                    int32_t num_steps, int32_t num_iterations, double *step_stats,
                                    double *iter_stats, void *workspace, size_t workspace_bytes,
                                    mbx_batched_plan *plan_out, void *stream);
MBX_API int mbx_vcd_batched_prepare2(const mbx_scan *scans, int32_t num_scans, const int32_t *schedule,
                                     int32_t num_steps, int32_t num_iterations, double *step_stats,
                                     double *iter_stats, void *workspace, size_t workspace_bytes, int32_t flags,
                                     mbx_batched_plan *plan_out, void *stream);

/* One subset update for every scan of the batch: eight persistent launches, each walking the packed work list
 * of all scans (no host synchronisation; capturable in a CUDA graph).  Replaces one vcd_subset_updater call
 * (tomography_model.py:1343-1542) per scan. */
MBX_API int mbx_vcd_batched_step(const mbx_batched_plan *plan, int32_t step, void *stream);

/* Number of stages of one batched subset step, and one stage on its own (the step is stages 0..7 in order:
 * back projection, delta, forward projection, line-search partials, alpha, recon update, error update, l1).
 * Running the stages of a step one by one in order is the same as mbx_vcd_batched_step; it lets a caller
 * time each stage with events. */
#define MBX_BATCHED_STAGES 8
MBX_API int mbx_vcd_batched_stage(const mbx_batched_plan *plan, int32_t step, int32_t stage, void *stream);

/* Per-scan iteration statistics into iter_stats[iteration] (inputs of the reference's fm_rmse and NMAE,
 * tomography_model.py:1219-1220). */
MBX_API int mbx_vcd_batched_iteration_stats(const mbx_batched_plan *plan, int32_t iteration, void *stream);

/* The VCD set-up of every scan of the batch, as batched stages (no host synchronisation; capturable): direct
 * recon initialisation (FBP / FDK filter of the scan's sinogram into its error sinogram, back projection over its
 * full_indices into its flat recon, zero elsewhere), forward projection of that recon, the alpha rescale that
 * minimises ||y - alpha A x||_W (float64 sums), error sinogram y - alpha A x and recon alpha x, and the Hessian
 * diagonal (back projection of the weights, or of ones, with squared coefficients over every pixel).  Replaces
 * the set-up of vcd_recon (tomography_model.py:1110-1152) with direct_recon (:934-964) and
 * compute_hessian_diagonal (:679-708), run once per scan in the reference.  Needs every scan's sinogram and
 * full_indices at prepare time (else MBX_ERR_UNSUPPORTED). */
MBX_API int mbx_vcd_batched_setup(const mbx_batched_plan *plan, void *stream);

/* New per-call parameters of a prepared batch: each scan's fm_constant and qp, and the subset schedule
 * (num_steps * num_scans entries, as at prepare).  scans must describe the same batch as at prepare (same count,
 * sizes and buffers); only fm_constant and qp are read from it.  Enqueues host-to-device copies on the stream
 * (from pageable host memory: not capturable; call it between graph replays).  With mbx_vcd_batched_refresh this
 * lets one prepared plan, and graphs captured from it, reconstruct new data of the same batch shape: the
 * reference recomputes regularisation, partitions and subset orders on every recon call
 * (tomography_model.py:1024-1035, 1281). */
MBX_API int mbx_vcd_batched_update(const mbx_batched_plan *plan, const mbx_scan *scans, int32_t num_scans,
                                   const int32_t *schedule, void *stream);

/* Recomputes the chunk bounding boxes of every scan's subsets from the partition buffers, after the caller has
 * written new partitions into them, and for a batch prepared with MBX_BATCHED_PLAN_FORWARD builds the planned
 * forward projections of those subsets (no host synchronisation; capturable). */
MBX_API int mbx_vcd_batched_refresh(const mbx_batched_plan *plan, void *stream);

/* ---- FBP / FDK filtering ---------------------------------------------------------------------- */

/* Direct-recon filtering of a sinogram (num_views, R, C) into out (same shape).
 * Parallel beam: ramp filter x 1/delta_voxel^2, 'valid' convolution per row, x pi/num_views
 * (replaces ParallelBeamModel.fbp_filter, parallel_beam.py:303-348).
 * Cone beam: pre-weight D/sqrt(D^2+u^2+v^2), filter x delta_det_row/(delta_voxel^3 magnification),
 * convolution, x pi/num_views (replaces ConeBeamModel.fdk_filter, cone_beam.py:779-846).
 * The filter is generate_direct_recon_filter 'ramp' (tomography_utils.py:4-35). */
MBX_API int mbx_direct_filter(const mbx_geom *g, const float *sinogram, float *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MBIRJAX_B200_H */
