/*
 * u3dg.h - C ABI of the B200 (sm_100a) 3D Gaussian Splatting trainer.
 *
 * This is the drop-in boundary for the CPU splat core of
 * Abner0907/univeral_3d_reconstruction_system (engine/src/splat). Every entry point
 * names the reference interface it replaces (file:line inside that project).
 *
 * Conventions
 *  - Every function returns an int status (U3DG_OK = 0). On failure the thread-local
 *    message of u3dg_last_error() says what went wrong. Nothing here throws or aborts.
 *  - Arrays passed to entry points without a "_dev" suffix are HOST memory; the library
 *    copies them to and from the GPU. The trainer keeps its state on the GPU between calls.
 *  - Gaussian parameters use the reference's GaussianModel layout
 *    (engine/include/u3d/splat/GaussianModel.h:23-37): five separate float arrays
 *    means[3n], scales[3n] (log sigma), quats[4n] (w,x,y,z, not normalised),
 *    opacities[n] (logit), colors[3n] (SH degree-0 coefficient).
 *  - Images are height*width*3 interleaved RGB (row-major), float in 0..1 for renders and
 *    uint8 for training targets, as in the reference (Trainer.h:13-18, Rasterizer.h:43-45).
 *  - One trainer or rasterizer object must not be used from two threads at once; separate
 *    objects are independent and may run concurrently.
 */
#ifndef U3DG_H
#define U3DG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define U3DG_ABI_VERSION 1

/* Status codes. */
#define U3DG_OK 0
#define U3DG_ERR_INVALID_ARG 1
#define U3DG_ERR_OOM 2
#define U3DG_ERR_CUDA 3
#define U3DG_ERR_TIMEOUT 4
#define U3DG_ERR_CAPACITY 5
#define U3DG_ERR_IO 6
#define U3DG_ERR_NO_DEVICE 7
#define U3DG_ERR_STATE 8

/* Pinhole camera, world-to-camera pose in the OpenCV convention (x right, y down, z forward),
 * p_cam = R p_world + t, R row-major. Same fields as RenderCamera
 * (engine/include/u3d/splat/Rasterizer.h:13-21). */
typedef struct u3dg_camera {
    int width;
    int height;
    float fx, fy, cx, cy;
    float R[9];
    float t[3];
} u3dg_camera;

/* RasterSettings (engine/include/u3d/splat/Rasterizer.h:23-32). */
typedef struct u3dg_raster_settings {
    int tile_size;           /* 16 by default; 8, 16, 32 and 64 are supported */
    float near_plane;        /* 0.01 */
    float eps2d;             /* 0.3, low-pass filter added to the 2D covariance */
    float background[3];     /* 0, 0, 0 */
    float min_alpha;         /* 1/255; contributions below are skipped */
    float min_transmittance; /* 1e-4; compositing stops below */
} u3dg_raster_settings;

/* LearningRates (engine/include/u3d/splat/Adam.h:8-14). means is relative to the scene extent. */
typedef struct u3dg_learning_rates {
    float means, scales, quats, opacities, colors;
} u3dg_learning_rates;

/* TrainOptions (engine/include/u3d/splat/Trainer.h:20-38). */
typedef struct u3dg_train_options {
    int iterations;
    int max_gaussians;
    float ssim_lambda;
    u3dg_learning_rates lr;
    float means_lr_final;
    float densify_grad_threshold;
    float percent_dense;
    int refine_start;
    int refine_stop;
    int refine_interval;
    int opacity_reset_interval; /* 0 = never */
    float prune_opacity;
    unsigned int seed;
    u3dg_raster_settings raster;
} u3dg_train_options;

/* TrainStats (engine/include/u3d/splat/Trainer.h:40-45). loss and psnr are exponential
 * moving averages over the training iterations. */
typedef struct u3dg_train_stats {
    int iteration;
    float loss;
    float psnr;
    uint64_t gaussians;
} u3dg_train_stats;

/* LossValue (engine/include/u3d/splat/Loss.h:9-13). */
typedef struct u3dg_loss_value {
    float total;
    float l1;
    float ssim;
} u3dg_loss_value;

/* Views of a GaussianModel (engine/include/u3d/splat/GaussianModel.h:23-37). For inputs the
 * pointers are read; for outputs they must hold `count` entries of each array. */
typedef struct u3dg_model {
    float *means;
    float *scales;
    float *quats;
    float *opacities;
    float *colors;
    size_t count;
} u3dg_model;

/* TrainImage (engine/include/u3d/splat/Trainer.h:13-18): camera + uint8 RGB target. */
typedef struct u3dg_image {
    u3dg_camera camera;
    const uint8_t *rgb; /* height * width * 3 */
} u3dg_image;

/* Per-phase device time of the trainer's steps, filled when profiling is on. */
typedef struct u3dg_phase_times {
    int steps;           /* steps accumulated */
    float project_ms;    /* projection kernel */
    float sort_ms;       /* depth sort + tile binning (scan, emit, tile sort, ranges) */
    float forward_ms;    /* tile compositing forward */
    float loss_ms;       /* L1 + D-SSIM forward and backward */
    float backward_ms;   /* tile compositing backward */
    float update_ms;     /* per-Gaussian chain rule fused with Adam */
    float densify_ms;    /* densify / prune / opacity reset (on the steps that run them) */
    float total_ms;      /* whole steps, first to last event */
    uint64_t intersections; /* sum over the profiled steps of tile-Gaussian intersections */
    uint64_t visible;       /* sum over the profiled steps of visible Gaussians */
    uint64_t gaussians;     /* sum over the profiled steps of the Gaussian count */
    uint64_t pixels;        /* sum over the profiled steps of rendered pixels */
} u3dg_phase_times;

typedef struct u3dg_trainer u3dg_trainer;
typedef struct u3dg_rasterizer u3dg_rasterizer;
typedef struct u3dg_adam u3dg_adam;

/* ------------------------------------------------------------------ library */

/* Message of the last failing call on this thread ("" if none). */
const char *u3dg_last_error(void);
/* U3DG_ABI_VERSION of the loaded library. */
int u3dg_abi_version(void);
/* Number of CUDA kernels this library has launched in this process (all devices, all objects). */
uint64_t u3dg_launch_count(void);
/* Number of CUDA devices visible (0 without a GPU; never fails). */
int u3dg_device_count(void);
/* Selects the CUDA device used by objects created afterwards on this thread. */
int u3dg_set_device(int device);

/* Defaults of RasterSettings (Rasterizer.h:23-32) and TrainOptions (Trainer.h:20-38). */
void u3dg_raster_settings_default(u3dg_raster_settings *out);
void u3dg_train_options_default(u3dg_train_options *out);
/* TrainOptions::forIterations (engine/src/splat/Trainer.cpp:26-35). */
void u3dg_train_options_for_iterations(int iterations, u3dg_train_options *out);

/* ------------------------------------------------------------------ trainer */

/* Trainer::Trainer (engine/include/u3d/splat/Trainer.h:50-51, engine/src/splat/Trainer.cpp:37-51).
 * Copies the initial model and all images to the GPU; the host buffers may be freed afterwards.
 * Device buffers are sized once for options->max_gaussians (at least initial->count). */
int u3dg_trainer_create(const u3dg_model *initial, const u3dg_image *images, int image_count,
                        float scene_extent, const u3dg_train_options *options, u3dg_trainer **out);
/* Trainer::Trainer as u3dg_trainer_create, except that the images are copied to the GPU by a host
 * thread while the first steps already run: views are sent in the order the first epoch uses them
 * and each step waits (on the GPU) only for its own view, so a short run does not wait for every
 * image first. Results are identical to u3dg_trainer_create's. The caller's pixel buffers
 * (images[k].rgb) must stay valid and unchanged until u3dg_trainer_wait_uploads returns or the
 * trainer is destroyed; the image array itself and the model may be freed on return. (The
 * reference's Trainer owns its images, which it takes by value: a caller that keeps them alive
 * beside the trainer, as the C++ drop-in does, loses nothing.) */
int u3dg_trainer_create_background_upload(const u3dg_model *initial, const u3dg_image *images, int image_count,
                                          float scene_extent, const u3dg_train_options *options,
                                          u3dg_trainer **out);
/* Blocks until every image of a trainer created with background upload is on the GPU; afterwards
 * the caller may release its pixel buffers. Returns at once for other trainers. */
int u3dg_trainer_wait_uploads(u3dg_trainer *trainer);
/* Trainer::step (Trainer.cpp:53-103), `count` times. Returns without work once done, like the
 * reference. The work is queued on the trainer's CUDA stream; only densification steps wait
 * for the GPU (they read back the split count to draw the split samples on the host). */
int u3dg_trainer_step(u3dg_trainer *trainer, int count);
/* Trainer::done / Trainer::iteration (Trainer.h:53-54). */
int u3dg_trainer_done(const u3dg_trainer *trainer, int *done);
int u3dg_trainer_iteration(const u3dg_trainer *trainer, int *iteration);
/* Trainer::stats (Trainer.h:56). Waits for the queued steps. */
int u3dg_trainer_stats(u3dg_trainer *trainer, u3dg_train_stats *out);
/* Current Gaussian count (GaussianModel::size). Waits for the queued steps. */
int u3dg_trainer_size(u3dg_trainer *trainer, size_t *count);
/* Trainer::model (Trainer.h:55): copies the current model into host arrays of capacity `capacity`
 * Gaussians (U3DG_ERR_CAPACITY if too small; *count is set either way). */
int u3dg_trainer_download(u3dg_trainer *trainer, u3dg_model *out, size_t capacity, size_t *count);
/* writeSplatPly(path, trainer.model()) (Reconstructor.cpp:350-355, SplatPly.cpp:261-282) in one call:
 * the trainer's current model is copied from the GPU into a temporary host copy and written; the same
 * bytes as u3dg_trainer_download followed by u3dg_write_splat_ply. */
int u3dg_trainer_write_splat_ply(u3dg_trainer *trainer, const char *path);
/* Trainer::evaluatePsnr (Trainer.cpp:180-192): mean PSNR over all training views. */
int u3dg_trainer_eval_psnr(u3dg_trainer *trainer, float *psnr);
/* Trainer::render (Trainer.cpp:194-197): rgb gets height*width*3 floats. */
int u3dg_trainer_render(u3dg_trainer *trainer, const u3dg_camera *camera, float *rgb);
/* CUDA stream (cudaStream_t) the trainer queues its work on. */
int u3dg_trainer_stream(u3dg_trainer *trainer, void **stream);
/* Blocks until every queued step has finished on the GPU. */
int u3dg_trainer_synchronize(u3dg_trainer *trainer);
/* Per-phase CUDA-event timing of the following steps (enable != 0), read back with
 * u3dg_trainer_phase_times (which waits and then resets the accumulators). Timing adds one event
 * pair per phase and waits for each step; leave it off for throughput runs. */
int u3dg_trainer_set_profiling(u3dg_trainer *trainer, int enable);
int u3dg_trainer_phase_times(u3dg_trainer *trainer, u3dg_phase_times *out);
/* Tile-Gaussian intersection buffers. Steps never wait for the GPU to learn their intersection count:
 * a step that overflows the buffers does no update, and the trainer grows the buffers and replays it
 * (bit-identical to a run that never overflowed). set_intersection_capacity sizes the buffers (they
 * still grow on demand); replays reports how many steps were replayed so far. */
int u3dg_trainer_set_intersection_capacity(u3dg_trainer *trainer, size_t capacity);
int u3dg_trainer_replays(u3dg_trainer *trainer, int *replays);
/* Device time in milliseconds of `count` steps, measured with CUDA events recorded on the
 * trainer's stream right before the first and after the last step (host waits on both sides). */
int u3dg_trainer_time_steps(u3dg_trainer *trainer, int count, float *ms);
/* No reference counterpart. Runs of 10 steps with no densification, opacity reset or profiling
 * among them, when every view has the same size, are launched as one CUDA graph whose kernels read
 * each step's view and learning rates from device memory (on by default; results are identical to
 * step-by-step launches). set_graphs turns this on (1) or off (0); graph_launches reports how many
 * graph launches ran so far. */
int u3dg_trainer_set_graphs(u3dg_trainer *trainer, int enable);
int u3dg_trainer_graph_launches(u3dg_trainer *trainer, long long *launches);
/* No reference counterpart. Compositing schedule: forward_block is the pixel block edge of the
 * forward kernel for tiles of 16 and 32 pixels, 8 (default: several 8x8 CTAs walk each tile list) or
 * 16; forward_depth and backward_depth are the list entries each thread of the forward and of the
 * backward kernel stages per shared-memory batch, 1 (default) or 2 (deeper batches halve the block
 * barriers per Gaussian at the cost of shared memory). The rendered images, gradients and trained
 * models are bit-identical for every setting. */
int u3dg_trainer_set_raster_schedule(u3dg_trainer *trainer, int forward_block, int forward_depth,
                                     int backward_depth);
/* No reference counterpart. Tile culling (on by default): a Gaussian is listed only in the tiles of
 * its rectangle that its contributing ellipse (alpha >= min_alpha) can reach, with a conservative
 * margin; the trained models are bit-identical with it on (1) or off (0). */
int u3dg_trainer_set_tile_culling(u3dg_trainer *trainer, int enable);
void u3dg_trainer_destroy(u3dg_trainer *trainer);

/* ------------------------------------------------------------------ rasterizer (unit boundary) */

/* Rasterizer::Rasterizer (engine/include/u3d/splat/Rasterizer.h:41). */
int u3dg_rasterizer_create(u3dg_rasterizer **out);
/* Rasterizer::forward (Rasterizer.h:43-45, engine/src/splat/Rasterizer.cpp:263-330): projection,
 * tile binning and front-to-back compositing; rgb gets height*width*3 floats. The per-Gaussian and
 * per-pixel state stays on the GPU for u3dg_rasterizer_backward. */
int u3dg_rasterizer_forward(u3dg_rasterizer *r, const u3dg_model *model, const u3dg_camera *camera,
                            const u3dg_raster_settings *settings, float *rgb);
/* Rasterizer::backward (Rasterizer.h:47-51, Rasterizer.cpp:334-545): ADDS dL/dparams to `grads`
 * (host arrays of the model's size); if mean2d_grad_ndc is not NULL (n floats) ADDS the
 * |dL/dmean2d| NDC statistic to it. */
int u3dg_rasterizer_backward(u3dg_rasterizer *r, const u3dg_model *model, const float *dl_drgb,
                             u3dg_model *grads, float *mean2d_grad_ndc);
/* Rasterizer::radii (Rasterizer.h:53-54): n ints, 0 = not visible. */
int u3dg_rasterizer_radii(u3dg_rasterizer *r, int *radii, size_t n);
/* Projected state of the last forward (Rasterizer.h:65-74, Rasterizer.cpp:179-201); any pointer
 * may be NULL. mean2d 2n, conic 3n, cov2d 3n, depth n, rgb 3n, alpha n, rect 4n, flags n. */
int u3dg_rasterizer_projection(u3dg_rasterizer *r, size_t n, float *mean2d, float *conic, float *cov2d,
                               float *depth, float *rgb, float *alpha, int *rect, uint8_t *flags);
/* Tile lists of the last forward (m_tileOffsets / m_tileList, Rasterizer.h:76-80): offsets gets
 * tiles+1 ints; list gets up to list_capacity ints; *list_length the full length. */
int u3dg_rasterizer_tiles(u3dg_rasterizer *r, int *tiles_x, int *tiles_y, int *offsets, size_t offsets_capacity,
                          int *list, size_t list_capacity, size_t *list_length);
/* Per-pixel state of the last forward (m_finalT, m_nContrib, Rasterizer.h:82-84). */
int u3dg_rasterizer_pixel_state(u3dg_rasterizer *r, float *final_t, int *n_contrib, size_t pixels);
/* No reference counterpart (the trainers' tile culling at the unit boundary): with enable = 1 the
 * following forwards list each Gaussian only in the tiles of its rectangle that its contributing
 * ellipse (alpha >= min_alpha) can reach, as the trainers do by default; every tile list is then an
 * order-preserving subsequence of Rasterizer::binTiles' list (Rasterizer.cpp:206-261) and images,
 * pixel state and gradients are unchanged. 0 (the default) keeps the reference's lists. */
int u3dg_rasterizer_set_tile_culling(u3dg_rasterizer *r, int enable);
void u3dg_rasterizer_destroy(u3dg_rasterizer *r);

/* Tile binning of Rasterizer::binTiles (Rasterizer.cpp:206-261) on the GPU, from given projected
 * records (depth n, radius n, rect 4n): the depth radix sort and the tile bucketing. Used to check
 * the sort order bit for bit on identical inputs. offsets gets tiles_x*tiles_y+1 ints. */
int u3dg_bin_tiles(const float *depth, const int *radius, const int *rect, size_t n, int tiles_x, int tiles_y,
                   int *offsets, int *list, size_t list_capacity, size_t *list_length);

/* Trainer::densifyAndPrune (engine/src/splat/Trainer.cpp:105-169) on a given state, through the same
 * GPU code path the trainer uses. model, adam_m and adam_v are host arrays with room for `capacity`
 * Gaussians of which model->count are valid; they are densified in place and *count gets the new
 * size (U3DG_ERR_CAPACITY if it exceeds capacity). grad_accum / grad_count (model->count entries) are
 * the densification statistics. Split samples come from std::mt19937(seed) through
 * std::normal_distribution<float>, drawn in the reference's order. counts3 (may be NULL) gets the
 * numbers of pruned, cloned and split Gaussians. */
int u3dg_densify_and_prune(u3dg_model *model, u3dg_model *adam_m, u3dg_model *adam_v, const float *grad_accum,
                           const int *grad_count, size_t capacity, float scene_extent,
                           const u3dg_train_options *options, int opacity_was_reset, unsigned int seed, size_t *count,
                           int *counts3);

/* ------------------------------------------------------------------ batched training */

/* No reference counterpart (the reference trains one scene per Trainer). Trains `scenes` scenes at
 * once on the current device: scene s starts from initial[s] with images[s][0 .. image_counts[s])
 * and options[s] (each with its own schedule and Gaussian cap). Every scene keeps its own trainer and
 * stream; u3dg_batch_step advances each scene by `count` iterations (or to its end), interleaving the
 * scenes so their kernels run concurrently and running steps through each scene's step graph where
 * it can. With autotune != 0, each scene's tile size (8, 16 or 32) and compositing schedule (the
 * settings of u3dg_trainer_set_raster_schedule; same results for any) are chosen at creation from
 * short timed runs on throwaway trainers; tile_size reports the tile and the tuned ms per step (0
 * without autotune), schedule the compositing settings as well. batch_trainer
 * returns a borrowed handle for the per-scene queries of the u3dg_trainer_* API (download, stats,
 * eval_psnr, ...); destroying it is a no-op, the batch owns it. time_steps steps like batch_step and
 * reports the device time from one event that all scene streams wait on to the last stream's end. */
typedef struct u3dg_batch u3dg_batch;
int u3dg_batch_create(const u3dg_model *initial, const u3dg_image *const *images, const int *image_counts,
                      const float *extents, const u3dg_train_options *options, int scenes, int autotune,
                      u3dg_batch **out);
int u3dg_batch_step(u3dg_batch *batch, int count);
int u3dg_batch_time_steps(u3dg_batch *batch, int count, float *ms);
int u3dg_batch_size(u3dg_batch *batch, int *scenes);
int u3dg_batch_trainer(u3dg_batch *batch, int scene, u3dg_trainer **out);
int u3dg_batch_tile_size(u3dg_batch *batch, int scene, int *tile, float *tuned_ms_per_step);
int u3dg_batch_schedule(u3dg_batch *batch, int scene, int *tile, int *forward_block, int *forward_depth,
                        int *backward_depth, float *tuned_ms_per_step);
/* Rounds in which every unfinished scene ran its next 10 steps as one CUDA graph launch holding all
 * scenes (scenes whose buffers stayed put since the previous round), and how often that graph was
 * recorded. Either pointer may be NULL. */
int u3dg_batch_graph_launches(u3dg_batch *batch, long long *launches, long long *captures);
void u3dg_batch_destroy(u3dg_batch *batch);

/* ------------------------------------------------------------------ loss */

/* photometricLoss (engine/include/u3d/splat/Loss.h:18-19, engine/src/splat/Loss.cpp:47-184):
 * (1-lambda) L1 + lambda (1 - SSIM), 11x11 Gaussian window (sigma 1.5, zero padding). render and
 * target are height*width*3 floats; grad (same size) receives dLoss/drender. */
int u3dg_photometric_loss(const float *render, const float *target, int width, int height, float lambda,
                          float *grad, u3dg_loss_value *out);
/* psnr (Loss.h:21, Loss.cpp:187-196): double accumulation, 99 dB when MSE <= 1e-12. */
int u3dg_psnr(const float *a, const float *b, size_t count, float *out);
/* No reference counterpart: u3dg_photometric_loss on DEVICE pointers (render, target, grad are
 * height*width*3 floats in device memory of the current device) that allocates nothing. Temporaries
 * live in a fixed 11.2 MB device array per device, so width*height must be <= 640*480 and the image
 * at most 2048 loss blocks of 32x16 pixels; larger images return U3DG_ERR_CAPACITY. Work runs on
 * `stream` (a cudaStream_t; NULL = the default stream), and the call synchronises it before
 * returning (it returns the loss values on the host). The first call in each device context (the
 * first on a device, and the first after a cudaDeviceReset there) resolves the array's address in
 * that context; make it before any stream capture begins on that device. Calls on one device share
 * the array and are serialised by a per-device lock. out may be NULL. Same results as
 * u3dg_photometric_loss. */
int u3dg_photometric_loss_noalloc(const float *render, const float *target, int width, int height, float lambda,
                                  float *grad, u3dg_loss_value *out, void *stream);

/* ------------------------------------------------------------------ Adam */

/* Adam (engine/include/u3d/splat/Adam.h:18-31, engine/src/splat/Adam.cpp). Moments live on the
 * GPU; params are host arrays updated in place. */
int u3dg_adam_create(size_t count, u3dg_adam **out);
/* Adam::step (Adam.cpp:68-78). */
int u3dg_adam_step(u3dg_adam *adam, u3dg_model *params, const u3dg_model *grads, const u3dg_learning_rates *lr);
/* Adam::compact (Adam.cpp:40-44): keep has count bytes. */
int u3dg_adam_compact(u3dg_adam *adam, const uint8_t *keep, size_t count);
/* Adam::grow (Adam.cpp:46-60). */
int u3dg_adam_grow(u3dg_adam *adam, size_t count);
/* Adam::resetOpacityMoments (Adam.cpp:62-66). */
int u3dg_adam_reset_opacity_moments(u3dg_adam *adam);
/* Copies the first and second moments out (either may be NULL). */
int u3dg_adam_moments(u3dg_adam *adam, u3dg_model *m, u3dg_model *v);
void u3dg_adam_destroy(u3dg_adam *adam);

/* ------------------------------------------------------------------ crop (engine/include/u3d/splat/Crop.h) */

/* CropBox (Crop.h:9-19): an axis-aligned box in model coordinates. */
typedef struct u3dg_crop_box {
    float min[3], max[3];
} u3dg_crop_box;
/* cropModel (Crop.h:21-23, engine/src/splat/Crop.cpp:44-52) on the GPU: keeps the Gaussians whose
 * centre lies inside box (bounds included) and whose sigmoid(opacity) is at least min_opacity, in
 * order. Call with out == NULL to get *count first; capacity is out's size. */
int u3dg_crop_model(const u3dg_model *model, const u3dg_crop_box *box, float min_opacity, u3dg_model *out,
                    size_t capacity, size_t *count);
/* suggestCropBox (Crop.h:25-31, Crop.cpp:54-57) on the GPU: per axis, the low / high quantiles of the
 * centres of Gaussians at least 0.3 opaque (all centres when none is), widened by margin of the
 * box size (at least 1e-4) on each side. */
int u3dg_suggest_crop_box(const u3dg_model *model, float low_fraction, float high_fraction, float margin,
                          u3dg_crop_box *out);
/* modelBounds (Crop.h:33-35, Crop.cpp:59-62): the 0.5 % / 99.5 % quantiles of all centres plus 10 %. */
int u3dg_model_bounds(const u3dg_model *model, u3dg_crop_box *out);
/* No reference counterpart (cropModel applied to the trainer's model where it lives): crops the
 * trainer's model on the GPU, with its Adam moments, without a round trip through the host; training
 * may continue afterwards (densification statistics restart at zero). */
int u3dg_trainer_crop(u3dg_trainer *trainer, const u3dg_crop_box *box, float min_opacity);
/* suggestCropBox / modelBounds of the trainer's model (low_fraction < 0: modelBounds). */
int u3dg_trainer_suggest_crop_box(u3dg_trainer *trainer, float low_fraction, float high_fraction, float margin,
                                  u3dg_crop_box *out);

/* ------------------------------------------------------------------ model I/O and init (host) */

/* initGaussiansFromPoints (engine/include/u3d/splat/GaussianModel.h:41,
 * engine/src/splat/GaussianModel.cpp:68-144): xyz 3n, rgb 3n (0..1, NULL = grey); out arrays n (host
 * memory). The hash grid is built on the host and the 27-cell nearest-neighbour search runs on the
 * current GPU; the result is bit-identical to the reference's. Needs a GPU (U3DG_ERR_NO_DEVICE). */
int u3dg_init_gaussians_from_points(const float *xyz, const float *rgb, size_t n, u3dg_model *out);
/* writeSplatPly (engine/include/u3d/splat/SplatPly.h:12, engine/src/splat/SplatPly.cpp:261-282). */
int u3dg_write_splat_ply(const char *path, const u3dg_model *model);
/* No reference counterpart (the reference trainer keeps SH degree 0): writeSplatPly plus the higher-order
 * SH coefficients as the common 3DGS properties f_rest_0 .. f_rest_{3K-1} after f_dc_2, channel-major
 * (f_rest_{c*K + k} = sh_rest[(i*K + k)*3 + c], K = (degree+1)^2 - 1, the layout u3dg_render_sh
 * takes); degree 1..3. u3dg_read_splat_ply and the reference's reader ignore the extra properties. */
int u3dg_write_splat_ply_sh(const char *path, const u3dg_model *model, const float *sh_rest, int degree);
/* readSplatPly (SplatPly.h:17-18, SplatPly.cpp:284-342). Call with out == NULL to get *count first.
 * is_splat (may be NULL) reports whether the file held Gaussians or a plain point cloud. */
int u3dg_read_splat_ply(const char *path, u3dg_model *out, size_t capacity, size_t *count, int *is_splat);

/* ------------------------------------------------------------------ ground-truth rendering */

/* Renders a model whose colours are real spherical harmonics of degree 0..3 (3DGS convention:
 * rgb = max(0.5 + sum_l sum_m C_lm Y_lm(dir) * coeff, 0), dir = normalised mean - camera centre).
 * sh_rest holds ((degree+1)^2 - 1) * 3 floats per Gaussian, coefficient-major
 * (k-th coefficient of Gaussian i at sh_rest[(i * K + k) * 3 + ch]); NULL or degree 0 = DC only,
 * which is exactly Rasterizer::forward. No reference counterpart (the reference is DC only,
 * Rasterizer.cpp:189-194); used to render the synthetic scenes' ground truth. */
int u3dg_render_sh(const u3dg_model *model, const float *sh_rest, int degree, const u3dg_camera *camera,
                   const u3dg_raster_settings *settings, float *rgb);
/* u3dg_render_sh over `count` cameras with the model uploaded once; every view is quantised like
 * TrainImage::quantize (engine/src/splat/Trainer.cpp:10-16: lround(clamp(v, 0, 1) * 255)) into
 * rgb8, views back to back (sum of width*height*3 bytes). */
int u3dg_render_views_sh(const u3dg_model *model, const float *sh_rest, int degree, const u3dg_camera *cameras,
                         int count, const u3dg_raster_settings *settings, uint8_t *rgb8);

/* ------------------------------------------------------------------ learned warm-start */

/* No reference counterpart: the reference initialises with initGaussiansFromPoints
 * (engine/src/splat/GaussianModel.cpp:68-144), which stays the fallback and the reference point of
 * every comparison. A small FP32 MLP (134 -> 128 -> 128 -> 128 -> 11, ReLU) maps each SfM point's
 * neighbourhood feature to its initial Gaussian: residual log-scales and DC colour over the plain initialisation, quaternion and logit
 * opacity. Features (134 floats per point): 16 nearest points' relative positions (divided by the
 * plain-init scale, 48) and log distances (16), their colours (48), colour samples minus 0.5 from the 7
 * nearest views that see the point (21), and the fraction of those views found (1). Training, inference
 * and gradients run on the GPU. */
#define U3DG_MLP_INPUTS 134
#define U3DG_MLP_OUTPUTS 11
#define U3DG_MLP_PARAMS 51723

typedef struct u3dg_mlp u3dg_mlp;

/* Number of parameters (U3DG_MLP_PARAMS): per layer W (out x in, row-major) then b. */
int u3dg_mlp_param_count(void);
/* params (U3DG_MLP_PARAMS floats) or NULL for a seeded He-uniform initialisation whose output layer
 * starts at the plain initialisation. */
int u3dg_mlp_create(const float *params, unsigned int seed, u3dg_mlp **out);
int u3dg_mlp_params(u3dg_mlp *mlp, float *out);
/* y (n x 11) = network(x (n x 134)). */
int u3dg_mlp_forward(u3dg_mlp *mlp, const float *x, size_t n, float *y);
/* Weighted mean squared error against t (n x 11) with per-output weights (11, NULL = defaults), and
 * its gradient with respect to every parameter (grad: U3DG_MLP_PARAMS floats, may be NULL). */
int u3dg_mlp_loss_grad(u3dg_mlp *mlp, const float *x, const float *t, const float *weights, size_t n, float *loss,
                       float *grad);
/* Adam (lr, beta 0.9 / 0.999, eps 1e-8) over `epochs` shuffled passes (std::mt19937(seed)) of whole
 * batches; epoch_loss (epochs floats, may be NULL) gets each epoch's mean batch loss. */
int u3dg_mlp_train(u3dg_mlp *mlp, const float *x, const float *t, const float *weights, size_t n, int epochs,
                   int batch, float lr, unsigned int seed, float *epoch_loss);
void u3dg_mlp_destroy(u3dg_mlp *mlp);

/* The k (1, 3 or 16) nearest points of every query (brute force on the GPU; ties by lower index);
 * idx / dist2 get nq * k entries (-1 / FLT_MAX when fewer points exist). exclude_self skips the point
 * whose index equals the query's. */
int u3dg_knn(const float *queries, size_t nq, const float *points, size_t np, int k, int exclude_self, int *idx,
             float *dist2);
/* The 134-float feature of every point (features: n x 134). */
int u3dg_warmstart_features(const float *xyz, const float *rgb, size_t n, const u3dg_image *images, int count,
                            float *features);
/* Initial model of n points through the network (out: n Gaussians); mlp == NULL gives exactly
 * initGaussiansFromPoints. A point whose prediction is not finite keeps its plain initialisation; the
 * predicted opacity is floored at 0.05 (below the pruning threshold the first densification would
 * remove the Gaussian). */
int u3dg_warmstart_init(u3dg_mlp *mlp, const float *xyz, const float *rgb, size_t n, const u3dg_image *images,
                        int count, u3dg_model *out);

#ifdef __cplusplus
}
#endif

#endif /* U3DG_H */
