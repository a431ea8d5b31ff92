/* nprush.h — C ABI of libnprush_cuda.so, the B200 (sm_100a) implementation of
 * nprush's differentiable splat / Bezier rasterisation hot path.
 *
 * The reference (wooningeire/nprush) exposes this path through TypeScript
 * manager classes over WebGPU.  Each entry point below names the reference
 * method it replaces (file:line in src/lib/gpu/).  All functions:
 *   - are extern "C", take plain pointers and sizes, and return int status
 *     (NPS_OK = 0, negative on error); nps_last_error() gives a thread-local
 *     message for the last failure on the calling thread;
 *   - enqueue work on the context's CUDA stream and return without waiting,
 *     except the read_* functions, which wait for the copy to finish;
 *   - are not thread-safe per context: one host thread drives one context,
 *     as one JS thread drives one GPUDevice queue in the reference.
 * Matrices are 16 floats, column-major (WGSL mat4x4f as uploaded by
 * Float32Array from wgpu-matrix).  Images are row-major, y = 0 at the top.
 */
#ifndef NPRUSH_H
#define NPRUSH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  NPS_OK = 0,
  NPS_ERR_INVALID = -1,   /* bad argument (null handle, size 0, size mismatch) */
  NPS_ERR_CUDA = -2,      /* CUDA runtime error (message in nps_last_error) */
  NPS_ERR_NOMEM = -3,     /* device allocation failed */
  NPS_ERR_CAPACITY = -4,  /* a work buffer was too small; sizes were grown, retry */
  NPS_ERR_TIMEOUT = -5,   /* a bounded device-side wait gave up */
  NPS_ERR_STATE = -6      /* call order violated (e.g. dispatch before set_target) */
};

/* Where a pointer argument lives. */
enum {
  NPS_MEM_HOST = 0,          /* host memory: copied before the call returns */
  NPS_MEM_DEVICE = 1,        /* device memory: copied on the context stream */
  NPS_MEM_DEVICE_BORROW = 2  /* device memory kept by reference until replaced
                                (like a texture view bound into a bind group) */
};

typedef struct nps_ctx nps_ctx;
typedef struct nps_splat_opt nps_splat_opt;
typedef struct nps_bezier_opt nps_bezier_opt;
typedef struct nps_gs nps_gs;

/* ---------------------------------------------------------------- context */
/* Replaces requestGpu() (requestGpu.ts:16-64): binds a CUDA device and stream. */
int nps_create(int device, nps_ctx** out);
int nps_destroy(nps_ctx* ctx);
/* Waits for all work queued on the context stream (the reference never waits). */
int nps_sync(nps_ctx* ctx);
/* Uses an external CUDA stream (cudaStream_t) instead of the context's own. */
int nps_set_stream(nps_ctx* ctx, void* cuda_stream);
/* Stable sort of n (key, value) pairs of device memory by the low `bits`
 * bits of the keys (1..32), in place, on the context's stream; waits for it.
 * The library's onesweep radix sort (no reference counterpart: the reference
 * builds its tile lists without sorting, splat_backward.wgsl:199-210): one
 * histogram kernel, then one kernel per 8-bit digit whose tiles find their
 * output offsets by a bounded decoupled look-back.  spin_limit bounds the
 * polls of one unpublished tile status (0 = the default, 2^20); stall_tile
 * (tests; 0xffffffff = none) is treated as never published.  Returns
 * NPS_ERR_TIMEOUT when a look-back gave up (the output is then unsorted but
 * nothing outside the buffers is written).  Allocates its work buffers per
 * call. */
int nps_sort_pairs(nps_ctx* ctx, uint32_t* keys, uint32_t* vals, uint32_t n, int bits, uint32_t spin_limit,
                   uint32_t stall_tile);
const char* nps_last_error(void);
const char* nps_version(void);

/* ============================================= splats, reference semantics
 * Parameter record: 16 floats per splat, the reference's AoS layout
 * (splat_forward.wgsl:1-6): pos.xyz, sx | r, g, b, opacity | qw, qx, qy, qz |
 * sy, shape_a, shape_b, sz.  Gradients are the reference's fixed-point i32
 * sums (splat_backward.wgsl:436-455); Adam state m, v is 16 floats per splat.
 */
/* new GpuSplatOptimizerManager({numSplats}) (GpuSplatOptimizerManager.ts:43-125).
 * Parameters start zeroed (all splats dead); upload them with write_params. */
int nps_splat_opt_create(nps_ctx* ctx, uint32_t num_splats, nps_splat_opt** out);
int nps_splat_opt_destroy(nps_splat_opt* opt);
/* queue.writeBuffer(splatBuffer, first*64, ...) (GpuSplatOptimizerManager.ts:93). */
int nps_splat_opt_write_params(nps_splat_opt* opt, const float* splats, uint32_t first, uint32_t count, int mem);
/* Optimizer state for tests and checkpoints: the i32 gradient accumulators
 * (N*16), Adam m, v (N*16 f32 each), the step counter t and grad_accum (N f32).
 * Null pointers are skipped. */
int nps_splat_opt_write_state(nps_splat_opt* opt, const int32_t* grads, const float* adam_m, const float* adam_v,
                              float adam_t, const float* grad_accum, int mem);
int nps_splat_opt_read_state(nps_splat_opt* opt, float* splats, int32_t* grads, float* adam_m, float* adam_v,
                             float* adam_t, float* grad_accum);
/* writeSplatVPMatrix(vp, vpInv, blur) (GpuSplatOptimizerManager.ts:281-301),
 * for num_views views (16 floats each).  blur_enabled is stored, unused, as in
 * the reference backward. */
int nps_splat_opt_write_vp(nps_splat_opt* opt, const float* vp, const float* vp_inv, uint32_t num_views,
                           int blur_enabled);
/* setBackwardTarget(colour, depth, w, h) (GpuSplatOptimizerManager.ts:303-317):
 * rgba num_views*h*w*4 floats (.rgb used), depth num_views*h*w floats
 * (reciprocal encoding 1 - 0.1/w, 1.0 = background). */
int nps_splat_opt_set_target(nps_splat_opt* opt, const float* rgba, const float* depth, uint32_t width,
                             uint32_t height, uint32_t num_views, int mem);
/* dispatch(encoder) (GpuSplatOptimizerManager.ts:365-388): backward over all
 * views, Adam step, and ADC on every 25th call. */
int nps_splat_opt_dispatch(nps_splat_opt* opt);
/* The three stages of dispatch, separately (splat_backward / splat_step /
 * splat_adc).  backward optionally writes the fp32 composite the backward
 * computes (num_views*h*w*4: r, g, b, reciprocal depth) to out_rgbd (device).
 * A backward whose raster's bounded record-staging wait or sort look-back
 * gave up leaves invalid gradients; the next backward reports it with
 * NPS_ERR_TIMEOUT (and runs nothing further).  Work memory grows with the
 * views and tiles: besides the pair lists, 32 KB of transmittance
 * checkpoints per (view, 16 x 16 tile) (655 MB for 8 views at 800 x 800);
 * an allocation that fails returns NPS_ERR_NOMEM. */
int nps_splat_opt_backward(nps_splat_opt* opt, float* out_rgbd_device);
int nps_splat_opt_step(nps_splat_opt* opt);
int nps_splat_opt_adc(nps_splat_opt* opt);
/* Headless GpuSplatForwardPipelineManager.dispatch(enc, clear=true)
 * (GpuSplatForwardPipelineManager.ts:114-137, splat_forward.wgsl:42-156):
 * fp32 composite of all splats (index 0 in front), w < 0.1 culled, splats
 * whose centre lies outside 0 <= z <= w (past the far plane) clipped away as
 * the pipeline clips their quads, alpha < 0.001 discarded, cleared to
 * colour 0.05 / depth 1.  out_rgba and out_depth
 * are device buffers of h*w*4 floats each (depth replicated in rgb, alpha in a). */
int nps_splat_opt_render(nps_splat_opt* opt, const float* vp, uint32_t width, uint32_t height, float* out_rgba,
                         float* out_depth);
/* GpuSplatForwardPipelineManager.dispatch(enc, clear=false), the pass that
 * loads its attachments: the same draw blended over the current contents of
 * rgba and depth (device h*w*4 floats each, read and written in place; depth
 * may be null), colour alpha and depth alpha accumulating as a + dst.a (1 - a)
 * per fragment (the pipeline's blend state, GpuSplatForwardPipelineManager.ts:64-77). */
int nps_splat_opt_render_load(nps_splat_opt* opt, const float* vp, uint32_t width, uint32_t height, float* rgba,
                              float* depth);
/* Device pointers of the library-owned buffers (splatBuffer, gradBuffer,
 * Adam m / v, grad_accum), for zero-copy access; valid until destroy. */
int nps_splat_opt_buffers(nps_splat_opt* opt, float** splats, int32_t** grads, float** adam_m, float** adam_v,
                          float** grad_accum);

/* ADC without device allocation.  No counterpart in the reference.  For
 * callers that cannot let the library allocate device memory: applications
 * that give their whole device-memory budget to their own arena or pool, and
 * ones that share the GPU with latency-critical work (a render loop), where
 * cudaMalloc / cudaFree may synchronise the device.  Runs the splat ADC
 * (splat_adc.wgsl:28-87, same kernel as nps_splat_opt_adc) on caller-owned
 * device buffers: splats N*16, adam_m / adam_v N*16 (16-byte aligned),
 * grad_accum N floats (4-byte aligned); misaligned pointers return
 * NPS_ERR_INVALID.  Its scratch (dead-slot list + result word) is a fixed
 * array compiled into the library: at most 262144 splats (larger N returns
 * NPS_ERR_CAPACITY), and every GPU that loads the library holds that 1 MiB
 * until exit.  Allocates nothing.  The first call on a device looks up the
 * array's device address (with that device current) and keeps it for the
 * process, so make the first call before any stream capture, and do not call
 * it again on a device after cudaDeviceReset (the kept address belongs to the
 * destroyed context).  Calls share the array, which keeps the last call's contents;
 * calls that overlap on the GPU (different streams, or different host
 * threads) race on it.  Runs on cuda_stream (null = legacy default stream) of
 * the current device; clones_host (may be null) receives the number of clones
 * and splits, which makes the call wait for the stream. */
int nps_splat_adc_noalloc(float* splats, float* adam_m, float* adam_v, float* grad_accum, uint32_t num_splats,
                          float adam_t, void* cuda_stream, uint32_t* clones_host);

typedef struct nps_stats {
  uint64_t pairs;          /* (tile, primitive) pairs overlapped in the last backward, all views (splats:
                              the binning sorts only those that can fall among a tile's first 1024,
                              reserved[1]) */
  uint64_t pairs_capped;   /* pairs composited after the per-tile cap */
  uint32_t max_tile_len;   /* longest tile list before the cap */
  uint32_t adc_clones;     /* clones + splits performed by the last ADC */
  uint32_t step_count;     /* dispatch() calls so far */
  uint32_t reserved[3];    /* Splats: [1] pairs kept by the cap-aware binning, [2] bounded device waits
                              that gave up (a backward after one returns NPS_ERR_TIMEOUT).
                              Bezier: [0] spawns.  Gaussians: [0] kernel launches per replay of the
                              captured train step (its graph's kernel nodes), [1] graph replays that
                              skipped their update (pair overflow), [2] bounded device waits
                              that gave up (raster record staging, sort look-back) */
} nps_stats;
int nps_splat_opt_stats(nps_splat_opt* opt, nps_stats* out);
/* Bound of the backward raster's waits for its staged records (polls of the
 * mbarrier; 0 = the default, 2^22) and, for tests, one batch of tile 0 (view
 * 0) whose copies are never issued (0xffffffff = none), so that its wait runs
 * out on a normal input: the raster's CTA for that tile stops, and the next
 * backward returns NPS_ERR_TIMEOUT.  No counterpart in the reference. */
int nps_splat_opt_set_wait_guard(nps_splat_opt* opt, uint32_t spin_limit, uint32_t stall_batch);
/* Sets the manager's stepCount (GpuSplatOptimizerManager.ts:380, dispatch()
 * calls so far; ADC runs when it reaches a multiple of 25): a restored
 * checkpoint continues the ADC schedule. */
int nps_splat_opt_set_step_count(nps_splat_opt* opt, uint32_t count);

/* ========================================== Bezier strokes, reference semantics
 * Record: 20 floats per curve (bezier_forward.wgsl:1-7): p0.xyz, width |
 * p1.xyz, softness | p2.xyz, _ | p3.xyz, _ | r, g, b, a.  18 optimised
 * parameters, fixed-point i32 gradients (bezier_backward.wgsl:536-558), Adam m,
 * v 18 floats per curve, ADC accumulators grad_accum / loss_accum (1 float per
 * curve each) and the 512 x 512 i32 pixel_loss map. */
/* new GpuBezierOptimizerManager({numBeziers}) (GpuBezierOptimizerManager.ts:46-267). */
int nps_bezier_opt_create(nps_ctx* ctx, uint32_t num_beziers, nps_bezier_opt** out);
int nps_bezier_opt_destroy(nps_bezier_opt* opt);
/* queue.writeBuffer(bezierBuffer, first*80, ...) (GpuBezierOptimizerManager.ts:102). */
int nps_bezier_opt_write_params(nps_bezier_opt* opt, const float* beziers, uint32_t first, uint32_t count, int mem);
int nps_bezier_opt_write_state(nps_bezier_opt* opt, const int32_t* grads, const float* adam_m, const float* adam_v,
                               float adam_t, const float* grad_accum, const float* loss_accum,
                               const int32_t* pixel_loss, int mem);
int nps_bezier_opt_read_state(nps_bezier_opt* opt, float* beziers, int32_t* grads, float* adam_m, float* adam_v,
                              float* adam_t, float* grad_accum, float* loss_accum, int32_t* pixel_loss);
/* writeVPMatrix + writeVPInvMatrix (GpuBezierOptimizerManager.ts:269-288) for
 * num_views views; the Adam step's offscreen kill and the ADC use the first. */
int nps_bezier_opt_write_vp(nps_bezier_opt* opt, const float* vp, const float* vp_inv, uint32_t num_views);
/* writeMode (:290), writeBgPenalty (:298), writeMaxWidth (:309),
 * writeKillThresholds (:318), setAdcPeriod (:328), writeNoKill (:332). */
int nps_bezier_opt_write_mode(nps_bezier_opt* opt, float mode);
int nps_bezier_opt_write_bg_penalty(nps_bezier_opt* opt, float weight);
int nps_bezier_opt_write_max_width(nps_bezier_opt* opt, float max_width);
int nps_bezier_opt_write_kill_thresholds(nps_bezier_opt* opt, float alpha_thresh, float width_thresh);
int nps_bezier_opt_set_adc_period(nps_bezier_opt* opt, uint32_t period);
int nps_bezier_opt_write_no_kill(nps_bezier_opt* opt, int no_kill);
/* setBackwardTarget(target, targetDepth, bg, bgDepth, normal, w, h)
 * (GpuBezierOptimizerManager.ts:341-368): RGBA textures num_views*h*w*4
 * floats, depth textures num_views*h*w floats. */
int nps_bezier_opt_set_target(nps_bezier_opt* opt, const float* target_rgba, const float* target_depth,
                              const float* bg_rgba, const float* bg_depth, const float* normal_rgba, uint32_t width,
                              uint32_t height, uint32_t num_views, int mem);
/* dispatch(encoder) (GpuBezierOptimizerManager.ts:370-406): backward over all
 * views, Adam step (gradients / (w*h)), ADC every adc_period calls. */
int nps_bezier_opt_dispatch(nps_bezier_opt* opt);
/* The stages of dispatch separately; backward optionally writes the composite
 * (num_views*h*w*4: r, g, b, reciprocal depth) to out_rgbd (device).  Its
 * work memory includes 37 KB of transmittance checkpoints per (view, 16 x 16
 * tile). */
int nps_bezier_opt_backward(nps_bezier_opt* opt, float* out_rgbd_device);
int nps_bezier_opt_step(nps_bezier_opt* opt);
int nps_bezier_opt_adc(nps_bezier_opt* opt);
/* Headless GpuBezierForwardPipelineManager.dispatch (GpuBezierForwardPipelineManager.ts:131-148,
 * bezier_forward.wgsl:48-182): fp32 premultiplied composite of all curves
 * (curve 0 in front) over bg_rgba (device h*w*4, null = cleared to 0), with
 * an optional single-channel brush texture (device brush_h*brush_w, sampled
 * bilinearly at level 0, u repeat / v clamp; null = analytic coverage only).
 * out_rgba: device h*w*4. */
int nps_bezier_opt_render(nps_bezier_opt* opt, const float* vp, uint32_t width, uint32_t height, const float* bg_rgba,
                          const float* brush, uint32_t brush_w, uint32_t brush_h, float* out_rgba);
int nps_bezier_opt_buffers(nps_bezier_opt* opt, float** beziers, int32_t** grads, float** adam_m, float** adam_v,
                           float** grad_accum, float** loss_accum, int32_t** pixel_loss);
int nps_bezier_opt_stats(nps_bezier_opt* opt, nps_stats* out);
/* Sets the manager's stepCount (GpuBezierOptimizerManager.ts:398). */
int nps_bezier_opt_set_step_count(nps_bezier_opt* opt, uint32_t count);

/* ====================================== 3D Gaussians (the trainer)
 * No counterpart in the reference, which fits linear-parameter generalised
 * splats; this trainer keeps the reference's fit-a-scene call pattern
 * (GpuSplatOptimizerManager: write params, write camera(s), set target(s),
 * dispatch) for standard 3D Gaussians.  Parameter record: 64 floats per
 * Gaussian (256 B): mean xyz | log-scale xyz | quaternion wxyz | opacity logit |
 * pad | SH coefficients 16 x rgb (coefficient-major) | pad.  Loss: 0.8 L1 +
 * 0.2 (1 - SSIM) unless nps_gs_set_loss chooses another.  All views of a step
 * are processed by every launch. */
int nps_gs_create(nps_ctx* ctx, uint32_t capacity, uint32_t sh_degree, nps_gs** out);
int nps_gs_destroy(nps_gs* gs);
/* Upload records [first, first+count); the active count grows to cover them. */
int nps_gs_write_params(nps_gs* gs, const float* params, uint32_t first, uint32_t count, int mem);
int nps_gs_set_count(nps_gs* gs, uint32_t count);
int nps_gs_write_state(nps_gs* gs, const float* adam_m, const float* adam_v, uint32_t step, int mem);
/* Host copies of the active records (null pointers skipped); adc_grad / adc_denom
 * are the accumulated view-space gradient norms and visibility counts. */
/* ADC accumulators of the first `count` Gaussians (sum of view-space gradient
 * norms, number of views that saw each one); null pointers are skipped. */
int nps_gs_write_adc_stats(nps_gs* gs, const float* adc_grad, const float* adc_denom, int mem);
int nps_gs_read_state(nps_gs* gs, float* params, float* grads, float* adam_m, float* adam_v, float* adc_grad,
                      float* adc_denom);
/* Learning rates: mean, log-scale, quaternion, opacity logit, SH DC, SH rest. */
int nps_gs_set_lr(nps_gs* gs, const float* lr6);
int nps_gs_set_background(nps_gs* gs, float r, float g, float b);
/* Target images: num_targets x h x w x 4 floats (rgb used), resident on the device. */
int nps_gs_set_targets(nps_gs* gs, const float* rgba, uint32_t width, uint32_t height, uint32_t num_targets, int mem);
/* Image size for rendering without targets (set_targets sets it too). */
/* Targets uploaded from host memory without stalling the step in flight: the
 * images host_images[ids[i]] (W x H x 4 floats each; page-locked memory lets
 * the copy run concurrently) go to a staging buffer on a copy stream, then to
 * the targets in stream order, after every step already queued.  Target i is
 * then ids[i]'s image.  For a training loop that uploads the next step's
 * targets while the current step runs (no reference counterpart). */
int nps_gs_upload_targets(nps_gs* gs, const float* host_images, const uint32_t* ids, uint32_t n_ids, uint32_t w,
                          uint32_t h);
/* (loss, mean L1, mean SSIM) of the last loss computed, waiting for it. */
int nps_gs_read_loss(nps_gs* gs, float* loss3_host);
int nps_gs_set_image_size(nps_gs* gs, uint32_t width, uint32_t height);
/* Cameras of the next step: num_views view-projection matrices (+ inverses),
 * and for each the index of its target image (null = 0, 1, 2, ...). */
int nps_gs_set_views(nps_gs* gs, const float* vp, const float* vp_inv, const uint32_t* target_ids, uint32_t num_views);
/* Paired differentiable rendering: forward keeps only per-record and per-pixel
 * state (final transmittance + last contributor); backward replays. */
int nps_gs_forward(nps_gs* gs, float* out_rgba_device);
/* Fused loss of the last forward against the targets; loss3 (host, may be
 * null) = {loss, mean L1, mean SSIM} (L1 + D-SSIM) or {loss, mean L1, mean
 * squared error} (L1, L2).  Also stores dL/dimage for backward. */
int nps_gs_loss(nps_gs* gs, float* loss3);
/* Loss of the fused path (no reference counterpart; the reference's splat
 * loss is L2 on colour plus a depth term, splat_backward.wgsl:250-257):
 * kind NPS_GS_LOSS_L1_DSSIM = (1 - w) mean|x - y| + w (1 - mean SSIM) with an
 * 11 x 11 Gaussian window (sigma 1.5) and w = ssim_weight (default: this
 * kind, w = 0.2); NPS_GS_LOSS_L1 = mean|x - y|; NPS_GS_LOSS_L2 = mean
 * (x - y)^2; means over the 3 H W colour values of the views.  ssim_weight
 * in [0, 1] (ignored by L1 and L2). */
enum { NPS_GS_LOSS_L1_DSSIM = 0, NPS_GS_LOSS_L1 = 1, NPS_GS_LOSS_L2 = 2 };
int nps_gs_set_loss(nps_gs* gs, int kind, float ssim_weight);
/* dl_dimage: device num_views*h*w*4 floats, or null for the fused loss gradient. */
int nps_gs_backward(nps_gs* gs, const float* dl_dimage_device);
/* The same backward with dL/dimage in host memory (num_views*h*w*4 floats,
 * copied before the backward runs): the paired call for hosts that hold no
 * device memory of their own (a TypeScript caller through Deno FFI). */
int nps_gs_backward_host(nps_gs* gs, const float* dl_dimage_host);
int nps_gs_adam(nps_gs* gs);
/* forward + loss + backward + Adam.  In graph mode the first call (and any
 * call after the step's shape changed: Gaussian count, views, image size,
 * targets) runs eagerly to size every buffer and then captures the whole
 * step as one CUDA graph; later calls replay it with no host synchronisation
 * inside the step.  A replay whose tile pairs exceed the captured capacity
 * (25% above the capturing step's) skips its parameter update; the next call
 * grows the capacity and recaptures (nps_stats.reserved[1] counts skips). */
int nps_gs_train_step(nps_gs* gs, float* loss3);
int nps_gs_set_graph(nps_gs* gs, int enable);
/* Host copies of the last forward's image (num_views*h*w*4: rgb, final T) and
 * of dL/dimage from the last nps_gs_loss (null pointers skipped). */
int nps_gs_read_image(nps_gs* gs, float* rgba_host, float* dl_dimage_host);
/* Tiles and raster variants (no reference counterpart; the reference's
 * tile is its 16 x 16 workgroup, splat_backward.wgsl:136).  The binning
 * cuts the image into T x T tiles, T = 8, 16 (default) or 32
 * (nps_gs_set_tile); the deterministic backward and forms 0 and 2 below
 * need 16.
 * Two forms of the forward and backward raster kernels, each for several
 * (pixels per thread, records staged per batch); T * T / ppt threads cover a
 * tile:
 *   form 0, one CTA per (tile, view), records double-buffered, T = 16:
 *     (1, 256), (2, 128), (2, 256), (4, 64), (4, 128);
 *   form 1, persistent and warp-specialised: a fixed grid of CTAs pulls the
 *     (view, tile) items of all views from a queue ordered longest first; in
 *     each CTA one producer warp stages batches of records into a 3-slot ring
 *     (bulk copies completing on mbarriers) while the consumer warps
 *     composite or differentiate, with no CTA-wide barrier in the loop:
 *     T = 8: (1 or 2, 64 or 128); T = 16: (1, 128), (2 or 4, 64 or 128);
 *     T = 32: (4, 64 or 128);
 *   form 2, the kernels of form 0 with a 1D grid whose blocks take the
 *     (view, tile) items longest first (the forward by list length, the
 *     backward by its last contributor), so the longest tiles start first
 *     and the grid's tail is short: T = 16, the (ppt, stage) of form 0.
 * nps_gs_set_raster selects one per pass for the current tile (a stage of 0
 * means the form's default: 256 / ppt for form 0, 128 for form 1);
 * nps_gs_set_variant selects form 0; nps_gs_set_tile changes the tile (and
 * switches to that tile's default persistent variants where the current ones
 * do not serve it); nps_gs_get_raster reports tile, forward form, ppt, stage,
 * backward form, ppt, stage (choice7).  nps_gs_autotune_raster bins the
 * current views at every tile size (timing the binning), times every variant
 * of each tile, forward and backward, and keeps the tile with the smallest
 * binning + fastest forward + fastest backward, with those variants; with
 * cache_path it first looks the workload up in that text file (device,
 * image size, views, SH degree, Gaussian count to ~19%, deterministic mode)
 * and appends its choice.  choice7 (may be null) as nps_gs_get_raster;
 * times_ms99 (may be null): for T = 8, 16, 32 in turn, 33 floats: binning,
 * then the forward and then the backward time of the 16 variants (0, 1,
 * 256), (0, 2, 128), (0, 2, 256), (0, 4, 64), (0, 4, 128), (1, 1, 64),
 * (1, 1, 128), (1, 2, 64), (1, 2, 128), (1, 4, 64), (1, 4, 128), (2, 1,
 * 256), (2, 2, 128), (2, 2, 256), (2, 4, 64), (2, 4, 128) (0 where a variant
 * does not serve the tile; -1 throughout when the choice came from the
 * cache).  nps_gs_autotune is the same tuner reporting only ppt and stage
 * (choice4) and the 16 x 16 form-0 times (times_ms10). */
int nps_gs_set_tile(nps_gs* gs, uint32_t tile);
int nps_gs_set_raster(nps_gs* gs, int fwd_form, int fwd_ppt, int fwd_stage, int bwd_form, int bwd_ppt,
                      int bwd_stage);
int nps_gs_set_variant(nps_gs* gs, int fwd_ppt, int fwd_stage, int bwd_ppt, int bwd_stage);
int nps_gs_get_raster(nps_gs* gs, int* choice7);
int nps_gs_autotune_raster(nps_gs* gs, const char* cache_path, int* choice7, float* times_ms99);
int nps_gs_autotune(nps_gs* gs, const char* cache_path, int* choice4, float* times_ms10);
/* Bounded waits of the radix sorts (depth keys, tile keys).  The sorts are
 * onesweep radix sorts: each tile of keys finds its output offsets by a
 * decoupled look-back over the tiles before it, polling each unpublished
 * tile status at most spin_limit times (0 = the default, 2^20).  A
 * look-back that gives up counts a timeout (nps_stats.reserved[2]); the
 * sort's output is then wrong but stays inside its buffers, the train step
 * skips its Adam update, and the next forward or train step returns
 * NPS_ERR_TIMEOUT.  stall_tile (tests; 0xffffffff = none) names one tile whose
 * status is treated as never published, which makes a look-back run out on a
 * normal input. */
int nps_gs_set_sort_guard(nps_gs* gs, uint32_t spin_limit, uint32_t stall_tile);
/* Deterministic mode: the backward reduces each (view, Gaussian) gradient in
 * two passes (per-pair tile sums stored, then summed per record in sorted-pair
 * order) instead of with float atomics, so repeated runs are bit-identical.
 * Costs a pair-sized buffer (40 B per pair) and a second sort. */
int nps_gs_set_deterministic(nps_gs* gs, int enable);
/* Gradient accumulation for views launched one at a time (the plain per-view
 * trainer): with accumulate != 0 backward adds to the gradient buffer instead
 * of overwriting it; loss_views (0 = the views of each call) is the number of
 * views the loss is averaged over, so that V single-view calls sum to the
 * gradient of one V-view call.  The ADC statistic is always the NDC-space
 * gradient of each view's own loss. */
int nps_gs_set_accumulate(nps_gs* gs, int accumulate, uint32_t loss_views);
/* Checkpoint (no reference counterpart: the reference never reads its GPU
 * state back).  File: a 104-byte little-endian header (magic "NPSGSCK1",
 * version, count, SH degree, Adam step, ADC seed, loss views, learning rates,
 * background, SSIM weight, loss kind) followed by params, Adam m, Adam v (count x 64
 * floats each) and the two ADC accumulators (count floats each).  Load
 * requires count <= capacity and the same SH degree. */
int nps_gs_save(nps_gs* gs, const char* path);
/* Number of Gaussians (changes with write_params, set_count, ADC and load). */
int nps_gs_count(nps_gs* gs, uint32_t* count);
int nps_gs_load(nps_gs* gs, const char* path);
/* Adaptive density control (the plain threshold rule): prune Gaussians with
 * opacity < prune_opacity; densify those whose average view-space gradient
 * norm (accumulated by backward, averaged over the views that saw them) is
 * >= grad_thresh — split into two (scales / 1.6, means drawn from the parent)
 * if their largest scale exceeds split_scale, else clone — while the capacity
 * allows; compacts records and Adam state, resets the accumulators.
 * counts4 (host, may be null) = {count before, count after, densified, pruned}.
 * The k-th call on a trainer samples split children with seed k. */
int nps_gs_adc(nps_gs* gs, float grad_thresh, float split_scale, float prune_opacity, uint32_t* counts4);
/* Learned ADC.  Record float 63 (padding) carries a lineage id: set it with
 * nps_gs_assign_ids (id = base + index); clones and split children inherit it.
 * nps_gs_adc_features writes, for the current Gaussians, the policy's 16-float
 * feature vectors (features_dev, n x 16), the plain rule's decision
 * (plain_dev, may be null: 0 keep, 1 clone, 2 split, 3 prune) and the ids
 * (ids_dev, may be null); step_frac is the position in the ADC schedule.
 * nps_gs_adc_policy applies the network's argmax decision per Gaussian (keep /
 * clone / split / prune), falling back to the plain rule where a Gaussian's
 * logits are not finite or for every Gaussian when policy is null; then
 * densifies within the capacity and compacts like nps_gs_adc.
 * fallback_host (may be null) = Gaussians decided by the plain rule. */
int nps_gs_assign_ids(nps_gs* gs, uint32_t base);
/* Logit given to "keep" in the policy's decision (default 0 = argmax); a
 * positive margin makes the network clone, split or prune only when that
 * logit exceeds keep's by the margin. */
int nps_gs_set_policy_margin(nps_gs* gs, float margin);
int nps_gs_adc_features(nps_gs* gs, float step_frac, float grad_thresh, float split_scale, float prune_opacity,
                        float* features_dev, uint8_t* plain_dev, uint32_t* ids_dev);
typedef struct nps_mlp nps_mlp;
typedef struct nps_pt nps_pt;
typedef struct nps_mesh nps_mesh;
int nps_gs_adc_policy(nps_gs* gs, nps_mlp* policy, float step_frac, float grad_thresh, float split_scale,
                      float prune_opacity, uint32_t* counts4, uint32_t* fallback_host);
/* PSNR (dB) of each view of the last forward against its target, rgb in [0, 1]. */
int nps_gs_psnr(nps_gs* gs, float* psnr_host);
int nps_gs_buffers(nps_gs* gs, float** params, float** grads, float** adam_m, float** adam_v, float** image,
                   float** dl_dimage);
/* Device pointers of the ADC accumulators (count floats each; valid until the
 * next ADC or load, which may swap buffers).  Used to sum them over ranks. */
int nps_gs_adc_buffers(nps_gs* gs, float** adc_grad, float** adc_denom);
int nps_gs_stats(nps_gs* gs, nps_stats* out);
/* Per-stage device timing with CUDA events on the context stream (off by
 * default).  Stages: 0 preprocess, 1 depth sort, 2 pair emit, 3 tile sort,
 * 4 tile ranges, 5 forward raster, 6 loss, 7 backward raster, 8 projection
 * backward, 9 Adam.  stage_times waits for the stream, adds the recorded
 * intervals to the totals, and returns totals (ms) and counts per stage. */
int nps_gs_set_timing(nps_gs* gs, int enable);
int nps_gs_stage_times(nps_gs* gs, double* ms, uint64_t* calls, uint32_t n, int reset);


/* ---- target preprocessing --------------------------------------------------
 * Device images: H x W float4 RGBA, 16-byte aligned (depth images use .x),
 * processed on the context's stream.  The reference stores into rgba8unorm
 * textures; quantize != 0 applies that conversion (clamp to [0, 1], round to
 * the nearest of 256 levels, ties to even), otherwise the stored floats are
 * returned.  Alpha is written as 1. */
/* Replaces GpuBlurPipelineManager's pass (src/lib/gpu/blur.wgsl:23-48): 2r+1
 * taps along (dir_x, dir_y), edge-clamped, weights exp(-i^2 / (2 sigma^2));
 * flags bit 0: input sRGB, bit 1: output sRGB. */
int nps_blur(nps_ctx* ctx, const float* src_rgba, float* dst_rgba, uint32_t w, uint32_t h, int32_t dir_x,
             int32_t dir_y, int32_t radius, uint32_t flags, float sigma, int quantize);
/* Replaces GpuDepthAwareBlurPipelineManager's pass (depth_aware_blur.wgsl:12-53):
 * (2r+1)^2 bilateral window with spatial, colour and depth sigmas 10, 0.5, 0.5. */
int nps_depth_aware_blur(nps_ctx* ctx, const float* color_rgba, const float* depth_rgba, float* dst_rgba, uint32_t w,
                         uint32_t h, int32_t radius, int quantize);
/* The splat edge pass (splat_edge.wgsl:13-44): Sobel magnitude of the depth,
 * edge-clamped, through smoothstep(thr_min, thr_max, .) (the reference's
 * SPLAT_EDGE_THRESHOLD_MIN / _MAX, constants.ts:40-41: 0.02, 0.06). */
int nps_splat_edge(nps_ctx* ctx, const float* depth_rgba, float* dst_rgba, uint32_t w, uint32_t h, float thr_min,
                   float thr_max, int quantize);

/* ---- learned ADC policy network (no reference counterpart) ----------------
 * 16 -> 64 -> 64 -> 3 MLP with ReLU; the three logits (clone, split, prune)
 * and a fixed 0 logit for keep form a softmax.  Parameters: one fp32 vector of
 * nps_mlp_num_params() floats: W1 [64x16], b1 [64], W2 [64x64], b2 [64],
 * W3 [3x64], b3 [3] (row-major, out x in).  Products run on the tensor cores
 * with bf16 operands and fp32 accumulation. */
int nps_mlp_num_params(void);
int nps_mlp_create(nps_ctx* ctx, nps_mlp** out);
int nps_mlp_destroy(nps_mlp* mlp);
int nps_mlp_init(nps_mlp* mlp, uint64_t seed);
int nps_mlp_set_params(nps_mlp* mlp, const float* params_host);
int nps_mlp_get_params(nps_mlp* mlp, float* params_host);
/* logits_dev [n x 3] of features_dev [n x 16] (device pointers, 16-byte aligned). */
int nps_mlp_forward(nps_mlp* mlp, const float* features_dev, uint32_t n, float* logits_dev);
/* Gradient of the mean class-weighted cross-entropy of one batch (labels:
 * 0 keep, 1 clone, 2 split, 3 prune; class_w4 may be null for 1s). */
int nps_mlp_grads(nps_mlp* mlp, const float* features_dev, const uint8_t* labels_dev, uint32_t n,
                  const float* class_w4, float* grads_host, float* loss_host);
/* Mini-batch Adam (lr, betas 0.9 / 0.999, eps 1e-8) for `epochs` passes over
 * device-resident samples, reshuffled each epoch from `seed`; per-epoch mean
 * loss and accuracy to the host arrays when given. */
int nps_mlp_train(nps_mlp* mlp, const float* features_dev, const uint8_t* labels_dev, uint32_t n,
                  const float* class_w4, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                  float* loss_curve, float* acc_curve);

/* ---- path-traced targets (GpuPathTracePipelineManager.ts) -------------------
 * buildBvh (bvh.ts:202-223) alone, on the host (no device needed):
 * `vertices` are n_vertices x 12 floats [px py pz, nx ny nz, r g b a, u v],
 * `indices` n_tris x 3; nodes must hold max(1, 2 n_tris - 1) x 8 floats,
 * tri_indices n_tris x 3.  The SAH tree is the reference's bit for bit
 * (8 floats per node, leaf flag 0x80000000 in data1). */
int nps_bvh_build(const float* vertices, uint32_t n_vertices, const uint32_t* indices, uint32_t n_tris,
                  float* nodes, uint32_t* tri_indices, uint32_t* n_nodes);
/* Replaces setMeshes (GpuPathTracePipelineManager.ts:103-151): the
 * concatenated meshes (host arrays, layout as nps_bvh_build; colour alpha
 * below 0.5 marks a perfect mirror), their BVH built on the host and
 * uploaded with the geometry.  The environment starts as one white texel. */
int nps_pt_create(nps_ctx* ctx, const float* vertices, uint32_t n_vertices, const uint32_t* indices, uint32_t n_tris,
                  nps_pt** out);
int nps_pt_destroy(nps_pt* pt);
/* The uploaded BVH, as buildBvh returns it (BvhResult.nodes / triIndices). */
int nps_pt_bvh_size(nps_pt* pt, uint32_t* n_nodes, uint32_t* n_tris);
int nps_pt_read_bvh(nps_pt* pt, float* nodes, uint32_t* tri_indices);
/* The env_tex binding (path_trace.wgsl:31): w x h float4, host or device
 * pointer; sampled bilinearly, u repeating, v clamped (:204-208). */
int nps_pt_set_env(nps_pt* pt, const float* rgba, uint32_t w, uint32_t h);
/* Replaces dispatch()'s path-trace pass (path_trace.wgsl:222-268) for
 * n_frames consecutive frames starting at `frame`: each adds one sample per
 * pixel to accum_rgba (device, w x h float4: radiance sums and the sample
 * count), as n_frames dispatches would.  inv_view_proj: 16 floats,
 * column-major (writeInvViewProjMat).  Asynchronous on the context stream. */
int nps_pt_trace(nps_pt* pt, const float* inv_view_proj, uint32_t frame, uint32_t n_frames, float* accum_rgba,
                 uint32_t w, uint32_t h);
/* Rays that gave up because the traversal visited more nodes than the tree
 * has (cannot happen for a BVH built here; a guard against corruption). */
int nps_pt_overflows(nps_pt* pt, uint32_t* count);
/* dispatch()'s resolve pass (path_trace_resolve.wgsl:20-30): mean radiance
 * x 4 through c / (c + 1), alpha 1; quantize != 0 rounds to the rgba8unorm
 * levels the reference's output texture holds. */
int nps_pt_resolve(nps_ctx* ctx, const float* accum_rgba, float* out_rgba, uint32_t w, uint32_t h, int quantize);

/* ---- mesh render pass (GpuMeshRenderPipelineManager.ts, envmap.wgsl) --------
 * nps_mesh_create replaces the manager's constructor mesh plus setGroundMesh
 * (GpuMeshRenderPipelineManager.ts:41-160): the meshes concatenated in draw
 * order, vertices n_vertices x 12 floats [pos, normal, rgba, uv], indices
 * n_tris x 3 (host arrays). */
int nps_mesh_create(nps_ctx* ctx, const float* vertices, uint32_t n_vertices, const uint32_t* indices,
                    uint32_t n_tris, nps_mesh** out);
int nps_mesh_destroy(nps_mesh* mesh);
/* The matcap texture (mesh.wgsl:9-10, linear, clamped) and the environment
 * panorama (envmap.wgsl:17-18, linear, u repeating, v clamped): w x h
 * float4, host or device pointer; both start as one white texel. */
int nps_mesh_set_matcap(nps_mesh* mesh, const float* rgba, uint32_t w, uint32_t h);
int nps_mesh_set_env(nps_mesh* mesh, const float* rgba, uint32_t w, uint32_t h);
/* setPbrMesh (GpuMeshRenderPipelineManager.ts:161-248): triangles from
 * first_tri on (the PBR mesh, drawn last) use mesh.wgsl's vert_pbr / frag_pbr
 * (:72-121): albedo and tangent-space normal map (w x h float4, host
 * pointers), sampled linearly with repeat; srgb != 0 decodes the albedo
 * texels from sRGB first, as the reference's sRGB texture view does. */
int nps_mesh_set_pbr(nps_mesh* mesh, uint32_t first_tri, const float* albedo_rgba, uint32_t aw, uint32_t ah, int srgb,
                     const float* normal_rgba, uint32_t nw, uint32_t nh);
/* One mesh render pass as the viewer's optimisation pass draws it
 * (GpuRunner.svelte.ts:611-634): the environment background (draw_env = 0:
 * the clear colour 0.05), then the mesh through mesh.wgsl's vert / frag with
 * back faces culled (counter-clockwise front) and depth "less" in draw order.
 * uniforms52: the shared uniform buffer (GpuUniformsBufferManager.ts, 208
 * bytes: viewProj, view, shadingMode (0 normals, 1 matcap), 3 pad,
 * invViewProj; matrices column-major).  Writes color_rgba (the shaded colour)
 * and depth_rgba (1 - 0.1 / max(w, 0.1) per fragment, 1 where no triangle):
 * device w x h float4 images, at most 16384 x 16384; quantize != 0 rounds
 * them to the 8-bit levels of the reference's targets.  The triangles'
 * clamped pixel boxes together must hold fewer than 2^42 pixels (2^32 work
 * chunks of 1024 pixels; e.g. four million full-screen triangles at
 * 1024 x 1024).  Asynchronous on the context stream. */
int nps_mesh_render(nps_mesh* mesh, const float* uniforms52, float* color_rgba, float* depth_rgba, uint32_t w,
                    uint32_t h, int draw_env, int quantize);

#ifdef __cplusplus
}
#endif
#endif /* NPRUSH_H */
