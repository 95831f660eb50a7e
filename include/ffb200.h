/*
 * ffb200.h -- C ABI of the B200 fractal-flame render path.
 *
 * Two layers, both plain C (pointers and sizes, no CUDA or torch types):
 *
 *  1. The drop-in: the exports of the reference's engine module
 *     (calibas/fflame-rust wasm/python/src/lib.rs), with the same JSON
 *     protocol -- `fae_call({"fn": "render", "config": <.fae JSON>, "width",
 *     "height", "iterations"?, "iterations_per_thread"?, "transparent"?,
 *     "premultiplied"?})` answers RGBA8 bytes as the output and
 *     {width, height, iterations, ms, iterations_per_thread} as the info
 *     (wasm/python/src/render.rs:45-91).  A status of 1 carries the error's
 *     text as the output.  OUTPUT and INFO are owned by the library, per
 *     calling thread, valid until that thread's next fae_call.
 *
 *  2. The typed render API, the C mirror of the reference's Rust surface
 *     `render(device, queue, RenderJob) -> Result<RenderOutput, RenderError>`
 *     (src/renderer/render.rs:48-466), plus the stages the render is made of
 *     (histogram, density estimation, tone map, variation probe), which the
 *     parity tests and the benchmark call directly.
 *
 * Every function returns an ffb_status; ffb_last_error() holds the message
 * of the calling thread's last failure.  Nothing here falls back to the CPU:
 * without a CUDA device the calls fail with FFB_ERR_NO_DEVICE.
 */
#ifndef FFB200_H
#define FFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ drop-in --- */

/* wasm/python/src/lib.rs:49-55: a request buffer in the library's memory. */
uint8_t* fae_alloc(size_t len);
/* wasm/python/src/lib.rs:57-62: frees a fae_alloc'd buffer. */
void fae_free(uint8_t* ptr, size_t len);
/* wasm/python/src/lib.rs:64-72: the last call's output bytes. */
const uint8_t* fae_output_ptr(void);
size_t fae_output_len(void);
/* wasm/python/src/lib.rs:74-82: the last call's info JSON. */
const uint8_t* fae_info_ptr(void);
size_t fae_info_len(void);
/* wasm/python/src/lib.rs:84-101: one call; 0, or 1 with the error's text
 * as the output.  Calls: "info", "variations", "render", "flame_import"
 * ({xml}: the configs, lib.rs:214-218), "encode_png"
 * ({config, width, height, iterations, ms, iterations_per_thread} with the
 * RGBA8 frame as `data`: the PNG as the output, lib.rs:227-232). */
int32_t fae_call(const uint8_t* req, size_t req_len, const uint8_t* data, size_t data_len);

/* ---------------------------------------------------------- typed API --- */

/* RenderError (src/renderer/render.rs:312-330) and the failures this build adds. */
typedef enum {
    FFB_OK = 0,
    FFB_ERR_INVALID = 1,        /* a bad argument */
    FFB_ERR_CONFIG = 2,         /* the config did not parse or asks for what this build lacks */
    FFB_ERR_TOO_LARGE = 3,      /* RenderError::TooLarge */
    FFB_ERR_OUT_OF_MEMORY = 4,  /* RenderError::OutOfMemory */
    FFB_ERR_CUDA = 5,           /* a CUDA call failed */
    FFB_ERR_COMPILE = 6,        /* NVRTC rejected the specialised kernel */
    FFB_ERR_CANCELLED = 7,      /* RenderError::Cancelled */
    FFB_ERR_NO_DEVICE = 8       /* no CUDA device */
} ffb_status;

enum { FFB_RNG_PCG = 0, FFB_RNG_PHILOX = 1 };       /* ffb_job.rng */
enum { FFB_MATH_PRECISE = 0, FFB_MATH_SFU = 1 };    /* ffb_job.math */

/* RenderJob (src/renderer/render.rs:48-137).  Zero means "default". */
typedef struct {
    uint32_t width, height;            /* output size */
    uint64_t iterations;               /* plotted samples of the internal render; 0: config max_iterations x ss^2 */
    uint32_t iterations_per_thread;    /* dispatch length of the PCG stream (0: 1024, the CLI's) */
    uint32_t burn_in;                  /* 0: 20 (render.rs:126) */
    uint32_t walkers;                  /* 0: sized to the budget */
    uint32_t supersample;              /* 1 or 2 (src/export/supersample.rs); 0: 1 */
    int32_t rng;                       /* FFB_RNG_* (default FFB_RNG_PHILOX) ; -1 = default */
    int32_t math;                      /* FFB_MATH_* */
    int32_t transparent;               /* 0 opaque, 1 straight alpha, 2 premultiplied */
    int32_t threads;                   /* threads a block (0: 128; the sorted schedule: one block a
                                          multiprocessor holding its share of the walkers) -- under the
                                          sorted schedule also the group the walkers are sorted within */
    uint64_t seed;                     /* 0: the config's (12345 under deterministic_rng) */
    uint32_t walker0;                  /* first walker id of this shard (multi-GPU sharding) */
    uint32_t schedule;                 /* 0 auto, 1 one walker a thread, 2 transform-sorted (same orbits) */
    uint32_t count_bits;               /* 32 (0): u32 count + FP32 colour sums (16 B a pixel); 64: exact
                                          integer accumulation -- u64 count and u64 colour sums in 24-bit
                                          fixed point (32 B a pixel), independent of the atomics' order
                                          (the exact count of accumulate.wgsl:185-199) */
    uint32_t accumulate;               /* 0 auto (tile-sorted above a 512 MB histogram, else direct),
                                          1 direct (a splat's atomics on the histogram), 2
                                          tile-sorted (samples emitted as records, sorted by 64x64 tile,
                                          summed in shared-memory bins; exact mode: the same bits as direct;
                                          32-bit mode: the same counts, colour sums in another FP32 order) */
    uint32_t plot;                     /* 0 auto, 1 inline (each walker plots its own samples), 2 deferred:
                                          the chaos kernel stores its samples and a plot kernel (the final
                                          chain, palette, symmetry copies, splat) runs beside the next
                                          launch on a second stream; 3 fused: plot warps in the walkers'
                                          own blocks take the samples through shared memory (no sample
                                          leaves the multiprocessor); the same histogram (Philox stream, no
                                          spatial filter, direct accumulation; fused also without an xaos
                                          orbit refresh; otherwise deferred or inline) */
    /* RenderProgress (src/renderer/render.rs:293-301, 624-693): `progress`
       is called after each launch of the chaos game with the plotted
       samples submitted so far and the render's total; `cancelled`
       returning nonzero before a launch stops the render (status
       FFB_ERR_CANCELLED, the histogram partial).  NULL: none.  With either
       set at most two launches are in flight, so a cancel takes effect
       within one launch of the chaos game. */
    void (*progress)(void* user, uint64_t current, uint64_t total);
    int (*cancelled)(void* user);
    void* progress_user;
} ffb_job;

/* RenderOutput (src/renderer/render.rs:207-218). */
typedef struct {
    uint32_t width, height;
    uint64_t total_iterations;         /* plotted samples (post burn-in) */
    uint64_t inframe_samples;          /* samples splatted into the frame */
    double render_time_ms;             /* device time of the whole render */
    uint64_t h2d_bytes;                /* host->device bytes this call copied */
    uint64_t d2h_bytes;                /* device->host bytes this call copied */
    uint32_t kernel_launches;          /* this library's kernels launched by this call */
    uint32_t reserved;
} ffb_output;

typedef struct ffb_renderer ffb_renderer;   /* FlameRenderer: a device, a stream, the module cache */

/* The calling thread's last error message ("" when none). */
const char* ffb_last_error(void);

/* sizeof(ffb_job) and sizeof(ffb_output), for bindings to check their layouts. */
void ffb_struct_sizes(size_t* job_bytes, size_t* output_bytes);
/* Build version and the device it would use. */
const char* ffb_version(void);

/* Apophysis / JWildfire `.flame` XML -> `.fae` configs (src/flame_xml.rs:
 * 41-425): *out is a JSON array of config objects, one a <flame> /
 * <jwf-flame> element, in a buffer of the library's valid until the calling
 * thread's next call.  The configs are 2-D (this build's path); a flame
 * with a 3-D camera is refused with the reason.  Needs no GPU. */
int ffb_flame_import(const char* xml, size_t xml_len, const char** out, size_t* out_len);

/* A frame (width*height*4 RGBA8 bytes) as the PNG the reference's CLI
 * writes: the config (.fae JSON) and the render's numbers in tEXt chunks
 * under src/png_metadata.rs:144-183's keys (Software, Resolution,
 * Iterations, RenderTime, IterationsPerThread, SpeedFactor, ConfigChecksum
 * "sha256:<hex>", Config, BackgroundColor, Exposure, Gamma, ToneCurve, ...).
 * `rgba` must hold width*height*4 bytes.  *out points at a buffer of the
 * library's, valid until the calling thread's next call.  Host memory
 * only; needs no GPU. */
int ffb_encode_png(const char* config, size_t config_len, const uint8_t* rgba, uint32_t width, uint32_t height,
                   uint64_t iterations, double ms, uint32_t iterations_per_thread, const uint8_t** out, size_t* out_len);

int ffb_renderer_create(int device, ffb_renderer** out);
void ffb_renderer_destroy(ffb_renderer* r);

/* A full render: config (.fae JSON) -> RGBA8 into the host buffer `rgba`
 * (width*height*4 bytes).  The timed region of the reference's
 * render_with (render.rs:483-804) plus the readback. */
int ffb_render(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job,
               uint8_t* rgba, ffb_output* out);

/* The same render with the RGBA8 result left in device memory (`d_rgba`,
 * width*height*4 bytes); `stream` is a cudaStream_t or NULL for the
 * renderer's own.  Returns once the work is enqueued when `sync` is 0. */
int ffb_render_device(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job,
                      void* d_rgba, void* stream, int sync, ffb_output* out);

/* The chaos game alone into a histogram read back to the host: `counts`
 * (w*h u32 hits) and `rgb` (w*h*3 f32 colour sums) at the internal size
 * (width*ss x height*ss).  The high-resolution export's readback path
 * (src/export/high_res.rs:2139-2175). */
int ffb_histogram(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job,
                  uint32_t* counts, float* rgb, ffb_output* out);

/* The same with counts as f32: the only form of a histogram the spatial
 * filter (filter_radius > 0: a bilateral Gaussian on each batch's
 * histogram, compute_kernel.rs:1663-1725) made fractional; ffb_histogram
 * refuses those. */
int ffb_histogram_f32(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job,
                      float* counts, float* rgb, ffb_output* out);

/* The spatial filter alone on a host histogram (u32 counts, rgb sums) of
 * one batch: out is w*h*4 floats (r, g, b, count) after the row and column
 * passes; sigma in pixels, sigma_d in counts.  The filter's parity entry. */
int ffb_hist_filter(ffb_renderer* r, const uint32_t* counts, const float* rgb, uint32_t w, uint32_t h, float sigma,
                    float sigma_d, float* out);

/* The same in exact mode (job->count_bits taken as 64): counts is w*h u64
 * hits, rgb the colour sums (f32 of the exact fixed-point sums). */
int ffb_histogram_u64(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job,
                      uint64_t* counts, float* rgb, ffb_output* out);

/* The tone map of a host histogram (counts as f32, colour sums), with the
 * config's tone-map settings and the given sample density:
 * tonemap.wgsl:224-590.  ss 1: rgba is w*h*4 bytes and `rgba_f` (if not
 * NULL) w*h*4 floats before quantisation; ss 2: rgba is (w/2)*(h/2)*4 after
 * the firefly downsample. */
int ffb_tonemap(ffb_renderer* r, const char* config, size_t config_len, const float* counts, const float* rgb,
                uint32_t w, uint32_t h, uint32_t ss, double sample_density, int32_t transparent,
                uint8_t* rgba, float* rgba_f);

/* Density estimation of a host histogram (counts, colour sums): radii in
 * histogram pixels.  Output counts and sums as f32. */
int ffb_density_estimate(ffb_renderer* r, const uint32_t* counts, const float* rgb, uint32_t w, uint32_t h,
                         float max_radius, float min_radius, float curve, float* out_counts, float* out_rgb);

/* Density estimation that allocates nothing, for callers that may not
 * allocate device memory while they run: an application whose own pool owns
 * the device, or a frame loop whose memory is fixed at start-up.  No
 * counterpart in the reference: an addition beside ffb_density_estimate.
 * d_hist: w*h float4 (r, g, b sums, u32 count bits), the layout
 * ffb_chaos_device writes; d_out: w*h float4 (r, g, b, count as f32); both
 * on the current device; stream NULL is the default stream.  Returns once
 * the work is queued.  The weight table lives in one static device array of
 * 65536 entries (1 MiB) shared by every call on a device:
 * FFB_ERR_TOO_LARGE when the radii need more (the table grows as
 * max_radius^(1/curve)), and calls whose work overlaps on the GPU race on
 * it.  The first call on a device looks up the array's address and should
 * come before any stream capture. */
int ffb_density_estimate_static(const void* d_hist, uint32_t w, uint32_t h, float max_radius, float min_radius,
                                float curve, void* d_out, void* stream);

/* The variation probe (shaders/core/main_template.wgsl:1467-1567): every
 * transform of the config (normals, then the final chain) at `npts`
 * points (x, y pairs), RNG slot = transform*npts + point.  `out` holds
 * n_transforms*npts (x, y) pairs.  `math` as ffb_job.math. */
int ffb_probe(ffb_renderer* r, const char* config, size_t config_len, const float* pts, uint32_t npts, int32_t math,
              float* out, uint32_t out_pairs);

/* One transform step at n points with explicit draw words (64 a point: the
 * iteration's slots, 0 the pick, 1 the opacity, then each variation's):
 * affine, variations, post (with_affine) or the variations alone.  The
 * single-step parity entry; `xform` >= normals selects a final. */
int ffb_apply_points(ffb_renderer* r, const char* config, size_t config_len, int32_t xform, uint32_t n,
                     const float* xs, const float* ys, const float* words, int32_t with_affine, int32_t math,
                     float* xo, float* yo);

/* ---- multi-GPU building blocks (one renderer a rank; the caller owns the
 * collectives).  The render of a walker shard into a caller-owned device
 * histogram (width*ss x height*ss float4: r, g, b sums and the u32 count's
 * bits), cleared here. */
int ffb_chaos_device(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job, void* d_hist,
                     void* stream, ffb_output* out);
/* Split a device histogram into a u32 count plane and an f32 rgb plane
 * (pixels*3), each summable by a collective in its own type, and back. */
int ffb_hist_pack(ffb_renderer* r, const void* d_hist, uint64_t pixels, void* d_counts, void* d_rgb, void* stream);
int ffb_hist_unpack(ffb_renderer* r, const void* d_counts, const void* d_rgb, uint64_t pixels, void* d_hist, void* stream);
/* Density estimation and tone map of output rows [row0, row0+rows) of a
 * summed histogram holding `total_samples` plotted samples, into `d_rgba`
 * (rows*width*4 bytes).  The DE halo is read from the whole histogram. */
int ffb_finish_device(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job, const void* d_hist,
                      uint64_t total_samples, uint32_t row0, uint32_t rows, void* d_rgba, void* stream);
/* The same from a window of the summed histogram: d_hist holds internal rows
 * [hist_row0, hist_row0 + hist_rows) (width*ss float4 a row), which must
 * cover the band's rows and the density-estimation reach around them
 * (ceil(radius * ss) rows each side, clamped to the image) -- what a rank
 * receives from a reduce-scatter of row windows (the exchange step planned
 * in place of the reference's single-GPU accumulate, accumulate.wgsl:115-230;
 * the reference renders on one device).  FFB_ERR_INVALID when it does not. */
int ffb_finish_band(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job, const void* d_hist,
                    uint32_t hist_row0, uint32_t hist_rows, uint64_t total_samples, uint32_t row0, uint32_t rows,
                    void* d_rgba, void* stream);

/* ---- the differentiable render: an addition beside the reference's render
 * (which has no gradients).  The chaos game with a bilinear splat and a
 * linearly interpolated palette, the log tone map in linear light (alpha 1),
 * and the gradient of a loss with respect to
 * theta = [n_xf*6 affine a..f | n_xf*n_var variation weights, transform-major
 * | n_xf colours], each plotted sample differentiated through the last
 * `window` iterations of its walker (default 16) from walker states
 * checkpointed every `checkpoint` iterations (default 64).  Philox stream,
 * no final transforms, supersampling or density estimation; log tone map,
 * clip highlights.  job->count_bits 64 accumulates the histogram in u64
 * fixed point (2^-32 units): the same bits whatever the order of the
 * atomics, so renders at nearby theta differ only by theta (finite
 * differences at small steps).  Device pointers; `stream` is a cudaStream_t passed
 * through as given (NULL: the legacy default stream); calls only enqueue. */
typedef struct ffb_diff ffb_diff;
int ffb_diff_create(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job, uint32_t window,
                    uint32_t checkpoint, ffb_diff** out);
/* ffb_specialize for the differentiable render's module (no device needed). */
int ffb_diff_specialize(const char* config, size_t config_len, uint32_t window, uint32_t checkpoint, size_t* cubin_bytes,
                        char* source, size_t source_len);
/* theta's shape: transforms, variations (and their names, comma-separated,
 * in theta's order), walkers and iterations a walker (burn-in included). */
int ffb_diff_layout(ffb_diff* d, uint32_t* n_xforms, uint32_t* n_variations, uint32_t* walkers, uint32_t* iterations,
                    char* names, size_t names_cap);
/* The config's own theta (host, n_xf*(7+n_var) floats). */
int ffb_diff_theta(ffb_diff* d, float* theta);
/* Forward at d_theta: the image (width*height float4, linear rgb, 1) and, if
 * d_hist is not NULL, a copy of the histogram (r, g, b sums, weight). */
int ffb_diff_forward(ffb_diff* d, const float* d_theta, float* d_image, float* d_hist, void* stream);
/* dL/dtheta (n_xf*(7+n_var) doubles) of the most recent forward, given
 * dL/dimage (width*height float4; alpha ignored), and, if d_grad_hist is
 * not NULL, dL/dhistogram (width*height float4). */
int ffb_diff_backward(ffb_diff* d, const float* d_grad_image, double* d_grad_theta, float* d_grad_hist, void* stream);
/* The most recent forward's plotted and in-frame samples (synchronises `stream`). */
int ffb_diff_samples(ffb_diff* d, uint64_t* plotted, uint64_t* inframe, void* stream);
/* Each variation's value and Jacobian at n points for transform `xform`
 * (host buffers; words as ffb_apply_points): out is n*n_var*6 floats
 * (vx, vy, dvx/dx, dvx/dy, dvy/dx, dvy/dy). */
int ffb_diff_jacobians(ffb_diff* d, int32_t xform, uint32_t n, const float* xs, const float* ys, const float* words, float* out);
void ffb_diff_destroy(ffb_diff* d);

/* ---- batches: many flames in one persistent launch a structure group,
 * tone-mapped in one launch, the device work captured as a CUDA graph.
 * The batched addition beside the reference's one-flame render. */
typedef struct {
    const char* config;      /* .fae JSON */
    size_t config_len;
    uint32_t width, height;  /* output size (no supersampling in batches) */
    uint64_t iterations;     /* this flame's plotted-sample budget */
    uint64_t seed;           /* this flame's stream key (0: the config's) */
} ffb_batch_item;
typedef struct ffb_batch ffb_batch;
/* Parse, specialise and upload every flame; with `tune`, time candidate
 * (threads a block, iterations a walker) pairs on 1/64 of every budget and
 * keep the fastest; capture the batch as a graph.  common: rng, math,
 * burn_in, transparent, threads / iterations_per_thread (used when not tuning). */
int ffb_batch_create(ffb_renderer* r, const ffb_batch_item* items, uint32_t n, const ffb_job* common, int32_t tune,
                     ffb_batch** out);
/* Replay the batch (stream NULL: the renderer's).  `ms`: device time. */
int ffb_batch_run(ffb_batch* b, void* stream, int32_t sync, double* ms);
/* Item `index`'s RGBA8 (width*height*4 host bytes) and its plotted samples. */
int ffb_batch_output(ffb_batch* b, uint32_t index, uint8_t* rgba, uint64_t* plotted);
int ffb_batch_info(ffb_batch* b, uint64_t* total_samples, uint32_t* threads, uint32_t* iters_per_walker, uint32_t* groups);
void ffb_batch_destroy(ffb_batch* b);

/* Compile the chaos-game kernel of a config's structure for sm_100a with
 * NVRTC, without a device (the shader builder's build step,
 * src/shader_builder_v2.rs:2337; src/shader_cache.rs).  Writes the CUBIN
 * size to *cubin_bytes and, if `source` is not NULL, up to source_len
 * bytes of the generated source.  Needs no GPU. */
int ffb_specialize(const char* config, size_t config_len, int32_t rng, int32_t math, size_t* cubin_bytes,
                   char* source, size_t source_len);
/* The module a render of `job` would compile (its rng, math, count_bits,
 * accumulation and plot modes; width and height may be 0): as ffb_specialize. */
int ffb_specialize_job(const char* config, size_t config_len, const ffb_job* job, size_t* cubin_bytes, char* source,
                       size_t source_len);

/* The splat-throughput microbenchmark: `samples` random splats of `kind`
 * (0: the 4-atomic splat, 1: one u32 atomic, 2: one f32x4 reduction) into
 * a histogram of `pixels`; returns the device milliseconds. */
int ffb_atomic_bench(ffb_renderer* r, uint32_t pixels, uint64_t samples, int32_t kind, double* ms);
/* The splat kernel's own throughput (no reference counterpart; a
 * measurement beside the render boundary): `job` rendered with deferred
 * plotting (plot 0 or 2; refused otherwise), each plot launch run alone
 * after its chaos launch on one stream.  *plot_ms: the plot launches'
 * summed device milliseconds; *samples: the records they plotted (post-
 * burn-in iterations); *inframe: the splats they made. */
int ffb_plot_bench(ffb_renderer* r, const char* config, size_t config_len, const ffb_job* job, double* plot_ms,
                   uint64_t* samples, uint64_t* inframe);

#ifdef __cplusplus
}
#endif

#endif /* FFB200_H */
