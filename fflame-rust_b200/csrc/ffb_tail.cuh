// ffb_tail.cuh -- host interface of the ahead-of-time kernels (ffb_tail.cu):
// density estimation, the tone map with the fused 2x firefly downsample,
// and the splat-throughput microbenchmark.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ffb {

// Per-pixel tone-map constants, derived on the host (in double) from the
// flame's ToneMap and the render's sample density (tonemap.wgsl:94-590).
struct TonemapArgs {
    int mode;              // 0 linear, 1 log, 2 density
    int highlight;         // 0 clip, 1 max_norm, 2 reinhard, 3 filmic
    int use_curve;
    int transparent;       // 0 opaque, 1 straight, 2 premultiplied
    int levels_enabled;
    int count_is_float;    // histogram .w holds a float count (after DE) instead of u32 bits
    const ulonglong4* exact;             // if not null: the exact histogram (r, g, b in 2^-24, count), read instead
    float exposure, inv_gamma, density_scale;
    float ls_a;            // k1 / (prefilter_white * ln 10)
    float ls_b;            // white_level * k2
    float white_level;
    float gamma_threshold, funcval;
    float vib, notvib;
    float saturation, hue_shift;
    float alpha_blend_low, alpha_blend_high;
    float levels_low, levels_high, levels_gamma, levels_density;
    float bg_lin[3];
};

// hist: wi*hi float4 (r, g, b sums, count).  ss = 1: out is wi*hi RGBA8 (and
// out_f, if not null, the float RGBA before quantisation); ss = 2: out is
// (wi/2)*(hi/2) RGBA8 after the firefly downsample.
cudaError_t launch_tonemap(const float4* hist, int wi, int hi, int ss, const TonemapArgs& a, const float* curve_lut,
                           uint8_t* out, float4* out_f, cudaStream_t s);

// One flame of a batched tone map: its histogram, output, size, the first
// output pixel's index in the batch's pixel sequence, its constants.
struct TonemapJob {
    const float4* hist;        // internal-resolution histogram (or DE output)
    uint8_t* out;              // output RGBA8
    const float* lut;
    long long px0;             // first OUTPUT pixel's index in the batch
    int w, h;                  // internal size
    int ss;                    // 1, or 2 (fused firefly downsample)
    TonemapArgs a;
};
cudaError_t launch_tonemap_batch(const TonemapJob* jobs, int n_jobs, long long total_px, cudaStream_t s);

// Density estimation table: entry c (counts 0..n-1, the last entry serving
// every larger count): (max accepted d^2, 1/h^2, 1/normaliser, reach).
// Computes output rows [y_lo, y_lo + h_out) into `out` (row y_lo first),
// reading sources from the whole w x h histogram (`exact`, when given,
// instead of `hist`).
cudaError_t launch_density_estimate(const float4* hist, const ulonglong4* exact, int w, int h,
                                    const float4* table, int table_n, int radius, int y_lo, int h_out, float4* out, cudaStream_t s,
                                    int count_f = 0);

// The spatial filter of one batch (histogram_blur.wgsl): `batch` (u32
// counts) filtered along rows into `tmp`, then along columns and added into
// `acc` (float counts).  sigma in pixels, sigma_d in counts.
cudaError_t launch_hist_filter(const float4* batch, float4* tmp, float4* acc, int w, int h, float sigma, float sigma_d,
                               cudaStream_t s);

// Density estimation of all w x h rows with the weight table in a file-scope
// device array of kDeStaticEntries entries instead of allocated memory (the
// contract is at its definition in ffb_tail.cu). de_static_entries: the
// table's length for these radii, or -1 when it exceeds the array.
constexpr int kDeStaticEntries = 65536;
int de_static_entries(double r_max, double r_min, double curve);
cudaError_t density_estimate_static(const float4* hist, int w, int h, double r_max, double r_min, double curve,
                                    float4* out, cudaStream_t s);

// The differentiable render's tone map (ffb_diff_tail.cu): n pixels of a
// bilinear histogram (r, g, b sums, weight) to linear-light RGBA (alpha 1),
// and its vector-Jacobian product dh = J^T dimg per pixel.  `samples` is the
// forward pass's device counter of plotted samples; npx, area and white give
// the sample density's constants as tonemap_args derives them.
cudaError_t launch_diff_tonemap(const float4* hist, size_t n, const TonemapArgs& a, const float* lut, const uint64_t* samples,
                                double npx, double area, double white, float4* out, cudaStream_t s);
cudaError_t launch_diff_tonemap_vjp(const float4* hist, const float4* dimg, size_t n, const TonemapArgs& a, const float* lut,
                                    const uint64_t* samples, double npx, double area, double white, float4* dh, cudaStream_t s);

// Tile-sorted accumulation (ffb_tiles.cu): one pass over a launch's records
// (u64: pixel index | palette index << 32) into the histogram `hist` --
// the exact one (ulonglong4 a pixel) when `exact`, else the u32-count /
// FP32-colour one (float4 a pixel) -- by 64x64-pixel tiles.  The records are n_segs
// segments of seg_cap (one a chaos block), followed by the segments' counts
// (u32 each).  Scratch: count/fill n_tiles words, off/work_off n_tiles + 1,
// work 2, band_fill tiles_y, band_part_off kMaxBands + 1, then (16-byte
// aligned) 1024 uint4 for the palette's fixed-point colours; tmp n_segs * seg_cap
// u64 (the band-grouped records); sorted n_segs * seg_cap words.
struct TileGeom { int w, h, tiles_x, tiles_y, n_tiles; };
constexpr int kMaxTiles = 16384, kMaxBands = 512, kMaxCols = 512;
cudaError_t launch_tile_pass(const unsigned long long* rec, unsigned long long seg_cap, int n_segs, const TileGeom& g,
                             unsigned slice, unsigned* count, unsigned* off, unsigned* fill, unsigned* work_off, unsigned* work,
                             unsigned* band_fill, unsigned* band_part_off, unsigned long long* tmp, unsigned* sorted,
                             const float4* pal, int pal_n, void* hist, bool exact, int n_sm, cudaStream_t s);

// The deterministic accumulation's u64 sums (2^-32 units) as float4.
cudaError_t launch_fixed_to_float(const ulonglong4* fx, size_t n, float4* out, cudaStream_t s);

// Histogram <-> (u32 count plane, f32 rgb plane), for collectives.
cudaError_t launch_pack(const float4* hist, size_t n, unsigned* cnt, float* rgb, cudaStream_t s);
cudaError_t launch_unpack(const unsigned* cnt, const float* rgb, size_t n, float4* hist, cudaStream_t s);

// Splat-throughput microbenchmark: `n_ops` random-address atomic splats of
// the given kind into `buf` (n_words u32 words): kind 0 = 4 scalar atomics a
// sample (the splat), 1 = one u32 atomic, 2 = one vector f32x4 reduction.
cudaError_t launch_atomic_bench(uint32_t* buf, uint32_t n_pixels, uint64_t n_samples, int kind, int blocks, cudaStream_t s);

}  // namespace ffb
