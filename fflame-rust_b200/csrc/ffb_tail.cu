// ffb_tail.cu -- ahead-of-time sm_100a kernels of the render tail.
//
// * density estimation: a variable-width Gaussian gather over the histogram
//   (this build's DE; no reference counterpart -- the reference writes
//   flam3's DE attributes unused, src/flame_xml.rs:1488-1490);
// * the log-density tone map (shaders/tonemap.wgsl:94-590) with the mean
//   colour of accumulate.wgsl:115-230 and, at 2x supersampling, the
//   firefly-clamped 2x2 downsample of src/export/supersample.rs:132-167
//   fused into the same kernel, so the supersampled RGBA8 never exists;
// * a splat-throughput microbenchmark (the L2 atomic roofline).
//
// All three are HBM/L2-bound byte work: no tensor cores; one thread per
// output pixel, coalesced along rows.

#include "ffb_tail.cuh"

namespace ffb {

namespace {

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

__device__ __forceinline__ float3 rgb_to_hsv(float3 c) {                 // tonemap.wgsl:152-184
    float mx = fmaxf(fmaxf(c.x, c.y), c.z), mn = fminf(fminf(c.x, c.y), c.z), d = mx - mn;
    float h = 0.f, s = 0.f;
    if (d > 0.00001f) {
        s = d / mx;
        if (c.x >= mx) h = (c.y - c.z) / d; else if (c.y >= mx) h = 2.0f + (c.z - c.x) / d; else h = 4.0f + (c.x - c.y) / d;
        h *= 60.0f; if (h < 0.f) h += 360.0f;
    }
    return make_float3(h, s, mx);
}
__device__ __forceinline__ float3 hsv_to_rgb(float3 c) {                 // tonemap.wgsl:187-220
    float h = c.x, s = c.y, v = c.z;
    if (s <= 0.f) return make_float3(v, v, v);
    float hh = h >= 360.0f ? 0.0f : h;
    hh /= 60.0f;
    unsigned i = (unsigned)hh;
    float ff = hh - (float)i;
    float p = v * (1.f - s), q = v * (1.f - s * ff), t = v * (1.f - s * (1.f - ff));
    switch (i) { case 0: return make_float3(v, t, p); case 1: return make_float3(q, v, p); case 2: return make_float3(p, v, t);
                 case 3: return make_float3(p, q, v); case 4: return make_float3(t, p, v); default: return make_float3(v, p, q); }
}
__device__ __forceinline__ float curve_sample(const float* lut, float x) {
    // Linear filter, clamp-to-edge, read at u = (255x + 0.5)/256 (tonemap.wgsl:478-485).
    float t = clampf(x * 255.0f, 0.0f, 255.0f);
    int i0 = (int)floorf(t);
    int i1 = min(i0 + 1, 255);
    float fr = t - (float)i0;
    return lut[i0] * (1.0f - fr) + lut[i1] * fr;
}
__device__ __forceinline__ float smooth(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.f, 1.f);
    return t * t * (3.f - 2.f * t);
}

// One pixel of the tone map: cnt = hits, sum = colour sums.  Returns the
// RGBA before quantisation.
__device__ float4 tonemap_px(const TonemapArgs& A, const float* lut, float cnt, float3 sum) {
    float3 mean = make_float3(0.f, 0.f, 0.f);
    if (cnt > 0.f) {                                                     // accumulate.wgsl:205-210
        mean = make_float3(clampf(sum.x / cnt, 0.f, 1.f), clampf(sum.y / cnt, 0.f, 1.f), clampf(sum.z / cnt, 0.f, 1.f));
    }
    const float bucket = cnt * 100.0f;                                   // tonemap.wgsl:252
    float3 color;
    float alpha = 0.f;
    const float g = A.inv_gamma;
    if (A.mode == 0) {
        color = make_float3(powf(mean.x * A.exposure, g), powf(mean.y * A.exposure, g), powf(mean.z * A.exposure, g));
        alpha = clampf(bucket * 0.01f * A.density_scale, 0.f, 1.f);
    } else if (A.mode == 2) {
        float nd = clampf(bucket * 0.01f * A.exposure, 0.f, 1.f);
        float gd = powf(nd, g);
        color = make_float3(gd, gd, gd);
        alpha = nd;
    } else {
        // brightness_scale (tonemap.wgsl:94-112), log10(1+x) through log1p.
        float ls = 0.f;
        if (!(bucket < 0.001f)) ls = A.ls_a * log1pf(A.ls_b * bucket) / (A.white_level * bucket);
        const float fp0 = ls * (mean.x * bucket), fp1 = ls * (mean.y * bucket), fp2 = ls * (mean.z * bucket);
        const float fp3 = ls * bucket * A.white_level;
        if (fp3 > 0.f) {
            if (fp3 <= A.gamma_threshold) {
                float fr = fp3 / A.gamma_threshold;
                alpha = (1.f - fr) * fp3 * A.funcval + fr * powf(fp3, g);
            } else alpha = powf(fp3, g);
        }
        const float l2 = fp3 > 0.f ? A.vib * alpha / fp3 : 0.f;
        if (A.notvib > 0.f)
            color = make_float3(l2 * fp0 + A.notvib * powf(fp0, g), l2 * fp1 + A.notvib * powf(fp1, g), l2 * fp2 + A.notvib * powf(fp2, g));
        else
            color = make_float3(l2 * fp0, l2 * fp1, l2 * fp2);
    }
    if (A.saturation != 1.0f || A.hue_shift != 0.0f) {                   // tonemap.wgsl:371-401
        float3 h = rgb_to_hsv(color);
        if (A.hue_shift != 0.0f) { h.x += A.hue_shift; if (h.x < 0.f) h.x += 360.f; else if (h.x >= 360.f) h.x -= 360.f; }
        if (A.saturation != 1.0f) h.y = clampf(h.y * A.saturation, 0.f, 1.f);
        color = hsv_to_rgb(h);
    }
    if (A.mode == 1) { color.x *= A.exposure; color.y *= A.exposure; color.z *= A.exposure; }
    color = make_float3(fmaxf(color.x, 0.f), fmaxf(color.y, 0.f), fmaxf(color.z, 0.f));
    if (A.highlight == 1) {                                              // tonemap.wgsl:414-477
        float m = fmaxf(color.x, fmaxf(color.y, color.z));
        if (m > 1.f) color = make_float3(color.x / m, color.y / m, color.z / m);
    } else if (A.highlight == 2) {
        float lum = 0.2126f * color.x + 0.7152f * color.y + 0.0722f * color.z;
        if (lum > 1e-6f) { float s = (lum / (1.f + lum)) / lum; color = make_float3(color.x * s, color.y * s, color.z * s); }
        color = make_float3(fminf(color.x, 1.f), fminf(color.y, 1.f), fminf(color.z, 1.f));
    } else if (A.highlight == 3) {
        auto aces = [](float x) { return clampf((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f), 0.f, 1.f); };
        color = make_float3(aces(color.x), aces(color.y), aces(color.z));
    } else {
        color = make_float3(fminf(color.x, 1.f), fminf(color.y, 1.f), fminf(color.z, 1.f));
    }
    float3 fc = color;
    if (A.use_curve && bucket > 0.001f)                                  // tonemap.wgsl:486-493
        fc = make_float3(curve_sample(lut, color.x), curve_sample(lut, color.y), curve_sample(lut, color.z));
    float lev = 1.f;                                                     // apply_levels, tonemap.wgsl:124-149
    if (A.levels_density > 0.f) {
        float nd = cnt / A.levels_density;
        if (A.levels_high <= A.levels_low) lev = nd > A.levels_low ? 1.f : 0.f;
        else {
            float cl = clampf((nd - A.levels_low) / (A.levels_high - A.levels_low), 0.f, 1.f);
            lev = (A.levels_gamma != 1.0f && A.levels_gamma > 0.f) ? powf(cl, A.levels_gamma) : cl;
        }
    }
    const float lin_a = clampf(bucket * 0.01f * A.density_scale, 0.f, 1.f);   // tonemap.wgsl:514-529
    const float gam_a = clampf(alpha, 0.f, 1.f);
    const float bt = smooth(A.alpha_blend_low, A.alpha_blend_high, gam_a);
    const float base_a = gam_a + (lin_a - gam_a) * bt;
    const float fa = A.levels_enabled ? fminf(base_a, lev) : base_a;
    const float inv22 = 1.0f / 2.2f;
    if (A.transparent != 0) {                                            // tonemap.wgsl:531-577
        float3 os = make_float3(powf(fmaxf(fc.x * fa, 0.f), inv22), powf(fmaxf(fc.y * fa, 0.f), inv22), powf(fmaxf(fc.z * fa, 0.f), inv22));
        if (A.transparent == 2) return make_float4(os.x, os.y, os.z, fa);
        float cov = fmaxf(os.x, fmaxf(os.y, os.z));
        if (cov > 0.f) return make_float4(os.x / cov, os.y / cov, os.z / cov, cov);
        return make_float4(0.f, 0.f, 0.f, cov);
    }
    float3 f = make_float3(A.bg_lin[0] * (1.f - fa) + fc.x * fa, A.bg_lin[1] * (1.f - fa) + fc.y * fa, A.bg_lin[2] * (1.f - fa) + fc.z * fa);
    return make_float4(powf(f.x, inv22), powf(f.y, inv22), powf(f.z, inv22), 1.0f);   // tonemap.wgsl:582-589
}

__device__ __forceinline__ float hist_count(const float4& v, int count_is_float) {
    return count_is_float ? v.w : (float)__float_as_uint(v.w);
}

__device__ __forceinline__ uchar4 quantise(float4 o) {
    return make_uchar4((unsigned char)rintf(clampf(o.x, 0.f, 1.f) * 255.f), (unsigned char)rintf(clampf(o.y, 0.f, 1.f) * 255.f),
                       (unsigned char)rintf(clampf(o.z, 0.f, 1.f) * 255.f), (unsigned char)rintf(clampf(o.w, 0.f, 1.f) * 255.f));
}

__global__ void __launch_bounds__(256) k_tonemap1(const float4* __restrict__ hist, int n, TonemapArgs A, const float* __restrict__ lut_g,
                                                  uchar4* __restrict__ out, float4* __restrict__ out_f) {
    __shared__ float lut[256];
    lut[threadIdx.x] = lut_g[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = hist[i];
    const float4 o = tonemap_px(A, lut, hist_count(v, A.count_is_float), make_float3(v.x, v.y, v.z));
    out[i] = quantise(o);
    if (out_f) out_f[i] = o;
}

// 2x: tone map the four internal pixels of an output pixel, quantise each
// to 8 bits, then the firefly clamp and box (supersample.rs:132-167).
__global__ void __launch_bounds__(256) k_tonemap2(const float4* __restrict__ hist, int wi, int ow, int oh, TonemapArgs A,
                                                  const float* __restrict__ lut_g, uchar4* __restrict__ out) {
    __shared__ float lut[256];
    lut[threadIdx.x] = lut_g[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ow * oh) return;
    const int ox = i % ow, oy = i / ow;
    float s[4][4], lum[4];
    const int dx[4] = {0, 1, 0, 1}, dy[4] = {0, 0, 1, 1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 v = hist[(size_t)(oy * 2 + dy[k]) * wi + (ox * 2 + dx[k])];
        const uchar4 q = quantise(tonemap_px(A, lut, hist_count(v, A.count_is_float), make_float3(v.x, v.y, v.z)));
        s[k][0] = q.x; s[k][1] = q.y; s[k][2] = q.z; s[k][3] = q.w;
        lum[k] = s[k][0] + 2.0f * s[k][1] + s[k][2];
    }
    // median of four = mean of the middle two
    float a = lum[0], b = lum[1], c = lum[2], d = lum[3], t;
    if (a > b) { t = a; a = b; b = t; }
    if (c > d) { t = c; c = d; d = t; }
    if (a > c) { t = a; a = c; c = t; }
    if (b > d) { t = b; b = d; d = t; }
    if (b > c) { t = b; b = c; c = t; }
    const float median = 0.5f * (b + c);
    const float cap = median * 4.0f + 64.0f;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float sc = lum[k] > cap ? cap / lum[k] : 1.0f;
        acc[0] += s[k][0] * sc; acc[1] += s[k][1] * sc; acc[2] += s[k][2] * sc; acc[3] += s[k][3];
    }
    unsigned char r[4];
#pragma unroll
    for (int c2 = 0; c2 < 4; ++c2) r[c2] = (unsigned char)clampf(roundf(acc[c2] * 0.25f), 0.f, 255.f);
    out[i] = make_uchar4(r[0], r[1], r[2], r[3]);
}

// Density estimation, gather form: output pixel p sums, over sources q in
// the (2R+1)^2 window, w(|p-q|, count_q) * (rgb_q, count_q).  The source
// window is staged in shared memory per 32x8 tile.
constexpr int DE_TX = 32, DE_TY = 8;
__global__ void __launch_bounds__(DE_TX * DE_TY) k_density(const float4* __restrict__ hist, int w, int h, const float4* __restrict__ tab,
                                                           int tab_n, int R, float4* __restrict__ out) {
    extern __shared__ float4 tile[];                                     // (TX+2R) x (TY+2R) sources
    const int tw = DE_TX + 2 * R, th = DE_TY + 2 * R;
    const int x0 = blockIdx.x * DE_TX - R, y0 = blockIdx.y * DE_TY - R;
    for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
        const int sx = x0 + i % tw, sy = y0 + i / tw;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (sx >= 0 && sy >= 0 && sx < w && sy < h) {
            const float4 hv = hist[(size_t)sy * w + sx];
            v = make_float4(hv.x, hv.y, hv.z, (float)__float_as_uint(hv.w));
        }
        tile[i] = v;
    }
    __syncthreads();
    const int lx = threadIdx.x % DE_TX, ly = threadIdx.x / DE_TX;
    const int px = blockIdx.x * DE_TX + lx, py = blockIdx.y * DE_TY + ly;
    if (px >= w || py >= h) return;
    float ar = 0.f, ag = 0.f, ab = 0.f, ac = 0.f;
    for (int dy = -R; dy <= R; ++dy) {
        const float4* row = tile + (ly + R + dy) * tw + (lx + R);
        for (int dx = -R; dx <= R; ++dx) {
            const float4 v = row[dx];
            if (v.w <= 0.f) continue;
            const int ci = v.w < (float)(tab_n - 1) ? (int)v.w : tab_n - 1;
            const float4 e = tab[ci];
            const float d2 = (float)(dx * dx + dy * dy);
            if (d2 > e.x) continue;
            const float wt = __expf(-4.5f * d2 * e.y) * e.z;
            ar += wt * v.x; ag += wt * v.y; ab += wt * v.z; ac += wt * v.w;
        }
    }
    out[(size_t)py * w + px] = make_float4(ar, ag, ab, ac);
}

// Random-address splat microbenchmark (the L2 atomic peak this kernel
// class can reach).  A cheap integer hash gives the addresses.
__global__ void k_atomic_bench(uint32_t* __restrict__ buf, uint32_t n_pixels, uint64_t n_samples, int kind) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 12345u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_samples; i += stride) {
        h ^= h << 13; h ^= h >> 17; h ^= h << 5;
        const uint32_t px = h % n_pixels;
        float* p = reinterpret_cast<float*>(buf) + (size_t)px * 4;
        if (kind == 0) {
            atomicAdd(p + 0, 0.25f); atomicAdd(p + 1, 0.5f); atomicAdd(p + 2, 0.75f);
            atomicAdd(reinterpret_cast<uint32_t*>(p + 3), 1u);
        } else if (kind == 1) {
            atomicAdd(reinterpret_cast<uint32_t*>(p + 3), 1u);
        } else {
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(0.25f), "f"(0.5f), "f"(0.75f), "f"(1.0f) : "memory");
        }
    }
}

}  // namespace

cudaError_t launch_tonemap(const float4* hist, int wi, int hi, int ss, const TonemapArgs& a, const float* curve_lut,
                           uint8_t* out, float4* out_f, cudaStream_t s) {
    if (ss == 1) {
        const int n = wi * hi;
        k_tonemap1<<<(n + 255) / 256, 256, 0, s>>>(hist, n, a, curve_lut, reinterpret_cast<uchar4*>(out), out_f);
    } else if (ss == 2) {
        const int ow = wi / 2, oh = hi / 2, n = ow * oh;
        k_tonemap2<<<(n + 255) / 256, 256, 0, s>>>(hist, wi, ow, oh, a, curve_lut, reinterpret_cast<uchar4*>(out));
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_density_estimate(const float4* hist, int w, int h, const float4* table, int table_n, int radius,
                                    float4* out, cudaStream_t s) {
    const size_t smem = (size_t)(DE_TX + 2 * radius) * (DE_TY + 2 * radius) * sizeof(float4);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_density, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((w + DE_TX - 1) / DE_TX, (h + DE_TY - 1) / DE_TY);
    k_density<<<grid, DE_TX * DE_TY, smem, s>>>(hist, w, h, table, table_n, radius, out);
    return cudaGetLastError();
}

cudaError_t launch_atomic_bench(uint32_t* buf, uint32_t n_pixels, uint64_t n_samples, int kind, int blocks, cudaStream_t s) {
    k_atomic_bench<<<blocks, 256, 0, s>>>(buf, n_pixels, n_samples, kind);
    return cudaGetLastError();
}

}  // namespace ffb
