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

#include <algorithm>
#include <cmath>
#include <mutex>

namespace ffb {

namespace {

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

struct D3 { double x, y, z; };
__device__ __forceinline__ double clampd(double v, double lo, double hi) { return fmin(fmax(v, lo), hi); }

__device__ __forceinline__ D3 rgb_to_hsv(D3 c) {                         // tonemap.wgsl:152-184
    double mx = fmax(fmax(c.x, c.y), c.z), mn = fmin(fmin(c.x, c.y), c.z), d = mx - mn;
    double h = 0.0, s = 0.0;
    if (d > 0.00001) {
        s = d / mx;
        if (c.x >= mx) h = (c.y - c.z) / d; else if (c.y >= mx) h = 2.0 + (c.z - c.x) / d; else h = 4.0 + (c.x - c.y) / d;
        h *= 60.0; if (h < 0.0) h += 360.0;
    }
    return {h, s, mx};
}
__device__ __forceinline__ D3 hsv_to_rgb(D3 c) {                         // tonemap.wgsl:187-220
    double h = c.x, s = c.y, v = c.z;
    if (s <= 0.0) return {v, v, v};
    double hh = h >= 360.0 ? 0.0 : h;
    hh /= 60.0;
    unsigned i = (unsigned)hh;
    double ff = hh - (double)i;
    double p = v * (1.0 - s), q = v * (1.0 - s * ff), t = v * (1.0 - s * (1.0 - ff));
    switch (i) { case 0: return {v, t, p}; case 1: return {q, v, p}; case 2: return {p, v, t};
                 case 3: return {p, q, v}; case 4: return {t, p, v}; default: return {v, p, q}; }
}
__device__ __forceinline__ double curve_sample(const float* lut, double x) {
    // Linear filter, clamp-to-edge, read at u = (255x + 0.5)/256 (tonemap.wgsl:478-485).
    double t = clampd(x * 255.0, 0.0, 255.0);
    int i0 = (int)floor(t);
    int i1 = min(i0 + 1, 255);
    double fr = t - (double)i0;
    return (double)lut[i0] * (1.0 - fr) + (double)lut[i1] * fr;
}
__device__ __forceinline__ double smooth(double e0, double e1, double x) {
    double t = clampd((x - e0) / (e1 - e0), 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}

// AgX (Troy Sobotka's view transform, Benjamin Wrensch's minimal fit;
// tonemap.wgsl:444-477): into AgX's inset gamut, log2 encoded over
// [-12.47393, 4.026069] stops, the fit's sixth-order sigmoid, for the Punchy
// look a power of 1.35 and saturation 1.4 about Rec.709 luma, then the outset
// gamut, clamped, decoded by a power of 2.2.
__device__ D3 agx(D3 c, bool punchy) {
    D3 v{0.842479062253094 * c.x + 0.0784335999999992 * c.y + 0.0792237451477643 * c.z,
         0.0423282422610123 * c.x + 0.878468636469772 * c.y + 0.0791661274605434 * c.z,
         0.0423756549057051 * c.x + 0.0784336 * c.y + 0.879142973793104 * c.z};
    const double lo = -12.47393, hi = 4.026069;
    auto enc = [&](double x) {
        const double t = (clampd(log2(fmax(x, 1.0e-10)), lo, hi) - lo) / (hi - lo);
        const double t2 = t * t, t4 = t2 * t2;
        return 15.5 * t4 * t2 - 40.14 * t4 * t + 31.96 * t4 - 6.868 * t2 * t + 0.4298 * t2 + 0.1191 * t - 0.00232;
    };
    v = {enc(v.x), enc(v.y), enc(v.z)};
    if (punchy) {
        v = {pow(fmax(v.x, 0.0), 1.35), pow(fmax(v.y, 0.0), 1.35), pow(fmax(v.z, 0.0), 1.35)};
        const double l = 0.2126 * v.x + 0.7152 * v.y + 0.0722 * v.z;
        v = {l + 1.4 * (v.x - l), l + 1.4 * (v.y - l), l + 1.4 * (v.z - l)};
    }
    const D3 o{1.19687900512017 * v.x - 0.0980208811401368 * v.y - 0.0990297440797205 * v.z,
               -0.0528968517574562 * v.x + 1.15190312990417 * v.y - 0.0989611768448433 * v.z,
               -0.0529716355144438 * v.x - 0.0980434501171241 * v.y + 1.15107367264116 * v.z};
    return {pow(clampd(o.x, 0.0, 1.0), 2.2), pow(clampd(o.y, 0.0, 1.0), 2.2), pow(clampd(o.z, 0.0, 1.0), 2.2)};
}

// One pixel of the tone map: cnt = hits, sum = colour sums.  Returns the
// RGBA before quantisation.  Computed in FP64: the pass is bound by HBM
// (16 bytes in, 4 out a pixel), so the double arithmetic is free, and the
// ill-conditioned corners (HSV near grey, the gamma threshold blend) keep
// the result within 1e-5 of an exact evaluation.
__device__ D3 tonemap_rgb(const TonemapArgs& A, const float* lut, double cnt, D3 sum, double& fa_out) {
    D3 mean{0.0, 0.0, 0.0};
    if (cnt > 0.0) mean = {clampd(sum.x / cnt, 0.0, 1.0), clampd(sum.y / cnt, 0.0, 1.0), clampd(sum.z / cnt, 0.0, 1.0)};   // accumulate.wgsl:205-210
    const double bucket = cnt * 100.0;                                   // tonemap.wgsl:252
    D3 color;
    double alpha = 0.0;
    const double g = A.inv_gamma;
    if (A.mode == 0) {
        color = {pow(mean.x * A.exposure, g), pow(mean.y * A.exposure, g), pow(mean.z * A.exposure, g)};
        alpha = clampd(bucket * 0.01 * A.density_scale, 0.0, 1.0);
    } else if (A.mode == 2) {
        double nd = clampd(bucket * 0.01 * A.exposure, 0.0, 1.0);
        double gd = pow(nd, g);
        color = {gd, gd, gd};
        alpha = nd;
    } else {
        // brightness_scale (tonemap.wgsl:94-112), log10(1+x) through log1p.
        double ls = 0.0;
        if (!(bucket < 0.001)) ls = A.ls_a * log1p(A.ls_b * bucket) / (A.white_level * bucket);
        const double fp0 = ls * (mean.x * bucket), fp1 = ls * (mean.y * bucket), fp2 = ls * (mean.z * bucket);
        const double fp3 = ls * bucket * A.white_level;
        if (fp3 > 0.0) {
            if (fp3 <= A.gamma_threshold) {
                double fr = fp3 / A.gamma_threshold;
                alpha = (1.0 - fr) * fp3 * A.funcval + fr * pow(fp3, g);
            } else alpha = pow(fp3, g);
        }
        const double l2 = fp3 > 0.0 ? A.vib * alpha / fp3 : 0.0;
        if (A.notvib > 0.0)
            color = {l2 * fp0 + A.notvib * pow(fp0, g), l2 * fp1 + A.notvib * pow(fp1, g), l2 * fp2 + A.notvib * pow(fp2, g)};
        else
            color = {l2 * fp0, l2 * fp1, l2 * fp2};
    }
    if (A.saturation != 1.0 || A.hue_shift != 0.0) {                     // tonemap.wgsl:371-401
        D3 h = rgb_to_hsv(color);
        if (A.hue_shift != 0.0) { h.x += A.hue_shift; if (h.x < 0.0) h.x += 360.0; else if (h.x >= 360.0) h.x -= 360.0; }
        if (A.saturation != 1.0) h.y = clampd(h.y * A.saturation, 0.0, 1.0);
        color = hsv_to_rgb(h);
    }
    if (A.mode == 1) { color.x *= A.exposure; color.y *= A.exposure; color.z *= A.exposure; }
    color = {fmax(color.x, 0.0), fmax(color.y, 0.0), fmax(color.z, 0.0)};
    if (A.highlight == 1) {                                              // tonemap.wgsl:414-477
        double m = fmax(color.x, fmax(color.y, color.z));
        if (m > 1.0) color = {color.x / m, color.y / m, color.z / m};
    } else if (A.highlight == 2) {
        double lum = 0.2126 * color.x + 0.7152 * color.y + 0.0722 * color.z;
        if (lum > 1e-6) { double s = (lum / (1.0 + lum)) / lum; color = {color.x * s, color.y * s, color.z * s}; }
        color = {fmin(color.x, 1.0), fmin(color.y, 1.0), fmin(color.z, 1.0)};
    } else if (A.highlight == 3) {
        auto aces = [](double x) { return clampd((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0); };
        color = {aces(color.x), aces(color.y), aces(color.z)};
    } else if (A.highlight == 4 || A.highlight == 5) {
        color = agx(color, A.highlight == 5);
    } else {
        color = {fmin(color.x, 1.0), fmin(color.y, 1.0), fmin(color.z, 1.0)};
    }
    D3 fc = color;
    if (A.use_curve && bucket > 0.001)                                   // tonemap.wgsl:486-493
        fc = {curve_sample(lut, color.x), curve_sample(lut, color.y), curve_sample(lut, color.z)};
    double lev = 1.0;                                                    // apply_levels, tonemap.wgsl:124-149
    if (A.levels_density > 0.0) {
        double nd = cnt / (double)A.levels_density;
        if (A.levels_high <= A.levels_low) lev = nd > A.levels_low ? 1.0 : 0.0;
        else {
            double cl = clampd((nd - A.levels_low) / ((double)A.levels_high - A.levels_low), 0.0, 1.0);
            lev = (A.levels_gamma != 1.0f && A.levels_gamma > 0.0f) ? pow(cl, (double)A.levels_gamma) : cl;
        }
    }
    const double lin_a = clampd(bucket * 0.01 * A.density_scale, 0.0, 1.0);   // tonemap.wgsl:514-529
    const double gam_a = clampd(alpha, 0.0, 1.0);
    const double bt = smooth(A.alpha_blend_low, A.alpha_blend_high, gam_a);
    const double base_a = gam_a + (lin_a - gam_a) * bt;
    fa_out = A.levels_enabled ? fmin(base_a, lev) : base_a;
    return fc;
}

__device__ double4 tonemap_px(const TonemapArgs& A, const float* lut, double cnt, D3 sum) {
    double fa;
    const D3 fc = tonemap_rgb(A, lut, cnt, sum, fa);
    const double inv22 = 1.0 / 2.2;
    if (A.transparent != 0) {                                            // tonemap.wgsl:531-577
        D3 os = {pow(fmax(fc.x * fa, 0.0), inv22), pow(fmax(fc.y * fa, 0.0), inv22), pow(fmax(fc.z * fa, 0.0), inv22)};
        if (A.transparent == 2) return make_double4(os.x, os.y, os.z, fa);
        double cov = fmax(os.x, fmax(os.y, os.z));
        if (cov > 0.0) return make_double4(os.x / cov, os.y / cov, os.z / cov, cov);
        return make_double4(0.0, 0.0, 0.0, cov);
    }
    D3 f = {A.bg_lin[0] * (1.0 - fa) + fc.x * fa, A.bg_lin[1] * (1.0 - fa) + fc.y * fa, A.bg_lin[2] * (1.0 - fa) + fc.z * fa};
    return make_double4(pow(f.x, inv22), pow(f.y, inv22), pow(f.z, inv22), 1.0);   // tonemap.wgsl:582-589
}

__device__ __forceinline__ double hist_count(const TonemapArgs& A, const float4& v, size_t i) {
    if (A.count_is_float) return (double)v.w;
    if (A.exact) return (double)A.exact[i].w;
    return (double)__float_as_uint(v.w);
}
__device__ __forceinline__ D3 hist_rgb(const TonemapArgs& A, const float4& v, size_t i) {
    if (A.exact && !A.count_is_float) {
        const ulonglong4 e = A.exact[i];
        const double q = 1.0 / 16777216.0;
        return D3{(double)e.x * q, (double)e.y * q, (double)e.z * q};
    }
    return D3{v.x, v.y, v.z};
}

__device__ __forceinline__ uchar4 quantise(double4 o) {
    return make_uchar4((unsigned char)rint(clampd(o.x, 0.0, 1.0) * 255.0), (unsigned char)rint(clampd(o.y, 0.0, 1.0) * 255.0),
                       (unsigned char)rint(clampd(o.z, 0.0, 1.0) * 255.0), (unsigned char)rint(clampd(o.w, 0.0, 1.0) * 255.0));
}

__global__ void __launch_bounds__(256) k_tonemap1(const float4* __restrict__ hist, int n, TonemapArgs A, const float* __restrict__ lut_g,
                                                  uchar4* __restrict__ out, float4* __restrict__ out_f) {
    __shared__ float lut[256];
    lut[threadIdx.x] = lut_g[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = A.exact && !A.count_is_float ? make_float4(0.f, 0.f, 0.f, 0.f) : hist[i];
    const double4 o = tonemap_px(A, lut, hist_count(A, v, (size_t)i), hist_rgb(A, v, (size_t)i));
    out[i] = quantise(o);
    if (out_f) out_f[i] = make_float4((float)o.x, (float)o.y, (float)o.z, (float)o.w);
}

// 2x: tone map the four internal pixels of an output pixel, quantise each
// to 8 bits, then the firefly clamp and box (supersample.rs:132-167).
__device__ __forceinline__ uchar4 tonemap2_px(const TonemapArgs& A, const float* lut, const float4* __restrict__ hist, int wi, int ox, int oy) {
    float s[4][4], lum[4];
    const int dx[4] = {0, 1, 0, 1}, dy[4] = {0, 0, 1, 1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const size_t idx = (size_t)(oy * 2 + dy[k]) * wi + (ox * 2 + dx[k]);
        const float4 v = A.exact && !A.count_is_float ? make_float4(0.f, 0.f, 0.f, 0.f) : hist[idx];
        const uchar4 q = quantise(tonemap_px(A, lut, hist_count(A, v, idx), hist_rgb(A, v, idx)));
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
    return make_uchar4(r[0], r[1], r[2], r[3]);
}

__global__ void __launch_bounds__(256) k_tonemap2(const float4* __restrict__ hist, int wi, int ow, int oh, TonemapArgs A,
                                                  const float* __restrict__ lut_g, uchar4* __restrict__ out) {
    __shared__ float lut[256];
    lut[threadIdx.x] = lut_g[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ow * oh) return;
    out[i] = tonemap2_px(A, lut, hist, wi, i % ow, i / ow);
}

// Many flames in one launch: a grid-stride over the concatenated OUTPUT
// pixels of every flame, each finding its flame by binary search over px0.
__global__ void __launch_bounds__(256) k_tonemap_batch(const TonemapJob* __restrict__ jobs, int n_jobs, long long total) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_jobs - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].px0 <= g) lo = mid; else hi = mid - 1;
        }
        const TonemapJob& J = jobs[lo];
        const size_t i = (size_t)(g - J.px0);
        if (J.ss == 2) {
            const int ow = J.w / 2;
            reinterpret_cast<uchar4*>(J.out)[i] = tonemap2_px(J.a, J.lut, J.hist, J.w, (int)(i % ow), (int)(i / ow));
        } else {
            const float4 v = J.a.exact && !J.a.count_is_float ? make_float4(0.f, 0.f, 0.f, 0.f) : J.hist[i];
            const double4 o = tonemap_px(J.a, J.lut, hist_count(J.a, v, i), hist_rgb(J.a, v, i));
            reinterpret_cast<uchar4*>(J.out)[i] = quantise(o);
        }
    }
}

// Density estimation, gather form: output pixel p sums, over sources q in
// the (2R+1)^2 window, w(|p-q|, count_q) * (rgb_q, count_q).  Each block
// stages its 32x16 tile's source window in shared memory once, with every
// source's table entry resolved (its accepted d^2, 4.5/h^2, and its values
// premultiplied by the normaliser), so a neighbour outside its disc costs
// one 8-byte shared load and a compare; and the window shrinks to the
// largest radius any staged source actually has (dense regions, where
// every count is high, gather over a few pixels only).
constexpr int DE_TX = 32, DE_TY = 16;
__global__ void __launch_bounds__(DE_TX * DE_TY) k_density(const float4* __restrict__ hist, const ulonglong4* __restrict__ exact,
                                                           int w, int h, const float4* __restrict__ tab,
                                                           int tab_n, int R, int y_lo, int h_out, float4* __restrict__ out,
                                                           int count_f) {
    extern __shared__ float4 de_smem[];
    const int tw = DE_TX + 2 * R, th = DE_TY + 2 * R, n = tw * th;
    float4* val = de_smem;                                                // (rgb, count) / normaliser
    float2* par = reinterpret_cast<float2*>(de_smem + n);                 // (accepted d^2, 4.5 / h^2)
    __shared__ int reach;
    if (threadIdx.x == 0) reach = 0;
    __syncthreads();
    const int x0 = blockIdx.x * DE_TX - R, y0 = y_lo + blockIdx.y * DE_TY - R;
    int my_reach = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int sx = x0 + i % tw, sy = y0 + i / tw;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 pr = make_float2(-1.0f, 0.0f);                              // empty: never accepted
        if (sx >= 0 && sy >= 0 && sx < w && sy < h) {
            const size_t si = (size_t)sy * w + sx;
            float4 hv;
            unsigned long long c;
            if (exact) {
                const ulonglong4 q = exact[si];
                c = q.w;
                const double f = 1.0 / 16777216.0;
                hv = make_float4((float)((double)q.x * f), (float)((double)q.y * f), (float)((double)q.z * f), 0.f);
            } else {
                hv = hist[si];
                // A filtered histogram holds fractional counts: the table
                // entry of the count rounded up, the count itself as weight.
                c = count_f ? (unsigned long long)ceilf(fmaxf(hv.w, 0.0f)) : (unsigned long long)__float_as_uint(hv.w);
            }
            if (c > 0ull) {
                const float4 e = tab[c < (unsigned long long)(tab_n - 1) ? c : (unsigned long long)(tab_n - 1)];
                const float cf = count_f ? hv.w : (float)c;
                v = make_float4(hv.x * e.z, hv.y * e.z, hv.z * e.z, cf * e.z);
                pr = make_float2(e.x, 4.5f * e.y);
                my_reach = max(my_reach, (int)e.w);
            }
        }
        val[i] = v;
        par[i] = pr;
    }
    atomicMax(&reach, my_reach);
    __syncthreads();
    const int rb = min(R, reach);
    const int lx = threadIdx.x % DE_TX, ly = threadIdx.x / DE_TX;
    const int px = blockIdx.x * DE_TX + lx, py = y_lo + blockIdx.y * DE_TY + ly;
    if (px >= w || py >= h || py >= y_lo + h_out) return;
    float ar = 0.f, ag = 0.f, ab = 0.f, ac = 0.f;
    for (int dy = -rb; dy <= rb; ++dy) {
        const int row = (ly + R + dy) * tw + (lx + R);
        for (int dx = -rb; dx <= rb; ++dx) {
            const float2 pp = par[row + dx];
            const float d2 = (float)(dx * dx + dy * dy);
            if (d2 > pp.x) continue;
            const float wt = __expf(-pp.y * d2);
            const float4 v = val[row + dx];
            ar += wt * v.x; ag += wt * v.y; ab += wt * v.z; ac += wt * v.w;
        }
    }
    out[(size_t)(py - y_lo) * w + px] = make_float4(ar, ag, ab, ac);
}

// Histogram planes for a collective: AoS (r, g, b, count bits) <-> a u32
// count plane and an f32 (r, g, b) plane, each summable by NCCL in its own type.
__global__ void k_pack(const float4* __restrict__ hist, size_t n, unsigned* __restrict__ cnt, float* __restrict__ rgb) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float4 v = hist[i];
        cnt[i] = __float_as_uint(v.w);
        rgb[3 * i] = v.x; rgb[3 * i + 1] = v.y; rgb[3 * i + 2] = v.z;
    }
}
__global__ void k_unpack(const unsigned* __restrict__ cnt, const float* __restrict__ rgb, size_t n, float4* __restrict__ hist) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        hist[i] = make_float4(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], __uint_as_float(cnt[i]));
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

cudaError_t launch_tonemap_batch(const TonemapJob* jobs, int n_jobs, long long total_px, cudaStream_t s) {
    k_tonemap_batch<<<148 * 16, 256, 0, s>>>(jobs, n_jobs, total_px);
    return cudaGetLastError();
}

cudaError_t launch_density_estimate(const float4* hist, const ulonglong4* exact, int w, int h,
                                    const float4* table, int table_n, int radius, int y_lo, int h_out, float4* out, cudaStream_t s,
                                    int count_f) {
    const size_t smem = (size_t)(DE_TX + 2 * radius) * (DE_TY + 2 * radius) * (sizeof(float4) + sizeof(float2));
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_density, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((w + DE_TX - 1) / DE_TX, (h_out + DE_TY - 1) / DE_TY);
    k_density<<<grid, DE_TX * DE_TY, smem, s>>>(hist, exact, w, h, table, table_n, radius, y_lo, h_out, out, count_f);
    return cudaGetLastError();
}

// The spatial filter (shaders/histogram_blur.wgsl:38-119): one separable
// pass of a bilateral Gaussian, spatial sigma `sigma` pixels (taps within
// min(ceil(3 sigma), 8), clamped to the edge), density sigma `sigma_d`
// (weight exp(-(d_tap - d_centre)^2 / 2 sigma_d^2)); the centre density of
// both passes is the batch's unfiltered one (`orig`).  dir 0 filters rows,
// 1 columns.  `src_u32`/`orig_u32`: .w holds u32 count bits, else a float.
// `accumulate`: add the result into `dst` (count as float) instead of
// storing it.  Counts and colours stay FP32 (the reference truncates its
// x100 fixed-point values to u32 after each pass).
__global__ void __launch_bounds__(256) k_hist_filter(const float4* __restrict__ src, int src_u32, const float4* __restrict__ orig,
                                                     int orig_u32, int w, int h, int dir, float sigma, float sigma_d,
                                                     float4* __restrict__ dst, int accumulate) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= w || y >= h) return;
    const float sg = fmaxf(sigma, 0.0001f);
    const int kh = min((int)ceilf(3.0f * sg), 8);
    const float inv_2s2 = 1.0f / (2.0f * sg * sg);
    const size_t c = (size_t)y * w + x;
    const float4 oc = orig[c];
    const float dc = orig_u32 ? (float)__float_as_uint(oc.w) : oc.w;
    const float sd = fmaxf(sigma_d, 0.01f);
    const float inv_2sd2 = 1.0f / (2.0f * sd * sd);
    float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
    float wt = 0.0f;
    for (int k = -kh; k <= kh; ++k) {
        const int nx = dir == 0 ? min(max(x + k, 0), w - 1) : x;
        const int ny = dir == 0 ? y : min(max(y + k, 0), h - 1);
        const float4 t = src[(size_t)ny * w + nx];
        const float td = src_u32 ? (float)__float_as_uint(t.w) : t.w;
        const float fk = (float)k;
        const float ws = expf(-fk * fk * inv_2s2);
        const float dd = td - dc;
        const float wd = expf(-dd * dd * inv_2sd2);
        const float wk = ws * wd;
        sum.x += t.x * wk; sum.y += t.y * wk; sum.z += t.z * wk; sum.w += td * wk;
        wt += wk;
    }
    const float inv = 1.0f / fmaxf(wt, 1e-6f);
    const float4 r = make_float4(sum.x * inv, sum.y * inv, sum.z * inv, sum.w * inv);
    if (accumulate) {
        float4 a = dst[c];
        a.x += r.x; a.y += r.y; a.z += r.z; a.w += r.w;
        dst[c] = a;
    } else {
        dst[c] = r;
    }
}

cudaError_t launch_hist_filter(const float4* batch, float4* tmp, float4* acc, int w, int h, float sigma, float sigma_d,
                               cudaStream_t s) {
    const dim3 grid((w + 255) / 256, h);
    k_hist_filter<<<grid, 256, 0, s>>>(batch, 1, batch, 1, w, h, 0, sigma, sigma_d, tmp, 0);
    k_hist_filter<<<grid, 256, 0, s>>>(tmp, 0, batch, 1, w, h, 1, sigma, sigma_d, acc, 1);
    return cudaGetLastError();
}

cudaError_t launch_pack(const float4* hist, size_t n, unsigned* cnt, float* rgb, cudaStream_t s) {
    k_pack<<<148 * 8, 256, 0, s>>>(hist, n, cnt, rgb);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const unsigned* cnt, const float* rgb, size_t n, float4* hist, cudaStream_t s) {
    k_unpack<<<148 * 8, 256, 0, s>>>(cnt, rgb, n, hist);
    return cudaGetLastError();
}

cudaError_t launch_atomic_bench(uint32_t* buf, uint32_t n_pixels, uint64_t n_samples, int kind, int blocks, cudaStream_t s) {
    k_atomic_bench<<<blocks, 256, 0, s>>>(buf, n_pixels, n_samples, kind);
    return cudaGetLastError();
}

// ---- density estimation without allocation ---------------------------------
//
// Some callers cannot allocate device memory while they render. Examples: an
// application that hands the whole device to its own memory pool and must
// account for every byte; a host framework whose allocator must not be bypassed;
// a frame loop that has fixed its memory at start-up and may not grow it.
// The density-estimation gather needs one buffer besides its input and output:
// the weight table. This variant keeps that table in a file-scope device array
// with a fixed maximum, not in memory allocated per call.
//
// * The array holds kDeStaticEntries entries (1 MiB). A table that needs more
//   is refused before any work is queued. The table's length grows as
//   max_radius^(1/curve); min_radius > 0 shortens it.
// * Set-up: the first call on a device, with that device current, looks up
//   the array's device address (cudaGetSymbolAddress) and keeps it for later
//   calls on that device. That first call should come before any stream
//   capture. The kept address belongs to the device's context at set-up: if
//   that context is destroyed and another made (cudaDeviceReset, or a primary
//   context released and retained again), the next call sees the new
//   context's id and looks the address up again.
// * Every call on a device shares the one array. Calls whose work overlaps on
//   the GPU race on it: two streams, or a call queued while another's DE
//   kernel has not yet run. Order them on one stream or with events.
// * Nothing in the array has to start at zero: each call writes every entry
//   its DE kernel reads, earlier on the same stream.
// * The table is computed on the host, in the same double arithmetic as the
//   allocating path. It reaches the device in launch parameters (chunks of
//   kDeChunk entries), so no memcpy or staging buffer is involved.

static __device__ __align__(256) float4 g_de_scratch[kDeStaticEntries];

namespace {

constexpr int kMaxDevices = 64;
constexpr int kDeChunk = 1024;                 // 16 KiB of launch parameters a chunk

struct DeChunk { float4 e[kDeChunk]; };

__global__ void k_de_store(const __grid_constant__ DeChunk c, int n, float4* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = c.e[i];
}

std::mutex g_de_static_mu;
struct DeStaticSlot {
    unsigned long long ctx_id = 0;   // the context the address belongs to (0: none yet)
    float4* ptr = nullptr;
};
DeStaticSlot g_de_static[kMaxDevices];

// The unique id of the calling thread's current context (0 when none is
// current), through the driver's entry points so this library needs no link
// to libcuda.  Ids are never reused within a process, unlike context handles.
unsigned long long current_context_id() {
    typedef int (*GetCurrent)(void**);
    typedef int (*GetId)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess) get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess) get_id = (GetId)f;
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

cudaError_t de_static_scratch(float4** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_de_static_mu);
    DeStaticSlot& slot = g_de_static[dev];
    unsigned long long id = current_context_id();
    if (!slot.ptr || id == 0 || id != slot.ctx_id) {
        float4* ptr = nullptr;
        e = cudaGetSymbolAddress((void**)&ptr, g_de_scratch);   // makes the device's primary context current if none is
        if (e != cudaSuccess) return e;
        slot.ptr = ptr;
        slot.ctx_id = id ? id : current_context_id();
    }
    *out = slot.ptr;
    return cudaSuccess;
}

// Entry c of the DE table: (max accepted d^2, 1/h^2, 1/normaliser, reach),
// h(c) = max(min_radius, max_radius / c^curve), weights exp(-4.5 d^2 / h^2)
// over integer offsets with d^2 <= h^2; count 0 has no disc.
float4 de_entry(int c, double r_max, double r_min, double curve) {
    const double h = c == 0 ? 0.0 : std::max(r_min, r_max / std::pow((double)c, curve));
    const double h2 = h * h;
    const double dmax2 = c == 0 ? -1.0 : std::floor(h2);
    const int rr = (int)std::floor(std::sqrt(std::max(dmax2, 0.0)));
    double norm = 0.0;
    for (int dy = -rr; dy <= rr; ++dy)
        for (int dx = -rr; dx <= rr; ++dx) {
            const double d2 = dx * dx + dy * dy;
            if (d2 <= h2) norm += std::exp(-4.5 * d2 / h2);
        }
    if (c == 0) norm = 1.0;
    return make_float4((float)dmax2, h2 > 0 ? (float)(1.0 / h2) : 0.0f, (float)(1.0 / norm), (float)rr);
}

}  // namespace

int de_static_entries(double r_max, double r_min, double curve) {
    // Entries 0..c; the table ends at the first c >= 1 whose disc is below a
    // pixel or at the minimum radius (every larger count shares it).
    for (int c = 1;; ++c) {
        const double h = std::max(r_min, r_max / std::pow((double)c, curve));
        if (h < 1.0 || h <= r_min) return c + 1;
        if (c + 2 > kDeStaticEntries) return -1;
    }
}

cudaError_t density_estimate_static(const float4* hist, int w, int h, double r_max, double r_min, double curve,
                                    float4* out, cudaStream_t s) {
    const int n = de_static_entries(r_max, r_min, curve);
    if (n < 0) return cudaErrorInvalidValue;
    float4* tab = nullptr;
    cudaError_t e = de_static_scratch(&tab);
    if (e != cudaSuccess) return e;
    DeChunk chunk;
    for (int c0 = 0; c0 < n; c0 += kDeChunk) {
        const int m = std::min(kDeChunk, n - c0);
        for (int j = 0; j < m; ++j) chunk.e[j] = de_entry(c0 + j, r_max, r_min, curve);
        k_de_store<<<(m + 255) / 256, 256, 0, s>>>(chunk, m, tab + c0);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return launch_density_estimate(hist, nullptr, w, h, tab, n, (int)std::floor(r_max), 0, h, out, s, 0);
}

}  // namespace ffb
