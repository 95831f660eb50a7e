// ffb_diff_tail.cu -- the differentiable render's tone map (ahead-of-time
// sm_100a kernels).
//
// The log-density tone map of ffb_tail.cu (tonemap.wgsl:94-590: log
// brightness, gamma with its threshold blend, vibrancy, clip, curve LUT,
// levels, alpha blend, background) in FP32, returned in linear light (the
// display encode pow(., 1/2.2) is left out: its slope is unbounded at black)
// with alpha 1.  The vector-Jacobian product evaluates the same function on
// dual numbers carrying the derivatives with respect to the pixel's four
// histogram channels (r, g, b sums, weight), so forward and backward share
// one definition.  The sample density comes from the forward pass's device
// counter, so neither pass waits for the host.  HBM-bound: 16 B in and 16 B
// out a pixel forward, 32 B in and 16 B out backward.

#include "ffb_tail.cuh"

#include <algorithm>

namespace ffb {

namespace {

struct DF {
    float v, d[4];
};
__device__ __forceinline__ DF dfc(float c) { return DF{c, {0.f, 0.f, 0.f, 0.f}}; }
__device__ __forceinline__ DF operator+(DF a, DF b) { return DF{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2], a.d[3] + b.d[3]}}; }
__device__ __forceinline__ DF operator-(DF a, DF b) { return DF{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2], a.d[3] - b.d[3]}}; }
__device__ __forceinline__ DF operator*(DF a, DF b) {
    return DF{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2], a.d[3] * b.v + a.v * b.d[3]}};
}
__device__ __forceinline__ DF operator/(DF a, DF b) {
    const float q = a.v / b.v, ib = 1.0f / b.v;
    return DF{q, {(a.d[0] - q * b.d[0]) * ib, (a.d[1] - q * b.d[1]) * ib, (a.d[2] - q * b.d[2]) * ib, (a.d[3] - q * b.d[3]) * ib}};
}
__device__ __forceinline__ DF operator*(DF a, float s) { return DF{a.v * s, {a.d[0] * s, a.d[1] * s, a.d[2] * s, a.d[3] * s}}; }
__device__ __forceinline__ DF operator*(float s, DF a) { return a * s; }
__device__ __forceinline__ DF operator-(float s, DF a) { return DF{s - a.v, {-a.d[0], -a.d[1], -a.d[2], -a.d[3]}}; }
__device__ __forceinline__ DF operator/(DF a, float s) { return a * (1.0f / s); }
__device__ __forceinline__ DF chain(DF a, float v, float dv) { return DF{v, {a.d[0] * dv, a.d[1] * dv, a.d[2] * dv, a.d[3] * dv}}; }

__device__ __forceinline__ float val(float x) { return x; }
__device__ __forceinline__ float val(DF x) { return x.v; }
template <class S> __device__ __forceinline__ S cst(float c);
template <> __device__ __forceinline__ float cst<float>(float c) { return c; }
template <> __device__ __forceinline__ DF cst<DF>(float c) { return dfc(c); }

__device__ __forceinline__ float log1p_s(float x) { return log1pf(x); }
__device__ __forceinline__ DF log1p_s(DF x) { return chain(x, log1pf(x.v), 1.0f / (1.0f + x.v)); }
// x^g for x > 0, 0 (and slope 0) otherwise.
__device__ __forceinline__ float pow_s(float x, float g) { return x > 0.0f ? powf(x, g) : 0.0f; }
__device__ __forceinline__ DF pow_s(DF x, float g) {
    if (!(x.v > 0.0f)) return dfc(0.0f);
    const float p = powf(x.v, g);
    return chain(x, p, g * p / x.v);
}
template <class S> __device__ __forceinline__ S clamp_s(S x, float lo, float hi) {
    if (val(x) < lo) return cst<S>(lo);
    if (val(x) > hi) return cst<S>(hi);
    return x;
}
template <class S> __device__ __forceinline__ S min_s(S a, S b) { return val(b) < val(a) ? b : a; }
template <class S> __device__ __forceinline__ S smooth_s(float e0, float e1, S x) {
    S t = clamp_s<S>((x - cst<S>(e0)) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
// Curve LUT: linear filter, clamp-to-edge (tonemap.wgsl:478-493).
template <class S> __device__ __forceinline__ S curve_s(const float* lut, S x) {
    const float t = fminf(fmaxf(val(x) * 255.0f, 0.0f), 255.0f);
    const int i0 = (int)floorf(t), i1 = min(i0 + 1, 255);
    const float fr = t - (float)i0;
    const float v = lut[i0] * (1.0f - fr) + lut[i1] * fr;
    const bool inside = val(x) * 255.0f > 0.0f && val(x) * 255.0f < 255.0f;
    if constexpr (sizeof(S) == sizeof(float)) return v;
    else return chain(x, v, inside ? (lut[i1] - lut[i0]) * 255.0f : 0.0f);
}

// One pixel: histogram (r, g, b sums, weight) -> linear-light rgb.
template <class S>
__device__ __forceinline__ void dtm_px(const TonemapArgs& A, const float* lut, float ls_b, float lev_d, S r, S g, S b, S cnt,
                                       S out[3]) {
    S m[3] = {cst<S>(0.f), cst<S>(0.f), cst<S>(0.f)};
    if (val(cnt) > 0.0f) { m[0] = clamp_s<S>(r / cnt, 0.f, 1.f); m[1] = clamp_s<S>(g / cnt, 0.f, 1.f); m[2] = clamp_s<S>(b / cnt, 0.f, 1.f); }
    const S bucket = cnt * 100.0f;
    S ls = cst<S>(0.f);
    if (!(val(bucket) < 0.001f)) ls = A.ls_a * log1p_s(ls_b * bucket) / (A.white_level * bucket);
    S fp[3] = {ls * (m[0] * bucket), ls * (m[1] * bucket), ls * (m[2] * bucket)};
    const S fp3 = ls * bucket * A.white_level;
    const float gma = A.inv_gamma;
    S alpha = cst<S>(0.f);
    if (val(fp3) > 0.0f) {
        if (val(fp3) <= A.gamma_threshold) {
            const S fr = fp3 / A.gamma_threshold;
            alpha = (1.0f - fr) * fp3 * A.funcval + fr * pow_s(fp3, gma);
        } else alpha = pow_s(fp3, gma);
    }
    const S l2 = val(fp3) > 0.0f ? A.vib * alpha / fp3 : cst<S>(0.f);
    S col[3];
    for (int c = 0; c < 3; ++c) {
        col[c] = A.notvib > 0.0f ? l2 * fp[c] + A.notvib * pow_s(fp[c], gma) : l2 * fp[c];
        col[c] = col[c] * A.exposure;
        if (val(col[c]) < 0.0f) col[c] = cst<S>(0.f);
        if (val(col[c]) > 1.0f) col[c] = cst<S>(1.f);
        if (A.use_curve && val(bucket) > 0.001f) col[c] = curve_s<S>(lut, col[c]);
    }
    S lev = cst<S>(1.f);
    if (lev_d > 0.0f) {
        const S nd = cnt / lev_d;
        if (A.levels_high <= A.levels_low) lev = cst<S>(val(nd) > A.levels_low ? 1.f : 0.f);
        else {
            const S cl = clamp_s<S>((nd - cst<S>(A.levels_low)) / (A.levels_high - A.levels_low), 0.f, 1.f);
            lev = (A.levels_gamma != 1.0f && A.levels_gamma > 0.0f) ? pow_s(cl, A.levels_gamma) : cl;
        }
    }
    const S lin_a = clamp_s<S>(bucket * (0.01f * A.density_scale), 0.f, 1.f);
    const S gam_a = clamp_s<S>(alpha, 0.f, 1.f);
    const S bt = smooth_s<S>(A.alpha_blend_low, A.alpha_blend_high, gam_a);
    const S base = gam_a + (lin_a - gam_a) * bt;
    const S fa = A.levels_enabled ? min_s<S>(base, lev) : base;
    for (int c = 0; c < 3; ++c) out[c] = A.bg_lin[c] * (1.0f - fa) + col[c] * fa;
}

struct DensityArgs {
    const unsigned long long* samples;   // plotted samples of the forward pass
    double npx, area, white;
};

__device__ __forceinline__ void density_consts(const DensityArgs& D, float& ls_b, float& lev_d) {
    // tonemap_args' k2 and levels density, from the device sample count.
    const double sd = fmax((double)D.samples[0] / D.npx, 1e-6);
    const double k2 = 1.0 / (D.area * D.white * sd);
    ls_b = (float)(D.white * k2);
    lev_d = (float)sd;
}

__global__ void k_diff_tonemap(const float4* __restrict__ hist, size_t n, TonemapArgs A, const float* __restrict__ lut_g,
                               DensityArgs D, float4* __restrict__ out) {
    __shared__ float lut[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    float ls_b, lev_d;
    density_consts(D, ls_b, lev_d);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float4 h = hist[i];
        float o[3];
        dtm_px<float>(A, lut, ls_b, lev_d, h.x, h.y, h.z, h.w, o);
        out[i] = make_float4(o[0], o[1], o[2], 1.0f);
    }
}

__global__ void k_diff_tonemap_vjp(const float4* __restrict__ hist, const float4* __restrict__ dimg, size_t n, TonemapArgs A,
                                   const float* __restrict__ lut_g, DensityArgs D, float4* __restrict__ dh) {
    __shared__ float lut[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    float ls_b, lev_d;
    density_consts(D, ls_b, lev_d);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float4 h = hist[i], g = dimg[i];
        DF r{h.x, {1.f, 0.f, 0.f, 0.f}}, gg{h.y, {0.f, 1.f, 0.f, 0.f}}, b{h.z, {0.f, 0.f, 1.f, 0.f}}, c{h.w, {0.f, 0.f, 0.f, 1.f}};
        DF o[3];
        dtm_px<DF>(A, lut, ls_b, lev_d, r, gg, b, c, o);
        float4 v;
        v.x = g.x * o[0].d[0] + g.y * o[1].d[0] + g.z * o[2].d[0];
        v.y = g.x * o[0].d[1] + g.y * o[1].d[1] + g.z * o[2].d[1];
        v.z = g.x * o[0].d[2] + g.y * o[1].d[2] + g.z * o[2].d[2];
        v.w = g.x * o[0].d[3] + g.y * o[1].d[3] + g.z * o[2].d[3];
        dh[i] = v;
    }
}

__global__ void k_fixed_to_float(const ulonglong4* __restrict__ fx, size_t n, float4* __restrict__ out) {
    const double s = 2.3283064365386963e-10;              // 2^-32
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const ulonglong4 v = fx[i];
        out[i] = make_float4((float)((double)v.x * s), (float)((double)v.y * s), (float)((double)v.z * s), (float)((double)v.w * s));
    }
}

}  // namespace

cudaError_t launch_fixed_to_float(const ulonglong4* fx, size_t n, float4* out, cudaStream_t s) {
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_fixed_to_float<<<blocks, 256, 0, s>>>(fx, n, out);
    return cudaGetLastError();
}

cudaError_t launch_diff_tonemap(const float4* hist, size_t n, const TonemapArgs& a, const float* lut, const uint64_t* samples,
                                double npx, double area, double white, float4* out, cudaStream_t s) {
    DensityArgs D{(const unsigned long long*)samples, npx, area, white};
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_diff_tonemap<<<blocks, 256, 0, s>>>(hist, n, a, lut, D, out);
    return cudaGetLastError();
}

cudaError_t launch_diff_tonemap_vjp(const float4* hist, const float4* dimg, size_t n, const TonemapArgs& a, const float* lut,
                                    const uint64_t* samples, double npx, double area, double white, float4* dh, cudaStream_t s) {
    DensityArgs D{(const unsigned long long*)samples, npx, area, white};
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_diff_tonemap_vjp<<<blocks, 256, 0, s>>>(hist, dimg, n, a, lut, D, dh);
    return cudaGetLastError();
}

}  // namespace ffb
