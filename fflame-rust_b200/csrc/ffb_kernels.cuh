// ffb_kernels.cuh -- the chaos-game kernels, compiled per flame structure
// by NVRTC after ffb_device.cuh and the generated ffb_normal / ffb_finals.

// One flame in a launch.  A launch covers jobs[0..n_jobs); job j owns
// blocks [block0, block0 + ceil(n_walkers / blockDim)).
struct ffb_launch {
    const float* table;        // FFB_TABLE_SIZE floats
    const float4* palette;     // pal_n entries: linear rgb, 1
    float4* hist;              // width*height: (r sum, g sum, b sum, count bits)
    float4* walkers;           // n_walkers: (x, y, colour index, fuse bits)
    u64* counters;             // [0] in-frame splats
    u32 n_walkers, walker0, block0, n_xf;
    u32 seed_lo, seed_hi, burn_in, ipt;
    u64 it0;
    u32 n_iters, pal_n;
    int width, height;
    float zoom, pan_x, pan_y, cos_r, sin_r;
};

__device__ __forceinline__ int ffb_select(const float* __restrict__ sm, int n_xf, float u) {
    // utilities.wgsl:35-54: first i with u*total <= cumsum_i (f32, left to right).
    const float t = u * sm[T_TOTAL];
    int k = n_xf - 1;
    bool found = false;
#pragma unroll
    for (int i = 0; i < FFB_MAXX; ++i) {
        bool hit = (i < n_xf) && !found && (t <= sm[T_CUM + i]);
        k = hit ? i : k;
        found = found || hit;
    }
    return k;
}

__device__ __forceinline__ int ffb_palette_index(float ci, u32 n) {
    // Nearest sampling, clamp-to-edge (gpu/buffers.rs:1867-1876).
    float t = floorf(ci * (float)n);
    if (!(t >= 0.0f)) return 0;
    if (t > (float)(n - 1)) return (int)n - 1;
    return (int)t;
}

// Splat one sample: exact u32 count, FP32 colour sums.
__device__ __forceinline__ void ffb_splat(float4* __restrict__ hist, u32 idx, float4 c) {
    float* p = reinterpret_cast<float*>(hist + idx);
    atomicAdd(p + 0, c.x);
    atomicAdd(p + 1, c.y);
    atomicAdd(p + 2, c.z);
    atomicAdd(reinterpret_cast<u32*>(p + 3), 1u);
}

extern "C" __global__ void __launch_bounds__(FFB_THREADS)
ffb_chaos(const ffb_launch* __restrict__ jobs, int n_jobs) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    // The job owning this block (block-uniform binary search).
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].block0 <= blockIdx.x) lo = mid; else hi = mid - 1;
    }
    const ffb_launch& J = jobs[lo];
    for (int i = threadIdx.x; i < FFB_TABLE_SIZE; i += blockDim.x) sm[i] = J.table[i];
    float4* pal = ffb_smem4 + FFB_TABLE_VEC4;
    for (u32 i = threadIdx.x; i < J.pal_n; i += blockDim.x) pal[i] = J.palette[i];
    __syncthreads();

    const u32 w = (blockIdx.x - J.block0) * blockDim.x + threadIdx.x;
    if (w >= J.n_walkers) return;
    const u32 gw = J.walker0 + w;
    const int n_xf = (int)J.n_xf;
    float x, y, ci;
    u32 fuse;
    const u64 it0 = J.it0, it1 = J.it0 + J.n_iters;
    if (it0 == 0) {
        ci = 0.0f;
        fuse = J.burn_in;
#if FFB_RNG_MODE == 1
        uint4 o = philox4(J.seed_lo, J.seed_hi, gw, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        x = u24(o.x) * 2.0f - 1.0f;
        y = u24(o.y) * 2.0f - 1.0f;
#else
        x = 0.0f; y = 0.0f;   // drawn at it == 0 below
#endif
    } else {
        float4 s = J.walkers[w];
        x = s.x; y = s.y; ci = s.z; fuse = __float_as_uint(s.w);
    }
    const float scale = (float)min(J.width, J.height) * 0.25f;
    const float cx = (float)J.width * 0.5f, cy = (float)J.height * 0.5f;
    u32 inframe = 0;
#if FFB_RNG_MODE == 0
    PcgRng rng;
    rng.state = 0; rng.inc = 1;
#endif
    for (u64 it = it0; it < it1; ++it) {
#if FFB_RNG_MODE == 0
        // A dispatch boundary: the stream is re-seeded per dispatch and the
        // two start draws are consumed before the orbit resumes
        // (main_template.wgsl:25-55, 125-181; compute_kernel.rs:3541-3553).
        if (it == it0 || (J.ipt != 0 && it % J.ipt == 0)) {
            u32 d = J.ipt ? (u32)(it / J.ipt) : 0u;
            rng.init(gw, J.seed_lo + d * 2654435761u);
            float s0 = rng.draw(0), s1 = rng.draw(0);
            if (it == 0) { x = s0 * 2.0f - 1.0f; y = s1 * 2.0f - 1.0f; }
        }
#else
        PhiloxRng rng;
        rng.fill(J.seed_lo, J.seed_hi, gw, it);
#endif
        const int k = ffb_select(sm, n_xf, rng.draw(0));                     // main_template.wgsl:198-223
        const bool plot = rng.draw(1) < sm[T_XF + F_OPAC * FFB_MAXX + k];       // main_template.wgsl:249
        const float* q = sm + T_XF + k;
        float ax = q[F_A * FFB_MAXX] * x + q[F_B * FFB_MAXX] * y + q[F_E * FFB_MAXX];
        float ay = q[F_C * FFB_MAXX] * x + q[F_D * FFB_MAXX] * y + q[F_F * FFB_MAXX];
        ffb_normal(sm, k, ax, ay, rng);                                         // main_template.wgsl:366-376
#if FFB_HAS_POST
        if (q[F_POST * FFB_MAXX] > 0.5f) {                                      // main_template.wgsl:380-384
            float px = q[F_PA * FFB_MAXX] * ax + q[F_PB * FFB_MAXX] * ay + q[F_PE * FFB_MAXX];
            float py = q[F_PC * FFB_MAXX] * ax + q[F_PD * FFB_MAXX] * ay + q[F_PF * FFB_MAXX];
            ax = px; ay = py;
        }
#endif
        if (!(fabsf(ax) <= 1e32f) || !(fabsf(ay) <= 1e32f)) {                  // main_template.wgsl:449-479
#if FFB_RNG_MODE == 1
            uint4 o = philox4(J.seed_lo, J.seed_hi, gw, (u32)it, 0xFFFFFFFFu, (u32)(it >> 32));
            x = u24(o.x) * 2.0f - 1.0f;
            y = u24(o.y) * 2.0f - 1.0f;
#else
            x = rng.draw(0) * 2.0f - 1.0f;
            y = rng.draw(0) * 2.0f - 1.0f;
#endif
            fuse = J.burn_in;
            continue;
        }
        x = ax; y = ay;
        ci = ci * q[F_C1 * FFB_MAXX] + q[F_C2 * FFB_MAXX];                       // main_template.wgsl:496-508
        if (fuse > 0u) { fuse -= 1u; continue; }                               // main_template.wgsl:510-514
        float fx = x, fy = y;
        ffb_finals(sm, fx, fy, rng);                                            // main_template.wgsl:663-717
        const float4 c = pal[ffb_palette_index(ci, J.pal_n)];                   // main_template.wgsl:766-772
        // world_to_pixel (utilities.wgsl:417-450).
        float tx = fx - J.pan_x, ty = fy - J.pan_y;
        float rx = tx * J.cos_r - ty * J.sin_r;
        float ry = tx * J.sin_r + ty * J.cos_r;
        rx = rx * J.zoom; ry = ry * J.zoom;
        const float pxf = floorf(cx + rx * scale), pyf = floorf(cy + ry * scale);
        if (plot && pxf >= 0.0f && pyf >= 0.0f && pxf < (float)J.width && pyf < (float)J.height) {
            const u32 idx = (u32)pyf * (u32)J.width + (u32)pxf;
            ffb_splat(J.hist, idx, c);
            ++inframe;
        }
    }
    J.walkers[w] = make_float4(x, y, ci, __uint_as_float(fuse));
    // In-frame splat count (count conservation: sum of the count plane).
    // Lanes past n_walkers have returned, so reduce over the live ones.
    const unsigned live = __activemask();
    const u32 tot = __reduce_add_sync(live, inframe);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(live) - 1) && tot) atomicAdd(J.counters, (u64)tot);
}

// The variation probe (main_template.wgsl:1467-1567): transform xi's
// apply_variations at point pi, slot = xi*npts + pi, the RNG seeded
// rng_init(slot, 0x9E3779B9); the affine is not applied.  Finals (xi >=
// n_xf) run their whole chain step.
extern "C" __global__ void ffb_probe(const float* __restrict__ table, int n_xf, int n_all, const float2* __restrict__ pts,
                                     int npts, float2* __restrict__ out) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n_all * npts) return;
    const int xi = slot / npts, pi = slot % npts;
    float x = pts[pi].x, y = pts[pi].y;
    if (fabsf(x) < 1.17549435e-38f) x = copysignf(0.0f, x);
    if (fabsf(y) < 1.17549435e-38f) y = copysignf(0.0f, y);
    PcgRng rng;
    rng.init((u32)slot, 0x9E3779B9u);
    if (xi < n_xf) ffb_normal(table, xi, x, y, rng);
    else ffb_final_one(table, xi - n_xf, x, y, rng, false);
    out[slot] = make_float2(x, y);
}

// Single-step parity: transform xi (affine, variations, post) at n points
// with given draw words (16 a point).  xi >= n_xf selects final xi - n_xf.
extern "C" __global__ void ffb_apply_points(const float* __restrict__ table, int n_xf, int xi, int n,
                                            const float* __restrict__ xs, const float* __restrict__ ys,
                                            const float* __restrict__ words, int with_affine,
                                            float* __restrict__ xo, float* __restrict__ yo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ArrayRng rng{words + (size_t)i * 16};
    float x = xs[i], y = ys[i];
    if (xi < n_xf) {
        const float* q = table + T_XF + xi;
        if (with_affine) {
            float ax = q[F_A * FFB_MAXX] * x + q[F_B * FFB_MAXX] * y + q[F_E * FFB_MAXX];
            float ay = q[F_C * FFB_MAXX] * x + q[F_D * FFB_MAXX] * y + q[F_F * FFB_MAXX];
            x = ax; y = ay;
        }
        ffb_normal(table, xi, x, y, rng);
        if (with_affine && q[F_POST * FFB_MAXX] > 0.5f) {
            float px = q[F_PA * FFB_MAXX] * x + q[F_PB * FFB_MAXX] * y + q[F_PE * FFB_MAXX];
            float py = q[F_PC * FFB_MAXX] * x + q[F_PD * FFB_MAXX] * y + q[F_PF * FFB_MAXX];
            x = px; y = py;
        }
    } else {
        ffb_final_one(table, xi - n_xf, x, y, rng, with_affine != 0);
    }
    xo[i] = x; yo[i] = y;
}
