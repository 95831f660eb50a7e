// ffb_diff.cuh -- the differentiable render's chaos-game kernels, compiled
// per flame structure by NVRTC after ffb_device.cuh, ffb_kernels.cuh,
// ffb_diff_jac.cuh and the generated ffb_normal / ffb_dnormal.
//
// An addition beside the reference's render (which has no gradients):
//   * forward: the chaos game of ffb_chaos (Philox stream) with a bilinear
//     splat at the un-floored pixel coordinate minus one half and the palette
//     sampled with linear interpolation between texel centres, so the
//     histogram is piecewise-smooth in the parameters; each walker's state is
//     checkpointed every FFB_CKPT iterations;
//   * adjoint: each walker re-runs one checkpoint interval at a time, last to
//     first, and walks it backwards.  Every plotted sample is differentiated
//     through the FFB_WINDOW iterations ending with the one that produced it
//     (transform choices held fixed): a sliding window of FFB_WINDOW adjoints
//     lives in registers, the sum of the window feeds the parameter gradient
//     of each step, and each adjoint is carried back through the step's
//     Jacobian until it leaves the window.  Parameter gradients accumulate in
//     a thread-private column of shared memory (no atomics), reduced per
//     block and added to the global gradient in double.
//
// Parameters (theta): [n_xf*6 affine a, b, c, d, e, f | n_xf*FFB_NVN
// variation weights, transform-major | n_xf colours].

struct ffb_diff_args {
    const float* table;          // FFB_TABLE_SIZE floats (theta applied)
    const float4* palette;       // pal_n: linear rgb, 1
    float4* hist;                // width*height: r, g, b sums, weight
    float4* ckpt;                // n_ckpt * n_walkers: x, y, colour index, fuse bits
    const float4* dh;            // dL/dhist, width*height
    double* grad;                // theta layout
    u64* counters;               // [0] plotted samples, [1] in-frame samples
    ulonglong4* fixed;           // if not null: deterministic accumulation (r, g, b, weight in 2^-32 units) instead of hist
    u32 n_walkers, walker0, n_xf, pal_n;
    u32 seed_lo, seed_hi, burn_in, n_iters;
    int width, height;
    float zoom, pan_x, pan_y, cos_r, sin_r;
};

enum { DS_RESPAWN = 1u << 8, DS_PLOTTED = 1u << 9, DS_SAMPLE = 1u << 10 };

// One iteration once transform k is picked: affine, variations, post,
// bad-value respawn, colour, fuse (ffb_step without finals and splat).
// Returns k | flags.
__device__ __forceinline__ u32 ffb_dstep(const float* __restrict__ sm, const ffb_diff_args& A, int k, bool plot,
                                         PhiloxRng& rng, u32 gw, u64 it, float& x, float& y, float& ci, u32& fuse) {
    const float* q = sm + T_XF + k;
    float ax = q[F_A * FFB_MAXX] * x + q[F_B * FFB_MAXX] * y + q[F_E * FFB_MAXX];
    float ay = q[F_C * FFB_MAXX] * x + q[F_D * FFB_MAXX] * y + q[F_F * FFB_MAXX];
    ffb_normal(sm, k, ax, ay, rng);
#if FFB_HAS_POST
    if (q[F_POST * FFB_MAXX] > 0.5f) {
        float px = q[F_PA * FFB_MAXX] * ax + q[F_PB * FFB_MAXX] * ay + q[F_PE * FFB_MAXX];
        float py = q[F_PC * FFB_MAXX] * ax + q[F_PD * FFB_MAXX] * ay + q[F_PF * FFB_MAXX];
        ax = px; ay = py;
    }
#endif
    if (!(fabsf(ax) <= 1e32f) || !(fabsf(ay) <= 1e32f)) {
        uint4 o = philox4(A.seed_lo, A.seed_hi, gw, (u32)it, 0xFFFFFFFFu, (u32)(it >> 32));
        x = u24(o.x) * 2.0f - 1.0f;
        y = u24(o.y) * 2.0f - 1.0f;
        fuse = A.burn_in;
        return (u32)k | DS_RESPAWN;
    }
    x = ax; y = ay;
    ci = ci * q[F_C1 * FFB_MAXX] + q[F_C2 * FFB_MAXX];
    if (fuse > 0u) { fuse -= 1u; return (u32)k; }
    return (u32)k | DS_PLOTTED | (plot ? DS_SAMPLE : 0u);
}

// The bilinear footprint's origin and fractions: u = world_to_pixel's
// continuous x minus 0.5 (the same float operations as the oracle).
__device__ __forceinline__ bool ffb_dcam(const ffb_diff_args& A, float x, float y, float& u, float& v) {
    const float scale = (float)min(A.width, A.height) * 0.25f;
    const float cx = (float)A.width * 0.5f, cy = (float)A.height * 0.5f;
    float tx = x - A.pan_x, ty = y - A.pan_y;
    float rx = tx * A.cos_r - ty * A.sin_r;
    float ry = tx * A.sin_r + ty * A.cos_r;
    rx = rx * A.zoom; ry = ry * A.zoom;
    u = (cx + rx * scale) - 0.5f;
    v = (cy + ry * scale) - 0.5f;
    return u > -1.0f && u < (float)A.width && v > -1.0f && v < (float)A.height;
}

// Palette sampled with linear interpolation between texel centres (clamped
// at the ends): colour and d colour / d index.
__device__ __forceinline__ void ffb_dpal(const float4* __restrict__ pal, u32 n, float ci, float3& col, float3& dcol) {
    const float t = ci * (float)n - 0.5f;
    int i0 = 0;
    float fr = 0.0f;
    bool inside = false;
    if (!(t > 0.0f)) i0 = 0;
    else if (t >= (float)(n - 1)) i0 = (int)n - 1;
    else { i0 = (int)floorf(t); fr = t - (float)i0; inside = true; }
    const int i1 = min(i0 + 1, (int)n - 1);
    const float4 p0 = pal[i0], p1 = pal[i1];
    col = make_float3(p0.x * (1.0f - fr) + p1.x * fr, p0.y * (1.0f - fr) + p1.y * fr, p0.z * (1.0f - fr) + p1.z * fr);
    const float sc = inside ? (float)n : 0.0f;
    dcol = make_float3((p1.x - p0.x) * sc, (p1.y - p0.y) * sc, (p1.z - p0.z) * sc);
}

__device__ __forceinline__ void ffb_red4(float4* p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

__device__ __forceinline__ void ffb_dstage(const ffb_diff_args& A, float* sm, float4*& pal) {
    for (int i = threadIdx.x; i < FFB_TABLE_SIZE; i += blockDim.x) sm[i] = A.table[i];
    pal = reinterpret_cast<float4*>(sm) + FFB_TABLE_VEC4;
    for (u32 i = threadIdx.x; i < A.pal_n; i += blockDim.x) pal[i] = A.palette[i];
}

__device__ __forceinline__ void ffb_dstart(const ffb_diff_args& A, u32 gw, float& x, float& y) {
    uint4 o = philox4(A.seed_lo, A.seed_hi, gw, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
    x = u24(o.x) * 2.0f - 1.0f;
    y = u24(o.y) * 2.0f - 1.0f;
}

// Forward: one walker a thread, all iterations.
extern "C" __global__ void __launch_bounds__(FFB_THREADS) ffb_diff_forward(const ffb_diff_args A) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    float4* pal;
    ffb_dstage(A, sm, pal);
    __syncthreads();
    const u32 w = blockIdx.x * blockDim.x + threadIdx.x;
    u32 plotted = 0, inframe = 0;
    if (w < A.n_walkers) {
        const u32 gw = A.walker0 + w;
        float x, y, ci = 0.0f;
        u32 fuse = A.burn_in;
        ffb_dstart(A, gw, x, y);
        for (u32 it = 0; it < A.n_iters; ++it) {
            if (it % FFB_CKPT == 0u) A.ckpt[(size_t)(it / FFB_CKPT) * A.n_walkers + w] = make_float4(x, y, ci, __uint_as_float(fuse));
            PhiloxRng rng;
            rng.fill(A.seed_lo, A.seed_hi, gw, it);
            const int k = ffb_select(sm, (int)A.n_xf, rng.draw(0));
            const bool plot = rng.draw(1) < sm[T_XF + F_OPAC * FFB_MAXX + k];
            const u32 fl = ffb_dstep(sm, A, k, plot, rng, gw, it, x, y, ci, fuse);
            plotted += (fl & DS_PLOTTED) ? 1u : 0u;
            if (!(fl & DS_SAMPLE)) continue;
            float u, v;
            if (!ffb_dcam(A, x, y, u, v)) continue;
            float3 col, dcol;
            ffb_dpal(pal, A.pal_n, ci, col, dcol);
            const float fu = floorf(u), fv = floorf(v);
            const int i0 = (int)fu, j0 = (int)fv;
            const float fx = u - fu, fy = v - fv, gx = 1.0f - fx, gy = 1.0f - fy;
            const float wgt[4] = {gx * gy, fx * gy, gx * fy, fx * fy};
            ++inframe;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int i = i0 + (c & 1), j = j0 + (c >> 1);
                if (i < 0 || j < 0 || i >= A.width || j >= A.height) continue;
                const size_t idx = (size_t)j * A.width + i;
                if (A.fixed) {
                    // Integer sums: the same bits whatever the atomics' order.
                    unsigned long long* p = reinterpret_cast<unsigned long long*>(A.fixed + idx);
                    atomicAdd(p + 0, __float2ull_rn(wgt[c] * col.x * 4294967296.0f));
                    atomicAdd(p + 1, __float2ull_rn(wgt[c] * col.y * 4294967296.0f));
                    atomicAdd(p + 2, __float2ull_rn(wgt[c] * col.z * 4294967296.0f));
                    atomicAdd(p + 3, __float2ull_rn(wgt[c] * 4294967296.0f));
                } else {
                    ffb_red4(A.hist + idx, wgt[c] * col.x, wgt[c] * col.y, wgt[c] * col.z, wgt[c]);
                }
            }
        }
    }
    const unsigned live = __activemask();
    const u32 tp = __reduce_add_sync(live, plotted), ti = __reduce_add_sync(live, inframe);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(live) - 1)) {
        if (tp) atomicAdd(A.counters, (u64)tp);
        if (ti) atomicAdd(A.counters + 1, (u64)ti);
    }
}

// Index of parameter p of the shared-memory gradient layout in theta:
// [MAXX*6 affine | MAXX*NVN weights | MAXX colours] -> theta's n_xf layout.
__device__ __forceinline__ int ffb_dparam_index(int p, int n_xf) {
    if (p < FFB_MAXX * 6) { const int k = p / 6; return k < n_xf ? p : -1; }
    p -= FFB_MAXX * 6;
    if (p < FFB_MAXX * FFB_NVN) { const int k = p / FFB_NVN; return k < n_xf ? n_xf * 6 + p : -1; }
    p -= FFB_MAXX * FFB_NVN;
    return p < n_xf ? n_xf * (6 + FFB_NVN) + p : -1;
}

// Adjoint: one walker a thread.
extern "C" __global__ void __launch_bounds__(FFB_THREADS) ffb_diff_adjoint(const ffb_diff_args A) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    float4* pal;
    ffb_dstage(A, sm, pal);
    const int P = blockDim.x, tid = threadIdx.x;
    float* s_grad = reinterpret_cast<float*>(pal + A.pal_n);         // [FFB_NPARAM][P]
    float* gt = s_grad + tid;
    for (int p = 0; p < FFB_NPARAM; ++p) gt[p * P] = 0.0f;
    __syncthreads();
    const u32 w = blockIdx.x * P + tid;
    if (w < A.n_walkers) {
        const u32 gw = A.walker0 + w;
        const float zs = A.zoom * ((float)min(A.width, A.height) * 0.25f);
        float rx[FFB_WINDOW], ry[FFB_WINDOW], rc[FFB_WINDOW];
#pragma unroll
        for (int r = 0; r < FFB_WINDOW; ++r) { rx[r] = 0.0f; ry[r] = 0.0f; rc[r] = 0.0f; }
        int since = FFB_WINDOW;                          // steps since the newest adjoint entered the window
        float4 loc[FFB_CKPT];
        const int n_seg = (int)((A.n_iters + FFB_CKPT - 1) / FFB_CKPT);
        for (int seg = n_seg - 1; seg >= 0; --seg) {
            const u32 it0 = (u32)seg * FFB_CKPT;
            const int n = (int)min((u32)FFB_CKPT, A.n_iters - it0);
            const float4 st = A.ckpt[(size_t)seg * A.n_walkers + w];
            {
                float x = st.x, y = st.y, ci = st.z;
                u32 fuse = __float_as_uint(st.w);
                for (int i = 0; i < n; ++i) {
                    const u32 it = it0 + (u32)i;
                    PhiloxRng rng;
                    rng.fill(A.seed_lo, A.seed_hi, gw, it);
                    const int k = ffb_select(sm, (int)A.n_xf, rng.draw(0));
                    const bool plot = rng.draw(1) < sm[T_XF + F_OPAC * FFB_MAXX + k];
                    const u32 fl = ffb_dstep(sm, A, k, plot, rng, gw, it, x, y, ci, fuse);
                    loc[i] = make_float4(x, y, ci, __uint_as_float(fl));
                }
            }
            for (int i = n - 1; i >= 0; --i) {
                const float4 post = loc[i];
                const float px = i > 0 ? loc[i - 1].x : st.x, py = i > 0 ? loc[i - 1].y : st.y;
                const u32 fl = __float_as_uint(post.w);
                const int k = (int)(fl & 0xFFu);
                // The window slides one step: the oldest adjoint leaves, this
                // step's sample (if any) enters.
#pragma unroll
                for (int r = FFB_WINDOW - 1; r > 0; --r) { rx[r] = rx[r - 1]; ry[r] = ry[r - 1]; rc[r] = rc[r - 1]; }
                rx[0] = 0.0f; ry[0] = 0.0f; rc[0] = 0.0f;
                ++since;
                float u, v;
                if ((fl & DS_SAMPLE) && ffb_dcam(A, post.x, post.y, u, v)) {
                    float3 col, dcol;
                    ffb_dpal(pal, A.pal_n, post.z, col, dcol);
                    const float fu = floorf(u), fv = floorf(v);
                    const int i0 = (int)fu, j0 = (int)fv;
                    const float fx = u - fu, fy = v - fv, gx = 1.0f - fx, gy = 1.0f - fy;
                    const float wgt[4] = {gx * gy, fx * gy, gx * fy, fx * fy};
                    float sc[4], dci = 0.0f;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int ii = i0 + (c & 1), jj = j0 + (c >> 1);
                        sc[c] = 0.0f;
                        if (ii < 0 || jj < 0 || ii >= A.width || jj >= A.height) continue;
                        const float4 G = A.dh[(size_t)jj * A.width + ii];
                        sc[c] = G.x * col.x + G.y * col.y + G.z * col.z + G.w;
                        dci += wgt[c] * (G.x * dcol.x + G.y * dcol.y + G.z * dcol.z);
                    }
                    const float dfx = -gy * sc[0] + gy * sc[1] - fy * sc[2] + fy * sc[3];
                    const float dfy = -gx * sc[0] - fx * sc[1] + gx * sc[2] + fx * sc[3];
                    rx[0] = zs * (A.cos_r * dfx + A.sin_r * dfy);
                    ry[0] = zs * (-A.sin_r * dfx + A.cos_r * dfy);
                    rc[0] = dci;
                    since = 0;
                }
                if (since >= FFB_WINDOW) continue;              // the window is empty
                if (fl & DS_RESPAWN) {
                    // The new point does not depend on the old one or on theta;
                    // the colour index is not updated on this step.
#pragma unroll
                    for (int r = 0; r < FFB_WINDOW; ++r) { rx[r] = 0.0f; ry[r] = 0.0f; }
                    continue;
                }
                float lx = 0.0f, ly = 0.0f, mc = 0.0f;
#pragma unroll
                for (int r = 0; r < FFB_WINDOW; ++r) { lx += rx[r]; ly += ry[r]; mc += rc[r]; }
                const float* q = sm + T_XF + k;
                const float a = q[F_A * FFB_MAXX], b = q[F_B * FFB_MAXX], c = q[F_C * FFB_MAXX], d = q[F_D * FFB_MAXX];
                const float qx = a * px + b * py + q[F_E * FFB_MAXX];
                const float qy = c * px + d * py + q[F_F * FFB_MAXX];
                // Adjoint at the variations' output (through the post affine).
                float p00 = 1.0f, p01 = 0.0f, p10 = 0.0f, p11 = 1.0f;
#if FFB_HAS_POST
                if (q[F_POST * FFB_MAXX] > 0.5f) {
                    p00 = q[F_PA * FFB_MAXX]; p01 = q[F_PB * FFB_MAXX]; p10 = q[F_PC * FFB_MAXX]; p11 = q[F_PD * FFB_MAXX];
                }
#endif
                const float ax = p00 * lx + p10 * ly, ay = p01 * lx + p11 * ly;
                PhiloxRng rng;
#if FFB_NSLOTS > 2
                rng.fill(A.seed_lo, A.seed_hi, gw, it0 + (u32)i);
#endif
                float4 J;
                ffb_dnormal(sm, k, qx, qy, rng, ax, ay, gt + (FFB_MAXX * 6 + k * FFB_NVN) * P, P, J);
                const float ux = J.x * ax + J.z * ay, uy = J.y * ax + J.w * ay;   // J^T (ax, ay)
                float* ga = gt + (k * 6) * P;
                ga[0] += ux * px; ga[P] += ux * py; ga[2 * P] += uy * px; ga[3 * P] += uy * py; ga[4 * P] += ux; ga[5 * P] += uy;
                gt[(FFB_MAXX * (6 + FFB_NVN) + k) * P] += mc * (1.0f - q[F_C1 * FFB_MAXX]);   // d ci / d colour = (1 - speed) / 2
                // M^T = A^T J^T P^T carries every adjoint in the window back one step.
                const float j00 = J.x * p00 + J.z * p10, j01 = J.x * p01 + J.z * p11;   // (P J)^T rows
                const float j10 = J.y * p00 + J.w * p10, j11 = J.y * p01 + J.w * p11;
                const float m00 = a * j00 + c * j10, m01 = a * j01 + c * j11;
                const float m10 = b * j00 + d * j10, m11 = b * j01 + d * j11;
                const float c1 = q[F_C1 * FFB_MAXX];
#pragma unroll
                for (int r = 0; r < FFB_WINDOW; ++r) {
                    const float nx = m00 * rx[r] + m01 * ry[r];
                    const float ny = m10 * rx[r] + m11 * ry[r];
                    rx[r] = nx; ry[r] = ny; rc[r] *= c1;
                }
            }
        }
    }
    __syncthreads();
    for (int p = tid; p < FFB_NPARAM; p += P) {
        const int gi = ffb_dparam_index(p, (int)A.n_xf);
        if (gi < 0) continue;
        float s = 0.0f;
        const float* col = s_grad + p * P;
        for (int t = 0; t < P; ++t) s += col[t];
        if (s != 0.0f) atomicAdd(A.grad + gi, (double)s);
    }
}

// Theta into the coefficient table: affine, variation weights and the
// colour term color * (1 - speed) / 2 of each normal transform.
// oms[k] = 1 - speed_k.  One block.
extern "C" __global__ void ffb_diff_theta(const float* __restrict__ theta, const float* __restrict__ base,
                                          const float* __restrict__ oms, float* __restrict__ table, int n_xf) {
    for (int i = threadIdx.x; i < FFB_TABLE_SIZE; i += blockDim.x) table[i] = base[i];
    __syncthreads();
    for (int i = threadIdx.x; i < n_xf * 6; i += blockDim.x) {
        const int k = i / 6, f = i % 6;
        table[T_XF + f * FFB_MAXX + k] = theta[i];
    }
    for (int i = threadIdx.x; i < n_xf * FFB_NVN; i += blockDim.x) {
        const int k = i / FFB_NVN, j = i % FFB_NVN;
        table[T_VW + j * FFB_MAXX + k] = theta[n_xf * 6 + i];
    }
    for (int k = threadIdx.x; k < n_xf; k += blockDim.x)
        table[T_XF + F_C2 * FFB_MAXX + k] = theta[n_xf * (6 + FFB_NVN) + k] * oms[k] / 2.0f;
}

// Each normal variation's value and Jacobian at n points for transform k:
// out[(p * FFB_NVN + j) * 6 ..] = (vx, vy, J).  Draw words as ffb_apply_points.
extern "C" __global__ void ffb_dprobe(const float* __restrict__ table, int k, int n, const float* __restrict__ xs,
                                      const float* __restrict__ ys, const float* __restrict__ words, float* __restrict__ out) {
    __shared__ float sm[FFB_TABLE_SIZE];
    for (int i = threadIdx.x; i < FFB_TABLE_SIZE; i += blockDim.x) sm[i] = table[i];
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    ArrayRng rng{words + (size_t)p * FFB_APPLY_WORDS};
    for (int j = 0; j < FFB_NVN; ++j) {
        float vx, vy;
        float4 J;
        ffb_dvar_one(sm, j, k, xs[p], ys[p], rng, vx, vy, J);
        float* o = out + ((size_t)p * FFB_NVN + j) * 6;
        o[0] = vx; o[1] = vy; o[2] = J.x; o[3] = J.y; o[4] = J.z; o[5] = J.w;
    }
}
