// ffb_kernels.cuh -- the chaos-game kernels, compiled per flame structure
// by NVRTC after ffb_device.cuh and the generated ffb_normal / ffb_finals.

// One flame in a launch.  A launch covers jobs[0..n_jobs); job j owns
// blocks [block0, block0 + ceil(n_walkers / blockDim)).
struct ffb_launch {
    const float* table;        // FFB_TABLE_SIZE floats
    const float4* palette;     // pal_n entries: linear rgb, 1
    void* hist;                // width*height: float4 (r, g, b sums, count bits); exact mode: ulonglong4 (r, g, b, count)
    float4* walkers;           // n_walkers: (x, y, colour index, fuse bits)
    u64* counters;             // [0] in-frame splats
    u32 n_walkers, walker0, block0, n_xf;
    u32 seed_lo, seed_hi, burn_in, ipt;
    u64 it0;
    u32 n_iters, pal_n;
    int width, height;
    float zoom, pan_x, pan_y, cos_r, sin_r;
    float4* rec;               // deferred plotting: n_iters x n_walkers samples (x, y, ci, flags)
    float* rec_draws;          // and their final chain's draws, FFB_NFD planes of the same length
    float* state;              // FFB_NSTATE planes of n_walkers: the walkers' variation state (slot-major)
    u32 ring_prod, ring_depth; // fused plotting: producer threads a block, iteration slots of the ring
};

// The walker context of walker gw at iteration it.
__device__ __forceinline__ FfbCtx ffb_ctx(const ffb_launch& J, u32 gw, u64 it) {
    FfbCtx c;
    c.st = J.state + (gw - J.walker0);
    c.stride = J.n_walkers;
    c.vc = 0.0f;
    c.k0 = J.seed_lo; c.k1 = J.seed_hi; c.gw = gw; c.it = it;
    return c;
}

#if FFB_NSTATE > 0
// A starting walker's variation state: zero (var<private> thread_state,
// main_template.wgsl:117-122), then each `wgsl_state_init` that draws --
// klein_group's previous generator, floor(r * 4) (klein_group_misc.rs:227-231).
// With the reference's stream the draw is taken at every dispatch start
// (ffb_pcg_dispatch); with the counter-based stream it is Philox counter
// (walker, 0xFFFFFFFE, entry / 4 + 256 d, 0xFFFFFFFF) for a walker (re)started
// at dispatch d.
__device__ __forceinline__ void ffb_state_fresh(const float* __restrict__ sm, const ffb_launch& J, u32 gw, u32 d = 0u) {
    float* st = J.state + (gw - J.walker0);
    for (int s = 0; s < FFB_NSTATE; ++s) st[(size_t)s * J.n_walkers] = 0.0f;
#ifdef FFB_SPEED
    for (int s = 0; s < 3; ++s) st[(size_t)(FFB_SPEED_SLOT + s) * J.n_walkers] = 1.0f;   // main_template.wgsl:43
#endif
#if FFB_RNG_MODE == 1
    for (int i = 0; i < FFB_NINIT; ++i) {
        const uint4 o = philox4(J.seed_lo, J.seed_hi, gw, 0xFFFFFFFEu, (u32)(i >> 2) | (d << 8), 0xFFFFFFFFu);
        const u32 wd = (i & 3) == 0 ? o.x : (i & 3) == 1 ? o.y : (i & 3) == 2 ? o.z : o.w;
        st[(size_t)ffb_u32(sm[T_INIT + i]) * J.n_walkers] = floorf(u24(wd) * 4.0f);
    }
#else
    (void)sm; (void)d;
#endif
}
#endif

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

#ifdef FFB_XAOS
// Xaos (utilities.wgsl:106-137): the pick from the previous transform's
// row, whose running sums of weight_i x xaos[prev][i] (f32, left to right)
// and total the table holds at T_XAOS + prev * (FFB_MAXX + 1).
__device__ __forceinline__ int ffb_select_xaos(const float* __restrict__ sm, int n_xf, float u, int prev) {
    const float* row = sm + T_XAOS + prev * (FFB_MAXX + 1);
    const float t = u * row[0];
    int k = n_xf - 1;
    bool found = false;
#pragma unroll
    for (int i = 0; i < FFB_MAXX; ++i) {
        bool hit = (i < n_xf) && !found && (t <= row[1 + i]);
        k = hit ? i : k;
        found = found || hit;
    }
    return k;
}
// A starting walker's previous transform (main_template.wgsl:163-179): an
// unconditioned pick at a Kronecker point of its index, so every range of
// walkers starts in each closed group of the chain in proportion.
__device__ __forceinline__ int ffb_xaos_first(const float* __restrict__ sm, int n_xf, u32 gw, u32 seed) {
    const u32 ou = gw * 2654435769u + seed;
    return ffb_select(sm, n_xf, (float)(ou >> 8u) * (1.0f / 16777216.0f));
}
#define FFB_PICK(u, prev) ffb_select_xaos(sm, n_xf, (u), (prev))
// The stored walker state packs the previous transform above the burn-in left.
#define FFB_PACK_FUSE(fuse, prev) ((fuse) | ((u32)(prev) << 24))
#else
#define FFB_PICK(u, prev) ffb_select(sm, n_xf, (u))
#define FFB_PACK_FUSE(fuse, prev) (fuse)
#endif

__device__ __forceinline__ int ffb_palette_index(float ci, u32 n) {
    // Nearest sampling, clamp-to-edge (gpu/buffers.rs:1867-1876).
    float t = floorf(ci * (float)n);
    if (!(t >= 0.0f)) return 0;
    if (t > (float)(n - 1)) return (int)n - 1;
    return (int)t;
}

// Splat one sample: exact u32 count, FP32 colour sums.  Warp-aggregated:
// the lanes of a warp splatting the same pixel with the same palette entry
// find each other (__match_any_sync on a 64-bit key) and their lowest lane
// adds n * colour and n once, so a hot pixel (an attractor's fixed point)
// costs one atomic per warp instead of one per lane.  A lone lane adds
// exactly what it would have alone.
//
// Exact mode (FFB_EXACT): the pixel is four u64 (r, g, b, count), colour in
// 24-bit fixed point (round(c * 2^24) a sample): integer sums, exact to
// 2^40 hits a pixel and independent of the order of the atomics.
__device__ __forceinline__ void ffb_splat(void* __restrict__ hist_v, u32 idx, float4 c, int pal_idx) {
#ifdef FFB_NO_AGGREGATION
    const u32 n = 1u;
    const bool lead = true;
#else
    const unsigned live = __activemask();
    const unsigned long long key = ((unsigned long long)idx << 16) | (unsigned)pal_idx;
    const unsigned peers = __match_any_sync(live, key);
    const bool lead = (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1);
    const u32 n = __popc(peers);
#endif
    if (!lead) return;
#ifdef FFB_EXACT
    unsigned long long* p = reinterpret_cast<unsigned long long*>(reinterpret_cast<ulonglong4*>(hist_v) + idx);
    const unsigned long long nn = n;
    atomicAdd(p + 0, nn * (unsigned long long)__float2uint_rn(c.x * 16777216.0f));
    atomicAdd(p + 1, nn * (unsigned long long)__float2uint_rn(c.y * 16777216.0f));
    atomicAdd(p + 2, nn * (unsigned long long)__float2uint_rn(c.z * 16777216.0f));
    atomicAdd(p + 3, nn);
#else
    float* p = reinterpret_cast<float*>(reinterpret_cast<float4*>(hist_v) + idx);
    if (n == 1u) {
        atomicAdd(p + 0, c.x);
        atomicAdd(p + 1, c.y);
        atomicAdd(p + 2, c.z);
    } else {
        const float fn = (float)n;
        atomicAdd(p + 0, fn * c.x);
        atomicAdd(p + 1, fn * c.y);
        atomicAdd(p + 2, fn * c.z);
    }
    atomicAdd(reinterpret_cast<u32*>(p + 3), n);
#endif
}

#ifdef FFB_EMIT
// Tile-sorted accumulation, first stage: instead of the splat, each sample
// becomes a record (pixel index | palette index << 32).  Block b owns
// segment b of the launch's record buffer (`hist`): threads x iterations x
// symmetry copies records, as many as its walkers can produce, behind a
// cursor in shared memory that each warp advances once for all its lanes;
// the block's count follows the segments (ffb_emit_finish).  A record past
// the segment (impossible by its size) sets counters[3].
__shared__ u32 ffb_s_emit;

__device__ __forceinline__ u64 ffb_seg_cap(const ffb_launch& J, u32 copies) {
    return (u64)blockDim.x * J.n_iters * copies;
}

__device__ __forceinline__ void ffb_emit(const ffb_launch& J, bool valid, u32 idx, int pal_idx, u32 copies) {
    const unsigned live = __activemask();
    const unsigned m = __ballot_sync(live, valid);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(live) - 1;
    u32 base = 0;
    if (lane == leader) base = atomicAdd(&ffb_s_emit, (u32)__popc(m));
    base = __shfl_sync(live, base, leader);
    if (valid) {
        const u64 cap = ffb_seg_cap(J, copies);
        const u64 slot = (u64)base + (u64)__popc(m & ((1u << lane) - 1u));
        if (slot < cap) reinterpret_cast<u64*>(J.hist)[(u64)blockIdx.x * cap + slot] = (u64)idx | ((u64)pal_idx << 32);
        else atomicOr(reinterpret_cast<unsigned int*>(J.counters + 3), 1u);
    }
}

// Every thread of the block: the block's record count after the segments.
__device__ __forceinline__ void ffb_emit_finish(const ffb_launch& J, u32 copies) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const u64 cap = ffb_seg_cap(J, copies);
        u32* counts = reinterpret_cast<u32*>(reinterpret_cast<u64*>(J.hist) + (u64)gridDim.x * cap);
        counts[blockIdx.x] = (u32)min((u64)ffb_s_emit, cap);
    }
}
#endif

__device__ __forceinline__ u32 ffb_copies(const float* __restrict__ sm) {
#if FFB_SYM_KIND != 0
    return (u32)sm[T_SYM];
#else
    return 1u;
#endif
}

// The job owning this block (block-uniform binary search) and its tables
// staged in shared memory.  The launch record itself stays in global
// memory: its fields are block-uniform, read-only loads (a copy in shared
// memory measured 4-8 % slower walkers).
__device__ __forceinline__ const ffb_launch& ffb_stage(const ffb_launch* __restrict__ jobs, int n_jobs, float* sm, float4*& pal) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].block0 <= blockIdx.x) lo = mid; else hi = mid - 1;
    }
    const ffb_launch& J = jobs[lo];
    for (int i = threadIdx.x; i < FFB_TABLE_SIZE; i += blockDim.x) sm[i] = J.table[i];
    pal = reinterpret_cast<float4*>(sm) + FFB_TABLE_VEC4;
    for (u32 i = threadIdx.x; i < J.pal_n; i += blockDim.x) pal[i] = J.palette[i];
#ifdef FFB_EMIT
    if (threadIdx.x == 0) ffb_s_emit = 0u;
#endif
    __syncthreads();
    return J;
}

// A walker's start (main_template.wgsl:25-55) or its stored state; `prev`
// the previous transform of an xaos walk.
__device__ __forceinline__ void ffb_start(const float* __restrict__ sm, const ffb_launch& J, u32 w, u32 gw, float& x, float& y,
                                          float& ci, u32& fuse, int& prev) {
    prev = 0;
    if (J.it0 == 0) {
        ci = 0.0f;
        fuse = J.burn_in;
#if FFB_NSTATE > 0
        ffb_state_fresh(sm, J, gw);
#endif
#ifdef FFB_XAOS
        prev = ffb_xaos_first(sm, (int)J.n_xf, gw, J.seed_lo);
#endif
#if FFB_RNG_MODE == 1
        uint4 o = philox4(J.seed_lo, J.seed_hi, gw, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        x = u24(o.x) * 2.0f - 1.0f;
        y = u24(o.y) * 2.0f - 1.0f;
#else
        x = 0.0f; y = 0.0f;   // drawn at it == 0 by ffb_pcg_dispatch
#endif
    } else {
        float4 s = J.walkers[w];
        x = s.x; y = s.y; ci = s.z; fuse = __float_as_uint(s.w);
#ifdef FFB_XAOS
        prev = (int)(fuse >> 24);
        fuse &= 0xFFFFFFu;
#endif
    }
}

#if FFB_RNG_MODE == 0
// A dispatch boundary of the reference's stream: re-seeded per dispatch, the
// two start draws consumed before the orbit resumes (main_template.wgsl:25-55,
// 125-181; compute_kernel.rs:3541-3553).
__device__ __forceinline__ void ffb_pcg_dispatch(const float* __restrict__ sm, const ffb_launch& J, PcgRng& rng, u32 gw, u64 it,
                                                 float& x, float& y, float& ci, u32& fuse, int& prev) {
    if (it == J.it0 || (J.ipt != 0 && it % J.ipt == 0)) {
        u32 d = J.ipt ? (u32)(it / J.ipt) : 0u;
        const u32 seed_d = J.seed_lo + d * 2654435761u;
        rng.init(gw, seed_d);
        float s0 = rng.draw(0), s1 = rng.draw(0);
        bool fresh = it == 0;
#ifdef FFB_REFRESH
        // Orbit refresh (main_template.wgsl:125-145, compute_kernel.rs:45-60):
        // this dispatch starts the walkers w with (w + seed) % period == 0
        // again -- point from the start draws, colour 0, burn-in, the
        // stratified first pick, fresh state.
        if (!fresh && J.ipt != 0 && it % J.ipt == 0 && (gw + seed_d) % (u32)FFB_REFRESH == 0u) {
            fresh = true;
            ci = 0.0f;
            fuse = J.burn_in;
#ifdef FFB_XAOS
            prev = ffb_xaos_first(sm, (int)J.n_xf, gw, seed_d);
#endif
#if FFB_NSTATE > 0
            ffb_state_fresh(sm, J, gw, d);
#endif
        }
#endif
        if (fresh) { x = s0 * 2.0f - 1.0f; y = s1 * 2.0f - 1.0f; }
#if FFB_NINIT > 0
        // The state-init block (main_template.wgsl:117-122) draws every
        // dispatch; a resumed orbit then restores its state over it.
        for (int i = 0; i < FFB_NINIT; ++i) {
            const float r = rng.draw(0);
            if (fresh) J.state[(size_t)ffb_u32(J.table[T_INIT + i]) * J.n_walkers + (gw - J.walker0)] = floorf(r * 4.0f);
        }
#endif
    }
    (void)sm; (void)ci; (void)fuse; (void)prev;
}
#endif

#if defined(FFB_REFRESH) && FFB_RNG_MODE == 1
// Orbit refresh with the counter-based stream: at each dispatch boundary
// (every ipt iterations) the walkers w with (w + seed_d) % period == 0 start
// again, seed_d = seed + d * 2654435761 as the reference's dispatch seeds;
// the point from Philox counter (walker, 0xFFFFFFFF, d, 0xFFFFFFFD).
__device__ __forceinline__ void ffb_refresh(const float* __restrict__ sm, const ffb_launch& J, u32 gw, u64 it, float& x, float& y,
                                            float& ci, u32& fuse, int& prev) {
    if (it == 0 || J.ipt == 0 || it % J.ipt != 0) return;
    const u32 d = (u32)(it / J.ipt);
    const u32 seed_d = J.seed_lo + d * 2654435761u;
    if ((gw + seed_d) % (u32)FFB_REFRESH != 0u) return;
    const uint4 o = philox4(J.seed_lo, J.seed_hi, gw, 0xFFFFFFFFu, d, 0xFFFFFFFDu);
    x = u24(o.x) * 2.0f - 1.0f;
    y = u24(o.y) * 2.0f - 1.0f;
    ci = 0.0f;
    fuse = J.burn_in;
#ifdef FFB_XAOS
    prev = ffb_xaos_first(sm, (int)J.n_xf, gw, seed_d);
#endif
#if FFB_NSTATE > 0
    ffb_state_fresh(sm, J, gw, d);
#endif
    (void)prev;
}
#endif

#if FFB_SYM_KIND != 0
// Copy k of a plotted point under the flame's post-symmetry
// (utilities.wgsl:470-568): point mode rotates copy k by k*2pi/order about
// the centre; the axis modes pan by half the separation, pre-rotate by
// -rotation about the centre, and reflect copy 1.
__device__ __forceinline__ void ffb_sym_copy(const float* __restrict__ sm, int k, float& x, float& y) {
    const float cx = sm[T_SYM + 1], cy = sm[T_SYM + 2];
#if FFB_SYM_KIND == 3
    if (k == 0) return;
    const float cs = sm[T_SYM + 6 + 2 * k], sn = sm[T_SYM + 7 + 2 * k];
    const float dx = x - cx, dy = y - cy;
    x = dx * cs - dy * sn + cx;
    y = dx * sn + dy * cs + cy;
#else
#if FFB_SYM_KIND == 1
    y = y + sm[T_SYM + 3];
#else
    x = x + sm[T_SYM + 3];
#endif
    const float cs = sm[T_SYM + 4], sn = sm[T_SYM + 5];
    const float dx = x - cx, dy = y - cy;
    x = dx * cs - dy * sn + cx;
    y = dx * sn + dy * cs + cy;
    if (k == 1) {
#if FFB_SYM_KIND == 1
        y = 2.0f * cy - y;
#else
        x = 2.0f * cx - x;
#endif
    }
#endif
}
#endif

// The plot of a kept sample of transform k: its final chain, the palette,
// the symmetry copies, world_to_pixel and the splat (main_template.wgsl:663-1320).
template <class R>
__device__ __forceinline__ void ffb_plot_sample(const float* __restrict__ sm, const float4* __restrict__ pal, const ffb_launch& J,
                                                int k, float x, float y, float ci, bool plot, R& rng, FfbCtx& ctx, float cx,
                                                float cy, float scale, u32& inframe) {
    float fx = x, fy = y;
    ffb_finals(sm, k, fx, fy, rng, ctx);                                    // main_template.wgsl:663-717
#ifdef FFB_HIDE
    if (ctx.hide) plot = false;                                             // main_template.wgsl:725-731
#endif
#ifdef FFB_SPEED
    // Speed mode plots the walker's own colour (main_template.wgsl:770-772);
    // a key of its lane keeps the warp's splats apart.
    const float* wc = ctx.st + (size_t)FFB_SPEED_SLOT * ctx.stride;
    const float4 c = make_float4(wc[0], wc[ctx.stride], wc[2 * (size_t)ctx.stride], 1.0f);
    const int pal_idx = 0x8000 | (int)(threadIdx.x & 31u);
    (void)ci;
#else
    const int pal_idx = ffb_palette_index(ci, J.pal_n);
    const float4 c = pal[pal_idx];                                          // main_template.wgsl:766-772
#endif
#if FFB_SYM_KIND != 0
    const int ncopy = (int)sm[T_SYM];                                       // main_template.wgsl:747-755, 858-870
    for (int sk = 0; sk < ncopy; ++sk) {
        float sx = fx, sy = fy;
        ffb_sym_copy(sm, sk, sx, sy);
#else
    {
        const float sx = fx, sy = fy;
#endif
        // world_to_pixel (utilities.wgsl:417-450).
        float tx = sx - J.pan_x, ty = sy - J.pan_y;
        float rx = tx * J.cos_r - ty * J.sin_r;
        float ry = tx * J.sin_r + ty * J.cos_r;
        rx = rx * J.zoom; ry = ry * J.zoom;
        const float pxf = floorf(cx + rx * scale), pyf = floorf(cy + ry * scale);
        const bool hit = plot && pxf >= 0.0f && pyf >= 0.0f && pxf < (float)J.width && pyf < (float)J.height;
#ifdef FFB_EMIT
        ffb_emit(J, hit, hit ? (u32)pyf * (u32)J.width + (u32)pxf : 0u, pal_idx, ffb_copies(sm));
        inframe += hit ? 1u : 0u;
#else
        if (hit) {
            const u32 idx = (u32)pyf * (u32)J.width + (u32)pxf;
            ffb_splat(J.hist, idx, c, pal_idx);
            ++inframe;
        }
#endif
    }
}

#ifdef FFB_DEFER
// Deferred plotting: the chaos kernel stores each iteration's sample (its
// point after the transform, colour index, plot flag, transform) and the
// draws of the finals' slots; ffb_plot (or the plotting warps of
// ffb_chaos_fused) applies the rest.  A record a walker and iteration:
// (x, y, ci, flags) with flags bit 1 a kept sample, bit 0 its opacity draw
// passed, bits 8-15 the transform picked; 0 for burn-in and respawns.  The
// final chain's draws go to planes `stride` apart.
struct FfbRec {
    float4* rec;
    float* draws;
    u64 stride;
};
// The record of walker gw at iteration it in the launch's global buffers.
__device__ __forceinline__ FfbRec ffb_rec_at(const ffb_launch& J, u32 gw, u64 it) {
    const u64 ri = (it - J.it0) * (u64)J.n_walkers + (u64)(gw - J.walker0);
    return FfbRec{J.rec + ri, J.rec_draws + ri, (u64)J.n_iters * J.n_walkers};
}
#define FFB_DEFER_SKIP(R) (*(R).rec = make_float4(0.f, 0.f, 0.f, 0.f))
template <class R>
__device__ __forceinline__ void ffb_defer_store(const FfbRec& rs, int k, float x, float y, float ci, bool plot, R& rng) {
    *rs.rec = make_float4(x, y, ci, __uint_as_float(2u | (plot ? 1u : 0u) | ((u32)k << 8)));
    ffb_capture_final_draws(rng, rs.draws, rs.stride);
}
// The stored draws handed back by slot.
struct SlotRng {
    const float* d;
    __device__ __forceinline__ float draw(int slot) { return d[slot - FFB_FIN_SLOT0]; }
    __device__ __forceinline__ u32 word(int slot) { return ffb_word_of(draw(slot)); }
};
#else
struct FfbRec {};
#define FFB_DEFER_SKIP(R) ((void)0)
#endif

// The rest of an iteration once transform k is picked and the opacity draw
// made: affine, variations, post, bad-value respawn, colour, fuse, finals,
// palette, world_to_pixel and the splat (main_template.wgsl:366-1320).
template <bool PER_XFORM, class R>
__device__ __forceinline__ void ffb_step(const float* __restrict__ sm, const float4* __restrict__ pal, const ffb_launch& J,
                                         int k, bool plot, R& rng, u32 gw, u64 it, float& x, float& y, float& ci, u32& fuse,
                                         float cx, float cy, float scale, u32& inframe, const FfbRec* slot = nullptr) {
    const float* q = sm + T_XF + k;
#ifdef FFB_DEFER
    const FfbRec rs = slot ? *slot : ffb_rec_at(J, gw, it);
#else
    (void)slot;
#endif
    FfbCtx ctx = ffb_ctx(J, gw, it);
#ifdef FFB_DC
    // Step 1 of the colour flow with a colour-writing variation
    // (main_template.wgsl:294-306): c_base, the register vc starting there.
    const float cb = ci * q[F_C1 * FFB_MAXX] + q[F_C2 * FFB_MAXX];
    ctx.vc = cb;
#endif
    float ax = q[F_A * FFB_MAXX] * x + q[F_B * FFB_MAXX] * y + q[F_E * FFB_MAXX];
    float ay = q[F_C * FFB_MAXX] * x + q[F_D * FFB_MAXX] * y + q[F_F * FFB_MAXX];
    if (PER_XFORM) ffb_normal_k(sm, k, ax, ay, rng, ctx);                   // main_template.wgsl:366-376
    else ffb_normal(sm, k, ax, ay, rng, ctx);
#if FFB_HAS_POST
    if (q[F_POST * FFB_MAXX] > 0.5f) {                                      // main_template.wgsl:380-384
        float px = q[F_PA * FFB_MAXX] * ax + q[F_PB * FFB_MAXX] * ay + q[F_PE * FFB_MAXX];
        float py = q[F_PC * FFB_MAXX] * ax + q[F_PD * FFB_MAXX] * ay + q[F_PF * FFB_MAXX];
        ax = px; ay = py;
    }
#endif
#if FFB_NLNK > 0
    ffb_linked(sm, k, ax, ay, rng, ctx);                                    // main_template.wgsl:320-360
#endif
#ifdef FFB_HIDE
    if (ctx.hide) { FFB_DEFER_SKIP(rs); return; }                          // main_template.wgsl:389-400: the point reverts
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
        FFB_DEFER_SKIP(rs);
        return;
    }
#ifdef FFB_SPEED
    {   // Speed colour (main_template.wgsl:483, 491-493; utilities.wgsl:148-156):
        // the step's length, log-scaled into the palette, mixed into the
        // walker's colour by speed_factor.
        const float dx = ax - x, dy = ay - y;
        const float sp = sqrtf(dx * dx + dy * dy);
        const float ns = fminf(fmaxf(FLOG(sp * 10.0f + 1.0f) / 3.0f, 0.0f), 1.0f);
        const float4 sc = pal[ffb_palette_index(ns, J.pal_n)];
        const float t = sm[T_SPEED];
        float* wc = ctx.st + (size_t)FFB_SPEED_SLOT * ctx.stride;
        const size_t sd = ctx.stride;
        wc[0] = wc[0] * (1.0f - t) + sc.x * t;
        wc[sd] = wc[sd] * (1.0f - t) + sc.y * t;
        wc[2 * sd] = wc[2 * sd] * (1.0f - t) + sc.z * t;
    }
#endif
    x = ax; y = ay;
#ifdef FFB_DC
    ci = cb + q[F_DC * FFB_MAXX] * (ctx.vc - cb);                          // main_template.wgsl:486-490
#else
    ci = ci * q[F_C1 * FFB_MAXX] + q[F_C2 * FFB_MAXX];                       // main_template.wgsl:496-508
#endif
    if (fuse > 0u) { fuse -= 1u; FFB_DEFER_SKIP(rs); return; }            // main_template.wgsl:510-514
#ifdef FFB_DEFER
    ffb_defer_store(rs, k, x, y, ci, plot, rng);
#else
    ffb_plot_sample(sm, pal, J, k, x, y, ci, plot, rng, ctx, cx, cy, scale, inframe);
#endif
}

__device__ __forceinline__ void ffb_count_inframe(const ffb_launch& J, u32 inframe) {
    // In-frame splat count (count conservation: the sum of the count plane).
    const unsigned live = __activemask();
    const u32 tot = __reduce_add_sync(live, inframe);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(live) - 1) && tot) atomicAdd(J.counters, (u64)tot);
}

// One walker's whole launch (the body of ffb_chaos).
__device__ __forceinline__ void ffb_chaos_walker(const float* __restrict__ sm, const float4* __restrict__ pal,
                                                 const ffb_launch& J, u32 w) {
    const u32 gw = J.walker0 + w;
    const int n_xf = (int)J.n_xf;
    float x, y, ci;
    u32 fuse;
    int prev;
    ffb_start(sm, J, w, gw, x, y, ci, fuse, prev);
    const float scale = (float)min(J.width, J.height) * 0.25f;
    const float cx = (float)J.width * 0.5f, cy = (float)J.height * 0.5f;
    u32 inframe = 0;
#if FFB_RNG_MODE == 0
    PcgRng rng;
    rng.state = 0; rng.inc = 1;
#endif
    const u64 it1 = J.it0 + J.n_iters;
    for (u64 it = J.it0; it < it1; ++it) {
#if FFB_RNG_MODE == 0
        ffb_pcg_dispatch(sm, J, rng, gw, it, x, y, ci, fuse, prev);
#else
#ifdef FFB_REFRESH
        ffb_refresh(sm, J, gw, it, x, y, ci, fuse, prev);
#endif
        PhiloxRng rng;
        rng.fill(J.seed_lo, J.seed_hi, gw, it);
#endif
        const int k = FFB_PICK(rng.draw(0), prev);                            // main_template.wgsl:198-223
        prev = k;
        const bool plot = rng.draw(1) < sm[T_XF + F_OPAC * FFB_MAXX + k];       // main_template.wgsl:249
        ffb_step<false>(sm, pal, J, k, plot, rng, gw, it, x, y, ci, fuse, cx, cy, scale, inframe);
    }
    (void)prev;
    J.walkers[w] = make_float4(x, y, ci, __uint_as_float(FFB_PACK_FUSE(fuse, prev)));
    ffb_count_inframe(J, inframe);
}

// One walker a thread, for the whole launch.
extern "C" __global__ void __launch_bounds__(FFB_THREADS)
ffb_chaos(const ffb_launch* __restrict__ jobs, int n_jobs) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    float4* pal;
    const ffb_launch& J = ffb_stage(jobs, n_jobs, sm, pal);
    const u32 w = (blockIdx.x - J.block0) * blockDim.x + threadIdx.x;
    if (w < J.n_walkers) ffb_chaos_walker(sm, pal, J, w);
#ifdef FFB_EMIT
    ffb_emit_finish(J, ffb_copies(sm));                  // every thread reaches its barrier
#endif
}

// Transform-coherent scheduling.  A thread holds a walker only for one
// iteration: after each walker picks its transform, the block regroups the
// walkers by transform (a counting sort through shared memory, the state
// travelling with the walker's id), so a warp runs mostly one transform and
// the variation branches of ffb_normal are warp-uniform.  Every walker still
// draws from its own counter-based stream, keyed by its id, so the orbits
// are bit-identical to ffb_chaos's; only which thread carries them changes.
extern "C" __global__ void __launch_bounds__(1024, 1)
ffb_chaos_sorted(const ffb_launch* __restrict__ jobs, int n_jobs) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    float4* pal;
    const ffb_launch& J = ffb_stage(jobs, n_jobs, sm, pal);
    const int P = blockDim.x, tid = threadIdx.x, lane = tid & 31;
    float* s_x = reinterpret_cast<float*>(pal + J.pal_n);
    float* s_y = s_x + P;
    float* s_ci = s_y + P;
    u32* s_fuse = reinterpret_cast<u32*>(s_ci + P);
    u32* s_kp = s_fuse + P;                     // k | plot << 31
    u32* s_wid = s_kp + P;
    u32* s_r0 = s_wid + P;                      // philox words 2, 3 / pcg state, inc
    u32* s_r1 = s_r0 + P;
    u32* s_cnt = s_r1 + P;                      // [2][FFB_MAXX + 1], ping-pong by iteration
    const int NC = FFB_MAXX + 1;
    for (int i = tid; i < 2 * NC; i += P) s_cnt[i] = 0u;
    const u32 w0 = (blockIdx.x - J.block0) * P + tid;
    bool active = w0 < J.n_walkers;
    u32 wid = J.walker0 + w0;
    float x = 0.f, y = 0.f, ci = 0.f;
    u32 fuse = 0;
    int prev = 0;                                // the held walker's previous transform (xaos)
    if (active) ffb_start(sm, J, w0, wid, x, y, ci, fuse, prev);
    const int n_xf = (int)J.n_xf;
    const float scale = (float)min(J.width, J.height) * 0.25f;
    const float cx = (float)J.width * 0.5f, cy = (float)J.height * 0.5f;
    u32 inframe = 0;
#if FFB_RNG_MODE == 0
    PcgRng rng;
    rng.state = 0; rng.inc = 1;
#endif
    __syncthreads();
    const u64 it1 = J.it0 + J.n_iters;
    int par = 0;
    for (u64 it = J.it0; it < it1; ++it, par ^= 1) {
        u32* cnt = s_cnt + par * NC;
        int k = FFB_MAXX;                        // inactive threads sort last
        bool plot = false;
        u32 r0 = 0, r1 = 0;
        if (active) {
#if FFB_RNG_MODE == 0
            ffb_pcg_dispatch(sm, J, rng, wid, it, x, y, ci, fuse, prev);
            k = FFB_PICK(rng.draw(0), prev);
            plot = rng.draw(1) < sm[T_XF + F_OPAC * FFB_MAXX + k];
            r0 = rng.state; r1 = rng.inc;
#else
#ifdef FFB_REFRESH
            ffb_refresh(sm, J, wid, it, x, y, ci, fuse, prev);
#endif
            PhiloxRng rng;
            rng.fill(J.seed_lo, J.seed_hi, wid, it);
            k = FFB_PICK(rng.draw(0), prev);
            plot = rng.draw(1) < sm[T_XF + F_OPAC * FFB_MAXX + k];
            r0 = __float_as_uint(rng.w[2]); r1 = __float_as_uint(rng.w[3]);
#endif
        }
        // Counting sort by transform: warp-aggregated counts, then each
        // walker's slot = (walkers of lower transforms) + its rank.
        const unsigned grp = __match_any_sync(0xffffffffu, k);
        const int leader = __ffs(grp) - 1;
        const u32 rank = __popc(grp & ((1u << lane) - 1u));
        u32 base = 0;
        if (lane == leader) base = atomicAdd(&cnt[k], (u32)__popc(grp));
        base = __shfl_sync(0xffffffffu, base, leader);
        u32* nxt = s_cnt + (par ^ 1) * NC;
        __syncthreads();                                                        // counts complete
        for (int i = tid; i < NC; i += P) nxt[i] = 0u;                          // next iteration's counters
        u32 off = 0;
#pragma unroll 4
        for (int j = 0; j < k; ++j) off += cnt[j];
        const u32 slot = off + base + rank;
        s_x[slot] = x; s_y[slot] = y; s_ci[slot] = ci; s_fuse[slot] = fuse;
        s_kp[slot] = (u32)k | (plot ? 0x80000000u : 0u);
        s_wid[slot] = wid; s_r0[slot] = r0; s_r1[slot] = r1;
        __syncthreads();                                                        // states regrouped
        x = s_x[tid]; y = s_y[tid]; ci = s_ci[tid]; fuse = s_fuse[tid];
        const u32 kp = s_kp[tid];
        k = (int)(kp & 0x7FFFFFFFu);
        plot = (kp >> 31) != 0u;
        prev = k;                                // the gathered walker's transform, its next pick's row
        wid = s_wid[tid];
        active = k < FFB_MAXX;
        if (active) {
#if FFB_RNG_MODE == 0
            rng.state = s_r0[tid]; rng.inc = s_r1[tid];
            ffb_step<true>(sm, pal, J, k, plot, rng, wid, it, x, y, ci, fuse, cx, cy, scale, inframe);
#else
            PhiloxRng rng;
            rng.w[2] = __uint_as_float(s_r0[tid]);
            rng.w[3] = __uint_as_float(s_r1[tid]);
            rng.fill_from(1, J.seed_lo, J.seed_hi, wid, it);
            ffb_step<true>(sm, pal, J, k, plot, rng, wid, it, x, y, ci, fuse, cx, cy, scale, inframe);
#endif
        }
    }
    (void)prev;
    if (active) J.walkers[wid - J.walker0] = make_float4(x, y, ci, __uint_as_float(FFB_PACK_FUSE(fuse, prev)));
    ffb_count_inframe(J, inframe);
#ifdef FFB_EMIT
    ffb_emit_finish(J, ffb_copies(sm));
#endif
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
    // State as a probe thread starts it (zero) and vc = 0.5 (main_template.wgsl:1510-1512).
    float st[FFB_NSTATE > 0 ? FFB_NSTATE : 1];
    for (int s = 0; s < (FFB_NSTATE > 0 ? FFB_NSTATE : 1); ++s) st[s] = 0.0f;
    FfbCtx ctx{st, 1u, 0.5f, 0u, 0u, (u32)slot, 0ull};
    if (xi < n_xf) ffb_normal(table, xi, x, y, rng, ctx);
    else ffb_final_one(table, xi - n_xf, x, y, rng, ctx, false);
    out[slot] = make_float2(x, y);
}

// Single-step parity: transform xi (affine, variations, post) at n points
// with given draw words (FFB_APPLY_WORDS a point).  xi >= n_xf selects final xi - n_xf.
extern "C" __global__ void ffb_apply_points(const float* __restrict__ table, int n_xf, int xi, int n,
                                            const float* __restrict__ xs, const float* __restrict__ ys,
                                            const float* __restrict__ words, int with_affine,
                                            float* __restrict__ xo, float* __restrict__ yo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ArrayRng rng{words + (size_t)i * FFB_APPLY_WORDS};
    float st[FFB_NSTATE > 0 ? FFB_NSTATE : 1];
    for (int s = 0; s < (FFB_NSTATE > 0 ? FFB_NSTATE : 1); ++s) st[s] = 0.0f;
    FfbCtx ctx{st, 1u, 0.5f, 0u, 0u, (u32)i, 0ull};
    float x = xs[i], y = ys[i];
    if (xi < n_xf) {
        const float* q = table + T_XF + xi;
        if (with_affine) {
            float ax = q[F_A * FFB_MAXX] * x + q[F_B * FFB_MAXX] * y + q[F_E * FFB_MAXX];
            float ay = q[F_C * FFB_MAXX] * x + q[F_D * FFB_MAXX] * y + q[F_F * FFB_MAXX];
            x = ax; y = ay;
        }
        ffb_normal(table, xi, x, y, rng, ctx);
        if (with_affine && q[F_POST * FFB_MAXX] > 0.5f) {
            float px = q[F_PA * FFB_MAXX] * x + q[F_PB * FFB_MAXX] * y + q[F_PE * FFB_MAXX];
            float py = q[F_PC * FFB_MAXX] * x + q[F_PD * FFB_MAXX] * y + q[F_PF * FFB_MAXX];
            x = px; y = py;
        }
    } else {
        ffb_final_one(table, xi - n_xf, x, y, rng, ctx, with_affine != 0);
    }
    xo[i] = x; yo[i] = y;
}

#ifdef FFB_DEFER
// The plot of one launch's stored samples (the tail ffb_chaos defers): a
// thread a record, grid-striding; samples are independent, so this kernel
// has the parallelism the walkers' chains lack.
extern "C" __global__ void __launch_bounds__(384) ffb_plot(const ffb_launch* __restrict__ jobs, int n_jobs) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    float4* pal;
    const ffb_launch& J = ffb_stage(jobs, n_jobs, sm, pal);
    const float scale = (float)min(J.width, J.height) * 0.25f;
    const float cx = (float)J.width * 0.5f, cy = (float)J.height * 0.5f;
    const u64 n = (u64)J.n_iters * J.n_walkers;
    u32 inframe = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const float4 r = J.rec[i];
        const u32 fl = __float_as_uint(r.w);
        if (!(fl & 2u)) continue;
        float fd[FFB_NFD > 0 ? FFB_NFD : 1];
#pragma unroll
        for (int m = 0; m < FFB_NFD; ++m) fd[m] = J.rec_draws[(u64)m * n + i];
        SlotRng rng{fd};
        FfbCtx ctx{nullptr, 0u, 0.0f, 0u, 0u, 0u, 0ull};                // deferred finals carry no state
        ffb_plot_sample(sm, pal, J, (int)((fl >> 8) & 0xFFu), r.x, r.y, r.z, (fl & 1u) != 0u, rng, ctx, cx, cy, scale, inframe);
    }
    ffb_count_inframe(J, inframe);
}
#endif

#if defined(FFB_DEFER) && FFB_RNG_MODE == 1 && !defined(FFB_REFRESH)
// ---------------------------------------------------------------------------
// Fused plotting: the walkers and the plot of their samples in one block.
//
// The first J.ring_prod threads of a block are producer warps: they carry the
// block's walkers through the transform-sorted schedule of ffb_chaos_sorted
// and, instead of plotting, write each iteration's samples (the deferred
// records) into a ring of J.ring_depth iteration slots in shared memory.  The
// other warps of the block are consumer warps: they take the slots in order
// and apply the plot tail -- the final chain, the palette, the symmetry
// copies, world_to_pixel and the warp-aggregated splat.  A sample never goes
// to HBM on its way from the walker to the histogram, and the plot's long
// independent work fills the issue slots the walkers' dependent chains and
// their sorting barrier leave empty.
//
// Hand-over: full[d] (one arrival a producer warp) completes when slot d
// holds an iteration's records, empty[d] (one arrival a consumer warp) when
// it has been plotted; a slot's u-th use waits on phase parity u & 1.  Every
// wait is bounded: past FFB_WAIT_LIMIT polls the kernel sets bit 63 of the
// in-frame counter (the host reports the render failed) and goes on, so no
// miscounted hand-over can hang the GPU.
//
// One barrier an iteration among the producers: the counter-based stream
// gives every walker's pick ahead of time (it depends only on the walker's
// id, the iteration and, with xaos, the previous pick), so the picks of
// iteration j + 2 are counted while iteration j runs, and iteration j + 1's
// sort needs only its scatter and gather around a single barrier.  Counters
// are kept in three rotating sets, slot ranks and walker state in two.
// Orbits are those of ffb_chaos and ffb_chaos_sorted, bit for bit.

#define FFB_WAIT_LIMIT (1u << 21)
#define FFB_WAIT_HINT_NS 2000

__device__ __forceinline__ u32 ffb_smem_addr(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void ffb_mbar_init(u64* b, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(ffb_smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void ffb_mbar_arrive(u64* b) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(ffb_smem_addr(b)) : "memory");
}
// One poll: the thread may sleep up to FFB_WAIT_HINT_NS in it, and wakes when
// the phase completes.
__device__ __forceinline__ bool ffb_mbar_test(u64* b, u32 parity) {
    u32 ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(ffb_smem_addr(b)), "r"(parity), "n"(FFB_WAIT_HINT_NS)
                 : "memory");
    return ok != 0u;
}
// Wait for phase `parity` of b: at most FFB_WAIT_LIMIT polls (a few seconds).
// A wait that gives up marks the block aborted (`abort`, shared memory) and
// the render failed (bit 63 of the in-frame counter); an aborted block waits
// no more, so it runs to its end at once whatever went wrong.
__device__ __forceinline__ void ffb_mbar_wait(u64* b, u32 parity, volatile u32* abort, const ffb_launch& J) {
    if (*abort) return;
    for (u32 n = 0; n < FFB_WAIT_LIMIT; ++n)
        if (ffb_mbar_test(b, parity)) return;
    *abort = 1u;
    atomicOr(J.counters, 1ull << 63);
}
// The producers' barrier (named barrier 1, producer threads only).
__device__ __forceinline__ void ffb_prod_sync(u32 n_threads) {
    asm volatile("bar.sync 1, %0;" ::"r"(n_threads) : "memory");
}

// A walker's pick at iteration it: the transform, its opacity draw, and the
// two variation words of Philox block 0 (slots 2, 3).
struct FfbPick {
    int k;
    bool plot;
    float w2, w3;
};
__device__ __forceinline__ FfbPick ffb_pick_at(const float* __restrict__ sm, const ffb_launch& J, int n_xf, u32 wid, u64 it,
                                               int prev) {
    const uint4 o = philox4(J.seed_lo, J.seed_hi, wid, (u32)it, 0u, (u32)(it >> 32));
    FfbPick p;
    p.k = FFB_PICK(u24(o.x), prev);                                              // main_template.wgsl:198-223
    p.plot = u24(o.y) < sm[T_XF + F_OPAC * FFB_MAXX + p.k];                      // main_template.wgsl:249
    p.w2 = u24(o.z);
    p.w3 = u24(o.w);
    (void)prev;
    return p;
}
__device__ __forceinline__ u32 ffb_pack_pick(int k, bool plot) { return (u32)k | (plot ? 0x8000u : 0u); }

// Count transform k into cnt (warp-aggregated; every lane of the warp takes part).
__device__ __forceinline__ void ffb_count_pick(u32* cnt, int k) {
    const unsigned grp = __match_any_sync(0xffffffffu, k);
    if ((int)(threadIdx.x & 31u) == __ffs(grp) - 1) atomicAdd(&cnt[k], (u32)__popc(grp));
}
// The sorted slot of a walker with transform k: walkers of lower transforms
// (complete counts) + its rank among those of k (a running count).
__device__ __forceinline__ u32 ffb_sort_slot(const u32* cnt, u32* rnk, int k) {
    const int lane = (int)(threadIdx.x & 31u);
    const unsigned grp = __match_any_sync(0xffffffffu, k);
    const int leader = __ffs(grp) - 1;
    u32 base = 0;
    if (lane == leader) base = atomicAdd(&rnk[k], (u32)__popc(grp));
    base = __shfl_sync(0xffffffffu, base, leader);
    // Walkers of lower transforms: every count loaded at once (independent
    // shared loads), summed under a predicate -- no loop whose length, and
    // chain of dependent loads, follows k.
    u32 off = 0;
#pragma unroll
    for (int i = 0; i < FFB_MAXX; ++i) {
        const u32 c = cnt[i];
        off += i < k ? c : 0u;
    }
    return off + base + (u32)__popc(grp & ((1u << lane) - 1u));
}

// Shared memory of the fused kernel after the table and palette.
struct FfbFused {
    u64* full;          // ring_depth mbarriers
    u64* empty;         // ring_depth mbarriers
    u32* abort;         // set when a wait gave up
    u32* cnt;           // 3 sets of FFB_MAXX + 1 transform counts
    u32* rnk;           // 2 sets of FFB_MAXX + 1 running ranks
    u32* st;            // 2 sets of 10 planes of ring_prod words: the regrouped walkers
    float4* ring;       // ring_depth x ring_prod records
    float* ring_draws;  // FFB_NFD planes of ring_depth x ring_prod final-chain draws
};
#define FFB_FUSED_PLANES 10
enum { FS_X, FS_Y, FS_CI, FS_FUSE, FS_WID, FS_KP, FS_A2, FS_A3, FS_B2, FS_B3 };

__device__ __forceinline__ void ffb_fused_put(const FfbFused& S, int set, u32 P, u32 slot, float x, float y, float ci, u32 fuse,
                                              u32 wid, u32 kp, float a2, float a3, float b2, float b3) {
    u32* b = S.st + (size_t)set * FFB_FUSED_PLANES * P + slot;
    b[FS_X * P] = __float_as_uint(x); b[FS_Y * P] = __float_as_uint(y); b[FS_CI * P] = __float_as_uint(ci);
    b[FS_FUSE * P] = fuse; b[FS_WID * P] = wid; b[FS_KP * P] = kp;
    b[FS_A2 * P] = __float_as_uint(a2); b[FS_A3 * P] = __float_as_uint(a3);
    b[FS_B2 * P] = __float_as_uint(b2); b[FS_B3 * P] = __float_as_uint(b3);
}
__device__ __forceinline__ void ffb_fused_get(const FfbFused& S, int set, u32 P, u32 slot, float& x, float& y, float& ci, u32& fuse,
                                              u32& wid, u32& kp, float& a2, float& a3, float& b2, float& b3) {
    const u32* b = S.st + (size_t)set * FFB_FUSED_PLANES * P + slot;
    x = __uint_as_float(b[FS_X * P]); y = __uint_as_float(b[FS_Y * P]); ci = __uint_as_float(b[FS_CI * P]);
    fuse = b[FS_FUSE * P]; wid = b[FS_WID * P]; kp = b[FS_KP * P];
    a2 = __uint_as_float(b[FS_A2 * P]); a3 = __uint_as_float(b[FS_A3 * P]);
    b2 = __uint_as_float(b[FS_B2 * P]); b3 = __uint_as_float(b[FS_B3 * P]);
}

// Producer warps: the block's walkers, sorted by transform every iteration.
// Thread state after each gather: the walker's point, colour index, fuse and
// id, its picks for this iteration (k, plot; words a2, a3) and the next
// (kn, plotn; words b2, b3).
__device__ __forceinline__ void ffb_fused_producer(const float* __restrict__ sm, const float4* __restrict__ pal, const ffb_launch& J,
                                                   const FfbFused& S) {
    const u32 P = J.ring_prod, D = J.ring_depth;
    const int tid = (int)threadIdx.x, lane = tid & 31;
    const int NC = FFB_MAXX + 1;
    const int n_xf = (int)J.n_xf;
    const u32 n = J.n_iters;
    const u32 w0 = (blockIdx.x - J.block0) * P + (u32)tid;
    bool active = w0 < J.n_walkers;
    u32 wid = J.walker0 + w0;
    float x = 0.f, y = 0.f, ci = 0.f;
    u32 fuse = 0;
    int prev = 0;
    if (active) ffb_start(sm, J, w0, wid, x, y, ci, fuse, prev);
    const float scale = (float)min(J.width, J.height) * 0.25f;
    const float cx = (float)J.width * 0.5f, cy = (float)J.height * 0.5f;
    // The first two iterations' picks, counted into sets 0 and 1.
    FfbPick p0{FFB_MAXX, false, 0.f, 0.f}, p1{FFB_MAXX, false, 0.f, 0.f};
    if (active) {
        p0 = ffb_pick_at(sm, J, n_xf, wid, J.it0, prev);
        if (n > 1) p1 = ffb_pick_at(sm, J, n_xf, wid, J.it0 + 1, p0.k);
    }
    ffb_count_pick(S.cnt, p0.k);
    if (n > 1) ffb_count_pick(S.cnt + NC, p1.k);
    ffb_prod_sync(P);
    {
        const u32 slot = ffb_sort_slot(S.cnt, S.rnk, p0.k);
        ffb_fused_put(S, 0, P, slot, x, y, ci, fuse, wid, ffb_pack_pick(p0.k, p0.plot) | (ffb_pack_pick(p1.k, p1.plot) << 16),
                      p0.w2, p0.w3, p1.w2, p1.w3);
    }
    ffb_prod_sync(P);
    u32 kp;
    float a2, a3, b2, b3;
    ffb_fused_get(S, 0, P, (u32)tid, x, y, ci, fuse, wid, kp, a2, a3, b2, b3);
    u32 inframe = 0;
    for (u32 j = 0; j < n; ++j) {
        const u64 it = J.it0 + j;
        const u32 d = j % D;
        const int k = (int)(kp & 0x7FFFu);
        const bool plot = (kp & 0x8000u) != 0u;
        active = k < FFB_MAXX;
        // The pick two iterations ahead (independent of this step's point:
        // its Philox rounds overlap the step's latency), counted after it.
        const int kn = (int)((kp >> 16) & 0x7FFFu);
        const bool pn = (kp >> 31) != 0u;
        FfbPick p2{FFB_MAXX, false, 0.f, 0.f};
        if (active && j + 2 < n) p2 = ffb_pick_at(sm, J, n_xf, wid, it + 2, kn);
        // This iteration's records go to ring slot d once the consumers are done with its last use.
        if (j >= D) ffb_mbar_wait(&S.empty[d], ((j / D) - 1u) & 1u, S.abort, J);
        const FfbRec rs{S.ring + (size_t)d * P + tid, S.ring_draws + (size_t)d * P + tid, (u64)D * P};
        if (active) {
            PhiloxRng rng;
            rng.w[0] = 0.f;
            rng.w[1] = 0.f;
            rng.w[2] = a2;
            rng.w[3] = a3;
            rng.fill_from(1, J.seed_lo, J.seed_hi, wid, it);
            ffb_step<true>(sm, pal, J, k, plot, rng, wid, it, x, y, ci, fuse, cx, cy, scale, inframe, &rs);
        } else {
            FFB_DEFER_SKIP(rs);
        }
        __syncwarp();
        if (lane == 0) ffb_mbar_arrive(&S.full[d]);
        if (j + 1 == n) {
            prev = k;
            break;
        }
        // Count the pick two ahead (set (j + 2) % 3).
        if (j + 2 < n) ffb_count_pick(S.cnt + ((j + 2) % 3) * NC, p2.k);
        // Counters whose last reader ran before the previous barrier: zero them for their next use.
        for (int i = tid; i < NC; i += (int)P) {
            S.cnt[(j % 3) * NC + i] = 0u;
            S.rnk[(j % 2) * NC + i] = 0u;
        }
        // Regroup by next iteration's transform.
        const u32 slot = ffb_sort_slot(S.cnt + ((j + 1) % 3) * NC, S.rnk + ((j + 1) % 2) * NC, kn);
        ffb_fused_put(S, (int)((j + 1) % 2), P, slot, x, y, ci, fuse, wid,
                      ffb_pack_pick(kn, pn) | (ffb_pack_pick(p2.k, p2.plot) << 16), b2, b3, p2.w2, p2.w3);
        ffb_prod_sync(P);
        ffb_fused_get(S, (int)((j + 1) % 2), P, (u32)tid, x, y, ci, fuse, wid, kp, a2, a3, b2, b3);
    }
    (void)inframe;
    if (active) J.walkers[wid - J.walker0] = make_float4(x, y, ci, __uint_as_float(FFB_PACK_FUSE(fuse, prev)));
}

// Consumer warps: plot each ring slot's records, slot after slot.
__device__ __forceinline__ void ffb_fused_consumer(const float* __restrict__ sm, const float4* __restrict__ pal, const ffb_launch& J,
                                                   const FfbFused& S) {
    const u32 P = J.ring_prod, D = J.ring_depth;
    const u32 C = blockDim.x - P;
    const u32 c = threadIdx.x - P;
    const int lane = (int)(threadIdx.x & 31u);
    const float scale = (float)min(J.width, J.height) * 0.25f;
    const float cx = (float)J.width * 0.5f, cy = (float)J.height * 0.5f;
    u32 inframe = 0;
    // A pass covers one slot (a pass over two slots, giving every thread of
    // 576 work against 448 records, measured 7 % slower: 61.1 ms a frame
    // against 57.1).
    const u32 G = 1u;
    for (u32 j = 0; j < J.n_iters; j += G) {
        const u32 g = min(G, J.n_iters - j);
        for (u32 q = 0; q < g; ++q) ffb_mbar_wait(&S.full[(j + q) % D], ((j + q) / D) & 1u, S.abort, J);
        for (u32 i = c; i < g * P; i += C) {
            const u32 d = (j + i / P) % D, e = i % P;
            const float4 r = S.ring[(size_t)d * P + e];
            const u32 fl = __float_as_uint(r.w);
            if (!(fl & 2u)) continue;
            float fd[FFB_NFD > 0 ? FFB_NFD : 1];
#pragma unroll
            for (int m = 0; m < FFB_NFD; ++m) fd[m] = S.ring_draws[(size_t)m * D * P + (size_t)d * P + e];
            SlotRng rng{fd};
            FfbCtx ctx{nullptr, 0u, 0.0f, 0u, 0u, 0u, 0ull};                     // deferred finals carry no state
            ffb_plot_sample(sm, pal, J, (int)((fl >> 8) & 0xFFu), r.x, r.y, r.z, (fl & 1u) != 0u, rng, ctx, cx, cy, scale,
                            inframe);
        }
        __syncwarp();
        if (lane == 0)
            for (u32 q = 0; q < g; ++q) ffb_mbar_arrive(&S.empty[(j + q) % D]);
    }
    ffb_count_inframe(J, inframe);
}

// One block: ring_prod producer threads (a multiple of 32) and the rest
// consumers (a multiple of 32).  Shared memory after the table and palette:
// 2 x ring_depth mbarriers, the abort word (8 bytes), 5 x (FFB_MAXX + 1)
// counters, 2 x 10 x ring_prod
// walker words, up to 12 bytes of padding, ring_depth x ring_prod records of
// 16 bytes and FFB_NFD x ring_depth x ring_prod draws.
extern "C" __global__ void __launch_bounds__(1024, 1) ffb_chaos_fused(const ffb_launch* __restrict__ jobs, int n_jobs) {
    extern __shared__ float4 ffb_smem4[];
    float* sm = reinterpret_cast<float*>(ffb_smem4);
    float4* pal;
    const ffb_launch& J = ffb_stage(jobs, n_jobs, sm, pal);
    const u32 P = J.ring_prod, D = J.ring_depth;
    const int NC = FFB_MAXX + 1;
    FfbFused S;
    S.full = reinterpret_cast<u64*>(pal + J.pal_n);
    S.empty = S.full + D;
    S.abort = reinterpret_cast<u32*>(S.empty + D);
    S.cnt = S.abort + 2;
    S.rnk = S.cnt + 3 * NC;
    S.st = S.rnk + 2 * NC;
    // The ring starts at the next 16-byte boundary after the walker planes.
    S.ring = reinterpret_cast<float4*>((reinterpret_cast<size_t>(S.st + 2 * FFB_FUSED_PLANES * P) + 15) & ~(size_t)15);
    S.ring_draws = reinterpret_cast<float*>(S.ring + (size_t)D * P);
    // Launch-shape guard (the host sizes the block; a mismatch would miscount the hand-overs).
    const bool ok = P >= 32 && P % 32 == 0 && P < blockDim.x && (blockDim.x - P) % 32 == 0 && D >= 2;
    if (threadIdx.x == 0 && ok) {
        for (u32 i = 0; i < D; ++i) {
            ffb_mbar_init(&S.full[i], P / 32);
            ffb_mbar_init(&S.empty[i], (blockDim.x - P) / 32);
        }
    }
    for (int i = (int)threadIdx.x; i < 5 * NC + 2; i += (int)blockDim.x) S.abort[i] = 0u;
    __syncthreads();
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(J.counters, 1ull << 63);
        return;
    }
    if (threadIdx.x < P) ffb_fused_producer(sm, pal, J, S);
    else ffb_fused_consumer(sm, pal, J, S);
}
#endif
