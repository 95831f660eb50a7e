// ffb_tiles.cu -- tile-sorted accumulation into the exact histogram
// (ahead-of-time sm_100a kernels).
//
// When the exact histogram (32 B a pixel) is several times the L2, a direct
// splat pays for every sample with four 64-bit atomics on lines that mostly
// miss the L2.  The tiled path replaces them, per launch of the chaos game,
// by the stages of a counting sort:
//   1. the chaos kernel emits one 8-byte record a sample (ffb_emit) into
//      its block's segment of the record buffer;
//   2. k_tile_count: records per 64x64-pixel tile (shared-memory counters);
//   3. k_tile_scan: tile offsets, the accumulate's work list (slices of at
//      most `slice` records a tile) and the second scatter's work list;
//   4. two scatter passes that write coalesced runs: k_band_scatter groups
//      a block's records by band of 64 rows in shared memory and writes each
//      band's run at the band's next free place; k_tile_scatter does the
//      same within a band by tile column, writing 4-byte records (tile-local
//      pixel | palette index << 12) in tile order;
//   5. k_tile_accumulate: persistent blocks take slices from the work list,
//      sum them in shared memory (u32 count; u64 colour in 2^-24 units, the
//      same integers the direct exact splat adds, kept as 32-bit halves with
//      the carry taken from the returned old value) and add the tile to the
//      histogram with plain read-modify-writes (with atomics when a hot tile
//      is split over several slices).
// The integer sums make the result the same bits as the direct path.
// The same passes serve the u32-count / FP32-colour histogram (float4 a
// pixel): k_tile_accumulate_f32 sums a slice in shared memory (u32 count,
// FP32 colour) and adds it with one 16-byte read-modify-write a pixel, so
// the count plane is the direct splat's exactly and the colour sums differ
// from it only by the order of the FP32 additions.  The reference's
// counterpart is the sample-emit path for histograms larger
// than one storage binding (main_template.wgsl:1324-1353,
// shaders/core/accumulate_samples.wgsl, src/export/high_res.rs:2139-2175).

#include "ffb_tail.cuh"

#include <algorithm>
#include <cstdint>

namespace ffb {

namespace {

typedef unsigned long long u64t;

__device__ __forceinline__ unsigned tile_of(unsigned idx, const TileGeom& g, unsigned& local) {
    const unsigned y = idx / (unsigned)g.w, x = idx - y * (unsigned)g.w;
    local = (y & 63u) * 64u + (x & 63u);
    return (y >> 6) * (unsigned)g.tiles_x + (x >> 6);
}

// Records: segment s holds seg_n[s] <= seg_cap records from rec + s * seg_cap.
__global__ void k_tile_count(const u64t* __restrict__ rec, u64t seg_cap, int n_segs, const unsigned* __restrict__ seg_n,
                             TileGeom g, unsigned* __restrict__ count) {
    extern __shared__ unsigned s_cnt[];
    for (int t = threadIdx.x; t < g.n_tiles; t += blockDim.x) s_cnt[t] = 0u;
    __syncthreads();
    for (int sg = blockIdx.x; sg < n_segs; sg += gridDim.x) {
        const u64t* r = rec + (u64t)sg * seg_cap;
        const unsigned n = (unsigned)min((u64t)seg_n[sg], seg_cap);
        for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
            unsigned local;
            atomicAdd(&s_cnt[tile_of((unsigned)r[i], g, local)], 1u);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < g.n_tiles; t += blockDim.x)
        if (s_cnt[t]) atomicAdd(&count[t], s_cnt[t]);
}

// One block: exclusive scans of the tile counts (-> offsets, in tile order,
// which is band-major, so a band's tiles are contiguous) and of the slices a
// tile needs (-> the accumulate's work list); the band pass's work list
// (parts of at most `range` records of a band); clears the fill cursors and
// the work counter.
__global__ void k_tile_scan(const unsigned* __restrict__ count, TileGeom g, unsigned slice, unsigned range,
                            unsigned* __restrict__ off, unsigned* __restrict__ fill, unsigned* __restrict__ work_off,
                            unsigned* __restrict__ work, unsigned* __restrict__ band_fill, unsigned* __restrict__ band_part_off) {
    __shared__ unsigned s_a[1024], s_b[1024];
    const int n_tiles = g.n_tiles;
    const int per = (n_tiles + blockDim.x - 1) / blockDim.x;
    const int t0 = threadIdx.x * per, t1 = min(t0 + per, n_tiles);
    unsigned a = 0, b = 0;
    for (int t = t0; t < t1; ++t) { a += count[t]; b += (count[t] + slice - 1) / slice; }
    s_a[threadIdx.x] = a;
    s_b[threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned ra = 0, rb = 0;
        for (unsigned i = 0; i < blockDim.x; ++i) {
            const unsigned va = s_a[i], vb = s_b[i];
            s_a[i] = ra; s_b[i] = rb;
            ra += va; rb += vb;
        }
        work[0] = rb;          // work items
        work[1] = 0;           // work counter
        off[n_tiles] = ra;
        work_off[n_tiles] = rb;
    }
    __syncthreads();
    a = s_a[threadIdx.x];
    b = s_b[threadIdx.x];
    for (int t = t0; t < t1; ++t) {
        off[t] = a;
        work_off[t] = b;
        fill[t] = 0u;
        a += count[t];
        b += (count[t] + slice - 1) / slice;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned rp = 0;
        for (int y = 0; y < g.tiles_y; ++y) {
            band_part_off[y] = rp;
            band_fill[y] = 0u;
            const unsigned n = off[(y + 1) * g.tiles_x] - off[y * g.tiles_x];
            rp += (n + range - 1) / range;
        }
        band_part_off[g.tiles_y] = rp;
    }
}

// Pass A: block (segment, part) takes `range` records of a segment, groups
// them by band of 64 rows in shared memory and writes each band's run
// contiguously (coalesced) at the band's next free place in `tmp`.
__global__ void k_band_scatter(const u64t* __restrict__ rec, u64t seg_cap, int parts, const unsigned* __restrict__ seg_n,
                               TileGeom g, unsigned range, const unsigned* __restrict__ off, unsigned* __restrict__ band_fill,
                               u64t* __restrict__ tmp) {
    extern __shared__ u64t s_stage[];                          // [range]
    unsigned short* s_band = reinterpret_cast<unsigned short*>(s_stage + range);
    __shared__ unsigned s_cnt[kMaxBands], s_loc[kMaxBands], s_base[kMaxBands];
    const int sg = blockIdx.x / parts, part = blockIdx.x % parts;
    const u64t n_seg = min((u64t)seg_n[sg], seg_cap);
    const u64t r0 = (u64t)part * range;
    if (r0 >= n_seg) return;
    const unsigned n = (unsigned)min((u64t)range, n_seg - r0);
    const u64t* r = rec + (u64t)sg * seg_cap + r0;
    const int nb = g.tiles_y;
    for (int y = threadIdx.x; y < nb; y += blockDim.x) s_cnt[y] = 0u;
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&s_cnt[((unsigned)r[i] / (unsigned)g.w) >> 6], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int y = 0; y < nb; ++y) { s_loc[y] = acc; acc += s_cnt[y]; }
    }
    __syncthreads();
    for (int y = threadIdx.x; y < nb; y += blockDim.x) {
        const unsigned c = s_cnt[y];
        if (c) s_base[y] = off[y * g.tiles_x] + atomicAdd(&band_fill[y], c);
        s_cnt[y] = 0u;
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        const u64t v = r[i];
        const unsigned y = ((unsigned)v / (unsigned)g.w) >> 6;
        const unsigned pos = s_loc[y] + atomicAdd(&s_cnt[y], 1u);
        s_stage[pos] = v;
        s_band[pos] = (unsigned short)y;
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned y = s_band[i];
        tmp[s_base[y] + (i - s_loc[y])] = s_stage[i];
    }
}

// Pass B: work item (band, part) takes `range` records of one band of `tmp`,
// groups them by tile column and writes each tile's run contiguously as
// 4-byte records (tile-local pixel | palette index << 12).
__global__ void k_tile_scatter(const u64t* __restrict__ tmp, TileGeom g, unsigned range, const unsigned* __restrict__ off,
                               const unsigned* __restrict__ band_part_off, unsigned* __restrict__ fill, unsigned* __restrict__ sorted) {
    extern __shared__ unsigned s_st[];                         // [range]
    unsigned short* s_col = reinterpret_cast<unsigned short*>(s_st + range);
    __shared__ unsigned s_cnt[kMaxCols], s_loc[kMaxCols], s_base[kMaxCols];
    const unsigned item = blockIdx.x;
    if (item >= band_part_off[g.tiles_y]) return;
    int lo = 0, hi = g.tiles_y - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (band_part_off[mid] <= item) lo = mid; else hi = mid - 1;
    }
    const int y = lo;
    const unsigned b0 = off[y * g.tiles_x], b1 = off[(y + 1) * g.tiles_x];
    const unsigned r0 = b0 + (item - band_part_off[y]) * range;
    const unsigned n = min(range, b1 - r0);
    const int nc = g.tiles_x;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) s_cnt[c] = 0u;
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&s_cnt[((unsigned)tmp[r0 + i] % (unsigned)g.w) >> 6], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int c = 0; c < nc; ++c) { s_loc[c] = acc; acc += s_cnt[c]; }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        const unsigned k = s_cnt[c];
        if (k) s_base[c] = off[y * g.tiles_x + c] + atomicAdd(&fill[y * g.tiles_x + c], k);
        s_cnt[c] = 0u;
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        const u64t v = tmp[r0 + i];
        unsigned local;
        const unsigned t = tile_of((unsigned)v, g, local);
        const unsigned c = t - (unsigned)(y * g.tiles_x);
        const unsigned pos = s_loc[c] + atomicAdd(&s_cnt[c], 1u);
        s_st[pos] = local | ((unsigned)(v >> 32) << 12);
        s_col[pos] = (unsigned short)c;
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned c = s_col[i];
        sorted[s_base[c] + (i - s_loc[c])] = s_st[i];
    }
}

// 64-bit sums from 32-bit shared-memory atomics: add to the low word and
// carry into the high word when it wraps (seen in the returned old value).
__device__ __forceinline__ void add64_lohi(unsigned* lo, unsigned* hi, unsigned v) {
    const unsigned old = atomicAdd(lo, v);
    if (old + v < old) atomicAdd(hi, 1u);
}

__global__ void __launch_bounds__(512) k_tile_accumulate(const unsigned* __restrict__ sorted, const unsigned* __restrict__ off,
                                                         const unsigned* __restrict__ work_off, unsigned* __restrict__ work,
                                                         unsigned slice, const uint4* __restrict__ pal_fx,
                                                         TileGeom g, ulonglong4* __restrict__ hist) {
    extern __shared__ unsigned s_acc[];
    unsigned* s_n = s_acc;                                // [4096] each: count, then (lo, hi) of r, g, b
    unsigned* s_rl = s_n + 4096;
    unsigned* s_rh = s_rl + 4096;
    unsigned* s_gl = s_rh + 4096;
    unsigned* s_gh = s_gl + 4096;
    unsigned* s_bl = s_gh + 4096;
    unsigned* s_bh = s_bl + 4096;
    __shared__ unsigned s_item;
    const unsigned items = work[0];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(&work[1], 1u);
        for (int i = threadIdx.x; i < 7 * 4096; i += blockDim.x) s_acc[i] = 0u;
        __syncthreads();
        const unsigned item = s_item;
        if (item >= items) break;
        // The tile owning this work item: last t with work_off[t] <= item.
        int lo = 0, hi = g.n_tiles - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (work_off[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const int t = lo;
        const unsigned slices = work_off[t + 1] - work_off[t];
        const unsigned k = item - work_off[t];
        const unsigned i0 = off[t] + k * slice, i1 = min(i0 + slice, off[t + 1]);
        for (unsigned i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const unsigned v = sorted[i];
            const unsigned li = v & 4095u;
            const uint4 c = __ldg(pal_fx + (v >> 12));           // palette colour in 2^-24 units (L1)
            atomicAdd(&s_n[li], 1u);
            add64_lohi(&s_rl[li], &s_rh[li], c.x);
            add64_lohi(&s_gl[li], &s_gh[li], c.y);
            add64_lohi(&s_bl[li], &s_bh[li], c.z);
        }
        __syncthreads();
        const int tx = t % g.tiles_x, ty = t / g.tiles_x;
        for (int li = threadIdx.x; li < 4096; li += blockDim.x) {
            const unsigned n = s_n[li];
            if (!n) continue;
            const int x = tx * 64 + (li & 63), y = ty * 64 + (li >> 6);
            ulonglong4* p = hist + (size_t)y * g.w + x;
            const u64t r = ((u64t)s_rh[li] << 32) | s_rl[li], gg = ((u64t)s_gh[li] << 32) | s_gl[li];
            const u64t b = ((u64t)s_bh[li] << 32) | s_bl[li];
            if (slices == 1) {
                ulonglong4 h = *p;
                h.x += r; h.y += gg; h.z += b; h.w += n;
                *p = h;
            } else {
                u64t* q = reinterpret_cast<u64t*>(p);
                atomicAdd(q + 0, r);
                atomicAdd(q + 1, gg);
                atomicAdd(q + 2, b);
                atomicAdd(q + 3, (u64t)n);
            }
        }
    }
}

// The u32-count / FP32-colour histogram's slices: the tile's pixels as
// shared-memory bins (u32 count, FP32 r, g, b: 64 KB), summed with shared
// atomics, then added to the histogram -- one 16-byte read-modify-write a
// pixel when the tile is one slice, atomics when a hot tile is split over
// several (its slices run in any order on any block).
__global__ void __launch_bounds__(512) k_tile_accumulate_f32(const unsigned* __restrict__ sorted, const unsigned* __restrict__ off,
                                                             const unsigned* __restrict__ work_off, unsigned* __restrict__ work,
                                                             unsigned slice, const float4* __restrict__ pal, TileGeom g,
                                                             float4* __restrict__ hist) {
    extern __shared__ unsigned s_acc[];
    unsigned* s_n = s_acc;                                        // [4096] counts
    float* s_r = reinterpret_cast<float*>(s_n + 4096);            // [4096] each: r, g, b sums
    float* s_g = s_r + 4096;
    float* s_b = s_g + 4096;
    __shared__ unsigned s_item;
    const unsigned items = work[0];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(&work[1], 1u);
        for (int i = threadIdx.x; i < 4 * 4096; i += blockDim.x) s_acc[i] = 0u;
        __syncthreads();
        const unsigned item = s_item;
        if (item >= items) break;
        int lo = 0, hi = g.n_tiles - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (work_off[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const int t = lo;
        const unsigned slices = work_off[t + 1] - work_off[t];
        const unsigned k = item - work_off[t];
        const unsigned i0 = off[t] + k * slice, i1 = min(i0 + slice, off[t + 1]);
        for (unsigned i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const unsigned v = sorted[i];
            const unsigned li = v & 4095u;
            const float4 c = __ldg(pal + (v >> 12));                // linear palette colour (L1)
            atomicAdd(&s_n[li], 1u);
            atomicAdd(&s_r[li], c.x);
            atomicAdd(&s_g[li], c.y);
            atomicAdd(&s_b[li], c.z);
        }
        __syncthreads();
        const int tx = t % g.tiles_x, ty = t / g.tiles_x;
        for (int li = threadIdx.x; li < 4096; li += blockDim.x) {
            const unsigned n = s_n[li];
            if (!n) continue;
            const int x = tx * 64 + (li & 63), y = ty * 64 + (li >> 6);
            float4* p = hist + (size_t)y * g.w + x;
            if (slices == 1) {
                float4 h = *p;
                h.x += s_r[li]; h.y += s_g[li]; h.z += s_b[li];
                h.w = __uint_as_float(__float_as_uint(h.w) + n);
                *p = h;
            } else {
                float* q = reinterpret_cast<float*>(p);
                atomicAdd(q + 0, s_r[li]);
                atomicAdd(q + 1, s_g[li]);
                atomicAdd(q + 2, s_b[li]);
                atomicAdd(reinterpret_cast<unsigned*>(q + 3), n);
            }
        }
    }
}

// The palette's colours as the exact splat's integers: round(c * 2^24).
__global__ void k_pal_fixed(const float4* __restrict__ pal, int n, uint4* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = pal[i];
        out[i] = make_uint4(__float2uint_rn(c.x * 16777216.0f), __float2uint_rn(c.y * 16777216.0f),
                            __float2uint_rn(c.z * 16777216.0f), 0u);
    }
}

}  // namespace

cudaError_t launch_tile_pass(const unsigned long long* rec, unsigned long long seg_cap, int n_segs, const TileGeom& g,
                             unsigned slice, unsigned* count, unsigned* off, unsigned* fill, unsigned* work_off, unsigned* work,
                             unsigned* band_fill, unsigned* band_part_off, unsigned long long* tmp, unsigned* sorted,
                             const float4* pal, int pal_n, void* hist, bool exact, int n_sm, cudaStream_t s) {
    const unsigned* seg_n = reinterpret_cast<const unsigned*>(rec + seg_cap * (unsigned long long)n_segs);
    cudaError_t e;
    if (g.n_tiles > kMaxTiles || g.tiles_y > kMaxBands || g.tiles_x > kMaxCols || pal_n > 1024) return cudaErrorInvalidValue;
    const unsigned range = 8192;
    const size_t smem_a = (size_t)range * 10, smem_b = (size_t)range * 6;
    const size_t smem_c = (size_t)g.n_tiles * 4, smem_acc = 7 * 4096 * 4;
    // After the band work list, rounded up to 16 bytes (the scratch has the slack).
    uint4* pal_fx = reinterpret_cast<uint4*>((reinterpret_cast<uintptr_t>(band_part_off + kMaxBands + 1) + 15) & ~(uintptr_t)15);
    if ((e = cudaFuncSetAttribute(k_tile_count, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxTiles * 4)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_band_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_tile_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b)) != cudaSuccess) return e;
    const size_t smem_f32 = 4 * 4096 * 4;
    if (exact && (e = cudaFuncSetAttribute(k_tile_accumulate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_acc)) != cudaSuccess)
        return e;
    if (!exact && (e = cudaFuncSetAttribute(k_tile_accumulate_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_f32)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(count, 0, (size_t)g.n_tiles * 4, s)) != cudaSuccess) return e;
    k_tile_count<<<std::min(n_sm * 4, n_segs), 512, smem_c, s>>>(rec, seg_cap, n_segs, seg_n, g, count);
    k_tile_scan<<<1, 1024, 0, s>>>(count, g, slice, range, off, fill, work_off, work, band_fill, band_part_off);
    const int parts = (int)((seg_cap + range - 1) / range);
    k_band_scatter<<<n_segs * parts, 512, smem_a, s>>>(rec, seg_cap, parts, seg_n, g, range, off, band_fill, tmp);
    const unsigned long long total_cap = seg_cap * (unsigned long long)n_segs;
    const unsigned items_max = (unsigned)((total_cap + range - 1) / range) + (unsigned)g.tiles_y;
    k_tile_scatter<<<items_max, 512, smem_b, s>>>(tmp, g, range, off, band_part_off, fill, sorted);
    if (exact) {
        k_pal_fixed<<<(pal_n + 255) / 256, 256, 0, s>>>(pal, pal_n, pal_fx);
        k_tile_accumulate<<<n_sm * 2, 512, smem_acc, s>>>(sorted, off, work_off, work, slice, pal_fx, g,
                                                          static_cast<ulonglong4*>(hist));
    } else {
        k_tile_accumulate_f32<<<n_sm * 3, 512, smem_f32, s>>>(sorted, off, work_off, work, slice, pal, g, static_cast<float4*>(hist));
    }
    return cudaGetLastError();
}

}  // namespace ffb
