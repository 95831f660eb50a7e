// ffb_runtime.cpp -- the render driver and the C ABI (include/ffb200.h).
//
// FlameRenderer's job (src/renderer/compute_kernel.rs:374-3600,
// src/renderer/render.rs:371-804) done the B200 way: the flame is parsed
// on the host, its structure compiled once by NVRTC for sm_100a (kept in a
// module cache, the counterpart of src/shader_cache.rs), its numbers
// uploaded as a small table; one persistent-walker launch runs the whole
// sample budget (the reference's host loop of ~120 dispatches with an
// accumulate pass every 4 becomes a handful of launches into one exact-count
// histogram), and one fused kernel tone-maps (and 2x-downsamples) it.
// No CPU fallback: without a CUDA device every call fails.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvrtc.h>

#include "../../include/ffb200.h"
#include "ffb_codegen.hpp"
#include "ffb_flame.hpp"
#include "ffb_json.hpp"
#include "ffb_png.hpp"
#include "ffb_flame_xml.hpp"
#include "ffb_tail.cuh"

#define FFB_API extern "C" __attribute__((visibility("default")))

namespace ffb {
namespace {

thread_local std::string g_err;

// Draw words a point of the single-step entries (FFB_APPLY_WORDS on the device).
constexpr size_t kApplyWords = 64;

struct Fail {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string& m) { throw Fail{code, m}; }

void ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    int code = (e == cudaErrorMemoryAllocation) ? FFB_ERR_OUT_OF_MEMORY
               : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? FFB_ERR_NO_DEVICE : FFB_ERR_CUDA;
    fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int guard(F&& f) {
    try {
        f();
        g_err.clear();
        return FFB_OK;
    } catch (const Fail& e) {
        g_err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "out of host memory";
        return FFB_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_err = e.what();
        return FFB_ERR_CONFIG;
    }
}

// Host mirror of the device-side launch record (ffb_kernels.cuh, ffb_launch).
struct Launch {
    const void* table;
    const void* palette;
    void* hist;
    void* walkers;
    void* counters;
    uint32_t n_walkers, walker0, block0, n_xf;
    uint32_t seed_lo, seed_hi, burn_in, ipt;
    uint64_t it0;
    uint32_t n_iters, pal_n;
    int32_t width, height;
    float zoom, pan_x, pan_y, cos_r, sin_r;
    void* rec;          // deferred plotting: the launch's samples
    void* rec_draws;    // and their final chain's draws
    void* state;        // the walkers' variation state (slot-major planes of n_walkers)
    uint32_t ring_prod, ring_depth;   // fused plotting: producer threads a block, iteration slots of the ring
};
static_assert(sizeof(Launch) == 152, "launch record layout");

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    void* ensure(size_t bytes) {
        if (bytes <= n && p) return p;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        ck(cudaMalloc(&p, std::max<size_t>(bytes, 256)), "cudaMalloc");
        n = std::max<size_t>(bytes, 256);
        return p;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

// Page-locked host memory the readback lands in (a copy from the device to
// pageable memory goes through the driver's staging buffer at a fraction of
// the link's rate).
struct HostBuf {
    void* p = nullptr;
    size_t n = 0;
    void* ensure(size_t bytes) {
        if (bytes <= n && p) return p;
        if (p) cudaFreeHost(p);
        p = nullptr; n = 0;
        ck(cudaMallocHost(&p, std::max<size_t>(bytes, 256)), "cudaMallocHost");
        n = std::max<size_t>(bytes, 256);
        return p;
    }
    void release() { if (p) cudaFreeHost(p); p = nullptr; n = 0; }
};

struct Module {
    std::string key;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t chaos = nullptr, chaos_sorted = nullptr, probe = nullptr, apply = nullptr;
    cudaKernel_t plot = nullptr;   // deferred-plot modules only
    cudaKernel_t fused = nullptr;  // deferred-plot modules of the counter-based stream without orbit refresh
    int smem_attr_plot = 0, smem_attr_fused = 0;
    // Differentiable-render modules (ffb_diff.cuh) only.
    cudaKernel_t dforward = nullptr, dadjoint = nullptr, dtheta = nullptr, dprobe = nullptr;
    int smem_attr = 0, smem_attr_sorted = 0, smem_attr_dadj = 0;
    int pins = 0;                  // batches holding this module (not evicted while > 0)
};

std::string nvrtc_options_key() { return "sm_100a|c++17|ftz|prec-div|prec-sqrt|nofmad"; }

// Whether a module's source compiles ffb_chaos_fused (ffb_kernels.cuh): a
// deferred-plot module of the counter-based stream without orbit refresh.
bool fused_capable(const std::string& src) {
    return src.find("#define FFB_DEFER 1") != std::string::npos && src.find("#define FFB_RNG_MODE 1") != std::string::npos &&
           src.find("#define FFB_REFRESH") == std::string::npos;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

// Objects that borrow a renderer's modules: when the renderer goes first it
// orphans them (their modules are unloaded with it), so destroying them
// later frees only their own device memory and touches nothing else.
static void batch_orphan(ffb_batch* b);
static void diff_orphan(ffb_diff* d);

struct ffb_renderer {
    int device = 0;
    int n_sm = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    std::list<Module> cache;     // most recent first
    DevBuf hist, walkers, table, palette, counters, jobs, rgba, de_out, de_tab, lut, f_out, tmp_in;
    DevBuf tile_rec, tile_tmp, tile_sorted, tile_meta;      // tile-sorted accumulation scratch
    DevBuf filt_batch, filt_tmp;                            // spatial filter: a batch's histogram, the row pass
    DevBuf vstate;                                          // stateful variations / subflames: per-walker state
    HostBuf readback;                                       // fae_call's RGBA8 on its way to the caller
    // Deferred plotting: the plot kernel's stream, double-buffered sample
    // records, events ordering the two streams.
    cudaStream_t plot_stream = nullptr;
    cudaEvent_t ev_main[2] = {nullptr, nullptr}, ev_plot[2] = {nullptr, nullptr}, ev_start = nullptr;
    DevBuf rec[2], rec_draws[2];
    cudaEvent_t ev_flight[2] = {nullptr, nullptr};          // RenderProgress: launches in flight
    // ffb_plot_bench: when set, each plot launch runs after its chaos launch
    // on the render's stream and its device time is added here.
    double* plot_timing = nullptr;
    cudaEvent_t ev_p[2] = {nullptr, nullptr};
    void ensure_flight_events() {
        for (auto& e : ev_flight)
            if (!e) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    }
    void ensure_plot_stream() {
        if (plot_stream) return;
        ck(cudaStreamCreateWithFlags(&plot_stream, cudaStreamNonBlocking), "plot stream");
        for (int i = 0; i < 2; ++i) {
            ck(cudaEventCreateWithFlags(&ev_main[i], cudaEventDisableTiming), "event");
            ck(cudaEventCreateWithFlags(&ev_plot[i], cudaEventDisableTiming), "event");
        }
        ck(cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming), "event");
    }
    uint64_t h2d = 0, d2h = 0;      // bytes copied by the current call
    uint32_t launches = 0;          // kernels launched by the current call
    std::set<ffb_batch*> batches;   // live objects borrowing this renderer's modules
    std::set<ffb_diff*> diffs;

    void reset_counts() { h2d = d2h = 0; launches = 0; }
    void fill_counts(ffb_output* o) const { if (o) { o->h2d_bytes = h2d; o->d2h_bytes = d2h; o->kernel_launches = launches; } }

    ~ffb_renderer() {
        cudaSetDevice(device);
        cudaDeviceSynchronize();
        for (ffb_batch* b : batches) batch_orphan(b);
        for (ffb_diff* d : diffs) diff_orphan(d);
        batches.clear();
        diffs.clear();
        if (stream) cudaStreamSynchronize(stream);
        for (auto& m : cache) if (m.lib) cudaLibraryUnload(m.lib);
        for (DevBuf* b : {&hist, &walkers, &table, &palette, &counters, &jobs, &rgba, &de_out, &de_tab, &lut, &f_out, &tmp_in,
                          &tile_rec, &tile_tmp, &tile_sorted, &tile_meta, &filt_batch, &filt_tmp, &vstate, &rec[0], &rec[1],
                          &rec_draws[0], &rec_draws[1]}) b->release();
        readback.release();
        if (plot_stream) {
            cudaStreamSynchronize(plot_stream);
            for (int i = 0; i < 2; ++i) { cudaEventDestroy(ev_main[i]); cudaEventDestroy(ev_plot[i]); }
            cudaEventDestroy(ev_start);
            cudaStreamDestroy(plot_stream);
        }
        for (auto e : ev_flight) if (e) cudaEventDestroy(e);
        for (auto e : ev_p) if (e) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    Module& module_for(const std::string& src) {
        for (auto it = cache.begin(); it != cache.end(); ++it)
            if (it->key == src) { cache.splice(cache.begin(), cache, it); return cache.front(); }
        Module m;
        m.key = src;
        compile(src, m);
        cache.push_front(std::move(m));
        while (cache.size() > 32) {                         // src/shader_cache.rs keeps an LRU too
            auto victim = cache.end();
            for (auto it = std::prev(cache.end()); ; --it) {
                if (it->pins == 0 && it != cache.begin()) { victim = it; break; }
                if (it == cache.begin()) break;
            }
            if (victim == cache.end()) break;              // everything pinned: keep growing
            if (victim->lib) cudaLibraryUnload(victim->lib);
            cache.erase(victim);
        }
        return cache.front();
    }

    static void compile(const std::string& src, Module& m) {
        std::vector<char> cubin = nvrtc_cubin(src);
        ck(cudaLibraryLoadData(&m.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0), "cudaLibraryLoadData");
        ck(cudaLibraryGetKernel(&m.chaos, m.lib, "ffb_chaos"), "cudaLibraryGetKernel(ffb_chaos)");
        ck(cudaLibraryGetKernel(&m.chaos_sorted, m.lib, "ffb_chaos_sorted"), "cudaLibraryGetKernel(ffb_chaos_sorted)");
        ck(cudaLibraryGetKernel(&m.probe, m.lib, "ffb_probe"), "cudaLibraryGetKernel(ffb_probe)");
        ck(cudaLibraryGetKernel(&m.apply, m.lib, "ffb_apply_points"), "cudaLibraryGetKernel(ffb_apply_points)");
        if (src.find("#define FFB_DEFER 1") != std::string::npos) {
            ck(cudaLibraryGetKernel(&m.plot, m.lib, "ffb_plot"), "cudaLibraryGetKernel(ffb_plot)");
            if (fused_capable(src)) ck(cudaLibraryGetKernel(&m.fused, m.lib, "ffb_chaos_fused"), "cudaLibraryGetKernel(ffb_chaos_fused)");
        }
        if (src.find("ffb_diff_forward") != std::string::npos) {
            ck(cudaLibraryGetKernel(&m.dforward, m.lib, "ffb_diff_forward"), "cudaLibraryGetKernel(ffb_diff_forward)");
            ck(cudaLibraryGetKernel(&m.dadjoint, m.lib, "ffb_diff_adjoint"), "cudaLibraryGetKernel(ffb_diff_adjoint)");
            ck(cudaLibraryGetKernel(&m.dtheta, m.lib, "ffb_diff_theta"), "cudaLibraryGetKernel(ffb_diff_theta)");
            ck(cudaLibraryGetKernel(&m.dprobe, m.lib, "ffb_dprobe"), "cudaLibraryGetKernel(ffb_dprobe)");
        }
    }

    static std::vector<char> nvrtc_cubin(const std::string& src) {
        nvrtcProgram prog;
        if (nvrtcCreateProgram(&prog, src.c_str(), "ffb_flame.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
            fail(FFB_ERR_COMPILE, "nvrtcCreateProgram failed");
        const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--ftz=true", "--prec-div=true",
                              "--prec-sqrt=true", "--fmad=false", "-lineinfo"};
        nvrtcResult r = nvrtcCompileProgram(prog, (int)(sizeof(opts) / sizeof(opts[0])), opts);
        if (r != NVRTC_SUCCESS) {
            size_t n = 0;
            nvrtcGetProgramLogSize(prog, &n);
            std::string log(n, '\0');
            nvrtcGetProgramLog(prog, &log[0]);
            nvrtcDestroyProgram(&prog);
            fail(FFB_ERR_COMPILE, std::string("NVRTC: ") + nvrtcGetErrorString(r) + "\n" + log);
        }
        size_t n = 0;
        nvrtcGetCUBINSize(prog, &n);
        std::vector<char> cubin(n);
        nvrtcGetCUBIN(prog, cubin.data());
        nvrtcDestroyProgram(&prog);
        return cubin;
    }

    void begin() { ck(cudaSetDevice(device), "cudaSetDevice"); }
};

namespace ffb {
namespace {

constexpr uint32_t kMaxDim = 32768;                           // config/defaults.rs MAX_IMAGE_DIM

struct Prepared {
    Flame flame;
    Plan plan;
    std::vector<float> table, palette;
    uint32_t ss = 1, wi = 0, hi = 0, walkers = 0, burn_in = 20, ipt = 1024, threads = 128;
    uint64_t target = 0, per_walker = 0, seed = 0;
    int rng = RNG_PHILOX, math = MATH_PRECISE;
    uint32_t schedule = 0;
    uint32_t count_bits = 32;
    uint32_t accumulate = 0;    // 0 auto, 1 direct, 2 tile-sorted
    bool threads_set = false;   // the job chose the block size (the sorted schedule's sorting group too)
    uint32_t plot = 0;          // 0 auto, 1 inline, 2 deferred (the plot in its own kernel)
    void (*progress)(void*, uint64_t, uint64_t) = nullptr;   // RenderProgress (render.rs:293-301)
    int (*cancelled)(void*) = nullptr;
    void* progress_user = nullptr;
};

// Whether a render accumulates by tiles: tile-sorted accumulation asked
// for -- or auto with a histogram above 512 MB (4x the L2, where the direct
// splat's atomics mostly miss it) -- a tile grid the sort's shared-memory
// counters hold, and a palette of at most 1024 entries.  Measured at
// 7680x4320: exact (1.06 GB), 1e10 samples, 546 ms tiled against 585
// direct; u32 / FP32 (531 MB), 3e9 samples, 213 against 259.  At
// 3840x2160 (u32 / FP32, 133 MB, 1e9 samples) the direct splat, deferred
// beside the walkers, wins: 57 ms against 82.
bool tiled_accumulation(const Prepared& P) {
    if (P.accumulate == 1) return false;
    if (P.flame.color_mode != 0) return false;      // records hold a palette index, not a walker's colour
    const double px_bytes = P.count_bits == 64 ? 32.0 : 16.0;
    if (P.accumulate == 0 && (P.flame.filter.on() || (double)P.wi * (double)P.hi * px_bytes <= 512e6)) return false;
    const int tx = (int)((P.wi + 63) / 64), ty = (int)((P.hi + 63) / 64);
    return tx * ty <= kMaxTiles && tx <= kMaxCols && ty <= kMaxBands && P.flame.palette_size <= 1024;
}

Prepared prepare(const char* config, size_t len, const ffb_job* job, bool need_size = true) {
    if (!config) fail(FFB_ERR_INVALID, "config is NULL");
    if (!job) fail(FFB_ERR_INVALID, "job is NULL");
    Prepared P;
    try { P.flame = parse_config_text(std::string(config, len)); }
    catch (const std::exception& e) {
        std::string m = e.what();
        fail(m.rfind("TooLarge", 0) == 0 ? FFB_ERR_TOO_LARGE : FFB_ERR_CONFIG, "config did not parse: " + m);
    }
    P.ss = job->supersample ? job->supersample : 1;
    if (P.ss != 1 && P.ss != 2) fail(FFB_ERR_INVALID, "supersample must be 1 or 2");
    if (need_size) {
        if (job->width == 0 || job->height == 0) fail(FFB_ERR_INVALID, "width and height must be nonzero");   // render.rs:259-264
        if (job->width > kMaxDim || job->height > kMaxDim) fail(FFB_ERR_TOO_LARGE, "width and height must be at most 32768");
    }
    P.wi = job->width * P.ss;
    P.hi = job->height * P.ss;
    P.rng = job->rng < 0 ? RNG_PHILOX : job->rng;
    if (P.rng != RNG_PCG && P.rng != RNG_PHILOX) fail(FFB_ERR_INVALID, "rng must be 0 (pcg) or 1 (philox)");
    P.math = job->math;
    if (P.math != MATH_PRECISE && P.math != MATH_SFU) fail(FFB_ERR_INVALID, "math must be 0 (precise) or 1 (sfu)");
    P.threads = job->threads ? job->threads : 128;
    P.threads_set = job->threads != 0;
    if (P.threads % 32 || P.threads > 1024) fail(FFB_ERR_INVALID, "threads must be a multiple of 32, at most 1024");
    P.burn_in = job->burn_in ? job->burn_in : 20;
    // An xaos walker's stored state holds its previous transform above the burn-in left.
    if (!P.flame.xaos.empty() && P.burn_in >= (1u << 24)) fail(FFB_ERR_INVALID, "burn_in must be below 2^24 with xaos");
    if (P.flame.orbit_refresh && P.flame.filter.on())
        fail(FFB_ERR_INVALID, "the spatial filter with an xaos chain that needs orbit refresh is not supported by this build");
    P.ipt = job->iterations_per_thread ? job->iterations_per_thread : 1024;
    P.target = job->iterations ? job->iterations : P.flame.max_iterations * (uint64_t)P.ss * P.ss;
    uint64_t w = job->walkers;
    if (!w) w = std::min<uint64_t>(148ull * 2048, std::max<uint64_t>(4096, P.target / 1024));
    w = (w + 31) / 32 * 32;
    if (w > 0xFFFFFFFFull) fail(FFB_ERR_INVALID, "too many walkers");
    P.walkers = (uint32_t)w;
    P.per_walker = (P.target + w - 1) / w;
    if (P.rng == RNG_PCG) {
        // Launch chunks stay on dispatch boundaries of the PCG stream.
        if (P.per_walker + P.burn_in > (uint64_t)P.ipt * 0xFFFFFFFFull) fail(FFB_ERR_INVALID, "budget too large for the pcg stream");
    }
    P.seed = job->seed ? job->seed : P.flame.seed;
    P.schedule = job->schedule;
    if (P.schedule > 2) fail(FFB_ERR_INVALID, "schedule must be 0 (auto), 1 (plain) or 2 (sorted)");
    P.count_bits = job->count_bits ? job->count_bits : 32;
    if (P.count_bits != 32 && P.count_bits != 64) fail(FFB_ERR_INVALID, "count_bits must be 32 or 64");
    P.accumulate = job->accumulate;
    if (P.accumulate > 2) fail(FFB_ERR_INVALID, "accumulate must be 0 (auto), 1 (direct) or 2 (tile-sorted)");
    if (P.accumulate == 2 && P.flame.color_mode != 0)
        fail(FFB_ERR_INVALID, "tile-sorted accumulation records palette indices: not with the speed colour mode");
    if (P.accumulate == 2 && P.flame.filter.on())
        fail(FFB_ERR_INVALID, "tile-sorted accumulation adds into the render's histogram: not with the spatial filter's batches");
    P.plot = job->plot;
    if (P.plot > 3) fail(FFB_ERR_INVALID, "plot must be 0 (auto), 1 (inline), 2 (deferred) or 3 (fused)");
    P.progress = job->progress;
    P.cancelled = job->cancelled;
    P.progress_user = job->progress_user;
    const bool tiled = tiled_accumulation(P);
    // Deferred plotting needs the counter-based stream (a launch of any
    // length resumes it) and plots straight into the histogram.
    // Auto: deferred for the sorted schedule over enough walkers to fill
    // the machine (measured on the 1080p ss2 frame: 51 ms against 66).
    const bool can_defer = P.rng == RNG_PHILOX && !tiled && !P.flame.filter.on() && P.walkers <= (1u << 23);
    const bool defer = can_defer && (P.plot >= 2 || (P.plot == 0 && P.schedule != 1 && P.walkers >= 16384));
    P.plan = make_plan(P.flame, P.rng, P.math, 0, P.threads_set ? P.threads : 128, false, P.count_bits == 64, 0, 0, tiled, defer);
    P.table = make_table(P.plan, P.flame);
    P.palette = palette_table(P.flame);
    return P;
}

// The tone map's constants (tonemap.wgsl:94-112, 224-590;
// compute_kernel.rs:1796-1866, 3813-3866), in double, for a render at
// wi x hi with `samples` plotted samples.
TonemapArgs tonemap_args(const Flame& f, uint32_t wi, uint32_t hi, double sample_density, int transparent, bool count_is_float) {
    const ToneMap& t = f.tm;
    TonemapArgs a{};
    a.mode = t.mode;
    a.highlight = t.highlight;
    a.use_curve = t.use_curve ? 1 : 0;
    a.transparent = transparent;
    a.levels_enabled = t.levels_enabled ? 1 : 0;
    a.count_is_float = count_is_float ? 1 : 0;
    a.exposure = t.exposure;
    const double g = t.gamma == 0.0f ? (double)t.gamma : 1.0 / (double)t.gamma;
    a.inv_gamma = (float)g;
    a.density_scale = t.density_scale;
    const double ppu = (double)std::min(wi, hi) * 0.25 * (double)f.zoom;
    const double area = (double)wi * (double)hi / (ppu * ppu);
    const double pw = 67108864.0, bright_adjust = 2.3;
    const double k1 = bright_adjust * (double)t.brightness * 268.0 * pw / 256.0;
    const double k2 = 1.0 / (area * (double)t.white_level * sample_density);
    a.ls_a = (float)(k1 / (pw * std::log(10.0)));
    a.ls_b = (float)((double)t.white_level * k2);
    a.white_level = t.white_level;
    a.gamma_threshold = t.gamma_threshold;
    a.funcval = t.gamma_threshold != 0.0f ? (float)std::pow((double)t.gamma_threshold, g - 1.0) : 0.0f;
    const double vib = std::nearbyint((double)t.vibrancy * 256.0);
    a.vib = (float)vib;
    a.notvib = (float)(256.0 - vib);
    a.saturation = t.saturation;
    a.hue_shift = t.hue_shift;
    a.alpha_blend_low = t.alpha_blend_low;
    a.alpha_blend_high = t.alpha_blend_high;
    a.levels_low = t.levels_low;
    a.levels_high = t.levels_high;
    a.levels_gamma = t.levels_gamma;
    a.levels_density = (float)sample_density;
    for (int k = 0; k < 3; ++k) a.bg_lin[k] = (float)std::pow(std::max((double)t.background[k], 0.0), 2.2);
    return a;
}

// Density-estimation table (see ffb_tail.cu): entry c for counts 0..n-2,
// entry n-1 for every larger count.
std::vector<float> de_table(double r_max, double r_min, double curve, int& n_out, int& radius) {
    radius = (int)std::floor(r_max);
    auto h_of = [&](double c) { return std::max(r_min, r_max / std::pow(c, curve)); };
    std::vector<float> t;
    int c = 0;
    for (;; ++c) {
        double h = c == 0 ? 0.0 : h_of((double)c);
        double h2 = h * h;
        double dmax2 = c == 0 ? -1.0 : std::floor(h2);
        double norm = 0.0;
        int rr = (int)std::floor(std::sqrt(std::max(dmax2, 0.0)));
        for (int dy = -rr; dy <= rr; ++dy)
            for (int dx = -rr; dx <= rr; ++dx) {
                double d2 = dx * dx + dy * dy;
                if (d2 <= h2) norm += std::exp(-4.5 * d2 / h2);
            }
        if (c == 0) norm = 1.0;
        t.push_back((float)dmax2);
        t.push_back(h2 > 0 ? (float)(1.0 / h2) : 0.0f);
        t.push_back((float)(1.0 / norm));
        t.push_back((float)rr);                        // the disc's reach in whole pixels
        // Past this count every larger one has the same disc and weights.
        if (c >= 1 && (h < 1.0 || h <= r_min)) break;
        if (c > 10000000) fail(FFB_ERR_INVALID, "density estimation table too large");
    }
    n_out = (int)(t.size() / 4);
    return t;
}

void check_de(const Flame& f, uint32_t ss) {
    if (f.de.max_radius * ss > 36.0f) fail(FFB_ERR_INVALID, "density estimation radius too large (at most 36 histogram pixels)");
}

// The render's plotted samples -- each walker's iterations past its burn-in
// (OrbitFuses::dispatch, compute_kernel.rs:85-101).  With orbit refresh a
// walker restarted at dispatch d (every ipt iterations, (w + seed_d) %
// period == 0, seed_d = seed + d * 2654435761) burns in again.
uint64_t plotted_samples(const Prepared& P, uint32_t walker0) {
    const uint32_t period = P.flame.orbit_refresh;
    if (!period || P.ipt == 0) return (uint64_t)P.walkers * P.per_walker;
    const uint64_t total = P.per_walker + P.burn_in, ipt = P.ipt;
    uint64_t plotted = 0;
    for (uint32_t w = 0; w < P.walkers; ++w) {
        const uint32_t gw = walker0 + w;
        uint64_t left = P.burn_in;
        for (uint64_t it0 = 0; it0 < total; it0 += ipt) {
            const uint64_t n = std::min(ipt, total - it0);
            const uint32_t seed_d = (uint32_t)P.seed + (uint32_t)(it0 / ipt) * 2654435761u;
            if (it0 > 0 && (gw + seed_d) % period == 0u) left = P.burn_in;
            const uint64_t burnt = std::min(left, n);
            plotted += n - burnt;
            left -= burnt;
        }
    }
    return plotted;
}

// The in-frame count a render read back.  Bit 63 is set by a kernel whose
// bounded wait gave up (ffb_chaos_fused's hand-over): the render is void.
void check_inframe(uint64_t v) {
    if (v >> 63) fail(FFB_ERR_CUDA, "the fused plot hand-over timed out on the device; the render is incomplete");
}

// Fused plotting's block shape: consumer threads (the plot warps) beside the
// producers, ring slots (iterations in flight between the two), iterations
// a launch.
#ifndef FFB_FUSED_CONSUMERS
#define FFB_FUSED_CONSUMERS 576
#endif
#ifndef FFB_FUSED_RING
#define FFB_FUSED_RING 8
#endif
constexpr uint32_t kFusedConsumers = FFB_FUSED_CONSUMERS;
constexpr uint32_t kFusedRing = FFB_FUSED_RING;
constexpr uint64_t kFusedIters = 4096;

// Shared memory of ffb_chaos_fused after its table and palette (the layout
// ffb_kernels.cuh carves): mbarriers, the abort word, counters, two sets of ten walker
// planes, padding to 16 bytes, the record ring and its draw planes.
int fused_smem_bytes(uint32_t prod, uint32_t ring, int nc, int nfd) {
    return (int)(2 * ring * 8 + 8 + 5 * (uint32_t)nc * 4 + 2 * 10 * prod * 4 + 16 + ring * prod * 16 + (uint32_t)nfd * ring * prod * 4);
}

// Chaos game of a prepared flame into r->hist (wi*hi float4, cleared here).
void run_chaos(ffb_renderer* r, const Prepared& P, cudaStream_t s, uint32_t walker0, uint64_t* inframe_out,
               float4* ext_hist = nullptr) {
    Module& m = r->module_for(P.plan.source);
    const size_t npx = (size_t)P.wi * P.hi;
    // Exact mode: four u64 a pixel (ulonglong4); otherwise float4.
    const size_t px_bytes = P.plan.exact ? 32 : 16;
    const bool filt = P.flame.filter.on();
    if (filt && (ext_hist || P.plan.exact))
        fail(FFB_ERR_INVALID, "the spatial filter (filter_radius) works on this library's own u32 histogram: "
                              "not with count_bits 64 or a caller's device histogram");
    float4* hist = ext_hist ? ext_hist : (float4*)r->hist.ensure(npx * px_bytes);
    ck(cudaMemsetAsync(hist, 0, npx * px_bytes, s), "clear histogram");
    // Spatial filter (compute_kernel.rs:1663-1725): each batch splats into
    // its own histogram, which is filtered and added into `hist` (counts as
    // float).  A batch is `ipt` iterations of every walker, the reference's
    // dispatch.
    float4* batch = filt ? (float4*)r->filt_batch.ensure(npx * 16) : nullptr;
    float4* ftmp = filt ? (float4*)r->filt_tmp.ensure(npx * 16) : nullptr;
    void* d_table = r->table.ensure(P.table.size() * 4);
    ck(cudaMemcpyAsync(d_table, P.table.data(), P.table.size() * 4, cudaMemcpyHostToDevice, s), "upload table");
    r->h2d += P.table.size() * 4;
    void* d_pal = r->palette.ensure(P.palette.size() * 4);
    ck(cudaMemcpyAsync(d_pal, P.palette.data(), P.palette.size() * 4, cudaMemcpyHostToDevice, s), "upload palette");
    r->h2d += P.palette.size() * 4;
    void* d_walk = r->walkers.ensure((size_t)P.walkers * 16);
    uint64_t* d_cnt = (uint64_t*)r->counters.ensure(64);
    ck(cudaMemsetAsync(d_cnt, 0, 64, s), "clear counters");
    const uint32_t pal_n = (uint32_t)(P.palette.size() / 4);
    const bool sorted = P.schedule != 1;
    // Sorted schedule: about one block a multiprocessor holding its share
    // of the walkers (the regrouping works within a block).
    uint32_t threads = P.threads;
    if (sorted) {
        uint32_t per_sm = (P.walkers + (uint32_t)r->n_sm - 1) / (uint32_t)r->n_sm;
        threads = std::min<uint32_t>(1024, std::max<uint32_t>(64, (per_sm + 31) / 32 * 32));
        if (P.threads_set) threads = std::min<uint32_t>(1024, std::max<uint32_t>(32, (P.threads + 31) / 32 * 32));
    }
    // Fused plotting (ffb_job.plot 3): producer warps (the sorted walkers)
    // and consumer warps (the plot) in one block, the samples handed over in
    // shared memory.  The deferred-plot module carries the kernel.
    const bool fused = P.plan.defer && P.plot == 3 && sorted && m.fused != nullptr;
    uint32_t consumers = 0, ring = 0;
    if (fused) {
        consumers = kFusedConsumers;
        ring = kFusedRing;
        uint32_t per_sm = (P.walkers + (uint32_t)r->n_sm - 1) / (uint32_t)r->n_sm;
        threads = std::min<uint32_t>(1024 - consumers, std::max<uint32_t>(64, (per_sm + 31) / 32 * 32));
        if (P.threads_set) threads = std::min<uint32_t>(1024 - consumers, std::max<uint32_t>(32, (P.threads + 31) / 32 * 32));
    }
    int smem = ((P.plan.table_size + 3) / 4) * 16 + (int)pal_n * 16;
    int nfd_fused = 0;
    if (fused) {
        for (auto& fi : P.plan.fin) for (const VarDef* v : fi.vars) nfd_fused += v->draws;
        // A shallower ring where a deep one would not fit the 227 KB of a block.
        while (ring > 2 && smem + fused_smem_bytes(threads, ring, P.plan.maxx + 1, nfd_fused) > 227 * 1024) ring /= 2;
        smem += fused_smem_bytes(threads, ring, P.plan.maxx + 1, nfd_fused);
    } else if (sorted) {
        smem += (int)threads * 8 * 4 + 2 * (P.plan.maxx + 1) * 4;
    }
    const void* kfn = fused ? (const void*)m.fused : sorted ? (const void*)m.chaos_sorted : (const void*)m.chaos;
    int& attr = fused ? m.smem_attr_fused : sorted ? m.smem_attr_sorted : m.smem_attr;
    if (smem > 48 * 1024 && attr < smem) {
        ck(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attribute");
        attr = smem;
    }
    const uint64_t total_iters = P.per_walker + P.burn_in;
    uint64_t chunk = 1ull << 16;
    if (P.rng == RNG_PCG) {
        if (chunk < P.ipt) fail(FFB_ERR_INVALID, "the pcg stream's dispatch does not fit a launch");
        chunk = chunk / P.ipt * P.ipt;
    }
    if (filt) chunk = P.ipt;
    // Deferred plotting: launches of kDeferIters iterations, each followed
    // by the plot of its samples on the plot stream, which overlaps the
    // next launch (two record buffers).  The plot kernel runs two blocks of
    // 384 threads a multiprocessor: with the sorted chaos kernel's block
    // (448 threads x 48 registers) that is 1216 threads and 51K registers,
    // so both stay resident (measured 1080p ss2 frames: one plot block
    // 58.6 ms, two 54.2, three -- which no longer fit beside the chaos
    // block -- 55.5-57.8, eight 77.7; 256 iterations a launch measured best
    // of 64-512).
    const bool defer = P.plan.defer && !fused;
    constexpr uint64_t kDeferIters = 256;
    constexpr unsigned kPlotThreads = 384;
#ifndef FFB_PLOT_BLOCKS
#define FFB_PLOT_BLOCKS 2
#endif
    constexpr unsigned kPlotBlocksPerSm = FFB_PLOT_BLOCKS;
    // At most 2^27 records (2 GiB) a buffer.
    if (defer) chunk = std::max<uint64_t>(16, std::min<uint64_t>(kDeferIters, (1ull << 27) / P.walkers));
    if (fused) chunk = kFusedIters;
    const uint32_t blocks = (P.walkers + threads - 1) / threads;
    const double rot = P.flame.rotation;
    Launch L{};
    L.table = d_table; L.palette = d_pal; L.hist = filt ? batch : hist; L.walkers = d_walk; L.counters = d_cnt;
    L.n_walkers = P.walkers; L.walker0 = walker0; L.block0 = 0; L.n_xf = (uint32_t)P.flame.xf.size();
    // Stateful variations and subflames: their slots of every walker (set
    // by the first launch, carried between launches like the walkers).
    L.state = P.plan.n_state > 0 ? r->vstate.ensure((size_t)P.walkers * (size_t)P.plan.n_state * 4) : nullptr;
    L.seed_lo = (uint32_t)P.seed; L.seed_hi = (uint32_t)(P.seed >> 32); L.burn_in = P.burn_in; L.ipt = P.ipt;
    L.pal_n = pal_n; L.width = (int32_t)P.wi; L.height = (int32_t)P.hi;
    L.zoom = P.flame.zoom; L.pan_x = (float)P.flame.pan_x; L.pan_y = (float)P.flame.pan_y;
    L.cos_r = (float)std::cos(rot); L.sin_r = (float)std::sin(rot);
    L.ring_prod = fused ? threads : 0;
    L.ring_depth = fused ? ring : 0;
    // Tile-sorted accumulation: launches sized so one launch's records (one
    // a walker slot, iteration and symmetry copy at most) fit the record
    // buffer, about 2^29 of them; each launch is followed by the
    // sort-and-sum pass into the exact histogram.
    TileGeom tg{};
    uint64_t cap = 0;
    if (P.plan.emit) {
        const uint64_t copies = (uint64_t)P.flame.sym.copies();
        uint64_t per = std::max<uint64_t>(64, (1ull << 29) / ((uint64_t)blocks * threads * copies)) / 64 * 64;
        if (P.rng == RNG_PCG) per = std::max<uint64_t>(P.ipt, per / P.ipt * P.ipt);
        chunk = std::min<uint64_t>(chunk, per);
        // One segment a block: its threads x the launch's iterations x copies.
        cap = (uint64_t)blocks * threads * std::min<uint64_t>(chunk, total_iters) * copies;
        if (cap >= (1ull << 32)) fail(FFB_ERR_TOO_LARGE, "too many walkers for tile-sorted accumulation");
        tg.w = (int)P.wi; tg.h = (int)P.hi;
        tg.tiles_x = (int)((P.wi + 63) / 64); tg.tiles_y = (int)((P.hi + 63) / 64);
        tg.n_tiles = tg.tiles_x * tg.tiles_y;
        r->tile_rec.ensure(cap * 8 + (size_t)blocks * 4);
        r->tile_tmp.ensure(cap * 8);
        r->tile_sorted.ensure(cap * 4);
        r->tile_meta.ensure(((size_t)tg.n_tiles * 4 + 4 + (size_t)tg.tiles_y + kMaxBands + 1) * 4 + 16 + 1024 * 16);
        L.hist = r->tile_rec.p;
    }
    const size_t n_chunks = (size_t)((total_iters + chunk - 1) / chunk);
    Launch* d_jobs = (Launch*)r->jobs.ensure(sizeof(Launch) * std::max<size_t>(1, n_chunks));
    int nfd = 0;
    if (defer) {
        for (auto& fi : P.plan.fin) for (const VarDef* v : fi.vars) nfd += v->draws;
        const size_t nrec = (size_t)chunk * P.walkers;
        r->ensure_plot_stream();
        for (int b = 0; b < 2; ++b) {
            r->rec[b].ensure(nrec * 16);
            r->rec_draws[b].ensure(std::max<size_t>(4, nrec * 4 * (size_t)nfd));
        }
    }
    std::vector<Launch> ls;
    for (uint64_t it0 = 0; it0 < total_iters; it0 += chunk) {
        L.it0 = it0;
        L.n_iters = (uint32_t)std::min<uint64_t>(chunk, total_iters - it0);
        if (defer) { L.rec = r->rec[ls.size() % 2].p; L.rec_draws = r->rec_draws[ls.size() % 2].p; }
        ls.push_back(L);
    }
    ck(cudaMemcpyAsync(d_jobs, ls.data(), ls.size() * sizeof(Launch), cudaMemcpyHostToDevice, s), "upload launches");
    r->h2d += ls.size() * sizeof(Launch);
    const int smem_plot = ((P.plan.table_size + 3) / 4) * 16 + (int)pal_n * 16;
    if (defer) {
        if (smem_plot > 48 * 1024 && m.smem_attr_plot < smem_plot) {
            ck(cudaFuncSetAttribute((const void*)m.plot, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_plot), "smem attribute");
            m.smem_attr_plot = smem_plot;
        }
        ck(cudaEventRecord(r->ev_start, s), "event");                          // the clears and uploads before
        ck(cudaStreamWaitEvent(r->plot_stream, r->ev_start, 0), "plot stream waits");
    }
    // RenderProgress: a cancel is looked at before each launch, progress
    // reported after it; with either, at most two launches are in flight
    // (each waits for the one two before it).
    const bool watched = P.progress || P.cancelled;
    if (watched) r->ensure_flight_events();
    const uint64_t plotted_total = (uint64_t)P.walkers * P.per_walker;
    for (size_t i = 0; i < ls.size(); ++i) {
        Launch* jp = d_jobs + i;
        int nj = 1;
        void* args[] = {&jp, &nj};
        if (watched && i >= 2) ck(cudaEventSynchronize(r->ev_flight[i % 2]), "launch in flight");
        if (P.cancelled && P.cancelled(P.progress_user)) {
            ck(cudaStreamSynchronize(s), "cancel");
            if (defer) ck(cudaStreamSynchronize(r->plot_stream), "cancel");
            fail(FFB_ERR_CANCELLED, "render cancelled");
        }
        if (filt) ck(cudaMemsetAsync(batch, 0, npx * 16, s), "clear batch histogram");
        if (defer && i >= 2) ck(cudaStreamWaitEvent(s, r->ev_plot[i % 2], 0), "record buffer free");
        ck(cudaLaunchKernel(kfn, dim3(blocks), dim3(threads + consumers), args, (size_t)smem, s), "launch ffb_chaos");
        r->launches += 1;
        if (watched) {
            ck(cudaEventRecord(r->ev_flight[i % 2], s), "event");
            if (P.progress) {
                const uint64_t end = ls[i].it0 + ls[i].n_iters;
                const uint64_t done = end > P.burn_in ? std::min<uint64_t>((uint64_t)P.walkers * (end - P.burn_in), plotted_total) : 0;
                P.progress(P.progress_user, done, plotted_total);
            }
        }
        if (defer && r->plot_timing) {
            // The plot kernel alone: after its chaos launch, on the same
            // stream, timed by events (a measurement mode, not a render's).
            ck(cudaEventRecord(r->ev_p[0], s), "event");
            ck(cudaLaunchKernel((const void*)m.plot, dim3((unsigned)r->n_sm * kPlotBlocksPerSm), dim3(kPlotThreads), args, (size_t)smem_plot,
                                s), "launch ffb_plot");
            ck(cudaEventRecord(r->ev_p[1], s), "event");
            ck(cudaEventSynchronize(r->ev_p[1]), "plot launch");
            float t = 0.f;
            ck(cudaEventElapsedTime(&t, r->ev_p[0], r->ev_p[1]), "event time");
            *r->plot_timing += t;
            r->launches += 1;
        } else if (defer) {
            ck(cudaEventRecord(r->ev_main[i % 2], s), "event");
            ck(cudaStreamWaitEvent(r->plot_stream, r->ev_main[i % 2], 0), "plot waits for its samples");
            ck(cudaLaunchKernel((const void*)m.plot, dim3((unsigned)r->n_sm * kPlotBlocksPerSm), dim3(kPlotThreads), args, (size_t)smem_plot,
                                r->plot_stream), "launch ffb_plot");
            ck(cudaEventRecord(r->ev_plot[i % 2], r->plot_stream), "event");
            r->launches += 1;
            if (i + 1 == ls.size()) {
                ck(cudaStreamWaitEvent(s, r->ev_plot[i % 2], 0), "render waits for the last plot");
                if (i >= 1) ck(cudaStreamWaitEvent(s, r->ev_plot[(i + 1) % 2], 0), "render waits for the plots");
            }
        }
        if (filt) {
            // The batch's plotted samples, as the reference counts them (compute_kernel.rs:1413-1421):
            // its walkers' iterations past the burn-in.
            const uint64_t a = std::max<uint64_t>(ls[i].it0, P.burn_in), b = ls[i].it0 + ls[i].n_iters;
            const double samples = (double)P.walkers * (double)(b > a ? b - a : 0);
            // sigma_d = mean density x 100^(2 blur_edges - 1), here in counts (the reference's
            // densities are counts x 100; its floor of 1 is 0.01 count).
            const double sd = samples / (double)npx * std::pow(100.0, 2.0 * (double)P.flame.filter.blur_edges - 1.0);
            ck(launch_hist_filter(batch, ftmp, hist, (int)P.wi, (int)P.hi, P.flame.filter.radius, (float)sd, s), "spatial filter");
            r->launches += 2;
        }
        if (P.plan.emit) {
            unsigned* count = (unsigned*)r->tile_meta.p;
            unsigned* fill = count + tg.n_tiles;
            unsigned* off = fill + tg.n_tiles;
            unsigned* work_off = off + tg.n_tiles + 1;
            unsigned* work = work_off + tg.n_tiles + 1;
            unsigned* band_fill = work + 2;
            unsigned* band_part_off = band_fill + tg.tiles_y;
            const uint64_t seg_cap = (uint64_t)threads * ls[i].n_iters * (uint64_t)P.flame.sym.copies();
            ck(launch_tile_pass((const unsigned long long*)r->tile_rec.p, seg_cap, (int)blocks, tg, 1u << 18, count, off, fill,
                                work_off, work, band_fill, band_part_off, (unsigned long long*)r->tile_tmp.p,
                                (unsigned*)r->tile_sorted.p, (const float4*)d_pal, (int)pal_n, (void*)hist, P.count_bits == 64,
                                r->n_sm, s),
               "tile-sorted accumulation");
            r->launches += 5;
        }
    }
    if (P.plan.emit) {
        // The launches are sized so no segment can overflow; a set flag
        // would mean lost samples, so it is checked rather than assumed.
        uint64_t flag = 0;
        ck(cudaMemcpyAsync(&flag, d_cnt + 3, 8, cudaMemcpyDeviceToHost, s), "read overflow flag");
        ck(cudaStreamSynchronize(s), "tile-sorted accumulation");
        if (flag) fail(FFB_ERR_CUDA, "tile-sorted accumulation: record segment overflow");
    }
    if (inframe_out) {
        ck(cudaMemcpyAsync(inframe_out, d_cnt, 8, cudaMemcpyDeviceToHost, s), "read counters");
        r->d2h += 8;
    }
}

// Density estimation of output rows [y_lo, y_lo + h_out) of a w x h
// histogram into r->de_out (count as float; row y_lo first).
float4* run_de(ffb_renderer* r, const float4* hist, uint32_t w, uint32_t h, double r_max, double r_min, double curve, cudaStream_t s,
               uint32_t y_lo = 0, uint32_t h_out = 0, const ulonglong4* exact = nullptr, bool count_f = false) {
    if (h_out == 0) h_out = h - y_lo;
    int n = 0, radius = 0;
    std::vector<float> tab = de_table(r_max, r_min, curve, n, radius);
    float4* d_tab = (float4*)r->de_tab.ensure(tab.size() * 4);
    ck(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, s), "upload DE table");
    r->h2d += tab.size() * 4;
    float4* out = (float4*)r->de_out.ensure((size_t)w * h_out * sizeof(float4));
    ck(launch_density_estimate(hist, exact, (int)w, (int)h, d_tab, n, radius, (int)y_lo, (int)h_out, out, s, count_f ? 1 : 0),
       "density estimation");
    r->launches += 1;
    return out;
}

const float* upload_lut(ffb_renderer* r, const Flame& f, cudaStream_t s) {
    std::vector<float> lut = curve_lut(f.tm);
    float* d = (float*)r->lut.ensure(256 * 4);
    ck(cudaMemcpyAsync(d, lut.data(), 256 * 4, cudaMemcpyHostToDevice, s), "upload curve");
    r->h2d += 256 * 4;
    return d;
}

// The tail of a render: density estimation (if configured) and the tone map
// of output rows [row0, row0 + rows) of a summed histogram holding
// `samples` plotted samples, into `d_rgba` (that band, row0 first).
// `hist` holds internal rows [hist_row0, hist_row0 + hist_rows) of the
// histogram (the whole of it by default): a band's rows and the DE reach
// around them are enough, since density estimation reads no source farther
// than its radius.
void finish_device(ffb_renderer* r, const Prepared& P, const float4* hist, uint64_t samples, uint32_t row0, uint32_t rows,
                   int transparent, void* d_rgba, cudaStream_t s, uint32_t hist_row0 = 0, uint32_t hist_rows = 0) {
    const uint32_t ss = P.ss;
    if (hist_rows == 0) hist_rows = P.hi - hist_row0;
    const uint32_t y_lo = row0 * ss - hist_row0, h_band = rows * ss;
    const float4* src = P.plan.exact ? nullptr : hist + (size_t)y_lo * P.wi;
    bool count_f = P.flame.filter.on();              // a filtered histogram holds float counts
    const ulonglong4* ex = P.plan.exact ? (const ulonglong4*)hist : nullptr;
    if (ex) src = nullptr;
    if (P.flame.de.max_radius > 0.0f) {
        src = run_de(r, ex ? nullptr : hist, P.wi, hist_rows, (double)P.flame.de.max_radius * ss, (double)P.flame.de.min_radius * ss,
                     (double)P.flame.de.curve, s, y_lo, h_band, ex, count_f);
        count_f = true;
    }
    const double sd = std::max((double)samples / ((double)P.wi * (double)P.hi), 1e-6);   // compute_kernel.rs:1796-1840
    TonemapArgs a = tonemap_args(P.flame, P.wi, P.hi, sd, transparent, count_f);
    if (!count_f && ex) a.exact = ex + (size_t)y_lo * P.wi;
    const float* lut = upload_lut(r, P.flame, s);
    ck(launch_tonemap(src, (int)P.wi, (int)h_band, (int)ss, a, lut, (uint8_t*)d_rgba, nullptr, s), "tone map");
    r->launches += 1;
}

// One whole render into device RGBA8 `d_rgba`.
void render_device(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, void* d_rgba, cudaStream_t s,
                   bool sync, ffb_output* out) {
    Prepared P = prepare(config, len, job);
    check_de(P.flame, P.ss);
    ck(cudaEventRecord(r->ev0, s), "event");
    uint64_t* h_inframe = nullptr;
    static thread_local uint64_t inframe_slot;
    if (sync) h_inframe = &inframe_slot;
    run_chaos(r, P, s, job->walker0, h_inframe);
    const uint64_t plotted = plotted_samples(P, job->walker0);
    finish_device(r, P, (const float4*)r->hist.p, plotted, 0, job->height, job->transparent, d_rgba, s);
    ck(cudaEventRecord(r->ev1, s), "event");
    if (out) {
        out->width = job->width; out->height = job->height;
        out->total_iterations = plotted;
        out->inframe_samples = 0;
        out->render_time_ms = 0.0;
    }
    if (sync) {
        ck(cudaStreamSynchronize(s), "render");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, r->ev0, r->ev1), "event time");
        check_inframe(*h_inframe);
        if (out) { out->render_time_ms = ms; out->inframe_samples = *h_inframe; }
    }
    r->fill_counts(out);
}

// ------------------------------------------------------------ fae_call ---
thread_local std::vector<uint8_t> g_output, g_info;
std::mutex g_fae_mu;
std::unique_ptr<ffb_renderer> g_fae_renderer;

ffb_renderer* fae_renderer() {
    if (!g_fae_renderer) {
        ffb_renderer* r = nullptr;
        int st = ffb_renderer_create(0, &r);
        if (st != FFB_OK) fail(st, g_err.empty() ? "no CUDA device" : g_err);
        g_fae_renderer.reset(r);
    }
    return g_fae_renderer.get();
}

std::string variations_json() {
    std::string s = "[";
    bool first = true;
    for (const VarDef* v : registry_all()) {
        if (!first) s += ",";
        first = false;
        s += "{\"name\":" + JsonWriter::quote(v->name) + ",\"params\":[";
        for (int j = 0; j < v->nparams; ++j) s += (j ? "," : "") + JsonWriter::quote(v->pname[j]);
        s += "]}";
    }
    return s + "]";
}

uint32_t u32_arg(const Json& r, const char* k) {
    const Json* v = r.get(k);
    if (!v || v->kind != Json::Number || v->num < 0) fail(FFB_ERR_INVALID, std::string("`") + k + "` (a number) is missing");
    return (uint32_t)v->num;
}

// A frame as the PNG the reference's CLI writes (wasm/python/src/render.rs:97-103,
// src/png_metadata.rs:61-183): the config, the render's numbers and the
// tone map's settings in tEXt chunks.
std::vector<uint8_t> encode_png_bytes(const std::string& config, const uint8_t* rgba, size_t len, uint32_t w, uint32_t h,
                                      uint64_t iterations, double ms, uint32_t ipt) {
    if (!rgba || len != (size_t)w * h * 4)
        fail(FFB_ERR_INVALID, std::to_string(len) + " bytes are not " + std::to_string(w) + "x" + std::to_string(h) + " RGBA");
    if (w == 0 || h == 0) fail(FFB_ERR_INVALID, "width and height must be nonzero");
    Flame f;
    PngInfo in;
    try {
        JsonPtr j = json_parse(config);
        f = parse_config(*j);
        in.speed_factor = (float)j->number_or("speed_factor", 0.5);
    } catch (const std::exception& e) { fail(FFB_ERR_CONFIG, std::string("config did not parse: ") + e.what()); }
    in.software = ffb_version();
    in.build_date = __DATE__ " " __TIME__;
    for (int k = 0; k < 3; ++k) in.background[k] = f.tm.background[k];
    in.exposure = f.tm.exposure;
    in.gamma = f.tm.gamma;
    in.tone_curve = f.tm.curve.size() > 2;
    in.variations = f.local.size();
    try { return png_encode(rgba, w, h, png_metadata(config, w, h, iterations, ms, ipt, in)); }
    catch (const std::exception& e) { fail(FFB_ERR_INVALID, e.what()); }
}

void fae_dispatch(const Json& r, const uint8_t* data, size_t data_len, std::vector<uint8_t>& out, std::string& info) {
    const Json* fn = r.get("fn");
    if (!fn || fn->kind != Json::String) fail(FFB_ERR_INVALID, "`fn` is missing");
    const std::string& f = fn->str;
    if (f == "info") {
        info = std::string("{\"result\":{\"version\":") + JsonWriter::quote(ffb_version()) +
               ",\"engines\":[\"flame\"],\"device\":\"cuda sm_100a\"}}";
    } else if (f == "variations") {
        info = "{\"result\":" + variations_json() + "}";
    } else if (f == "render") {
        const Json* c = r.get("config");
        if (!c || c->kind != Json::String) fail(FFB_ERR_INVALID, "`config` (a string) is missing");
        ffb_job job{};
        job.width = u32_arg(r, "width");
        job.height = u32_arg(r, "height");
        if (const Json* it = r.get("iterations"); it && it->kind == Json::Number && it->num > 0) job.iterations = (uint64_t)it->num;
        if (const Json* it = r.get("iterations_per_thread"); it && it->kind == Json::Number) job.iterations_per_thread = (uint32_t)it->num;
        job.iterations_per_thread = job.iterations_per_thread ? job.iterations_per_thread : 1024;   // DEFAULT_EXPORT_ITERATIONS_PER_THREAD
        const bool tr = r.bool_or("transparent", false), pm = r.bool_or("premultiplied", false);
        job.transparent = tr ? (pm ? 2 : 1) : 0;
        job.supersample = (uint32_t)r.number_or("supersample", 1.0);
        job.rng = (int32_t)r.number_or("rng", -1.0);
        job.walkers = (uint32_t)r.number_or("walkers", 0.0);
        job.count_bits = r.bool_or("exact", false) ? 64 : 32;
        {
            const std::string acc = r.string_or("accumulate", "auto");
            if (acc != "auto" && acc != "direct" && acc != "tiled")
                fail(FFB_ERR_INVALID, "accumulate must be \"auto\", \"direct\" or \"tiled\"");
            job.accumulate = acc == "direct" ? 1u : acc == "tiled" ? 2u : 0u;
        }
        ffb_renderer* R = fae_renderer();
        std::lock_guard<std::mutex> lk(R->mu);
        R->begin();
        const size_t n_out = (size_t)job.width * job.height * 4;
        void* d = R->rgba.ensure(n_out);
        ffb_output o{};
        R->reset_counts();
        render_device(R, c->str.data(), c->str.size(), &job, d, R->stream, true, &o);
        uint8_t* staged = (uint8_t*)R->readback.ensure(n_out);
        ck(cudaMemcpyAsync(staged, d, n_out, cudaMemcpyDeviceToHost, R->stream), "readback");
        R->d2h += n_out;
        ck(cudaStreamSynchronize(R->stream), "readback");
        out.assign(staged, staged + n_out);
        JsonWriter w;
        w.begin().num("width", job.width).num("height", job.height).num("iterations", (double)o.total_iterations)
            .num("ms", o.render_time_ms).num("iterations_per_thread", job.iterations_per_thread).end();
        info = w.s();
    } else if (f == "flame_import") {                                   // wasm/python/src/lib.rs:214-218
        const Json* x = r.get("xml");
        if (!x || x->kind != Json::String) fail(FFB_ERR_INVALID, "`xml` (a string) is missing");
        std::vector<std::string> cfgs;
        try { cfgs = flame_xml_import(x->str); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, e.what()); }
        std::string a = "[";
        for (size_t i = 0; i < cfgs.size(); ++i) a += (i ? "," : "") + JsonWriter::quote(cfgs[i]);
        info = "{\"result\":" + a + "]}";
    } else if (f == "encode_png") {                                     // wasm/python/src/lib.rs:227-232
        const Json* c = r.get("config");
        if (!c || c->kind != Json::String) fail(FFB_ERR_INVALID, "`config` (a string) is missing");
        out = encode_png_bytes(c->str, data, data_len, u32_arg(r, "width"), u32_arg(r, "height"),
                               (uint64_t)r.number_or("iterations", 0.0), r.number_or("ms", 0.0),
                               (uint32_t)r.number_or("iterations_per_thread", 0.0));
        info = "null";
    } else {
        fail(FFB_ERR_INVALID, "`" + f + "` is not supported by this build (render, encode_png, flame_import, info, variations)");
    }
}

}  // namespace
}  // namespace ffb

// ================================================================ ABI ====
FFB_API const char* ffb_last_error(void) { return g_err.c_str(); }
FFB_API const char* ffb_version(void) { return "ffb200 0.1.0 (sm_100a)"; }
FFB_API void ffb_struct_sizes(size_t* job_bytes, size_t* output_bytes) {
    if (job_bytes) *job_bytes = sizeof(ffb_job);
    if (output_bytes) *output_bytes = sizeof(ffb_output);
}

FFB_API int ffb_flame_import(const char* xml, size_t xml_len, const char** out, size_t* out_len) {
    static thread_local std::string json;
    return guard([&] {
        if (!xml || !out || !out_len) fail(FFB_ERR_INVALID, "NULL argument");
        std::vector<std::string> cfgs;
        try { cfgs = flame_xml_import(std::string(xml, xml_len)); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, e.what()); }
        json = "[";
        for (size_t i = 0; i < cfgs.size(); ++i) json += (i ? "," : "") + cfgs[i];
        json += "]";
        *out = json.c_str();
        *out_len = json.size();
    });
}

FFB_API int ffb_encode_png(const char* config, size_t config_len, const uint8_t* rgba, uint32_t width, uint32_t height,
                           uint64_t iterations, double ms, uint32_t iterations_per_thread, const uint8_t** out, size_t* out_len) {
    static thread_local std::vector<uint8_t> png;
    return guard([&] {
        if (!config || !out || !out_len) fail(FFB_ERR_INVALID, "NULL argument");
        png = encode_png_bytes(std::string(config, config_len), rgba, (size_t)width * height * 4, width, height, iterations, ms,
                               iterations_per_thread);
        *out = png.data();
        *out_len = png.size();
    });
}

FFB_API int ffb_renderer_create(int device, ffb_renderer** out) {
    return guard([&] {
        if (!out) fail(FFB_ERR_INVALID, "out is NULL");
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) fail(FFB_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
        if (device < 0 || device >= n) fail(FFB_ERR_INVALID, "no such device");
        auto r = std::make_unique<ffb_renderer>();
        r->device = device;
        r->begin();
        ck(cudaDeviceGetAttribute(&r->n_sm, cudaDevAttrMultiProcessorCount, device), "device attribute");
        ck(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaEventCreate(&r->ev0), "cudaEventCreate");
        ck(cudaEventCreate(&r->ev1), "cudaEventCreate");
        *out = r.release();
    });
}

FFB_API void ffb_renderer_destroy(ffb_renderer* r) { delete r; }

FFB_API int ffb_render(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, uint8_t* rgba, ffb_output* out) {
    return guard([&] {
        if (!r || !rgba || !job) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        const size_t bytes = (size_t)job->width * job->height * 4;
        void* d = r->rgba.ensure(bytes);
        ffb_output o{};
        r->reset_counts();
        render_device(r, config, len, job, d, r->stream, true, &o);
        ck(cudaMemcpyAsync(rgba, d, bytes, cudaMemcpyDeviceToHost, r->stream), "readback");
        r->d2h += bytes;
        ck(cudaStreamSynchronize(r->stream), "readback");
        r->fill_counts(&o);
        if (out) *out = o;
    });
}

FFB_API int ffb_render_device(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, void* d_rgba, void* stream,
                              int sync, ffb_output* out) {
    return guard([&] {
        if (!r || !d_rgba || !job) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        r->reset_counts();
        render_device(r, config, len, job, d_rgba, stream ? (cudaStream_t)stream : r->stream, sync != 0, out);
    });
}

FFB_API int ffb_histogram(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, uint32_t* counts, float* rgb,
                          ffb_output* out) {
    return guard([&] {
        if (!r || !job) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Prepared P = prepare(config, len, job);
        if (P.flame.filter.on()) fail(FFB_ERR_INVALID, "a filtered histogram holds fractional counts: use ffb_histogram_f32");
        r->reset_counts();
        uint64_t inframe = 0;
        ck(cudaEventRecord(r->ev0, r->stream), "event");
        run_chaos(r, P, r->stream, job->walker0, &inframe);
        ck(cudaEventRecord(r->ev1, r->stream), "event");
        const size_t npx = (size_t)P.wi * P.hi;
        std::vector<float> h(npx * 4);
        ck(cudaMemcpyAsync(h.data(), r->hist.p, npx * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "histogram");
        check_inframe(inframe);
        for (size_t i = 0; i < npx; ++i) {
            if (counts) { uint32_t c; std::memcpy(&c, &h[i * 4 + 3], 4); counts[i] = c; }
            if (rgb) { rgb[i * 3] = h[i * 4]; rgb[i * 3 + 1] = h[i * 4 + 1]; rgb[i * 3 + 2] = h[i * 4 + 2]; }
        }
        if (out) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r->ev0, r->ev1);
            out->width = P.wi; out->height = P.hi;
            out->total_iterations = plotted_samples(P, job->walker0);
            out->inframe_samples = inframe;
            out->render_time_ms = ms;
            r->fill_counts(out);
            out->d2h_bytes += npx * 16;
        }
    });
}

FFB_API int ffb_histogram_f32(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, float* counts, float* rgb,
                              ffb_output* out) {
    return guard([&] {
        if (!r || !job) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Prepared P = prepare(config, len, job);
        if (P.count_bits != 32) fail(FFB_ERR_INVALID, "ffb_histogram_f32 reads the u32 / filtered histogram (count_bits 32)");
        r->reset_counts();
        uint64_t inframe = 0;
        ck(cudaEventRecord(r->ev0, r->stream), "event");
        run_chaos(r, P, r->stream, job->walker0, &inframe);
        ck(cudaEventRecord(r->ev1, r->stream), "event");
        const size_t npx = (size_t)P.wi * P.hi;
        std::vector<float> h(npx * 4);
        ck(cudaMemcpyAsync(h.data(), r->hist.p, npx * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "histogram");
        check_inframe(inframe);
        const bool f = P.flame.filter.on();
        for (size_t i = 0; i < npx; ++i) {
            if (counts) { uint32_t c; std::memcpy(&c, &h[i * 4 + 3], 4); counts[i] = f ? h[i * 4 + 3] : (float)c; }
            if (rgb) { rgb[i * 3] = h[i * 4]; rgb[i * 3 + 1] = h[i * 4 + 1]; rgb[i * 3 + 2] = h[i * 4 + 2]; }
        }
        if (out) {
            *out = ffb_output{};
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r->ev0, r->ev1);
            out->width = P.wi; out->height = P.hi;
            out->total_iterations = plotted_samples(P, job->walker0);
            out->inframe_samples = inframe;
            out->render_time_ms = ms;
            r->fill_counts(out);
        }
    });
}

FFB_API int ffb_hist_filter(ffb_renderer* r, const uint32_t* counts, const float* rgb, uint32_t w, uint32_t h, float sigma,
                            float sigma_d, float* out) {
    return guard([&] {
        if (!r || !counts || !rgb || !out) fail(FFB_ERR_INVALID, "NULL argument");
        if (w == 0 || h == 0 || w > kMaxDim || h > kMaxDim) fail(FFB_ERR_INVALID, "bad histogram size");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        const size_t npx = (size_t)w * h;
        std::vector<float> in(npx * 4);
        for (size_t i = 0; i < npx; ++i) {
            in[i * 4] = rgb[i * 3]; in[i * 4 + 1] = rgb[i * 3 + 1]; in[i * 4 + 2] = rgb[i * 3 + 2];
            std::memcpy(&in[i * 4 + 3], &counts[i], 4);
        }
        float4* batch = (float4*)r->filt_batch.ensure(npx * 16);
        float4* tmp = (float4*)r->filt_tmp.ensure(npx * 16);
        float4* acc = (float4*)r->f_out.ensure(npx * 16);
        ck(cudaMemcpyAsync(batch, in.data(), npx * 16, cudaMemcpyHostToDevice, r->stream), "upload");
        ck(cudaMemsetAsync(acc, 0, npx * 16, r->stream), "clear");
        ck(launch_hist_filter(batch, tmp, acc, (int)w, (int)h, sigma, sigma_d, r->stream), "spatial filter");
        ck(cudaMemcpyAsync(out, acc, npx * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "spatial filter");
    });
}

FFB_API int ffb_histogram_u64(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, uint64_t* counts, float* rgb,
                              ffb_output* out) {
    return guard([&] {
        if (!r || !job || !counts) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        ffb_job j = *job;
        j.count_bits = 64;
        Prepared P = prepare(config, len, &j);
        r->reset_counts();
        uint64_t inframe = 0;
        ck(cudaEventRecord(r->ev0, r->stream), "event");
        run_chaos(r, P, r->stream, j.walker0, &inframe);
        ck(cudaEventRecord(r->ev1, r->stream), "event");
        const size_t npx = (size_t)P.wi * P.hi;
        std::vector<unsigned long long> h(npx * 4);
        ck(cudaMemcpyAsync(h.data(), r->hist.p, npx * 32, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "histogram");
        check_inframe(inframe);
        for (size_t i = 0; i < npx; ++i) {
            counts[i] = h[i * 4 + 3];
            if (rgb) for (int q = 0; q < 3; ++q) rgb[i * 3 + q] = (float)((double)h[i * 4 + q] / 16777216.0);
        }
        if (out) {
            *out = ffb_output{};
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r->ev0, r->ev1);
            out->width = P.wi; out->height = P.hi;
            out->total_iterations = plotted_samples(P, job->walker0);
            out->inframe_samples = inframe;
            out->render_time_ms = ms;
            r->fill_counts(out);
        }
    });
}

FFB_API int ffb_tonemap(ffb_renderer* r, const char* config, size_t len, const float* counts, const float* rgb, uint32_t w,
                        uint32_t h, uint32_t ss, double sample_density, int32_t transparent, uint8_t* rgba, float* rgba_f) {
    return guard([&] {
        if (!r || !counts || !rgb || !rgba) fail(FFB_ERR_INVALID, "NULL argument");
        if (ss != 1 && ss != 2) fail(FFB_ERR_INVALID, "ss must be 1 or 2");
        if (w == 0 || h == 0 || (ss == 2 && (w % 2 || h % 2))) fail(FFB_ERR_INVALID, "bad size");
        if (rgba_f && ss != 1) fail(FFB_ERR_INVALID, "float output at ss 1 only");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Flame f;
        try { f = parse_config_text(std::string(config, len)); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, std::string("config did not parse: ") + e.what()); }
        const size_t npx = (size_t)w * h;
        std::vector<float> hv(npx * 4);
        for (size_t i = 0; i < npx; ++i) { hv[i * 4] = rgb[i * 3]; hv[i * 4 + 1] = rgb[i * 3 + 1]; hv[i * 4 + 2] = rgb[i * 3 + 2]; hv[i * 4 + 3] = counts[i]; }
        float4* d_in = (float4*)r->tmp_in.ensure(npx * 16);
        ck(cudaMemcpyAsync(d_in, hv.data(), npx * 16, cudaMemcpyHostToDevice, r->stream), "upload");
        TonemapArgs a = tonemap_args(f, w, h, sample_density, transparent, true);
        const float* lut = upload_lut(r, f, r->stream);
        const size_t out_px = ss == 1 ? npx : npx / 4;
        void* d_out = r->rgba.ensure(out_px * 4);
        float4* d_f = rgba_f ? (float4*)r->f_out.ensure(npx * 16) : nullptr;
        ck(launch_tonemap(d_in, (int)w, (int)h, (int)ss, a, lut, (uint8_t*)d_out, d_f, r->stream), "tone map");
        ck(cudaMemcpyAsync(rgba, d_out, out_px * 4, cudaMemcpyDeviceToHost, r->stream), "readback");
        if (rgba_f) ck(cudaMemcpyAsync(rgba_f, d_f, npx * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "tone map");
    });
}

// Density-estimation parameters a caller passes: written so that NaN fails
// every comparison and is refused with the out-of-range values.
static bool de_params_ok(float max_radius, float min_radius, float curve) {
    return max_radius > 0.f && max_radius <= 36.f && min_radius >= 0.f && std::isfinite(min_radius) && curve >= 0.f &&
           std::isfinite(curve);
}

FFB_API int ffb_density_estimate(ffb_renderer* r, const uint32_t* counts, const float* rgb, uint32_t w, uint32_t h,
                                 float max_radius, float min_radius, float curve, float* out_counts, float* out_rgb) {
    return guard([&] {
        if (!r || !counts || !rgb || !out_counts || !out_rgb) fail(FFB_ERR_INVALID, "NULL argument");
        if (!de_params_ok(max_radius, min_radius, curve)) fail(FFB_ERR_INVALID, "bad DE parameters: max_radius in (0, 36], min_radius >= 0, curve >= 0, all finite");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        const size_t npx = (size_t)w * h;
        std::vector<float> hv(npx * 4);
        for (size_t i = 0; i < npx; ++i) {
            hv[i * 4] = rgb[i * 3]; hv[i * 4 + 1] = rgb[i * 3 + 1]; hv[i * 4 + 2] = rgb[i * 3 + 2];
            std::memcpy(&hv[i * 4 + 3], &counts[i], 4);
        }
        float4* d_in = (float4*)r->tmp_in.ensure(npx * 16);
        ck(cudaMemcpyAsync(d_in, hv.data(), npx * 16, cudaMemcpyHostToDevice, r->stream), "upload");
        float4* o = run_de(r, d_in, w, h, max_radius, min_radius, curve, r->stream);
        std::vector<float> ov(npx * 4);
        ck(cudaMemcpyAsync(ov.data(), o, npx * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "density estimation");
        for (size_t i = 0; i < npx; ++i) {
            out_rgb[i * 3] = ov[i * 4]; out_rgb[i * 3 + 1] = ov[i * 4 + 1]; out_rgb[i * 3 + 2] = ov[i * 4 + 2];
            out_counts[i] = ov[i * 4 + 3];
        }
    });
}

FFB_API int ffb_density_estimate_static(const void* d_hist, uint32_t w, uint32_t h, float max_radius, float min_radius,
                                        float curve, void* d_out, void* stream) {
    return guard([&] {
        if (!d_hist || !d_out) fail(FFB_ERR_INVALID, "NULL argument");
        if (w == 0 || h == 0 || w > 65536 || h > 65536) fail(FFB_ERR_INVALID, "histogram size must be 1..65536 on each side");
        if (!de_params_ok(max_radius, min_radius, curve)) fail(FFB_ERR_INVALID, "bad DE parameters: max_radius in (0, 36], min_radius >= 0, curve >= 0, all finite");
        if (de_static_entries(max_radius, min_radius, curve) < 0)
            fail(FFB_ERR_TOO_LARGE, "density estimation table needs more than " + std::to_string(kDeStaticEntries) +
                                        " entries, the static scratch's size: raise min_radius or curve");
        ck(density_estimate_static((const float4*)d_hist, (int)w, (int)h, max_radius, min_radius, curve, (float4*)d_out,
                                   (cudaStream_t)stream),
           "density estimation (static scratch)");
    });
}

FFB_API int ffb_probe(ffb_renderer* r, const char* config, size_t len, const float* pts, uint32_t npts, int32_t math, float* out,
                      uint32_t out_pairs) {
    return guard([&] {
        if (!r || !pts || !out) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Flame f;
        try { f = parse_config_text(std::string(config, len)); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, std::string("config did not parse: ") + e.what()); }
        Plan p = make_plan(f, RNG_PCG, math, 0, 128);
        std::vector<float> tab = make_table(p, f);
        const int n_all = (int)(f.xf.size() + f.fin_used.size());
        if (out_pairs < (uint32_t)n_all * npts) fail(FFB_ERR_INVALID, "output too small");
        Module& m = r->module_for(p.source);
        void* d_tab = r->table.ensure(tab.size() * 4);
        ck(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        float* d_pts = (float*)r->tmp_in.ensure((size_t)npts * 8);
        ck(cudaMemcpyAsync(d_pts, pts, (size_t)npts * 8, cudaMemcpyHostToDevice, r->stream), "upload");
        float* d_out = (float*)r->f_out.ensure((size_t)n_all * npts * 8);
        int nx = (int)f.xf.size(), np = (int)npts;
        const float* tp = (const float*)d_tab;
        void* args[] = {&tp, &nx, (void*)&n_all, &d_pts, &np, &d_out};
        const int total = n_all * np;
        ck(cudaLaunchKernel((const void*)m.probe, dim3((total + 127) / 128), dim3(128), args, 0, r->stream), "launch ffb_probe");
        ck(cudaMemcpyAsync(out, d_out, (size_t)total * 8, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "probe");
    });
}

FFB_API int ffb_apply_points(ffb_renderer* r, const char* config, size_t len, int32_t xform, uint32_t n, const float* xs,
                             const float* ys, const float* words, int32_t with_affine, int32_t math, float* xo, float* yo) {
    return guard([&] {
        if (!r || !xs || !ys || !words || !xo || !yo) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Flame f;
        try { f = parse_config_text(std::string(config, len)); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, std::string("config did not parse: ") + e.what()); }
        const int n_all = (int)(f.xf.size() + f.fin_used.size());
        if (xform < 0 || xform >= n_all) fail(FFB_ERR_INVALID, "no such transform");
        Plan p = make_plan(f, RNG_PHILOX, math, 0, 128);
        std::vector<float> tab = make_table(p, f);
        Module& m = r->module_for(p.source);
        void* d_tab = r->table.ensure(tab.size() * 4);
        ck(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        const size_t nn = n;
        float* d_in = (float*)r->tmp_in.ensure(nn * 4 * 2 + nn * kApplyWords * 4);
        float* d_x = d_in, *d_y = d_in + nn, *d_w = d_in + 2 * nn;
        ck(cudaMemcpyAsync(d_x, xs, nn * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        ck(cudaMemcpyAsync(d_y, ys, nn * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        ck(cudaMemcpyAsync(d_w, words, nn * kApplyWords * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        float* d_out = (float*)r->f_out.ensure(nn * 8);
        float* d_xo = d_out, *d_yo = d_out + nn;
        int nx = (int)f.xf.size(), xi = xform, ni = (int)n, wa = with_affine;
        const float* tp = (const float*)d_tab;
        void* args[] = {&tp, &nx, &xi, &ni, &d_x, &d_y, &d_w, &wa, &d_xo, &d_yo};
        ck(cudaLaunchKernel((const void*)m.apply, dim3((n + 127) / 128), dim3(128), args, 0, r->stream), "launch ffb_apply_points");
        ck(cudaMemcpyAsync(xo, d_xo, nn * 4, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaMemcpyAsync(yo, d_yo, nn * 4, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "apply points");
    });
}

FFB_API int ffb_chaos_device(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, void* d_hist, void* stream,
                             ffb_output* out) {
    return guard([&] {
        if (!r || !job || !d_hist) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        r->reset_counts();
        Prepared P = prepare(config, len, job);
        if (P.count_bits != 32) fail(FFB_ERR_INVALID, "device histograms hold u32 counts (count_bits 32)");
        cudaStream_t s = stream ? (cudaStream_t)stream : r->stream;
        run_chaos(r, P, s, job->walker0, nullptr, (float4*)d_hist);
        if (out) {
            *out = ffb_output{};
            out->width = P.wi; out->height = P.hi;
            out->total_iterations = plotted_samples(P, job->walker0);
            r->fill_counts(out);
        }
    });
}

FFB_API int ffb_hist_pack(ffb_renderer* r, const void* d_hist, uint64_t pixels, void* d_counts, void* d_rgb, void* stream) {
    return guard([&] {
        if (!r || !d_hist || !d_counts || !d_rgb) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        ck(launch_pack((const float4*)d_hist, pixels, (unsigned*)d_counts, (float*)d_rgb, stream ? (cudaStream_t)stream : r->stream), "pack");
    });
}

FFB_API int ffb_hist_unpack(ffb_renderer* r, const void* d_counts, const void* d_rgb, uint64_t pixels, void* d_hist, void* stream) {
    return guard([&] {
        if (!r || !d_hist || !d_counts || !d_rgb) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        ck(launch_unpack((const unsigned*)d_counts, (const float*)d_rgb, pixels, (float4*)d_hist, stream ? (cudaStream_t)stream : r->stream), "unpack");
    });
}

FFB_API int ffb_finish_device(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, const void* d_hist,
                              uint64_t total_samples, uint32_t row0, uint32_t rows, void* d_rgba, void* stream) {
    return guard([&] {
        if (!r || !job || !d_hist || !d_rgba) fail(FFB_ERR_INVALID, "NULL argument");
        if (rows == 0 || row0 + rows > job->height) fail(FFB_ERR_INVALID, "row band outside the image");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Prepared P = prepare(config, len, job);
        check_de(P.flame, P.ss);
        finish_device(r, P, (const float4*)d_hist, total_samples, row0, rows, job->transparent, d_rgba,
                      stream ? (cudaStream_t)stream : r->stream);
    });
}

FFB_API int ffb_finish_band(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, const void* d_hist,
                            uint32_t hist_row0, uint32_t hist_rows, uint64_t total_samples, uint32_t row0, uint32_t rows,
                            void* d_rgba, void* stream) {
    return guard([&] {
        if (!r || !job || !d_hist || !d_rgba) fail(FFB_ERR_INVALID, "NULL argument");
        if (rows == 0 || row0 + rows > job->height) fail(FFB_ERR_INVALID, "row band outside the image");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Prepared P = prepare(config, len, job);
        check_de(P.flame, P.ss);
        if (P.plan.exact) fail(FFB_ERR_INVALID, "histogram bands hold u32 counts (count_bits 32)");
        // The window must hold the band and the DE reach around it (clamped to the image).
        const uint32_t reach = P.flame.de.max_radius > 0.0f ? (uint32_t)std::ceil((double)P.flame.de.max_radius * P.ss) : 0u;
        const uint32_t y_lo = row0 * P.ss, y_hi = (row0 + rows) * P.ss;
        const uint32_t need_lo = y_lo > reach ? y_lo - reach : 0u, need_hi = std::min<uint32_t>(P.hi, y_hi + reach);
        if ((uint64_t)hist_row0 + hist_rows > P.hi || hist_row0 > need_lo || hist_row0 + hist_rows < need_hi)
            fail(FFB_ERR_INVALID, "the histogram window must hold internal rows [" + std::to_string(need_lo) + ", " +
                                      std::to_string(need_hi) + "): the band and the density-estimation reach around it");
        finish_device(r, P, (const float4*)d_hist, total_samples, row0, rows, job->transparent, d_rgba,
                      stream ? (cudaStream_t)stream : r->stream, hist_row0, hist_rows);
    });
}

FFB_API int ffb_specialize_job(const char* config, size_t len, const ffb_job* job, size_t* cubin_bytes, char* source,
                               size_t source_len) {
    return guard([&] {
        Prepared P = prepare(config, len, job, false);
        std::vector<char> cubin = ffb_renderer::nvrtc_cubin(P.plan.source);
        if (cubin_bytes) *cubin_bytes = cubin.size();
        if (source && source_len) {
            size_t n = std::min(source_len - 1, P.plan.source.size());
            std::memcpy(source, P.plan.source.data(), n);
            source[n] = 0;
        }
    });
}

FFB_API int ffb_specialize(const char* config, size_t len, int32_t rng, int32_t math, size_t* cubin_bytes, char* source,
                           size_t source_len) {
    return guard([&] {
        if (!config) fail(FFB_ERR_INVALID, "config is NULL");
        Flame f;
        try { f = parse_config_text(std::string(config, len)); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, std::string("config did not parse: ") + e.what()); }
        Plan p = make_plan(f, rng, math, 0, 128);
        std::vector<char> cubin = ffb_renderer::nvrtc_cubin(p.source);
        if (cubin_bytes) *cubin_bytes = cubin.size();
        if (source && source_len) {
            size_t n = std::min(source_len - 1, p.source.size());
            std::memcpy(source, p.source.data(), n);
            source[n] = 0;
        }
    });
}

FFB_API int ffb_atomic_bench(ffb_renderer* r, uint32_t pixels, uint64_t samples, int32_t kind, double* ms) {
    return guard([&] {
        if (!r || !ms || pixels == 0) fail(FFB_ERR_INVALID, "bad argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        uint32_t* buf = (uint32_t*)r->hist.ensure((size_t)pixels * 16);
        ck(cudaMemsetAsync(buf, 0, (size_t)pixels * 16, r->stream), "clear");
        int dev_sms = 148;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, r->device);
        ck(launch_atomic_bench(buf, pixels, samples / 16, kind, dev_sms * 8, r->stream), "warm-up");
        ck(cudaEventRecord(r->ev0, r->stream), "event");
        ck(launch_atomic_bench(buf, pixels, samples, kind, dev_sms * 8, r->stream), "atomic bench");
        ck(cudaEventRecord(r->ev1, r->stream), "event");
        ck(cudaStreamSynchronize(r->stream), "atomic bench");
        float t = 0.f;
        ck(cudaEventElapsedTime(&t, r->ev0, r->ev1), "event time");
        *ms = t;
    });
}


// The splat kernel's own throughput: a deferred-plot render of `job` (the
// sorted schedule's records, ffb_plot applying the final chain, palette,
// symmetry copies and the warp-aggregated splat) with each plot launch run
// alone after its chaos launch; *plot_ms = the plot launches' summed device
// time, *inframe = the splats they made, *samples = the records plotted.
FFB_API int ffb_plot_bench(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, double* plot_ms, uint64_t* samples,
                           uint64_t* inframe) {
    return guard([&] {
        if (!r || !job || !plot_ms) fail(FFB_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        Prepared P = prepare(config, len, job);
        if (!P.plan.defer || P.plot == 3)
            fail(FFB_ERR_INVALID, "ffb_plot_bench times deferred plotting (plot 0 or 2): this job does not defer its plot");
        for (auto& e : r->ev_p)
            if (!e) ck(cudaEventCreate(&e), "event");
        r->reset_counts();
        double t = 0.0;
        uint64_t n_in = 0;
        r->plot_timing = &t;
        try {
            run_chaos(r, P, r->stream, job->walker0, &n_in);
            ck(cudaStreamSynchronize(r->stream), "plot bench");
        } catch (...) {
            r->plot_timing = nullptr;
            throw;
        }
        r->plot_timing = nullptr;
        check_inframe(n_in);
        *plot_ms = t;
        if (inframe) *inframe = n_in;
        if (samples) *samples = plotted_samples(P, job->walker0);
    });
}

// =============================================================== batches ===
// Many flames in one persistent launch a structure group (the batched
// addition beside the reference's one-flame-a-call render, render.rs:483-804):
// walkers a flame sized to its budget, every block owning walkers of one
// flame (ffb_chaos_sorted finds its flame by binary search over block0),
// one batched tone-map launch, the device work captured once as a CUDA graph
// and replayed.  Threads a block and iterations a walker are picked by
// timing candidates on a scaled-down copy of the batch.

namespace ffb {
namespace {

struct BatchFlame {
    Prepared P;
    uint64_t budget = 0;
    uint32_t group = 0;
    uint32_t walkers = 0, per_walker = 0;
    size_t hist_off = 0, walk_off = 0, rgba_off = 0, tab_off = 0, pal_off = 0;
};

struct BatchDe {
    size_t flame = 0, off = 0;
    int n = 0, radius = 0;
    std::vector<float> table;
};

struct BatchGroup {
    Module* mod = nullptr;
    std::string src;
    int table_size = 0, maxx = 0, max_pal = 0;
    std::vector<uint32_t> members;
};

}  // namespace
}  // namespace ffb

struct ffb_batch {
    ffb_renderer* r = nullptr;
    int device = 0;
    std::vector<BatchFlame> flames;
    std::vector<BatchGroup> groups;
    DevBuf hist, walk, rgba, tables, palettes, counters, launches, tjobs, luts, de, detab;
    uint32_t threads = 256, iters = 1024;
    bool plain = false;          // one walker a thread (ffb_chaos) instead of the transform-sorted kernel
    uint64_t total_samples = 0;
    std::vector<BatchDe> de_tabs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rng = RNG_PHILOX, transparent = 0;
    ~ffb_batch() {
        for (auto& G : groups) if (G.mod) G.mod->pins -= 1;
        groups.clear();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (DevBuf* b : {&hist, &walk, &rgba, &tables, &palettes, &counters, &launches, &tjobs, &luts, &de, &detab}) b->release();
    }
};

namespace ffb {
namespace {

// Walkers and launch records of every group for (threads, iters), scaling
// each budget by 1/`scale` (the tuner's trial runs); enqueues the clears,
// the chaos launches and the tone map on `s`.
void batch_enqueue(ffb_batch* B, uint32_t threads, uint32_t iters, uint64_t scale, cudaStream_t s, bool tonemap,
                   bool upload = true) {
    ffb_renderer* r = B->r;
    size_t walk_total = 0;
    for (auto& F : B->flames) {
        // The walkers of the full budget whatever the scale (a tuning run
        // keeps the real run's occupancy), each walking its share of the
        // scaled budget.
        const uint64_t budget = std::max<uint64_t>(1, F.budget / scale);
        uint64_t w = (F.budget + iters - 1) / iters;
        w = std::max<uint64_t>(w, threads);
        w = (w + threads - 1) / threads * threads;
        F.walkers = (uint32_t)w;
        F.per_walker = (uint32_t)std::max<uint64_t>(1, (budget + w - 1) / w);
        F.walk_off = walk_total;
        walk_total += w;
    }
    void* d_walk = B->walk.ensure(walk_total * 16);
    size_t hist_bytes = 0;
    for (auto& F : B->flames) hist_bytes = std::max(hist_bytes, (F.hist_off + (size_t)F.P.wi * F.P.hi) * 16);
    ck(cudaMemsetAsync(B->hist.p, 0, hist_bytes, s), "clear histograms");
    ck(cudaMemsetAsync(B->counters.p, 0, B->flames.size() * 8, s), "clear counters");
    std::vector<Launch> all;
    std::vector<size_t> first;
    for (auto& G : B->groups) {
        first.push_back(all.size());
        uint32_t block0 = 0;
        for (uint32_t j : G.members) {
            BatchFlame& F = B->flames[j];
            const Prepared& P = F.P;
            Launch L{};
            L.table = (const float*)B->tables.p + F.tab_off;
            L.palette = (const float*)B->palettes.p + F.pal_off;
            L.hist = (float4*)B->hist.p + F.hist_off;
            L.walkers = (float4*)d_walk + F.walk_off;
            L.counters = (uint64_t*)B->counters.p + j;
            L.n_walkers = F.walkers; L.walker0 = 0; L.block0 = block0; L.n_xf = (uint32_t)P.flame.xf.size();
            L.seed_lo = (uint32_t)P.seed; L.seed_hi = (uint32_t)(P.seed >> 32); L.burn_in = P.burn_in; L.ipt = P.ipt;
            L.it0 = 0; L.n_iters = F.per_walker + P.burn_in;
            L.pal_n = (uint32_t)(P.palette.size() / 4);
            L.width = (int32_t)P.wi; L.height = (int32_t)P.hi;
            L.zoom = P.flame.zoom; L.pan_x = (float)P.flame.pan_x; L.pan_y = (float)P.flame.pan_y;
            L.cos_r = (float)std::cos((double)P.flame.rotation); L.sin_r = (float)std::sin((double)P.flame.rotation);
            block0 += F.walkers / threads;
            all.push_back(L);
        }
    }
    // Under graph capture (upload false) the records uploaded by the
    // identical uncaptured call before are reused: a capture may not copy
    // from pageable host memory, nor allocate.
    Launch* d_l = (Launch*)B->launches.ensure(all.size() * sizeof(Launch));
    if (upload) ck(cudaMemcpyAsync(d_l, all.data(), all.size() * sizeof(Launch), cudaMemcpyHostToDevice, s), "upload launches");
    for (size_t g = 0; g < B->groups.size(); ++g) {
        BatchGroup& G = B->groups[g];
        uint32_t blocks = 0;
        for (uint32_t j : G.members) blocks += B->flames[j].walkers / threads;
        int smem = ((G.table_size + 3) / 4) * 16 + G.max_pal * 16;
        if (!B->plain) smem += (int)threads * 8 * 4 + 2 * (G.maxx + 1) * 4;
        const void* kfn = B->plain ? (const void*)G.mod->chaos : (const void*)G.mod->chaos_sorted;
        int& attr = B->plain ? G.mod->smem_attr : G.mod->smem_attr_sorted;
        if (smem > 48 * 1024 && attr < smem) {
            ck(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attribute");
            attr = smem;
        }
        Launch* jp = d_l + first[g];
        int nj = (int)G.members.size();
        void* args[] = {&jp, &nj};
        ck(cudaLaunchKernel(kfn, dim3(blocks), dim3(threads), args, (size_t)smem, s), "launch batch");
        r->launches += 1;
    }
    if (!tonemap) return;
    // Density estimation, flame by flame, into the DE arena (same layout as
    // the histograms); the tone map then reads the float counts there.
    if (upload) {
        B->de_tabs.clear();
        for (size_t j = 0; j < B->flames.size(); ++j) {
            const Flame& fl = B->flames[j].P.flame;
            if (fl.de.max_radius <= 0.0f) continue;
            BatchDe d;
            d.flame = j;
            const uint32_t ss = B->flames[j].P.ss;
            d.table = de_table((double)fl.de.max_radius * ss, (double)fl.de.min_radius * ss, (double)fl.de.curve, d.n, d.radius);
            B->de_tabs.push_back(std::move(d));
        }
        size_t tab_floats = 0;
        for (auto& d : B->de_tabs) { d.off = tab_floats; tab_floats += d.table.size(); }
        std::vector<float> all_tabs(tab_floats);
        for (auto& d : B->de_tabs) std::copy(d.table.begin(), d.table.end(), all_tabs.begin() + d.off);
        if (tab_floats) {
            ck(cudaMemcpyAsync(B->detab.ensure(tab_floats * 4), all_tabs.data(), tab_floats * 4, cudaMemcpyHostToDevice, s), "upload DE tables");
            B->de.ensure(hist_bytes);
        }
    }
    for (auto& d : B->de_tabs) {
        BatchFlame& F = B->flames[d.flame];
        ck(launch_density_estimate((const float4*)B->hist.p + F.hist_off, nullptr, (int)F.P.wi, (int)F.P.hi,
                                   (const float4*)((const float*)B->detab.p + d.off), d.n, d.radius, 0, (int)F.P.hi,
                                   (float4*)B->de.p + F.hist_off, s), "batch density estimation");
        r->launches += 1;
    }
    std::vector<TonemapJob> tj;
    long long px = 0;
    for (size_t j = 0; j < B->flames.size(); ++j) {
        BatchFlame& F = B->flames[j];
        const bool has_de = F.P.flame.de.max_radius > 0.0f;
        TonemapJob J{};
        J.hist = (const float4*)(has_de ? B->de.p : B->hist.p) + F.hist_off;
        J.out = (uint8_t*)B->rgba.p + F.rgba_off;
        J.lut = (const float*)B->luts.p + 256 * j;
        J.px0 = px;
        J.w = (int)F.P.wi; J.h = (int)F.P.hi;
        J.ss = (int)F.P.ss;
        const uint64_t plotted = (uint64_t)F.walkers * F.per_walker;
        const double sd = std::max((double)plotted / ((double)F.P.wi * (double)F.P.hi), 1e-6);
        J.a = tonemap_args(F.P.flame, F.P.wi, F.P.hi, sd, B->transparent, has_de);
        tj.push_back(J);
        px += (long long)(F.P.wi / F.P.ss) * (F.P.hi / F.P.ss);
    }
    TonemapJob* d_tj = (TonemapJob*)B->tjobs.ensure(tj.size() * sizeof(TonemapJob));
    if (upload) ck(cudaMemcpyAsync(d_tj, tj.data(), tj.size() * sizeof(TonemapJob), cudaMemcpyHostToDevice, s), "upload tone-map jobs");
    ck(launch_tonemap_batch(d_tj, (int)tj.size(), px, s), "batched tone map");
    r->launches += 1;
}

}  // namespace
}  // namespace ffb

FFB_API int ffb_batch_create(ffb_renderer* r, const ffb_batch_item* items, uint32_t n, const ffb_job* common, int32_t tune,
                             ffb_batch** out) {
    return guard([&] {
        if (!r || !items || !common || !out || n == 0) fail(FFB_ERR_INVALID, "bad argument");
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        auto B = std::make_unique<ffb_batch>();
        B->r = r;
        B->rng = common->rng < 0 ? RNG_PHILOX : common->rng;
        B->transparent = common->transparent;
        // Parse every flame; one transform capacity for the whole batch so
        // flames that differ only in their transform count share a module.
        int maxx = 1;
        B->flames.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            ffb_job j = *common;
            j.width = items[i].width; j.height = items[i].height; j.iterations = items[i].iterations;
            j.seed = items[i].seed;
            if (j.iterations == 0) fail(FFB_ERR_INVALID, "every batch item needs its sample budget");
            B->flames[i].P = prepare(items[i].config, items[i].config_len, &j);
            if (!B->flames[i].P.flame.xaos.empty())
                fail(FFB_ERR_INVALID, "item " + std::to_string(i) + ": xaos flames are not batched; render it alone");
            if (B->flames[i].P.plan.n_state > 0)
                fail(FFB_ERR_INVALID, "item " + std::to_string(i) + ": flames with stateful variations or subflames are not "
                                      "batched; render it alone");
            if (B->flames[i].P.flame.filter.on())
                fail(FFB_ERR_INVALID, "item " + std::to_string(i) + ": the spatial filter (filter_radius) is not batched; render it alone");
            check_de(B->flames[i].P.flame, B->flames[i].P.ss);
            B->flames[i].budget = j.iterations;
            maxx = std::max<int>(maxx, (int)B->flames[i].P.flame.xf.size());
        }
        std::map<std::string, uint32_t> by_src;
        size_t hist_px = 0, rgba_bytes = 0, tab_floats = 0, pal_floats = 0;
        for (uint32_t i = 0; i < n; ++i) {
            BatchFlame& F = B->flames[i];
            F.P.plan = make_plan(F.P.flame, B->rng, F.P.math, maxx, 128);
            F.P.table = make_table(F.P.plan, F.P.flame);
            auto it = by_src.find(F.P.plan.source);
            if (it == by_src.end()) {
                it = by_src.emplace(F.P.plan.source, (uint32_t)B->groups.size()).first;
                BatchGroup G;
                G.src = F.P.plan.source;
                G.table_size = F.P.plan.table_size;
                G.maxx = F.P.plan.maxx;
                B->groups.push_back(G);
            }
            F.group = it->second;
            BatchGroup& G = B->groups[F.group];
            G.members.push_back(i);
            G.max_pal = std::max<int>(G.max_pal, (int)(F.P.palette.size() / 4));
            F.hist_off = hist_px; hist_px += (size_t)F.P.wi * F.P.hi;
            F.rgba_off = rgba_bytes; rgba_bytes += (size_t)(F.P.wi / F.P.ss) * (F.P.hi / F.P.ss) * 4;
            F.tab_off = tab_floats; tab_floats += (F.P.table.size() + 3) / 4 * 4;
            F.pal_off = pal_floats; pal_floats += F.P.palette.size();
            B->total_samples += F.budget;
        }
        for (auto& G : B->groups) { G.mod = &r->module_for(G.src); G.mod->pins += 1; }
        B->hist.ensure(hist_px * 16);
        B->rgba.ensure(rgba_bytes);
        B->counters.ensure(n * 8);
        std::vector<float> tabs(tab_floats), pals(pal_floats), luts((size_t)n * 256);
        for (uint32_t i = 0; i < n; ++i) {
            BatchFlame& F = B->flames[i];
            std::copy(F.P.table.begin(), F.P.table.end(), tabs.begin() + F.tab_off);
            std::copy(F.P.palette.begin(), F.P.palette.end(), pals.begin() + F.pal_off);
            std::vector<float> lut = curve_lut(F.P.flame.tm);
            std::copy(lut.begin(), lut.end(), luts.begin() + (size_t)i * 256);
        }
        cudaStream_t s = r->stream;
        ck(cudaMemcpyAsync(B->tables.ensure(tabs.size() * 4), tabs.data(), tabs.size() * 4, cudaMemcpyHostToDevice, s), "upload tables");
        ck(cudaMemcpyAsync(B->palettes.ensure(pals.size() * 4), pals.data(), pals.size() * 4, cudaMemcpyHostToDevice, s), "upload palettes");
        ck(cudaMemcpyAsync(B->luts.ensure(luts.size() * 4), luts.data(), luts.size() * 4, cudaMemcpyHostToDevice, s), "upload curves");
        // Autotune: time each (schedule, threads, iterations a walker) on
        // 1/16 and 1/8 of every budget with the full run's walkers, and
        // extrapolate linearly in the iterations walked (burn-in included)
        // to the full run: the intercept is the per-flame work that does
        // not grow with the budget (histogram clears, density estimation,
        // tone map).  Scaling one trial's time by the iteration ratio
        // alone charged that fixed work more to shapes whose trials walk
        // a larger share of burn-in: it picked 256 threads x 256
        // iterations (4.59 s) over 128 x 4096 (3.87 s) on a 256-flame set.
        // The transform-sorted kernel regroups walkers so a warp runs one
        // transform's variations; where every transform carries the same
        // variations (the sort removes no divergence) one walker a thread
        // saves the regrouping.  The one-walker kernel's blocks are the
        // modules' 128 threads (its launch bounds).
        B->threads = common->threads ? (uint32_t)common->threads : 256;
        B->iters = common->iterations_per_thread ? common->iterations_per_thread : 1024;
        B->plain = common->schedule == 1;
        if (B->plain) B->threads = 128;
        if (tune) {
            double best = 1e30;
            bool best_plain = B->plain;
            struct Cand { bool plain; uint32_t t; };
            std::vector<Cand> cands;
            if (common->schedule != 1) for (uint32_t t : {128u, 256u, 512u}) cands.push_back({false, t});
            if (common->schedule != 2) cands.push_back({true, 128u});
            const uint32_t cand_i[] = {256, 1024, 4096};
            for (const Cand& c : cands)
                for (uint32_t it : cand_i) {
                    const uint32_t t = c.t;
                    B->plain = c.plain;
                    // (time ms, iterations walked) at 1/16 and 1/8; the
                    // first call of a shape also sizes its buffers.
                    double ms[2], walked[2], full = 0;
                    batch_enqueue(B.get(), t, it, 16, s, false);
                    for (int k = 0; k < 2; ++k) {
                        ck(cudaEventRecord(r->ev0, s), "event");
                        batch_enqueue(B.get(), t, it, k ? 8 : 16, s, false);
                        ck(cudaEventRecord(r->ev1, s), "event");
                        ck(cudaStreamSynchronize(s), "tune");
                        float e = 0.f;
                        ck(cudaEventElapsedTime(&e, r->ev0, r->ev1), "event time");
                        ms[k] = e;
                        walked[k] = 0;
                        for (auto& F : B->flames) walked[k] += (double)F.walkers * (double)(F.per_walker + F.P.burn_in);
                    }
                    for (auto& F : B->flames) {
                        const uint64_t per_full = (F.budget + F.walkers - 1) / F.walkers;
                        full += (double)F.walkers * (double)(per_full + F.P.burn_in);
                    }
                    const double slope = walked[1] > walked[0] ? (ms[1] - ms[0]) / (walked[1] - walked[0]) : 0.0;
                    const double per = slope > 0.0 ? ms[1] + slope * (full - walked[1]) : ms[1] * full / walked[1];
                    if (per < best) { best = per; B->threads = t; B->iters = it; best_plain = c.plain; }
                }
            B->plain = best_plain;
        }
        // Size the buffers for the real run, then capture it as a graph.
        batch_enqueue(B.get(), B->threads, B->iters, 1, s, true);
        ck(cudaStreamSynchronize(s), "batch warm-up");
        ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            batch_enqueue(B.get(), B->threads, B->iters, 1, s, true, false);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        ck(cudaStreamEndCapture(s, &B->graph), "end capture");
        ck(cudaGraphInstantiate(&B->exec, B->graph, 0), "graph instantiate");
        B->device = r->device;
        r->batches.insert(B.get());
        *out = B.release();
    });
}

FFB_API int ffb_batch_run(ffb_batch* b, void* stream, int32_t sync, double* ms) {
    return guard([&] {
        if (!b) fail(FFB_ERR_INVALID, "NULL batch");
        if (!b->r) fail(FFB_ERR_INVALID, "the batch's renderer was destroyed");
        ffb_renderer* r = b->r;
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        cudaStream_t s = stream ? (cudaStream_t)stream : r->stream;
        ck(cudaEventRecord(r->ev0, s), "event");
        ck(cudaGraphLaunch(b->exec, s), "graph launch");
        ck(cudaEventRecord(r->ev1, s), "event");
        if (sync || ms) {
            ck(cudaStreamSynchronize(s), "batch");
            float t = 0.f;
            ck(cudaEventElapsedTime(&t, r->ev0, r->ev1), "event time");
            if (ms) *ms = t;
        }
    });
}

FFB_API int ffb_batch_output(ffb_batch* b, uint32_t index, uint8_t* rgba, uint64_t* plotted) {
    return guard([&] {
        if (!b || index >= b->flames.size()) fail(FFB_ERR_INVALID, "no such batch item");
        if (!b->r) fail(FFB_ERR_INVALID, "the batch's renderer was destroyed");
        ffb_renderer* r = b->r;
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        const BatchFlame& F = b->flames[index];
        if (rgba) {
            const size_t bytes = (size_t)(F.P.wi / F.P.ss) * (F.P.hi / F.P.ss) * 4;
            ck(cudaMemcpyAsync(rgba, (uint8_t*)b->rgba.p + F.rgba_off, bytes, cudaMemcpyDeviceToHost, r->stream), "readback");
            ck(cudaStreamSynchronize(r->stream), "readback");
        }
        if (plotted) *plotted = (uint64_t)F.walkers * F.per_walker;
    });
}

FFB_API int ffb_batch_info(ffb_batch* b, uint64_t* total_samples, uint32_t* threads, uint32_t* iters_per_walker, uint32_t* groups) {
    return guard([&] {
        if (!b) fail(FFB_ERR_INVALID, "NULL batch");
        uint64_t t = 0;
        for (auto& F : b->flames) t += (uint64_t)F.walkers * F.per_walker;
        if (total_samples) *total_samples = t;
        if (threads) *threads = b->threads;
        if (iters_per_walker) *iters_per_walker = b->iters;
        if (groups) *groups = (uint32_t)b->groups.size();
    });
}

static void batch_orphan(ffb_batch* b) {
    for (auto& G : b->groups) G.mod = nullptr;
    b->r = nullptr;
}

FFB_API void ffb_batch_destroy(ffb_batch* b) {
    if (!b) return;
    if (b->r) {
        std::lock_guard<std::mutex> lk(b->r->mu);
        cudaSetDevice(b->r->device);
        cudaStreamSynchronize(b->r->stream);
        b->r->batches.erase(b);
        delete b;
        return;
    }
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    delete b;
}

// ------------------------------------------------------- differentiable ----
// The differentiable render (ffb_diff.cuh, ffb_diff_tail.cu): no reference
// counterpart.  One object holds a specialised module, the base coefficient
// table, the histogram of the last forward pass and the walkers'
// checkpoints; theta lives in the caller's device memory.

namespace ffb {
namespace {

// Host mirror of ffb_diff_args (ffb_diff.cuh).
struct DiffArgs {
    const void* table;
    const void* palette;
    void* hist;
    void* ckpt;
    const void* dh;
    void* grad;
    void* counters;
    void* fixed;
    uint32_t n_walkers, walker0, n_xf, pal_n;
    uint32_t seed_lo, seed_hi, burn_in, n_iters;
    int32_t width, height;
    float zoom, pan_x, pan_y, cos_r, sin_r;
};
static_assert(sizeof(DiffArgs) == 128, "diff launch record layout");

}  // namespace
}  // namespace ffb

struct ffb_diff {
    ffb_renderer* r = nullptr;
    int device = 0;
    Prepared P;
    Module* mod = nullptr;
    uint32_t n_xf = 0, nvn = 0, n_params = 0, n_iters = 0, n_ckpt = 0, window = 0, ckpt = 0;
    uint32_t smem_fwd = 0, smem_adj = 0;
    TonemapArgs ta{};
    double area = 0, white = 0, npx = 0;
    DevBuf table, base, oms, palette, lut, hist, ckpts, counters, dh, fixed;
    bool exact = false;                 // deterministic accumulation (job count_bits 64)

    ~ffb_diff() {
        for (DevBuf* b : {&table, &base, &oms, &palette, &lut, &hist, &ckpts, &counters, &dh, &fixed}) b->release();
        if (mod) mod->pins -= 1;
    }

    DiffArgs args(cudaStream_t) const {
        DiffArgs a{};
        a.table = table.p; a.palette = palette.p; a.hist = hist.p; a.ckpt = ckpts.p; a.dh = dh.p; a.grad = nullptr;
        a.counters = counters.p;
        a.fixed = exact ? fixed.p : nullptr;
        a.n_walkers = P.walkers; a.walker0 = 0; a.n_xf = n_xf; a.pal_n = (uint32_t)(P.palette.size() / 4);
        a.seed_lo = (uint32_t)P.seed; a.seed_hi = (uint32_t)(P.seed >> 32); a.burn_in = P.burn_in; a.n_iters = n_iters;
        a.width = (int32_t)P.wi; a.height = (int32_t)P.hi;
        const double rot = (double)P.flame.rotation;
        a.zoom = P.flame.zoom; a.pan_x = (float)P.flame.pan_x; a.pan_y = (float)P.flame.pan_y;
        a.cos_r = (float)std::cos(rot); a.sin_r = (float)std::sin(rot);
        return a;
    }
};

FFB_API int ffb_diff_create(ffb_renderer* r, const char* config, size_t len, const ffb_job* job, uint32_t window,
                            uint32_t checkpoint, ffb_diff** out) {
    return guard([&] {
        if (!r || !out) fail(FFB_ERR_INVALID, "NULL argument");
        *out = nullptr;
        if (window == 0) window = 16;
        if (checkpoint == 0) checkpoint = 64;
        if (window > 32) fail(FFB_ERR_INVALID, "window must be at most 32 iterations");
        if (checkpoint > 256) fail(FFB_ERR_INVALID, "checkpoint interval must be at most 256 iterations");
        if (!job) fail(FFB_ERR_INVALID, "job is NULL");
        ffb_job j = *job;
        j.rng = RNG_PHILOX;
        const bool exact = job->count_bits == 64;
        if (job->count_bits != 0 && job->count_bits != 32 && !exact) fail(FFB_ERR_INVALID, "count_bits must be 32 or 64");
        j.count_bits = 32;
        std::unique_ptr<ffb_diff> d(new ffb_diff);
        d->exact = exact;
        d->P = prepare(config, len, &j);
        if (d->P.flame.filter.on()) fail(FFB_ERR_INVALID, "the differentiable render has no spatial filter (filter_radius)");
        const Flame& f = d->P.flame;
        if (d->P.ss != 1) fail(FFB_ERR_INVALID, "the differentiable render has no supersampling");
        if (!f.fin_used.empty() || !f.lnk_used.empty())
            fail(FFB_ERR_CONFIG, "the differentiable render takes no final or linked transforms");
        if (f.de.max_radius > 0.0f) fail(FFB_ERR_CONFIG, "the differentiable render takes no density estimation");
        if (f.sym.kind != 0) fail(FFB_ERR_CONFIG, "the differentiable render takes no post-symmetry");
        if (job->transparent) fail(FFB_ERR_INVALID, "the differentiable render is opaque");
        if (f.tm.mode != 1 || f.tm.highlight != 0 || f.tm.saturation != 1.0f || f.tm.hue_shift != 0.0f)
            fail(FFB_ERR_CONFIG, "the differentiable tone map is the log mode with clip highlights and no HSV adjustment");
        const uint64_t iters = d->P.per_walker + d->P.burn_in;
        if (iters > 0xFFFFFFFFull) fail(FFB_ERR_INVALID, "too many iterations a walker");
        d->n_iters = (uint32_t)iters;
        d->window = window;
        d->ckpt = checkpoint;
        d->n_ckpt = (d->n_iters + checkpoint - 1) / checkpoint;
        std::lock_guard<std::mutex> lk(r->mu);
        r->begin();
        d->r = r;
        d->P.plan = make_plan(f, RNG_PHILOX, d->P.math, 0, (int)d->P.threads, false, false, (int)window, (int)checkpoint);
        d->P.table = make_table(d->P.plan, f);
        d->n_xf = (uint32_t)f.xf.size();
        d->nvn = (uint32_t)d->P.plan.normal.size();
        d->n_params = d->n_xf * (7 + d->nvn);
        Module& m = r->module_for(d->P.plan.source);
        m.pins += 1;
        d->mod = &m;
        std::vector<float> oms(d->n_xf);
        for (uint32_t k = 0; k < d->n_xf; ++k) oms[k] = 1.0f - f.xf[k].speed;
        std::vector<float> lut = curve_lut(f.tm);
        auto up = [&](DevBuf& b, const void* src, size_t bytes) {
            ck(cudaMemcpyAsync(b.ensure(bytes), src, bytes, cudaMemcpyHostToDevice, r->stream), "upload");
        };
        up(d->base, d->P.table.data(), d->P.table.size() * 4);
        d->table.ensure(d->P.table.size() * 4);
        up(d->oms, oms.data(), oms.size() * 4);
        up(d->palette, d->P.palette.data(), d->P.palette.size() * 4);
        up(d->lut, lut.data(), lut.size() * 4);
        d->npx = (double)d->P.wi * (double)d->P.hi;
        d->hist.ensure((size_t)d->P.wi * d->P.hi * 16);
        d->dh.ensure((size_t)d->P.wi * d->P.hi * 16);
        d->ckpts.ensure((size_t)d->n_ckpt * d->P.walkers * 16);
        d->counters.ensure(16);
        if (exact) d->fixed.ensure((size_t)d->P.wi * d->P.hi * 32);
        ck(cudaStreamSynchronize(r->stream), "upload");
        d->ta = tonemap_args(f, d->P.wi, d->P.hi, 1.0, 0, true);
        const double ppu = (double)std::min(d->P.wi, d->P.hi) * 0.25 * (double)f.zoom;
        d->area = d->npx / (ppu * ppu);
        d->white = f.tm.white_level;
        const uint32_t table_bytes = (uint32_t)((d->P.plan.table_size + 3) / 4) * 16;
        d->smem_fwd = table_bytes + (uint32_t)(d->P.palette.size() / 4) * 16;
        d->smem_adj = d->smem_fwd + (uint32_t)d->P.plan.maxx * (7 + d->nvn) * d->P.threads * 4;
        if (d->smem_adj > 227 * 1024) fail(FFB_ERR_TOO_LARGE, "too many parameters for the adjoint's shared memory: use fewer threads");
        if (d->smem_adj > 48 * 1024) {
            ck(cudaFuncSetAttribute((const void*)m.dadjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d->smem_adj), "smem attribute");
        }
        if (d->smem_fwd > 48 * 1024) {
            ck(cudaFuncSetAttribute((const void*)m.dforward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d->smem_fwd), "smem attribute");
        }
        d->device = r->device;
        r->diffs.insert(d.get());
        *out = d.release();
    });
}

FFB_API int ffb_diff_specialize(const char* config, size_t len, uint32_t window, uint32_t checkpoint, size_t* cubin_bytes,
                                char* source, size_t source_len) {
    return guard([&] {
        if (!config) fail(FFB_ERR_INVALID, "config is NULL");
        Flame f;
        try { f = parse_config_text(std::string(config, len)); }
        catch (const std::exception& e) { fail(FFB_ERR_CONFIG, std::string("config did not parse: ") + e.what()); }
        Plan p = make_plan(f, RNG_PHILOX, MATH_PRECISE, 0, 128, false, false, window ? (int)window : 16, checkpoint ? (int)checkpoint : 64);
        std::vector<char> cubin = ffb_renderer::nvrtc_cubin(p.source);
        if (cubin_bytes) *cubin_bytes = cubin.size();
        if (source && source_len) {
            size_t n = std::min(source_len - 1, p.source.size());
            std::memcpy(source, p.source.data(), n);
            source[n] = 0;
        }
    });
}

FFB_API int ffb_diff_layout(ffb_diff* d, uint32_t* n_xforms, uint32_t* n_variations, uint32_t* walkers, uint32_t* iterations,
                            char* names, size_t names_cap) {
    return guard([&] {
        if (!d) fail(FFB_ERR_INVALID, "NULL object");
        if (n_xforms) *n_xforms = d->n_xf;
        if (n_variations) *n_variations = d->nvn;
        if (walkers) *walkers = d->P.walkers;
        if (iterations) *iterations = d->n_iters;
        if (names) {
            std::string s;
            for (size_t j = 0; j < d->P.plan.normal.size(); ++j) s += (j ? "," : "") + std::string(d->P.plan.normal[j]->name);
            if (s.size() + 1 > names_cap) fail(FFB_ERR_INVALID, "names buffer too small");
            std::memcpy(names, s.c_str(), s.size() + 1);
        }
    });
}

FFB_API int ffb_diff_theta(ffb_diff* d, float* theta) {
    return guard([&] {
        if (!d || !theta) fail(FFB_ERR_INVALID, "NULL argument");
        const Flame& f = d->P.flame;
        for (uint32_t k = 0; k < d->n_xf; ++k) {
            const XForm& x = f.xf[k];
            const float a[6] = {x.a, x.b, x.c, x.d, x.e, x.f};
            for (int i = 0; i < 6; ++i) theta[k * 6 + i] = a[i];
            for (uint32_t j = 0; j < d->nvn; ++j) theta[d->n_xf * 6 + k * d->nvn + j] = x.var_weight(d->P.plan.normal[j]);
            theta[d->n_xf * (6 + d->nvn) + k] = x.color;
        }
    });
}

FFB_API int ffb_diff_forward(ffb_diff* d, const float* d_theta, float* d_image, float* d_hist, void* stream) {
    return guard([&] {
        if (!d || !d_theta || !d_image) fail(FFB_ERR_INVALID, "NULL argument");
        if (!d->r) fail(FFB_ERR_INVALID, "the differentiable render's renderer was destroyed");
        ck(cudaSetDevice(d->r->device), "cudaSetDevice");
        cudaStream_t s = (cudaStream_t)stream;
        Module& m = *d->mod;
        {
            const float* th = d_theta;
            const void* bp = d->base.p;
            const void* op = d->oms.p;
            void* tp = d->table.p;
            int nx = (int)d->n_xf;
            void* a[] = {&th, &bp, &op, &tp, &nx};
            ck(cudaLaunchKernel((const void*)m.dtheta, dim3(1), dim3(256), a, 0, s), "launch ffb_diff_theta");
        }
        const size_t hb = (size_t)d->P.wi * d->P.hi * 16;
        if (d->exact) ck(cudaMemsetAsync(d->fixed.p, 0, hb * 2, s), "clear histogram");
        else ck(cudaMemsetAsync(d->hist.p, 0, hb, s), "clear histogram");
        ck(cudaMemsetAsync(d->counters.p, 0, 16, s), "clear counters");
        DiffArgs A = d->args(s);
        void* a[] = {&A};
        const uint32_t blocks = (d->P.walkers + d->P.threads - 1) / d->P.threads;
        ck(cudaLaunchKernel((const void*)m.dforward, dim3(blocks), dim3(d->P.threads), a, d->smem_fwd, s), "launch ffb_diff_forward");
        if (d->exact) ck(launch_fixed_to_float((const ulonglong4*)d->fixed.p, (size_t)d->npx, (float4*)d->hist.p, s), "fixed to float");
        ck(launch_diff_tonemap((const float4*)d->hist.p, (size_t)d->npx, d->ta, (const float*)d->lut.p, (const uint64_t*)d->counters.p,
                               d->npx, d->area, d->white, (float4*)d_image, s), "differentiable tone map");
        if (d_hist) ck(cudaMemcpyAsync(d_hist, d->hist.p, hb, cudaMemcpyDeviceToDevice, s), "histogram copy");
    });
}

FFB_API int ffb_diff_backward(ffb_diff* d, const float* d_grad_image, double* d_grad_theta, float* d_grad_hist, void* stream) {
    return guard([&] {
        if (!d || !d_grad_image || !d_grad_theta) fail(FFB_ERR_INVALID, "NULL argument");
        if (!d->r) fail(FFB_ERR_INVALID, "the differentiable render's renderer was destroyed");
        ck(cudaSetDevice(d->r->device), "cudaSetDevice");
        cudaStream_t s = (cudaStream_t)stream;
        ck(launch_diff_tonemap_vjp((const float4*)d->hist.p, (const float4*)d_grad_image, (size_t)d->npx, d->ta, (const float*)d->lut.p,
                                   (const uint64_t*)d->counters.p, d->npx, d->area, d->white, (float4*)d->dh.p, s),
           "tone map gradient");
        ck(cudaMemsetAsync(d_grad_theta, 0, (size_t)d->n_params * 8, s), "clear gradient");
        DiffArgs A = d->args(s);
        A.grad = d_grad_theta;
        void* a[] = {&A};
        const uint32_t blocks = (d->P.walkers + d->P.threads - 1) / d->P.threads;
        ck(cudaLaunchKernel((const void*)d->mod->dadjoint, dim3(blocks), dim3(d->P.threads), a, d->smem_adj, s), "launch ffb_diff_adjoint");
        if (d_grad_hist)
            ck(cudaMemcpyAsync(d_grad_hist, d->dh.p, (size_t)d->P.wi * d->P.hi * 16, cudaMemcpyDeviceToDevice, s), "gradient copy");
    });
}

FFB_API int ffb_diff_samples(ffb_diff* d, uint64_t* plotted, uint64_t* inframe, void* stream) {
    return guard([&] {
        if (!d) fail(FFB_ERR_INVALID, "NULL object");
        ck(cudaSetDevice(d->device), "cudaSetDevice");
        uint64_t c[2] = {0, 0};
        ck(cudaMemcpyAsync(c, d->counters.p, 16, cudaMemcpyDeviceToHost, (cudaStream_t)stream), "readback");
        ck(cudaStreamSynchronize((cudaStream_t)stream), "readback");
        if (plotted) *plotted = c[0];
        if (inframe) *inframe = c[1];
    });
}

FFB_API int ffb_diff_jacobians(ffb_diff* d, int32_t xform, uint32_t n, const float* xs, const float* ys, const float* words, float* out) {
    return guard([&] {
        if (!d || !xs || !ys || !words || !out) fail(FFB_ERR_INVALID, "NULL argument");
        if (!d->r) fail(FFB_ERR_INVALID, "the differentiable render's renderer was destroyed");
        if (xform < 0 || (uint32_t)xform >= d->n_xf) fail(FFB_ERR_INVALID, "no such transform");
        std::lock_guard<std::mutex> lk(d->r->mu);
        d->r->begin();
        ffb_renderer* r = d->r;
        const size_t nn = n;
        float* d_in = (float*)r->tmp_in.ensure(nn * 4 * 2 + nn * kApplyWords * 4);
        float* d_x = d_in, *d_y = d_in + nn, *d_w = d_in + 2 * nn;
        ck(cudaMemcpyAsync(d_x, xs, nn * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        ck(cudaMemcpyAsync(d_y, ys, nn * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        ck(cudaMemcpyAsync(d_w, words, nn * kApplyWords * 4, cudaMemcpyHostToDevice, r->stream), "upload");
        const size_t ob = nn * d->nvn * 6 * 4;
        float* d_out = (float*)r->f_out.ensure(std::max<size_t>(ob, 4));
        const void* tp = d->base.p;
        int k = xform, ni = (int)n;
        void* a[] = {&tp, &k, &ni, &d_x, &d_y, &d_w, &d_out};
        ck(cudaLaunchKernel((const void*)d->mod->dprobe, dim3((n + 127) / 128), dim3(128), a, 0, r->stream), "launch ffb_dprobe");
        ck(cudaMemcpyAsync(out, d_out, ob, cudaMemcpyDeviceToHost, r->stream), "readback");
        ck(cudaStreamSynchronize(r->stream), "jacobians");
    });
}

static void diff_orphan(ffb_diff* d) {
    d->mod = nullptr;
    d->r = nullptr;
}

FFB_API void ffb_diff_destroy(ffb_diff* d) {
    if (!d) return;
    if (d->r) {
        std::lock_guard<std::mutex> lk(d->r->mu);
        cudaSetDevice(d->r->device);
        cudaDeviceSynchronize();
        d->r->diffs.erase(d);
        delete d;
        return;
    }
    cudaSetDevice(d->device);
    cudaDeviceSynchronize();
    delete d;
}

// ------------------------------------------------------------ drop-in ----
FFB_API uint8_t* fae_alloc(size_t len) { return (uint8_t*)std::malloc(std::max<size_t>(len, 1)); }
FFB_API void fae_free(uint8_t* ptr, size_t) { std::free(ptr); }
FFB_API const uint8_t* fae_output_ptr(void) { return g_output.data(); }
FFB_API size_t fae_output_len(void) { return g_output.size(); }
FFB_API const uint8_t* fae_info_ptr(void) { return g_info.data(); }
FFB_API size_t fae_info_len(void) { return g_info.size(); }

FFB_API int32_t fae_call(const uint8_t* req, size_t req_len, const uint8_t* data, size_t data_len) {
    std::vector<uint8_t> out;
    std::string info;
    int st = guard([&] {
        std::string text(req ? (const char*)req : "", req ? req_len : 0);
        JsonPtr j;
        try { j = json_parse(text); }
        catch (const std::exception& e) { fail(FFB_ERR_INVALID, std::string("request is not JSON: ") + e.what()); }
        std::lock_guard<std::mutex> lk(g_fae_mu);
        fae_dispatch(*j, data, data_len, out, info);
    });
    if (st == FFB_OK) {
        g_output = std::move(out);
        g_info.assign(info.begin(), info.end());
        return 0;
    }
    g_output.assign(g_err.begin(), g_err.end());
    g_info.clear();
    return 1;
}
