// ffb_flame.hpp -- the flame description the render path consumes.
//
// The `.fae` / `.fflame` JSON subset of the 2-D flame path
// (src/config/fractal_config.rs:178-520, src/scene/transforms.rs:337-420,
// 1348-1558, 2016-2091), the variation registry subset this build carries
// (src/variations/defs/mod.rs:446, positions kept as registry ids), the
// per-flame local variation order (src/scene/transforms.rs:40-70, 668-682,
// 2297-2319), the palette table (src/scene/palette.rs:265-360, 453-482,
// 684-800) and the tone-map parameters (src/config/defaults.rs:18-52,
// src/renderer/compute_kernel.rs:1796-1866).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "ffb_json.hpp"

namespace ffb {

// A variation's packed parameter row: its user parameters, then the values
// its `wgsl_init` derives from them (VariationDef::slot_count,
// src/variations/definition.rs:452-454).  klein_group's 6 + 16 is the widest.
constexpr int kMaxVarSlots = 24;

enum VarFlags {
    VF_XF = 1,        // Feature::NeedsTransform reading the affine: the body takes its transform's a..f
    VF_W = 2,         // the body reads its own weight (transforms[id].variations[idx])
    VF_PRE = 4,       // VariationPhase::Pre: temp = V(temp), before the weighted sum
    VF_POST = 8,      // VariationPhase::Post: result = V(result), after it
    VF_JAC = 16,      // has a Jacobian (dj_*) for the differentiable render
    VF_DC = 32,       // Feature::WritesColor: may write the iteration's colour register (vc)
    VF_SUB = 64,      // steps a subflame (subflame_wf, pre_subflame_wf): generated, not a plain body
    VF_REPLACE = 128, // Feature::Replace: its w * V(p) overwrites the normal phase's sum, after the others
    VF_HIDE = 256,    // Feature::CanHide: the body sets (or clears) the iteration's hide flag
};

struct VarDef {
    const char* name;
    int id;            // position in the reference's ALL_VARIATIONS
    int draws;         // Feature::NeedsRng: draws the body takes, in its order
    int nparams;       // user parameters
    const char* pname[kMaxVarSlots];
    float pdef[kMaxVarSlots];
    const char* fn;    // device function name
    int flags;         // VarFlags
    int nderived;      // init_param_count
    // The variation's `wgsl_init` restated on the host in f32: user -> derived.
    void (*derive)(const float* user, float* out);
    // Per-walker state a call carries to the next (state_count,
    // definition.rs; the 2-D slots this build keeps), and the draws its
    // `wgsl_state_init` takes at every dispatch start (klein_group's one).
    int state = 0;
    int init_draws = 0;
    int slots() const { return nparams + nderived; }
    bool needs_rng() const { return draws > 0; }
};

const VarDef* registry_find(const std::string& name);
const std::vector<const VarDef*>& registry_all();

struct XForm {
    float a = 1, b = 0, c = 0, d = 1, e = 0, f = 0;
    float pa = 1, pb = 0, pc = 0, pd = 1, pe = 0, pf = 0;
    bool post = false;
    float weight = 1, color = 0.5f, speed = 0, opacity = 1;
    // Step 3 of the colour flow when a variation writes the colour register
    // (main_template.wgsl:294-306, 486-490); a `.fflame` without the field
    // reads 0 (transforms.rs:1533-1540).
    float direct_color = 0;
    // (variation, weight) in the transform's dispatch order.
    std::vector<std::pair<const VarDef*, float>> vars;
    // "name.param" -> value
    std::vector<std::pair<std::string, float>> params;
    std::vector<int> final_att;   // indices into the finals pool
    std::vector<int> linked_att;  // indices into the linked pool
    float param(const VarDef* v, int j) const;
    // The packed row: user parameters, then the derived values.
    void slot_values(const VarDef* v, float* out) const;
    float var_weight(const VarDef* v) const;
};

struct CurvePt { float x, y; };

struct ToneMap {
    int mode = 1;              // 0 linear, 1 logarithmic, 2 density
    int highlight = 0;         // 0 clip, 1 max_norm, 2 reinhard, 3 filmic, 4 agx, 5 agx_punchy
    float exposure = 1.0f, gamma = 4.0f, gamma_threshold = 5.0f, brightness = 4.0f, vibrancy = 1.0f;
    float white_level = 200.0f, saturation = 1.0f, hue_shift = 0.0f;
    float alpha_blend_low = 0.3f, alpha_blend_high = 0.8f, density_scale = 1.0f;
    bool levels_enabled = true;
    float levels_low = 0.0f, levels_high = 10.0f, levels_gamma = 0.5f;
    float background[3] = {0, 0, 0};
    bool use_curve = true;
    std::vector<CurvePt> curve{{0.f, 0.f}, {1.f, 1.f}};
};

struct DensityEstimation {
    float max_radius = 0.0f;   // final-image pixels; 0 = off
    float min_radius = 0.0f;
    float curve = 0.4f;
};

// Plot-time symmetry (scene/transforms.rs:2093-2190, GpuPostSymmetry in
// gpu/buffers.rs:936-966): every kept sample is plotted once per copy.
struct PostSym {
    int kind = 0;              // 0 none, 1 x axis (reflects y), 2 y axis (reflects x), 3 point
    int order = 3;             // point mode: copies, clamped to 1..32
    float cx = 0.0f, cy = 0.0f;
    float distance = 1.25f;    // axis modes: total separation of the pair
    float rotation = 0.0f;     // axis modes: pre-rotation, radians (rotation_deg.to_radians())
    int copies() const { return kind == 0 ? 1 : kind == 3 ? order : 2; }
};

// The spatial filter (Apophysis `filter`; fractal_config.rs:381-395,
// compute_kernel.rs:1663-1725): a bilateral Gaussian on each batch's
// histogram before it is accumulated; off at radius 0.
struct SpatialFilter {
    float radius = 0.0f;       // Gaussian sigma in pixels
    float blur_edges = 0.0f;   // 0 strict edge preservation .. 1 near-uniform
    bool on() const { return radius > 0.0f; }
};

// A subflame (FractalConfig.subflames, gpu/buffers.rs:160-200): an inner
// flame that subflame_wf steps one visible iteration at a time, its normals
// picked by weight (no xaos) and its finals applied to the output.
struct SubFlame {
    std::vector<XForm> xf, fin;
};

// Attachments (transforms.rs:470-480; gpu/buffers.rs:600-680): each normal
// transform's linked chain -- transforms applied after it in the same
// iteration, their output the walker's next point -- and its final chain,
// applied at plot time only.  Indices past their pool are dropped and a
// chain holds at most kMaxAttach (the reference logs and does the same).
constexpr int kMaxAttach = 32;

struct Flame {
    std::vector<XForm> xf;              // normal transforms
    std::vector<XForm> lnk;             // linked transforms pool
    std::vector<XForm> fin;             // final transforms pool
    std::vector<int> fin_chain;         // the final chain every normal runs, when they share one
    bool fin_uniform = true;            // every normal has the same final chain
    std::vector<int> fin_used;          // finals some normal attaches, pool order
    std::vector<int> lnk_used;          // linked transforms some normal attaches, pool order
    std::vector<const VarDef*> local;   // local variation order (parent, then subflames)
    std::vector<SubFlame> sub;          // at most 8 (MAX_SUBFLAMES, buffers.rs:36-44)
    // The solo transform (Apophysis soloxform; gpu/buffers.rs:523-536):
    // every other normal transform still moves the walk but plots nothing
    // (opacity 0); -1 none.
    int solo = -1;
    SpatialFilter filter;
    // Xaos (utilities.wgsl:106-137): row-major n_xf x n_xf transition
    // weights, empty when every weight is 1 (Flame::has_xaos, xaos.rs:29-40).
    std::vector<float> xaos;
    // Orbit refresh (compute_kernel.rs:45-60; main_template.wgsl:125-145):
    // where the xaos walk decides which closed group an orbit ends in, every
    // dispatch restarts the walkers w with (w + the dispatch's seed) % 4 == 0.
    uint32_t orbit_refresh = 0;
    float zoom = 1.0f;
    double pan_x = 0.0, pan_y = 0.0;
    float rotation = 0.0f;
    PostSym sym;
    // palette
    std::vector<float> stop_pos, stop_col;
    int palette_size = 256;
    float palette_rotation = 0.0f;
    bool palette_reverse = false;
    // The lookup pipeline's squeeze and redistribution (palette.rs:485-800):
    // mode 0 linear (repeat count `palette_squeeze`), 1 geometric (octave
    // ratio `palette_squeeze_falloff`); then exponential redistribution.
    int palette_squeeze_mode = 0;
    float palette_squeeze = 1.0f, palette_squeeze_falloff = 0.5f, palette_log_strength = 0.0f;
    // Colour mode (palette.rs:8-18): 0 palette, 1 speed -- each walker
    // carries an RGB colour mixed toward the palette's entry at its step's
    // speed, clamp(ln(10 speed + 1) / 3, 0, 1), by `speed_factor`
    // (main_template.wgsl:483-508; utilities.wgsl:148-156).
    int color_mode = 0;
    float speed_factor = 0.5f;
    ToneMap tm;
    DensityEstimation de;
    uint64_t max_iterations = 1000000000ull;
    bool deterministic_rng = false;
    uint64_t seed = 12345;               // first dispatch seed, compute_kernel.rs:3541-3553
};

// Parse a `.fae` configuration.  Throws std::runtime_error with the reason.
Flame parse_config(const Json& cfg);
Flame parse_config_text(const std::string& text);

// The palette table the chaos game samples: `size` entries of linear RGB
// (f16 texels of the stop gradient, decoded with pow 2.2), RGBA f32.
std::vector<float> palette_table(const Flame& f);

// The tone curve LUT (tonemap.rs:289-304): 256 f16-rounded values.
std::vector<float> curve_lut(const ToneMap& tm);
float f16_round(float v);

}  // namespace ffb
