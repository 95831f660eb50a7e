// ffb_codegen.cpp -- see ffb_codegen.hpp.

#include "ffb_codegen.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <sstream>
#include <stdexcept>

#include "ffb_device_src.inc"

namespace ffb {

namespace {

constexpr int kSymBlock = 6 + 64;            // post-symmetry table block (floats)
constexpr int kMaxDrawSlots = 64;            // draws an iteration (pick, opacity, variations)

// Normal-phase variations: those a normal transform uses at a weight other
// than 0, in local order.  The reference emits every active variation and
// gates each on `xform.variations[idx] != 0.0` (shader_builder_v2.rs
// 2755-2763); one no transform uses never fires, so leaving it out changes
// nothing.
std::vector<const VarDef*> normal_vars(const Flame& f) {
    std::vector<const VarDef*> out;
    for (const VarDef* v : f.local) {
        bool used = false;
        for (auto& x : f.xf) used |= x.var_weight(v) != 0.0f;
        if (used) out.push_back(v);
    }
    return out;
}

std::vector<const VarDef*> final_vars(const Flame& f, const XForm& x) {
    std::vector<const VarDef*> out;
    for (const VarDef* v : f.local) if (x.var_weight(v) != 0.0f) out.push_back(v);
    return out;
}

// Where one call of a variation finds its inputs, as source expressions:
// its packed parameter row (`prm(q)`), its own weight and its transform's
// affine (`xf(0..5)` = a..f), and the first of its draw slots.
struct Site {
    std::function<std::string(int)> prm;
    std::string w;
    std::function<std::string(int)> xf;
    int slot = -1;
};

// Normal transform k's site (k a source expression).
Site normal_site(const Plan& p, int j, const std::string& k) {
    Site c;
    const int off = p.vp_off[j];
    c.prm = [off, k](int q) { return "sm[T_VP + " + std::to_string(off + q) + " * FFB_MAXX + " + k + "]"; };
    c.w = "sm[T_VW + " + std::to_string(j) + " * FFB_MAXX + " + k + "]";
    c.xf = [k](int f) { return "sm[T_XF + " + std::to_string(f) + " * FFB_MAXX + " + k + "]"; };
    c.slot = p.normal_slot[j];
    return c;
}

// Final c's site: its record q (affine at q[0..5], weights at q[13..]).
Site final_site(const Plan::Fin& fi, int j) {
    Site c;
    const int nv = (int)fi.vars.size(), off = 13 + nv + fi.prm_off[j];
    c.prm = [off](int q) { return "q[" + std::to_string(off + q) + "]"; };
    c.w = "q[" + std::to_string(13 + j) + "]";
    c.xf = [](int f) { return "q[" + std::to_string(f) + "]"; };
    c.slot = fi.slot[j];
    return c;
}

// `v_name(px, py[, rng, slot][, params...][, w][, a..f], ox, oy)`.
std::string call(const VarDef* v, const Site& c, const char* px = "x", const char* py = "y") {
    std::ostringstream o;
    o << v->fn << "(" << px << ", " << py;
    if (v->draws) o << ", rng, " << c.slot;
    for (int q = 0; q < v->slots(); ++q) o << ", " << c.prm(q);
    if (v->flags & VF_W) o << ", " << c.w;
    if (v->flags & VF_XF) for (int f = 0; f < 6; ++f) o << ", " << c.xf(f);
    o << ", ox, oy)";
    return o.str();
}

// The Jacobian of a variation body (ffb_diff_jac.cuh): "v_name" -> "dj_name".
// Only variations flagged VF_JAC have one; they take at most one draw.
std::string jcall(const VarDef* v, const Site& c) {
    std::ostringstream o;
    o << "dj_" << (v->fn + 2) << "(x, y";
    if (v->draws) o << ", rng.draw(" << c.slot << ")";
    for (int q = 0; q < v->slots(); ++q) o << ", " << c.prm(q);
    o << ")";
    return o.str();
}

// The three phases of apply_variations (shader_builder_v2.rs:2589-2800):
// Pre variations replace the input point in turn (`temp = V(temp)`), the
// others sum `w * V(temp)` from zero, Post variations replace the sum
// (`result = V(result)`); each gated on its weight, in local order within
// its phase.  `site(j)` locates variation j of `vars`; `gate` false drops
// the weight test (the per-transform form lists only the variations the
// transform uses).
void emit_phases(std::ostringstream& s, const std::vector<const VarDef*>& vars,
                 const std::function<Site(int)>& site, const char* ind, bool gate) {
    s << ind << "float tx = x, ty = y, rx = 0.0f, ry = 0.0f, ox, oy;\n";
    auto open = [&](const Site& c) {
        s << ind << "{ const float w = " << c.w << "; " << (gate ? "if (w != 0.0f) { " : "{ ");
    };
    for (int pass = 0; pass < 3; ++pass) {
        for (size_t j = 0; j < vars.size(); ++j) {
            const VarDef* v = vars[j];
            const int ph = (v->flags & VF_PRE) ? 0 : (v->flags & VF_POST) ? 2 : 1;
            if (ph != pass) continue;
            const Site c = site((int)j);
            open(c);
            if (ph == 0) s << call(v, c, "tx", "ty") << "; tx = ox; ty = oy;";
            else if (ph == 1) s << call(v, c, "tx", "ty") << "; rx = rx + w * ox; ry = ry + w * oy;";
            else s << call(v, c, "rx", "ry") << "; rx = ox; ry = oy;";
            s << " } }   // " << v->name << "\n";
        }
    }
}

// The differentiable render's generated functions and kernels.
void emit_diff(std::ostringstream& s, const Plan& p) {
    const int NVN = (int)p.normal.size();
    s << kDiffJacSrc << "\n";
    s << "#define FFB_WINDOW " << p.diff_window << "\n#define FFB_CKPT " << p.diff_ckpt << "\n";
    s << "#define FFB_NPARAM " << p.maxx * (7 + NVN) << "\n";
    // Normal phase of transform k for the adjoint: the weight gradient of
    // each variation (a . V_j(x, y)) into gw[j * P], and J = sum_j w_j J_j.
    s << "template <class R> __device__ __forceinline__ void ffb_dnormal(const float* __restrict__ sm, int k, float x, float y, R& rng, "
         "float ax, float ay, float* __restrict__ gw, int P, float4& J) {\n";
    s << "    J = make_float4(0.f, 0.f, 0.f, 0.f);\n    float ox, oy;\n";
    for (int j = 0; j < NVN; ++j) {
        const VarDef* v = p.normal[j];
        const Site c = normal_site(p, j, "k");
        s << "    { " << call(v, c) << "; const float g = ax * ox + ay * oy; if (isfinite(g)) gw["
          << j << " * P] += g;\n      const float w = " << c.w << "; if (w != 0.0f) { const float4 jj = "
          << jcall(v, c) << "; J.x += w * jj.x; J.y += w * jj.y; J.z += w * jj.z; J.w += w * jj.w; } }   // " << v->name << "\n";
    }
    s << "    if (!(isfinite(J.x) && isfinite(J.y) && isfinite(J.z) && isfinite(J.w))) J = make_float4(0.f, 0.f, 0.f, 0.f);\n}\n";
    // One normal variation's value and Jacobian (the probe).
    s << "template <class R> __device__ __forceinline__ void ffb_dvar_one(const float* __restrict__ sm, int j, int k, float x, float y, R& rng, "
         "float& ox, float& oy, float4& J) {\n    switch (j) {\n";
    for (int j = 0; j < NVN; ++j) {
        const VarDef* v = p.normal[j];
        const Site c = normal_site(p, j, "k");
        s << "    case " << j << ": " << call(v, c) << "; J = " << jcall(v, c) << "; break;\n";
    }
    s << "    default: ox = 0.f; oy = 0.f; J = make_float4(0.f, 0.f, 0.f, 0.f); break;\n    }\n}\n";
    s << kDiffSrc << "\n";
}

std::string jac_names() {
    std::string o;
    for (const VarDef* v : registry_all()) if (v->flags & VF_JAC) o += (o.empty() ? "" : ", ") + std::string(v->name);
    return o;
}

}  // namespace

Plan make_plan(const Flame& f, int rng_mode, int math_mode, int maxx, int threads, bool per_xform, bool exact,
               int diff_window, int diff_ckpt, bool emit, bool defer) {
    Plan p;
    p.exact = exact;
    p.emit = emit;
    p.defer = defer && !emit && diff_window == 0;
    p.diff_window = diff_window;
    p.diff_ckpt = diff_ckpt;
    p.rng_mode = rng_mode;
    p.math_mode = math_mode;
    p.per_xform = per_xform;
    p.threads = threads;
    p.maxx = std::max<int>(maxx, (int)f.xf.size());
    p.normal = normal_vars(f);
    // Draw slots: 0 the transform pick, 1 the opacity test, then each
    // NeedsRng variation's draws (consecutive, in its body's order): the
    // normal phase's in local order, then each final's.
    int slot = 2, vp = 0;
    for (const VarDef* v : p.normal) {
        p.normal_slot.push_back(v->draws ? slot : -1);
        slot += v->draws;
        p.vp_off.push_back(vp);
        vp += v->slots();
    }
    p.vp_slots = vp;
    for (int c : f.fin_chain) {
        Plan::Fin fi;
        fi.vars = final_vars(f, f.fin[c]);
        int fo = 0;
        for (const VarDef* v : fi.vars) {
            fi.slot.push_back(v->draws ? slot : -1);
            slot += v->draws;
            fi.prm_off.push_back(fo);
            fo += v->slots();
        }
        fi.prm_slots = fo;
        p.fin.push_back(fi);
    }
    p.n_slots = slot;
    // Philox words live in registers (4 a block): a bound keeps them there.
    if (p.n_slots > kMaxDrawSlots)
        throw std::runtime_error("the flame's variations take " + std::to_string(p.n_slots - 2) +
                                 " random draws an iteration, over the " + std::to_string(kMaxDrawSlots - 2) + " this build carries");
    if (diff_window > 0) {
        // The adjoint differentiates the weighted sum through each
        // variation's Jacobian; a variation without one (or outside the
        // normal phase) cannot be differentiated here.
        auto need = [](const VarDef* v) {
            if (!(v->flags & VF_JAC))
                throw std::runtime_error("variation `" + std::string(v->name) +
                                         "` has no Jacobian in this build; the differentiable render supports " + jac_names());
        };
        for (const VarDef* v : p.normal) need(v);
        for (auto& fi : p.fin) for (const VarDef* v : fi.vars) need(v);
        if (!f.xaos.empty()) throw std::runtime_error("the differentiable render has no xaos");
    }
    for (auto& x : f.xf) p.has_post |= x.post;
    const int M = p.maxx, NVN = (int)p.normal.size();
    p.t_cum = 1;
    p.t_xf = p.t_cum + M;
    p.t_vw = p.t_xf + 16 * M;
    p.t_vp = p.t_vw + NVN * M;
    p.t_fin = p.t_vp + p.vp_slots * M;
    int off = p.t_fin;
    for (auto& fi : p.fin) { fi.off = off; off += 13 + (int)fi.vars.size() + fi.prm_slots; }
    p.sym_kind = f.sym.kind;
    p.t_sym = off;
    if (p.sym_kind != 0) off += kSymBlock;
    p.xaos = !f.xaos.empty();
    p.t_xaos = off;
    if (p.xaos) off += M * (M + 1);
    p.table_size = off;

    std::ostringstream s;
    s << "// generated by ffb_codegen for one flame structure\n";
    s << "#define FFB_MAXX " << M << "\n#define FFB_NVN " << NVN << "\n#define FFB_NFIN " << p.fin.size() << "\n";
    s << "#define FFB_HAS_POST " << (p.has_post ? 1 : 0) << "\n#define FFB_NSLOTS " << p.n_slots << "\n";
    s << "#define FFB_RNG_MODE " << rng_mode << "\n#define FFB_THREADS " << threads << "\n";
    if (math_mode == MATH_SFU) s << "#define FFB_SFU 1\n";
    if (exact) s << "#define FFB_EXACT 1\n";
    if (emit) s << "#define FFB_EMIT 1\n";
    int nfd = 0;
    for (auto& fi : p.fin) for (const VarDef* v : fi.vars) nfd += v->draws;
    if (p.defer) s << "#define FFB_DEFER 1\n#define FFB_NFD " << nfd << "\n";
    s << "#define FFB_SYM_KIND " << p.sym_kind << "\n#define T_SYM " << p.t_sym << "\n";
    if (p.xaos) s << "#define FFB_XAOS 1\n#define T_XAOS " << p.t_xaos << "\n";
    s << "#define FFB_TABLE_SIZE " << p.table_size << "\n#define FFB_TABLE_VEC4 " << (p.table_size + 3) / 4 << "\n";
    s << "#define T_TOTAL 0\n#define T_CUM " << p.t_cum << "\n#define T_XF " << p.t_xf << "\n#define T_VW " << p.t_vw
      << "\n#define T_VP " << p.t_vp << "\n";
    s << kDeviceSrc << "\n";
    // The normal phase (shader_builder_v2.rs:2714-2795): `result += w * V(p)`
    // from zero, in local order, each gated on its weight.
    s << "template <class R> __device__ __forceinline__ void ffb_normal(const float* __restrict__ sm, int k, float& x, float& y, R& rng) {\n";
    emit_phases(s, p.normal, [&](int j) { return normal_site(p, j, "k"); }, "    ", true);
    s << "    x = rx; y = ry;\n}\n";
    // Per-transform form for the sorted schedule, where k is (mostly)
    // warp-uniform: each case evaluates only its transform's variations, in
    // the same local order, straight-line (their chains overlap).
    s << "template <class R> __device__ __forceinline__ void ffb_normal_k(const float* __restrict__ sm, int k, float& x, float& y, R& rng) {\n";
    if (per_xform) {
        s << "    switch (k) {\n";
        for (size_t k = 0; k < f.xf.size(); ++k) {
            s << "    case " << k << ": {\n";
            std::vector<const VarDef*> used;
            std::vector<int> idx;
            for (int j = 0; j < NVN; ++j)
                if (f.xf[k].var_weight(p.normal[j]) != 0.0f) { used.push_back(p.normal[j]); idx.push_back(j); }
            emit_phases(s, used, [&](int u) { return normal_site(p, idx[u], std::to_string(k)); }, "        ", false);
            s << "        x = rx; y = ry;\n        return; }\n";
        }
        s << "    default: ffb_normal(sm, k, x, y, rng); return;\n    }\n";
    } else {
        s << "    ffb_normal(sm, k, x, y, rng);\n";
    }
    s << "}\n";
    // One final of the chain (main_template.wgsl:679-704): affine,
    // variations, post-affine; `aff` false evaluates the variations alone.
    s << "template <class R> __device__ __forceinline__ void ffb_final_one(const float* __restrict__ sm, int c, float& x, float& y, R& rng, bool aff) {\n";
    s << "    switch (c) {\n";
    for (size_t c = 0; c < p.fin.size(); ++c) {
        const Plan::Fin& fi = p.fin[c];
        s << "    case " << c << ": {\n        const float* q = sm + " << fi.off << ";\n";
        s << "        if (aff) { float ax = q[0] * x + q[1] * y + q[4]; float ay = q[2] * x + q[3] * y + q[5]; x = ax; y = ay; }\n";
        emit_phases(s, fi.vars, [&](int j) { return final_site(fi, j); }, "        ", true);
        s << "        if (aff && q[12] > 0.5f) { float px = q[6] * rx + q[7] * ry + q[10]; float py = q[8] * rx + q[9] * ry + q[11]; rx = px; ry = py; }\n";
        s << "        x = rx; y = ry;\n        break; }\n";
    }
    s << "    default: break;\n    }\n}\n";
    s << "template <class R> __device__ __forceinline__ void ffb_finals(const float* __restrict__ sm, float& x, float& y, R& rng) {\n";
    for (size_t c = 0; c < p.fin.size(); ++c) s << "    ffb_final_one(sm, " << c << ", x, y, rng, true);\n";
    s << "}\n";
    if (p.defer) {
        // The final chain's draws in the order it takes them (slot order),
        // for the deferred plot: one plane of `stride` a draw.
        s << "template <class R> __device__ __forceinline__ void ffb_capture_final_draws(R& rng, float* out, unsigned long long stride) {\n";
        int m = 0;
        for (auto& fi : p.fin)
            for (size_t j = 0; j < fi.vars.size(); ++j)
                for (int d = 0; d < fi.vars[j]->draws; ++d, ++m)
                    s << "    { const float v = rng.draw(" << fi.slot[j] + d << "); out[" << m << "ull * stride] = v; }\n";
        s << "    (void)rng; (void)out; (void)stride;\n}\n";
    }
    s << kKernelsSrc << "\n";
    if (diff_window > 0) emit_diff(s, p);
    p.source = s.str();
    return p;
}

bool plan_fits(const Plan& p, const Flame& f) {
    if ((int)f.xf.size() > p.maxx) return false;
    Plan q = make_plan(f, p.rng_mode, p.math_mode, p.maxx, p.threads, p.per_xform, p.exact, p.diff_window, p.diff_ckpt, p.emit,
                       p.defer);
    return q.source == p.source;
}

std::vector<float> make_table(const Plan& p, const Flame& f) {
    std::vector<float> t((size_t)p.table_size, 0.0f);
    const int M = p.maxx;
    // utilities.wgsl:35-54: total and running sums in f32, left to right.
    float total = 0.0f;
    for (auto& x : f.xf) total += x.weight;
    t[0] = total;
    float cum = 0.0f;
    for (size_t k = 0; k < f.xf.size(); ++k) { cum += f.xf[k].weight; t[p.t_cum + k] = cum; }
    for (size_t k = f.xf.size(); k < (size_t)M; ++k) t[p.t_cum + k] = INFINITY;
    for (size_t k = 0; k < f.xf.size(); ++k) {
        const XForm& x = f.xf[k];
        const float rec[16] = {x.a, x.b, x.c, x.d, x.e, x.f, x.pa, x.pb, x.pc, x.pd, x.pe, x.pf,
                               x.post ? 1.0f : 0.0f,
                               (1.0f + x.speed) / 2.0f,                 // main_template.wgsl:499-500
                               x.color * (1.0f - x.speed) / 2.0f,
                               x.opacity};
        for (int fld = 0; fld < 16; ++fld) t[p.t_xf + fld * M + k] = rec[fld];
        for (size_t j = 0; j < p.normal.size(); ++j) {
            const VarDef* v = p.normal[j];
            t[p.t_vw + j * M + k] = x.var_weight(v);
            float row[kMaxVarSlots];
            x.slot_values(v, row);
            for (int q = 0; q < v->slots(); ++q) t[p.t_vp + (size_t)(p.vp_off[j] + q) * M + k] = row[q];
        }
    }
    if (p.sym_kind != 0) {
        // Post-symmetry block: copies, centre, half the pair's separation,
        // cos/sin of the axis modes' pre-rotation (-rotation), then cos/sin
        // of each point-mode copy's angle k * 2pi / order
        // (utilities.wgsl:470-568), computed here in f32.
        const PostSym& y = f.sym;
        float* q = t.data() + p.t_sym;
        q[0] = (float)y.copies();
        q[1] = y.cx; q[2] = y.cy;
        q[3] = y.distance * 0.5f;
        q[4] = std::cos(-y.rotation); q[5] = std::sin(-y.rotation);
        for (int k = 0; k < 32; ++k) {
            const float th = ((float)k * 6.28318530717958647692f) / (float)std::max(y.order, 1);
            q[6 + 2 * k] = std::cos(th);
            q[7 + 2 * k] = std::sin(th);
        }
    }
    if (p.xaos) {
        // Each previous transform's row: total, then the running sums of
        // weight_i x xaos[prev][i] in f32, left to right (utilities.wgsl:110-137).
        const size_t n = f.xf.size();
        for (int r = 0; r < M; ++r) {
            float* row = t.data() + p.t_xaos + (size_t)r * (M + 1);
            float cum = 0.0f;
            for (int i = 0; i < M; ++i) {
                if ((size_t)i < n && (size_t)r < n) { cum += f.xf[i].weight * f.xaos[(size_t)r * n + i]; row[1 + i] = cum; }
                else row[1 + i] = INFINITY;
            }
            row[0] = (size_t)r < n ? cum : 0.0f;
        }
    }
    for (size_t c = 0; c < p.fin.size(); ++c) {
        const Plan::Fin& fi = p.fin[c];
        const XForm& x = f.fin[f.fin_chain[c]];
        const float rec[13] = {x.a, x.b, x.c, x.d, x.e, x.f, x.pa, x.pb, x.pc, x.pd, x.pe, x.pf, x.post ? 1.0f : 0.0f};
        for (int q = 0; q < 13; ++q) t[fi.off + q] = rec[q];
        const int nv = (int)fi.vars.size();
        for (int j = 0; j < nv; ++j) {
            t[fi.off + 13 + j] = x.var_weight(fi.vars[j]);
            float row[kMaxVarSlots];
            x.slot_values(fi.vars[j], row);
            for (int q = 0; q < fi.vars[j]->slots(); ++q) t[fi.off + 13 + nv + fi.prm_off[j] + q] = row[q];
        }
    }
    return t;
}

}  // namespace ffb
