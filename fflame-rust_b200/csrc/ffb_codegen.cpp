// ffb_codegen.cpp -- see ffb_codegen.hpp.

#include "ffb_codegen.hpp"

#include <algorithm>
#include <cmath>
#include <sstream>

#include "ffb_device_src.inc"

namespace ffb {

namespace {

constexpr int kSymBlock = 6 + 64;            // post-symmetry table block (floats)

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

std::string call(const VarDef* v, const std::string& prm0, const std::string& prm1, int slot) {
    std::ostringstream o;
    o << v->fn << "(x, y";
    if (v->needs_rng) o << ", rng.draw(" << slot << ")";
    if (v->nparams >= 1) o << ", " << prm0;
    if (v->nparams >= 2) o << ", " << prm1;
    o << ", ox, oy)";
    return o.str();
}

// The Jacobian of a variation body (ffb_diff.cuh): "v_name" -> "dj_name".
std::string jcall(const VarDef* v, const std::string& prm0, const std::string& prm1, int slot) {
    std::ostringstream o;
    o << "dj_" << (v->fn + 2) << "(x, y";
    if (v->needs_rng) o << ", rng.draw(" << slot << ")";
    if (v->nparams >= 1) o << ", " << prm0;
    if (v->nparams >= 2) o << ", " << prm1;
    o << ")";
    return o.str();
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
        std::ostringstream w, a0, a1;
        w << "sm[T_VW + " << j << " * FFB_MAXX + k]";
        a0 << "sm[T_VP + " << (2 * j) << " * FFB_MAXX + k]";
        a1 << "sm[T_VP + " << (2 * j + 1) << " * FFB_MAXX + k]";
        s << "    { " << call(v, a0.str(), a1.str(), p.normal_slot[j]) << "; const float g = ax * ox + ay * oy; if (isfinite(g)) gw["
          << j << " * P] += g;\n      const float w = " << w.str() << "; if (w != 0.0f) { const float4 jj = "
          << jcall(v, a0.str(), a1.str(), p.normal_slot[j])
          << "; J.x += w * jj.x; J.y += w * jj.y; J.z += w * jj.z; J.w += w * jj.w; } }   // " << v->name << "\n";
    }
    s << "    if (!(isfinite(J.x) && isfinite(J.y) && isfinite(J.z) && isfinite(J.w))) J = make_float4(0.f, 0.f, 0.f, 0.f);\n}\n";
    // One normal variation's value and Jacobian (the probe).
    s << "template <class R> __device__ __forceinline__ void ffb_dvar_one(const float* __restrict__ sm, int j, int k, float x, float y, R& rng, "
         "float& ox, float& oy, float4& J) {\n    switch (j) {\n";
    for (int j = 0; j < NVN; ++j) {
        const VarDef* v = p.normal[j];
        std::ostringstream a0, a1;
        a0 << "sm[T_VP + " << (2 * j) << " * FFB_MAXX + k]";
        a1 << "sm[T_VP + " << (2 * j + 1) << " * FFB_MAXX + k]";
        s << "    case " << j << ": " << call(v, a0.str(), a1.str(), p.normal_slot[j]) << "; J = "
          << jcall(v, a0.str(), a1.str(), p.normal_slot[j]) << "; break;\n";
    }
    s << "    default: ox = 0.f; oy = 0.f; J = make_float4(0.f, 0.f, 0.f, 0.f); break;\n    }\n}\n";
    s << kDiffSrc << "\n";
}

}  // namespace

Plan make_plan(const Flame& f, int rng_mode, int math_mode, int maxx, int threads, bool per_xform, bool exact,
               int diff_window, int diff_ckpt, bool emit) {
    Plan p;
    p.exact = exact;
    p.emit = emit;
    p.diff_window = diff_window;
    p.diff_ckpt = diff_ckpt;
    p.rng_mode = rng_mode;
    p.math_mode = math_mode;
    p.per_xform = per_xform;
    p.threads = threads;
    p.maxx = std::max<int>(maxx, (int)f.xf.size());
    p.normal = normal_vars(f);
    int slot = 2;                                   // 0: transform pick, 1: opacity
    for (const VarDef* v : p.normal) p.normal_slot.push_back(v->needs_rng ? slot++ : -1);
    for (int c : f.fin_chain) {
        Plan::Fin fi;
        fi.vars = final_vars(f, f.fin[c]);
        for (const VarDef* v : fi.vars) fi.slot.push_back(v->needs_rng ? slot++ : -1);
        p.fin.push_back(fi);
    }
    p.n_slots = slot;
    for (auto& x : f.xf) p.has_post |= x.post;
    const int M = p.maxx, NVN = (int)p.normal.size();
    p.t_cum = 1;
    p.t_xf = p.t_cum + M;
    p.t_vw = p.t_xf + 16 * M;
    p.t_vp = p.t_vw + NVN * M;
    p.t_fin = p.t_vp + 2 * NVN * M;
    int off = p.t_fin;
    for (auto& fi : p.fin) { fi.off = off; off += 13 + 3 * (int)fi.vars.size(); }
    p.sym_kind = f.sym.kind;
    p.t_sym = off;
    if (p.sym_kind != 0) off += kSymBlock;
    p.table_size = off;

    std::ostringstream s;
    s << "// generated by ffb_codegen for one flame structure\n";
    s << "#define FFB_MAXX " << M << "\n#define FFB_NVN " << NVN << "\n#define FFB_NFIN " << p.fin.size() << "\n";
    s << "#define FFB_HAS_POST " << (p.has_post ? 1 : 0) << "\n#define FFB_NSLOTS " << p.n_slots << "\n";
    s << "#define FFB_RNG_MODE " << rng_mode << "\n#define FFB_THREADS " << threads << "\n";
    if (math_mode == MATH_SFU) s << "#define FFB_SFU 1\n";
    if (exact) s << "#define FFB_EXACT 1\n";
    if (emit) s << "#define FFB_EMIT 1\n";
    s << "#define FFB_SYM_KIND " << p.sym_kind << "\n#define T_SYM " << p.t_sym << "\n";
    s << "#define FFB_TABLE_SIZE " << p.table_size << "\n#define FFB_TABLE_VEC4 " << (p.table_size + 3) / 4 << "\n";
    s << "#define T_TOTAL 0\n#define T_CUM " << p.t_cum << "\n#define T_XF " << p.t_xf << "\n#define T_VW " << p.t_vw
      << "\n#define T_VP " << p.t_vp << "\n";
    s << kDeviceSrc << "\n";
    // The normal phase (shader_builder_v2.rs:2714-2795): `result += w * V(p)`
    // from zero, in local order, each gated on its weight.
    s << "template <class R> __device__ __forceinline__ void ffb_normal(const float* __restrict__ sm, int k, float& x, float& y, R& rng) {\n";
    s << "    float rx = 0.0f, ry = 0.0f, ox, oy;\n";
    for (int j = 0; j < NVN; ++j) {
        const VarDef* v = p.normal[j];
        std::ostringstream w, a0, a1;
        w << "sm[T_VW + " << j << " * FFB_MAXX + k]";
        a0 << "sm[T_VP + " << (2 * j) << " * FFB_MAXX + k]";
        a1 << "sm[T_VP + " << (2 * j + 1) << " * FFB_MAXX + k]";
        s << "    { const float w = " << w.str() << "; if (w != 0.0f) { " << call(v, a0.str(), a1.str(), p.normal_slot[j])
          << "; rx = rx + w * ox; ry = ry + w * oy; } }   // " << v->name << "\n";
    }
    s << "    x = rx; y = ry;\n}\n";
    // Per-transform form for the sorted schedule, where k is (mostly)
    // warp-uniform: each case evaluates only its transform's variations, in
    // the same local order, straight-line (their chains overlap).
    s << "template <class R> __device__ __forceinline__ void ffb_normal_k(const float* __restrict__ sm, int k, float& x, float& y, R& rng) {\n";
    if (per_xform) {
        s << "    float rx = 0.0f, ry = 0.0f, ox, oy;\n    switch (k) {\n";
        for (size_t k = 0; k < f.xf.size(); ++k) {
            s << "    case " << k << ": {\n";
            for (int j = 0; j < NVN; ++j) {
                const VarDef* v = p.normal[j];
                if (f.xf[k].var_weight(v) == 0.0f) continue;
                std::ostringstream w, a0, a1;
                w << "sm[T_VW + " << j << " * FFB_MAXX + " << k << "]";
                a0 << "sm[T_VP + " << (2 * j) << " * FFB_MAXX + " << k << "]";
                a1 << "sm[T_VP + " << (2 * j + 1) << " * FFB_MAXX + " << k << "]";
                s << "        { const float w = " << w.str() << "; " << call(v, a0.str(), a1.str(), p.normal_slot[j])
                  << "; rx = rx + w * ox; ry = ry + w * oy; }   // " << v->name << "\n";
            }
            s << "        break; }\n";
        }
        s << "    default: ffb_normal(sm, k, x, y, rng); return;\n    }\n    x = rx; y = ry;\n";
    } else {
        s << "    ffb_normal(sm, k, x, y, rng);\n";
    }
    s << "}\n";
    // One final of the chain (main_template.wgsl:679-704): affine,
    // variations, post-affine; `aff` false evaluates the variations alone.
    s << "template <class R> __device__ __forceinline__ void ffb_final_one(const float* __restrict__ sm, int c, float& x, float& y, R& rng, bool aff) {\n";
    s << "    float rx = 0.0f, ry = 0.0f, ox, oy;\n    switch (c) {\n";
    for (size_t c = 0; c < p.fin.size(); ++c) {
        const Plan::Fin& fi = p.fin[c];
        s << "    case " << c << ": {\n        const float* q = sm + " << fi.off << ";\n";
        s << "        if (aff) { float ax = q[0] * x + q[1] * y + q[4]; float ay = q[2] * x + q[3] * y + q[5]; x = ax; y = ay; }\n";
        const int nv = (int)fi.vars.size();
        for (int j = 0; j < nv; ++j) {
            std::ostringstream w, a0, a1;
            w << "q[" << 13 + j << "]";
            a0 << "q[" << 13 + nv + 2 * j << "]";
            a1 << "q[" << 13 + nv + 2 * j + 1 << "]";
            s << "        { const float w = " << w.str() << "; if (w != 0.0f) { " << call(fi.vars[j], a0.str(), a1.str(), fi.slot[j])
              << "; rx = rx + w * ox; ry = ry + w * oy; } }   // " << fi.vars[j]->name << "\n";
        }
        s << "        if (aff && q[12] > 0.5f) { float px = q[6] * rx + q[7] * ry + q[10]; float py = q[8] * rx + q[9] * ry + q[11]; rx = px; ry = py; }\n";
        s << "        x = rx; y = ry;\n        break; }\n";
    }
    s << "    default: break;\n    }\n}\n";
    s << "template <class R> __device__ __forceinline__ void ffb_finals(const float* __restrict__ sm, float& x, float& y, R& rng) {\n";
    for (size_t c = 0; c < p.fin.size(); ++c) s << "    ffb_final_one(sm, " << c << ", x, y, rng, true);\n";
    s << "}\n";
    s << kKernelsSrc << "\n";
    if (diff_window > 0) emit_diff(s, p);
    p.source = s.str();
    return p;
}

bool plan_fits(const Plan& p, const Flame& f) {
    if ((int)f.xf.size() > p.maxx) return false;
    Plan q = make_plan(f, p.rng_mode, p.math_mode, p.maxx, p.threads, p.per_xform, p.exact, p.diff_window, p.diff_ckpt, p.emit);
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
            for (int q = 0; q < v->nparams; ++q) t[p.t_vp + (2 * j + q) * M + k] = x.param(v, q);
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
    for (size_t c = 0; c < p.fin.size(); ++c) {
        const Plan::Fin& fi = p.fin[c];
        const XForm& x = f.fin[f.fin_chain[c]];
        const float rec[13] = {x.a, x.b, x.c, x.d, x.e, x.f, x.pa, x.pb, x.pc, x.pd, x.pe, x.pf, x.post ? 1.0f : 0.0f};
        for (int q = 0; q < 13; ++q) t[fi.off + q] = rec[q];
        const int nv = (int)fi.vars.size();
        for (int j = 0; j < nv; ++j) {
            t[fi.off + 13 + j] = x.var_weight(fi.vars[j]);
            for (int q = 0; q < fi.vars[j]->nparams; ++q) t[fi.off + 13 + nv + 2 * j + q] = x.param(fi.vars[j], q);
        }
    }
    return t;
}

}  // namespace ffb
